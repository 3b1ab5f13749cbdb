// Path-replay adjoint instantiations of the wave kernels (the backward pass
// of ymrt_render_backward / ymrt_render_backward_ex), compiled apart from the
// forward kernels so that the library builds in parallel. Surface adjoint
// shading is instantiated on surface_features() (its closest hits are the
// forward k_extend's); with media, one instantiation with every feature
// serves both free flight and shading.
#include "wave_device.cuh"

namespace ym {

namespace {

template <uint32_t kS>
void surface_adjoint_shade(const WaveArgs& w, const WaveOptions& opt) {
  const ShadowQueue none{};
  k_shade<false, false, true, kS><<<w.blocks, kTraceBlock, 0, w.stream>>>(w.A, w.ctl, w.H, w.B, w.jobs, w.counters,
                                                                          none, opt.grads, opt.grad_materials);
}

}  // namespace

void launch_adjoint_extend_media(const WaveArgs& w, const WaveOptions& opt) {
  // free flight with the density-grid terms (one instantiation, all features)
  const auto k = k_extend<true, kFeatAll, true>;
  k<<<w.trace_blocks, w.trace_block, traversal_shared_bytes(w.trace_block), w.stream>>>(w.A, w.ctl, w.H, w.jobs, w.counters,
                                                                           opt.grid_grads, opt.grid_tex, w.ray_order);
}

void launch_adjoint_shade(bool volumes, uint32_t features, const WaveArgs& w, const WaveOptions& opt) {
  if (volumes) {
    const ShadowQueue none{};
    k_shade<true, false, true, kFeatAll><<<w.blocks, kTraceBlock, 0, w.stream>>>(
        w.A, w.ctl, w.H, w.B, w.jobs, w.counters, none, opt.grads, opt.grad_materials, opt.grid_grads, opt.grid_tex);
    return;
  }
  switch (surface_features(features)) {
    case 0: surface_adjoint_shade<0>(w, opt); break;
    case kFeatSpheres: surface_adjoint_shade<kFeatSpheres>(w, opt); break;
    case kFeatTextures: surface_adjoint_shade<kFeatTextures>(w, opt); break;
    default: surface_adjoint_shade<kFeatSpheres | kFeatTextures>(w, opt); break;
  }
}

void prepare_adjoint_kernels() { allow_trace_shared(k_extend<true, kFeatAll, true>); }

cudaError_t upload_slots_adjoint(const DeviceScene* scenes, const uint32_t* slots, uint32_t n, const uint32_t* primes,
                                 const uint32_t* prime_sums, cudaStream_t stream) {
  return upload_slots_here(scenes, slots, n, primes, prime_sums, stream);
}

cudaError_t read_bound_adjoint(BoundRecord* out, bool clear, cudaStream_t stream) {
  return read_bound_here(out, clear, stream);
}

}  // namespace ym
