// Volume-scattering instantiations of the wave kernels (k_extend with free
// flight through media, k_shade with volume vertices and media next-event
// estimation), compiled apart from the surface kernels so that the library
// builds in parallel. Media kernels are instantiated on media_features(): the
// sphere bit and one bit for the full texture node set.
#include "wave_device.cuh"

namespace ym {

namespace {

template <uint32_t kF>
void media_extend(const WaveArgs& w) {
  const auto k = k_extend<true, kF>;
  k<<<w.trace_blocks, w.trace_block, traversal_shared_bytes(w.trace_block), w.stream>>>(w.A, w.ctl, w.H, w.jobs, w.counters, nullptr,
                                                                   kEmpty, w.ray_order);
}

template <uint32_t kF>
void media_shade(const WaveArgs& w) {
  const ShadowQueue none{};
  k_shade<true, false, false, kF><<<w.blocks, kTraceBlock, 0, w.stream>>>(w.A, w.ctl, w.H, w.B, w.jobs, w.counters,
                                                                          none);
}

constexpr uint32_t kAllNodes = kFeatGrids | kFeatTextures;

}  // namespace

void launch_media_extend(uint32_t features, const WaveArgs& w) {
  switch (media_features(features)) {
    case 0: media_extend<0>(w); break;
    case kFeatSpheres: media_extend<kFeatSpheres>(w); break;
    case kAllNodes: media_extend<kAllNodes>(w); break;
    default: media_extend<kAllNodes | kFeatSpheres>(w); break;
  }
}

void launch_media_shade(uint32_t features, const WaveArgs& w) {
  switch (media_features(features)) {
    case 0: media_shade<0>(w); break;
    case kFeatSpheres: media_shade<kFeatSpheres>(w); break;
    case kAllNodes: media_shade<kAllNodes>(w); break;
    default: media_shade<kAllNodes | kFeatSpheres>(w); break;
  }
}

void prepare_media_kernels() {
  allow_trace_shared(k_extend<true, 0>);
  allow_trace_shared(k_extend<true, kFeatSpheres>);
  allow_trace_shared(k_extend<true, kAllNodes>);
  allow_trace_shared(k_extend<true, kAllNodes | kFeatSpheres>);
}

cudaError_t upload_slots_media(const DeviceScene* scenes, const uint32_t* slots, uint32_t n, const uint32_t* primes,
                               const uint32_t* prime_sums, cudaStream_t stream) {
  return upload_slots_here(scenes, slots, n, primes, prime_sums, stream);
}

cudaError_t read_bound_media(BoundRecord* out, bool clear, cudaStream_t stream) {
  return read_bound_here(out, clear, stream);
}

}  // namespace ym
