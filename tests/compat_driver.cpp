// Test driver for libymrt_compat.so: the reference editor's calling sequence
// against the reference-named launchers, beside the same frames rendered
// through the C ABI directly.
//
// TEST INFRASTRUCTURE ONLY (compiled and run by tests/test_gpu_compat.py).
//
// The launchers are declared here with the reference's argument kinds
// (references, RenderSetting, RayCounter, the queue structs), as
// src/core/RenderModule.cpp:14-28, 36-42 declares them; its structs are
// replaced by stand-ins of the same layout where the driver touches them
// (RayCounter, RayCounterData, src/SceneDefines.h:114-124) and by empty
// types where it only passes them on. run_frame restates the counter
// protocol of RenderModule::PathTracingExecuteTask
// (src/core/RenderModule.cpp:494-653): clear the counters, then generation,
// trace and shading batch after batch until no tiles are left and no rays
// are in flight, copying the counters between host and device in between.
//
// usage: compat_driver <scene.ymtmp> <halton_perm.u32> <width> <height> <spp> <frames> <max_frames> <out_compat> <out_direct>
//        [<editor_compat> <editor_direct>]
// The optional outputs hold, per side: the editor view's beauty (float4 per
// pixel) and primitive index (uint32 per pixel), the editor view after
// PostProcessingEditorView (outline of the instance at the image centre),
// and the accumulated image after PostProcessingPathTracing.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <vector>

#include "ymrt.h"
#include "ymrt_compat.h"

using RenderSetting = ymrt_render_setting;  // byte-compatible with the reference's
struct RayCounter {
  uint32_t shading_ray_counter;
  uint32_t hit_counter;
  uint32_t shadow_ray_counter;
};
struct RayCounterData {
  RayCounter* ray_counter_device;
  RayCounter* ray_counter_host;
};
struct ShadingRayData {};
struct HitData {};
struct ShadowRayData {};
struct Scene;
struct HaltonEnumerator;
struct vec4 {
  float x, y, z, w;
};

extern "C" {
void AllocateRayCounter(RayCounterData& ray_counter_data);
void ReleaseRayCounter(RayCounterData& ray_counter_data);
void AllocateShadingRayData(ShadingRayData& shading_ray_data);
void ReleaseShadingRayData(ShadingRayData& shading_ray_data);
void AllocateHitData(HitData& hit_data);
void ReleaseHitData(HitData& hit_data);
void AllocateShadowRayData(ShadowRayData& shadow_ray_data);
void ReleaseShadowRayData(ShadowRayData& shadow_ray_data);
void RayGenerationPathTracing(int current_frame_index, const RenderSetting& render_setting, Scene* scene_device,
                              HaltonEnumerator* halton_enumerator_device, RayCounter* ray_counter_device,
                              uint32_t next_tile_index, uint32_t tile_count_this_batch, uint32_t width, uint32_t height,
                              uint32_t tile_count_x, uint32_t tile_count_y, ShadingRayData& shading_ray_data,
                              cudaStream_t& stream);
void RayTracePathTracing(int current_frame_index, const RenderSetting& render_setting, Scene* scene_device,
                         RayCounter* ray_counter_device, RayCounter* ray_counter_host, uint32_t width, uint32_t height,
                         vec4* noise_image, ShadingRayData& shading_ray_data, HitData& hit_data, cudaStream_t& stream);
void RayShadingPathTracing(int current_frame_index, const RenderSetting& render_setting, Scene* scene_device,
                           RayCounter* ray_counter_device, RayCounter* ray_counter_host, uint32_t width,
                           uint32_t height, vec4* noise_image, ShadingRayData& shading_ray_data, HitData& hit_data,
                           ShadowRayData& shadow_ray_data, cudaStream_t& stream);
void AccumulateImagePathTracing(const vec4* noise_image, vec4* accumulated_image, uint32_t width, uint32_t height,
                                int frame_index, const int max_accumulate_frame, cudaStream_t& stream);
void RayGenerationEditorView(int current_frame_index, const RenderSetting& render_setting, Scene* scene_device,
                             RayCounter* ray_counter_device, uint32_t next_tile_index, uint32_t tile_count_this_batch,
                             uint32_t width, uint32_t height, uint32_t tile_count_x, uint32_t tile_count_y,
                             ShadingRayData& shading_ray_data, cudaStream_t& stream);
void RayTraceEditorView(int current_frame_index, const RenderSetting& render_setting, Scene* scene_device,
                        RayCounter* ray_counter_device, RayCounter* ray_counter_host, uint32_t width, uint32_t height,
                        vec4* beauty, uint32_t* primitive_index, ShadingRayData& shading_ray_data, HitData& hit_data,
                        cudaStream_t& stream);
void RayShadingEditorView(int current_frame_index, const RenderSetting& render_setting, Scene* scene_device,
                          RayCounter* ray_counter_device, RayCounter* ray_counter_host, uint32_t width, uint32_t height,
                          vec4* beauty, uint32_t* primitive_index, ShadingRayData& shading_ray_data,
                          HitData& hit_data, ShadowRayData& shadow_ray_data, cudaStream_t& stream);
void PostProcessingEditorView(vec4* image, uint32_t* primitive_index, uint32_t width, uint32_t height,
                              uint32_t clicked_primitive_index, float gamma, float exposure, bool draw_selected_effect,
                              cudaStream_t& stream);
void PostProcessingPathTracing(vec4* image, uint32_t width, uint32_t height, float gamma, float exposure,
                               cudaStream_t& stream);
}

namespace {

constexpr uint32_t kMaxRayCount = 1u << 20;  // MAX_RAY_COUNT, src/SceneDefines.h:9-15
constexpr uint32_t kTilePixels = 256;        // TILE_PIXEL_COUNT (16 x 16)

void cuda(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

int generation_calls = 0;

void run_frame(int frame, const RenderSetting& rs, RayCounterData& counters, ShadingRayData& srd, HitData& hd,
               ShadowRayData& sd, uint32_t w, uint32_t h, vec4* noise, cudaStream_t& stream) {
  cuda(cudaMemsetAsync(noise, 0, sizeof(vec4) * w * h, stream), "clear noise");
  cuda(cudaStreamSynchronize(stream), "sync");
  const uint32_t spp = (uint32_t)rs.ssp;
  const uint32_t tiles_x = (w + 15) / 16, tiles_y = (h + 15) / 16, total = tiles_x * tiles_y;
  uint32_t next_tile = 0;
  RayCounter* host = counters.ray_counter_host;
  RayCounter* dev = counters.ray_counter_device;
  host->hit_counter = host->shading_ray_counter = host->shadow_ray_counter = 0;
  cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
  cuda(cudaStreamSynchronize(stream), "sync");
  while (host->shading_ray_counter > 0 || next_tile < total) {
    const uint32_t batch = (kMaxRayCount - host->shading_ray_counter) / (kTilePixels * spp);
    RayGenerationPathTracing(frame, rs, nullptr, nullptr, dev, next_tile, batch, w, h, tiles_x, tiles_y, srd, stream);
    ++generation_calls;
    next_tile += batch;
    host->shading_ray_counter += batch * spp * kTilePixels;
    cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    RayTracePathTracing(frame, rs, nullptr, dev, host, w, h, noise, srd, hd, stream);
    cuda(cudaMemcpyAsync(host, dev, sizeof(RayCounter), cudaMemcpyDeviceToHost, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    host->shading_ray_counter = 0;
    cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    RayShadingPathTracing(frame, rs, nullptr, dev, host, w, h, noise, srd, hd, sd, stream);
    cuda(cudaMemcpyAsync(host, dev, sizeof(RayCounter), cudaMemcpyDeviceToHost, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    host->hit_counter = 0;
    cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
  }
}

// RenderModule::EditorViewExecuteTask's loop (src/core/RenderModule.cpp:366-492):
// batches of MAX_RAY_COUNT rays, re-queued pass-through rays, counters
// copied between host and device around every stage.
void run_editor_frame(int frame, const RenderSetting& rs, RayCounterData& counters, ShadingRayData& srd, HitData& hd,
                      ShadowRayData& sd, uint32_t w, uint32_t h, vec4* beauty, uint32_t* prim, cudaStream_t& stream) {
  const uint32_t tiles_x = (w + 15) / 16, tiles_y = (h + 15) / 16, total = tiles_x * tiles_y;
  uint32_t next_tile = 0;
  RayCounter* host = counters.ray_counter_host;
  RayCounter* dev = counters.ray_counter_device;
  host->hit_counter = host->shading_ray_counter = host->shadow_ray_counter = 0;
  cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
  cuda(cudaStreamSynchronize(stream), "sync");
  while (host->shading_ray_counter > 0 || next_tile < total) {
    const uint32_t batch = (kMaxRayCount - host->shading_ray_counter) / kTilePixels;
    RayGenerationEditorView(frame, rs, nullptr, dev, next_tile, batch, w, h, tiles_x, tiles_y, srd, stream);
    next_tile += batch;
    host->shading_ray_counter += batch * kTilePixels;
    cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    RayTraceEditorView(frame, rs, nullptr, dev, host, w, h, beauty, prim, srd, hd, stream);
    cuda(cudaMemcpyAsync(host, dev, sizeof(RayCounter), cudaMemcpyDeviceToHost, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    host->shading_ray_counter = 0;
    cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    RayShadingEditorView(frame, rs, nullptr, dev, host, w, h, beauty, prim, srd, hd, sd, stream);
    cuda(cudaMemcpyAsync(host, dev, sizeof(RayCounter), cudaMemcpyDeviceToHost, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
    host->hit_counter = 0;
    cuda(cudaMemcpyAsync(dev, host, sizeof(RayCounter), cudaMemcpyHostToDevice, stream), "counter");
    cuda(cudaStreamSynchronize(stream), "sync");
  }
}

void save_raw(FILE* f, const void* dev, size_t bytes) {
  std::vector<unsigned char> h(bytes);
  cuda(cudaMemcpy(h.data(), dev, bytes, cudaMemcpyDeviceToHost), "read back");
  if (std::fwrite(h.data(), 1, bytes, f) != bytes) throw std::runtime_error("writing");
}

void save(const char* path, const vec4* dev, size_t n) {
  std::vector<vec4> h(n);
  cuda(cudaMemcpy(h.data(), dev, sizeof(vec4) * n, cudaMemcpyDeviceToHost), "read back");
  FILE* f = std::fopen(path, "wb");
  if (!f || std::fwrite(h.data(), sizeof(vec4), n, f) != n) throw std::runtime_error("writing the image");
  std::fclose(f);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 10 && argc != 12) {
    std::fprintf(stderr, "usage: %s scene perm width height spp frames max_frames out_compat out_direct\n", argv[0]);
    return 2;
  }
  try {
    const int w = std::atoi(argv[3]), h = std::atoi(argv[4]), spp = std::atoi(argv[5]);
    const int frames = std::atoi(argv[6]), max_frames = std::atoi(argv[7]);
    std::vector<uint32_t> perm;
    {
      FILE* f = std::fopen(argv[2], "rb");
      if (!f) throw std::runtime_error("cannot open the Halton table");
      uint32_t v;
      while (std::fread(&v, 4, 1, f) == 1) perm.push_back(v);
      std::fclose(f);
    }
    ymrt_context* ctx = nullptr;
    if (ymrt_create(0, &ctx) != YMRT_OK) throw std::runtime_error("ymrt_create");
    ymrt_host_scene* hs = nullptr;
    char err[512];
    if (ymrt_scene_load_ymtmp(argv[1], w, h, &hs, err, sizeof(err)) != YMRT_OK) throw std::runtime_error(err);
    ymrt_scene* scene = nullptr;
    if (ymrt_scene_upload(ctx, hs, perm.data(), perm.size(), &scene) != YMRT_OK)
      throw std::runtime_error(ymrt_last_error(ctx));
    if (ymrt_compat_bind(ctx, scene) != YMRT_OK) throw std::runtime_error("ymrt_compat_bind");

    RenderSetting rs{};
    rs.ssp = spp;
    rs.ray_depth = 8;
    rs.gamma = 2.2f;
    rs.exposure = 1.0f;
    rs.max_frame_count = max_frames;
    rs.sampler_type = 1;
    rs.enable_shape_light = 1;

    // the editor's side: its queues (not allocated by the shim) and counters
    RayCounterData counters{};
    ShadingRayData srd;
    HitData hd;
    ShadowRayData sd;
    AllocateRayCounter(counters);
    AllocateShadingRayData(srd);
    AllocateHitData(hd);
    AllocateShadowRayData(sd);
    cudaStream_t stream;
    cuda(cudaStreamCreate(&stream), "stream");
    const size_t n = (size_t)w * h;
    vec4 *noise, *acc, *noise2, *acc2;
    cuda(cudaMalloc(&noise, sizeof(vec4) * n), "alloc");
    cuda(cudaMalloc(&acc, sizeof(vec4) * n), "alloc");
    cuda(cudaMalloc(&noise2, sizeof(vec4) * n), "alloc");
    cuda(cudaMalloc(&acc2, sizeof(vec4) * n), "alloc");
    cuda(cudaMemset(acc, 0, sizeof(vec4) * n), "clear");
    cuda(cudaMemset(acc2, 0, sizeof(vec4) * n), "clear");
    for (int frame = 1; frame <= frames; ++frame) {
      run_frame(frame, rs, counters, srd, hd, sd, (uint32_t)w, (uint32_t)h, noise, stream);
      AccumulateImagePathTracing(noise, acc, (uint32_t)w, (uint32_t)h, frame, max_frames, stream);
      // the same frame through the C ABI
      ymrt_stats st;
      if (ymrt_render_forward(scene, &rs, frame, reinterpret_cast<float*>(noise2), 1, &st) != YMRT_OK)
        throw std::runtime_error(ymrt_last_error(ctx));
      if (!(max_frames > 0 && frame - 1 >= max_frames) &&
          ymrt_accumulate(scene, reinterpret_cast<float*>(noise2), reinterpret_cast<float*>(acc2), frame) != YMRT_OK)
        throw std::runtime_error(ymrt_last_error(ctx));
    }
    save(argv[8], acc, n);
    save(argv[9], acc2, n);
    if (argc == 12) {
      // the editor view through the launchers and directly, then post-processing
      vec4 *eb, *eb2;
      uint32_t *ep, *ep2;
      cuda(cudaMalloc(&eb, sizeof(vec4) * n), "alloc");
      cuda(cudaMalloc(&eb2, sizeof(vec4) * n), "alloc");
      cuda(cudaMalloc(&ep, sizeof(uint32_t) * n), "alloc");
      cuda(cudaMalloc(&ep2, sizeof(uint32_t) * n), "alloc");
      cuda(cudaMemset(eb, 0, sizeof(vec4) * n), "clear");
      cuda(cudaMemset(eb2, 0, sizeof(vec4) * n), "clear");
      cuda(cudaMemset(ep, 0xFF, sizeof(uint32_t) * n), "clear");
      cuda(cudaMemset(ep2, 0xFF, sizeof(uint32_t) * n), "clear");
      RayCounterData ec{};
      AllocateRayCounter(ec);
      run_editor_frame(1, rs, ec, srd, hd, sd, (uint32_t)w, (uint32_t)h, eb, ep, stream);
      ReleaseRayCounter(ec);
      if (ymrt_render_editor_view(scene, &rs, (uint32_t)w, (uint32_t)h, reinterpret_cast<float*>(eb2), ep2, 1) != YMRT_OK)
        throw std::runtime_error(ymrt_last_error(ctx));
      uint32_t centre = 0;
      cuda(cudaMemcpy(&centre, ep + (size_t)(h / 2) * w + w / 2, sizeof(uint32_t), cudaMemcpyDeviceToHost), "read");
      FILE* fa = std::fopen(argv[10], "wb");
      FILE* fb = std::fopen(argv[11], "wb");
      if (!fa || !fb) throw std::runtime_error("opening the editor outputs");
      save_raw(fa, eb, sizeof(vec4) * n);
      save_raw(fa, ep, sizeof(uint32_t) * n);
      save_raw(fb, eb2, sizeof(vec4) * n);
      save_raw(fb, ep2, sizeof(uint32_t) * n);
      PostProcessingEditorView(eb, ep, (uint32_t)w, (uint32_t)h, centre, 2.2f, 1.0f, true, stream);
      if (ymrt_post_process(ctx, reinterpret_cast<float*>(eb2), ep2, (uint32_t)w, (uint32_t)h, centre, 2.2f, 1.0f, 1, 1) !=
          YMRT_OK)
        throw std::runtime_error(ymrt_last_error(ctx));
      save_raw(fa, eb, sizeof(vec4) * n);
      save_raw(fb, eb2, sizeof(vec4) * n);
      PostProcessingPathTracing(acc, (uint32_t)w, (uint32_t)h, 2.2f, 1.0f, stream);
      if (ymrt_post_process(ctx, reinterpret_cast<float*>(acc2), nullptr, (uint32_t)w, (uint32_t)h, 0xFFFFFFFFu, 2.2f,
                            1.0f, 0, 1) != YMRT_OK)
        throw std::runtime_error(ymrt_last_error(ctx));
      save_raw(fa, acc, sizeof(vec4) * n);
      save_raw(fb, acc2, sizeof(vec4) * n);
      std::fclose(fa);
      std::fclose(fb);
      std::printf("editor_centre %u\n", centre);
    }
    ReleaseRayCounter(counters);
    ReleaseShadingRayData(srd);
    ReleaseHitData(hd);
    ReleaseShadowRayData(sd);
    ymrt_compat_bind(ctx, nullptr);
    ymrt_scene_free(scene);
    ymrt_host_scene_free(hs);
    ymrt_destroy(ctx);
    std::printf("generation_calls %d\n", generation_calls);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "compat_driver: %s\n", e.what());
    return 1;
  }
  return 0;
}
