// Headless device driver for the YMRT reference's own wavefront kernels,
// rebuilt for sm_100a (the "reference CUDA" baseline).
//
// TEST AND BASELINE INFRASTRUCTURE ONLY. Built by oracle/build_ref.py
// (build_gpu) into oracle/_ref/libymrt_refgpu.so from the reference sources
// where they lie; only tests/ and bench.py load it, to time the reference's
// kernels beside ymrt_b200's and to compare their outputs. The ymrt_b200
// product never links or calls it.
//
// What it does, in the reference's own terms:
//  * loads a .ymtmp scene with the reference's parser and scene module
//    (src/core/YMParser.cpp:2330), which uploads each mesh to the device as it
//    is created (src/GeometryDefines.h:171-174 TriangleMesh::Upload);
//  * prepares it as GuiModule::UpdateScene does (shared with the host oracle,
//    oracle/ref_prepare.h) and copies every scene array to the device the way
//    UpdateScene's device block does (src/core/GuiModule.cpp:173-272);
//  * allocates the wave queues with the reference's own AllocateRayCounter /
//    AllocateShadingRayData / AllocateHitData / AllocateShadowRayData
//    (src/Shading.cu:1067-1163, MAX_RAY_COUNT = 1 Mi rays);
//  * renders a frame with the wave loop of RenderModule::PathTracingExecuteTask
//    (src/core/RenderModule.cpp:494-653), calling the reference's stage
//    launchers RayGenerationPathTracing, RayTracePathTracing and
//    RayShadingPathTracing (src/Shading.cu:1727, 1903, 2304) on one stream,
//    with the same host synchronisation after each stage.
//
// The kernels are the reference's, compiled from a build-time copy of
// src/Shading.cu with one read rewritten (RayTransfer::GetMaxPriorityRecord
// returns a reference to a temporary; the copy reads the priority directly).
// Device time is taken with CUDA events around the wave loop.
#include YMRT_SHADING_SOURCE

#include "core/SceneModule.h"
#include "core/YMParser.h"

#include "ref_prepare.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>

using namespace YMRT;

namespace {

struct GpuContext {
  std::shared_ptr<SceneModule> module;
  std::vector<uint32_t> instance_old_index;
  Scene device_scene{};  // host copy of the Scene struct, its arrays on the device
  std::vector<void*> owned;
  RenderSetting setting{};
  int width = 0, height = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  RayCounterData counters{};
  ShadingRayData shading{};
  HitData hits{};
  ShadowRayData shadow{};
  glm::vec4* image = nullptr;
  double last_ms = 0.0, last_wall_ms = 0.0;
  bool profile_stages = false;
  cudaEvent_t st0 = nullptr, st1 = nullptr;
  double stage_ms[3] = {0.0, 0.0, 0.0};  // generation, trace, shading (profiled frames only)
  uint32_t waves = 0;
  std::string error;
  // path-vertex recording (ymrefgpu_set_recorder)
  uint32_t* rec_watch = nullptr;
  uint32_t* rec_out = nullptr;
  uint32_t* rec_count = nullptr;
  uint32_t rec_capacity = 0;
};

constexpr int kRecordWords = 24;

// Appends the hit-queue entries of watched pixels to the record array (see
// ymrefgpu_set_recorder): pixel, depth, flags (1 hit, 2 volume, 4 back),
// instance, triangle, t, origin[3], direction[3], barycentrics[3],
// throughput[3], received light[3], sample index, 2 unused.
__global__ void k_record_hits(HitData hits, uint32_t n_hits, uint32_t width, uint32_t n_pixels,
                              const uint32_t* __restrict__ watch, uint32_t* out, uint32_t* count, uint32_t capacity) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n_hits) return;
  const uint32_t pixel = (uint32_t)hits.hit_data_pixel_position_y[i] * width + (uint32_t)hits.hit_data_pixel_position_x[i];
  if (pixel >= n_pixels || !((watch[pixel >> 5] >> (pixel & 31u)) & 1u)) return;
  const uint32_t k = atomicAdd(count, 1u);
  if (k >= capacity) return;
  const HitRecord h = hits.hit_data_hit_record[i];
  const Ray ray = hits.hit_data_ray[i];
  const glm::vec3 tp = hits.hit_data_throughput[i], light = hits.hit_data_received_light[i];
  uint32_t* o = out + (size_t)k * kRecordWords;
  o[0] = pixel;
  o[1] = (uint32_t)hits.hit_data_ray_depth[i];
  o[2] = 1u | (h.volume_hit ? 2u : 0u) | (h.hit_back ? 4u : 0u);
  o[3] = h.hit_instance_idx;
  o[4] = h.hit_triangle_idx;
  o[5] = __float_as_uint(h.hit_t);
  for (int c = 0; c < 3; ++c) {
    o[6 + c] = __float_as_uint(ray.origin[c]);
    o[9 + c] = __float_as_uint(ray.direction[c]);
    o[12 + c] = __float_as_uint(h.hit_barycentric[c]);
    o[15 + c] = __float_as_uint(tp[c]);
    o[18 + c] = __float_as_uint(light[c]);
  }
  o[21] = (uint32_t)hits.hit_data_pixel_sample_index[i];
  o[22] = o[23] = 0u;
}

template <typename T>
bool upload(GpuContext* c, T** dst, const T* src, size_t count) {
  *dst = nullptr;
  if (count == 0) return true;
  void* p = nullptr;
  if (cudaMalloc(&p, sizeof(T) * count) != cudaSuccess) return false;
  c->owned.push_back(p);
  if (cudaMemcpy(p, src, sizeof(T) * count, cudaMemcpyHostToDevice) != cudaSuccess) return false;
  *dst = static_cast<T*>(p);
  return true;
}

}  // namespace

extern "C" {

// Same settings block as the host oracle's (oracle/ref_harness.cpp).
struct YmrefGpuSettings {
  int spp;
  int ray_depth;
  int sampler_type;
  int enable_shape_light;
  int enable_distant_light;
  int enable_volume_scattering;
  int enable_env_light;
  int enable_russian_roulette;
  int enable_indirect_clamp;
  float indirect_limit;
};

const char* ymrefgpu_last_error(void* handle) { return static_cast<GpuContext*>(handle)->error.c_str(); }

void* ymrefgpu_scene_load(const char* path, const uint32_t* halton_perm, size_t perm_len, int width, int height,
                          int device) {
  size_t table = 0;
  for (uint32_t i = 0; i < prime_count; ++i) table += primes[i];
  if (perm_len != table || width <= 0 || height <= 0) return nullptr;
  if (cudaSetDevice(device) != cudaSuccess) return nullptr;
  auto c = new GpuContext();
  c->device = device;
  c->width = width;
  c->height = height;
  try {
    c->module = std::make_shared<SceneModule>();
    SceneParser parser;
    if (!parser.parsing_scene(path, c->module)) {
      delete c;
      return nullptr;
    }
    SceneModule& m = *c->module;
    GuiModule::PrepareScene(m, halton_perm, perm_len, width, height, &c->instance_old_index);
    Scene host = GuiModule::HostScene(m);
    Scene& d = c->device_scene;
    ImageTileCache empty_cache;
    std::memset(&empty_cache, 0, sizeof(empty_cache));
    bool ok = upload(c, &d.camera, host.camera, CAMERA_COUNT) &&
              upload(c, &d.geometries, host.geometries, host.geometry_count) &&
              upload(c, &d.primitive_instances, host.primitive_instances, host.primitive_instance_count) &&
              upload(c, &d.top_nodes, host.top_nodes, host.top_node_count) &&
              upload(c, &d.transforms, host.transforms, host.transform_count) &&
              upload(c, &d.i_transforms, host.i_transforms, host.transform_count) &&
              upload(c, &d.materials, host.materials, host.material_count) &&
              upload(c, &d.distant_lights, host.distant_lights, host.distant_light_count) &&
              upload(c, &d.shape_lights, host.shape_lights, host.shape_light_count) &&
              upload(c, &d.shape_light_sample_table, host.shape_light_sample_table, host.shape_light_count) &&
              upload(c, &d.volumes, host.volumes, host.volume_count) &&
              upload(c, &d.textures, host.textures, host.texture_count) &&
              upload(c, &d.image_tile_cache, &empty_cache, 1) &&
              upload(c, &d.sampler_data.halton_permute_table, halton_perm, perm_len) &&
              upload(c, &d.sampler_data.sobol_matrices, (const uint32_t*)sobol_matrices32, (size_t)4096 * 32) &&
              upload(c, &d.render_setting, &c->setting, 1);
    d.camera_count = CAMERA_COUNT;
    d.geometry_count = host.geometry_count;
    d.primitive_instance_count = host.primitive_instance_count;
    d.top_node_count = host.top_node_count;
    d.transform_count = host.transform_count;
    d.material_count = host.material_count;
    d.distant_light_count = host.distant_light_count;
    d.shape_light_count = host.shape_light_count;
    d.volume_count = host.volume_count;
    d.texture_count = host.texture_count;
    if (!ok) throw std::runtime_error("scene upload failed");
    AllocateRayCounter(c->counters);
    AllocateShadingRayData(c->shading);
    AllocateHitData(c->hits);
    AllocateShadowRayData(c->shadow);
    CUDA_CHECK(cudaStreamCreate(&c->stream));
    CUDA_CHECK(cudaEventCreate(&c->ev0));
    CUDA_CHECK(cudaEventCreate(&c->ev1));
    CUDA_CHECK(cudaEventCreate(&c->st0));
    CUDA_CHECK(cudaEventCreate(&c->st1));
    CUDA_CHECK(cudaMalloc(&c->image, sizeof(glm::vec4) * (size_t)width * height));
  } catch (const std::exception& e) {
    fprintf(stderr, "ymrefgpu_scene_load: %s\n", e.what());
    delete c;
    return nullptr;
  }
  return c;
}

void ymrefgpu_scene_free(void* handle) {
  auto c = static_cast<GpuContext*>(handle);
  if (!c) return;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  try {
    ReleaseRayCounter(c->counters);
    ReleaseShadingRayData(c->shading);
    ReleaseHitData(c->hits);
    ReleaseShadowRayData(c->shadow);
  } catch (...) {
  }
  if (c->rec_watch) cudaFree(c->rec_watch);
  if (c->rec_out) cudaFree(c->rec_out);
  if (c->rec_count) cudaFree(c->rec_count);
  for (void* p : c->owned) cudaFree(p);
  if (c->image) cudaFree(c->image);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->st0) cudaEventDestroy(c->st0);
  if (c->st1) cudaEventDestroy(c->st1);
  if (c->stream) cudaStreamDestroy(c->stream);
  c->module.reset();  // frees the meshes' device copies
  delete c;
}

int ymrefgpu_set_settings(void* handle, const YmrefGpuSettings* s) {
  auto c = static_cast<GpuContext*>(handle);
  RenderSetting& r = c->setting;
  r.ssp = s->spp;
  r.ray_depth = s->ray_depth;
  r.sampler_type = s->sampler_type;
  r.enable_shape_light = s->enable_shape_light;
  r.enable_distant_light = s->enable_distant_light != 0;
  r.enable_volume_scattering = s->enable_volume_scattering != 0;
  r.enable_env_light = s->enable_env_light != 0;
  r.enable_russian_roulette = s->enable_russian_roulette != 0;
  r.enable_indirect_clamp = s->enable_indirect_clamp != 0;
  r.indirect_limit = s->indirect_limit;
  cudaSetDevice(c->device);
  return cudaMemcpy(c->device_scene.render_setting, &r, sizeof(RenderSetting), cudaMemcpyHostToDevice) == cudaSuccess
             ? 0
             : -1;
}

// Renders one frame (tiles [tile_begin, tile_end), 0/0 = all) into the
// context's device image and copies it to out_rgba when that is not null.
// Returns 0, or -1 on a CUDA error (message in ymrefgpu_last_error).
int ymrefgpu_render_frame(void* handle, int frame_index, int tile_begin, int tile_end, float* out_rgba) {
  auto c = static_cast<GpuContext*>(handle);
  if (frame_index < 1 || tile_begin < 0) return -1;
  try {
    CUDA_CHECK(cudaSetDevice(c->device));
    const RenderSetting& rs = c->setting;
    const uint32_t w = c->width, h = c->height;
    const uint32_t tiles_x = (w + TILE_X_RES - 1) / TILE_X_RES;
    const uint32_t tiles_y = (h + TILE_Y_RES - 1) / TILE_Y_RES;
    const uint32_t total = tiles_x * tiles_y;
    const uint32_t t_end = tile_end <= 0 ? total : std::min<uint32_t>((uint32_t)tile_end, total);
    const bool partial = tile_begin > 0 || t_end < total;
    const uint32_t spp = (uint32_t)rs.ssp;
    if (spp == 0 || spp * TILE_PIXEL_COUNT > MAX_RAY_COUNT) return -1;

    CUDA_CHECK(cudaMemsetAsync(c->image, 0, sizeof(glm::vec4) * (size_t)w * h, c->stream));
    Scene* scene_device = nullptr;
    HaltonEnumerator* halton_device = nullptr;
    CUDA_CHECK(cudaMalloc(&scene_device, sizeof(Scene)));
    CUDA_CHECK(cudaMemcpyAsync(scene_device, &c->device_scene, sizeof(Scene), cudaMemcpyHostToDevice, c->stream));
    HaltonEnumerator halton(w, h);
    CUDA_CHECK(cudaMalloc(&halton_device, sizeof(HaltonEnumerator)));
    CUDA_CHECK(cudaMemcpyAsync(halton_device, &halton, sizeof(HaltonEnumerator), cudaMemcpyHostToDevice, c->stream));
    RayCounter* counter_host = c->counters.ray_counter_host;
    RayCounter* counter_device = c->counters.ray_counter_device;
    counter_host->hit_counter = 0;
    counter_host->shading_ray_counter = 0;
    counter_host->shadow_ray_counter = 0;
    CUDA_CHECK(cudaMemcpyAsync(counter_device, counter_host, sizeof(RayCounter), cudaMemcpyHostToDevice, c->stream));
    CUDA_CHECK(cudaStreamSynchronize(c->stream));

    const auto wall0 = std::chrono::steady_clock::now();
    CUDA_CHECK(cudaEventRecord(c->ev0, c->stream));
    uint32_t next_tile = (uint32_t)tile_begin;
    c->stage_ms[0] = c->stage_ms[1] = c->stage_ms[2] = 0.0;
    c->waves = 0;
    // Optional per-stage device times (events around each stage launcher; the
    // loop synchronises after every stage anyway).
    auto stage_begin = [&]() {
      if (c->profile_stages) CUDA_CHECK(cudaEventRecord(c->st0, c->stream));
    };
    auto stage_end = [&](int k) {
      if (!c->profile_stages) return;
      CUDA_CHECK(cudaEventRecord(c->st1, c->stream));
      CUDA_CHECK(cudaEventSynchronize(c->st1));
      float ms = 0.0f;
      CUDA_CHECK(cudaEventElapsedTime(&ms, c->st0, c->st1));
      c->stage_ms[k] += ms;
    };
    while (counter_host->shading_ray_counter > 0 || next_tile < t_end) {
      uint32_t batch = (MAX_RAY_COUNT - counter_host->shading_ray_counter) / (TILE_PIXEL_COUNT * spp);
      if (partial) batch = std::min(batch, t_end - next_tile);  // the full-frame loop is the reference's, uncapped
      ++c->waves;
      stage_begin();
      RayGenerationPathTracing(frame_index, rs, scene_device, halton_device, counter_device, next_tile, batch, w, h,
                               tiles_x, tiles_y, c->shading, c->stream);
      stage_end(0);
      next_tile += batch;
      counter_host->shading_ray_counter += batch * spp * TILE_PIXEL_COUNT;
      CUDA_CHECK(cudaMemcpyAsync(counter_device, counter_host, sizeof(RayCounter), cudaMemcpyHostToDevice, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));

      stage_begin();
      RayTracePathTracing(frame_index, rs, scene_device, counter_device, counter_host, w, h, c->image, c->shading,
                          c->hits, c->stream);
      stage_end(1);
      CUDA_CHECK(cudaMemcpyAsync(counter_host, counter_device, sizeof(RayCounter), cudaMemcpyDeviceToHost, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
      if (c->rec_out && counter_host->hit_counter > 0) {
        const uint32_t n_hits = counter_host->hit_counter;
        k_record_hits<<<(n_hits + 255) / 256, 256, 0, c->stream>>>(c->hits, n_hits, w, w * h, c->rec_watch, c->rec_out,
                                                                  c->rec_count, c->rec_capacity);
        CUDA_CHECK(cudaGetLastError());
        CUDA_CHECK(cudaStreamSynchronize(c->stream));
      }
      counter_host->shading_ray_counter = 0;
      CUDA_CHECK(cudaMemcpyAsync(counter_device, counter_host, sizeof(RayCounter), cudaMemcpyHostToDevice, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));

      stage_begin();
      RayShadingPathTracing(frame_index, rs, scene_device, counter_device, counter_host, w, h, c->image, c->shading,
                            c->hits, c->shadow, c->stream);
      stage_end(2);
      CUDA_CHECK(cudaMemcpyAsync(counter_host, counter_device, sizeof(RayCounter), cudaMemcpyDeviceToHost, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
      counter_host->hit_counter = 0;
      CUDA_CHECK(cudaMemcpyAsync(counter_device, counter_host, sizeof(RayCounter), cudaMemcpyHostToDevice, c->stream));
      CUDA_CHECK(cudaStreamSynchronize(c->stream));
      if (counter_host->shading_ray_counter > MAX_RAY_COUNT) throw std::runtime_error("wave queue overflow");
    }
    CUDA_CHECK(cudaEventRecord(c->ev1, c->stream));
    CUDA_CHECK(cudaEventSynchronize(c->ev1));
    c->last_wall_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - wall0).count();
    float ms = 0.0f;
    CUDA_CHECK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
    c->last_ms = ms;
    CUDA_CHECK(cudaFree(scene_device));
    CUDA_CHECK(cudaFree(halton_device));
    if (out_rgba)
      CUDA_CHECK(cudaMemcpy(out_rgba, c->image, sizeof(glm::vec4) * (size_t)w * h, cudaMemcpyDeviceToHost));
  } catch (const std::exception& e) {
    c->error = e.what();
    return -1;
  }
  return 0;
}

// Device time (CUDA events on the render stream) and host wall time of the
// last frame's wave loop, in milliseconds.
double ymrefgpu_last_render_ms(void* handle) { return static_cast<GpuContext*>(handle)->last_ms; }
double ymrefgpu_last_wall_ms(void* handle) { return static_cast<GpuContext*>(handle)->last_wall_ms; }

// Per-stage device times of the last frame rendered with profiling on
// (generation, trace, shading, in ms) and its wave count.
void ymrefgpu_set_profiling(void* handle, int on) { static_cast<GpuContext*>(handle)->profile_stages = on != 0; }

// Path-vertex recording for parity diagnostics: during the renders that
// follow, after every trace stage a harness kernel reads the hit queue the
// reference's trace stage wrote (hit record, ray, throughput, received light,
// pixel, depth: src/Shading.cu:1880-1902) and appends the entries of watched
// pixels (one bit per pixel in watch_bits, host memory, width*height bits)
// to a device array of `capacity` records of 24 words, the layout
// ymrt_debug_record_paths writes. The reference's kernels are not changed;
// only vertices that hit something are queued there, so misses are not
// recorded. capacity <= 0 stops recording and frees the arrays. Returns 0,
// or -1 when the device arrays cannot be set up.
int ymrefgpu_set_recorder(void* handle, const uint32_t* watch_bits, int capacity) {
  auto c = static_cast<GpuContext*>(handle);
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  if (c->rec_watch) cudaFree(c->rec_watch);
  if (c->rec_out) cudaFree(c->rec_out);
  if (c->rec_count) cudaFree(c->rec_count);
  c->rec_watch = nullptr;
  c->rec_out = nullptr;
  c->rec_count = nullptr;
  c->rec_capacity = 0;
  if (capacity <= 0 || !watch_bits) return 0;
  const size_t words = ((size_t)c->width * c->height + 31) / 32;
  if (cudaMalloc(&c->rec_watch, words * 4) != cudaSuccess ||
      cudaMalloc(&c->rec_out, (size_t)kRecordWords * 4 * (size_t)capacity) != cudaSuccess ||
      cudaMalloc(&c->rec_count, 4) != cudaSuccess ||
      cudaMemcpy(c->rec_watch, watch_bits, words * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(c->rec_count, 0, 4) != cudaSuccess) {
    ymrefgpu_set_recorder(handle, nullptr, 0);
    return -1;
  }
  c->rec_capacity = (uint32_t)capacity;
  return 0;
}
// Copies the records written so far (at most `capacity`) into out; returns
// how many were recorded (those past the recorder's capacity are counted,
// not written), or -1.
int ymrefgpu_read_records(void* handle, void* out, int capacity) {
  auto c = static_cast<GpuContext*>(handle);
  cudaSetDevice(c->device);
  if (cudaDeviceSynchronize() != cudaSuccess || !c->rec_count) return -1;
  uint32_t n = 0;
  if (cudaMemcpy(&n, c->rec_count, 4, cudaMemcpyDeviceToHost) != cudaSuccess) return -1;
  const uint32_t kept = std::min<uint32_t>(std::min<uint32_t>(n, c->rec_capacity), (uint32_t)std::max(capacity, 0));
  if (kept && cudaMemcpy(out, c->rec_out, (size_t)kRecordWords * 4 * kept, cudaMemcpyDeviceToHost) != cudaSuccess)
    return -1;
  return (int)n;
}
uint32_t ymrefgpu_last_stage_ms(void* handle, double* out3) {
  auto c = static_cast<GpuContext*>(handle);
  for (int k = 0; k < 3; ++k) out3[k] = c->stage_ms[k];
  return c->waves;
}

}  // extern "C"
