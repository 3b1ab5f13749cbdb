// C ABI of ymrt_b200 (include/ymrt.h): contexts, scene upload, the frame
// loop that drives the wavefront kernels, and the known-answer entry points.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ymrt.h"
#include "../../include/ymrt_compat.h"
#include "kernels.h"
#include "scene_host.h"

using namespace ym;

struct ymrt_host_scene {
  HostScene s;
};

namespace {

thread_local std::string g_last_error;

// Device allocations still to fail on purpose (ymrt_debug_fail_allocations):
// a host-side fault injection for the error paths of allocation failures.
std::atomic<int> g_failing_allocations{0};

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t bytes = 0;
  ~DeviceBuffer() { release(); }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    bytes = 0;
  }
  cudaError_t ensure(size_t n) {
    if (n <= bytes && ptr) return cudaSuccess;
    release();
    if (g_failing_allocations.load() > 0 && g_failing_allocations.fetch_sub(1) > 0) return cudaErrorMemoryAllocation;
    cudaError_t e = cudaMalloc(&ptr, n ? n : 16);
    if (e == cudaSuccess) bytes = n;
    return e;
  }
  template <typename T>
  T* as() const {
    return static_cast<T*>(ptr);
  }
};

std::vector<uint32_t> first_primes(int n) {
  std::vector<uint32_t> p;
  for (uint32_t c = 2; (int)p.size() < n; ++c) {
    bool prime = true;
    for (uint32_t q : p) {
      if (q * q > c) break;
      if (c % q == 0) {
        prime = false;
        break;
      }
    }
    if (prime) p.push_back(c);
  }
  return p;
}

}  // namespace

struct ymrt_context {
  int device = 0;
  cudaStream_t stream = nullptr;
  std::string error;
  uint32_t capacity = 1u << 21;
  // two path pools (ping-pong), one hit pool, counters
  DeviceBuffer pool_buf[2], hit_buf, counters_buf, image_buf, jobs_buf;
  PathPool pool[2]{};
  HitPool hits{};
  uint32_t pool_capacity = 0;
  WaveCounters* counters_host = nullptr;  // pinned
  WaveControl* ctl_host = nullptr;        // pinned
  DeviceBuffer ctl_buf;
  // CUDA graph of the wave loop (a while-loop node around two waves), cached
  // for the memory and options it was captured with
  bool graph_loop = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  std::vector<uintptr_t> graph_key;
  void drop_graph() {
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    graph_exec = nullptr;
    graph = nullptr;
    graph_key.clear();
  }
  cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
  bool profiling = false;
  cudaEvent_t ev_stage[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  std::vector<uint32_t> primes, prime_sums;
  WaveCounters batch_counters{};  // frame totals across the launch groups of one batch
  // wave options (ymrt_set_option)
  bool sort_hits = true;
  uint32_t trace_block = 128;  // threads per block of k_extend / k_connect (YMRT_OPT_TRACE_BLOCK)
  bool defer_shadows = true;
  bool sort_rays = true;  // YMRT_OPT_SORT_RAYS
  DeviceBuffer shadow_buf;
  ShadowQueue shadow_queue{};
  // pinned host staging of scene uploads (grown on demand, kept)
  void* staging = nullptr;
  size_t staging_bytes = 0;
  // device buffers of freed scenes' packed uploads, kept for the next upload
  // (at most kSpareSceneBuffers, the largest), so that replacing a scene
  // does not allocate
  static constexpr size_t kSpareSceneBuffers = 2;
  std::vector<std::unique_ptr<DeviceBuffer>> spare_scene_buffers;
  std::unique_ptr<DeviceBuffer> take_spare(size_t n) {
    size_t best = spare_scene_buffers.size();
    for (size_t k = 0; k < spare_scene_buffers.size(); ++k)
      if (spare_scene_buffers[k]->bytes >= n &&
          (best == spare_scene_buffers.size() || spare_scene_buffers[k]->bytes < spare_scene_buffers[best]->bytes))
        best = k;
    if (best == spare_scene_buffers.size()) return std::unique_ptr<DeviceBuffer>(new DeviceBuffer());
    std::unique_ptr<DeviceBuffer> b = std::move(spare_scene_buffers[best]);
    spare_scene_buffers.erase(spare_scene_buffers.begin() + (long)best);
    return b;
  }
  void keep_spare(std::unique_ptr<DeviceBuffer> b) {
    spare_scene_buffers.push_back(std::move(b));
    std::sort(spare_scene_buffers.begin(), spare_scene_buffers.end(),
              [](const std::unique_ptr<DeviceBuffer>& a, const std::unique_ptr<DeviceBuffer>& c) {
                return a->bytes > c->bytes;
              });
    while (spare_scene_buffers.size() > kSpareSceneBuffers) spare_scene_buffers.pop_back();
  }
  cudaError_t ensure_staging(size_t n) {
    if (n <= staging_bytes && staging) return cudaSuccess;
    if (staging) cudaFreeHost(staging);
    staging = nullptr;
    staging_bytes = 0;
    cudaError_t e = cudaMallocHost(&staging, n);
    if (e == cudaSuccess) staging_bytes = n;
    return e;
  }

  int fail(int code, const std::string& msg) {
    error = msg;
    g_last_error = msg;
    return code;
  }
  int cuda_fail(cudaError_t e, const char* what) {
    return fail(e == cudaErrorMemoryAllocation ? YMRT_ERR_OOM : YMRT_ERR_CUDA,
                std::string(what) + ": " + cudaGetErrorString(e));
  }

  int ensure_pools() {
    if (pool_capacity == capacity) return YMRT_OK;
    const size_t n = capacity;
    const size_t pool_bytes =
        n * (4 * sizeof(float4) + 2 * sizeof(uint2) + sizeof(uint4) + sizeof(RayTransfer) + sizeof(uint32_t) + 1) + 64;
    for (int k = 0; k < 2; ++k) {
      cudaError_t e = pool_buf[k].ensure(pool_bytes);
      if (e != cudaSuccess) return cuda_fail(e, "allocating path pool");
      char* p = pool_buf[k].as<char>();
      PathPool& P = pool[k];
      P.ray_o = reinterpret_cast<float4*>(p); p += n * sizeof(float4);
      P.ray_d = reinterpret_cast<float4*>(p); p += n * sizeof(float4);
      P.throughput = reinterpret_cast<float4*>(p); p += n * sizeof(float4);
      P.radiance = reinterpret_cast<float4*>(p); p += n * sizeof(float4);
      P.sampler = reinterpret_cast<uint4*>(p); p += n * sizeof(uint4);
      P.pixel_flags = reinterpret_cast<uint2*>(p); p += n * sizeof(uint2);
      P.last_hit = reinterpret_cast<uint2*>(p); p += n * sizeof(uint2);
      P.transfer = reinterpret_cast<RayTransfer*>(p); p += n * sizeof(RayTransfer);
      p = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(p) + 15) & ~uintptr_t(15));
      P.path_id = reinterpret_cast<uint32_t*>(p); p += n * sizeof(uint32_t);
      P.transfer_count = reinterpret_cast<uint8_t*>(p);
      P.capacity = capacity;
    }
    const size_t hit_bytes = n * (sizeof(float4) + sizeof(uint4) + kMaxNearby * sizeof(uint4) +
                                  kMaxBoundaryRecord * sizeof(float) + sizeof(uint32_t) + 1) +
                             kRayBinWords * sizeof(uint32_t) + 2 * n * sizeof(uint32_t) + 16;
    cudaError_t e = hit_buf.ensure(hit_bytes);
    if (e != cudaSuccess) return cuda_fail(e, "allocating hit pool");
    char* h = hit_buf.as<char>();
    hits.bary_t = reinterpret_cast<float4*>(h); h += n * sizeof(float4);
    hits.ids = reinterpret_cast<uint4*>(h); h += n * sizeof(uint4);
    hits.nearby = reinterpret_cast<uint4*>(h); h += n * kMaxNearby * sizeof(uint4);
    hits.vol_w = reinterpret_cast<float*>(h); h += n * kMaxBoundaryRecord * sizeof(float);
    hits.order = reinterpret_cast<uint32_t*>(h); h += n * sizeof(uint32_t);
    hits.ray_bins = reinterpret_cast<uint32_t*>(h); h += kRayBinWords * sizeof(uint32_t);
    hits.ray_key = reinterpret_cast<uint32_t*>(h); h += n * sizeof(uint32_t);
    hits.ray_order = reinterpret_cast<uint32_t*>(h); h += n * sizeof(uint32_t);
    hits.bucket = reinterpret_cast<uint8_t*>(h);
    pool_capacity = capacity;
    shadow_queue = ShadowQueue{};
    return YMRT_OK;
  }

  // Deferred shadow rays: at most kShadowRaysPerVertex per shaded path.
  static constexpr uint32_t kShadowRaysPerVertex = 4;
  int ensure_shadow_queue() {
    const size_t n = (size_t)pool_capacity * kShadowRaysPerVertex;
    if (shadow_queue.capacity == n) return YMRT_OK;
    cudaError_t e = shadow_buf.ensure(n * (3 * sizeof(float4) + sizeof(uint32_t)));
    if (e != cudaSuccess) return cuda_fail(e, "allocating shadow-ray queue");
    float4* q = shadow_buf.as<float4>();
    shadow_queue = ShadowQueue{q, q + n, q + 2 * n, reinterpret_cast<uint32_t*>(q + 3 * n), (uint32_t)n};
    return YMRT_OK;
  }
};

namespace {

// Whether a default material reads any texture (parameters, normal or bump map).
bool material_textures(const DefaultMtl& d) {
  const uint32_t tex[] = {d.diffuse_albedo_tex, d.alpha_x_tex, d.specular_albedo_tex, d.alpha_y_tex,
                          d.specular_weight_tex, d.metalness_tex, d.transmission_weight_tex, d.normal_mapping_tex,
                          d.bump_mapping_tex, d.coat_albedo_tex, d.coat_weight_tex, d.coat_thickness_tex,
                          d.coat_roughness_x_tex, d.coat_roughness_y_tex};
  for (uint32_t t : tex)
    if (t != kEmpty) return true;
  return false;
}

// DeviceScene::textured: a material reads textures, or a medium's density
// graph holds a solid node beyond fBm (both need the full node set).
bool uses_textures(const std::vector<Material>& materials, const std::vector<Texture>& textures) {
  for (const Material& m : materials)
    if (m.material_type == kDefaultMtl && material_textures(m.default_mtl)) return true;
  for (const Texture& t : textures)
    if ((t.type >= kTexChecker && t.type <= kTexWave && t.type != kTexFbm) || t.type == kTexImage) return true;
  return false;
}

// Shading bucket of a hit on `inst`: pass-through boundaries, lights and
// invalid materials share the cheap bucket; a default material's bucket is
// the set of lobes its constant parameters switch on (the lobes
// init_layered_lobes builds), so hits in one bucket run the same BSDF code.
uint32_t shading_bucket(const HostScene& s, const Instance& inst) {
  if (inst.treat_as_boundary || inst.material_idx >= s.materials.size()) return kBucketCheap;
  const Material& m = s.materials[inst.material_idx];
  if (m.material_type != kDefaultMtl) return kBucketCheap;
  const DefaultMtl& d = m.default_mtl;
  if (material_textures(d)) return kBucketLobes + 31u;  // lobes vary over the surface
  const bool not_metal = d.metalness < 1.0f;
  uint32_t mask = 0;
  if (d.coat_weight > 0.0f) mask |= 1u;
  if (d.metalness > 0.0f) mask |= 2u;
  if (not_metal && d.specular_weight > 0.0f) mask |= 4u;
  if (not_metal && d.transmission_weight > 0.0f) mask |= 8u;
  if (not_metal && d.transmission_weight < 1.0f) mask |= 16u;
  return kBucketLobes + mask;
}

}  // namespace

namespace {

// Constant-memory scene slots (kMaxSceneSlots per device) are shared by every
// context on a device. A call leases the slots it uploads scenes into for as
// long as its kernels may read them, so that calls from several contexts on
// one device (one context per host thread) never overwrite each other's
// scenes; it waits while another call holds too many. The lease ends after
// the call's stream is synchronised.
struct DeviceSlots {
  std::mutex m;
  std::condition_variable cv;
  uint64_t used = 0;  // bit k: slot k leased
};
DeviceSlots g_device_slots[128];

class SlotLease {
 public:
  SlotLease(ymrt_context* ctx, uint32_t n);
  ~SlotLease();
  SlotLease(const SlotLease&) = delete;
  SlotLease& operator=(const SlotLease&) = delete;
  bool ok() const { return ok_; }
  const uint32_t* slots() const { return slots_; }
  uint32_t slot(size_t k) const { return slots_[k]; }
  // Uploads scenes[k] into the k-th leased slot (and the prime tables).
  cudaError_t upload(const DeviceScene* scenes, uint32_t n) const;

 private:
  ymrt_context* ctx_;
  uint64_t mask_ = 0;
  uint32_t slots_[kMaxSceneSlots] = {};
  uint32_t n_ = 0;
  bool ok_ = false;
};

}  // namespace

struct ymrt_scene {
  ymrt_context* ctx = nullptr;
  DeviceScene dev{};
  std::vector<Material> materials;  // host copy (material parameters can be updated)
  std::vector<Texture> textures;    // host copy (grid nodes can be attached)
  std::map<uint32_t, std::unique_ptr<DeviceBuffer>> grids;  // grid values per texture node
  std::vector<std::unique_ptr<DeviceBuffer>> buffers;
  int width = 0, height = 0;
  uint64_t triangles = 0;
  // top-level rebuilds on the device (ymrt_scene_set_transforms)
  struct TopLevel {
    uint32_t max_leaf = 3;
    uint32_t node_count = 0;                 // top-level wide nodes
    std::vector<uint32_t> file_index;        // file index of each instance (host copy)
    std::vector<vec3> transform_scales;      // each transform's own scale (host copy)
    bool prepared = false;
    int cur = 0;                             // which of the pairs below holds the current order
    DeviceBuffer inst[2], bucket[2], file_idx[2];
    DeviceBuffer scales, items, nodes, mid, kind, left, stack, wide, prims, offsets, inside, camera, counts;
  } top;

  template <typename T>
  cudaError_t upload(const std::vector<T>& v, const T** out) {
    buffers.emplace_back(new DeviceBuffer());
    DeviceBuffer& b = *buffers.back();
    cudaError_t e = b.ensure(std::max<size_t>(v.size() * sizeof(T), 16));
    if (e != cudaSuccess) return e;
    if (!v.empty()) e = cudaMemcpyAsync(b.ptr, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    *out = b.as<T>();
    return e;
  }

  // Packed upload: arrays gathered with pack() go to the device with one
  // allocation and one copy from the context's pinned staging buffer
  // (pack_commit), instead of an allocation and a pageable copy each. The
  // host arrays must stay unchanged until pack_commit returns; the device
  // pointers are set by pack_commit.
  struct PackItem {
    const void* src;
    size_t bytes;
    const void** out;
  };
  std::vector<PackItem> packed;
  std::vector<DeviceBuffer*> packed_buffers;  // the buffers pack_commit filled (returned to the context on free)
  template <typename T>
  void pack(const T* src, size_t count, const T** out) {
    packed.push_back(PackItem{src, count * sizeof(T), reinterpret_cast<const void**>(out)});
  }
  template <typename T>
  void pack(const std::vector<T>& v, const T** out) {
    pack(v.data(), v.size(), out);
  }
  cudaError_t pack_commit() {
    size_t total = 0;
    for (const PackItem& p : packed) total += (std::max<size_t>(p.bytes, 16) + 255) & ~size_t(255);
    cudaError_t e = cudaSuccess;
    if (total) {
      buffers.push_back(ctx->take_spare(total));
      DeviceBuffer& b = *buffers.back();
      packed_buffers.push_back(&b);
      // the staging buffer is reused: the previous upload's copy must be done
      if ((e = cudaStreamSynchronize(ctx->stream)) == cudaSuccess) e = b.ensure(total);
      if (e == cudaSuccess) e = ctx->ensure_staging(total);
      if (e == cudaSuccess) {
        unsigned char* host = static_cast<unsigned char*>(ctx->staging);
        // the host copies in pieces of at most 4 MiB, spread over a few
        // threads (one thread copies well below the bus's rate)
        struct Piece {
          unsigned char* dst;
          const unsigned char* src;
          size_t bytes;
        };
        std::vector<Piece> pieces;
        constexpr size_t kPiece = size_t(4) << 20;
        size_t at = 0;
        for (const PackItem& p : packed) {
          for (size_t o = 0; o < p.bytes; o += kPiece)
            pieces.push_back(Piece{host + at + o, static_cast<const unsigned char*>(p.src) + o,
                                   std::min(kPiece, p.bytes - o)});
          *p.out = b.as<unsigned char>() + at;
          at += (std::max<size_t>(p.bytes, 16) + 255) & ~size_t(255);
        }
        const size_t n_threads =
            std::min<size_t>({pieces.size(), (size_t)std::max(1u, std::thread::hardware_concurrency()), 8});
        auto copy_share = [&](size_t t) {
          for (size_t k = t; k < pieces.size(); k += n_threads) std::memcpy(pieces[k].dst, pieces[k].src, pieces[k].bytes);
        };
        if (n_threads <= 1 || total < (size_t(4) << 20)) {
          for (size_t t = 0; t < std::max<size_t>(n_threads, 1); ++t) copy_share(t);
        } else {
          std::vector<std::thread> pool;
          for (size_t t = 1; t < n_threads; ++t) pool.emplace_back(copy_share, t);
          copy_share(0);
          for (std::thread& th : pool) th.join();
        }
        e = cudaMemcpyAsync(b.ptr, host, total, cudaMemcpyHostToDevice, ctx->stream);
      }
    }
    packed.clear();
    return e;
  }
};

namespace {

SlotLease::SlotLease(ymrt_context* ctx, uint32_t n) : ctx_(ctx) {
  if (n == 0 || n > kMaxSceneSlots || ctx->device < 0 || ctx->device >= 128) return;
  DeviceSlots& d = g_device_slots[ctx->device];
  std::unique_lock<std::mutex> lk(d.m);
  d.cv.wait(lk, [&] { return (uint32_t)__builtin_popcountll(~d.used) >= n; });
  for (uint32_t k = 0; k < kMaxSceneSlots && n_ < n; ++k)
    if (!((d.used >> k) & 1ull)) {
      slots_[n_++] = k;
      mask_ |= 1ull << k;
    }
  d.used |= mask_;
  ok_ = true;
}

SlotLease::~SlotLease() {
  if (!mask_) return;
  cudaStreamSynchronize(ctx_->stream);  // no kernel of this call reads the slots any more
  DeviceSlots& d = g_device_slots[ctx_->device];
  {
    std::lock_guard<std::mutex> lk(d.m);
    d.used &= ~mask_;
  }
  d.cv.notify_all();
}

cudaError_t SlotLease::upload(const DeviceScene* scenes, uint32_t n) const {
  if (!ok_ || n > n_) return cudaErrorInvalidValue;
  return upload_constants(scenes, slots_, n, ctx_->primes.data(), ctx_->prime_sums.data(), ctx_->stream);
}

}  // namespace

extern "C" {

int ymrt_create(int device_ordinal, ymrt_context** out) {
  if (!out) return YMRT_ERR_INVALID;
  *out = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    g_last_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
    return YMRT_ERR_NO_DEVICE;
  }
  if (device_ordinal < 0 || device_ordinal >= n) {
    g_last_error = "device ordinal out of range";
    return YMRT_ERR_INVALID;
  }
  std::unique_ptr<ymrt_context> ctx(new (std::nothrow) ymrt_context());
  if (!ctx) return YMRT_ERR_OOM;
  ctx->device = device_ordinal;
  if ((e = cudaSetDevice(device_ordinal)) != cudaSuccess) return ctx->cuda_fail(e, "cudaSetDevice");
  if ((e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking)) != cudaSuccess)
    return ctx->cuda_fail(e, "cudaStreamCreate");
  if ((e = cudaEventCreate(&ctx->ev_start)) != cudaSuccess || (e = cudaEventCreate(&ctx->ev_stop)) != cudaSuccess)
    return ctx->cuda_fail(e, "cudaEventCreate");
  for (auto& ev : ctx->ev_stage)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return ctx->cuda_fail(e, "cudaEventCreate");
  if ((e = cudaMallocHost(&ctx->counters_host, sizeof(WaveCounters))) != cudaSuccess)
    return ctx->cuda_fail(e, "cudaMallocHost");
  if ((e = cudaMallocHost(&ctx->ctl_host, sizeof(WaveControl))) != cudaSuccess)
    return ctx->cuda_fail(e, "cudaMallocHost");
  if ((e = ctx->counters_buf.ensure(sizeof(WaveCounters))) != cudaSuccess) return ctx->cuda_fail(e, "cudaMalloc");
  ctx->primes = first_primes(kHaltonDims);
  ctx->prime_sums.resize(kHaltonDims);
  uint32_t acc = 0;
  for (int i = 0; i < kHaltonDims; ++i) {
    ctx->prime_sums[i] = acc;
    acc += ctx->primes[i];
  }
  *out = ctx.release();
  return YMRT_OK;
}

void ymrt_destroy(ymrt_context* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  for (auto& b : ctx->pool_buf) b.release();
  ctx->hit_buf.release();
  ctx->counters_buf.release();
  ctx->jobs_buf.release();
  ctx->image_buf.release();
  ctx->drop_graph();
  if (ctx->counters_host) cudaFreeHost(ctx->counters_host);
  if (ctx->ctl_host) cudaFreeHost(ctx->ctl_host);
  if (ctx->staging) cudaFreeHost(ctx->staging);
  ctx->spare_scene_buffers.clear();
  ctx->ctl_buf.release();
  if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
  if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
  for (auto& ev : ctx->ev_stage)
    if (ev) cudaEventDestroy(ev);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

const char* ymrt_last_error(const ymrt_context* ctx) { return ctx ? ctx->error.c_str() : g_last_error.c_str(); }

int ymrt_set_queue_capacity(ymrt_context* ctx, uint32_t paths) {
  if (!ctx) return YMRT_ERR_INVALID;
  ctx->capacity = paths ? paths : (1u << 21);
  return YMRT_OK;
}

int ymrt_set_profiling(ymrt_context* ctx, int enable) {
  if (!ctx) return YMRT_ERR_INVALID;
  ctx->profiling = enable != 0;
  return YMRT_OK;
}

int ymrt_set_option(ymrt_context* ctx, int option, int value) {
  if (!ctx) return YMRT_ERR_INVALID;
  switch (option) {
    case YMRT_OPT_SORT_HITS: ctx->sort_hits = value != 0; return YMRT_OK;
    case YMRT_OPT_DEFER_SHADOWS: ctx->defer_shadows = value != 0; return YMRT_OK;
    case YMRT_OPT_GRAPH_LOOP: ctx->graph_loop = value != 0; return YMRT_OK;
    case YMRT_OPT_SORT_RAYS: ctx->sort_rays = value != 0; return YMRT_OK;
    case YMRT_OPT_TRACE_BLOCK:
      if (value != 64 && value != 128 && value != 256)
        return ctx->fail(YMRT_ERR_INVALID, "YMRT_OPT_TRACE_BLOCK must be 64, 128 or 256");
      ctx->trace_block = (uint32_t)value;
      return YMRT_OK;
    default: return ctx->fail(YMRT_ERR_INVALID, "unknown option " + std::to_string(option));
  }
}

int ymrt_get_option(const ymrt_context* ctx, int option, int* value) {
  if (!ctx || !value) return YMRT_ERR_INVALID;
  switch (option) {
    case YMRT_OPT_SORT_HITS: *value = ctx->sort_hits ? 1 : 0; return YMRT_OK;
    case YMRT_OPT_DEFER_SHADOWS: *value = ctx->defer_shadows ? 1 : 0; return YMRT_OK;
    case YMRT_OPT_GRAPH_LOOP: *value = ctx->graph_loop ? 1 : 0; return YMRT_OK;
    case YMRT_OPT_TRACE_BLOCK: *value = (int)ctx->trace_block; return YMRT_OK;
    case YMRT_OPT_SORT_RAYS: *value = ctx->sort_rays ? 1 : 0; return YMRT_OK;
    default: return YMRT_ERR_INVALID;
  }
}

int ymrt_scene_load_ymtmp(const char* path, int width, int height, ymrt_host_scene** out, char* err, size_t err_len) {
  return ymrt_scene_load_ymtmp_ex(path, width, height, nullptr, out, err, err_len);
}

int ymrt_scene_load_ymtmp_ex(const char* path, int width, int height, const ymrt_load_options* options,
                             ymrt_host_scene** out, char* err, size_t err_len) {
  auto report = [&](int code, const std::string& msg) {
    g_last_error = msg;
    if (err && err_len) {
      std::strncpy(err, msg.c_str(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return code;
  };
  if (!path || !out) return report(YMRT_ERR_INVALID, "null argument");
  *out = nullptr;
  std::unique_ptr<ymrt_host_scene> hs(new (std::nothrow) ymrt_host_scene());
  if (!hs) return report(YMRT_ERR_OOM, "out of host memory");
  std::string msg;
  int rc;
  if (options) {
    if (options->max_leaf_triangles < 1 || options->max_leaf_triangles > 4)
      return report(YMRT_ERR_INVALID, "max_leaf_triangles must be 1..4");
    hs->s.max_leaf_prims = options->max_leaf_triangles;
  }
  try {
    rc = load_ymtmp(path, &hs->s, &msg);
    if (rc == YMRT_OK && options && options->override_camera) {
      hs->s.cam_from = vec3(options->camera_from[0], options->camera_from[1], options->camera_from[2]);
      hs->s.cam_look = vec3(options->camera_look[0], options->camera_look[1], options->camera_look[2]);
      hs->s.cam_fov_deg = gmax(options->camera_fov_deg, 0.01f);
    }
    if (rc == YMRT_OK) rc = prepare_scene(&hs->s, width, height, &msg);
  } catch (const std::exception& ex) {
    rc = YMRT_ERR_FORMAT;
    msg = std::string("malformed value in ") + path + ": " + ex.what();
  }
  if (rc != YMRT_OK) return report(rc, msg);
  *out = hs.release();
  return YMRT_OK;
}

int ymrt_scene_from_arrays(const ymrt_scene_desc* desc, int width, int height, const ymrt_load_options* options,
                           ymrt_host_scene** out, char* err, size_t err_len) {
  auto report = [&](int code, const std::string& msg) {
    g_last_error = msg;
    if (err && err_len) {
      std::strncpy(err, msg.c_str(), err_len - 1);
      err[err_len - 1] = 0;
    }
    return code;
  };
  if (!desc || !out) return report(YMRT_ERR_INVALID, "null argument");
  *out = nullptr;
  std::unique_ptr<ymrt_host_scene> hs(new (std::nothrow) ymrt_host_scene());
  if (!hs) return report(YMRT_ERR_OOM, "out of host memory");
  if (options) {
    if (options->max_leaf_triangles < 1 || options->max_leaf_triangles > 4)
      return report(YMRT_ERR_INVALID, "max_leaf_triangles must be 1..4");
    hs->s.max_leaf_prims = options->max_leaf_triangles;
  }
  std::string msg;
  int rc = load_arrays(desc, &hs->s, &msg);
  if (rc == YMRT_OK && options && options->override_camera) {
    hs->s.cam_from = vec3(options->camera_from[0], options->camera_from[1], options->camera_from[2]);
    hs->s.cam_look = vec3(options->camera_look[0], options->camera_look[1], options->camera_look[2]);
    hs->s.cam_fov_deg = gmax(options->camera_fov_deg, 0.01f);
  }
  if (rc == YMRT_OK) rc = prepare_scene(&hs->s, width, height, &msg);
  if (rc != YMRT_OK) return report(rc, msg);
  *out = hs.release();
  return YMRT_OK;
}

void ymrt_host_scene_free(ymrt_host_scene* scene) { delete scene; }

long long ymrt_host_scene_query(const ymrt_host_scene* hs, int what, int index, void* out, size_t cap) {
  if (!hs) return YMRT_ERR_INVALID;
  const HostScene& s = hs->s;
  auto copy = [&](const void* src, size_t count, size_t elem) -> long long {
    if (out && cap < count) return YMRT_ERR_INVALID;
    if (out && count) std::memcpy(out, src, count * elem);
    return (long long)count;
  };
  switch (what) {
    case YMRT_QUERY_COUNTS: {
      uint64_t c[8] = {s.instances.size(), s.meshes.size(), s.tri_corners.size() / 3, s.triangle_count_instanced,
                       s.shape_lights.size(), s.blas_nodes.size(), s.tlas_nodes.size(), s.materials.size()};
      return copy(c, 8, sizeof(uint64_t));
    }
    case YMRT_QUERY_INSTANCES: {
      std::vector<uint32_t> v;
      for (size_t i = 0; i < s.instances.size(); ++i) {
        const Instance& in = s.instances[i];
        v.insert(v.end(), {in.geometry_idx, in.transform_idx, in.material_idx, (uint32_t)in.inner_volume_idx,
                           (uint32_t)in.treat_as_boundary, s.instance_file_index[i]});
      }
      return copy(v.data(), v.size(), sizeof(uint32_t));
    }
    case YMRT_QUERY_LIGHTS: {
      std::vector<float> v;
      for (const ShapeLight& l : s.shape_lights) v.insert(v.end(), {u2f(l.instance_idx), u2f(l.triangle_idx), l.power, l.area});
      return copy(v.data(), v.size(), sizeof(float));
    }
    case YMRT_QUERY_LIGHT_TABLE:
      return copy(s.shape_light_table.data(), s.shape_light_table.size(), sizeof(float));
    case YMRT_QUERY_TRANSFORMS: {
      std::vector<float> v;
      for (size_t i = 0; i < s.transforms.size(); ++i) {
        const float* a = &s.transforms[i].m[0][0];
        const float* b = &s.i_transforms[i].m[0][0];
        v.insert(v.end(), a, a + 16);
        v.insert(v.end(), b, b + 16);
      }
      return copy(v.data(), v.size(), sizeof(float));
    }
    case YMRT_QUERY_CAMERA: {
      const CameraDesc& c = s.camera;
      const float v[14] = {c.position.x, c.position.y, c.position.z, c.u.x, c.u.y, c.u.z, c.v.x,
                           c.v.y,        c.v.z,        c.w.x,        c.w.y, c.w.z, c.aspect_ratio, c.tan_half_fov};
      return copy(v, 14, sizeof(float));
    }
    case YMRT_QUERY_MATERIALS:
      return copy(s.materials.data(), s.materials.size() * (sizeof(Material) / 4), 4);
    case YMRT_QUERY_VOLUMES:
      return copy(s.volumes.data(), s.volumes.size() * (sizeof(Volume) / 4), 4);
    case YMRT_QUERY_DISTANT_LIGHTS:
      return copy(s.distant_lights.data(), s.distant_lights.size() * (sizeof(DistantLight) / 4), 4);
    case YMRT_QUERY_TEXTURES: {
      std::vector<uint32_t> v;
      for (const Texture& t : s.textures) {
        uint32_t r[kTextureWords];
        texture_words(t, r);
        v.insert(v.end(), r, r + kTextureWords);
      }
      return copy(v.data(), v.size(), sizeof(uint32_t));
    }
    case YMRT_QUERY_TRIANGLES: {
      if (index < 0 || (size_t)index >= s.meshes.size()) return YMRT_ERR_INVALID;
      const std::vector<uint32_t>& t = s.meshes[index].tris;
      return copy(t.data(), t.size(), sizeof(uint32_t));
    }
    case YMRT_QUERY_GEOMETRIES: {
      std::vector<uint32_t> v;
      for (const HostMesh& m : s.meshes) v.insert(v.end(), {m.kind, f2u(m.radius)});
      return copy(v.data(), v.size(), sizeof(uint32_t));
    }
    case YMRT_QUERY_IMAGE_PIXELS: {
      if (index < 0) return YMRT_ERR_INVALID;
      auto it = s.images.find((uint32_t)index);
      if (it == s.images.end()) return YMRT_ERR_INVALID;
      return copy(it->second.data(), it->second.size(), sizeof(float));
    }
    case YMRT_QUERY_MESH_CORNERS: {
      if (index < 0 || (size_t)index >= s.meshes.size()) return YMRT_ERR_INVALID;
      const HostMesh& m = s.meshes[index];
      std::vector<float> v;
      for (size_t c = 0; c < m.pos_idx.size(); ++c) {
        const uint32_t pi = m.pos_idx[c], ni = m.nrm_idx[c];
        v.insert(v.end(), {m.pos[3 * pi], m.pos[3 * pi + 1], m.pos[3 * pi + 2], m.nrm[3 * ni], m.nrm[3 * ni + 1],
                           m.nrm[3 * ni + 2]});
        if (m.uv_idx.empty()) {
          v.insert(v.end(), {0.0f, 0.0f});
        } else {
          const uint32_t ti = m.uv_idx[c];
          v.insert(v.end(), {m.uv[2 * ti], m.uv[2 * ti + 1]});
        }
      }
      return copy(v.data(), v.size(), sizeof(float));
    }
    default:
      return YMRT_ERR_INVALID;
  }
}

int ymrt_scene_upload(ymrt_context* ctx, const ymrt_host_scene* hs, const uint32_t* halton_perm, size_t perm_len,
                      ymrt_scene** out) {
  if (!ctx || !hs || !out || !halton_perm) return YMRT_ERR_INVALID;
  *out = nullptr;
  size_t need = 0;
  for (uint32_t p : ctx->primes) need += p;
  if (perm_len != need)
    return ctx->fail(YMRT_ERR_INVALID, "halton permutation table must hold " + std::to_string(need) + " entries");
  const HostScene& s = hs->s;
  cudaSetDevice(ctx->device);
  std::unique_ptr<ymrt_scene> sc(new (std::nothrow) ymrt_scene());
  if (!sc) return YMRT_ERR_OOM;
  sc->ctx = ctx;
  sc->width = s.width;
  sc->height = s.height;
  sc->triangles = s.triangle_count_instanced;
  DeviceScene& D = sc->dev;
  cudaError_t e = cudaSuccess;
  // image pixels first (the texture nodes point at them), then every other
  // array in one packed upload
  std::vector<Texture> tex = s.textures;
  for (size_t k = 0; k < tex.size(); ++k) {
    if (tex[k].type != kTexImage) continue;
    auto it = s.images.find((uint32_t)k);
    const size_t n = (size_t)tex[k].width * tex[k].height * tex[k].channels;
    if (it == s.images.end() || it->second.size() != n)
      return ctx->fail(YMRT_ERR_INVALID, "image node " + std::to_string(k) + " has no pixels (ymrt_host_scene_set_image)");
    sc->pack(it->second, &tex[k].image);
  }
  e = sc->pack_commit();
#define UP(vec, field) sc->pack(vec, &D.field)
  UP(s.instances, instances);
  UP(s.transforms, transforms);
  UP(s.i_transforms, i_transforms);
  UP(s.tlas_nodes, tlas_nodes);
  UP(s.tlas_prims, tlas_prims);
  UP(s.geo_desc, geometries);
  UP(s.blas_nodes, blas_nodes);
  UP(s.wtris, wtris);
  UP(s.tri_corners, tri_corners);
  UP(s.all_pos_idx, pos_idx);
  UP(s.all_nrm_idx, nrm_idx);
  UP(s.all_uv_idx, uv_idx);
  UP(s.all_pos, positions);
  UP(s.all_nrm, normals);
  UP(s.all_uv, texcoords);
  UP(s.materials, materials);
  sc->materials = s.materials;
  UP(s.distant_lights, distant_lights);
  UP(s.shape_lights, shape_lights);
  UP(s.shape_light_table, shape_light_table);
  UP(s.volumes, volumes);
  UP(tex, textures);
  sc->textures = tex;
  std::vector<uint8_t> buckets(s.instances.size());
  for (size_t i = 0; i < s.instances.size(); ++i) buckets[i] = (uint8_t)shading_bucket(s, s.instances[i]);
  UP(buckets, inst_bucket);
#undef UP
  sc->pack(halton_perm, perm_len, &D.halton_perm);
  if (e == cudaSuccess) e = sc->pack_commit();
  else sc->packed.clear();
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "uploading scene");
  D.sampler_type = kSamplerHalton;
  D.instance_count = (uint32_t)s.instances.size();
  D.transform_count = (uint32_t)s.transforms.size();
  D.geometry_count = (uint32_t)s.geo_desc.size();
  D.sphere_count = 0;
  for (const GeometryDesc& g : s.geo_desc) D.sphere_count += g.kind == kGeoSphere ? 1u : 0u;
  D.material_count = (uint32_t)s.materials.size();
  D.distant_light_count = (uint32_t)s.distant_lights.size();
  D.shape_light_count = (uint32_t)s.shape_lights.size();
  D.volume_count = (uint32_t)s.volumes.size();
  D.texture_count = (uint32_t)s.textures.size();
  D.textured = uses_textures(s.materials, s.textures) ? 1u : 0u;
  D.camera = s.camera;
  D.width = s.width;
  D.height = s.height;
  // HaltonEnumerator constructor (src/HaltonEnumerator.h:13-38).
  {
    int scale2 = 1, exp2 = 0, scale3 = 1, exp3 = 0;
    while (scale2 < s.width) {
      scale2 *= 2;
      ++exp2;
    }
    while (scale3 < s.height) {
      scale3 *= 3;
      ++exp3;
    }
    struct MI {
      int x, y;
    };
    std::function<MI(int, int)> ee = [&](int a, int b) -> MI {
      if (b == 0) return MI{1, 0};
      const MI lo = ee(b, a % b);
      return MI{lo.y, lo.x - (a / b) * lo.y};
    };
    const int w = scale2, h = scale3;
    const MI mi = ee(h, w);
    const int inv2 = mi.x < 0 ? (mi.x + w) : (mi.x % w);
    const int inv3 = mi.y < 0 ? (mi.y + h) : (mi.y % h);
    D.halton_mx = h * inv2;
    D.halton_my = w * inv3;
    D.halton_increment = w * h;
    D.halton_x_scale = float(scale2);
    D.halton_y_scale = float(scale3);
    D.halton_exp2 = exp2;
    D.halton_exp3 = exp3;
  }
  sc->top.max_leaf = s.max_leaf_prims;
  sc->top.node_count = (uint32_t)s.tlas_nodes.size();
  sc->top.file_index = s.instance_file_index;
  sc->top.transform_scales = s.transform_scales;
  *out = sc.release();
  return YMRT_OK;
}

int ymrt_scene_set_sobol_matrices(ymrt_scene* scene, const uint32_t* matrices, size_t count) {
  if (!scene || !matrices) return YMRT_ERR_INVALID;
  if (count != (size_t)4096 * 32)
    return scene->ctx->fail(YMRT_ERR_INVALID, "Sobol generator matrices: expected 4096 x 32 words");
  cudaSetDevice(scene->ctx->device);
  std::vector<uint32_t> m(matrices, matrices + count);
  cudaError_t e = scene->upload(m, &scene->dev.sobol_matrices);
  if (e == cudaSuccess) e = cudaStreamSynchronize(scene->ctx->stream);
  if (e != cudaSuccess) return scene->ctx->cuda_fail(e, "uploading Sobol matrices");
  return YMRT_OK;
}

void ymrt_scene_free(ymrt_scene* scene) {
  if (!scene) return;
  cudaSetDevice(scene->ctx->device);
  cudaStreamSynchronize(scene->ctx->stream);
  // the packed upload's buffers go back to the context for the next upload
  for (std::unique_ptr<DeviceBuffer>& b : scene->buffers)
    if (b && b->ptr &&
        std::find(scene->packed_buffers.begin(), scene->packed_buffers.end(), b.get()) != scene->packed_buffers.end())
      scene->ctx->keep_spare(std::move(b));
  delete scene;
}

}  // extern "C"

namespace {

// Device memory one batch renders with: the context's queues, or the fixed
// array of the allocation-free entry point.
struct BatchMemory {
  PathPool pool[2];
  HitPool hits;
  WaveCounters* counters = nullptr;
  WaveControl* ctl = nullptr;
  JobDesc* jobs = nullptr;  // device job table
  uint32_t capacity = 0;
};

struct BatchResult {
  uint64_t paths = 0, waves = 0, launches = 0, hits = 0;
  double ms = 0.0;
  double stage_ms[5] = {0.0, 0.0, 0.0, 0.0, 0.0};  // generate, extend, sort, shade, connect
};

// Checks one render's arguments and fills its job (path range left at 0).
int make_job(ymrt_context* ctx, ymrt_scene* sc, const ymrt_render_setting* setting, int frame_index, int tile_begin,
             int tile_end, float4* image, JobDesc* job, DeviceScene* scene, float* record = nullptr,
             const float* dloss = nullptr) {
  static_assert(sizeof(ymrt_render_setting) == sizeof(RenderSetting), "render setting layout");
  if (!sc || !setting || !image) return ctx->fail(YMRT_ERR_INVALID, "null scene, setting or output");
  if (sc->ctx != ctx) return ctx->fail(YMRT_ERR_INVALID, "scene belongs to another context");
  RenderSetting rs;
  std::memcpy(&rs, setting, sizeof(rs));
  if (frame_index < 1) return ctx->fail(YMRT_ERR_INVALID, "frame_index starts at 1");
  if (rs.sampler_type > 2u)
    return ctx->fail(YMRT_ERR_UNSUPPORTED, "sampler_type must be 0 (PCG), 1 (Halton) or 2 (Sobol)");
  if (rs.sampler_type == 2u && !sc->dev.sobol_matrices)
    return ctx->fail(YMRT_ERR_INVALID, "the Sobol sampler needs its generator matrices (ymrt_scene_set_sobol_matrices)");
  if (tile_begin < 0) return ctx->fail(YMRT_ERR_INVALID, "tile_begin < 0");
  const uint32_t tiles_x = (sc->width + kTileRes - 1) / kTileRes, tiles_y = (sc->height + kTileRes - 1) / kTileRes;
  const uint32_t total_tiles = tiles_x * tiles_y;
  const uint32_t t_end = tile_end <= 0 ? total_tiles : std::min<uint32_t>((uint32_t)tile_end, total_tiles);
  const uint32_t t_begin = std::min<uint32_t>((uint32_t)tile_begin, t_end);
  std::memset(job, 0, sizeof(*job));
  *scene = sc->dev;
  scene->sampler_type = rs.sampler_type;
  job->width = (uint32_t)sc->width;
  job->height = (uint32_t)sc->height;
  if (rs.enable_volume_scattering && sc->dev.volume_count == 0) rs.enable_volume_scattering = false;
  job->setting = rs;
  job->image = image;
  job->frame_index = frame_index;
  job->spp = (uint32_t)std::max(rs.ssp, 1);
  job->tiles_x = tiles_x;
  job->tile_begin = t_begin;
  job->path_count = (unsigned long long)(t_end - t_begin) * kTilePixels * job->spp;
  if (job->path_count > 0xFFFFFFFFull) return ctx->fail(YMRT_ERR_INVALID, "a render of more than 2^32 paths");
  job->path_radiance = reinterpret_cast<float4*>(record);
  job->dloss = reinterpret_cast<const float4*>(dloss);
  return YMRT_OK;
}

// Gives every job the constant-memory slot of its (scene, sampler) pair;
// returns the slots' scenes.
std::vector<DeviceScene> assign_slots(std::vector<JobDesc>& jobs, const std::vector<DeviceScene>& job_scenes,
                                      const std::vector<const void*>& keys) {
  std::vector<DeviceScene> slots;
  std::vector<std::pair<const void*, uint32_t>> seen;
  for (size_t k = 0; k < jobs.size(); ++k) {
    const auto key = std::make_pair(keys[k], job_scenes[k].sampler_type);
    uint32_t slot = (uint32_t)seen.size();
    for (uint32_t q = 0; q < seen.size(); ++q)
      if (seen[q] == key) slot = q;
    if (slot == seen.size()) {
      seen.push_back(key);
      slots.push_back(job_scenes[k]);
    }
    jobs[k].scene_slot = slot;
  }
  return slots;
}

// Renders a batch of jobs (paths numbered job after job). The wave loop is
// planned on the device (k_plan / k_finish); the host either launches the
// whole loop as one CUDA graph (a while-loop node around two waves, captured
// once and reused while memory and options stay the same), or, with
// per-kernel profiling or graph_loop off, launches wave after wave and reads
// the loop condition after each. The job images must be zeroed by the caller.
int run_batch(ymrt_context* ctx, const BatchMemory& M, std::vector<JobDesc>& jobs, const WaveOptions& opt,
              bool profiling, bool use_graph, BatchResult* r) {
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  unsigned long long total = 0;
  for (JobDesc& j : jobs) {
    j.path_begin = total;
    total += j.path_count;
  }
  if ((e = cudaMemcpyAsync(M.jobs, jobs.data(), sizeof(JobDesc) * jobs.size(), cudaMemcpyHostToDevice, st)) !=
      cudaSuccess)
    return ctx->cuda_fail(e, "uploading the job table");
  WaveControl& c = *ctx->ctl_host;
  std::memset(&c, 0, sizeof(c));
  c.total = total;
  c.capacity = M.capacity;
  c.more = 1;
  // a path lives at most kMaxRayDepth scattering vertices plus its boundary
  // crossings: a generous bound on waves, reached only by a fault
  const unsigned long long bound = total / std::max<uint32_t>(M.capacity, 1u) * 80ull + 4096ull;
  c.max_waves = (uint32_t)std::min<unsigned long long>(bound, 1ull << 30);
  if ((e = cudaMemcpyAsync(M.ctl, &c, sizeof(c), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    return ctx->cuda_fail(e, "uploading the wave control");
  WaveOptions o = opt;
  o.capacity = M.capacity;
  if ((e = cudaMemsetAsync(M.counters, 0, sizeof(WaveCounters), st)) != cudaSuccess)
    return ctx->cuda_fail(e, "clearing the wave counters");
  if (M.hits.ray_bins && (e = cudaMemsetAsync(M.hits.ray_bins, 0, kRayBins * sizeof(uint32_t), st)) != cudaSuccess)
    return ctx->cuda_fail(e, "clearing the ray-grouping counts");
  prepare_persistent_grids();
  cudaEventRecord(ctx->ev_start, st);
  if (use_graph && !profiling) {
    const std::vector<uintptr_t> key = {
        (uintptr_t)M.pool[0].ray_o, (uintptr_t)M.pool[1].ray_o, (uintptr_t)M.hits.bary_t, (uintptr_t)M.ctl,
        (uintptr_t)M.jobs, (uintptr_t)M.counters, (uintptr_t)jobs.size(), (uintptr_t)o.volumes,
        (uintptr_t)o.sort_hits, (uintptr_t)o.defer_shadows, (uintptr_t)o.shadow_queue.o, M.capacity,
        (uintptr_t)o.trace_block, (uintptr_t)o.sort_rays,
        (uintptr_t)o.features, (uintptr_t)o.grid_grads, (uintptr_t)o.grid_tex,
        (uintptr_t)o.adjoint, (uintptr_t)o.grads, o.grad_materials};
    if (ctx->graph_key != key) {
      ctx->drop_graph();
      cudaGraph_t g = nullptr;
      if ((e = cudaGraphCreate(&g, 0)) != cudaSuccess) return ctx->cuda_fail(e, "cudaGraphCreate");
      cudaGraphConditionalHandle cond;
      e = cudaGraphConditionalHandleCreate(&cond, g, 1, cudaGraphCondAssignDefault);
      cudaGraphNodeParams params{};
      params.type = cudaGraphNodeTypeConditional;
      params.conditional.handle = cond;
      params.conditional.type = cudaGraphCondTypeWhile;
      params.conditional.size = 1;
      cudaGraphNode_t node;
      if (e == cudaSuccess) e = cudaGraphAddNode(&node, g, nullptr, 0, &params);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return ctx->cuda_fail(e, "building the wave-loop graph");
      }
      cudaGraph_t body = params.conditional.phGraph_out[0];
      e = cudaStreamBeginCaptureToGraph(st, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed);
      if (e == cudaSuccess) {
        launch_wave(M.pool[0], M.pool[1], M.hits, M.ctl, M.jobs, (uint32_t)jobs.size(), M.counters, o, nullptr, st,
                    (unsigned long long)cond);
        launch_wave(M.pool[1], M.pool[0], M.hits, M.ctl, M.jobs, (uint32_t)jobs.size(), M.counters, o, nullptr, st,
                    (unsigned long long)cond);
        e = cudaStreamEndCapture(st, &body);
      }
      cudaGraphExec_t exec = nullptr;
      if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, g, 0);
      if (e != cudaSuccess) {
        cudaGraphDestroy(g);
        return ctx->cuda_fail(e, "capturing the wave-loop graph");
      }
      ctx->graph = g;
      ctx->graph_exec = exec;
      ctx->graph_key = key;
    }
    if ((e = cudaGraphLaunch(ctx->graph_exec, st)) != cudaSuccess) return ctx->cuda_fail(e, "launching the wave loop");
    if ((e = cudaMemcpyAsync(&c, M.ctl, sizeof(c), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return ctx->cuda_fail(e, "reading the wave control");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "wave loop");
    r->launches += 1;
  } else {
    int a = 0;
    for (;;) {
      r->launches += launch_wave(M.pool[a], M.pool[a ^ 1], M.hits, M.ctl, M.jobs, (uint32_t)jobs.size(), M.counters,
                                 o, profiling ? ctx->ev_stage : nullptr, st);
      if ((e = cudaMemcpyAsync(&c, M.ctl, sizeof(c), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
        return ctx->cuda_fail(e, "reading the wave control");
      if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "wave");
      if (profiling) {
        for (int k = 0; k < 5; ++k) {
          float ms = 0.0f;
          cudaEventElapsedTime(&ms, ctx->ev_stage[k], ctx->ev_stage[k + 1]);
          r->stage_ms[k] += ms;
        }
      }
      if (!c.more) break;
      a ^= 1;
    }
  }
  cudaEventRecord(ctx->ev_stop, st);
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "frame");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
  r->ms = ms;
  r->paths = c.cursor;
  r->waves = c.waves;
  r->hits = c.hits;
  return YMRT_OK;
}

// Adds the last group's frame counters (in counters_host) to batch_counters.
void total_counters_add(ymrt_context* ctx, bool first) {
  WaveCounters& t = ctx->batch_counters;
  const WaveCounters& c = *ctx->counters_host;
  if (first) t = WaveCounters{};
  t.errors |= c.errors;
  t.tracking_caps += c.tracking_caps;
  t.extension_rays += c.extension_rays;
  t.shadow_rays += c.shadow_rays;
  t.tri_tests += c.tri_tests;
  t.node_visits += c.node_visits;
  t.shadow_tri_tests += c.shadow_tri_tests;
  t.shadow_node_visits += c.shadow_node_visits;
}

// Fills ymrt_stats from the frame's counters and turns device error flags
// into a status.
int finish_batch(ymrt_context* ctx, const BatchResult& r, ymrt_stats* stats) {
  const WaveCounters& c = *ctx->counters_host;
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->paths = r.paths;
    stats->extension_rays = c.extension_rays;
    stats->shadow_rays = c.shadow_rays;
    stats->waves = r.waves;
    stats->shaded_hits = r.hits;
    stats->node_visits = c.node_visits + c.shadow_node_visits;
    stats->triangle_tests = c.tri_tests + c.shadow_tri_tests;
    stats->shadow_node_visits = c.shadow_node_visits;
    stats->shadow_triangle_tests = c.shadow_tri_tests;
    stats->kernel_launches = r.launches;
    stats->ms_total = r.ms;
    stats->ms_generate = r.stage_ms[0];
    stats->ms_extend = r.stage_ms[1];
    stats->ms_sort = r.stage_ms[2];
    stats->ms_shade = r.stage_ms[3];
    stats->ms_connect = r.stage_ms[4];
    stats->device_errors = c.errors;
    stats->tracking_bound_hits = c.tracking_caps;
  }
  if (c.errors & kDevErrQueue) return ctx->fail(YMRT_ERR_OVERFLOW, "path queue overflow on the device");
  if (c.errors & kDevErrStack) return ctx->fail(YMRT_ERR_OVERFLOW, "traversal or nested-media stack overflow on the device");
  if (c.errors & kDevErrIter)
    return ctx->fail(YMRT_ERR_OVERFLOW, "a bounded device loop reached its limit (shadow-ray boundary crossings or "
                                        "waves of a frame; ymrt_debug_bound_record tells which)");
  return YMRT_OK;
}

// The features (kFeatSpheres, kFeatGrids, kFeatTextures) any of the batch's
// scenes uses.
uint32_t batch_features(const DeviceScene* scenes, size_t n) {
  uint32_t f = 0;
  for (size_t i = 0; i < n; ++i) {
    if (scenes[i].sphere_count != 0) f |= kFeatSpheres;
    if (scenes[i].grid_count != 0) f |= kFeatGrids;
    if (scenes[i].textured != 0) f |= kFeatTextures;
  }
  return f;
}

// Wave options for a batch: media kernels when any job scatters in media;
// shadow rays deferred unless a job clamps indirect light.
int batch_options(ymrt_context* ctx, const std::vector<JobDesc>& jobs, WaveOptions* opt) {
  opt->volumes = false;
  bool clamp = false;
  for (const JobDesc& j : jobs) {
    opt->volumes = opt->volumes || j.setting.enable_volume_scattering;
    clamp = clamp || j.setting.enable_indirect_clamp;
  }
  opt->sort_hits = ctx->sort_hits;
  opt->trace_block = ctx->trace_block;
  opt->sort_rays = ctx->sort_rays;
  opt->defer_shadows = ctx->defer_shadows && !opt->volumes && !clamp;
  if (opt->defer_shadows) {
    int rc = ctx->ensure_shadow_queue();
    if (rc != YMRT_OK) return rc;
    opt->shadow_queue = ctx->shadow_queue;
  }
  return YMRT_OK;
}

// The context's queues as batch memory, with room for n_jobs jobs.
int context_memory(ymrt_context* ctx, size_t n_jobs, BatchMemory* M) {
  int rc = ctx->ensure_pools();
  if (rc != YMRT_OK) return rc;
  cudaError_t e = ctx->counters_buf.ensure(sizeof(WaveCounters));
  if (e == cudaSuccess) e = ctx->ctl_buf.ensure(sizeof(WaveControl));
  if (e == cudaSuccess) e = ctx->jobs_buf.ensure(sizeof(JobDesc) * std::max<size_t>(n_jobs, 1));
  if (e != cudaSuccess) return ctx->cuda_fail(e, "allocating the job table");
  M->pool[0] = ctx->pool[0];
  M->pool[1] = ctx->pool[1];
  M->hits = ctx->hits;
  M->counters = ctx->counters_buf.as<WaveCounters>();
  M->ctl = ctx->ctl_buf.as<WaveControl>();
  M->jobs = ctx->jobs_buf.as<JobDesc>();
  M->capacity = ctx->capacity;
  return YMRT_OK;
}

}  // namespace

extern "C" {

int ymrt_render_tiles(ymrt_scene* sc, const ymrt_render_setting* setting, int frame_index, int tile_begin, int tile_end,
                      float* out_rgba, int out_on_device, ymrt_stats* stats) {
  if (!sc || !setting || !out_rgba) return YMRT_ERR_INVALID;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  float4* image = reinterpret_cast<float4*>(out_rgba);
  const size_t img_bytes = (size_t)sc->width * sc->height * sizeof(float4);
  if (!out_on_device) {
    if ((e = ctx->image_buf.ensure(img_bytes)) != cudaSuccess) return ctx->cuda_fail(e, "allocating image");
    image = ctx->image_buf.as<float4>();
  }
  std::vector<JobDesc> jobs(1);
  DeviceScene scene;
  int rc = make_job(ctx, sc, setting, frame_index, tile_begin, tile_end, image, &jobs[0], &scene);
  if (rc != YMRT_OK) return rc;
  BatchMemory M;
  if ((rc = context_memory(ctx, 1, &M)) != YMRT_OK) return rc;
  WaveOptions opt;
  if ((rc = batch_options(ctx, jobs, &opt)) != YMRT_OK) return rc;
  opt.features = batch_features(&scene, 1);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  jobs[0].scene_slot = lease.slot(0);
  if ((e = lease.upload(&scene, 1)) != cudaSuccess) return ctx->cuda_fail(e, "uploading constants");
  if ((e = cudaMemsetAsync(image, 0, img_bytes, st)) != cudaSuccess) return ctx->cuda_fail(e, "clearing the image");
  BatchResult r;
  if ((rc = run_batch(ctx, M, jobs, opt, ctx->profiling, ctx->graph_loop, &r)) != YMRT_OK) return rc;
  if (!out_on_device) {
    if ((e = cudaMemcpyAsync(out_rgba, image, img_bytes, cudaMemcpyDeviceToHost, st)) != cudaSuccess)
      return ctx->cuda_fail(e, "copying image");
  }
  if ((e = cudaMemcpyAsync(ctx->counters_host, M.counters, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return ctx->cuda_fail(e, "reading counters");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "frame");
  return finish_batch(ctx, r, stats);
}

int ymrt_render_batch(ymrt_context* ctx, const ymrt_job* jobs_in, int n_jobs, ymrt_stats* stats) {
  if (!ctx || !jobs_in || n_jobs <= 0) return YMRT_ERR_INVALID;
  if (n_jobs > (1 << 21)) return ctx->fail(YMRT_ERR_INVALID, "too many jobs in one batch (at most 2^21)");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  std::vector<JobDesc> all((size_t)n_jobs);
  std::vector<DeviceScene> scenes((size_t)n_jobs);
  std::vector<const void*> keys((size_t)n_jobs);
  for (int k = 0; k < n_jobs; ++k) {
    const ymrt_job& in = jobs_in[k];
    int rc = make_job(ctx, in.scene, &in.setting, in.frame_index, in.tile_begin, in.tile_end,
                      reinterpret_cast<float4*>(in.out_rgba_device), &all[k], &scenes[k], in.path_radiance_device);
    if (rc != YMRT_OK) return rc;
    keys[k] = in.scene;
  }
  BatchMemory M;
  int rc = context_memory(ctx, all.size(), &M);
  if (rc != YMRT_OK) return rc;
  for (const JobDesc& j : all) {
    e = cudaMemsetAsync(j.image, 0, (size_t)j.width * j.height * sizeof(float4), st);
    if (e == cudaSuccess && j.path_radiance)
      e = cudaMemsetAsync(j.path_radiance, 0, (size_t)j.path_count * sizeof(float4), st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "clearing an image or its path records");
  }
  // Launch groups of jobs whose (scene, sampler) pairs fit the constant-memory slots.
  BatchResult total;
  size_t k0 = 0;
  while (k0 < all.size()) {
    size_t k1 = k0;
    std::vector<std::pair<const void*, uint32_t>> seen;
    while (k1 < all.size()) {
      const auto key = std::make_pair(keys[k1], scenes[k1].sampler_type);
      bool found = false;
      for (const auto& q : seen) found = found || q == key;
      if (!found) {
        if (seen.size() == kMaxSceneSlots) break;
        seen.push_back(key);
      }
      ++k1;
    }
    std::vector<JobDesc> jobs(all.begin() + k0, all.begin() + k1);
    std::vector<DeviceScene> js(scenes.begin() + k0, scenes.begin() + k1);
    std::vector<const void*> ks(keys.begin() + k0, keys.begin() + k1);
    const std::vector<DeviceScene> slots = assign_slots(jobs, js, ks);
    WaveOptions opt;
    if ((rc = batch_options(ctx, jobs, &opt)) != YMRT_OK) return rc;
    opt.features = batch_features(slots.data(), slots.size());
    SlotLease lease(ctx, (uint32_t)slots.size());
    if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slots for this device");
    for (JobDesc& j : jobs) j.scene_slot = lease.slot(j.scene_slot);
    if ((e = lease.upload(slots.data(), (uint32_t)slots.size())) != cudaSuccess)
      return ctx->cuda_fail(e, "uploading constants");
    BatchResult r;
    if ((rc = run_batch(ctx, M, jobs, opt, ctx->profiling, ctx->graph_loop, &r)) != YMRT_OK) return rc;
    total.paths += r.paths;
    total.waves += r.waves;
    total.launches += r.launches;
    total.hits += r.hits;
    total.ms += r.ms;
    for (int q = 0; q < 5; ++q) total.stage_ms[q] += r.stage_ms[q];
    // counters are cleared per group: keep this group's totals
    if ((e = cudaMemcpyAsync(ctx->counters_host, M.counters, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st)) !=
        cudaSuccess)
      return ctx->cuda_fail(e, "reading counters");
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "batch");
    total_counters_add(ctx, k0 == 0);
    k0 = k1;
  }
  *ctx->counters_host = ctx->batch_counters;
  return finish_batch(ctx, total, stats);
}

unsigned long long ymrt_job_path_count(const ymrt_job* job) {
  if (!job || !job->scene) return 0;
  const ymrt_scene* sc = job->scene;
  const uint32_t tiles_x = (sc->width + kTileRes - 1) / kTileRes, tiles_y = (sc->height + kTileRes - 1) / kTileRes;
  const uint32_t total = tiles_x * tiles_y;
  const uint32_t t_end = job->tile_end <= 0 ? total : std::min<uint32_t>((uint32_t)job->tile_end, total);
  const uint32_t t_begin = std::min<uint32_t>((uint32_t)std::max(job->tile_begin, 0), t_end);
  return (unsigned long long)(t_end - t_begin) * kTilePixels * (uint32_t)std::max(job->setting.ssp, 1);
}

int ymrt_render_backward_ex(ymrt_context* ctx, const ymrt_job* jobs_in, int n_jobs, const ymrt_backward_targets* tg,
                            ymrt_stats* stats) {
  if (!ctx || !jobs_in || n_jobs <= 0 || !tg) return YMRT_ERR_INVALID;
  const bool materials = tg->material_grads_device && tg->n_materials > 0;
  const bool grid = tg->grid_grads_device != nullptr;
  if (!materials && !grid) return ctx->fail(YMRT_ERR_INVALID, "backward: no gradient requested");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  std::vector<JobDesc> jobs((size_t)n_jobs);
  std::vector<DeviceScene> scenes((size_t)n_jobs);
  std::vector<const void*> keys((size_t)n_jobs);
  bool volumes = false;
  for (int k = 0; k < n_jobs; ++k) {
    const ymrt_job& in = jobs_in[k];
    if (!in.path_radiance_device || !in.dloss_device)
      return ctx->fail(YMRT_ERR_INVALID, "backward: every job needs its recorded path radiance and dLoss/dImage");
    if (in.setting.enable_indirect_clamp)
      return ctx->fail(YMRT_ERR_UNSUPPORTED, "backward: the indirect clamp is not differentiated");
    if (grid) {
      if (!in.scene || tg->grid_texture >= in.scene->textures.size())
        return ctx->fail(YMRT_ERR_INVALID, "backward: grid texture index out of range");
      const Texture& t = in.scene->textures[tg->grid_texture];
      if (t.type != kTexGrid ||
          (uint64_t)t.grid_n[0] * (uint64_t)t.grid_n[1] * (uint64_t)t.grid_n[2] != tg->grid_values)
        return ctx->fail(YMRT_ERR_INVALID, "backward: the grid texture node is not a grid of grid_values values");
    }
    volumes = volumes || in.setting.enable_volume_scattering;
    int rc = make_job(ctx, in.scene, &in.setting, in.frame_index, in.tile_begin, in.tile_end,
                      reinterpret_cast<float4*>(in.out_rgba_device), &jobs[k], &scenes[k], in.path_radiance_device,
                      in.dloss_device);
    if (rc != YMRT_OK) return rc;
    keys[k] = in.scene;
  }
  if (grid && !volumes) return ctx->fail(YMRT_ERR_INVALID, "backward: grid gradients need volume scattering on");
  const std::vector<DeviceScene> slots = assign_slots(jobs, scenes, keys);
  if (slots.size() > kMaxSceneSlots) return ctx->fail(YMRT_ERR_INVALID, "backward: too many distinct scenes in one call");
  BatchMemory M;
  int rc = context_memory(ctx, jobs.size(), &M);
  if (rc != YMRT_OK) return rc;
  WaveOptions opt;
  opt.adjoint = true;
  opt.volumes = volumes;
  opt.trace_block = ctx->trace_block;
  opt.sort_rays = ctx->sort_rays;
  opt.features = batch_features(slots.data(), slots.size());
  opt.grads = materials ? tg->material_grads_device : nullptr;
  opt.grad_materials = materials ? tg->n_materials : 0;
  opt.grid_grads = grid ? tg->grid_grads_device : nullptr;
  opt.grid_tex = grid ? tg->grid_texture : kEmpty;
  SlotLease lease(ctx, (uint32_t)slots.size());
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slots for this device");
  for (JobDesc& j : jobs) j.scene_slot = lease.slot(j.scene_slot);
  if ((e = lease.upload(slots.data(), (uint32_t)slots.size())) != cudaSuccess)
    return ctx->cuda_fail(e, "uploading constants");
  if (materials &&
      (e = cudaMemsetAsync(tg->material_grads_device, 0, sizeof(float) * kGradParams * tg->n_materials, st)) !=
          cudaSuccess)
    return ctx->cuda_fail(e, "clearing the material gradients");
  if (grid && (e = cudaMemsetAsync(tg->grid_grads_device, 0, sizeof(float) * tg->grid_values, st)) != cudaSuccess)
    return ctx->cuda_fail(e, "clearing the grid gradients");
  BatchResult r;
  if ((rc = run_batch(ctx, M, jobs, opt, ctx->profiling, ctx->graph_loop, &r)) != YMRT_OK) return rc;
  if ((e = cudaMemcpyAsync(ctx->counters_host, M.counters, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return ctx->cuda_fail(e, "reading counters");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "backward");
  return finish_batch(ctx, r, stats);
}

int ymrt_render_backward(ymrt_context* ctx, const ymrt_job* jobs_in, int n_jobs, float* grads_device,
                         uint32_t n_materials, ymrt_stats* stats) {
  if (!ctx || !jobs_in || n_jobs <= 0 || !grads_device || n_materials == 0) return YMRT_ERR_INVALID;
  ymrt_backward_targets tg{};
  tg.material_grads_device = grads_device;
  tg.n_materials = n_materials;
  tg.grid_texture = kEmpty;
  return ymrt_render_backward_ex(ctx, jobs_in, n_jobs, &tg, stats);
}

int ymrt_scene_set_material_params(ymrt_scene* scene, uint32_t first, uint32_t count, const float* params) {
  if (!scene || !params) return YMRT_ERR_INVALID;
  if ((size_t)first + count > scene->materials.size())
    return scene->ctx->fail(YMRT_ERR_INVALID, "material range out of bounds");
  for (uint32_t k = 0; k < count; ++k) {
    Material& m = scene->materials[first + k];
    if (m.material_type != kDefaultMtl) continue;
    const float* q = params + 4 * k;
    m.default_mtl.diffuse_albedo = vec3(q[0], q[1], q[2]);
    m.default_mtl.alpha_x = q[3];
    m.default_mtl.alpha_y = q[3];
  }
  cudaSetDevice(scene->ctx->device);
  cudaError_t e = cudaMemcpyAsync(const_cast<Material*>(scene->dev.materials) + first, scene->materials.data() + first,
                                  sizeof(Material) * count, cudaMemcpyHostToDevice, scene->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(scene->ctx->stream);
  if (e != cudaSuccess) return scene->ctx->cuda_fail(e, "updating materials");
  return YMRT_OK;
}

int ymrt_host_scene_set_transforms(ymrt_host_scene* hs, uint32_t first, uint32_t count, const float* object_to_world,
                                   const float* world_to_object, const float* scales) {
  if (!hs || !object_to_world) return YMRT_ERR_INVALID;
  std::string err;
  const int rc = set_transforms(&hs->s, first, count, object_to_world, world_to_object, scales, &err);
  if (rc != YMRT_OK) g_last_error = err;
  return rc;
}

int ymrt_scene_set_transforms(ymrt_scene* sc, uint32_t first, uint32_t count, const float* object_to_world,
                              const float* world_to_object, const float* scales) {
  if (!sc || !object_to_world) return YMRT_ERR_INVALID;
  ymrt_context* ctx = sc->ctx;
  DeviceScene& D = sc->dev;
  auto& T = sc->top;
  if (first > D.transform_count || count > D.transform_count - first)
    return ctx->fail(YMRT_ERR_INVALID, "transform range out of bounds");
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const uint32_t n = D.instance_count;
  std::vector<mat4> m(count), mi(count);
  for (uint32_t k = 0; k < count; ++k) {
    std::memcpy(&m[k], object_to_world + 16 * (size_t)k, sizeof(mat4));
    if (world_to_object) std::memcpy(&mi[k], world_to_object + 16 * (size_t)k, sizeof(mat4));
    else mi[k] = mat4_inverse(m[k]);
    if (scales) {
      const float* q = scales + 3 * (size_t)k;
      T.transform_scales[first + k] = vmax(vec3(0.0001f), vec3(q[0], q[1], q[2]));
    }
  }
  cudaError_t e = cudaSuccess;
  if (count > 0) {
    // the scene's own transform arrays (uploaded by ymrt_scene_upload)
    e = cudaMemcpyAsync(const_cast<mat4*>(D.transforms) + first, m.data(), sizeof(mat4) * count,
                        cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(const_cast<mat4*>(D.i_transforms) + first, mi.data(), sizeof(mat4) * count,
                          cudaMemcpyHostToDevice, st);
  }
  const size_t nb = 2 * (size_t)n - 1;
  if (!T.prepared) {
    for (int k = 0; k < 2 && e == cudaSuccess; ++k) {
      e = T.inst[k].ensure(sizeof(Instance) * n);
      if (e == cudaSuccess) e = T.bucket[k].ensure(n);
      if (e == cudaSuccess) e = T.file_idx[k].ensure(sizeof(uint32_t) * n);
    }
    if (e == cudaSuccess) e = T.items.ensure(sizeof(BuildItem) * n);
    if (e == cudaSuccess) e = T.nodes.ensure(sizeof(BinNode) * nb);
    if (e == cudaSuccess) e = T.mid.ensure(nb);
    if (e == cudaSuccess) e = T.kind.ensure(nb);
    if (e == cudaSuccess) e = T.left.ensure(sizeof(uint32_t) * nb);
    if (e == cudaSuccess) e = T.stack.ensure(sizeof(uint32_t) * 2 * (7 * nb + 2));
    if (e == cudaSuccess) e = T.wide.ensure(sizeof(WideNode) * std::max<size_t>(2 * (size_t)n, 2));
    if (e == cudaSuccess) e = T.prims.ensure(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = T.offsets.ensure(sizeof(uint32_t) * n);
    if (e == cudaSuccess) e = T.inside.ensure(n);
    if (e == cudaSuccess) e = T.camera.ensure(sizeof(RayTransfer));
    if (e == cudaSuccess) e = T.counts.ensure(sizeof(uint32_t) * 4);
    if (e == cudaSuccess) e = T.scales.ensure(sizeof(vec3) * std::max<size_t>(T.transform_scales.size(), 1));
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(T.inst[0].ptr, D.instances, sizeof(Instance) * n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(T.bucket[0].ptr, D.inst_bucket, n, cudaMemcpyDeviceToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(T.file_idx[0].ptr, T.file_index.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "preparing the top-level rebuild");
    T.cur = 0;
    T.prepared = true;
  }
  if (e == cudaSuccess && !T.transform_scales.empty())
    e = cudaMemcpyAsync(T.scales.ptr, T.transform_scales.data(), sizeof(vec3) * T.transform_scales.size(),
                        cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "uploading transforms");
  const int c = T.cur, o = c ^ 1;
  TlasBuild b{};
  b.n = n;
  b.instances = T.inst[c].as<Instance>();
  b.instances_out = T.inst[o].as<Instance>();
  b.bucket = T.bucket[c].as<uint8_t>();
  b.bucket_out = T.bucket[o].as<uint8_t>();
  b.file_index = T.file_idx[c].as<uint32_t>();
  b.file_index_out = T.file_idx[o].as<uint32_t>();
  b.transforms = D.transforms;
  b.i_transforms = D.i_transforms;
  b.transform_scales = T.scales.as<vec3>();
  b.geometries = D.geometries;
  b.materials = D.materials;
  b.material_count = D.material_count;
  b.tri_corners = D.tri_corners;
  b.pos_idx = D.pos_idx;
  b.positions = D.positions;
  b.items = T.items.as<BuildItem>();
  b.nodes = T.nodes.as<BinNode>();
  b.mid = T.mid.as<uint8_t>();
  b.split_kind = T.kind.as<uint8_t>();
  b.split_left = T.left.as<uint32_t>();
  b.stack = T.stack.as<uint32_t>();
  b.wide = T.wide.as<WideNode>();
  b.prims = T.prims.as<uint32_t>();
  b.lights = const_cast<ShapeLight*>(D.shape_lights);
  b.light_table = const_cast<float*>(D.shape_light_table);
  b.light_count = D.shape_light_count;
  b.light_offsets = T.offsets.as<uint32_t>();
  b.inside = T.inside.as<uint8_t>();
  b.camera_transfer = T.camera.as<RayTransfer>();
  b.counts = T.counts.as<uint32_t>();
  launch_tlas_rebuild(b, T.max_leaf, D.camera.position, camera_media_ray(D.camera), st);
  uint32_t counts[4] = {};
  RayTransfer rt{};
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(counts, T.counts.ptr, sizeof(counts), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&rt, T.camera.ptr, sizeof(rt), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "rebuilding the top level");
  if (counts[2] != D.shape_light_count || counts[1] != n)
    return ctx->fail(YMRT_ERR_INVALID, "top-level rebuild: light or leaf count changed");
  T.cur = o;
  T.node_count = counts[0];
  D.instances = T.inst[o].as<Instance>();
  D.inst_bucket = T.bucket[o].as<uint8_t>();
  D.tlas_nodes = T.wide.as<WideNode>();
  D.tlas_prims = T.prims.as<uint32_t>();
  D.camera.transfer = rt;
  return YMRT_OK;
}

long long ymrt_scene_download(const ymrt_scene* sc, int what, void* out, size_t cap_bytes) {
  if (!sc) return YMRT_ERR_INVALID;
  const DeviceScene& D = sc->dev;
  const auto& T = sc->top;
  const void* src = nullptr;
  bool device = true;
  size_t bytes = 0;
  switch (what) {
    case YMRT_SCENE_TLAS_NODES: src = D.tlas_nodes; bytes = sizeof(WideNode) * T.node_count; break;
    case YMRT_SCENE_TLAS_PRIMS: src = D.tlas_prims; bytes = sizeof(uint32_t) * D.instance_count; break;
    case YMRT_SCENE_INSTANCES: src = D.instances; bytes = sizeof(Instance) * D.instance_count; break;
    case YMRT_SCENE_SHAPE_LIGHTS: src = D.shape_lights; bytes = sizeof(ShapeLight) * D.shape_light_count; break;
    case YMRT_SCENE_LIGHT_TABLE: src = D.shape_light_table; bytes = sizeof(float) * D.shape_light_count; break;
    case YMRT_SCENE_INSTANCE_BUCKETS: src = D.inst_bucket; bytes = D.instance_count; break;
    case YMRT_SCENE_CAMERA_MEDIA: src = &D.camera.transfer; bytes = sizeof(RayTransfer); device = false; break;
    case YMRT_SCENE_FILE_INDEX:
      bytes = sizeof(uint32_t) * D.instance_count;
      if (T.prepared) src = T.file_idx[T.cur].ptr;
      else {
        src = T.file_index.data();
        device = false;
      }
      break;
    default:
      return YMRT_ERR_INVALID;
  }
  if (!out) return (long long)bytes;
  if (cap_bytes < bytes) return YMRT_ERR_INVALID;
  if (!device) {
    std::memcpy(out, src, bytes);
    return (long long)bytes;
  }
  cudaSetDevice(sc->ctx->device);
  cudaError_t e = cudaMemcpyAsync(out, src, bytes, cudaMemcpyDeviceToHost, sc->ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(sc->ctx->stream);
  if (e != cudaSuccess) return sc->ctx->cuda_fail(e, "downloading the scene");
  return (long long)bytes;
}

int ymrt_scene_set_density_grid(ymrt_scene* scene, uint32_t texture_index, int nx, int ny, int nz,
                                const float* values, int store_half) {
  if (!scene || !values || nx < 1 || ny < 1 || nz < 1) return YMRT_ERR_INVALID;
  ymrt_context* ctx = scene->ctx;
  if (texture_index >= scene->textures.size()) return ctx->fail(YMRT_ERR_INVALID, "texture index out of range");
  const size_t n = (size_t)nx * (size_t)ny * (size_t)nz;
  if (n > (size_t)1 << 30) return ctx->fail(YMRT_ERR_INVALID, "grid larger than 2^30 values");
  float vmax = 0.0f;
  std::vector<uint16_t> half;
  if (store_half) half.resize(n);
  for (size_t i = 0; i < n; ++i) {
    float v = values[i];
    if (!std::isfinite(v)) return ctx->fail(YMRT_ERR_INVALID, "grid values must be finite");
    if (store_half) {
      half[i] = __half_as_ushort(__float2half_rn(v));
      v = __half2float(__ushort_as_half(half[i]));
    }
    vmax = std::max(vmax, v);
  }
  cudaSetDevice(ctx->device);
  std::unique_ptr<DeviceBuffer>& buf = scene->grids[texture_index];
  if (!buf) buf.reset(new DeviceBuffer());
  const size_t bytes = n * (store_half ? sizeof(uint16_t) : sizeof(float));
  cudaError_t e = buf->ensure(bytes);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(buf->ptr, store_half ? static_cast<const void*>(half.data()) : static_cast<const void*>(values),
                        bytes, cudaMemcpyHostToDevice, ctx->stream);
  Texture& t = scene->textures[texture_index];
  t = Texture{};
  t.type = kTexGrid;
  t.child[0] = t.child[1] = kEmpty;
  t.value = vmax;
  t.grid_n[0] = nx;
  t.grid_n[1] = ny;
  t.grid_n[2] = nz;
  t.grid_half = store_half ? 1 : 0;
  t.grid = buf->ptr;
  scene->dev.grid_count = 0;
  for (const Texture& x : scene->textures) scene->dev.grid_count += x.type == kTexGrid ? 1u : 0u;
  scene->dev.textured = uses_textures(scene->materials, scene->textures) ? 1u : 0u;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(const_cast<Texture*>(scene->dev.textures) + texture_index, &t, sizeof(Texture),
                        cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "uploading the density grid");
  return YMRT_OK;
}

int ymrt_scene_get_material_params(const ymrt_scene* scene, uint32_t first, uint32_t count, float* params) {
  if (!scene || !params || (size_t)first + count > scene->materials.size()) return YMRT_ERR_INVALID;
  for (uint32_t k = 0; k < count; ++k) {
    const Material& m = scene->materials[first + k];
    float* q = params + 4 * k;
    if (m.material_type != kDefaultMtl) {
      q[0] = q[1] = q[2] = q[3] = 0.0f;
      continue;
    }
    q[0] = m.default_mtl.diffuse_albedo.x;
    q[1] = m.default_mtl.diffuse_albedo.y;
    q[2] = m.default_mtl.diffuse_albedo.z;
    q[3] = m.default_mtl.alpha_x;
  }
  return YMRT_OK;
}

int ymrt_render_forward(ymrt_scene* sc, const ymrt_render_setting* setting, int frame_index, float* out_rgba,
                        int out_on_device, ymrt_stats* stats) {
  return ymrt_render_tiles(sc, setting, frame_index, 0, 0, out_rgba, out_on_device, stats);
}

}  // extern "C"

// ------------------------------------------------- allocation-free render ---
//
// Some callers cannot allocate device memory while they render: a host that
// hands the renderer a fixed memory budget up front (an embedding application
// with its own pool allocator, or a process that must not grow its footprint
// once its frame loop runs), or code that runs where a cudaMalloc would
// synchronise the device and stall other work. ymrt_render_tiles_noalloc
// serves them: instead of the context's path queues (allocated on first use)
// it places the path queues, the hit records and the wave counters in the
// fixed array below, which exists once per device for as long as the library
// is loaded.
//
// Limits: the array holds kNoAllocScratchBytes; one wave holds as many
// 16x16-pixel tiles of samples as fit (at least one tile of 256 * spp
// paths must fit, so spp is bounded by the array size). All calls share the
// array: calls that overlap on the GPU (from several host threads, or on
// several contexts of one device) race on it and must be serialised by the
// caller. The wave counters are cleared at the start of every call; the
// queues need no clearing (every slot is written before it is read).

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;  // 32 MiB per device
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device ordinal, looked up once per
// device (with that device current) and kept for the life of the process.
std::mutex g_noalloc_mutex;
void* g_noalloc_addr[128] = {};

constexpr size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Bytes one path slot needs across both path pools and the hit pool.
constexpr size_t kPoolSlotBytes =
    4 * sizeof(float4) + sizeof(uint4) + 2 * sizeof(uint2) + sizeof(RayTransfer) + sizeof(uint32_t) + 1;
constexpr size_t kHitSlotBytes = sizeof(float4) + sizeof(uint4) + kMaxNearby * sizeof(uint4) + sizeof(uint32_t) + 1;

uint32_t noalloc_capacity() {
  // counters, one job, and the alignment slack of the carved arrays
  const size_t fixed = align256(sizeof(WaveCounters)) + align256(sizeof(WaveControl)) + align256(sizeof(JobDesc)) + 20 * 256;
  return (uint32_t)((kNoAllocScratchBytes - fixed) / (2 * kPoolSlotBytes + kHitSlotBytes));
}

// Carves the two path pools, the hit pool and the counters out of `base`;
// returns the number of bytes used.
size_t carve(unsigned char* base, uint32_t n, PathPool pools[2], HitPool* hits, WaveCounters** counters,
             WaveControl** ctl, JobDesc** job) {
  size_t off = 0;
  auto take = [&](size_t bytes) {
    unsigned char* p = base + off;
    off = align256(off + bytes);
    return p;
  };
  *counters = reinterpret_cast<WaveCounters*>(take(sizeof(WaveCounters)));
  *ctl = reinterpret_cast<WaveControl*>(take(sizeof(WaveControl)));
  *job = reinterpret_cast<JobDesc*>(take(sizeof(JobDesc)));
  for (int k = 0; k < 2; ++k) {
    PathPool& P = pools[k];
    P.ray_o = reinterpret_cast<float4*>(take(n * sizeof(float4)));
    P.ray_d = reinterpret_cast<float4*>(P.ray_o + n);
    P.throughput = P.ray_d + n;
    P.radiance = P.throughput + n;
    P.sampler = reinterpret_cast<uint4*>(P.radiance + n);
    off = align256((reinterpret_cast<unsigned char*>(P.sampler + n)) - base);
    P.pixel_flags = reinterpret_cast<uint2*>(take(n * sizeof(uint2)));
    P.last_hit = reinterpret_cast<uint2*>(take(n * sizeof(uint2)));
    P.transfer = reinterpret_cast<RayTransfer*>(take(n * sizeof(RayTransfer)));
    P.path_id = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
    P.transfer_count = reinterpret_cast<uint8_t*>(take(n));
    P.capacity = n;
  }
  hits->bary_t = reinterpret_cast<float4*>(take(n * sizeof(float4)));
  hits->ids = reinterpret_cast<uint4*>(take(n * sizeof(uint4)));
  hits->nearby = reinterpret_cast<uint4*>(take(n * kMaxNearby * sizeof(uint4)));
  hits->vol_w = nullptr;  // volume scattering is not rendered by this entry point
  hits->order = reinterpret_cast<uint32_t*>(take(n * sizeof(uint32_t)));
  hits->bucket = reinterpret_cast<uint8_t*>(take(n));
  hits->ray_key = nullptr;  // continuing rays are traced in slot order here
  hits->ray_bins = nullptr;
  hits->ray_order = nullptr;
  return off;
}

}  // namespace

extern "C" {

uint32_t ymrt_noalloc_max_paths(void) { return noalloc_capacity(); }

int ymrt_render_tiles_noalloc(ymrt_scene* sc, const ymrt_render_setting* setting, int frame_index, int tile_begin,
                              int tile_end, float* out_rgba_device, ymrt_stats* stats) {
  if (!sc || !setting || !out_rgba_device) return YMRT_ERR_INVALID;
  ymrt_context* ctx = sc->ctx;
  std::vector<JobDesc> jobs(1);
  DeviceScene scene;
  int rc = make_job(ctx, sc, setting, frame_index, tile_begin, tile_end, reinterpret_cast<float4*>(out_rgba_device),
                    &jobs[0], &scene);
  if (rc != YMRT_OK) return rc;
  // (make_job has already turned off what the scene lacks, as for ymrt_render_tiles)
  if (jobs[0].setting.enable_distant_light)
    return ctx->fail(YMRT_ERR_UNSUPPORTED, "ymrt_render_tiles_noalloc: distant lights are not rendered by this entry point");
  if (jobs[0].setting.enable_volume_scattering)
    return ctx->fail(YMRT_ERR_UNSUPPORTED, "ymrt_render_tiles_noalloc: volume scattering is not rendered by this entry point");
  const uint32_t spp = jobs[0].spp;
  const uint32_t per_tile = (uint32_t)kTilePixels * spp;
  const uint32_t cap = noalloc_capacity();
  if (per_tile > cap)
    return ctx->fail(YMRT_ERR_INVALID, "ymrt_render_tiles_noalloc: one 16x16 tile at " + std::to_string(spp) +
                                           " spp needs " + std::to_string(per_tile) + " path slots; the fixed " +
                                           std::to_string(kNoAllocScratchBytes >> 20) + " MiB scratch array holds " +
                                           std::to_string(cap) + " (at most " + std::to_string(cap / kTilePixels) +
                                           " spp)");
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaSetDevice");
  if (ctx->device < 0 || ctx->device >= 128) return ctx->fail(YMRT_ERR_INVALID, "device ordinal out of range");
  unsigned char* base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_addr[ctx->device]) {
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr) return ctx->cuda_fail(e, "cudaGetSymbolAddress(scratch)");
      g_noalloc_addr[ctx->device] = ptr;
    }
    base = static_cast<unsigned char*>(g_noalloc_addr[ctx->device]);
  }
  BatchMemory M;
  if (carve(base, cap, M.pool, &M.hits, &M.counters, &M.ctl, &M.jobs) > kNoAllocScratchBytes)
    return ctx->fail(YMRT_ERR_OVERFLOW, "scratch layout exceeds the fixed array");
  M.capacity = cap;
  cudaStream_t st = ctx->stream;
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  jobs[0].scene_slot = lease.slot(0);
  if ((e = lease.upload(&scene, 1)) != cudaSuccess) return ctx->cuda_fail(e, "uploading constants");
  if ((e = cudaMemsetAsync(out_rgba_device, 0, (size_t)sc->width * sc->height * sizeof(float4), st)) != cudaSuccess)
    return ctx->cuda_fail(e, "clearing the image");
  WaveOptions opt;
  opt.features = batch_features(&scene, 1);
  BatchResult r;
  if ((rc = run_batch(ctx, M, jobs, opt, false, false, &r)) != YMRT_OK) return rc;
  if ((e = cudaMemcpyAsync(ctx->counters_host, M.counters, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return ctx->cuda_fail(e, "reading counters");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return ctx->cuda_fail(e, "frame");
  return finish_batch(ctx, r, stats);
}

int ymrt_accumulate(ymrt_scene* sc, const float* noise, float* acc, int frame_index) {
  if (!sc || !noise || !acc || frame_index < 1) return YMRT_ERR_INVALID;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  launch_accumulate(reinterpret_cast<const float4*>(noise), reinterpret_cast<float4*>(acc),
                    (uint32_t)sc->width * (uint32_t)sc->height, frame_index, ctx->stream);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  return e == cudaSuccess ? YMRT_OK : ctx->cuda_fail(e, "accumulate");
}

// ---- the reference's stage interface (include/ymrt_compat.h) ----

namespace {
struct CompatBinding {
  std::mutex m;
  ymrt_context* ctx = nullptr;
  ymrt_scene* scene = nullptr;
  bool frame_marked = false;
  int frame_index = 0;
  bool editor_marked = false;  // the editor view's current frame, as frame_marked
  int editor_frame = 0;
};
CompatBinding g_compat;

int compat_sync(void* stream) {
  if (!stream) return YMRT_OK;
  cudaError_t e = cudaStreamSynchronize(*static_cast<cudaStream_t*>(stream));
  if (e != cudaSuccess) {
    g_last_error = std::string("caller's stream: ") + cudaGetErrorString(e);
    return YMRT_ERR_CUDA;
  }
  return YMRT_OK;
}

int compat_clear_counter(void* device_counter) {
  if (!device_counter) return YMRT_ERR_INVALID;
  cudaError_t e = cudaMemset(device_counter, 0, 3 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e != cudaSuccess) {
    g_last_error = std::string("clearing the ray counter: ") + cudaGetErrorString(e);
    return YMRT_ERR_CUDA;
  }
  return YMRT_OK;
}
}  // namespace

int ymrt_compat_bind(ymrt_context* ctx, ymrt_scene* scene) {
  if (scene && (!ctx || scene->ctx != ctx)) return YMRT_ERR_INVALID;
  std::lock_guard<std::mutex> lk(g_compat.m);
  g_compat.ctx = ctx;
  g_compat.scene = scene;
  g_compat.frame_marked = false;
  return YMRT_OK;
}

int ymrt_compat_alloc_counter(void** host_counter, void** device_counter) {
  if (!host_counter || !device_counter) return YMRT_ERR_INVALID;
  *host_counter = std::calloc(1, 3 * sizeof(uint32_t));
  if (!*host_counter) return YMRT_ERR_OOM;
  cudaError_t e = cudaMalloc(device_counter, 3 * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(*device_counter, 0, 3 * sizeof(uint32_t));
  if (e != cudaSuccess) {
    std::free(*host_counter);
    *host_counter = nullptr;
    g_last_error = std::string("allocating the ray counter: ") + cudaGetErrorString(e);
    return YMRT_ERR_CUDA;
  }
  return YMRT_OK;
}

int ymrt_compat_free_counter(void* host_counter, void* device_counter) {
  std::free(host_counter);
  if (device_counter && cudaFree(device_counter) != cudaSuccess) return YMRT_ERR_CUDA;
  return YMRT_OK;
}

int ymrt_compat_generate(int frame_index, const ymrt_render_setting* setting, void* device_counter,
                         uint32_t next_tile, uint32_t tile_count, uint32_t width, uint32_t height, uint32_t tiles_x,
                         uint32_t tiles_y, void* stream) {
  (void)device_counter;
  (void)tile_count;
  std::lock_guard<std::mutex> lk(g_compat.m);
  if (!g_compat.scene || !setting) {
    g_last_error = "no scene bound (ymrt_compat_bind)";
    return YMRT_ERR_INVALID;
  }
  ymrt_scene* sc = g_compat.scene;
  if ((int)width != sc->width || (int)height != sc->height ||
      tiles_x != (width + 15) / 16 || tiles_y != (height + 15) / 16) {
    g_last_error = "frame size differs from the bound scene's";
    return YMRT_ERR_INVALID;
  }
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  if (next_tile == 0) {
    g_compat.frame_marked = true;
    g_compat.frame_index = frame_index;
  }
  return YMRT_OK;
}

int ymrt_compat_trace(int frame_index, const ymrt_render_setting* setting, void* device_counter, uint32_t width,
                      uint32_t height, float* noise_rgba, void* stream) {
  std::lock_guard<std::mutex> lk(g_compat.m);
  if (!g_compat.scene || !setting || !noise_rgba) {
    g_last_error = "no scene bound (ymrt_compat_bind) or null argument";
    return YMRT_ERR_INVALID;
  }
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  ymrt_scene* sc = g_compat.scene;
  if ((int)width != sc->width || (int)height != sc->height) {
    g_last_error = "frame size differs from the bound scene's";
    return YMRT_ERR_INVALID;
  }
  if (g_compat.frame_marked && g_compat.frame_index == frame_index) {
    g_compat.frame_marked = false;
    ymrt_stats st;
    rc = ymrt_render_tiles(sc, setting, frame_index, 0, 0, noise_rgba, 1, &st);
    if (rc != YMRT_OK) {
      g_last_error = sc->ctx->error;
      return rc;
    }
    if (st.device_errors) {
      g_last_error = "device errors while rendering";
      return YMRT_ERR_CUDA;
    }
  }
  return compat_clear_counter(device_counter);
}

int ymrt_compat_shade(int frame_index, const ymrt_render_setting* setting, void* device_counter, uint32_t width,
                      uint32_t height, float* noise_rgba, void* stream) {
  (void)frame_index;
  (void)setting;
  (void)width;
  (void)height;
  (void)noise_rgba;
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  return compat_clear_counter(device_counter);
}

int ymrt_compat_editor_generate(int frame_index, void* device_counter, uint32_t next_tile, uint32_t width,
                                uint32_t height, void* stream) {
  (void)device_counter;
  std::lock_guard<std::mutex> lk(g_compat.m);
  if (!g_compat.scene) {
    g_last_error = "no scene bound (ymrt_compat_bind)";
    return YMRT_ERR_INVALID;
  }
  if (width == 0 || height == 0) return YMRT_ERR_INVALID;
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  if (next_tile == 0) {
    g_compat.editor_marked = true;
    g_compat.editor_frame = frame_index;
  }
  return YMRT_OK;
}

int ymrt_compat_editor_trace(int frame_index, const ymrt_render_setting* setting, void* device_counter, uint32_t width,
                             uint32_t height, float* beauty_rgba, uint32_t* primitive_index, void* stream) {
  std::lock_guard<std::mutex> lk(g_compat.m);
  if (!g_compat.scene || !setting || !beauty_rgba || !primitive_index) {
    g_last_error = "no scene bound (ymrt_compat_bind) or null argument";
    return YMRT_ERR_INVALID;
  }
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  if (g_compat.editor_marked && g_compat.editor_frame == frame_index) {
    g_compat.editor_marked = false;
    rc = ymrt_render_editor_view(g_compat.scene, setting, width, height, beauty_rgba, primitive_index, 1);
    if (rc != YMRT_OK) {
      g_last_error = g_compat.scene->ctx->error;
      return rc;
    }
  }
  return compat_clear_counter(device_counter);
}

int ymrt_compat_editor_shade(void* device_counter, void* stream) {
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  return compat_clear_counter(device_counter);
}

int ymrt_compat_post_process(float* image_rgba, const uint32_t* primitive_index, uint32_t width, uint32_t height,
                             uint32_t selected, float gamma, float exposure, int outline, void* stream) {
  std::lock_guard<std::mutex> lk(g_compat.m);
  if (!g_compat.ctx) {
    g_last_error = "no context bound (ymrt_compat_bind)";
    return YMRT_ERR_INVALID;
  }
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  rc = ymrt_post_process(g_compat.ctx, image_rgba, primitive_index, width, height, selected, gamma, exposure, outline, 1);
  if (rc != YMRT_OK) g_last_error = g_compat.ctx->error;
  return rc;
}

int ymrt_compat_accumulate(const float* noise_rgba, float* acc_rgba, uint32_t width, uint32_t height, int frame_index,
                           int max_frames, void* stream) {
  if (max_frames > 0 && frame_index - 1 >= max_frames) return YMRT_OK;
  std::lock_guard<std::mutex> lk(g_compat.m);
  if (!g_compat.scene) {
    g_last_error = "no scene bound (ymrt_compat_bind)";
    return YMRT_ERR_INVALID;
  }
  if ((int)width != g_compat.scene->width || (int)height != g_compat.scene->height) {
    g_last_error = "frame size differs from the bound scene's";
    return YMRT_ERR_INVALID;
  }
  int rc = compat_sync(stream);
  if (rc != YMRT_OK) return rc;
  rc = ymrt_accumulate(g_compat.scene, noise_rgba, acc_rgba, frame_index);
  if (rc != YMRT_OK) g_last_error = g_compat.scene->ctx->error;
  return rc;
}

}  // extern "C"

namespace {
// Stages host arrays on the device for the known-answer kernels.
struct Staging {
  ymrt_context* ctx;
  std::vector<std::unique_ptr<DeviceBuffer>> bufs;
  cudaError_t err = cudaSuccess;
  template <typename T>
  T* in(const T* host, size_t n) {
    if (!host || err != cudaSuccess) return nullptr;
    bufs.emplace_back(new DeviceBuffer());
    if ((err = bufs.back()->ensure(n * sizeof(T))) != cudaSuccess) return nullptr;
    err = cudaMemcpyAsync(bufs.back()->ptr, host, n * sizeof(T), cudaMemcpyHostToDevice, ctx->stream);
    return bufs.back()->as<T>();
  }
  template <typename T>
  T* out(size_t n) {
    if (err != cudaSuccess) return nullptr;
    bufs.emplace_back(new DeviceBuffer());
    if ((err = bufs.back()->ensure(n * sizeof(T))) != cudaSuccess) return nullptr;
    return bufs.back()->as<T>();
  }
  template <typename T>
  void back(T* host, const T* dev, size_t n) {
    if (err == cudaSuccess && host) err = cudaMemcpyAsync(host, dev, n * sizeof(T), cudaMemcpyDeviceToHost, ctx->stream);
  }
};
}  // namespace

extern "C" {

int ymrt_debug_trace(ymrt_scene* sc, int n, const float* origin, const float* dir, const uint32_t* last_hit,
                     uint32_t* inst, uint32_t* tri, float* t, float* bary, int* back, int* nearby) {
  if (!sc || n < 0 || !origin || !dir || !inst || !tri || !t || !bary || !back || !nearby) return YMRT_ERR_INVALID;
  if (n == 0) return YMRT_OK;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  Staging sg{ctx};
  const float* d_o = sg.in(origin, 3 * (size_t)n);
  const float* d_d = sg.in(dir, 3 * (size_t)n);
  const uint32_t* d_lh = last_hit ? sg.in(last_hit, 2 * (size_t)n) : nullptr;
  uint32_t* d_inst = sg.out<uint32_t>(n);
  uint32_t* d_tri = sg.out<uint32_t>(n);
  float* d_t = sg.out<float>(n);
  float* d_b = sg.out<float>(3 * (size_t)n);
  int* d_back = sg.out<int>(n);
  int* d_nb = sg.out<int>(n);
  uint32_t* d_err = sg.out<uint32_t>(1);
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  cudaMemsetAsync(d_err, 0, sizeof(uint32_t), ctx->stream);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_debug_trace(lease.slot(0), n, d_o, d_d, d_lh, d_inst, d_tri, d_t, d_b, d_back, d_nb, d_err, ctx->stream);
  uint32_t errs = 0;
  sg.back(inst, d_inst, n);
  sg.back(tri, d_tri, n);
  sg.back(t, d_t, n);
  sg.back(bary, d_b, 3 * (size_t)n);
  sg.back(back, d_back, n);
  sg.back(nearby, d_nb, n);
  sg.back(&errs, d_err, 1);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "debug trace");
  if (errs) return ctx->fail(YMRT_ERR_OVERFLOW, "traversal stack overflow");
  return YMRT_OK;
}

int ymrt_debug_record_paths(ymrt_scene* sc, const ymrt_render_setting* setting, int frame_index, int tile_begin,
                            int tile_end, const uint32_t* watch_bits, uint32_t* records, int capacity, int* n_records,
                            float* out_rgba) {
  if (!sc || !setting || !watch_bits || !records || capacity < 0 || !n_records || !out_rgba) return YMRT_ERR_INVALID;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  cudaError_t e;
  const uint32_t n_pixels = (uint32_t)sc->width * sc->height;
  const size_t watch_words = (n_pixels + 31) / 32, img_bytes = (size_t)n_pixels * sizeof(float4);
  Staging sg{ctx};
  const uint32_t* d_watch = sg.in(watch_bits, watch_words);
  VertexRecord* d_rec = reinterpret_cast<VertexRecord*>(sg.out<uint32_t>((size_t)std::max(capacity, 1) * 24));
  uint32_t* d_count = sg.out<uint32_t>(1);
  float4* image = reinterpret_cast<float4*>(sg.out<float>(4 * (size_t)n_pixels));
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  if ((e = cudaMemsetAsync(d_count, 0, sizeof(uint32_t), st)) != cudaSuccess) return ctx->cuda_fail(e, "clearing");
  std::vector<JobDesc> jobs(1);
  DeviceScene scene;
  int rc = make_job(ctx, sc, setting, frame_index, tile_begin, tile_end, image, &jobs[0], &scene);
  if (rc != YMRT_OK) return rc;
  BatchMemory M;
  if ((rc = context_memory(ctx, 1, &M)) != YMRT_OK) return rc;
  WaveOptions opt;
  if ((rc = batch_options(ctx, jobs, &opt)) != YMRT_OK) return rc;
  opt.features = batch_features(&scene, 1);
  // shadow rays traced in the shading stage, so that the light each path
  // carries includes its next-event estimates, as the reference's does
  opt.defer_shadows = false;
  opt.recorder.watch = d_watch;
  opt.recorder.n_pixels = n_pixels;
  opt.recorder.out = d_rec;
  opt.recorder.count = d_count;
  opt.recorder.capacity = (uint32_t)capacity;
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  jobs[0].scene_slot = lease.slot(0);
  if ((e = lease.upload(&scene, 1)) != cudaSuccess) return ctx->cuda_fail(e, "uploading constants");
  if ((e = cudaMemsetAsync(image, 0, img_bytes, st)) != cudaSuccess) return ctx->cuda_fail(e, "clearing the image");
  BatchResult r;
  // waves launched from the host: the recorder is not part of the cached graph
  if ((rc = run_batch(ctx, M, jobs, opt, false, false, &r)) != YMRT_OK) return rc;
  uint32_t count = 0;
  sg.back(&count, d_count, 1);
  sg.back(out_rgba, reinterpret_cast<float*>(image), 4 * (size_t)n_pixels);
  if ((e = cudaMemcpyAsync(ctx->counters_host, M.counters, sizeof(WaveCounters), cudaMemcpyDeviceToHost, st)) !=
      cudaSuccess)
    return ctx->cuda_fail(e, "reading counters");
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess || sg.err != cudaSuccess)
    return ctx->cuda_fail(e != cudaSuccess ? e : sg.err, "recording paths");
  const uint32_t kept = std::min<uint32_t>(count, (uint32_t)capacity);
  if (kept && (e = cudaMemcpy(records, d_rec, (size_t)kept * sizeof(VertexRecord), cudaMemcpyDeviceToHost)) != cudaSuccess)
    return ctx->cuda_fail(e, "reading records");
  *n_records = (int)count;
  rc = finish_batch(ctx, r, nullptr);
  if (rc != YMRT_OK) return rc;
  return count > (uint32_t)capacity ? ctx->fail(YMRT_ERR_OVERFLOW, "more path vertices than the record capacity") : YMRT_OK;
}

int ymrt_debug_density(ymrt_scene* sc, uint32_t texture_index, int n, const float* points, float* out) {
  if (!sc || n < 0 || !points || !out) return YMRT_ERR_INVALID;
  if (texture_index >= sc->textures.size()) return sc->ctx->fail(YMRT_ERR_INVALID, "texture index out of range");
  if (n == 0) return YMRT_OK;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  Staging sg{ctx};
  const float* d_p = sg.in(points, 3 * (size_t)n);
  float* d_out = sg.out<float>(n);
  uint32_t* d_err = sg.out<uint32_t>(1);
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  cudaMemsetAsync(d_err, 0, sizeof(uint32_t), ctx->stream);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_debug_density(lease.slot(0), n, texture_index, d_p, d_out, d_err, ctx->stream);
  uint32_t errs = 0;
  sg.back(out, d_out, n);
  sg.back(&errs, d_err, 1);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "debug density");
  if (errs) return ctx->fail(YMRT_ERR_OVERFLOW, "texture graph too deep");
  return YMRT_OK;
}

int ymrt_host_scene_set_image(ymrt_host_scene* hs, uint32_t texture_index, const float* pixels, size_t count) {
  if (!hs || !pixels) return YMRT_ERR_INVALID;
  HostScene& s = hs->s;
  if (texture_index >= s.textures.size() || s.textures[texture_index].type != kTexImage) {
    g_last_error = "texture " + std::to_string(texture_index) + " is not an image node";
    return YMRT_ERR_INVALID;
  }
  const Texture& t = s.textures[texture_index];
  if (count != (size_t)t.width * t.height * t.channels) {
    g_last_error = "image node " + std::to_string(texture_index) + " holds " +
                   std::to_string((size_t)t.width * t.height * t.channels) + " samples";
    return YMRT_ERR_INVALID;
  }
  s.images[texture_index].assign(pixels, pixels + count);
  return YMRT_OK;
}

int ymrt_render_editor_view(ymrt_scene* sc, const ymrt_render_setting* setting, uint32_t width, uint32_t height,
                            float* beauty_rgba, uint32_t* primitive_index, int device_buffers) {
  if (!sc || !setting || !beauty_rgba || !primitive_index || width == 0 || height == 0) return YMRT_ERR_INVALID;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)width * height;
  Staging sg{ctx};
  float* d_b = beauty_rgba;
  uint32_t* d_p = primitive_index;
  if (!device_buffers) {
    d_b = const_cast<float*>(sg.in(beauty_rgba, 4 * n));
    d_p = const_cast<uint32_t*>(sg.in(primitive_index, n));
  }
  uint32_t* d_err = sg.out<uint32_t>(1);
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  cudaMemsetAsync(d_err, 0, sizeof(uint32_t), ctx->stream);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_editor_view((int)lease.slot(0), (int)width, (int)height, setting->enable_env_light ? 1 : 0, reinterpret_cast<float4*>(d_b), d_p,
                     d_err, ctx->stream);
  uint32_t errs = 0;
  if (!device_buffers) {
    sg.back(beauty_rgba, d_b, 4 * n);
    sg.back(primitive_index, d_p, n);
  }
  sg.back(&errs, d_err, 1);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "editor view");
  if (errs & kDevErrStack) return ctx->fail(YMRT_ERR_OVERFLOW, "traversal or nested-media stack overflow on the device");
  if (errs & kDevErrIter) return ctx->fail(YMRT_ERR_OVERFLOW, "a camera ray passed through too many boundaries");
  return YMRT_OK;
}

int ymrt_post_process(ymrt_context* ctx, float* image_rgba, const uint32_t* primitive_index, uint32_t width,
                      uint32_t height, uint32_t selected, float gamma, float exposure, int outline,
                      int device_buffers) {
  if (!ctx || !image_rgba || width == 0 || height == 0 || (outline && !primitive_index)) return YMRT_ERR_INVALID;
  cudaSetDevice(ctx->device);
  const size_t n = (size_t)width * height;
  Staging sg{ctx};
  float* d_i = image_rgba;
  const uint32_t* d_p = primitive_index;
  if (!device_buffers) {
    d_i = const_cast<float*>(sg.in(image_rgba, 4 * n));
    if (outline) d_p = sg.in(primitive_index, n);
  }
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  launch_post_process(reinterpret_cast<float4*>(d_i), d_p, (int)width, (int)height, selected, gamma, exposure,
                      outline != 0 && selected != kEmpty, ctx->stream);
  if (!device_buffers) sg.back(image_rgba, d_i, 4 * n);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "post process");
  return YMRT_OK;
}

int ymrt_debug_frame(ymrt_scene* sc, int n, const uint32_t* inst, const uint32_t* tri, const float* bary,
                     const int* back, const float* dir, float* out) {
  if (!sc || n < 0 || !inst || !tri || !bary || !back || !dir || !out) return YMRT_ERR_INVALID;
  if (n == 0) return YMRT_OK;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  Staging sg{ctx};
  const uint32_t* d_i = sg.in(inst, (size_t)n);
  const uint32_t* d_t = sg.in(tri, (size_t)n);
  const float* d_b = sg.in(bary, 3 * (size_t)n);
  const int* d_k = sg.in(back, (size_t)n);
  const float* d_d = sg.in(dir, 3 * (size_t)n);
  float* d_out = sg.out<float>(22 * (size_t)n);
  uint32_t* d_err = sg.out<uint32_t>(1);
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  cudaMemsetAsync(d_err, 0, sizeof(uint32_t), ctx->stream);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_debug_frame(lease.slot(0), n, d_i, d_t, d_b, d_k, d_d, d_out, d_err, ctx->stream);
  sg.back(out, d_out, 22 * (size_t)n);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "debug frame");
  return YMRT_OK;
}

int ymrt_debug_texture(ymrt_scene* sc, uint32_t texture_index, int n, const float* coords, float* rgb) {
  if (!sc || n < 0 || !coords || !rgb) return YMRT_ERR_INVALID;
  if (texture_index >= sc->textures.size()) return sc->ctx->fail(YMRT_ERR_INVALID, "texture index out of range");
  if (n == 0) return YMRT_OK;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  Staging sg{ctx};
  const float* d_c = sg.in(coords, 5 * (size_t)n);
  float* d_out = sg.out<float>(3 * (size_t)n);
  uint32_t* d_err = sg.out<uint32_t>(1);
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  cudaMemsetAsync(d_err, 0, sizeof(uint32_t), ctx->stream);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_debug_texture(lease.slot(0), n, texture_index, d_c, d_out, d_err, ctx->stream);
  uint32_t errs = 0;
  sg.back(rgb, d_out, 3 * (size_t)n);
  sg.back(&errs, d_err, 1);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "debug texture");
  if (errs) return ctx->fail(YMRT_ERR_OVERFLOW, "texture graph too deep");
  return YMRT_OK;
}

int ymrt_debug_occluded(ymrt_scene* sc, int n, const float* origin, const float* dir, const float* tmax, int* occluded) {
  if (!sc || n < 0 || !origin || !dir || !tmax || !occluded) return YMRT_ERR_INVALID;
  if (n == 0) return YMRT_OK;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  Staging sg{ctx};
  const float* d_o = sg.in(origin, 3 * (size_t)n);
  const float* d_d = sg.in(dir, 3 * (size_t)n);
  const float* d_tm = sg.in(tmax, (size_t)n);
  int* d_occ = sg.out<int>(n);
  uint32_t* d_err = sg.out<uint32_t>(1);
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  cudaMemsetAsync(d_err, 0, sizeof(uint32_t), ctx->stream);
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_debug_occluded(lease.slot(0), n, d_o, d_d, d_tm, d_occ, d_err, ctx->stream);
  uint32_t errs = 0;
  sg.back(occluded, d_occ, n);
  sg.back(&errs, d_err, 1);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "debug occluded");
  if (errs) return ctx->fail(YMRT_ERR_OVERFLOW, "traversal stack overflow");
  return YMRT_OK;
}

void ymrt_debug_fail_allocations(int count) { g_failing_allocations.store(count > 0 ? count : 0); }

int ymrt_debug_bound_record(ymrt_context* ctx, uint32_t* words, size_t n_words, int clear) {
  if (!ctx || (!words && n_words > 0)) return YMRT_ERR_INVALID;
  cudaSetDevice(ctx->device);
  std::vector<uint32_t> tmp(64, 0u);
  const cudaError_t e = read_bound_record(tmp.data(), (int)tmp.size(), clear != 0, ctx->stream);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "reading the bound record");
  std::memcpy(words, tmp.data(), sizeof(uint32_t) * std::min<size_t>(n_words, tmp.size()));
  return YMRT_OK;
}

int ymrt_debug_halton(ymrt_scene* sc, int n, const int* px, const int* py, const int* sample, int n_dims, uint64_t* index,
                      float* offset, float* dims) {
  if (!sc || n < 0 || n_dims < 0 || !px || !py || !sample || !index || !offset || (n_dims > 0 && !dims))
    return YMRT_ERR_INVALID;
  if (n == 0) return YMRT_OK;
  ymrt_context* ctx = sc->ctx;
  cudaSetDevice(ctx->device);
  Staging sg{ctx};
  const int* d_px = sg.in(px, n);
  const int* d_py = sg.in(py, n);
  const int* d_s = sg.in(sample, n);
  uint64_t* d_idx = sg.out<uint64_t>(n);
  float* d_off = sg.out<float>(2 * (size_t)n);
  float* d_dims = sg.out<float>(std::max<size_t>((size_t)n * n_dims, 1));
  if (sg.err != cudaSuccess) return ctx->cuda_fail(sg.err, "staging");
  SlotLease lease(ctx, 1);
  if (!lease.ok()) return ctx->fail(YMRT_ERR_INVALID, "no constant-memory scene slot for this device");
  if (const cudaError_t e0 = lease.upload(&sc->dev, 1); e0 != cudaSuccess) return ctx->cuda_fail(e0, "uploading constants");
  launch_debug_halton(lease.slot(0), n, d_px, d_py, d_s, n_dims, d_idx, d_off, d_dims, ctx->stream);
  sg.back(index, d_idx, n);
  sg.back(offset, d_off, 2 * (size_t)n);
  if (n_dims > 0) sg.back(dims, d_dims, (size_t)n * n_dims);
  cudaError_t e = cudaStreamSynchronize(ctx->stream);
  if (sg.err != cudaSuccess || e != cudaSuccess) return ctx->cuda_fail(sg.err != cudaSuccess ? sg.err : e, "debug halton");
  return YMRT_OK;
}

}  // extern "C"
