// Device-side buffers of one wave and the kernel launchers (kernels.cu).
#pragma once

#include <cstddef>

#include <cuda_runtime.h>

#include "ymrt_scene.h"

namespace ym {

// pixel_flags.y layout
constexpr uint32_t kFlagDepthMask = 0xFFu;        // path depth (1 = camera ray)
constexpr uint32_t kFlagNeverScatter = 1u << 8;
constexpr uint32_t kFlagCameraRay = 1u << 9;
constexpr uint32_t kFlagDead = 1u << 10;          // slot holds no live path
constexpr uint32_t kFlagJobShift = 11;            // render (job) of the batch the path belongs to (21 bits)

constexpr uint32_t kNearbyExplicit = 1u << 31;    // hit ids.w: nearby list stored in HitPool::nearby

// Shading buckets: k_extend files every hit under a bucket, a sort pass lists
// the hits bucket by bucket, and k_shade runs over that list, so each warp
// shades hits that take the same code path (lights and pass-through
// boundaries, volume scattering, or one combination of material lobes).
constexpr int kShadeBuckets = 35;
constexpr uint32_t kBucketCheap = 0;    // light, boundary pass-through, invalid material
constexpr uint32_t kBucketVolume = 1;   // scattering inside a medium
constexpr uint32_t kBucketLobes = 2;    // + bit mask of the material's lobes (coat, metal, specular, transmission, diffuse)
constexpr uint32_t kBucketMiss = 34;    // the ray left the scene: background, then the path ends
constexpr uint8_t kBucketNone = 0xFF;   // no path in this slot

constexpr uint32_t kDevErrStack = 1u;
constexpr uint32_t kDevErrQueue = 2u;
constexpr uint32_t kDevErrIter = 4u;

// Structure-of-arrays path state for `capacity` slots.
struct PathPool {
  float4* ray_o;        // origin xyz
  float4* ray_d;        // normalised direction xyz
  float4* throughput;   // rgb
  float4* radiance;     // rgb received so far
  uint2* pixel_flags;   // pixel index, flags
  uint2* last_hit;      // instance, triangle of the surface the ray leaves
  uint4* sampler;       // Halton sample index (lo, hi), dimension
  uint8_t* transfer_count;  // records in the nested-media stack
  RayTransfer* transfer;    // nested-media stack (read only when count > 0)
  uint32_t* path_id;        // the path's index within its job (for recording and replay)
  uint32_t capacity;
};

// Closest-hit results of one wave, indexed like the path pool.
struct HitPool {
  float4* bary_t;   // barycentrics (or the scattering position of a volume hit), t
  uint4* ids;       // instance, triangle, back face | volume hit << 1, nearby count | kNearbyExplicit
  uint4* nearby;    // kMaxNearby entries per slot: prim, t bits, back
  float* vol_w;     // kMaxBoundaryRecord medium-selection weights per slot (volume hits only)
  uint8_t* bucket;  // shading bucket per slot (kBucketNone: nothing to shade)
  uint32_t* order;  // slots to shade, bucket by bucket
  uint32_t* ray_order; // the continuing slots, grouped (null: rays are not grouped)
  uint32_t* ray_key;   // grouping key per continuing slot
  uint32_t* ray_bins;  // kRayBins counts, kRayBins offsets, kRayScanBlocks block offsets
};
// Continuing rays are traced grouped by origin cell and direction (k_ray_*):
// the origin's cell of a 2^kRayCellBits-per-axis grid over the scene, and the
// direction's cube face split into kRayDirSplit x kRayDirSplit squares.
constexpr uint32_t kRayCellBits = 4;
constexpr uint32_t kRayDirSplit = 4;
constexpr uint32_t kRayDirs = 6 * kRayDirSplit * kRayDirSplit;
constexpr uint32_t kRayBins = (1u << (3 * kRayCellBits)) * kRayDirs;
constexpr uint32_t kRayScanBlocks = (kRayBins + 1023) / 1024;  // at most 1024
static_assert(kRayScanBlocks <= 1024, "the block totals are scanned by one block");
constexpr size_t kRayBinWords = 2 * (size_t)kRayBins + kRayScanBlocks;

// One render of a batch (a single render is a batch of one): its scene,
// settings, output image and its range in the batch's path space (paths are
// numbered tile by tile, 256 * spp per 16x16 tile, job after job).
struct JobDesc {
  uint32_t scene_slot;            // c_scenes slot of the job's scene (with its sampler type)
  uint32_t width, height;
  RenderSetting setting;
  float4* image;                  // width * height float4, accumulated with atomics
  int frame_index;
  uint32_t spp;
  uint32_t tiles_x;
  uint32_t tile_begin;            // first tile rendered
  unsigned long long path_begin;  // first path of this job in the batch's path space
  unsigned long long path_count;  // tiles rendered * 256 * spp
  // differentiable rendering (null when unused)
  float4* path_radiance;          // forward: each path's radiance, by path index (accumulated: zero it first)
  const float4* dloss;            // adjoint: dLoss/dImage per pixel
  float* grads;                   // adjoint: dLoss/dParam, 4 per material (albedo rgb, roughness)
  uint32_t grad_materials;        // materials with gradient slots
};

// Deferred next-event shadow rays of one wave (traced by k_connect).
struct ShadowQueue {
  float4* o;   // origin xyz, maximum distance
  float4* d;   // normalised direction xyz, pixel index (bits)
  float4* c;   // contribution rgb, already weighted by throughput / spp; job index (bits)
  uint32_t* path;  // path index within the job (for per-path records)
  uint32_t capacity;
};

struct WaveCounters {
  // cleared at the start of every wave (the first kWaveClearBytes bytes)
  uint32_t next_count;             // paths written to the next pool
  uint32_t hit_count;              // hits (slots listed in HitPool::order when sorting)
  uint32_t shadow_count;           // rays written to the ShadowQueue
  uint32_t shadow_cursor;          // next ShadowQueue ray k_connect hands out
  uint32_t bucket_count[kShadeBuckets];
  uint32_t bucket_fill[kShadeBuckets];
  // cleared once per frame
  uint32_t errors;                 // kDevErr* bits
  // delta / ratio tracking loops that reached kMaxFreePath steps (the
  // reference's MAX_FREE_PATH_LENGTH, after which its loop stops and reports
  // a failed sample): reference behaviour, counted rather than raised. The
  // tracking functions reach it as the word after `errors`.
  uint32_t tracking_caps;
  unsigned long long extension_rays;
  unsigned long long shadow_rays;
  unsigned long long tri_tests;     // closest-hit queries
  unsigned long long node_visits;
  unsigned long long shadow_tri_tests;   // occlusion (and transmittance) queries
  unsigned long long shadow_node_visits;
};

constexpr size_t kWaveClearBytes = offsetof(WaveCounters, errors);
static_assert(offsetof(WaveCounters, tracking_caps) == offsetof(WaveCounters, errors) + sizeof(uint32_t),
              "the tracking functions count through errors + 1");

// Uploads scenes[k] into constant-memory slot slots[k] (k < n; slots ==
// nullptr: slot k) and the prime tables, in every translation unit that holds
// wave kernels (each has its own copy of the table).
cudaError_t upload_constants(const DeviceScene* scenes, const uint32_t* slots, uint32_t n, const uint32_t* primes,
                             const uint32_t* prime_sums, cudaStream_t stream);
constexpr uint32_t kMaxSceneSlots = 64;



// One wave: plans it on the device (k_plan: continuing paths, new paths to
// generate), generates the new camera paths after the continuing ones in A,
// traces them, lists the hits by shading bucket and shades them, writing
// continuing paths to B. With opt.defer_shadows (surfaces only; the caller
// turns it off for the indirect clamp, which needs a vertex's whole direct
// light at once) the shading kernel queues its shadow rays and k_connect
// traces them.
// ev (optional, 6 events) is recorded before generate, extend, sort, shade and
// connect and at the end. graph_condition: the handle of the CUDA graph's
// while-loop condition when the wave runs inside one (k_finish sets it).
// Returns the number of kernels launched.
// Wave control of one batch in device memory: k_plan fills it at the start
// of every wave and every kernel of the wave reads its sizes from it, so the
// wave loop takes no host decisions and can run as a CUDA graph.
struct WaveControl {
  unsigned long long cursor;      // next path of the batch to generate
  unsigned long long total;       // paths in the batch
  unsigned long long gen_cursor;  // first path generated in this wave
  unsigned long long hits;        // hits shaded so far
  uint32_t capacity;              // path slots per pool
  uint32_t live;                  // continuing paths at the start of this wave
  uint32_t gen;                   // paths generated in this wave
  uint32_t count;                 // live + gen
  uint32_t waves;                 // waves finished
  uint32_t max_waves;             // bound on waves (then YMRT_DEVERR_ITER)
  uint32_t more;                  // 1 while paths remain
  uint32_t reserved;
};

constexpr int kGradParams = 4;  // differentiated parameters per material: albedo r, g, b, roughness

// One path vertex as the closest-hit stage leaves it: the ray, what it hit
// (after volume free flight), the throughput and the light received so far.
// The debug recorder writes one per watched path per wave, so that a
// render's paths can be replayed vertex by vertex against another
// renderer's (ymrt_debug_record_paths).
struct VertexRecord {
  uint32_t pixel, depth;  // pixel index in the job's image; 1 = camera ray
  uint32_t flags;         // kVertexHit | kVertexVolume | kVertexBack
  uint32_t inst, tri;
  float t;
  float o[3], d[3];
  float bary[3];          // barycentrics, or the scattering position of a volume hit
  float throughput[3];
  float radiance[3];
  uint32_t path;          // path index within the job
  uint32_t pad[2];
};
static_assert(sizeof(VertexRecord) == 96, "VertexRecord is 24 words");
constexpr uint32_t kVertexHit = 1u, kVertexVolume = 2u, kVertexBack = 4u;
// Recording of the paths of watched pixels of job 0 (debug only; out ==
// nullptr turns it off).
struct PathRecorder {
  const uint32_t* watch = nullptr;  // one bit per pixel of job 0's image
  uint32_t n_pixels = 0;
  VertexRecord* out = nullptr;
  uint32_t* count = nullptr;        // records written (may exceed capacity: those past it are dropped)
  uint32_t capacity = 0;
};

struct WaveOptions {
  uint32_t capacity = 0;       // path slots per pool (sizes the grids)
  bool volumes = false;        // volume scattering kernels
  bool sort_hits = true;       // shade hits listed by shading bucket
  bool sort_rays = false;      // trace continuing rays grouped by origin cell and direction
  bool defer_shadows = false;  // queue surface shadow rays for k_connect (ignored with volumes)
  uint32_t features = kFeatAll;  // scene features of the batch (kFeatSpheres | kFeatGrids | kFeatTextures)
  ShadowQueue shadow_queue{};
  bool adjoint = false;        // path-replay adjoint pass (no deferral)
  float* grads = nullptr;      // adjoint: dLoss/dParam, kGradParams per material
  uint32_t grad_materials = 0;
  float* grid_grads = nullptr; // adjoint: dLoss/d(value) of the density grid at texture node grid_tex
  uint32_t grid_tex = 0xFFFFFFFFu;
  uint32_t trace_block = 128;  // threads per block of k_extend and k_connect (64, 128 or 256)
  PathRecorder recorder{};     // debug: vertices of watched paths after each closest-hit stage
};
// One wave's pools, control block, jobs and launch shape, for the launchers
// of the media (wave_media.cu) and adjoint (wave_adjoint.cu) kernels.
struct WaveArgs {
  PathPool A, B;
  HitPool H;
  WaveControl* ctl;
  const JobDesc* jobs;
  WaveCounters* counters;
  uint32_t blocks;  // kTraceBlock-thread blocks (one thread per pool slot)
  cudaStream_t stream;
  uint32_t trace_block;   // k_extend's threads per block
  uint32_t trace_blocks;  // k_extend's blocks (one thread per pool slot)
  const uint32_t* ray_order = nullptr;  // continuing slots in grouped order (null: slot order)
};
// Before any launch (and before any stream capture) on the current device:
// lets the k_extend instantiations of the media and adjoint units take a
// kMaxTraceBlock-thread block's dynamic shared memory.
void prepare_media_kernels();
void prepare_adjoint_kernels();
void launch_media_extend(uint32_t features, const WaveArgs& w);
void launch_media_shade(uint32_t features, const WaveArgs& w);
void launch_adjoint_extend_media(const WaveArgs& w, const WaveOptions& opt);
void launch_adjoint_shade(bool volumes, uint32_t features, const WaveArgs& w, const WaveOptions& opt);
cudaError_t upload_slots_media(const DeviceScene* scenes, const uint32_t* slots, uint32_t n, const uint32_t* primes,
                               const uint32_t* prime_sums, cudaStream_t stream);
cudaError_t upload_slots_adjoint(const DeviceScene* scenes, const uint32_t* slots, uint32_t n, const uint32_t* primes,
                                 const uint32_t* prime_sums, cudaStream_t stream);
struct BoundRecord;
cudaError_t read_bound_media(BoundRecord* out, bool clear, cudaStream_t stream);
cudaError_t read_bound_adjoint(BoundRecord* out, bool clear, cudaStream_t stream);

// Device buffers of a top-level rebuild (tlas_build.cu). The instance
// arrays are read in the current order and written in the build's order to
// the *_out buffers; the lights, light table and camera stack are written in
// place.
struct BuildItem;
struct BinNode;
struct TlasBuild {
  uint32_t n;  // instances
  const Instance* instances;
  Instance* instances_out;
  const uint8_t* bucket;
  uint8_t* bucket_out;
  const uint32_t* file_index;
  uint32_t* file_index_out;
  const mat4* transforms;
  const mat4* i_transforms;
  const vec3* transform_scales;
  const GeometryDesc* geometries;
  const Material* materials;
  uint32_t material_count;
  const uint32_t* tri_corners;
  const uint32_t* pos_idx;
  const float* positions;
  // build scratch
  BuildItem* items;       // n
  BinNode* nodes;         // 2n - 1
  uint8_t* mid;           // 2n - 1
  uint8_t* split_kind;    // 2n - 1
  uint32_t* split_left;   // 2n - 1
  uint32_t* stack;        // 2 * (7 * (2n - 1) + 2)
  // outputs
  WideNode* wide;         // top-level nodes (at most 2n)
  uint32_t* prims;        // n: instance per top-level leaf slot
  ShapeLight* lights;
  float* light_table;
  uint32_t light_count;   // entries the table holds (an edit keeps the count)
  uint32_t* light_offsets;  // n
  uint8_t* inside;          // n
  RayTransfer* camera_transfer;
  uint32_t* counts;         // [0] top-level nodes, [1] leaf slots, [2] light entries
};
void launch_tlas_rebuild(const TlasBuild& b, uint32_t max_leaf, vec3 cam_pos, vec3 cam_dir, cudaStream_t stream);

uint32_t launch_wave(const PathPool& A, const PathPool& B, const HitPool& H, WaveControl* ctl, const JobDesc* jobs,
                     uint32_t n_jobs, WaveCounters* counters, const WaveOptions& opt, cudaEvent_t* ev,
                     cudaStream_t stream, unsigned long long graph_condition = 0);
// Grid sizes of the persistent kernels for the current device (computed once).
void prepare_persistent_grids();
void launch_accumulate(const float4* noise, float4* acc, uint32_t n, int frame_index, cudaStream_t stream);
// Copies the device's bound record (dev_bound.cuh) into `words` (at most
// n_words 32-bit words) and optionally clears it.
cudaError_t read_bound_record(uint32_t* words, int n_words, bool clear, cudaStream_t stream);
// Known-answer launchers: each reads the scene in constant-memory slot `slot`.
// Density of texture node `tex` at object-space points (3 floats each).
void launch_debug_density(uint32_t slot, int n, uint32_t tex, const float* p, float* out, uint32_t* err, cudaStream_t stream);
void launch_debug_texture(uint32_t slot, int n, uint32_t tex, const float* c, float* out, uint32_t* err, cudaStream_t stream);
void launch_editor_view(int slot, int width, int height, int env_light, float4* beauty, uint32_t* primitive_index,
                        uint32_t* errors, cudaStream_t stream);
void launch_post_process(float4* image, const uint32_t* primitive_index, int width, int height, uint32_t selected,
                         float gamma, float exposure, bool outline, cudaStream_t stream);
void launch_debug_frame(uint32_t slot, int n, const uint32_t* inst, const uint32_t* tri, const float* bary, const int* back,
                        const float* dir, float* out, uint32_t* err, cudaStream_t stream);
void launch_debug_trace(uint32_t slot, int n, const float* o, const float* d, const uint32_t* lh, uint32_t* inst, uint32_t* tri,
                        float* t, float* bary, int* back, int* nearby, uint32_t* errors, cudaStream_t stream);
void launch_debug_occluded(uint32_t slot, int n, const float* o, const float* d, const float* tmax, int* occ, uint32_t* errors,
                           cudaStream_t stream);
void launch_debug_halton(uint32_t slot, int n, const int* px, const int* py, const int* sample, int n_dims, uint64_t* index,
                         float* offset, float* dims, cudaStream_t stream);

}  // namespace ym
