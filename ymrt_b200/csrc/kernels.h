// Device-side buffers of one wave and the kernel launchers (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "ymrt_scene.h"

namespace ym {

// pixel_flags.y layout
constexpr uint32_t kFlagDepthMask = 0xFFu;        // path depth (1 = camera ray)
constexpr uint32_t kFlagNeverScatter = 1u << 8;
constexpr uint32_t kFlagCameraRay = 1u << 9;
constexpr uint32_t kFlagDead = 1u << 10;          // slot holds no live path
constexpr uint32_t kFlagSampleShift = 11;         // sample index within the pixel (for non-Halton samplers)

constexpr uint32_t kNearbyExplicit = 1u << 31;    // hit ids.w: nearby list stored in HitPool::nearby

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
  uint32_t capacity;
};

// Closest-hit results of one wave, indexed like the path pool.
struct HitPool {
  float4* bary_t;   // barycentrics (or the scattering position of a volume hit), t
  uint4* ids;       // instance, triangle, back face | volume hit << 1, nearby count | kNearbyExplicit
  uint4* nearby;    // kMaxNearby entries per slot: prim, t bits, back
  float* vol_w;     // kMaxBoundaryRecord medium-selection weights per slot (volume hits only)
};

struct WaveCounters {
  uint32_t next_count;             // paths written to the next pool
  uint32_t errors;                 // kDevErr* bits
  unsigned long long extension_rays;
  unsigned long long shadow_rays;
  unsigned long long tri_tests;
  unsigned long long node_visits;
};

cudaError_t upload_constants(const DeviceScene& scene, const uint32_t* primes, const uint32_t* prime_sums,
                             cudaStream_t stream);
cudaError_t upload_setting(const RenderSetting& rs, cudaStream_t stream);
void launch_generate(const PathPool& P, uint32_t base, uint32_t count, uint32_t next_tile, uint32_t tiles_x,
                     int frame_index, uint32_t spp, cudaStream_t stream);
void launch_extend(const PathPool& P, uint32_t count, const HitPool& H, float4* image, WaveCounters* counters,
                   bool volumes, cudaStream_t stream);
void launch_shade(const PathPool& P, uint32_t count, const HitPool& H, const PathPool& Q, float4* image,
                  WaveCounters* counters, bool volumes, cudaStream_t stream);
void launch_accumulate(const float4* noise, float4* acc, uint32_t n, int frame_index, cudaStream_t stream);
void launch_debug_trace(int n, const float* o, const float* d, const uint32_t* lh, uint32_t* inst, uint32_t* tri,
                        float* t, float* bary, int* back, int* nearby, uint32_t* errors, cudaStream_t stream);
void launch_debug_occluded(int n, const float* o, const float* d, const float* tmax, int* occ, uint32_t* errors,
                           cudaStream_t stream);
void launch_debug_halton(int n, const int* px, const int* py, const int* sample, int n_dims, uint64_t* index,
                         float* offset, float* dims, cudaStream_t stream);

}  // namespace ym
