// Device code of the wave kernels shared by the translation units that
// instantiate them (kernels.cu: surfaces; wave_media.cu: volume scattering;
// wave_adjoint.cu: the path-replay adjoint). Each unit holds its own copy of
// the constant-memory scene table (dev_constants.cuh), which every upload
// writes.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "dev_sampler.cuh"
#include "dev_shade.cuh"
#include <cooperative_groups.h>

#include "dev_traverse.cuh"
#include "dev_volume.cuh"
#include "kernels.h"

namespace ym {

namespace cg = cooperative_groups;



// ---------------------------------------------------------------- paths ---

__device__ __forceinline__ void store_path(const PathPool& P, uint32_t i, vec3 o, vec3 d, vec3 tp, vec3 rad, uint32_t pixel,
                                           uint32_t flags, uint32_t last_inst, uint32_t last_tri, const PathSampler& hs,
                                           uint32_t path_id) {
  P.path_id[i] = path_id;
  P.ray_o[i] = make_float4(o.x, o.y, o.z, 0.0f);
  P.ray_d[i] = make_float4(d.x, d.y, d.z, 0.0f);
  P.throughput[i] = make_float4(tp.x, tp.y, tp.z, 0.0f);
  P.radiance[i] = make_float4(rad.x, rad.y, rad.z, 0.0f);
  P.pixel_flags[i] = make_uint2(pixel, flags);
  P.last_hit[i] = make_uint2(last_inst, last_tri);
  P.sampler[i] = make_uint4((uint32_t)hs.index, (uint32_t)(hs.index >> 32), hs.dim, hs.aux);
}

// Per-pixel accumulation (the reference adds the four channels with four
// float atomics, src/Shading.cu:1859-1862): one vector atomic that adds each
// channel atomically.
__device__ __forceinline__ void accumulate_pixel(float4* image, uint32_t pixel, vec3 light, float inv_spp) {
  atomicAdd(image + pixel, make_float4(light.x * inv_spp, light.y * inv_spp, light.z * inv_spp, inv_spp));
}

// A path ends: its radiance into its pixel, and (differentiable renders)
// into the job's per-path record.
__device__ __forceinline__ void finish_path(const JobDesc& J, uint32_t pixel, uint32_t path_id, vec3 rad,
                                            float inv_spp) {
  accumulate_pixel(J.image, pixel, rad, inv_spp);
  // added, not stored: deferred shadow rays of the path add to the same record
  if (J.path_radiance) atomicAdd(J.path_radiance + path_id, make_float4(rad.x, rad.y, rad.z, 0.0f));
}

template <bool kAdj>
__device__ __forceinline__ void end_path(const JobDesc& J, uint32_t pixel, uint32_t path_id, vec3 rad, float inv_spp) {
  if (!kAdj) finish_path(J, pixel, path_id, rad, inv_spp);
}

// Warp-aggregated slot allocation in the output pool.
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
  const uint32_t mask = __ballot_sync(0xFFFFFFFFu, want);
  if (!want) return kEmpty;
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(mask) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
  base = __shfl_sync(mask, base, leader);
  return base + (uint32_t)__popc(mask & ((1u << lane) - 1u));
}

__device__ __forceinline__ uint32_t flags_pack(int depth, bool never_scatter, bool camera_ray, uint32_t job) {
  return (uint32_t)depth | (never_scatter ? kFlagNeverScatter : 0u) | (camera_ray ? kFlagCameraRay : 0u) |
         (job << kFlagJobShift);
}

// ------------------------------------------------------------ generate ---

// The job holding path g of the batch's path space (binary search; jobs are
// in path order).
__device__ __forceinline__ uint32_t find_job(const JobDesc* __restrict__ jobs, uint32_t n_jobs, unsigned long long g) {
  uint32_t lo = 0, hi = n_jobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (jobs[mid].path_begin <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ void generate_path(const PathPool& P, uint32_t base, uint32_t tid,
                                              unsigned long long path_cursor, const JobDesc* __restrict__ jobs,
                                              uint32_t n_jobs);

// -------------------------------------------------------------- extend ---

// Counts this lane's hit under its shading bucket (kBucketNone: no hit), one
// atomic per bucket present in the warp, and the warp's hits in hit_count.
__device__ __forceinline__ void file_bucket(WaveCounters* counters, uint32_t bucket) {
  const bool has = bucket != kBucketNone;
  const uint32_t act = __ballot_sync(0xFFFFFFFFu, has);
  const uint32_t hits = __ballot_sync(0xFFFFFFFFu, has && bucket != kBucketMiss);
  const int lane = threadIdx.x & 31;
  if (lane == 0 && hits) atomicAdd(&counters->hit_count, (uint32_t)__popc(hits));
  if (!has) return;
  const uint32_t peers = __match_any_sync(act, bucket);
  if (lane == __ffs(peers) - 1) atomicAdd(&counters->bucket_count[bucket], (uint32_t)__popc(peers));
}

// Walks the wave's paths warp by warp (every lane of a warp takes part in each
// iteration, for the warp-collective bucket filing); the wave's size comes
// from the wave-control block, so any grid works (launched with one thread
// per pool slot, each thread takes at most one path).
//
// kF: the batch's scene features (kFeatSpheres, kFeatGrids); a batch without
// spheres or grids runs the instantiation without their code.
//
// kAdj (with kVol): the adjoint pass; each free-flight segment also adds its
// density-grid gradient terms to grid_grads, weighted by dLoss/dI times the
// radiance the path gathers after the segment (its recorded total minus what
// it gathered so far).
//
// ray_order (surfaces, optional): the continuing slots [0, live) in the order
// to trace them (k_ray_scatter: grouped by origin cell and direction), so that
// neighbouring lanes take similar walks; the new camera paths keep slot order.
//
// Launched with kTraceBlock threads by default, or any block size up to
// kMaxTraceBlock (YMRT_OPT_TRACE_BLOCK, tuned by ymrt_b200.autotune); the
// traversal stacks are in dynamic shared memory (traversal_shared_bytes).
// The launch bounds give 128 registers, four resident 128-thread blocks per
// SM: on the 1080p instanced frame 3.3% faster than five (102 registers,
// spills in the traversal loop) and 15% faster than three.
template <bool kVol, uint32_t kF, bool kAdj = false>
__global__ void __launch_bounds__(kMaxTraceBlock, 4 * kTraceBlock / kMaxTraceBlock) k_extend(PathPool P, const WaveControl* __restrict__ ctl, HitPool H,
                                                           const JobDesc* __restrict__ jobs, WaveCounters* counters,
                                                           float* grid_grads = nullptr, uint32_t grid_tex = kEmpty,
                                                           const uint32_t* __restrict__ ray_order = nullptr) {
  YM_TRAVERSAL_SHARED_DYNAMIC(s_stack);
  const uint32_t count = ctl->count;
  const uint32_t live = ray_order ? ctl->live : 0u;
  uint32_t tests = 0, nodes = 0, n_rays = 0;
  bool overflow = false;
  for (uint32_t warp_base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); warp_base < count;
       warp_base += gridDim.x * blockDim.x) {
  const uint32_t j = warp_base + (threadIdx.x & 31u);
  uint32_t i = j;
  if (j < live) {
    i = ray_order[j];
    if (i >= live) {  // not a continuing slot: the order is broken (never expected)
      atomicOr(&counters->errors, (uint32_t)kDevErrQueue);
      i = j;
    }
  }
  bool active = j < count;
  uint2 pf = active ? P.pixel_flags[i] : make_uint2(kEmpty, kFlagDead);
  if (active && (pf.y & kFlagDead)) active = false;
  uint32_t bucket = kBucketNone;
  if (active) {
    const JobDesc& J = jobs[pf.y >> kFlagJobShift];
    const uint32_t slot = J.scene_slot;
    const DeviceScene& S = c_scenes[slot];
    const float4 o4 = P.ray_o[i], d4 = P.ray_d[i];
    (void)J;
    const vec3 o(o4.x, o4.y, o4.z), d(d4.x, d4.y, d4.z);
    const uint2 lh = P.last_hit[i];
    TraversalStack st;
    st.bind(s_stack_entries, s_stack_t);
    ClosestHit ch;
    bool hit = trace_closest_impl<(kF & kFeatSpheres) != 0>(slot, st, o, d, kTMax, lh.x, lh.y, false, &ch, &tests, &nodes);
    overflow = overflow || st.overflow;
    bool volume_hit = false;
    vec3 vol_pos(0.0f);
    if (kVol && J.setting.enable_volume_scattering) {
      // volume free flight before the surface (src/Shading.cu:1828-1853)
      RayTransfer rt;
      rt.record_count = P.transfer_count[i];
      rt.max_priority_record_index = -1;
      if (rt.record_count > 0) rt = P.transfer[i];
      const uint4 s4 = P.sampler[i];
      PathSampler hs{(uint64_t)s4.x | ((uint64_t)s4.y << 32), s4.z, s4.w};
      int vidx[kMaxBoundaryRecord];
      const int n = current_volumes(rt, S.volume_count, vidx);
      vec3 trw(1.0f);
      float dist = 0.0f;
      float vw[kMaxBoundaryRecord];
      bool hv;
      if constexpr (kAdj) {
        MediumAdj am{vec3(0.0f), grid_tex, grid_grads};
        if (grid_grads && J.dloss) {
          const float4 dl = J.dloss[pf.x], lt = J.path_radiance[P.path_id[i]], r4 = P.radiance[i];
          const float inv_spp = 1.0f / gmax(J.setting.ssp, 1);
          am.scale = vec3(dl.x, dl.y, dl.z) * inv_spp * (vec3(lt.x, lt.y, lt.z) - vec3(r4.x, r4.y, r4.z));
        }
        hv = sample_volume_scattering<kF, true>(S, o, d, n, vidx, hit ? ch.t : kTMax, &trw, &dist, vw, hs,
                                                &counters->errors, &am);
      } else {
        hv = sample_volume_scattering<kF>(S, o, d, n, vidx, hit ? ch.t : kTMax, &trw, &dist, vw, hs,
                                          &counters->errors);
      }
      const float4 t4 = P.throughput[i];
      vec3 tp(t4.x, t4.y, t4.z);
      tp *= trw;
      P.throughput[i] = make_float4(tp.x, tp.y, tp.z, 0.0f);
      P.sampler[i] = make_uint4((uint32_t)hs.index, (uint32_t)(hs.index >> 32), hs.dim, hs.aux);
      if (hv) {
        volume_hit = true;
        vol_pos = o + d * dist;
        for (int k = 0; k < n; ++k) H.vol_w[(size_t)i * kMaxBoundaryRecord + k] = vw[k];
        if (!hit) {
          ch.inst = kEmpty;
          ch.tri = kEmpty;
          ch.back = 0;
          ch.t = kTMax;
          ch.nearby_count = 0;
        }
      }
      hit = hit || hv;
    }
    if (!hit) {
      // a miss: listed in its own bucket; k_shade adds the background and
      // ends the path (the miss branch of Ray_trace_path_tracing,
      // src/Shading.cu:1855-1864)
      H.ids[i] = make_uint4(kEmpty, kEmpty, 0u, 0u);
      bucket = kBucketMiss;
    } else {
      if (volume_hit) H.bary_t[i] = make_float4(vol_pos.x, vol_pos.y, vol_pos.z, ch.t);
      else H.bary_t[i] = make_float4(ch.b0, ch.b1, ch.b2, ch.t);
      uint32_t nearby_word = (uint32_t)ch.nearby_count;
      if (!(ch.nearby_count == 1 && ch.nearby[0].prim == ch.inst && ch.nearby[0].t == ch.t &&
            ch.nearby[0].back == ch.back)) {
        for (int k = 0; k < ch.nearby_count; ++k)
          H.nearby[(size_t)i * kMaxNearby + k] =
              make_uint4(ch.nearby[k].prim, __float_as_uint(ch.nearby[k].t), (uint32_t)ch.nearby[k].back, 0u);
        nearby_word |= kNearbyExplicit;
      }
      H.ids[i] = make_uint4(ch.inst, ch.tri, (uint32_t)ch.back | (volume_hit ? 2u : 0u), nearby_word);
      bucket = volume_hit ? kBucketVolume : (uint32_t)S.inst_bucket[ch.inst];
    }
  }
  if (j < count) H.bucket[i] = (uint8_t)bucket;
  file_bucket(counters, bucket);
  n_rays += __popc(__ballot_sync(0xFFFFFFFFu, active));
  }
  // counters: one atomic per warp
  uint32_t t_sum = tests, n_sum = nodes;
  for (int off = 16; off > 0; off >>= 1) {
    t_sum += __shfl_down_sync(0xFFFFFFFFu, t_sum, off);
    n_sum += __shfl_down_sync(0xFFFFFFFFu, n_sum, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (n_rays) atomicAdd(&counters->extension_rays, (unsigned long long)n_rays);
    if (t_sum) atomicAdd(&counters->tri_tests, (unsigned long long)t_sum);
    if (n_sum) atomicAdd(&counters->node_visits, (unsigned long long)n_sum);
  }
  if (overflow) atomicOr(&counters->errors, (uint32_t)kDevErrStack);
}

// --------------------------------------------------------------- shade ---

__device__ __forceinline__ int find_record(const RayTransfer& rt, uint32_t prim) {
  for (int r = rt.record_count - 1; r >= 0; --r)
    if (rt.records[r].prim_idx == prim) return r;
  return -1;
}
__device__ __forceinline__ int find_max_priority_record(const RayTransfer& rt) {
  if (rt.record_count == 0) return -1;
  uint32_t mp = rt.records[0].ior_priority;
  int mi = 0;
  for (int r = 1; r < rt.record_count; ++r)
    if (rt.records[r].ior_priority >= mp) {
      mp = rt.records[r].ior_priority;
      mi = r;
    }
  return mi;
}
// RayTransfer::PushRecord / PopRecord (src/Ray.h:179-224).
__device__ __forceinline__ bool push_record(RayTransfer& rt, uint32_t prim, float ior, uint32_t prio, int vol,
                                            uint32_t* errors) {
  if (rt.record_count == kMaxBoundaryRecord) {
    atomicOr(errors, (uint32_t)kDevErrStack);
    return false;
  }
  BoundaryRecord& r = rt.records[rt.record_count];
  r.prim_idx = prim;
  r.ior = ior;
  r.ior_priority = prio;
  r.vol_idx = vol;
  ++rt.record_count;
  if (rt.record_count == 1) {
    rt.max_priority_record_index = 0;
    return true;
  }
  if (prio >= rt.records[rt.max_priority_record_index].ior_priority) rt.max_priority_record_index = rt.record_count - 1;
  return true;
}
__device__ __forceinline__ void pop_record(RayTransfer& rt, int idx) {
  if (rt.record_count == 0 || !(idx >= 0 && idx < rt.record_count)) return;
  for (int k = idx + 1; k < rt.record_count; ++k) rt.records[k - 1] = rt.records[k];
  --rt.record_count;
  rt.max_priority_record_index = find_max_priority_record(rt);
}
// Material::FetchIOR (src/Material.h:262-278); a light material reports ior 1
// and priority 0.
__device__ __forceinline__ float fetch_ior(const Material& m, uint32_t* prio) {
  if (m.material_type == kDefaultMtl) {
    *prio = m.default_mtl.ior_priority;
    return m.default_mtl.ior_n;
  }
  *prio = 0;
  return 1.0f;
}
// BoundaryTransitionBunch (src/ShadingUtilities.cuh:954-990).
__device__ __forceinline__ void boundary_transition(const DeviceScene& S, RayTransfer& rt, const NearbyHit* nb, int n,
                                                    uint32_t* errors) {
  for (int k = 0; k < n; ++k) {
    if (nb[k].back) continue;
    const Instance inst = S.instances[nb[k].prim];
    uint32_t prio;
    const float ior = fetch_ior(S.materials[inst.material_idx], &prio);
    if (find_record(rt, nb[k].prim) == -1) push_record(rt, nb[k].prim, ior, prio, inst.inner_volume_idx, errors);
  }
  for (int k = 0; k < n; ++k) {
    if (!nb[k].back) continue;
    const int r = find_record(rt, nb[k].prim);
    if (r != -1) pop_record(rt, r);
  }
}
// RayTransfer::GetRayIOR / GetExIOR (src/Ray.h:239-258).
__device__ __forceinline__ float ray_ior(const RayTransfer& rt) {
  return rt.record_count > 0 ? rt.records[rt.max_priority_record_index].ior : 1.0f;
}
__device__ __forceinline__ float ex_ior(const RayTransfer& rt, uint32_t hit_prim) {
  uint32_t mp = 0;
  int mi = -1;
  for (int r = 0; r < rt.record_count; ++r) {
    if (rt.records[r].prim_idx == hit_prim) continue;
    if (rt.records[r].ior_priority >= mp) {
      mp = rt.records[r].ior_priority;
      mi = r;
    }
  }
  return mi == -1 ? 1.0f : rt.records[mi].ior;
}

// Closest boundary crossing of a ray (TraceVolume, src/ShadingUtilities.cuh:434-561)
// and the transmittance along a shadow ray through every medium it crosses
// (TraceTr, src/VolumeEval.cuh:420-468). `rt` is the shadow ray's own copy of
// the nested-media stack; `o`/`d`/`tmax` and the last hit are the shadow ray.
template <uint32_t kF, bool kAdj = false>
__device__ __noinline__ vec3 trace_tr(uint32_t scene, TraversalStack& st, vec3 o, vec3 d, float tmax,
                                      uint32_t last_inst, uint32_t last_tri, RayTransfer& rt, PathSampler& hs,
                                      uint32_t* errors, uint32_t* tests, uint32_t* nodes,
                                      const MediumAdj* am = nullptr) {
  const DeviceScene& S = c_scenes[scene];
  if (S.volume_count == 0) return vec3(1.0f);
  vec3 tr(1.0f);
  const float max_d = tmax;
  float traced = kTMin;
  float ray_t = tmax;
  int guard = 0;
  while (traced < max_d) {
    if (++guard > 4 * kMaxRayDepth) {
      atomicOr(errors, (uint32_t)kDevErrIter);
      note_bound(kBoundShadowCrossings, (uint32_t)(guard - 1), o, d, max_d - traced, last_inst, last_tri, &rt);
      break;
    }
    ClosestHit ch;
    const bool hit = trace_closest_impl<(kF & kFeatSpheres) != 0>(scene, st, o, d, ray_t, last_inst, last_tri, true, &ch, tests, nodes);
    if (!hit) {
      tr *= eval_tr<kF, kAdj>(S, o, d, rt, gmax(max_d - traced, 0.0f), hs, errors, am);
      break;
    }
    tr *= eval_tr<kF, kAdj>(S, o, d, rt, ch.t, hs, errors, am);
    traced += ch.t;
    vec3 hp, herr, hng;
    fetch_geometry_normal<kF>(S, ch.inst, ch.tri, vec3(ch.b0, ch.b1, ch.b2), &hp, &herr, &hng);
    boundary_transition(S, rt, ch.nearby, ch.nearby_count, errors);
    o = offset_ray_origin(hp, herr, d, hng);
    d = normalize(d);
    last_inst = ch.inst;
    last_tri = ch.tri;
    ray_t = kTMax;
  }
  return tr;
}

// DistantLight::SampleLi / EvalLi (src/Light.h:343-386).
__device__ __forceinline__ void distant_sample_li(const DeviceScene& S, const DistantLight& L, float u0, float u1, vec3* wi,
                                                  vec3* Li, float* pdf) {
  const mat4& otw = S.transforms[L.transform_idx];
  const float cone = 2.0f * kPi * (1.0f - L.cos_theta_max);
  vec3 cs(0.0f);
  if (cone < 1E-10f) {
    cs = vec3(0.0f, 1.0f, 0.0f);
  } else {
    const float c = (1.0f - u0) + u0 * L.cos_theta_max;
    const float sn = sqrtf(gmax(0.0f, 1.0f - c * c));
    const float phi = u1 * 2.0f * kPi;
    cs = vec3(cosf(phi) * sn, sinf(phi) * sn, c);
    cs = vec3(cs.x, cs.z, cs.y);
  }
  *wi = -normalize(transform_vector(otw, cs));
  *pdf = 1.0f / gmax(cone, 1E-10f);
  *Li = L.light_color * L.intensity;
}
__device__ __forceinline__ vec3 distant_eval_li(const DeviceScene& S, const DistantLight& L, vec3 wi, float* pdf) {
  const vec3 lwi = transform_vector(S.i_transforms[L.transform_idx], wi);
  const float c = -lwi.y;
  if (c < L.cos_theta_max) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  const float cone = 2.0f * kPi * (1.0f - L.cos_theta_max);
  *pdf = 1.0f / cone;
  return L.light_color * L.intensity * (*pdf);
}

// Shading-point context the light estimators share.
struct SurfaceNee {
  vec3 ray_dir, p, p_err, ng;
  uint32_t inst, tri;
  const RayTransfer* rt;
  const NearbyHit* nb;
  int n_nb;
  bool media;  // the render's enable_volume_scattering
  uint32_t slot;  // scene slot
};

// Transmittance of an unoccluded surface shadow ray (the volume part of the
// reference's EvalShapeLight / EvalDistantLight).
template <bool kVol, uint32_t kF, bool kAdj = false>
__device__ __forceinline__ vec3 surface_shadow_tr(const DeviceScene& S, TraversalStack& st, const SurfaceNee& c, vec3 so,
                                                  vec3 ldir, float maxd, bool tb, PathSampler& hs, uint32_t* errors,
                                                  uint32_t* tests, uint32_t* nodes, const MediumAdj* am = nullptr) {
  if (!kVol || !c.media) return vec3(1.0f);
  RayTransfer srt = *c.rt;
  if (tb) boundary_transition(S, srt, c.nb, c.n_nb, errors);
  return trace_tr<kF, kAdj>(c.slot, st, so, normalize(ldir), maxd, c.inst, c.tri, srt, hs, errors, tests, nodes, am);
}

// ------------------------------------------------- path-replay adjoint ---
//
// Gradients of an image loss with respect to each material's diffuse albedo
// (rgb) and roughness (alpha_x and alpha_y together), by path replay: the
// adjoint pass re-traces every path with its own sampler (same directions as
// the forward pass, which recorded each path's radiance), and at every
// surface vertex adds, for each parameter p of the vertex's material,
//   dLoss/dI . ( tp * dNEE/dp  +  L_after * (df/dp) / f )
// where L_after is the radiance the path gathers after the vertex (its
// recorded total minus what it gathered so far). Sampling and MIS weights are
// held fixed (detached), so only BSDF values are differentiated; df/dp is the
// central difference of the closed-form layered BSDF at the vertex's fixed
// directions.

constexpr int kMaxGradMaterials = 64;     // materials with shared-memory gradient slots per block
constexpr float kParamStep = 1e-3f;       // central-difference step of df/dp

struct AdjCtx {
  vec3 weight;                            // dLoss/dI (per path) * throughput: the weight of this vertex's NEE
  float g[kGradParams];                   // accumulated dLoss/dp
  float* grid_grads;                      // dLoss/d(density-grid value), or null
  uint32_t grid_tex;                      // the differentiated grid node
  // Per-lobe derivative data of the vertex's layered BSDF (channel-diagonal
  // in albedo: each channel's albedo moves only that channel of f):
  vec3 lambert_coeff;                     // the diffuse lobe's colour per unit albedo
  vec3 metal_n[2], metal_k[2];            // the conductor's complex IOR at albedo +-h
  float ax[2], ay[2];                     // the microfacet lobes' alpha at roughness +-h
};

// m: the material's parameters as read at the vertex. A parameter a texture
// supplies does not depend on the material's constant: its derivative is 0.
static __device__ __noinline__ void init_adjoint(AdjCtx& a, const LayeredBsdf& B, const DefaultMtl& m) {
  const bool albedo_const = m.diffuse_albedo_tex == kEmpty;
  const float ha = albedo_const ? kParamStep : 0.0f;
  const float hx = m.alpha_x_tex == kEmpty ? kParamStep : 0.0f;
  const float hy = m.alpha_y_tex == kEmpty ? kParamStep : 0.0f;
  a.lambert_coeff = vec3(0.0f);
  for (int i = 0; i < B.count; ++i)
    if (B.lobe[i].role == kRoleDiffuse && albedo_const)
      for (int c = 0; c < 3; ++c)
        a.lambert_coeff[c] = m.diffuse_albedo[c] > 0.0f ? B.lobe[i].albedo[c] / m.diffuse_albedo[c] : 0.0f;
  edge_tint_to_conductor(m.diffuse_albedo + vec3(ha), m.specular_albedo, &a.metal_n[0], &a.metal_k[0]);
  edge_tint_to_conductor(m.diffuse_albedo - vec3(ha), m.specular_albedo, &a.metal_n[1], &a.metal_k[1]);
  a.ax[0] = sqr(gclamp(m.alpha_x + hx, 0.001f, 0.999f));
  a.ax[1] = sqr(gclamp(m.alpha_x - hx, 0.001f, 0.999f));
  a.ay[0] = sqr(gclamp(m.alpha_y + hy, 0.001f, 0.999f));
  a.ay[1] = sqr(gclamp(m.alpha_y - hy, 0.001f, 0.999f));
  for (int k = 0; k < kGradParams; ++k) a.g[k] = 0.0f;
}

// Adds weight . (c * (df/dp) / f) for every parameter at the fixed
// directions (wo, wi) in the frame of B. df/d(albedo): exact for the diffuse
// lobe (linear), a central difference of the conductor's Fresnel term
// through its edge-tint IOR; df/d(roughness): central differences of the
// metal, specular and transmission lobes (the coat has its own roughness).
static __device__ __noinline__ void add_relative_grads(AdjCtx* a, const LayeredBsdf& B, vec3 wo, vec3 wi, vec3 weight,
                                                vec3 c) {
  float pdf;
  const float inv2h = 0.5f / kParamStep;
  vec3 f(0.0f), da(0.0f), dr(0.0f);
  for (int i = 0; i < B.count; ++i) {
    const Lobe& L = B.lobe[i];
    f += lobe_eval(L, wo, wi, &pdf);
    if (L.role == kRoleDiffuse) {
      Lobe u = L;
      u.albedo = a->lambert_coeff;
      da += lobe_eval(u, wo, wi, &pdf);
    }
    if (L.role == kRoleMetal) {
      Lobe hi = L, lo = L;
      hi.nt = a->metal_n[0];
      hi.kt = a->metal_k[0];
      lo.nt = a->metal_n[1];
      lo.kt = a->metal_k[1];
      da += (lobe_eval(hi, wo, wi, &pdf) - lobe_eval(lo, wo, wi, &pdf)) * inv2h;
    }
    if (L.role == kRoleMetal || L.role == kRoleSpecular || L.role == kRoleTransmission) {
      Lobe hi = L, lo = L;
      hi.ax = a->ax[0];
      hi.ay = a->ay[0];
      lo.ax = a->ax[1];
      lo.ay = a->ay[1];
      dr += (lobe_eval(hi, wo, wi, &pdf) - lobe_eval(lo, wo, wi, &pdf)) * inv2h;
    }
  }
  float rough = 0.0f;
  for (int ch = 0; ch < 3; ++ch) {
    if (!(f[ch] > 0.0f)) continue;
    const float s = weight[ch] * c[ch] / f[ch];
    a->g[ch] += s * da[ch];
    rough += s * dr[ch];
  }
  a->g[3] += rough;
}

// Where a surface shadow ray goes when shadow rays are deferred: the queue
// k_connect traces, the pixel it lights and the path's weight on it
// (throughput / spp).
struct ShadowEmit {
  ShadowQueue q;
  uint32_t* count;
  uint32_t* errors;
  uint32_t pixel;
  uint32_t job;
  uint32_t path;
  vec3 weight;
};

// Queues one shadow ray with its contribution (warp-aggregated slot claim
// over the lanes that reach this point together).
__device__ __forceinline__ void emit_shadow_ray(const ShadowEmit& em, vec3 o, vec3 d, float maxd, vec3 contribution) {
  cg::coalesced_group g = cg::coalesced_threads();
  uint32_t base = 0;
  if (g.thread_rank() == 0) base = atomicAdd(em.count, g.size());
  const uint32_t slot = g.shfl(base, 0) + g.thread_rank();
  if (slot >= em.q.capacity) {
    atomicOr(em.errors, kDevErrQueue);
    return;
  }
  const vec3 w = em.weight * contribution;
  em.q.o[slot] = make_float4(o.x, o.y, o.z, maxd);
  em.q.d[slot] = make_float4(d.x, d.y, d.z, __uint_as_float(em.pixel));
  em.q.c[slot] = make_float4(w.x, w.y, w.z, __uint_as_float(em.job));
  em.q.path[slot] = em.path;
}

// One next-event shadow ray of a surface vertex toward a light, with MIS
// weight `mis`, clamped BSDF value fc and radiance Lc; the light-selection
// pdf enters as (x * mul) / div, the form each estimator uses. Traced here
// (direct += its unoccluded contribution, times the media transmittance)
// or, with kDefer, queued for k_connect.
template <bool kVol, bool kDefer, uint32_t kF>
__device__ __forceinline__ void nee_shadow_ray(const DeviceScene& S, TraversalStack& st, const SurfaceNee& c,
                                               const ShadowEmit& em, vec3 so, vec3 ldir, float maxd, bool tb,
                                               float mis, vec3 fc, vec3 Lc, float mul, float div, vec3* direct,
                                               PathSampler& hs, uint32_t* shadow_rays, uint32_t* tests,
                                               uint32_t* nodes, uint32_t* errors, AdjCtx* adj = nullptr,
                                               const LayeredBsdf* B = nullptr) {
  ++*shadow_rays;
  if (kDefer) {
    emit_shadow_ray(em, so, normalize(ldir), maxd, ((mis * vec3(1.0f) * fc * Lc) * mul) / div);
    return;
  }
  if (!trace_occluded_impl<(kF & kFeatSpheres) != 0>(c.slot, st, so, normalize(ldir), maxd, tests, nodes)) {
    const PathSampler hs0 = hs;
    const vec3 tr = surface_shadow_tr<kVol, kF>(S, st, c, so, ldir, maxd, tb, hs, errors, tests, nodes);
    *direct += mis * tr * fc * Lc;
    if constexpr (kVol) {
      if (adj && adj->grid_grads && c.media) {
        // the transmittance's density-grid terms: replay its tracking with the
        // same samples, weighted by this ray's share of dLoss
        const MediumAdj am{adj->weight * (mul / div) * (mis * tr * fc * Lc), adj->grid_tex, adj->grid_grads};
        if (max_component(vabs(am.scale)) > 0.0f) {
          PathSampler h2 = hs0;
          surface_shadow_tr<kVol, kF, true>(S, st, c, so, ldir, maxd, tb, h2, errors, tests, nodes, &am);
        }
      }
    }
    if (adj) {
      // d(direct)/dp = mis * tr * fc * (df/dp)/f * Lc, scaled like the estimator
      const vec3 wo = B->to_local(-c.ray_dir), wi = B->to_local(ldir);
      add_relative_grads(adj, *B, wo, wi, adj->weight * (mul / div), mis * tr * fc * Lc);
    }
  }
}

// EvalShapeLight (src/Shading.cu:294-417).
template <bool kVol, bool kDefer, uint32_t kF>
__device__ __forceinline__ vec3 eval_shape_light(const DeviceScene& S, TraversalStack& st, const LayeredBsdf& B,
                                                 const SurfaceNee& c, const ShadowEmit& em, PathSampler& hs,
                                                 uint32_t* shadow_rays, uint32_t* tests, uint32_t* nodes,
                                                 uint32_t* errors, AdjCtx* adj = nullptr) {
  if (S.shape_light_count == 0) return vec3(0.0f);
  vec3 direct(0.0f);
  const vec3 wo = B.to_local(-c.ray_dir);
  float select_pdf = 0.0f;
  const int li = sample_light_power(S, sample1d(hs, S), &select_pdf);
  const ShapeLight L = S.shape_lights[li];
  const LightTri lt = load_light_tri<kF>(S, L);
  {
    float u0, u1;
    sample2d(hs, S, &u0, &u1);
    vec3 ldir(0.0f), lpos(0.0f), lerr(0.0f), lng(0.0f), Li(0.0f);
    float lpdf = 0.0f;
    const bool valid = light_sample_li<kF>(lt, L.area, c.p, u0, u1, &ldir, &lpos, &lerr, &lng, &Li, &lpdf);
    const vec3 lwi = B.to_local(ldir);
    float wpdf = 0.0f;
    const vec3 f = bsdf_eval(B, wo, lwi, &wpdf);
    if (max_component(f) > kMinColorEps && valid) {
      const vec3 so = offset_ray_origin(c.p, c.p_err, ldir, c.ng);
      const float maxd = length(offset_ray_origin(lpos, lerr, -ldir, lng) - c.p) * kShadowRayClamp;
      const bool tb = dot(-c.ray_dir, c.ng) * dot(ldir, c.ng) < 0.0f;
      const bool invalid = (!same_hemisphere(wo, lwi) && !tb) || (same_hemisphere(wo, lwi) && tb);
      if (!invalid)
        nee_shadow_ray<kVol, kDefer, kF>(S, st, c, em, so, ldir, maxd, tb, power_heuristic(lpdf, wpdf),
                                     vmin(f, vec3(kMaxColorClamp)), vmin(Li, vec3(kMaxColorClamp)),
                                     safe_rcp(select_pdf), 1.0f, &direct, hs, shadow_rays, tests, nodes, errors, adj, &B);
    }
  }
  {
    float u0, u1, u2;
    sample3d(hs, S, &u0, &u1, &u2);
    vec3 bw, bwi;
    float bpdf = 0.0f;
    if (bsdf_sample(B, wo, &bw, &bwi, &bpdf, u0, u1, u2)) {
      const vec3 ldir = B.to_world(bwi);
      vec3 lpos(0.0f), lerr(0.0f), lng(0.0f);
      float wpdf = 0.0f;
      const vec3 Li = light_eval_li<kF>(lt, L.area, c.p, ldir, &lpos, &lerr, &lng, &wpdf);
      if (max_component(Li) > kMinColorEps) {
        const vec3 so = offset_ray_origin(c.p, c.p_err, ldir, c.ng);
        const float maxd = length(offset_ray_origin(lpos, lerr, -ldir, lng) - c.p) * kShadowRayClamp;
        const bool tb = dot(-c.ray_dir, c.ng) * dot(ldir, c.ng) < 0.0f;
        const bool invalid = (!same_hemisphere(wo, bwi) && !tb) || (same_hemisphere(wo, bwi) && tb);
        if (!invalid)
          nee_shadow_ray<kVol, kDefer, kF>(S, st, c, em, so, ldir, maxd, tb, power_heuristic(bpdf, wpdf),
                                       vmin(bw, vec3(kMaxColorClamp)), vmin(Li, vec3(kMaxColorClamp)),
                                       safe_rcp(select_pdf), 1.0f, &direct, hs, shadow_rays, tests, nodes, errors, adj, &B);
      }
    }
  }
  return direct * safe_rcp(select_pdf);
}

// EvalDistantLight (src/Shading.cu:83-198).
template <bool kVol, bool kDefer, uint32_t kF>
__device__ __forceinline__ vec3 eval_distant_light(const DeviceScene& S, TraversalStack& st, const LayeredBsdf& B,
                                                   const SurfaceNee& c, const ShadowEmit& em, PathSampler& hs,
                                                   uint32_t* shadow_rays, uint32_t* tests, uint32_t* nodes,
                                                   uint32_t* errors, AdjCtx* adj = nullptr) {
  if (S.distant_light_count == 0) return vec3(0.0f);
  vec3 direct(0.0f);
  const vec3 wo = B.to_local(-c.ray_dir);
  const float select_pdf = 1.0f / float(S.distant_light_count);
  const int li = gmax(gmin((int)(sample1d(hs, S) * S.distant_light_count), (int)S.distant_light_count - 1), 0);
  const DistantLight L = S.distant_lights[li];
  {
    float u0, u1;
    sample2d(hs, S, &u0, &u1);
    vec3 ldir(0.0f), Li(0.0f);
    float lpdf = 0.0f;
    distant_sample_li(S, L, u0, u1, &ldir, &Li, &lpdf);
    const vec3 lwi = B.to_local(ldir);
    float wpdf = 0.0f;
    const vec3 f = bsdf_eval(B, wo, lwi, &wpdf);
    if (max_component(f) > kMinColorEps) {
      const vec3 so = offset_ray_origin(c.p, c.p_err, ldir, c.ng);
      const bool tb = dot(-c.ray_dir, c.ng) * dot(ldir, c.ng) < 0.0f;
      const bool invalid = (!same_hemisphere(wo, lwi) && !tb) || (same_hemisphere(wo, lwi) && tb);
      if (!invalid)
        nee_shadow_ray<kVol, kDefer, kF>(S, st, c, em, so, ldir, kTMax, tb, power_heuristic(lpdf, wpdf),
                                     vmin(f, vec3(kMaxColorClamp)), vmin(Li, vec3(kMaxColorClamp)), 1.0f,
                                     select_pdf, &direct, hs, shadow_rays, tests, nodes, errors, adj, &B);
    }
  }
  {
    float u0, u1, u2;
    sample3d(hs, S, &u0, &u1, &u2);
    vec3 bw, bwi;
    float bpdf = 0.0f;
    if (bsdf_sample(B, wo, &bw, &bwi, &bpdf, u0, u1, u2)) {
      const vec3 ldir = B.to_world(bwi);
      float wpdf = 0.0f;
      const vec3 Li = distant_eval_li(S, L, ldir, &wpdf);
      if (max_component(Li) > kMinColorEps) {
        const vec3 so = offset_ray_origin(c.p, c.p_err, ldir, c.ng);
        const bool tb = dot(-c.ray_dir, c.ng) * dot(ldir, c.ng) < 0.0f;
        const bool invalid = (!same_hemisphere(wo, bwi) && !tb) || (same_hemisphere(wo, bwi) && tb);
        if (!invalid)
          nee_shadow_ray<kVol, kDefer, kF>(S, st, c, em, so, ldir, kTMax, tb, power_heuristic(bpdf, wpdf),
                                       vmin(bw, vec3(kMaxColorClamp)), vmin(Li, vec3(kMaxColorClamp)), 1.0f,
                                       select_pdf, &direct, hs, shadow_rays, tests, nodes, errors, adj, &B);
      }
    }
  }
  return direct / select_pdf;
}

// Density-grid terms of one volume shadow ray's transmittance (the adjoint
// pass): its tracking replayed from the sampler state `hs` it started from,
// weighted by av->scale (dLoss/dI times throughput) times the ray's
// contribution to the estimate (contrib / select_pdf).
template <uint32_t kF>
__device__ __noinline__ void volume_shadow_grad(uint32_t slot, TraversalStack& st, vec3 pos, vec3 dir, float maxd,
                                                const RayTransfer& rt, PathSampler hs, vec3 contrib, float select_pdf,
                                                const MediumAdj* av, uint32_t* errors, uint32_t* tests,
                                                uint32_t* nodes) {
  if (!av || !av->grads || !(select_pdf > 0.0f)) return;
  const MediumAdj am{av->scale * contrib / select_pdf, av->grid_tex, av->grads};
  if (!(max_component(vabs(am.scale)) > 0.0f)) return;
  RayTransfer srt = rt;
  trace_tr<kF, true>(slot, st, pos, dir, maxd, kEmpty, kEmpty, srt, hs, errors, tests, nodes, &am);
}

// EvalVolumeShapeLight / EvalVolumeDistantLight (src/Shading.cu:202-291, 419-513):
// next-event estimation at a scattering point inside the media. kAdj: the
// adjoint pass, which also adds each shadow ray's density-grid terms (av).
template <uint32_t kF, bool kAdj = false>
__device__ __noinline__ vec3 eval_volume_lights(uint32_t slot, TraversalStack& st, bool distant, int n,
                                                const float* gs, const float* vw, vec3 ray_dir, const RayTransfer& rt,
                                                vec3 pos, PathSampler& hs, uint32_t* shadow_rays, uint32_t* tests,
                                                uint32_t* nodes, uint32_t* errors, const MediumAdj* av = nullptr) {
  const DeviceScene& S = c_scenes[slot];
  vec3 direct(0.0f);
  if (distant) {
    if (S.distant_light_count == 0 || n == 0) return vec3(0.0f);
    const float select_pdf = 1.0f / float(S.distant_light_count);
    const int li = gmax(gmin((int)(sample1d(hs, S) * S.distant_light_count), (int)S.distant_light_count - 1), 0);
    const DistantLight L = S.distant_lights[li];
    {
      float u0, u1;
      sample2d(hs, S, &u0, &u1);
      vec3 ldir(0.0f), Li(0.0f);
      float lpdf = 0.0f;
      distant_sample_li(S, L, u0, u1, &ldir, &Li, &lpdf);
      float wpdf = 0.0f;
      const float pw = eval_mixed_phases(vw, gs, n, -ray_dir, ldir, &wpdf);
      if (pw > kMinColorEps) {
        ++*shadow_rays;
        if (!trace_occluded_impl<(kF & kFeatSpheres) != 0>(slot, st, pos, normalize(ldir), kTMax, tests, nodes)) {
          RayTransfer srt = rt;
          const PathSampler hs0 = hs;
          const vec3 tr = trace_tr<kF>(slot, st, pos, normalize(ldir), kTMax, kEmpty, kEmpty, srt, hs, errors, tests, nodes);
          const float mis = power_heuristic(lpdf, wpdf);
          const vec3 contrib = mis * tr * gmin(pw, kMaxColorClamp) * vmin(Li, vec3(kMaxColorClamp));
          direct += contrib;
          if constexpr (kAdj)
            volume_shadow_grad<kF>(slot, st, pos, normalize(ldir), kTMax, rt, hs0, contrib, select_pdf, av, errors,
                                   tests, nodes);
        }
      }
    }
    {
      float u0, u1;
      sample2d(hs, S, &u0, &u1);
      vec3 pwi;
      float pspdf = 0.0f, pw = 0.0f;
      if (sample_mixed_phases(vw, gs, n, u0, u1, -ray_dir, &pw, &pwi, &pspdf)) {
        float wpdf = 0.0f;
        const vec3 Li = distant_eval_li(S, L, pwi, &wpdf);
        if (max_component(Li) > kMinColorEps) {
          ++*shadow_rays;
          if (!trace_occluded_impl<(kF & kFeatSpheres) != 0>(slot, st, pos, normalize(pwi), kTMax, tests, nodes)) {
            RayTransfer srt = rt;
            const PathSampler hs0 = hs;
            const vec3 tr = trace_tr<kF>(slot, st, pos, normalize(pwi), kTMax, kEmpty, kEmpty, srt, hs, errors, tests, nodes);
            const float mis = power_heuristic(pspdf, wpdf);
            const vec3 contrib = mis * tr * gmin(pw, kMaxColorClamp) * vmin(Li, vec3(kMaxColorClamp));
            direct += contrib;
            if constexpr (kAdj)
              volume_shadow_grad<kF>(slot, st, pos, normalize(pwi), kTMax, rt, hs0, contrib, select_pdf, av, errors,
                                     tests, nodes);
          }
        }
      }
    }
    return direct / select_pdf;
  }
  if (S.shape_light_count == 0 || n == 0) return vec3(0.0f);
  float select_pdf = 0.0f;
  const int li = sample_light_power(S, sample1d(hs, S), &select_pdf);
  const ShapeLight L = S.shape_lights[li];
  const LightTri lt = load_light_tri<kF>(S, L);
  {
    float u0, u1;
    sample2d(hs, S, &u0, &u1);
    vec3 ldir(0.0f), lpos(0.0f), lerr(0.0f), lng(0.0f), Li(0.0f);
    float lpdf = 0.0f;
    const bool valid = light_sample_li<kF>(lt, L.area, pos, u0, u1, &ldir, &lpos, &lerr, &lng, &Li, &lpdf);
    float wpdf = 0.0f;
    const float pw = eval_mixed_phases(vw, gs, n, -ray_dir, ldir, &wpdf);
    if (pw > kMinColorEps && valid) {
      const float maxd = length(offset_ray_origin(lpos, lerr, -ldir, lng) - pos) * kShadowRayClamp;
      ++*shadow_rays;
      if (!trace_occluded_impl<(kF & kFeatSpheres) != 0>(slot, st, pos, normalize(ldir), maxd, tests, nodes)) {
        RayTransfer srt = rt;
        const PathSampler hs0 = hs;
        const vec3 tr = trace_tr<kF>(slot, st, pos, normalize(ldir), maxd, kEmpty, kEmpty, srt, hs, errors, tests, nodes);
        const float mis = power_heuristic(lpdf, wpdf);
        const vec3 contrib = mis * tr * gmin(pw, kMaxColorClamp) * vmin(Li, vec3(kMaxColorClamp));
        direct += contrib;
        if constexpr (kAdj)
          volume_shadow_grad<kF>(slot, st, pos, normalize(ldir), maxd, rt, hs0, contrib, select_pdf, av, errors,
                                 tests, nodes);
      }
    }
  }
  {
    float u0, u1;
    sample2d(hs, S, &u0, &u1);
    vec3 pwi;
    float pspdf = 0.0f, pw = 0.0f;
    if (sample_mixed_phases(vw, gs, n, u0, u1, -ray_dir, &pw, &pwi, &pspdf)) {
      vec3 lpos(0.0f), lerr(0.0f), lng(0.0f);
      float wpdf = 0.0f;
      const vec3 Li = light_eval_li<kF>(lt, L.area, pos, pwi, &lpos, &lerr, &lng, &wpdf);
      if (max_component(Li) > kMinColorEps) {
        const float maxd = length(offset_ray_origin(lpos, lerr, -pwi, lng) - pos) * kShadowRayClamp;
        ++*shadow_rays;
        if (!trace_occluded_impl<(kF & kFeatSpheres) != 0>(slot, st, pos, normalize(pwi), maxd, tests, nodes)) {
          RayTransfer srt = rt;
          const PathSampler hs0 = hs;
          const vec3 tr = trace_tr<kF>(slot, st, pos, normalize(pwi), maxd, kEmpty, kEmpty, srt, hs, errors, tests, nodes);
          const float mis = power_heuristic(pspdf, wpdf);
          const vec3 contrib = mis * tr * gmin(pw, kMaxColorClamp) * vmin(Li, vec3(kMaxColorClamp));
          direct += contrib;
          if constexpr (kAdj)
            volume_shadow_grad<kF>(slot, st, pos, normalize(pwi), maxd, rt, hs0, contrib, select_pdf, av, errors,
                                   tests, nodes);
        }
      }
    }
  }
  return select_pdf > 0.0f ? (direct / select_pdf) : vec3(0.0f);
}

// kDefer (surfaces only, no indirect clamp): next-event shadow rays are queued
// for k_connect instead of traced here, which keeps traversal out of this
// kernel.
//
// kAdj (surfaces, inline shadow rays): the path-replay adjoint pass. Paths
// are shaded exactly as in the forward pass, nothing is added to the image,
// and each material vertex adds its terms of dLoss/dParam (see AdjCtx) to
// `grads` (per-block sums in shared memory, then one atomic per touched slot).
//
// Resident blocks per SM the register allocation is held to (measured on one
// box, CUDA-event A/B): forward surfaces four (128 registers, a few spills;
// the 1080p 64-spp bench frame 220.4 -> 217.4 ms against three at 168);
// forward media without the texture nodes three (168 registers, 1-2 KB of
// spills; the 1280x720 32-spp volumetric frame 925 -> 892 ms against two at
// 255, four 903 ms); forward media with the texture nodes two (255
// registers; three spill more and were slower, 892 -> 915 ms on the
// textured frame, and again with Perlin noise out of line, 745 -> 783 ms);
// the surface adjoint three (backward pass of 16 views
// 512² 16 spp 505 -> 487 ms); the media adjoint two.
template <bool kVol, bool kDefer, bool kAdj, uint32_t kF>
constexpr int shade_blocks_per_sm() {
  if (kAdj) return kVol ? 1 : 3;
  if (kVol) return (kF & kFeatTextures) ? 1 : 3;
  return 4;
}

template <bool kVol, bool kDefer, bool kAdj, uint32_t kF>
__global__ void __launch_bounds__(kTraceBlock, shade_blocks_per_sm<kVol, kDefer, kAdj, kF>()) k_shade(PathPool P, const WaveControl* __restrict__ ctl, HitPool H,
                                                       PathPool Q, const JobDesc* __restrict__ jobs,
                                                       WaveCounters* counters, ShadowQueue shadow_q,
                                                       float* grads = nullptr, uint32_t grad_materials = 0,
                                                       float* grid_grads = nullptr, uint32_t grid_tex = kEmpty) {
  static_assert(!(kVol && kDefer), "volume transmittance needs the path's sampler: shadow rays are traced inline");
  static_assert(!(kAdj && kDefer), "the adjoint pass traces its shadow rays inline");
  float* s_grad = nullptr;
  const uint32_t n_slots = min(grad_materials, (uint32_t)kMaxGradMaterials) * kGradParams;
  if constexpr (kAdj) {
    __shared__ float s_grad_buf[kMaxGradMaterials * kGradParams];
    s_grad = s_grad_buf;
    for (uint32_t k = threadIdx.x; k < n_slots; k += blockDim.x) s_grad[k] = 0.0f;
    __syncthreads();
  }
  const bool listed = H.order != nullptr;
  const uint32_t count = listed ? min(ctl->count, counters->hit_count) : ctl->count;
  uint32_t shadow_rays = 0, tests = 0, nodes = 0;
  bool overflow = false;
  for (uint32_t warp_base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); warp_base < count;
       warp_base += gridDim.x * blockDim.x) {
  // The path slot this lane shades: the t-th listed hit, or (hits not listed
  // by bucket) slot t itself when it holds a live path.
  const uint32_t t_idx = warp_base + (threadIdx.x & 31u);
  bool active = t_idx < count;
  const uint32_t i = active ? (listed ? H.order[t_idx] : t_idx) : 0u;
  bool alive = false;  // continues into Q
  const uint2 pf = active ? P.pixel_flags[i] : make_uint2(kEmpty, kFlagDead);
  if (pf.y & kFlagDead) active = false;  // a miss (already accumulated) or an empty slot

  vec3 new_o, new_d, tp, rad;
  uint32_t new_flags = 0, new_last_inst = kEmpty, new_last_tri = kEmpty;
  PathSampler hs{0, 0u, 0u};
  RayTransfer rt;
  rt.record_count = 0;
  rt.max_priority_record_index = -1;

  if (active) {
    const uint32_t job = pf.y >> kFlagJobShift;
    const JobDesc& J = jobs[job];
    const uint32_t slot = J.scene_slot;
    const DeviceScene& S = c_scenes[slot];
    const RenderSetting& rs = J.setting;
    uint32_t* errors = &counters->errors;
    const float4 o4 = P.ray_o[i], d4 = P.ray_d[i], t4 = P.throughput[i], r4 = P.radiance[i];
    const vec3 rd(d4.x, d4.y, d4.z);
    (void)o4;
    tp = vec3(t4.x, t4.y, t4.z);
    rad = vec3(r4.x, r4.y, r4.z);
    const uint4 s4 = P.sampler[i];
    hs.index = (uint64_t)s4.x | ((uint64_t)s4.y << 32);
    hs.dim = s4.z;
    hs.aux = s4.w;
    int depth = (int)(pf.y & kFlagDepthMask);
    bool never_scatter = (pf.y & kFlagNeverScatter) != 0;
    const uint32_t sample_bits = pf.y & ~(kFlagDepthMask | kFlagNeverScatter | kFlagCameraRay | kFlagDead);  // job
    const int n_rec = P.transfer_count[i];
    if (n_rec > 0) rt = P.transfer[i];
    const float4 bt = H.bary_t[i];
    const uint4 ids = H.ids[i];
    const vec3 bary(bt.x, bt.y, bt.z);
    const uint32_t inst_idx = ids.x, tri = ids.y;
    const int hit_back = (int)(ids.z & 1u);
    const bool volume_hit = kVol && (ids.z & 2u);
    const float inv_spp = 1.0f / gmax(rs.ssp, 1);
    TraversalStack st;
    if constexpr (!kDefer) {
      YM_TRAVERSAL_SHARED(s_stack);
      st.bind(s_stack_entries, s_stack_t);
    } else {
      st.sp = 0;
      st.overflow = false;
    }

    if (inst_idx == kEmpty && !volume_hit) {
      // a miss (Ray_trace_path_tracing, src/Shading.cu:1855-1864): the
      // background when the environment light is on, then the path ends
      if (rs.enable_env_light) rad += indirect_clamp(rs, tp * background(rd), depth);
      end_path<kAdj>(J, pf.x, P.path_id[i], rad, inv_spp);
    } else if (volume_hit) {
      // Ray_shading_path_tracing volume branch (src/Shading.cu:2066-2126).
      float vw[kMaxBoundaryRecord], gs[kMaxBoundaryRecord];
      int vidx[kMaxBoundaryRecord];
      const int n = current_volumes(rt, S.volume_count, vidx);
      for (int k = 0; k < n; ++k) {
        gs[k] = S.volumes[vidx[k]].g;
        vw[k] = H.vol_w[(size_t)i * kMaxBoundaryRecord + k];
      }
      const vec3 pos = bary;
      MediumAdj av{vec3(0.0f), grid_tex, grid_grads};
      if constexpr (kAdj) {
        const float4 dl = J.dloss[pf.x];
        av.scale = vec3(dl.x, dl.y, dl.z) * inv_spp * tp;  // dLoss/d(this vertex's light), before 1/select_pdf
      }
      if (rs.enable_distant_light)
        rad += indirect_clamp(rs, tp * eval_volume_lights<kF, kAdj>(slot, st, true, n, gs, vw, rd, rt, pos, hs,
                                                                    &shadow_rays, &tests, &nodes, errors,
                                                                    kAdj ? &av : nullptr), depth);
      if (rs.enable_shape_light)
        rad += indirect_clamp(rs, tp * eval_volume_lights<kF, kAdj>(slot, st, false, n, gs, vw, rd, rt, pos, hs,
                                                                    &shadow_rays, &tests, &nodes, errors,
                                                                    kAdj ? &av : nullptr), depth);
      vec3 wi;
      float pdf = 0.0f, pw = 0.0f;
      float u0, u1;
      sample2d(hs, S, &u0, &u1);
      bool terminate = !sample_mixed_phases(vw, gs, n, u0, u1, -rd, &pw, &wi, &pdf);
      if (!terminate) {
        tp *= pw;
        float rr = gmax(tp.x, gmax(tp.y, tp.z));
        rr = gmin(rr, 1.0f);
        if (depth + 1 > rs.ray_depth) {
          if (rs.enable_russian_roulette && sample1d(hs, S) < rr) tp /= gmax(rr, kMinColorEps);
          else terminate = true;
        }
      }
      if (!terminate) {
        new_o = pos;
        new_d = normalize(wi);
        depth += 1;
        if (depth > kMaxRayDepth) {
          terminate = true;
        } else {
          new_flags = flags_pack(depth, false, false, 0) | sample_bits;
          new_last_inst = kEmpty;
          new_last_tri = kEmpty;
          alive = true;
        }
      }
      if (terminate) end_path<kAdj>(J, pf.x, P.path_id[i], rad, inv_spp);
    } else {
      NearbyHit nb[kMaxNearby];
      const int n_nb = (int)(ids.w & 0xFFu);
      if (ids.w & kNearbyExplicit) {
        for (int k = 0; k < n_nb; ++k) {
          const uint4 e = H.nearby[(size_t)i * kMaxNearby + k];
          nb[k] = NearbyHit{e.x, __uint_as_float(e.y), (int)e.z};
        }
      } else {
        nb[0] = NearbyHit{inst_idx, bt.w, hit_back};
      }
      const SurfacePoint sp = fetch_surface<kF>(S, inst_idx, tri, bary);
      const Instance inst = S.instances[inst_idx];
      bool done = false;
      if (!(inst.material_idx < S.material_count)) {
        end_path<kAdj>(J, pf.x, P.path_id[i], rad, inv_spp);
        done = true;
      }
      const Material& mat = S.materials[done ? 0 : inst.material_idx];
      uint32_t prio = 0;
      if (!done) fetch_ior(mat, &prio);
      if (!done && rt.record_count != 0 && prio < rt.records[rt.max_priority_record_index].ior_priority) {
        // lower-priority boundary: pass straight through, no depth consumed
        boundary_transition(S, rt, nb, n_nb, errors);
        new_o = offset_ray_origin(sp.p, sp.p_err, rd, sp.ng);
        new_d = normalize(rd);
        new_flags = flags_pack(depth, never_scatter, false, 0) | sample_bits;
        new_last_inst = inst_idx;
        new_last_tri = tri;
        alive = true;
        done = true;
      }
      if (!done && inst.treat_as_boundary) {
        boundary_transition(S, rt, nb, n_nb, errors);
        new_o = offset_ray_origin(sp.p, sp.p_err, rd, sp.ng);
        new_d = normalize(rd);
        new_flags = flags_pack(depth, never_scatter, false, 0) | sample_bits;
        new_last_inst = inst_idx;
        new_last_tri = tri;
        alive = true;
        done = true;
      }
      if (!done && mat.material_type == kLightMtl) {
        if (never_scatter) rad += indirect_clamp(rs, tp * mat.light_mtl.light_color * mat.light_mtl.intensity, depth);
        end_path<kAdj>(J, pf.x, P.path_id[i], rad, inv_spp);
        done = true;
      }
      if (!done) {
        LayeredBsdf B;
        const DefaultMtl* mp = &mat.default_mtl;
        DefaultMtl mt;
        if constexpr ((kF & kFeatTextures) != 0) {
          if (material_textured(mat.default_mtl)) {
            // textured parameters, normal or bump mapping: read at the hit
            mt = mat.default_mtl;
            const TexCoord tc{sp.u, sp.v, sp.p_obj};
            init_shading_frame_mapped(B, mt, hit_back, rd, sp, S.i_transforms[inst.transform_idx], S, tc, errors);
            resolve_material_textures(mt, S.textures, tc, errors);
            mp = &mt;
          } else {
            init_shading_frame(B, hit_back, rd, sp.ng, sp.ns, sp.dpdu, sp.dpdv);
          }
        } else {
          init_shading_frame(B, hit_back, rd, sp.ng, sp.ns, sp.dpdu, sp.dpdv);
        }
        init_layered_lobes(B, *mp, rd, hit_back, ray_ior(rt), ex_ior(rt, inst_idx));
        const SurfaceNee nc{rd, sp.p, sp.p_err, sp.ng, inst_idx, tri, &rt, nb, n_nb, rs.enable_volume_scattering != 0,
                            slot};
        const ShadowEmit em{shadow_q, &counters->shadow_count, errors, pf.x, job, P.path_id[i], tp * inv_spp};
        AdjCtx adj_ctx;
        AdjCtx* adj = nullptr;
        vec3 delta(0.0f), l_total(0.0f);
        if constexpr (kAdj) {
          const float4 dl = J.dloss[pf.x];
          const float4 lt = J.path_radiance[P.path_id[i]];
          delta = vec3(dl.x, dl.y, dl.z) * inv_spp;  // dLoss/d(this path's radiance)
          l_total = vec3(lt.x, lt.y, lt.z);
          init_adjoint(adj_ctx, B, *mp);
          adj_ctx.weight = delta * tp;
          adj_ctx.grid_grads = grid_grads;
          adj_ctx.grid_tex = grid_tex;
          adj = &adj_ctx;
        }
        if (rs.enable_distant_light)
          rad += indirect_clamp(
              rs, tp * eval_distant_light<kVol, kDefer, kF>(S, st, B, nc, em, hs, &shadow_rays, &tests, &nodes, errors, adj),
              depth);
        if (rs.enable_shape_light)
          rad += indirect_clamp(
              rs, tp * eval_shape_light<kVol, kDefer, kF>(S, st, B, nc, em, hs, &shadow_rays, &tests, &nodes, errors, adj),
              depth);
        const vec3 wo = B.to_local(-rd);
        vec3 w, wi;
        float pdf = 0.0f;
        float u0, u1, u2;
        sample3d(hs, S, &u0, &u1, &u2);
        const bool valid = bsdf_sample(B, wo, &w, &wi, &pdf, u0, u1, u2);
        if constexpr (kAdj) {
          // the radiance gathered after this vertex, through the sampled BSDF value
          if (valid) add_relative_grads(&adj_ctx, B, wo, wi, delta, l_total - rad);
          const uint32_t m = inst.material_idx;
          for (int k = 0; k < kGradParams; ++k) {
            if (adj_ctx.g[k] == 0.0f) continue;
            if (m * kGradParams + k < n_slots) atomicAdd(&s_grad[m * kGradParams + k], adj_ctx.g[k]);
            else if (m < grad_materials) atomicAdd(&grads[m * kGradParams + k], adj_ctx.g[k]);
          }
        }
        if (!valid) {
          end_path<kAdj>(J, pf.x, P.path_id[i], rad, inv_spp);
        } else {
          tp *= w;
          float rr = gmax(tp.x, gmax(tp.y, tp.z));
          rr = gmin(rr, 1.0f);
          bool terminate = false;
          if (depth + 1 > rs.ray_depth) {
            if (rs.enable_russian_roulette && sample1d(hs, S) < rr) tp /= gmax(rr, kMinColorEps);
            else terminate = true;
          }
          if (!terminate) {
            const vec3 nd = B.to_world(wi);
            const bool tb = dot(-rd, sp.ng) * dot(nd, sp.ng) < 0.0f;
            const bool invalid = (!same_hemisphere(wo, wi) && !tb) || (same_hemisphere(wo, wi) && tb);
            if (invalid) {
              terminate = true;
            } else {
              if (tb) boundary_transition(S, rt, nb, n_nb, errors);
              new_o = offset_ray_origin(sp.p, sp.p_err, nd, sp.ng);
              new_d = normalize(nd);
              never_scatter = false;
              depth += 1;
              if (depth > kMaxRayDepth) {
                terminate = true;
              } else {
                new_flags = flags_pack(depth, false, false, 0) | sample_bits;
                new_last_inst = inst_idx;
                new_last_tri = tri;
                alive = true;
              }
            }
          }
          if (terminate) end_path<kAdj>(J, pf.x, P.path_id[i], rad, inv_spp);
        }
      }
    }
    overflow = overflow || st.overflow;
  }
  const uint32_t slot = warp_append(&counters->next_count, alive);
  if (alive) {
    if (slot < Q.capacity) {
      store_path(Q, slot, new_o, new_d, tp, rad, pf.x, new_flags, new_last_inst, new_last_tri, hs, P.path_id[i]);
      Q.transfer_count[slot] = (uint8_t)rt.record_count;
      if (rt.record_count > 0) Q.transfer[slot] = rt;
    } else {
      atomicOr(&counters->errors, (uint32_t)kDevErrQueue);
    }
  }
  }
  if (overflow) atomicOr(&counters->errors, (uint32_t)kDevErrStack);
  uint32_t s_sum = shadow_rays, t_sum = tests, n_sum = nodes;
  for (int off = 16; off > 0; off >>= 1) {
    s_sum += __shfl_down_sync(0xFFFFFFFFu, s_sum, off);
    t_sum += __shfl_down_sync(0xFFFFFFFFu, t_sum, off);
    n_sum += __shfl_down_sync(0xFFFFFFFFu, n_sum, off);
  }
  if ((threadIdx.x & 31) == 0) {
    if (s_sum) atomicAdd(&counters->shadow_rays, (unsigned long long)s_sum);
    if (t_sum) atomicAdd(&counters->shadow_tri_tests, (unsigned long long)t_sum);
    if (n_sum) atomicAdd(&counters->shadow_node_visits, (unsigned long long)n_sum);
  }
  if constexpr (kAdj) {
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < n_slots; k += blockDim.x)
      if (s_grad[k] != 0.0f) atomicAdd(&grads[k], s_grad[k]);
  }
}

// ------------------------------------------------------------- connect ---
//
// Traces the wave's queued shadow rays and adds each unoccluded ray's
// contribution to its pixel. Persistent (a GPU-sized grid) with warp-level
// work fetch (Aila & Laine, HPG 2009): a lane whose ray is done takes the next
// queued ray at once, one atomic per warp for all its idle lanes, instead of
// waiting for the warp's slowest ray; each loop iteration advances every busy
// lane by one step of its own walk (occluded_step).
template <uint32_t kF>
__global__ void __launch_bounds__(kMaxTraceBlock, kConnectBlocksPerSm * kTraceBlock / kMaxTraceBlock) k_connect(ShadowQueue Q,
                                                                             const JobDesc* __restrict__ jobs,
                                                                             WaveCounters* counters) {
  extern __shared__ __align__(16) uint32_t s_stack[];  // occluded_shared_bytes(blockDim.x)
  OccStack st;
  st.bind(s_stack);
  OccWalk w;
  const uint32_t n = min(counters->shadow_count, Q.capacity);
  const int lane = threadIdx.x & 31;
  uint32_t ray = kEmpty;   // queue index of this lane's ray (kEmpty: idle)
  bool exhausted = false;  // the queue has been handed out (warp-uniform)
  uint32_t tests = 0, nodes = 0;
  for (;;) {
    if (!exhausted) {
      const uint32_t idle = __ballot_sync(0xFFFFFFFFu, ray == kEmpty);
      if (idle) {
        const int leader = __ffs(idle) - 1;
        uint32_t base = 0;
        if (lane == leader) base = atomicAdd(&counters->shadow_cursor, (uint32_t)__popc(idle));
        base = __shfl_sync(0xFFFFFFFFu, base, leader);
        if (base + (uint32_t)__popc(idle) >= n) exhausted = true;
        if (ray == kEmpty) {
          const uint32_t t = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
          if (t < n) {
            const float4 o = Q.o[t], d = Q.d[t];
            const uint32_t job = __float_as_uint(Q.c[t].w);
            w.begin(jobs[job].scene_slot, vec3(o.x, o.y, o.z), vec3(d.x, d.y, d.z), o.w, st);
            ray = t;
          }
        }
      }
    }
    if (__ballot_sync(0xFFFFFFFFu, ray != kEmpty) == 0) break;
    if (ray != kEmpty) {
      const int r = occluded_step<(kF & kFeatSpheres) != 0>(w, st, &tests, &nodes);
      if (r != kWalkGoing) {
        if (r == kWalkClear) {
          const float4 c = Q.c[ray];
          const JobDesc& J = jobs[__float_as_uint(c.w)];
          atomicAdd(J.image + __float_as_uint(Q.d[ray].w), make_float4(c.x, c.y, c.z, 0.0f));
          if (J.path_radiance) {
            // the record holds radiance, the contribution is weighted by 1/spp
            const float spp = (float)gmax(J.setting.ssp, 1);
            atomicAdd(J.path_radiance + Q.path[ray], make_float4(c.x * spp, c.y * spp, c.z * spp, 0.0f));
          }
        }
        ray = kEmpty;
      }
    }
  }
  for (int off = 16; off > 0; off >>= 1) {
    tests += __shfl_down_sync(0xFFFFFFFFu, tests, off);
    nodes += __shfl_down_sync(0xFFFFFFFFu, nodes, off);
  }
  if (lane == 0) {
    if (tests) atomicAdd(&counters->shadow_tri_tests, (unsigned long long)tests);
    if (nodes) atomicAdd(&counters->shadow_node_visits, (unsigned long long)nodes);
  }
  if (st.overflow) atomicOr(&counters->errors, (uint32_t)kDevErrStack);
}

// Scene features a wave kernel is instantiated on. Surface kernels: the
// sphere and texture bits (grids are media). Media kernels: the sphere bit
// and one bit for the full texture node set (grids or the solid nodes beyond
// fBm switch on both). So each runs one of four instantiations.
constexpr uint32_t surface_features(uint32_t f) { return f & (kFeatSpheres | kFeatTextures); }
constexpr uint32_t media_features(uint32_t f) {
  return (f & (kFeatGrids | kFeatTextures)) ? (f | kFeatGrids | kFeatTextures) : (f & kFeatSpheres);
}

// Lets a k_extend instantiation take the dynamic shared memory of a
// kMaxTraceBlock-thread block (more than the default 48 KB).
template <typename K>
static void allow_trace_shared(K kernel) {
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       (int)traversal_shared_bytes(kMaxTraceBlock));
}

// Writes scenes[k] into this translation unit's constant slot slots[k]
// (k < n; slots == nullptr: slot k) and the prime tables.
static cudaError_t upload_slots_here(const DeviceScene* scenes, const uint32_t* slots, uint32_t n,
                                     const uint32_t* primes, const uint32_t* prime_sums, cudaStream_t stream) {
  if (n > (uint32_t)kMaxBatchScenes) return cudaErrorInvalidValue;
  cudaError_t e = cudaSuccess;
  uint32_t k = 0;
  while (k < n && e == cudaSuccess) {
    // one copy per run of consecutive slots
    const uint32_t first = slots ? slots[k] : k;
    if (first >= (uint32_t)kMaxBatchScenes) return cudaErrorInvalidValue;
    uint32_t run = 1;
    while (k + run < n && (slots ? slots[k + run] : k + run) == first + run) ++run;
    e = cudaMemcpyToSymbolAsync(c_scenes, scenes + k, sizeof(DeviceScene) * run, sizeof(DeviceScene) * first,
                                cudaMemcpyHostToDevice, stream);
    k += run;
  }
  if (e == cudaSuccess)
    e = cudaMemcpyToSymbolAsync(c_primes, primes, sizeof(uint32_t) * kHaltonDims, 0, cudaMemcpyHostToDevice, stream);
  if (e == cudaSuccess)
    e = cudaMemcpyToSymbolAsync(c_prime_sums, prime_sums, sizeof(uint32_t) * kHaltonDims, 0, cudaMemcpyHostToDevice,
                                stream);
  return e;
}

// This translation unit's bound record (dev_bound.cuh), optionally cleared.
static cudaError_t read_bound_here(BoundRecord* out, bool clear, cudaStream_t stream) {
  cudaError_t e = cudaMemcpyFromSymbolAsync(out, g_bound, sizeof(BoundRecord), 0, cudaMemcpyDeviceToHost, stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  if (e == cudaSuccess && clear) {
    const BoundRecord zero{};
    e = cudaMemcpyToSymbolAsync(g_bound, &zero, sizeof(zero), 0, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
  }
  return e;
}

}  // namespace ym
