// Volume media on the device: delta tracking through overlapping media,
// transmittance along shadow rays through medium boundaries and
// Henyey-Greenstein phase functions; densities are texture nodes
// (dev_texture.cuh).
//
// Follows src/VolumeEval.cuh (SampleTrHomogeneous :18-78,
// SampleTrHeterogeneous :80-214, EvalTrHomogeneous :253-267,
// EvalTrHeterogeneous :269-386, TraceTr :420-468, SampleMixedPhases
// :470-516, EvalMixedPhases :518-538) and src/Volume.h (EvalPhase,
// SamplePhase), in the reference's operand order.
#pragma once

#include <cuda_fp16.h>

#include "ymrt_scene.h"
#include "dev_sampler.cuh"
#include "dev_texture.cuh"

namespace ym {

__device__ __forceinline__ bool has_density(const DeviceScene& S, const Volume& v) {
  return v.density_texture_idx >= 0 && (uint32_t)v.density_texture_idx < S.texture_count;
}

// RayTransfer::GetCurrentVolumeIndices (src/Ray.h:131-145).
__device__ __forceinline__ int current_volumes(const RayTransfer& rt, uint32_t volume_count, int idx[kMaxBoundaryRecord]) {
  if (rt.record_count == 0 || rt.max_priority_record_index == -1) return 0;
  const uint32_t mp = rt.records[rt.max_priority_record_index].ior_priority;
  int n = 0;
  for (int r = rt.record_count - 1; r >= 0; --r)
    if (rt.records[r].ior_priority == mp && rt.records[r].vol_idx >= 0 && (uint32_t)rt.records[r].vol_idx < volume_count)
      idx[n++] = rt.records[r].vol_idx;
  return n;
}

// -------------------------------------------------------------- phases ---

// EvalPhase (src/Volume.h:21-27).
__device__ __forceinline__ float eval_phase(float g, vec3 wo, vec3 wi, float* pdf) {
  const float c = dot(wo, wi);
  const float t = 1.f + g * g + 2.f * g * c;
  *pdf = 0.25f * kInvPi * (1.f - g * g) * safe_rcp((t * sqrtf(gmax(t, 0.0f))));
  return *pdf;
}

// SamplePhase (src/Volume.h:28-47).
__device__ __forceinline__ void sample_phase(float g, float u0, float u1, vec3 wo, float* weight, vec3* wi, float* pdf) {
  float c;
  if (fabsf(g) < 1e-4f) {
    c = 1.f - 2.f * u0;
  } else {
    const float t = (1.f - g * g) * safe_rcp(1.f - g + 2.f * g * u0);
    c = (1.f + g * g - t * t) / (2.f * g);
  }
  const float s = sqrtf(gmax(0.0f, 1.0f - c * c));
  const float phi = 2.f * kPi * u1;
  vec3 w = wo, u, v;
  orthogonal_basis(w, u, v);
  *wi = u * s * cosf(phi) + v * s * sinf(phi) + w * c;
  eval_phase(g, wo, *wi, pdf);
  *weight = 1.0f;
}

// SampleMixedPhases (src/VolumeEval.cuh:470-516).
__device__ __forceinline__ bool sample_mixed_phases(const float* w, const float* gs, int n, float u0, float u1, vec3 wo,
                                                    float* weight, vec3* wi, float* pdf) {
  if (n == 0) return false;
  float cdf = 0.0f;
  int sel = -1;
  for (int i = 0; i < n; ++i) {
    if (u0 < cdf + w[i]) {
      sel = i;
      u0 = (u0 - cdf) * safe_rcp(w[i]);
      break;
    }
    cdf += w[i];
  }
  if (sel == -1) sel = n - 1;
  float ppdf = 0.0f;
  sample_phase(gs[sel], u0, u1, wo, weight, wi, &ppdf);
  float mixed_pdf = ppdf * w[sel];
  float mixed_g = (*weight) * ppdf * w[sel];
  for (int i = 0; i < n; ++i) {
    if (i == sel) continue;
    float p;
    mixed_g += w[i] * eval_phase(gs[i], wo, *wi, &p);
    mixed_pdf += w[i] * p;
  }
  *pdf = mixed_pdf;
  *weight = mixed_g * safe_rcp(mixed_pdf);
  return true;
}

// EvalMixedPhases (src/VolumeEval.cuh:518-538).
__device__ __forceinline__ float eval_mixed_phases(const float* w, const float* gs, int n, vec3 wo, vec3 wi, float* pdf) {
  if (n == 0) {
    *pdf = 0.0f;
    return 0.0f;
  }
  float mg = 0.0f, mp = 0.0f;
  for (int i = 0; i < n; ++i) {
    float sp = 0.0f;
    const float sg = eval_phase(gs[i], wo, wi, &sp);
    mg += w[i] * sg;
    mp += w[i] * sp;
  }
  *pdf = mp;
  return mg;
}

// ------------------------------------------------------- free flights ---

// SampleTrHomogeneous (src/VolumeEval.cuh:18-78).
__device__ __forceinline__ bool sample_tr_homogeneous(const DeviceScene& S, int n, const int* vidx, float t_max,
                                                      vec3* tr_weight, float* dist, float* vw, PathSampler& hs) {
  *tr_weight = vec3(1.0f);
  *dist = kFloatMax;
  vec3 m(0.0f), ms(0.0f);
  for (int i = 0; i < n; ++i) {
    const Volume& v = S.volumes[vidx[i]];
    m += v.sigma_t;
    ms += v.sigma_t * v.albedo;
  }
  const float csum = m.x + m.y + m.z;
  const vec3 cw = csum > 0.0f ? (m / csum) : vec3(1.0f / 3.0f);
  float u0 = sample1d(hs, S);
  int ch = 0;
  if (u0 < cw[0]) {
    ch = 0;
    u0 = u0 * safe_rcp(cw[0]);
  } else if (u0 < cw[0] + cw[1]) {
    ch = 1;
    u0 = (u0 - cw[0]) * safe_rcp(cw[1]);
  } else {
    ch = 2;
    u0 = (u0 - cw[0] - cw[1]) * safe_rcp(cw[2]);
  }
  const float fpl = m[ch] > 0.0f ? (-logf(1.0f - u0) / m[ch]) : kFloatMax;
  const bool scatter = fpl < t_max;
  const vec3 tr = vexp(-m * gmin(t_max, fpl));
  const float pdf = scatter ? (cw.x * m.x * tr.x + cw.y * m.y * tr.y + cw.z * m.z * tr.z)
                            : (cw.x * tr.x + cw.y * tr.y + cw.z * tr.z);
  if (!(fabsf(pdf) > 0.0f)) return false;
  const float vwt = 1.0f / float(n);
  for (int i = 0; i < n; ++i) vw[i] = vwt;
  *tr_weight = scatter ? (tr * ms / pdf) : (tr / pdf);
  *dist = fpl;
  return scatter;
}

// Majorant set-up shared by the heterogeneous estimators.
struct Majorant {
  vec3 m, cw, nf, mrcp;
  vec3 ro[kMaxBoundaryRecord], rd[kMaxBoundaryRecord];
  int ch;
};
__device__ __forceinline__ void volume_space_rays(const DeviceScene& S, int n, const int* vidx, vec3 o, vec3 d, float t_max,
                                                  Majorant& M) {
  M.m = vec3(0.0f);
  for (int i = 0; i < n; ++i) {
    const Volume& v = S.volumes[vidx[i]];
    float ub = 1.0f;
    if (has_density(S, v)) {
      const mat4& it = S.i_transforms[v.transform_idx];
      M.ro[i] = xform_point_glm(it, o);
      M.rd[i] = xform_dir_glm(it, d);
      ub = texture_upper_bound(S.textures[v.density_texture_idx]);
    }
    M.m += v.sigma_t * ub;
  }
  const float csum = M.m.x + M.m.y + M.m.z;
  M.cw = csum > 0.0f ? (M.m / csum) : vec3(1.0f / 3.0f);
}
template <uint32_t kF>
__device__ __forceinline__ void densities(const DeviceScene& S, int n, const int* vidx, const Majorant& M, float acc,
                                          vec3* mst, vec3* mss, uint32_t* errors) {
  *mst = vec3(0.0f);
  if (mss) *mss = vec3(0.0f);
  for (int i = 0; i < n; ++i) {
    const Volume& v = S.volumes[vidx[i]];
    float density = 1.0f;
    if (has_density(S, v))
      density = gmax(texture_eval<kF>(S.textures, (uint32_t)v.density_texture_idx, M.ro[i] + M.rd[i] * acc, errors).x, 0.0f);
    *mst += v.sigma_t * density;
    if (mss) *mss += v.sigma_t * v.albedo * density;
  }
}

// ---- density-grid gradients (the adjoint pass) ----
//
// A tracking estimator's value is f / p with f the product, over its
// tentative collisions x_j, of exp(-m * step) and
//   null collision:  m - sigma_t(x_j)           (delta and ratio tracking)
//   real collision:  sigma_s(x_j)               (delta tracking's last one)
// and p the sampling pdf. With the samples (and the majorant m, which the
// estimator's expectation does not depend on) held fixed, d(f/p)/d(g_k) for
// a grid value g_k is (f/p) times the sum over collisions of
//   null:  -d sigma_t(x_j)/d g_k / (m - sigma_t(x_j))
//   real:   d sigma_s(x_j)/d g_k / sigma_s(x_j)
// per colour channel, where sigma_t = sigma_t,vol * density and density is
// the grid's trilinear read, linear in g_k with weight w_k(x_j). `scale` is
// dLoss/d(radiance) times the radiance the estimator multiplies, per
// channel; each collision adds its terms to the eight grid cells it reads.
struct MediumAdj {
  vec3 scale;
  uint32_t grid_tex;   // the differentiated grid node
  float* grads;        // dLoss/d(grid value), x fastest
};

// grads += g * (trilinear weight of each of the eight cells read at p).
__device__ __forceinline__ void grid_scatter(const Texture& t, vec3 p, float g, float* grads) {
  int x[2], y[2], z[2];
  float wx, wy, wz;
  grid_axis(p.x, t.grid_n[0], &x[0], &x[1], &wx);
  grid_axis(p.y, t.grid_n[1], &y[0], &y[1], &wy);
  grid_axis(p.z, t.grid_n[2], &z[0], &z[1], &wz);
  const float fx[2] = {1.0f - wx, wx}, fy[2] = {1.0f - wy, wy}, fz[2] = {1.0f - wz, wz};
  for (int c = 0; c < 8; ++c) {
    const float w = fx[c & 1] * fy[(c >> 1) & 1] * fz[c >> 2];
    if (w == 0.0f) continue;
    const size_t k = ((size_t)z[c >> 2] * (size_t)t.grid_n[1] + (size_t)y[(c >> 1) & 1]) * (size_t)t.grid_n[0] +
                     (size_t)x[c & 1];
    atomicAdd(grads + k, g * w);
  }
}

// One tentative collision's terms: coef_t (per channel) multiplies
// d sigma_t / d density of each medium, coef_s multiplies d sigma_s / d density.
static __device__ __noinline__ void medium_grad(const DeviceScene& S, int n, const int* vidx, const vec3* ro, const vec3* rd,
                                         float acc, vec3 coef_t, vec3 coef_s, const MediumAdj& am) {
  for (int i = 0; i < n; ++i) {
    const Volume& v = S.volumes[vidx[i]];
    if (v.density_texture_idx != (int)am.grid_tex || !has_density(S, v)) continue;
    const Texture& t = S.textures[am.grid_tex];
    if (t.type != kTexGrid) continue;
    const vec3 p = ro[i] + rd[i] * acc;
    if (!(grid_eval(t, p) > 0.0f)) continue;  // the density is clamped at zero
    const float g = dot(coef_t, v.sigma_t) + dot(coef_s, v.sigma_t * v.albedo);
    if (g != 0.0f) grid_scatter(t, p, g, am.grads);
  }
}

// SampleTrHeterogeneous (src/VolumeEval.cuh:80-214): delta tracking against
// the summed majorant with channel-wise real / null collision probabilities.
// kAdj: also adds the segment's density-grid gradient terms (MediumAdj).
// `errors` is the frame's WaveCounters::errors: a loop that reaches
// kMaxFreePath steps stops there as the reference's does (a failed sample)
// and is counted in the word after it (WaveCounters::tracking_caps).
template <uint32_t kF, bool kAdj = false>
__device__ __noinline__ bool sample_tr_heterogeneous(const DeviceScene& S, int n, const int* vidx, vec3 o, vec3 d,
                                                     float t_max, vec3* tr_weight, float* dist, float* vw,
                                                     PathSampler& hs, uint32_t* errors,
                                                     const MediumAdj* am = nullptr) {
  *tr_weight = vec3(1.0f);
  *dist = kFloatMax;
  Majorant M;
  volume_space_rays(S, n, vidx, o, d, t_max, M);
  const float u0 = sample1d(hs, S);
  int ch = 0;
  if (u0 < M.cw[0]) ch = 0;
  else if (u0 < M.cw[0] + M.cw[1]) ch = 1;
  else ch = 2;
  if (!(M.m[ch] > 0.0f)) return false;
  const vec3 nf(safe_rcp(M.m.x + 1.0f), safe_rcp(M.m.y + 1.0f), safe_rcp(M.m.z + 1.0f));
  const vec3 mrcp(safe_rcp(M.m.x), safe_rcp(M.m.y), safe_rcp(M.m.z));
  vec3 tr(1.0f), pdf(1.0f);
  float acc = 0.0f;
  int it = 0;
  while (true) {
    if (it >= kMaxFreePath) {
      atomicAdd(errors + 1, 1u);  // WaveCounters::tracking_caps
      note_bound(kBoundDeltaTracking, (uint32_t)it, o, d, t_max - acc, kEmpty, kEmpty, nullptr, M.m, ch);
      break;
    }
    const float fpl = -logf(1.0f - sample1d(hs, S)) / M.m[ch];
    if (acc + fpl > t_max) {
      const vec3 ptr = vexp(-M.m * (t_max - acc));
      tr *= ptr * nf;
      pdf *= ptr * nf;
      acc += fpl;
      break;
    }
    acc += fpl;
    vec3 mst, mss;
    densities<kF>(S, n, vidx, M, acc, &mst, &mss, errors);
    vec3 real;
    real.x = gmin(M.m.x > 0.0f ? mst.x * mrcp.x : 0.0f, 1.0f);
    real.y = gmin(M.m.y > 0.0f ? mst.y * mrcp.y : 0.0f, 1.0f);
    real.z = gmin(M.m.z > 0.0f ? mst.z * mrcp.z : 0.0f, 1.0f);
    const vec3 fake = vec3(1.0f) - real;
    const vec3 ptr = vexp(-M.m * fpl);
    if (sample1d(hs, S) < real[ch]) {
      tr *= ptr * mss * nf;
      pdf *= ptr * M.m * real * nf;
      if constexpr (kAdj) {
        vec3 cs(0.0f);
        for (int c = 0; c < 3; ++c) cs[c] = mss[c] > 0.0f ? am->scale[c] / mss[c] : 0.0f;
        medium_grad(S, n, vidx, M.ro, M.rd, acc, vec3(0.0f), cs, *am);
      }
      break;
    } else {
      tr *= ptr * M.m * fake * nf;
      pdf *= ptr * M.m * fake * nf;
      if constexpr (kAdj) {
        vec3 ct(0.0f);
        for (int c = 0; c < 3; ++c) ct[c] = M.m[c] - mst[c] > 0.0f ? -am->scale[c] / (M.m[c] - mst[c]) : 0.0f;
        medium_grad(S, n, vidx, M.ro, M.rd, acc, ct, vec3(0.0f), *am);
      }
    }
    ++it;
  }
  const float vwt = 1.0f / float(n);
  for (int i = 0; i < n; ++i) vw[i] = vwt;
  *tr_weight = tr * safe_rcp(dot(M.cw, pdf));
  *dist = acc;
  return acc > t_max || it >= kMaxFreePath ? false : true;
}

// SampleVolumeScattering (src/VolumeEval.cuh:217-251).
template <uint32_t kF, bool kAdj = false>
__device__ __forceinline__ bool sample_volume_scattering(const DeviceScene& S, vec3 o, vec3 d, int n, const int* vidx,
                                                         float t_max, vec3* tr_weight, float* dist, float* vw,
                                                         PathSampler& hs, uint32_t* errors,
                                                         const MediumAdj* am = nullptr) {
  if (S.volume_count == 0 || n == 0) return false;
  bool het = false;
  for (int i = 0; i < n; ++i)
    if (has_density(S, S.volumes[vidx[i]])) {
      het = true;
      break;
    }
  if (het) return sample_tr_heterogeneous<kF, kAdj>(S, n, vidx, o, d, t_max, tr_weight, dist, vw, hs, errors, am);
  return sample_tr_homogeneous(S, n, vidx, t_max, tr_weight, dist, vw, hs);
}

// EvalTrHeterogeneous (src/VolumeEval.cuh:269-386): ratio-tracking style
// transmittance with Russian roulette after 32 steps. kAdj: also adds the
// density-grid gradient terms of its collisions (MediumAdj). The
// kMaxFreePath bound is counted as in sample_tr_heterogeneous.
template <uint32_t kF, bool kAdj = false>
__device__ __noinline__ vec3 eval_tr_heterogeneous(const DeviceScene& S, int n, const int* vidx, vec3 o, vec3 d,
                                                   float t_max, PathSampler& hs, uint32_t* errors,
                                                   const MediumAdj* am = nullptr) {
  Majorant M;
  volume_space_rays(S, n, vidx, o, d, t_max, M);
  const float u0 = sample1d(hs, S);
  int ch = 0;
  if (u0 < M.cw[0]) ch = 0;
  else if (u0 < M.cw[0] + M.cw[1]) ch = 1;
  else ch = 2;
  if (!(M.m[ch] > 0.0f)) return vec3(1.0f);
  const vec3 nf(safe_rcp(M.m.x + 1.0f), safe_rcp(M.m.y + 1.0f), safe_rcp(M.m.z + 1.0f));
  const vec3 mrcp(safe_rcp(M.m.x), safe_rcp(M.m.y), safe_rcp(M.m.z));
  vec3 tr(1.0f), pdf(1.0f);
  float acc = 0.0f;
  int it = 0;
  while (true) {
    if (it >= kMaxFreePath) {
      atomicAdd(errors + 1, 1u);  // WaveCounters::tracking_caps
      note_bound(kBoundRatioTracking, (uint32_t)it, o, d, t_max - acc, kEmpty, kEmpty, nullptr, M.m, ch);
      break;
    }
    const float fpl = -logf(1.0f - sample1d(hs, S)) / M.m[ch];
    if (acc + fpl > t_max) {
      const vec3 ptr = vexp(-M.m * (t_max - acc));
      tr *= ptr * nf;
      pdf *= ptr * nf;
      break;
    }
    acc += fpl;
    vec3 mst;
    densities<kF>(S, n, vidx, M, acc, &mst, nullptr, errors);
    vec3 real;
    real.x = gmin(M.m.x > 0.0f ? mst.x * mrcp.x : 0.0f, 1.0f);
    real.y = gmin(M.m.y > 0.0f ? mst.y * mrcp.y : 0.0f, 1.0f);
    real.z = gmin(M.m.z > 0.0f ? mst.z * mrcp.z : 0.0f, 1.0f);
    const vec3 fake = vec3(1.0f) - real;
    const vec3 ptr = vexp(-M.m * fpl);
    tr *= ptr * M.m * fake * nf;
    pdf *= ptr * M.m * nf;
    if constexpr (kAdj) {
      vec3 ct(0.0f);
      for (int c = 0; c < 3; ++c) ct[c] = M.m[c] - mst[c] > 0.0f ? -am->scale[c] / (M.m[c] - mst[c]) : 0.0f;
      medium_grad(S, n, vidx, M.ro, M.rd, acc, ct, vec3(0.0f), *am);
    }
    if (it + 1 > 32) {
      const vec3 pt = tr * safe_rcp(dot(M.cw, pdf));
      float rr = gmax(pt.x, gmax(pt.y, pt.z));
      rr = gmin(rr, 1.0f);
      if (sample1d(hs, S) < rr) tr /= gmax(rr, kMinColorEps);
      else break;
    }
    ++it;
  }
  return tr * safe_rcp(dot(M.cw, pdf));
}

// EvalTr (src/VolumeEval.cuh:388-418).
template <uint32_t kF, bool kAdj = false>
__device__ __forceinline__ vec3 eval_tr(const DeviceScene& S, vec3 o, vec3 d, const RayTransfer& rt, float t_max,
                                        PathSampler& hs, uint32_t* errors, const MediumAdj* am = nullptr) {
  if (S.volume_count == 0) return vec3(1.0f);
  int vidx[kMaxBoundaryRecord];
  const int n = current_volumes(rt, S.volume_count, vidx);
  if (n == 0) return vec3(1.0f);
  bool het = false;
  for (int i = 0; i < n; ++i)
    if (has_density(S, S.volumes[vidx[i]])) {
      het = true;
      break;
    }
  if (het) return eval_tr_heterogeneous<kF, kAdj>(S, n, vidx, o, d, t_max, hs, errors, am);
  vec3 m(0.0f);
  for (int i = 0; i < n; ++i) m += S.volumes[vidx[i]].sigma_t;
  return vexp(-m * t_max);
}

}  // namespace ym
