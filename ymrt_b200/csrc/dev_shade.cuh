// Surface shading on the device: hit reconstruction, the layered default
// material (coat / conductor / dielectric reflection / dielectric
// transmission / Lambert, one-sample lobe selection) and shape-light sampling.
//
// Each function states the reference function whose arithmetic it follows;
// expressions keep the reference's operand order (the kernels are built with
// -fmad=false, so every product and sum rounds as written), including the
// places where the reference mixes in double-precision literals.
#pragma once

#include "dev_texture.cuh"
#include "sphere.h"
#include "ymrt_scene.h"

namespace ym {

// ------------------------------------------------------------ hit data ---

struct SurfacePoint {
  vec3 p, p_err, p_obj, ns, ng, dpdu, dpdv;
  float u, v;  // texture coordinates
};

// FetchSphereShadingData (src/ShadingUtilities.cuh:639-711) in object space:
// `p` is the hit point the sphere test projected onto the sphere.
__device__ __forceinline__ void sphere_surface(float sphere_radius, vec3 p, SurfacePoint* sp) {
  const float radius = gmax(sphere_radius, kFloatEps);
  const vec3 n = p / radius;
  sp->p = p;
  sp->p_err = error_gamma(5) * vabs(p);
  sp->ns = n;
  sp->ng = n;
  const float theta = acosf(n.y);
  float phi = atan2f(n.z, n.x);
  if (phi < 0.0f) phi += kTwoPi;
  sp->u = 0.5f * phi * kInvPi;
  sp->v = theta * kInvPi;
  float sin_theta = 0.0f;
  if (1.0f - n.y * n.y > 0.0f) sin_theta = sqrtf(1.0f - n.y * n.y);
  float cos_phi, sin_phi;
  if (sin_theta > 0.0f) {
    cos_phi = n.x / sin_theta;
    sin_phi = n.z / sin_theta;
  } else {
    cos_phi = 1.0f;
    sin_phi = 0.0f;
  }
  sp->dpdu = vec3(-p.z, 0.0f, p.x) * kTwoPi;
  sp->dpdv = vec3(p.y * cos_phi, -radius * sin_theta, sin_phi * p.y) * kPi;
}

// FetchShadingData + FetchMeshShadingData / FetchSphereShadingData
// (src/ShadingUtilities.cuh:639-875). For a sphere `bary` is the object-space
// hit point and `tri` is EMPTY.
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ SurfacePoint fetch_surface(const DeviceScene& S, uint32_t inst_idx, uint32_t tri,
                                                      vec3 bary) {
  const Instance inst = S.instances[inst_idx];
  const GeometryDesc& g = S.geometries[inst.geometry_idx];
  if ((kF & kFeatSpheres) && g.kind == kGeoSphere) {
    SurfacePoint sp;
    sphere_surface(g.radius, bary, &sp);
    const mat4& otw = S.transforms[inst.transform_idx];
    const mat4& wto = S.i_transforms[inst.transform_idx];
    sp.p_obj = sp.p;
    sp.p = transform_position(otw, sp.p, &sp.p_err);
    sp.ns = normalize(transpose_transform_vector(wto, sp.ns));
    sp.ng = normalize(transpose_transform_vector(wto, sp.ng));
    sp.dpdu = transform_vector(otw, sp.dpdu);
    sp.dpdv = transform_vector(otw, sp.dpdv);
    return sp;
  }
  const uint32_t* tc = S.tri_corners + 3 * (size_t)(g.tri_offset + tri);
  const uint32_t c0 = tc[0], c1 = tc[1], c2 = tc[2];
  auto P = [&](uint32_t c) {
    const uint32_t vi = S.pos_idx[g.corner_offset + c];
    const float* q = S.positions + 3 * (size_t)(g.pos_offset + vi);
    return vec3(q[0], q[1], q[2]);
  };
  auto N = [&](uint32_t c) {
    const uint32_t vi = S.nrm_idx[g.corner_offset + c];
    const float* q = S.normals + 3 * (size_t)(g.nrm_offset + vi);
    return vec3(q[0], q[1], q[2]);
  };
  const vec3 p0 = P(c0), p1 = P(c1), p2 = P(c2);
  SurfacePoint sp;
  const float xs = fabsf(p0.x * bary.x) + fabsf(p1.x * bary.y) + fabsf(p2.x * bary.z);
  const float ys = fabsf(p0.y * bary.x) + fabsf(p1.y * bary.y) + fabsf(p2.y * bary.z);
  const float zs = fabsf(p0.z * bary.x) + fabsf(p1.z * bary.y) + fabsf(p2.z * bary.z);
  sp.p = p0 * bary.x + p1 * bary.y + p2 * bary.z;
  sp.p_err = error_gamma(7) * vec3(xs, ys, zs);
  const vec3 n0 = N(c0), n1 = N(c1), n2 = N(c2);
  sp.ns = n0 * bary.x + n1 * bary.y + n2 * bary.z;
  sp.ng = cross(p1 - p0, p2 - p0);
  float u0x = 0.0f, u0y = 0.0f, u1x = 1.0f, u1y = 0.0f, u2x = 1.0f, u2y = 1.0f;
  if (g.uv_offset >= 0) {
    const float* uvb = S.texcoords + 2 * (size_t)g.uv_offset;
    const uint32_t t0 = S.uv_idx[g.corner_offset + c0], t1 = S.uv_idx[g.corner_offset + c1],
                   t2 = S.uv_idx[g.corner_offset + c2];
    u0x = uvb[2 * t0]; u0y = uvb[2 * t0 + 1];
    u1x = uvb[2 * t1]; u1y = uvb[2 * t1 + 1];
    u2x = uvb[2 * t2]; u2y = uvb[2 * t2 + 1];
  }
  sp.u = u0x * bary.x + u1x * bary.y + u2x * bary.z;
  sp.v = u0y * bary.x + u1y * bary.y + u2y * bary.z;
  float du01 = u1x - u0x, dv01 = u1y - u0y;
  float du02 = u2x - u0x, dv02 = u2y - u0y;
  float det = du01 * dv02 - dv01 * du02;
  if (fabsf(det) < (float)1E-8f) {
    du01 = 1.0f; dv01 = 0.0f;
    du02 = 0.0f; dv02 = 1.0f;
    det = 1.0f;
  }
  const float idet = 1.0f / det;
  const vec3 dp01 = p1 - p0, dp02 = p2 - p0;
  sp.dpdu = (dv02 * dp01 - dv01 * dp02) * idet;
  sp.dpdv = (-du02 * dp01 + du01 * dp02) * idet;
  const mat4& otw = S.transforms[inst.transform_idx];
  const mat4& wto = S.i_transforms[inst.transform_idx];
  sp.p_obj = sp.p;
  sp.p = transform_position(otw, sp.p, &sp.p_err);
  sp.ns = normalize(transpose_transform_vector(wto, sp.ns));
  sp.ng = normalize(transpose_transform_vector(wto, sp.ng));
  sp.dpdu = transform_vector(otw, sp.dpdu);
  sp.dpdv = transform_vector(otw, sp.dpdv);
  return sp;
}

// FetchGeometryNormal with FetchMeshGeometryNormal / FetchSphereGeometryNormal
// (src/ShadingUtilities.cuh:877-952): position, error and normalised
// geometric normal only.
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ void fetch_geometry_normal(const DeviceScene& S, uint32_t inst_idx, uint32_t tri, vec3 bary,
                                                      vec3* p, vec3* p_err, vec3* ng) {
  const Instance inst = S.instances[inst_idx];
  const GeometryDesc& g = S.geometries[inst.geometry_idx];
  if ((kF & kFeatSpheres) && g.kind == kGeoSphere) {
    const float radius = gmax(g.radius, kFloatEps);
    *p = bary;
    *p_err = error_gamma(5) * vabs(bary);
    *ng = bary / radius;
  } else {
    const uint32_t* tc = S.tri_corners + 3 * (size_t)(g.tri_offset + tri);
    vec3 q[3];
    for (int k = 0; k < 3; ++k) {
      const uint32_t vi = S.pos_idx[g.corner_offset + tc[k]];
      const float* a = S.positions + 3 * (size_t)(g.pos_offset + vi);
      q[k] = vec3(a[0], a[1], a[2]);
    }
    const float xs = fabsf(q[0].x * bary.x) + fabsf(q[1].x * bary.y) + fabsf(q[2].x * bary.z);
    const float ys = fabsf(q[0].y * bary.x) + fabsf(q[1].y * bary.y) + fabsf(q[2].y * bary.z);
    const float zs = fabsf(q[0].z * bary.x) + fabsf(q[1].z * bary.y) + fabsf(q[2].z * bary.z);
    *p = q[0] * bary.x + q[1] * bary.y + q[2] * bary.z;
    *p_err = error_gamma(7) * vec3(xs, ys, zs);
    *ng = cross(q[1] - q[0], q[2] - q[0]);
  }
  const mat4& otw = S.transforms[inst.transform_idx];
  const mat4& wto = S.i_transforms[inst.transform_idx];
  *p = transform_position(otw, *p, p_err);
  *ng = normalize(transpose_transform_vector(wto, *ng));
}

// ---------------------------------------------------------- microfacet ---
// src/BSDF.cuh:19-176.


__device__ __forceinline__ vec3 reflect(vec3 wo, vec3 n) { return -wo + 2.0f * n * dot(n, wo); }

__device__ __forceinline__ bool refract(vec3 wo, vec3 n, float ni, float nt, vec3* wi) {
  const float ci = gmax(dot(wo, n), 0.0f);
  const float ci2 = sqr(ci);
  const float si2 = 1.0f - ci2;
  const float ct2 = 1.0f - sqr(ni / nt) * si2;
  if (!(ct2 > 0.0f)) return false;
  const float ct = sqrtf(ct2);
  *wi = normalize(-(ni / nt) * (wo - n * ci) - n * ct);
  return true;
}

// FresnelDielectricDielectric (src/BSDF.cuh:81-95), eta = nt / ni.
__device__ __forceinline__ float fresnel_dielectric(float eta, float cos_theta) {
  cos_theta = gmax(0.0f, cos_theta);
  const float s2 = 1.f - cos_theta * cos_theta;
  const float t0 = sqrtf(gmax(1.0f - (s2 / (eta * eta)), 0.0f));
  const float t1 = eta * t0;
  const float t2 = eta * cos_theta;
  const float rs = (cos_theta - t1) / gmax(cos_theta + t1, 1E-12f);
  const float rp = (t0 - t2) / gmax(t0 + t2, 1E-12f);
  return (float)(0.5 * (double)(rs * rs + rp * rp));
}

// FresnelDieletricConductor (src/BSDF.cuh:96-115).
__device__ __forceinline__ vec3 fresnel_conductor(vec3 eta, vec3 etak, float c) {
  const float c2 = c * c;
  const float s2 = 1.0f - c2;
  const vec3 eta2 = eta * eta;
  const vec3 etak2 = etak * etak;
  const vec3 t0 = eta2 - etak2 - s2;
  const vec3 a2pb2 = vsqrt(t0 * t0 + 4.0f * eta2 * etak2);
  const vec3 t1 = a2pb2 + c2;
  const vec3 a = vsqrt(0.5f * (a2pb2 + t0));
  const vec3 t2 = 2.0f * a * c;
  const vec3 rs = (t1 - t2) / (t1 + t2);
  const vec3 t3 = c2 * a2pb2 + s2 * s2;
  const vec3 t4 = t2 * s2;
  const vec3 rp = rs * (t3 - t4) / (t3 + t4);
  return 0.5f * (rp + rs);
}

// EdgeTintToConductiveFresnel (src/BSDF.cuh:123-134).
__device__ __forceinline__ void edge_tint_to_conductor(vec3 reflectivity, vec3 edge_tint, vec3* n, vec3* k) {
  const vec3 r = vclamp(reflectivity, vec3(0.f), vec3(0.99f));
  const vec3 g = edge_tint;
  const vec3 rs = vsqrt(r);
  const vec3 n_min = (vec3(1.0f) - r) / (vec3(1.0f) + r);
  const vec3 n_max = (vec3(1.0f) + rs) / (vec3(1.0f) - rs);
  *n = mix(n_max, n_min, g);
  vec3 k2 = ((*n + vec3(1.0f)) * (*n + vec3(1.0f)) * r - (*n - vec3(1.0f)) * (*n - vec3(1.0f))) / (vec3(1.0f) - r);
  k2 = vmax(k2, vec3(0.0f));
  *k = vsqrt(k2);
}

__device__ __forceinline__ float ggx_d(vec3 wh, float ax, float ay) {
  const float deno = kPi * ax * ay * sqr(sqr(wh.x / ax) + sqr(wh.y / ay) + sqr(wh.z));
  return 1.0f / gmax(deno, 1E-12f);
}
__device__ __forceinline__ float ggx_lambda(vec3 w, float ax, float ay) {
  if (fabsf(w.z) < 1E-8f) return 0.0f;
  return (-1.0f + sqrtf(1.0f + (sqr(w.x * ax) + sqr(w.y * ay)) / sqr(w.z))) * 0.5f;
}
__device__ __forceinline__ float ggx_g1(vec3 w, float ax, float ay) { return 1.0f / (1.0f + ggx_lambda(w, ax, ay)); }
__device__ __forceinline__ float ggx_g2(vec3 wo, vec3 wi, float ax, float ay) {
  return 1.0f / (1.0f + ggx_lambda(wo, ax, ay) + ggx_lambda(wi, ax, ay));
}

// SampleWh: visible-normal sampling (src/BSDF.cuh:158-176). The blend
// weight and the hemisphere-projection term are evaluated in double, as the
// reference's double literals make them.
__device__ __forceinline__ vec3 sample_wh(vec3 wo, float u0, float u1, float ax, float ay) {
  const vec3 wh = normalize(vec3(ax * wo.x, ay * wo.y, wo.z));
  const float lensq = wh.x * wh.x + wh.y * wh.y;
  const vec3 T1 = lensq > 0 ? vec3(-wh.y, wh.x, 0) * (1.0f / sqrtf(lensq)) : vec3(1, 0, 0);
  const vec3 T2 = cross(wh, T1);
  const float r = sqrtf(gmax(u0, 0.0f));
  const float phi = 2.0f * kPi * u1;
  const float t1 = r * cosf(phi);
  float t2 = r * sinf(phi);
  const float s = (float)(0.5 * (1.0 + (double)wh.z));
  t2 = (float)((1.0 - (double)s) * sqrt(1.0 - (double)(t1 * t1)) + (double)(s * t2));
  const vec3 Nh = t1 * T1 + t2 * T2 + sqrtf(gmax(0.0f, 1.0f - t1 * t1 - t2 * t2)) * wh;
  return normalize(vec3(ax * Nh.x, ay * Nh.y, gmax(0.0f, Nh.z)));
}

// --------------------------------------------------------------- lobes ---

enum LobeType : int { kLambert = 0, kReflect = 1, kTransmit = 2 };

// Which layer of DefaultMtl a lobe models (used by the adjoint pass).
constexpr int kRoleCoat = 0, kRoleMetal = 1, kRoleSpecular = 2, kRoleTransmission = 3, kRoleDiffuse = 4;

struct Lobe {
  int type;
  vec3 albedo;        // diffuse / specular / transmission albedo
  vec3 nt, kt;        // reflection: complex ior of the far side; transmission: nt.x
  float ni;
  float ax, ay;
  int is_metal;
  int role;           // kRole*
};

constexpr int kMaxLobes = 5;

struct LayeredBsdf {
  vec3 t, b, n;  // shading frame
  int count;
  float w[kMaxLobes];
  Lobe lobe[kMaxLobes];

  __device__ __forceinline__ vec3 to_local(vec3 v) const { return vec3(dot(v, t), dot(v, b), dot(v, n)); }
  __device__ __forceinline__ vec3 to_world(vec3 v) const { return v.x * t + v.y * b + v.z * n; }
};

// Lambert / MicrofacetReflection / MicrofacetTransmission ::Eval (src/BSDF.cuh:185-375).
// lobe_eval and lobe_sample are out of line: the layered BSDF's evaluation
// and sampling call them from several sites, and one copy of each keeps the
// shading kernels' instruction footprint small (A/B on one B200: textured
// 1280x720 32-spp frame 742 -> 717 ms, the instanced 1080p 64-spp bench frame
// 216.5 -> 215.3 ms, volumetric unchanged; lobe_eval alone out of line cost
// the bench frame 1.3%).
static __device__ __noinline__ vec3 lobe_eval(const Lobe& L, vec3 wo, vec3 wi, float* pdf) {
  if (L.type == kLambert) {
    if (!same_hemisphere(wo, wi)) {
      *pdf = 0.0f;
      return vec3(0.0f);
    }
    const float c = gmax(wi.z, 0.0f);
    *pdf = c * kInvPi;
    return L.albedo * c * kInvPi;
  }
  if (L.type == kReflect) {
    if (!same_hemisphere(wo, wi) || wo.z < 0.f || wi.z < 0.f) {
      *pdf = 0.0f;
      return vec3(0.0f);
    }
    vec3 wh = wi + wo;
    const float len = length(wh);
    if (fabsf(len) < 1E-8f) {
      *pdf = 0.0f;
      return vec3(0.0f);
    }
    wh /= len;
    const float D = ggx_d(wh, L.ax, L.ay);
    const float G1 = ggx_g1(wo, L.ax, L.ay);
    const float G2 = ggx_g2(wo, wi, L.ax, L.ay);
    const float i_ni = safe_rcp(L.ni);
    const float c = gmax(dot(wo, wh), 0.0f);
    const vec3 fr = L.is_metal ? fresnel_conductor(L.nt * i_ni, L.kt * i_ni, c) : vec3(fresnel_dielectric(L.nt.x * i_ni, c));
    *pdf = D * G1 * 0.25f / gmax(wo.z, 1E-8f);
    return L.albedo * D * G2 * 0.25f * fr / gmax(wo.z, 1E-8f);
  }
  // transmission
  const float ni = L.ni, nt = L.nt.x;
  if (same_hemisphere(wo, wi)) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  vec3 wh = -(ni * wo + nt * wi);
  if (!same_hemisphere(wo, wh)) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  const float len = length(wh);
  if (fabsf(len) < 1E-8f) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  wh /= len;
  const float D = ggx_d(wh, L.ax, L.ay);
  const float G1 = ggx_g1(wo, L.ax, L.ay);
  const float G2 = ggx_g2(wo, wi, L.ax, L.ay);
  const float dwh = sqr(nt) * fabsf(dot(wi, wh)) / gmax(sqr(ni * dot(wo, wh) + nt * dot(wi, wh)), 1E-12f);
  const float i_ni = safe_rcp(ni);
  const float c = gmax(dot(wo, wh), 0.0f);
  const float fr = fresnel_dielectric(nt * i_ni, c);
  *pdf = D * G1 * fabsf(dot(wo, wh)) * dwh / gmax(fabsf(wo.z), 1E-8f);
  return L.albedo * (1.0f - fr) * fabsf(dot(wo, wh) / gmax(fabsf(wo.z), 1E-8f)) * G2 * D * dwh * sqr(ni / nt);
}

// ::Sample of the three lobe types (src/BSDF.cuh:205-213, 258-283, 336-374).
static __device__ __noinline__ bool lobe_sample(const Lobe& L, float u0, float u1, vec3 wo, vec3* weight, vec3* wi,
                                                float* pdf) {
  if (L.type == kLambert) {
    const float radius = sqrtf(u0);
    const float phi = u1 * kTwoPi;
    const float dx = radius * cosf(phi), dy = radius * sinf(phi);
    const float r2 = dx * dx + dy * dy;
    *wi = vec3(dx, dy, r2 < 1.0f ? sqrtf(1.0f - r2) : 0.0f);
    const float c = gmax(wi->z, 0.0f);
    *pdf = c * kInvPi;
    *weight = L.albedo;
    return true;
  }
  const vec3 wh = sample_wh(wo, u0, u1, L.ax, L.ay);
  if (!same_hemisphere(wo, wh) || dot(wo, wh) < 0.0f) return false;
  if (L.type == kReflect) {
    *wi = reflect(wo, wh);
    if (!same_hemisphere(*wi, wo)) return false;
    const float D = ggx_d(wh, L.ax, L.ay);
    const float G1 = ggx_g1(wo, L.ax, L.ay);
    const float G2 = ggx_g2(wo, *wi, L.ax, L.ay);
    const float i_ni = safe_rcp(L.ni);
    const float c = gmax(dot(wo, wh), 0.0f);
    const vec3 fr = L.is_metal ? fresnel_conductor(L.nt * i_ni, L.kt * i_ni, c) : vec3(fresnel_dielectric(L.nt.x * i_ni, c));
    *pdf = D * G1 * 0.25f / gmax(wo.z, 1E-8f);
    *weight = L.albedo * G2 * fr / G1;
    return true;
  }
  const float ni = L.ni, nt = L.nt.x;
  if (!refract(wo, wh, ni, nt, wi)) return false;
  if (same_hemisphere(*wi, wo)) return false;
  const float D = ggx_d(wh, L.ax, L.ay);
  const float G1 = ggx_g1(wo, L.ax, L.ay);
  const float G2 = ggx_g2(*wi, wo, L.ax, L.ay);
  const float dwh = sqr(nt) * fabsf(dot(*wi, wh)) / gmax(sqr(ni * dot(wo, wh) + nt * dot(*wi, wh)), 1E-12f);
  const float i_ni = safe_rcp(ni);
  const float c = gmax(dot(wo, wh), 0.0f);
  const float fr = fresnel_dielectric(nt * i_ni, c);
  *pdf = D * G1 * fabsf(dot(wo, wh)) * dwh / gmax(fabsf(wo.z), 1E-8f);
  *weight = L.albedo * (1.0f - fr) * sqr(ni / nt) * G2 / G1;
  return true;
}

// MaterialBSDF::InitShadingSpace without normal or bump maps
// (src/BSDF.cuh:694-807).
__device__ __forceinline__ void init_shading_frame(LayeredBsdf& B, int hit_back, vec3 ray_dir, vec3 ng, vec3 ns, vec3 dpdu,
                                                   vec3 dpdv) {
  vec3 sn = ns;
  if (dot(ns, ng) < 0.0f) sn = -ns;
  vec3 sdpdu = dpdu;
  if (dot(cross(dpdu, dpdv), ng) < 0.0f) sdpdu = -dpdu;
  sdpdu = sdpdu - sn * dot(sdpdu, sn);
  if (!hit_back) {
    B.n = sn;
    B.t = normalize(sdpdu);
    B.b = cross(B.n, B.t);
  } else {
    B.n = -sn;
    B.t = -normalize(sdpdu);
    B.b = -cross(B.n, B.t);
  }
  if (dot(-ray_dir, B.n) < 0.0f) {
    B.n = reflect(B.n, dot(B.n, ng) > 0.0f ? ng : -ng);
    B.t = normalize(B.t - B.n * dot(B.t, B.n));
    B.b = hit_back ? -cross(B.n, B.t) : cross(B.n, B.t);
  }
}

// ------------------------------------------------------ textured surfaces ---

// A material texture read at a surface point: every node type (grids
// included), one out-of-line copy for all callers.
static __device__ __noinline__ vec3 surface_texture(const Texture* __restrict__ tex, uint32_t root, const TexCoord& tc,
                                             uint32_t* errors) {
  return texture_eval<kFeatGrids | kFeatTextures>(tex, root, tc, errors);
}

// Camera::TextureCoordinatesDifferential (src/Camera.h:56-140) with the
// reference's pixel-footprint scales (0.25, 0.25): the texture-coordinate
// footprint (du/dx, dv/dx, du/dy, dv/dy) of a pixel at a hit, from the
// offset camera rays' intersections with the hit's tangent plane (the
// offsets are added to the local -z axis in world-space directions, as the
// reference does). Zero when dp/du, dp/dv are degenerate in the plane the
// geometric normal selects.
__device__ __forceinline__ void tex_differentials(const CameraDesc& cam, vec3 p, vec3 ns, vec3 ng, vec3 dpdu, vec3 dpdv,
                                                  int width, int height, float sx, float sy, float d[4]) {
  vec3 look = cam.position - p;
  const float dist = length(look);
  look *= safe_rcp(dist);
  const vec3 right = normalize(cam.u - look * dot(cam.u, look));
  const vec3 up = cross(look, right);
  const float plane_h = 2.0f * cam.tan_half_fov;
  const float y_off = plane_h * sy / (float)height;
  const float plane_w = plane_h * cam.aspect_ratio;
  const float x_off = plane_w * sx / (float)width;
  auto min_abs = [](float f, float th) { return fabsf(f) < th ? (f > 0.0f ? th : -th) : f; };
  const vec3 dxd = normalize(vec3(0.0f, 0.0f, -1.0f) + right * x_off);
  const vec3 dyd = normalize(vec3(0.0f, 0.0f, -1.0f) + up * y_off);
  const vec3 ln(dot(ns, right), dot(ns, up), dot(ns, look));
  const vec3 lp(0.0f, 0.0f, -dist);
  const float tx = dot(ln, lp) / min_abs(dot(ln, dxd), 1E-4f);
  vec3 dpdx = (dxd * tx - lp) * safe_rcp(sx);
  const float ty = dot(ln, lp) / min_abs(dot(ln, dyd), 1E-4f);
  vec3 dpdy = (dyd * ty - lp) * safe_rcp(sy);
  dpdx = dpdx.x * right + dpdx.y * up + dpdx.z * look;
  dpdy = dpdy.x * right + dpdy.y * up + dpdy.z * look;
  const vec3 an = vabs(ng);
  int a0, a1;
  if (an.z > an.y && an.z > an.x) {
    a0 = 0;
    a1 = 1;
  } else if (an.y > an.x) {
    a0 = 0;
    a1 = 2;
  } else {
    a0 = 1;
    a1 = 2;
  }
  const float m00 = dpdu[a0], m01 = dpdv[a0], m10 = dpdu[a1], m11 = dpdv[a1];
  const float det = m00 * m11 - m10 * m01;
  if (fabsf(det) < 1E-7f) {
    d[0] = d[1] = d[2] = d[3] = 0.0f;
    return;
  }
  const float idet = 1.0f / det;
  d[0] = (m11 * dpdx[a0] - m01 * dpdx[a1]) * idet;
  d[1] = (-m10 * dpdx[a0] + m00 * dpdx[a1]) * idet;
  d[2] = (m11 * dpdy[a0] - m01 * dpdy[a1]) * idet;
  d[3] = (-m10 * dpdy[a0] + m00 * dpdy[a1]) * idet;
}

// MaterialBSDF::InitShadingSpace (src/BSDF.cuh:694-807) with normal mapping
// (the node's rgb * 2 - 1 as tangent-space normal) or bump mapping (the
// height node's first channel, differenced over the pixel's texture
// footprint, at least 0.0005, along the tangents).
static __device__ __noinline__ void init_shading_frame_mapped(LayeredBsdf& B, const DefaultMtl& m, int hit_back, vec3 ray_dir,
                                                       const SurfacePoint& sp, const mat4& wto, const DeviceScene& S,
                                                       const TexCoord& tc, uint32_t* errors) {
  vec3 sn = sp.ns;
  if (dot(sp.ns, sp.ng) < 0.0f) sn = -sp.ns;
  vec3 su = sp.dpdu;
  if (dot(cross(sp.dpdu, sp.dpdv), sp.ng) < 0.0f) su = -sp.dpdu;
  vec3 sv = sp.dpdv;
  su = su - sn * dot(su, sn);
  sv = sv - sn * dot(sv, sn);
  auto frame = [&](vec3 n, vec3 du) {
    if (!hit_back) {
      B.n = n;
      B.t = normalize(du);
      B.b = cross(B.n, B.t);
    } else {
      B.n = -n;
      B.t = -normalize(du);
      B.b = -cross(B.n, B.t);
    }
  };
  if (m.normal_mapping_tex != kEmpty) {
    frame(sn, su);
    const vec3 tn = normalize(surface_texture(S.textures, m.normal_mapping_tex, tc, errors) * 2.0f - vec3(1.0f));
    B.n = tn.x * B.t + tn.y * B.b + tn.z * B.n;
    B.t = normalize(B.t - B.n * dot(B.t, B.n));
    B.b = hit_back ? -cross(B.n, B.t) : cross(B.n, B.t);
  } else if (m.bump_mapping_tex != kEmpty) {
    float d[4];
    tex_differentials(S.camera, sp.p, sp.ns, sp.ng, sp.dpdu, sp.dpdv, S.width, S.height, 0.25f, 0.25f, d);
    const vec3 ou = transform_vector(wto, su), ov = transform_vector(wto, sv);
    float du = gmax((fabsf(d[0]) + fabsf(d[2])) * 0.5f, 0.0005f);
    if (!(du > 0.0f)) du = 0.0005f;
    TexCoord bc{tc.s + du, tc.t, tc.p + ou * du};
    const float hu = surface_texture(S.textures, m.bump_mapping_tex, bc, errors).x;
    float dv = gmax((fabsf(d[1]) + fabsf(d[3])) * 0.5f, 0.0005f);
    if (!(dv > 0.0f)) dv = 0.0005f;
    bc = TexCoord{tc.s, tc.t + dv, tc.p + ov * dv};
    const float hv = surface_texture(S.textures, m.bump_mapping_tex, bc, errors).x;
    const float h = surface_texture(S.textures, m.bump_mapping_tex, tc, errors).x;
    su = su + (hu - h) * safe_rcp(du) * sn;
    sv = sv + (hv - h) * safe_rcp(dv) * sn;
    sn = normalize(cross(su, sv));
    frame(sn, su);
  } else {
    frame(sn, su);
  }
  if (dot(-ray_dir, B.n) < 0.0f) {
    B.n = reflect(B.n, dot(B.n, sp.ng) > 0.0f ? sp.ng : -sp.ng);
    B.t = normalize(B.t - B.n * dot(B.t, B.n));
    B.b = hit_back ? -cross(B.n, B.t) : cross(B.n, B.t);
  }
}

// The textured parameters of a default material, read at the hit
// (DefaultMtlBSDF::InitBSDFSettings' fetch_float / fetch_color,
// src/BSDF.cuh:463-498): a float parameter takes its node's first channel.
// Unlike the constants, the values are not clamped at load.
static __device__ __noinline__ void resolve_material_textures(DefaultMtl& m, const Texture* __restrict__ tex,
                                                       const TexCoord& tc, uint32_t* errors) {
  auto f = [&](uint32_t t, float* v) {
    if (t != kEmpty) *v = surface_texture(tex, t, tc, errors).x;
  };
  auto c = [&](uint32_t t, vec3* v) {
    if (t != kEmpty) *v = surface_texture(tex, t, tc, errors);
  };
  f(m.coat_weight_tex, &m.coat_weight);
  f(m.metalness_tex, &m.metalness);
  f(m.alpha_x_tex, &m.alpha_x);
  f(m.alpha_y_tex, &m.alpha_y);
  f(m.specular_weight_tex, &m.specular_weight);
  f(m.transmission_weight_tex, &m.transmission_weight);
  c(m.diffuse_albedo_tex, &m.diffuse_albedo);
  c(m.specular_albedo_tex, &m.specular_albedo);
  f(m.coat_thickness_tex, &m.coat_thickness);
  f(m.coat_roughness_x_tex, &m.coat_roughness_x);
  f(m.coat_roughness_y_tex, &m.coat_roughness_y);
  c(m.coat_albedo_tex, &m.coat_albedo);
}

__device__ __forceinline__ bool material_textured(const DefaultMtl& m) {
  return (m.diffuse_albedo_tex & m.specular_albedo_tex & m.alpha_x_tex & m.alpha_y_tex & m.specular_weight_tex &
          m.metalness_tex & m.transmission_weight_tex & m.coat_albedo_tex & m.coat_weight_tex & m.coat_thickness_tex &
          m.coat_roughness_x_tex & m.coat_roughness_y_tex & m.normal_mapping_tex & m.bump_mapping_tex) != kEmpty;
}

// DefaultMtlBSDF::InitBSDFSettings with constant parameters (src/BSDF.cuh:453-618).
__device__ __forceinline__ void init_layered_lobes(LayeredBsdf& B, const DefaultMtl& m, vec3 ray_dir, int hit_back,
                                                   float ray_ior, float ex_ior) {
  const float ior_min = 0.0001f;
  const float coat_weight = m.coat_weight;
  const float ior_in = gmax(ray_ior, ior_min);
  const float ior_coat = gmax(m.coat_ior, ior_min);
  const float ior_out = gmax(hit_back ? ex_ior : m.ior_n, ior_min);
  const float eta_in_coat = ior_coat * safe_rcp(ior_in);
  const float eta_in_out = ior_out * safe_rcp(ior_in);
  const float cos_in = gmax(dot(B.n, -ray_dir), 0.0f);
  const float fr_in_coat = coat_weight > 0.0f ? fresnel_dielectric(eta_in_coat, cos_in) : 1.0f;
  const float fr_in_out = fresnel_dielectric(eta_in_out, cos_in);
  const float metalness = m.metalness;
  const float ax = sqr(gclamp(m.alpha_x, 0.001f, 0.999f));
  const float ay = sqr(gclamp(m.alpha_y, 0.001f, 0.999f));
  const float specular_weight = m.specular_weight;
  const float transmission_weight = m.transmission_weight;
  const vec3 diffuse_albedo = m.diffuse_albedo;
  const vec3 specular_albedo = m.specular_albedo;
  const float coat_thickness = m.coat_thickness;
  const float coat_ax = sqr(gclamp(m.coat_roughness_x, 0.001f, 0.999f));
  const float coat_ay = sqr(gclamp(m.coat_roughness_y, 0.001f, 0.999f));
  const vec3 coat_albedo = m.coat_albedo;
  const vec3 coat_sigma = -vlog(vmax(coat_albedo, vec3(1E-8f))) * coat_thickness;
  const vec3 coat_tr = vexp(-coat_sigma * safe_rcp(cos_in));

  float wsum = 0.0f;
  int n = 0;
  const vec3 coat_color = vec3(coat_weight * fr_in_coat);
  const float coat_lum = luminance(coat_color);
  if (coat_lum > 0.0f) {
    Lobe& L = B.lobe[n];
    L.type = kReflect;
    L.albedo = coat_color;
    L.ax = coat_ax;
    L.ay = coat_ay;
    L.nt = vec3(ior_coat);
    L.kt = vec3(0.0f);
    L.ni = ior_in;
    L.is_metal = 0;
    L.role = kRoleCoat;
    B.w[n] = coat_lum;
    wsum += coat_lum;
    ++n;
  }
  const vec3 tint = (1.0f - coat_weight * fr_in_coat) * linear_lerp(vec3(1.0f), coat_tr, coat_weight);
  const vec3 metal_color = tint * metalness;
  const float metal_lum = luminance(metal_color);
  if (metal_lum > 0.0f) {
    vec3 mn, mk;
    edge_tint_to_conductor(diffuse_albedo, specular_albedo, &mn, &mk);
    Lobe& L = B.lobe[n];
    L.type = kReflect;
    L.albedo = metal_color;
    L.ax = ax;
    L.ay = ay;
    L.nt = mn;
    L.kt = mk;
    L.ni = ior_in;
    L.is_metal = 1;
    L.role = kRoleMetal;
    B.w[n] = metal_lum;
    wsum += metal_lum;
    ++n;
  }
  const float spec_fr = fr_in_out;
  const vec3 spec_color = tint * (1.0f - metalness) * spec_fr * specular_weight * specular_albedo;
  const float spec_lum = luminance(spec_color);
  if (spec_lum > 0.0f) {
    Lobe& L = B.lobe[n];
    L.type = kReflect;
    L.albedo = spec_color;
    L.ax = ax;
    L.ay = ay;
    L.nt = vec3(ior_out);
    L.kt = vec3(0.0f);
    L.ni = ior_in;
    L.is_metal = 0;
    L.role = kRoleSpecular;
    B.w[n] = spec_lum;
    wsum += spec_lum;
    ++n;
  }
  const vec3 trans_color = tint * (1.0f - metalness) * (1.0f - spec_fr * specular_weight) * transmission_weight * specular_albedo;
  const float trans_lum = luminance(trans_color);
  if (trans_lum > 0.0f) {
    Lobe& L = B.lobe[n];
    L.type = kTransmit;
    L.albedo = trans_color;
    L.ax = ax;
    L.ay = ay;
    L.ni = ior_in;
    L.nt = vec3(ior_out);
    L.kt = vec3(0.0f);
    L.is_metal = 0;
    L.role = kRoleTransmission;
    B.w[n] = trans_lum;
    wsum += trans_lum;
    ++n;
  }
  const vec3 diff_color =
      tint * (1.0f - metalness) * (1.0f - spec_fr * specular_weight) * (1.0f - transmission_weight) * diffuse_albedo;
  const float diff_lum = luminance(diff_color);
  {
    Lobe& L = B.lobe[n];
    L.type = kLambert;
    L.albedo = diff_color;
    L.ax = L.ay = 0.0f;
    L.ni = 1.0f;
    L.nt = L.kt = vec3(0.0f);
    L.is_metal = 0;
    L.role = kRoleDiffuse;
    B.w[n] = diff_lum;
    wsum += diff_lum;
    ++n;
  }
  B.count = n;
  if (wsum > 0.0f) {
    const float iw = safe_rcp(wsum);
    for (int i = 0; i < n; ++i) B.w[i] *= iw;
  } else {
    const float iw = 1.0f / (float)n;
    for (int i = 0; i < n; ++i) B.w[i] = iw;
  }
}

// DefaultMtlBSDF::EvalWi (src/BSDF.cuh:619-632).
__device__ __forceinline__ vec3 bsdf_eval(const LayeredBsdf& B, vec3 wo, vec3 wi, float* pdf) {
  vec3 f(0.0f);
  float p = 0.0f;
  for (int i = 0; i < B.count; ++i) {
    float lp = 0.0f;
    f += lobe_eval(B.lobe[i], wo, wi, &lp);
    p += B.w[i] * lp;
  }
  *pdf = p;
  return f;
}

// DefaultMtlBSDF::SampleWi (src/BSDF.cuh:633-679).
__device__ __forceinline__ bool bsdf_sample(const LayeredBsdf& B, vec3 wo, vec3* weight, vec3* wi, float* pdf, float u0,
                                            float u1, float u2) {
  float cdf = 0.0f;
  int sel = -1;
  for (int i = 0; i < B.count; ++i) {
    if (u0 < cdf + B.w[i]) {
      sel = i;
      break;
    }
    cdf += B.w[i];
  }
  if (sel == -1) sel = B.count - 1;
  if (sel == -1) return false;
  float sp = 0.0f;
  if (!lobe_sample(B.lobe[sel], u1, u2, wo, weight, wi, &sp)) return false;
  float mix_pdf = sp * B.w[sel];
  vec3 mix_f = (*weight) * sp;
  for (int i = 0; i < B.count; ++i) {
    if (i == sel) continue;
    float lp;
    mix_f += lobe_eval(B.lobe[i], wo, *wi, &lp);
    mix_pdf += B.w[i] * lp;
  }
  *pdf = mix_pdf;
  *weight = mix_f * safe_rcp(mix_pdf);
  return true;
}

// -------------------------------------------------------------- lights ---

__device__ __forceinline__ float power_heuristic(float main_pdf, float vice_pdf) {
  return safe_rcp(1.0f + sqr(vice_pdf * safe_rcp(main_pdf)));
}

// SampleLightPower (src/Light.h:398-415).
__device__ __forceinline__ int sample_light_power(const DeviceScene& S, float u0, float* pdf) {
  const float* tab = S.shape_light_table;
  const int count = (int)S.shape_light_count;
  int left = 0, right = count;
  while (left < right) {
    const int mid = (left + right) / 2;
    if (tab[mid] <= u0) left = mid + 1;
    else right = mid;
  }
  const int idx = gmin(left, count - 1);
  *pdf = idx == 0 ? tab[idx] : (tab[idx] - tab[idx - 1]);
  return idx;
}

// One shape light: a triangle of a mesh instance, or a whole sphere.
struct LightTri {
  vec3 p0, p1, p2, n0, n1, n2, color;
  float intensity;
  const mat4* otw;
  const mat4* wto;
  bool sphere;
  float radius;
};
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ LightTri load_light_tri(const DeviceScene& S, const ShapeLight& L) {
  LightTri lt;
  const Instance inst = S.instances[L.instance_idx];
  const Material& mat = S.materials[inst.material_idx];
  const GeometryDesc& g = S.geometries[inst.geometry_idx];
  lt.color = mat.light_mtl.light_color;
  lt.intensity = mat.light_mtl.intensity;
  lt.otw = &S.transforms[inst.transform_idx];
  lt.wto = &S.i_transforms[inst.transform_idx];
  lt.sphere = (kF & kFeatSpheres) && g.kind == kGeoSphere;
  lt.radius = g.radius;
  if (lt.sphere) return lt;
  const uint32_t* tc = S.tri_corners + 3 * (size_t)(g.tri_offset + L.triangle_idx);
  vec3* P[3] = {&lt.p0, &lt.p1, &lt.p2};
  vec3* N[3] = {&lt.n0, &lt.n1, &lt.n2};
  for (int k = 0; k < 3; ++k) {
    const uint32_t vi = S.pos_idx[g.corner_offset + tc[k]];
    const float* a = S.positions + 3 * (size_t)(g.pos_offset + vi);
    *P[k] = vec3(a[0], a[1], a[2]);
    const uint32_t ni = S.nrm_idx[g.corner_offset + tc[k]];
    const float* b = S.normals + 3 * (size_t)(g.nrm_offset + ni);
    *N[k] = vec3(b[0], b[1], b[2]);
  }
  return lt;
}

// SampleCone (src/SampleUtilities.h:33-39).
__device__ __forceinline__ vec3 sample_cone(float u0, float u1, float cos_theta_max) {
  const float c = (1.0f - u0) + u0 * cos_theta_max;
  const float sn = sqrtf(gmax(0.0f, 1.0f - c * c));
  const float phi = u1 * 2.0f * kPi;
  return vec3(cosf(phi) * sn, sinf(phi) * sn, c);
}

// ShapeLight::SampleLi, spheres (src/Light.h:282-314): a direction in the
// cone the sphere subtends, solid-angle pdf. Both sphere-light functions are
// out of line: they run only for sphere lights, and inlined they would add
// registers to every light evaluation.
static __device__ __noinline__ bool sphere_light_sample_li(const LightTri& lt, vec3 position, float u0, float u1, vec3* wi,
                                                       vec3* lpos, vec3* lpos_err, vec3* lng, vec3* Li, float* pdf) {
  const vec3 op = transform_position(*lt.wto, position);
  const float lpo = length(op);
  const float r = lt.radius;
  if (lpo < r) {
    *pdf = 0.0f;
    return false;
  }
  const float ctm = sqrtf(gmax(sqr(lpo) - sqr(r), 0.0f)) / lpo;
  const float cone = 2.0f * kPi * (1.0f - ctm);
  vec3 cs = sample_cone(u0, u1, ctm);
  vec3 w = -op, u, v;
  orthogonal_basis(w, u, v);
  cs = cs.x * u + cs.y * v + cs.z * w;
  float t0, t1;
  sphere_solve(op, cs, r, &t0, &t1);
  vec3 ip = op + cs * t0;
  const float lio = length(ip);
  ip *= r * safe_rcp(lio);
  vec3 err = error_gamma(5) * vabs(ip);
  *lpos = transform_position(*lt.otw, ip, &err);
  *lpos_err = err;
  *lng = normalize(*lpos - get_translate(*lt.otw));
  *wi = normalize(transform_vector(*lt.otw, cs));
  *pdf = 1.0f / cone;
  *Li = lt.color * lt.intensity * cone;
  return true;
}

// ShapeLight::EvalLi, spheres (src/Light.h:163-200).
static __device__ __noinline__ vec3 sphere_light_eval_li(const LightTri& lt, vec3 position, vec3 wi, vec3* lpos,
                                                     vec3* lpos_err, vec3* lng, float* pdf) {
  const vec3 owi = transform_vector(*lt.wto, wi);
  const vec3 op = transform_position(*lt.wto, position);
  const float lpo = length(op);
  const float r = lt.radius;
  if (lpo < r) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  float t0, t1;
  if (!sphere_solve(op, owi, r, &t0, &t1)) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  const float ctm = sqrtf(gmax(sqr(lpo) - sqr(r), 0.0f)) / lpo;
  const float cone = 2.0f * kPi * (1.0f - ctm);
  const float ct = dot(normalize(owi), -op / lpo);
  if (ct < ctm) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  vec3 ip = op + owi * t0;
  const float lio = length(ip);
  ip *= r * safe_rcp(lio);
  vec3 err = error_gamma(5) * vabs(ip);
  *lpos = transform_position(*lt.otw, ip, &err);
  *lpos_err = err;
  *lng = normalize(*lpos - get_translate(*lt.otw));
  *pdf = 1.0f / cone;
  return lt.color * lt.intensity;
}

// ShapeLight::SampleLi, triangle meshes (src/Light.h:207-264), and spheres.
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ bool light_sample_li(const LightTri& lt, float area, vec3 position, float u0, float u1, vec3* wi,
                                                vec3* lpos, vec3* lpos_err, vec3* lng, vec3* Li, float* pdf) {
  if ((kF & kFeatSpheres) && lt.sphere) return sphere_light_sample_li(lt, position, u0, u1, wi, lpos, lpos_err, lng, Li, pdf);
  const vec3 geo_n = cross(lt.p1 - lt.p0, lt.p2 - lt.p0);
  const float su = sqrtf(gmax(0.0f, u0));
  const float bu = 1.0f - su;
  const float bv = u1 * su;
  const vec3 bary(bu, bv, 1.0f - bu - bv);
  const float xs = fabsf(lt.p0.x * bary.x) + fabsf(lt.p1.x * bary.y) + fabsf(lt.p2.x * bary.z);
  const float ys = fabsf(lt.p0.y * bary.x) + fabsf(lt.p1.y * bary.y) + fabsf(lt.p2.y * bary.z);
  const float zs = fabsf(lt.p0.z * bary.x) + fabsf(lt.p1.z * bary.y) + fabsf(lt.p2.z * bary.z);
  const vec3 sp = lt.p0 * bary.x + lt.p1 * bary.y + lt.p2 * bary.z;
  vec3 serr = error_gamma(7) * vec3(xs, ys, zs);
  const vec3 sn = lt.n0 * bary.x + lt.n1 * bary.y + lt.n2 * bary.z;
  const vec3 wn = normalize(xform_transpose_dir_glm(*lt.wto, sn));
  *lpos = transform_position(*lt.otw, sp, &serr);
  *lpos_err = serr;
  *lng = normalize(transpose_transform_vector(*lt.wto, geo_n));
  const float dist = length(*lpos - position);
  *wi = (*lpos - position) * safe_rcp(dist);
  const float ct = -dot(wn, *wi);
  if (ct <= 0.0f) {
    *pdf = 0.0f;
    return false;
  }
  *pdf = sqr(dist) * safe_rcp(area * ct);
  *Li = lt.color * lt.intensity / (*pdf);
  return true;
}

// ShapeLight::EvalLi, triangle meshes (src/Light.h:97-155), with
// RayIntersectTriangle's glm 3x3 inverse (src/Light.h:14-40).
template <uint32_t kF = kFeatAll>
__device__ __forceinline__ vec3 light_eval_li(const LightTri& lt, float area, vec3 position, vec3 wi, vec3* lpos,
                                              vec3* lpos_err, vec3* lng, float* pdf) {
  if ((kF & kFeatSpheres) && lt.sphere) return sphere_light_eval_li(lt, position, wi, lpos, lpos_err, lng, pdf);
  const vec3 geo_n = cross(lt.p1 - lt.p0, lt.p2 - lt.p0);
  const vec3 owi = transform_vector(*lt.wto, wi);
  const vec3 opos = transform_position(*lt.wto, position);
  const vec3 p20 = lt.p0 - lt.p2, p21 = lt.p1 - lt.p2;
  mat3 m;
  m.m[0][0] = p20.x; m.m[0][1] = p20.y; m.m[0][2] = p20.z;
  m.m[1][0] = p21.x; m.m[1][1] = p21.y; m.m[1][2] = p21.z;
  m.m[2][0] = -owi.x; m.m[2][1] = -owi.y; m.m[2][2] = -owi.z;
  const vec3 params = mul3(inverse3(m), opos - lt.p2);
  const float u = params.x, v = params.y, t = params.z;
  const float w = 1.0f - u - v;
  if (t < kTMin) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  const vec3 bary(u, v, w);
  if (!((u > 0.0f && u < 1.0f) && (v > 0.0f && v < 1.0f) && (w > 0.0f && w < 1.0f))) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  const float xs = fabsf(lt.p0.x * bary.x) + fabsf(lt.p1.x * bary.y) + fabsf(lt.p2.x * bary.z);
  const float ys = fabsf(lt.p0.y * bary.x) + fabsf(lt.p1.y * bary.y) + fabsf(lt.p2.y * bary.z);
  const float zs = fabsf(lt.p0.z * bary.x) + fabsf(lt.p1.z * bary.y) + fabsf(lt.p2.z * bary.z);
  const vec3 sp = lt.p0 * bary.x + lt.p1 * bary.y + lt.p2 * bary.z;
  vec3 serr = error_gamma(7) * vec3(xs, ys, zs);
  const vec3 sn = lt.n0 * bary.x + lt.n1 * bary.y + lt.n2 * bary.z;
  const vec3 wn = normalize(xform_transpose_dir_glm(*lt.wto, sn));
  const float ct = -dot(wn, wi);
  if (ct <= 0.0f) {
    *pdf = 0.0f;
    return vec3(0.0f);
  }
  *lpos = transform_position(*lt.otw, sp, &serr);
  *lpos_err = serr;
  *lng = normalize(transpose_transform_vector(*lt.wto, geo_n));
  const float dist = length(*lpos - position);
  *pdf = sqr(dist) * safe_rcp(area * ct);
  return lt.color * lt.intensity;
}

// Background gradient (src/Shading.cu:35-38).
__device__ __forceinline__ vec3 background(vec3 d) {
  return mix(vec3(1.0f), vec3(0.05f, 0.2f, 0.85f), d.y * 0.5f + 0.5f);
}

// indirect_light_clamp (src/Shading.cu:61-81).
__device__ __forceinline__ vec3 indirect_clamp(const RenderSetting& rs, vec3 c, int depth) {
  if (!(rs.enable_indirect_clamp && depth > 1)) return c;
  if (!(rs.indirect_limit > 0.0f)) return vec3(0.0f);
  const float lum = luminance(c);
  if (lum <= 1E-10f) return c;
  const float limit = rs.indirect_limit;
  const float pw = gmin(0.05f + 0.25f * (powf(lum / limit, 1.5f)), 1.0f);
  const float sf = powf(limit / (limit + lum), pw);
  return c * sf;
}

}  // namespace ym
