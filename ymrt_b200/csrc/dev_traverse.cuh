// Two-level ray traversal over compressed 8-wide BVHs (sm_100a).
//
// Semantics follow the reference's TraceRay / IntersectMeshObject /
// IntersectTri / IntersectSphereObject / BVHTraverseShadow
// (src/ShadingUtilities.cuh:54-276, 310-431, 563-635): world rays are carried into each instance with the
// instance's inverse transform (glm mat4*vec4 order), triangles are tested
// with the watertight test in the reference's exact float order (so t and the
// barycentrics are bit-identical), a hit is kept when TMIN <= t <= current t
// (a later hit at an equal t replaces the earlier one), and the "nearby hits"
// list for nested media records every instance whose hit lies within two
// ulps of the final t.
//
// The acceleration structure is this project's: each node holds 8 child boxes
// quantised to bytes on a per-node power-of-two grid (80-byte nodes, five
// 128-bit read-only loads), leaves hold up to three triangles stored as three
// float4 vertices (no index indirection), and the traversal stack lives in
// shared memory (spilling to a short local-memory tail). Box tests use fused
// multiply-adds and are widened by a few ulps so that they are conservative:
// they only decide which triangles are tested, never the hit itself.
#pragma once

#include "dev_constants.cuh"
#include "sphere.h"
#include "ymrt_scene.h"

namespace ym {

constexpr int kStackShared = 32;  // entries per thread in shared memory
constexpr int kStackLocal = 64;   // further entries per thread in local memory
constexpr int kTraceBlock = 128;  // threads per block of the traversal kernels (default)
constexpr int kMaxTraceBlock = 256;  // largest block k_extend and k_connect are launched with

// Stack entries carry the entry distance of the box that produced them, so a
// pop can drop entries that lie beyond the current closest hit. An entry with
// kInstanceEntry set names a top-level instance to enter.
constexpr uint32_t kInstanceEntry = 0x80000000u;

struct TraversalStack {
  uint32_t* sh;   // shared-memory column of this thread: entries (stride: the block's threads)
  float* sht;     // shared-memory column of this thread: entry distances
  uint32_t loc[kStackLocal];
  float loct[kStackLocal];
  int sp;
  int stride;
  bool overflow;
  __device__ __forceinline__ void bind(uint32_t* shared_entries, float* shared_t) {
    sh = shared_entries + threadIdx.x;
    sht = shared_t + threadIdx.x;
    stride = (int)blockDim.x;
    sp = 0;
    overflow = false;
  }
  __device__ __forceinline__ void push(uint32_t v, float t = 0.0f) {
    if (sp < kStackShared) {
      sh[sp * stride] = v;
      sht[sp * stride] = t;
    } else if (sp < kStackShared + kStackLocal) {
      loc[sp - kStackShared] = v;
      loct[sp - kStackShared] = t;
    } else {
      overflow = true;
      return;
    }
    ++sp;
  }
  __device__ __forceinline__ uint32_t pop(float* t) {
    --sp;
    if (sp < kStackShared) {
      *t = sht[sp * stride];
      return sh[sp * stride];
    }
    *t = loct[sp - kStackShared];
    return loc[sp - kStackShared];
  }
};

// Shared-memory backing of the traversal stacks of one kTraceBlock block.
#define YM_TRAVERSAL_SHARED(name)                                      \
  __shared__ uint32_t name##_entries[kStackShared * kTraceBlock];      \
  __shared__ float name##_t[kStackShared * kTraceBlock]
// The same, in the dynamic shared memory of a kernel launched with any block
// size up to kMaxTraceBlock (traversal_shared_bytes of it).
#define YM_TRAVERSAL_SHARED_DYNAMIC(name)                                              \
  extern __shared__ __align__(16) uint32_t name##_dyn[];                               \
  uint32_t* name##_entries = name##_dyn;                                               \
  float* name##_t = reinterpret_cast<float*>(name##_dyn + kStackShared * blockDim.x)
constexpr size_t traversal_shared_bytes(uint32_t block) { return (size_t)kStackShared * block * 8u; }

// The far end of the box-test interval for a ray whose closest hit so far is
// at t: boxes are widened by 1e-6 relative, and so is this bound, so a box
// entered beyond it cannot hold a hit at or near t.
__device__ __forceinline__ float widened_tmax(float t) { return __fmaf_rn(fabsf(t), 1e-6f, t); }

// Ray set-up shared by every triangle test of one object-space ray: the
// reference recomputes these in each IntersectTri call; they are the same
// numbers each time.
struct TriRay {
  vec3 o, d;
  int kx, ky, kz;
  float sx, sy, sz;
};
__device__ __forceinline__ TriRay make_tri_ray(vec3 o, vec3 d) {
  TriRay r;
  r.o = o;
  r.d = d;
  r.kz = max_dimension(vabs(d));
  r.kx = r.kz + 1; if (r.kx == 3) r.kx = 0;
  r.ky = r.kx + 1; if (r.ky == 3) r.ky = 0;
  const vec3 dd(d[r.kx], d[r.ky], d[r.kz]);
  r.sx = -dd.x / dd.z;
  r.sy = -dd.y / dd.z;
  r.sz = 1.f / dd.z;
  return r;
}

// Watertight ray/triangle test, IntersectTri (src/ShadingUtilities.cuh:54-134).
// Returns false when the edge tests fail; otherwise t (may be outside range)
// and the three unnormalised edge values with 1/den.
__device__ __forceinline__ bool tri_test(const TriRay& R, vec3 p0, vec3 p1, vec3 p2, float* t_out, float* e_out,
                                         float* inv_den_out) {
  p0 = p0 - R.o;
  p1 = p1 - R.o;
  p2 = p2 - R.o;
  p0 = vec3(p0[R.kx], p0[R.ky], p0[R.kz]);
  p1 = vec3(p1[R.kx], p1[R.ky], p1[R.kz]);
  p2 = vec3(p2[R.kx], p2[R.ky], p2[R.kz]);
  p0.x += R.sx * p0.z;
  p0.y += R.sy * p0.z;
  p1.x += R.sx * p1.z;
  p1.y += R.sy * p1.z;
  p2.x += R.sx * p2.z;
  p2.y += R.sy * p2.z;
  const float e0 = p1.x * p2.y - p1.y * p2.x;
  const float e1 = p2.x * p0.y - p2.y * p0.x;
  const float e2 = p0.x * p1.y - p0.y * p1.x;
  if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return false;
  const float den = e0 + e1 + e2;
  if (den == 0) return false;
  p0.z *= R.sz;
  p1.z *= R.sz;
  p2.z *= R.sz;
  const float inv = 1.0f / den;
  float t = e0 * p0.z + e1 * p1.z + e2 * p2.z;
  t *= inv;
  *t_out = t;
  e_out[0] = e0;
  e_out[1] = e1;
  e_out[2] = e2;
  *inv_den_out = inv;
  return true;
}

__device__ __forceinline__ void load_tri(const float4* __restrict__ wtris, uint32_t i, vec3* p0, vec3* p1, vec3* p2,
                                         uint32_t* id) {
  const float4 a = __ldg(wtris + 3 * (size_t)i);
  const float4 b = __ldg(wtris + 3 * (size_t)i + 1);
  const float4 c = __ldg(wtris + 3 * (size_t)i + 2);
  *p0 = vec3(a.x, a.y, a.z);
  *p1 = vec3(b.x, b.y, b.z);
  *p2 = vec3(c.x, c.y, c.z);
  *id = __float_as_uint(a.w);
}

// Per-ray constants for box tests.
struct BoxRay {
  float ox, oy, oz, ix, iy, iz;
};
__device__ __forceinline__ BoxRay make_box_ray(vec3 o, vec3 d) {
  BoxRay b;
  b.ox = o.x; b.oy = o.y; b.oz = o.z;
  b.ix = 1.0f / d.x; b.iy = 1.0f / d.y; b.iz = 1.0f / d.z;
  return b;
}

__device__ __forceinline__ float byte_of(uint32_t w, int k) { return (float)((w >> (8 * k)) & 0xFFu); }

// Tests the 8 child boxes of a node. Returns a mask of hit children; tnear
// receives each hit child's entry distance.
__device__ __forceinline__ uint32_t intersect_children(const uint4* __restrict__ nodes_u4, uint32_t node, const BoxRay& r,
                                                       float tmax, float tnear_out[8], uint32_t* imask,
                                                       uint32_t* child_base, uint32_t* prim_base, uint32_t meta[2]) {
  const uint4* p = nodes_u4 + 5 * (size_t)node;
  const uint4 w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3), w4 = __ldg(p + 4);
  const float nox = __uint_as_float(w0.x), noy = __uint_as_float(w0.y), noz = __uint_as_float(w0.z);
  const float sx = __uint_as_float((w0.w & 0xFFu) << 23);
  const float sy = __uint_as_float(((w0.w >> 8) & 0xFFu) << 23);
  const float sz = __uint_as_float(((w0.w >> 16) & 0xFFu) << 23);
  *imask = w0.w >> 24;
  *child_base = w1.x;
  *prim_base = w1.y;
  meta[0] = w1.z;
  meta[1] = w1.w;
  // t = (origin + q * scale - o) * inv = q * (scale * inv) + (origin - o) * inv
  const float ax = sx * r.ix, bx = (nox - r.ox) * r.ix;
  const float ay = sy * r.iy, by = (noy - r.oy) * r.iy;
  const float az = sz * r.iz, bz = (noz - r.oz) * r.iz;
  // byte planes: w2 = qlo_x[0..7], qlo_y[0..7]; w3 = qlo_z, qhi_x; w4 = qhi_y, qhi_z
  const bool negx = r.ix < 0.0f, negy = r.iy < 0.0f, negz = r.iz < 0.0f;
  uint32_t hits = 0;
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int k = c & 3;
    const uint32_t lox = c < 4 ? w2.x : w2.y, loy = c < 4 ? w2.z : w2.w;
    const uint32_t loz = c < 4 ? w3.x : w3.y, hix = c < 4 ? w3.z : w3.w;
    const uint32_t hiy = c < 4 ? w4.x : w4.y, hiz = c < 4 ? w4.z : w4.w;
    const float qlx = byte_of(lox, k), qhx = byte_of(hix, k);
    const float qly = byte_of(loy, k), qhy = byte_of(hiy, k);
    const float qlz = byte_of(loz, k), qhz = byte_of(hiz, k);
    const float t0x = __fmaf_rn(negx ? qhx : qlx, ax, bx), t1x = __fmaf_rn(negx ? qlx : qhx, ax, bx);
    const float t0y = __fmaf_rn(negy ? qhy : qly, ay, by), t1y = __fmaf_rn(negy ? qly : qhy, ay, by);
    const float t0z = __fmaf_rn(negz ? qhz : qlz, az, bz), t1z = __fmaf_rn(negz ? qlz : qhz, az, bz);
    float tn = fmaxf(fmaxf(t0x, t0y), fmaxf(t0z, 0.0f));
    float tf = fminf(fminf(t1x, t1y), fminf(t1z, tmax));
    tn = __fmaf_rn(-fabsf(tn), 1e-6f, tn);
    tf = __fmaf_rn(fabsf(tf), 1e-6f, tf);
    const uint32_t m = (c < 4 ? meta[0] : meta[1]) >> (8 * k) & 0xFFu;
    const bool occupied = ((*imask >> c) & 1u) || m != 0;
    if (occupied && tn <= tf) {
      hits |= 1u << c;
      tnear_out[c] = tn;
    }
  }
  return hits;
}

__device__ __forceinline__ uint32_t child_meta(const uint32_t meta[2], int c) {
  return (c < 4 ? meta[0] : meta[1]) >> (8 * (c & 3)) & 0xFFu;
}

// Branch-free ordering of the hit children of one node: keys hold the entry
// distance (non-negative, so its bits order like the float) with the child
// slot in the low three bits, misses sort last. The 19-comparator network is
// the optimal sorting network for 8 keys.
__device__ __forceinline__ void sort8(uint32_t k[8]) {
#define YM_CS(a, b)                         \
  {                                         \
    const uint32_t lo = min(k[a], k[b]);    \
    const uint32_t hi = max(k[a], k[b]);    \
    k[a] = lo;                              \
    k[b] = hi;                              \
  }
  YM_CS(0, 1) YM_CS(2, 3) YM_CS(4, 5) YM_CS(6, 7)
  YM_CS(0, 2) YM_CS(1, 3) YM_CS(4, 6) YM_CS(5, 7)
  YM_CS(1, 2) YM_CS(5, 6) YM_CS(0, 4) YM_CS(3, 7)
  YM_CS(1, 5) YM_CS(2, 6)
  YM_CS(1, 4) YM_CS(3, 6)
  YM_CS(2, 4) YM_CS(3, 5)
  YM_CS(3, 4)
#undef YM_CS
}

__device__ __forceinline__ uint32_t child_key(uint32_t mask, const float tnear[8], int c) {
  return ((mask >> c) & 1u) ? ((__float_as_uint(tnear[c]) & ~7u) | (uint32_t)c) : 0xFFFFFFFFu;
}

// Pushes the children in `mask` far-to-near (so the nearest pops first), each
// with its entry distance. Internal children push their node; in a top-level
// node, leaf children push their instances (tlas_prims) as instance entries.
__device__ __forceinline__ void push_children(TraversalStack& st, uint32_t internal, uint32_t leaves,
                                              const float tnear[8], const uint32_t meta[2], uint32_t child_base,
                                              uint32_t prim_base, const uint32_t* __restrict__ tlas_prims) {
  const uint32_t mask = internal | leaves;
  if (mask == 0) return;
  // one child's entries (a node, or the instances of a top-level leaf)
  auto push_one = [&](uint32_t key) {
    const int c = (int)(key & 7u);
    const float t = __uint_as_float(key & ~7u);
    const uint32_t m = child_meta(meta, c);
    if ((internal >> c) & 1u) {
      st.push(child_base + m, t);
    } else {
      for (uint32_t k = 0; k < (m >> 5); ++k) st.push(kInstanceEntry | __ldg(tlas_prims + prim_base + (m & 31u) + k), t);
    }
  };
  uint32_t key[8];
#pragma unroll
  for (int c = 0; c < 8; ++c) key[c] = child_key(mask, tnear, c);
  const int n = __popc(mask);
  if (n <= 2) {
    // one or two children: the nearest key is the least, the other the
    // greatest below 0xFFFFFFFF (the order the network gives)
    uint32_t lo = key[0], hi = 0u;
#pragma unroll
    for (int c = 1; c < 8; ++c) lo = min(lo, key[c]);
#pragma unroll
    for (int c = 0; c < 8; ++c) hi = max(hi, key[c] == 0xFFFFFFFFu ? 0u : key[c]);
    if (n == 2) push_one(hi);
    push_one(lo);
    return;
  }
  sort8(key);
#pragma unroll
  for (int j = 7; j >= 0; --j)
    if (key[j] != 0xFFFFFFFFu) push_one(key[j]);
}

// Sphere tests of the traversals, kept out of line so that their registers do
// not weigh on the triangle loop that surrounds them.
struct SphereTest {
  float t, px, py, pz;  // the hit, when hit != 0
  float xt;             // the extra crossing, when xhit != 0
  int hit, back, xhit, xback;
};
static __device__ __noinline__ SphereTest sphere_instance_test(float radius, vec3 o, vec3 d, float t_max) {
  SphereHit h{0.0f, vec3(0.0f), 0};
  SphereExtra x{false, kTMax, 0};
  SphereTest r;
  r.hit = sphere_intersect(radius, o, d, t_max, &h, &x);
  r.t = h.t;
  r.px = h.p.x;
  r.py = h.p.y;
  r.pz = h.p.z;
  r.back = h.back;
  r.xhit = x.hit;
  r.xt = x.t;
  r.xback = x.back;
  return r;
}
static __device__ __noinline__ bool sphere_occludes(float radius, vec3 o, vec3 d, float t_max) {
  SphereHit h;
  SphereExtra x;
  return sphere_intersect(radius, o, d, t_max, &h, &x);
}

// Results of one step of a resumable walk (ClosestWalk, occluded_step).
constexpr int kWalkGoing = 0, kWalkOccluded = 1, kWalkClear = 2;

struct NearbyHit {
  uint32_t prim;
  float t;
  int back;
};

struct ClosestHit {
  float t;
  float b0, b1, b2;
  uint32_t inst, tri;
  int back;
  int nearby_count;
  NearbyHit nearby[kMaxNearby];
};

// Closest hit of one world-space ray (TraceRay, src/ShadingUtilities.cuh:310-431)
// in the scene of constant-memory slot `scene`, as a resumable walk: one
// step() visits one node or enters one instance, so a persistent kernel can
// advance the lanes of a warp on different rays (k_extend); trace_closest_impl
// runs the steps to the end.
// `volume_only`: traverse only treat_as_boundary instances (TraceVolume, :434-561).
//
// One loop serves both levels: each step pops one entry -- a top-level node,
// an instance to enter, or a bottom-level node of the current instance -- so
// the lanes of a warp run the same node code whatever level they are in.
// Instance leaves are pushed in distance order with the internal nodes,
// bottom-level leaves are tested at once, and entries whose box begins beyond
// the closest hit so far are dropped when popped.
//
// kSpheres: the scene holds sphere geometry. The walk without sphere code is a
// separate instantiation, so scenes of meshes alone keep its register
// allocation (the sphere branch costs the triangle loop about 5%).
template <bool kSpheres>
struct ClosestWalk {
  uint32_t slot;
  vec3 wo, wd;
  BoxRay wray;
  uint32_t last_inst, last_tri;
  bool skip_enabled, volume_only, hit;
  float t_ray, t_upper, t_lower;
  int n_nearby;
  // the instance being traversed (inst_base < 0: none)
  int inst_base;
  uint32_t inst_idx, wtri_offset;
  vec3 od;
  TriRay tr;
  BoxRay br;
  bool skip_here, inst_hit, inst_sphere;
  float inst_t, hb0, hb1, hb2, extra_t;
  // hit_w / extra_w: the wide-BVH slot of the hit / extra triangle, or for a
  // sphere (inst_sphere) the back-face flag of its hit / extra crossing
  uint32_t hit_tri, hit_w, extra_w;

  __device__ __forceinline__ void begin(uint32_t scene, TraversalStack& st, vec3 o, vec3 d, float tmax,
                                        uint32_t li, uint32_t lt, bool vol_only) {
    slot = scene;
    wo = o;
    wd = d;
    wray = make_box_ray(o, d);
    last_inst = li;
    last_tri = lt;
    skip_enabled = li != kEmpty && lt != kEmpty;
    volume_only = vol_only;
    hit = false;
    t_ray = tmax;
    t_upper = t_lower = 0.0f;
    n_nearby = 0;
    inst_base = -1;
    inst_idx = wtri_offset = 0;
    od = vec3(0.0f);
    br = wray;
    skip_here = inst_hit = inst_sphere = false;
    inst_t = hb0 = hb1 = hb2 = 0.0f;
    extra_t = kTMax;
    hit_tri = kEmpty;
    hit_w = 0;
    extra_w = kEmpty;
    st.sp = 0;
    st.push(0, 0.0f);
  }

  // Leaving the instance: its hit (and the nearby-hit list) into `out`.
  __device__ __forceinline__ void leave_instance(const DeviceScene& S, ClosestHit* out) {
    NearbyHit* nb = out->nearby;
    if (inst_hit) {
      int back;
      if (kSpheres && inst_sphere) {
        back = (int)hit_w;
      } else {
        vec3 p0, p1, p2;
        uint32_t tid;
        load_tri(S.wtris, hit_w, &p0, &p1, &p2, &tid);
        const vec3 ng = normalize(cross(p1 - p0, p2 - p0));
        back = dot(ng, od) > 0.0f;
      }
      out->t = inst_t;
      out->b0 = hb0;
      out->b1 = hb1;
      out->b2 = hb2;
      out->inst = inst_idx;
      out->tri = hit_tri;
      out->back = back;
      hit = true;
      t_upper = next_float_up(next_float_up(t_ray));
      t_lower = next_float_down(next_float_down(t_ray));
      int head = 0, tail = n_nearby - 1;
      while (head <= tail) {
        if (nb[head].t > t_lower && nb[head].t < t_upper) ++head;
        else {
          const NearbyHit tmp = nb[head];
          nb[head] = nb[tail];
          nb[tail] = tmp;
          --tail;
        }
      }
      n_nearby = head;
      if (n_nearby < kMaxNearby) nb[n_nearby++] = NearbyHit{inst_idx, inst_t, back};
    } else if (hit && extra_w != kEmpty && extra_t > t_lower && extra_t < t_upper) {
      int back;
      if (kSpheres && inst_sphere) {
        back = (int)extra_w;
      } else {
        vec3 p0, p1, p2;
        uint32_t tid;
        load_tri(S.wtris, extra_w, &p0, &p1, &p2, &tid);
        const vec3 ng = normalize(cross(p1 - p0, p2 - p0));
        back = dot(ng, od) > 0.0f;
      }
      if (n_nearby < kMaxNearby) nb[n_nearby++] = NearbyHit{inst_idx, extra_t, back};
    }
    inst_base = -1;
  }

  // One step; kWalkGoing while entries remain, else kWalkClear (the walk is
  // over: `hit` says whether `out` holds a hit; out->nearby_count is set).
  __device__ __forceinline__ int step(TraversalStack& st, ClosestHit* out, uint32_t* tri_tests,
                                      uint32_t* node_visits) {
    const DeviceScene& S = c_scenes[slot];
    if (inst_base >= 0 && st.sp == inst_base) leave_instance(S, out);
    if (st.sp == 0) {
      out->nearby_count = n_nearby;
      return kWalkClear;
    }
    float etn;
    uint32_t e = st.pop(&etn);
    if (etn > widened_tmax(t_ray)) return kWalkGoing;
    if (e & kInstanceEntry) {
      inst_idx = e & ~kInstanceEntry;
      const Instance inst = S.instances[inst_idx];
      if (volume_only && !inst.treat_as_boundary) return kWalkGoing;
      const mat4& wto = S.i_transforms[inst.transform_idx];
      const vec3 oo = xform_point_glm(wto, wo);
      od = xform_dir_glm(wto, wd);
      const GeometryDesc& g = S.geometries[inst.geometry_idx];
      if (kSpheres && g.kind == kGeoSphere) {
        // a sphere is tested at once and left at the next step; its hit
        // point travels in the barycentric slots and its triangle is EMPTY
        ++*tri_tests;
        const SphereTest q = sphere_instance_test(g.radius, oo, od, t_ray);
        inst_sphere = true;
        inst_hit = q.hit != 0;
        if (inst_hit) {
          t_ray = q.t;
          inst_t = q.t;
          hb0 = q.px;
          hb1 = q.py;
          hb2 = q.pz;
          hit_tri = kEmpty;
          hit_w = (uint32_t)q.back;
        }
        extra_t = q.xhit ? q.xt : kTMax;
        extra_w = q.xhit ? (uint32_t)q.xback : kEmpty;
        inst_base = st.sp;
        return kWalkGoing;
      }
      inst_sphere = false;
      tr = make_tri_ray(oo, od);
      br = make_box_ray(oo, od);
      wtri_offset = g.wtri_offset;
      skip_here = skip_enabled && inst_idx == last_inst;
      inst_hit = false;
      extra_t = kTMax;
      extra_w = kEmpty;
      inst_base = st.sp;
      e = g.node_offset;  // continue with the instance's root in this step
    }
    const bool in_blas = inst_base >= 0;
    ++*node_visits;
    float tn[8];
    uint32_t imask, cbase, pbase, meta[2];
    const uint32_t hits = intersect_children(reinterpret_cast<const uint4*>(in_blas ? S.blas_nodes : S.tlas_nodes), e,
                                             in_blas ? br : wray, t_ray, tn, &imask, &cbase, &pbase, meta);
    uint32_t leaves = hits & ~imask;
    if (in_blas) {
      while (leaves) {
        const int c = __ffs(leaves) - 1;
        leaves &= leaves - 1;
        const uint32_t m = child_meta(meta, c);
        const uint32_t cnt = m >> 5, off = m & 31u;
        for (uint32_t q = 0; q < cnt; ++q) {
          const uint32_t wi = wtri_offset + pbase + off + q;
          vec3 p0, p1, p2;
          uint32_t tid;
          load_tri(S.wtris, wi, &p0, &p1, &p2, &tid);
          if (skip_here && tid == last_tri) continue;
          float t, ev[3], inv;
          ++*tri_tests;
          if (!tri_test(tr, p0, p1, p2, &t, ev, &inv)) continue;
          if (t >= kTMin && t < extra_t) {
            extra_t = t;
            extra_w = wi;
          }
          if (t < kTMin || t > t_ray) continue;
          t_ray = t;
          inst_hit = true;
          inst_t = t;
          hb0 = ev[0] * inv;
          hb1 = ev[1] * inv;
          hb2 = ev[2] * inv;
          hit_tri = tid;
          hit_w = wi;
        }
      }
      push_children(st, hits & imask, 0u, tn, meta, cbase, pbase, S.tlas_prims);
    } else {
      push_children(st, hits & imask, leaves, tn, meta, cbase, pbase, S.tlas_prims);
    }
    return kWalkGoing;
  }
};

// The whole walk of one ray (see ClosestWalk).
template <bool kSpheres>
static __device__ __noinline__ bool trace_closest_impl(uint32_t scene, TraversalStack& st, vec3 wo, vec3 wd,
                                                       float tmax, uint32_t last_inst, uint32_t last_tri,
                                                       bool volume_only, ClosestHit* out, uint32_t* tri_tests,
                                                       uint32_t* node_visits) {
  ClosestWalk<kSpheres> w;
  w.begin(scene, st, wo, wd, tmax, last_inst, last_tri, volume_only);
  while (w.step(st, out, tri_tests, node_visits) == kWalkGoing) {
  }
  return w.hit;
}

// Closest hit of one world-space ray in the scene of constant-memory slot
// `scene` (see trace_closest_impl). Out of line, so that its callers keep one
// call site whichever instantiation runs.
static __device__ __noinline__ bool trace_closest(uint32_t scene, TraversalStack& st, vec3 wo, vec3 wd, float tmax,
                                              uint32_t last_inst, uint32_t last_tri, bool volume_only,
                                              ClosestHit* out, uint32_t* tri_tests, uint32_t* node_visits) {
  if (c_scenes[scene].sphere_count != 0)
    return trace_closest_impl<true>(scene, st, wo, wd, tmax, last_inst, last_tri, volume_only, out, tri_tests,
                                    node_visits);
  return trace_closest_impl<false>(scene, st, wo, wd, tmax, last_inst, last_tri, volume_only, out, tri_tests,
                                   node_visits);
}

// Any hit within (TMIN, tmax] ignoring boundary-only instances
// (BVHTraverseShadow, src/ShadingUtilities.cuh:563-635). Same single loop as
// trace_closest; children are pushed unordered and the first hit ends it.
template <bool kSpheres>
__device__ __noinline__ bool trace_occluded_impl(uint32_t scene, TraversalStack& st, vec3 wo, vec3 wd, float tmax,
                                                 uint32_t* tri_tests, uint32_t* node_visits) {
  const DeviceScene& S = c_scenes[scene];
  const uint4* tlas = reinterpret_cast<const uint4*>(S.tlas_nodes);
  const uint4* blas = reinterpret_cast<const uint4*>(S.blas_nodes);
  const BoxRay wray = make_box_ray(wo, wd);
  int inst_base = -1;
  uint32_t wtri_offset = 0;
  TriRay tr;
  BoxRay br = wray;
  st.sp = 0;
  st.push(0, 0.0f);
  for (;;) {
    if (inst_base >= 0 && st.sp == inst_base) inst_base = -1;
    if (st.sp == 0) break;
    float etn;
    uint32_t e = st.pop(&etn);
    if (e & kInstanceEntry) {
      const Instance inst = S.instances[e & ~kInstanceEntry];
      if (inst.treat_as_boundary) continue;
      const mat4& wto = S.i_transforms[inst.transform_idx];
      const vec3 oo = xform_point_glm(wto, wo);
      const vec3 od = xform_dir_glm(wto, wd);
      const GeometryDesc& g = S.geometries[inst.geometry_idx];
      if (kSpheres && g.kind == kGeoSphere) {
        ++*tri_tests;
        if (sphere_occludes(g.radius, oo, od, tmax)) {
          st.sp = 0;
          return true;
        }
        continue;
      }
      tr = make_tri_ray(oo, od);
      br = make_box_ray(oo, od);
      wtri_offset = g.wtri_offset;
      inst_base = st.sp;
      e = g.node_offset;
    }
    const bool in_blas = inst_base >= 0;
    ++*node_visits;
    float tn[8];
    uint32_t imask, cbase, pbase, meta[2];
    const uint32_t hits =
        intersect_children(in_blas ? blas : tlas, e, in_blas ? br : wray, tmax, tn, &imask, &cbase, &pbase, meta);
    uint32_t leaves = hits & ~imask;
    uint32_t internal = hits & imask;
    while (internal) {
      const int c = __ffs(internal) - 1;
      internal &= internal - 1;
      st.push(cbase + child_meta(meta, c), tn[c]);
    }
    while (leaves) {
      const int c = __ffs(leaves) - 1;
      leaves &= leaves - 1;
      const uint32_t m = child_meta(meta, c);
      const uint32_t cnt = m >> 5, off = m & 31u;
      if (!in_blas) {
        for (uint32_t k = 0; k < cnt; ++k) st.push(kInstanceEntry | __ldg(S.tlas_prims + pbase + off + k), tn[c]);
        continue;
      }
      for (uint32_t q = 0; q < cnt; ++q) {
        vec3 p0, p1, p2;
        uint32_t tid;
        load_tri(S.wtris, wtri_offset + pbase + off + q, &p0, &p1, &p2, &tid);
        float t, ev[3], inv;
        ++*tri_tests;
        if (!tri_test(tr, p0, p1, p2, &t, ev, &inv)) continue;
        if (t < kTMin || t > tmax) continue;
        st.sp = 0;
        return true;
      }
    }
  }
  return false;
}

// ------------------------------------------------ resumable occlusion walk ---
//
// The any-hit query of trace_occluded_impl cut into steps, so that a
// persistent kernel can advance the lanes of a warp on different rays and
// hand a finished lane its next ray at once (k_connect). One step enters an
// instance and visits its root, or visits one node: its child boxes are
// tested, internal children pushed (unordered: any hit ends the query) and
// the triangles of its leaf children tested. Stack entries need no entry
// distance here, so the stack is entries only.
constexpr int kOccStackShared = 32;  // entries per thread in shared memory
constexpr int kConnectBlocksPerSm = 8;  // at kTraceBlock threads (the register budget of the launch bounds)
constexpr size_t occluded_shared_bytes(uint32_t block) { return (size_t)kOccStackShared * block * 4u; }

struct OccStack {
  uint32_t* sh;  // shared-memory column of this thread (stride: the block's threads)
  uint32_t loc[kStackLocal];
  int sp;
  int stride;
  bool overflow;
  __device__ __forceinline__ void bind(uint32_t* shared_entries) {
    sh = shared_entries + threadIdx.x;
    stride = (int)blockDim.x;
    sp = 0;
    overflow = false;
  }
  __device__ __forceinline__ void push(uint32_t v) {
    if (sp < kOccStackShared) sh[sp * stride] = v;
    else if (sp < kOccStackShared + kStackLocal) loc[sp - kOccStackShared] = v;
    else {
      overflow = true;
      return;
    }
    ++sp;
  }
  __device__ __forceinline__ uint32_t pop() {
    --sp;
    return sp < kOccStackShared ? sh[sp * stride] : loc[sp - kOccStackShared];
  }
};

struct OccWalk {
  uint32_t slot;       // scene slot
  vec3 wo, wd;         // world ray
  float tmax;
  BoxRay wray;
  int inst_base;       // stack depth below the current instance's entries (-1: top level)
  uint32_t wtri_offset;
  TriRay tr;           // the current instance's object-space ray
  BoxRay br;
  __device__ __forceinline__ void begin(uint32_t scene, vec3 o, vec3 d, float t_max, OccStack& st) {
    slot = scene;
    wo = o;
    wd = d;
    tmax = t_max;
    wray = make_box_ray(o, d);
    inst_base = -1;
    st.sp = 0;
    st.push(0);
  }
};

template <bool kSpheres>
__device__ __forceinline__ int occluded_step(OccWalk& w, OccStack& st, uint32_t* tri_tests, uint32_t* node_visits) {
  const DeviceScene& S = c_scenes[w.slot];
  if (w.inst_base >= 0 && st.sp == w.inst_base) w.inst_base = -1;
  if (st.sp == 0) return kWalkClear;
  uint32_t e = st.pop();
  if (e & kInstanceEntry) {
    const Instance inst = S.instances[e & ~kInstanceEntry];
    if (inst.treat_as_boundary) return kWalkGoing;
    const mat4& wto = S.i_transforms[inst.transform_idx];
    const vec3 oo = xform_point_glm(wto, w.wo);
    const vec3 od = xform_dir_glm(wto, w.wd);
    const GeometryDesc& g = S.geometries[inst.geometry_idx];
    if (kSpheres && g.kind == kGeoSphere) {
      ++*tri_tests;
      return sphere_occludes(g.radius, oo, od, w.tmax) ? kWalkOccluded : kWalkGoing;
    }
    w.tr = make_tri_ray(oo, od);
    w.br = make_box_ray(oo, od);
    w.wtri_offset = g.wtri_offset;
    w.inst_base = st.sp;
    e = g.node_offset;
  }
  const bool in_blas = w.inst_base >= 0;
  ++*node_visits;
  float tn[8];
  uint32_t imask, cbase, pbase, meta[2];
  const uint32_t hits = intersect_children(reinterpret_cast<const uint4*>(in_blas ? S.blas_nodes : S.tlas_nodes), e,
                                           in_blas ? w.br : w.wray, w.tmax, tn, &imask, &cbase, &pbase, meta);
  uint32_t leaves = hits & ~imask;
  uint32_t internal = hits & imask;
  while (internal) {
    const int c = __ffs(internal) - 1;
    internal &= internal - 1;
    st.push(cbase + child_meta(meta, c));
  }
  while (leaves) {
    const int c = __ffs(leaves) - 1;
    leaves &= leaves - 1;
    const uint32_t m = child_meta(meta, c);
    const uint32_t cnt = m >> 5, off = m & 31u;
    if (!in_blas) {
      for (uint32_t k = 0; k < cnt; ++k) st.push(kInstanceEntry | __ldg(S.tlas_prims + pbase + off + k));
      continue;
    }
    for (uint32_t q = 0; q < cnt; ++q) {
      vec3 p0, p1, p2;
      uint32_t tid;
      load_tri(S.wtris, w.wtri_offset + pbase + off + q, &p0, &p1, &p2, &tid);
      float t, ev[3], inv;
      ++*tri_tests;
      if (!tri_test(w.tr, p0, p1, p2, &t, ev, &inv)) continue;
      if (t < kTMin || t > w.tmax) continue;
      return kWalkOccluded;
    }
  }
  return kWalkGoing;
}

static __device__ __noinline__ bool trace_occluded(uint32_t scene, TraversalStack& st, vec3 wo, vec3 wd, float tmax,
                                               uint32_t* tri_tests, uint32_t* node_visits) {
  if (c_scenes[scene].sphere_count != 0) return trace_occluded_impl<true>(scene, st, wo, wd, tmax, tri_tests, node_visits);
  return trace_occluded_impl<false>(scene, st, wo, wd, tmax, tri_tests, node_visits);
}

}  // namespace ym
