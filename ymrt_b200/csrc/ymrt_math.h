// Small vector/matrix toolkit for the ymrt_b200 path tracer.
//
// Every operation evaluates in the same order, and at the same precision, as
// the expression the YMRT reference writes with glm 0.9.8 (external/glm in the
// reference tree): e.g. dot(a, b) = (a.x*b.x + a.y*b.y) + a.z*b.z
// (glm/detail/func_geometric.inl:54-61), normalize(v) = v * (1 / sqrt(dot(v, v)))
// (:88-96), mat4 * vec4 = (m0*x + m1*y) + (m2*z + m3*w)
// (glm/detail/type_mat4x4.inl:526-537), min(x, y) = y < x ? y : x
// (glm/detail/func_common.inl:15). The kernels are compiled with
// -fmad=false, so each expression is rounded exactly as written; where speed
// matters more than matching the reference bit for bit (BVH box tests) the
// code calls fmaf explicitly.
#pragma once

#include <cstdint>
#include <cmath>

#if defined(__CUDACC__)
#define YM_HD __host__ __device__ __forceinline__
#else
#define YM_HD inline
using std::isinf;
#endif

namespace ym {

constexpr float kPi = 3.14159265358f;        // ONE_PI, src/MathCommon.h:11
constexpr float kTwoPi = 6.28318530716f;     // TWO_PI
constexpr float kInvPi = 0.318309886183f;    // INV_PI
constexpr float kFloatEps = 1.569209E-07f;   // FLOAT_EPSILON
constexpr float kMinColorEps = 3.7252903E-9f;
constexpr float kMaxColorClamp = 1E16f;
constexpr float kShadowRayClamp = 0.9995f;
constexpr float kTMax = 1E36f;               // TMAX, src/Ray.h:9
constexpr float kTMin = 1E-7f;               // TMIN
constexpr float kFloatMax = 1E36f;           // YMRT_FLOAT_MAX
constexpr float kFloatMin = -1E36f;
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

YM_HD float gmin(float x, float y) { return y < x ? y : x; }
YM_HD float gmax(float x, float y) { return x < y ? y : x; }
YM_HD int gmin(int x, int y) { return y < x ? y : x; }
YM_HD int gmax(int x, int y) { return x < y ? y : x; }
YM_HD float gclamp(float x, float lo, float hi) { return gmin(gmax(x, lo), hi); }

YM_HD float error_gamma(int n) { return (n * kFloatEps) / (1.0f - n * kFloatEps); }

YM_HD float sqr(float x) { return x * x; }

YM_HD float safe_rcp(float f) { return fabsf(f) < 1E-30f ? (f > 0.0f ? 1E30f : -1E30f) : (1.0f / f); }

YM_HD uint32_t f2u(float f) {
  union { float f; uint32_t u; } c;
  c.f = f;
  return c.u;
}
YM_HD float u2f(uint32_t u) {
  union { float f; uint32_t u; } c;
  c.u = u;
  return c.f;
}

// NextFloatUp / NextFloatDown, src/MathCommon.h:263-297.
YM_HD float next_float_up(float f) {
  if (isinf(f) && f > 0.0f) return f;
  if (f == -0.0f) f = 0.0f;
  uint32_t ui = f2u(f);
  if (f >= 0.0f) ++ui; else --ui;
  return u2f(ui);
}
YM_HD float next_float_down(float f) {
  if (isinf(f) && f < 0.0f) return f;
  if (f == 0.0f) f = -0.0f;
  uint32_t ui = f2u(f);
  if (f <= 0.0f) ++ui; else --ui;
  return u2f(ui);
}

struct vec3 {
  float x, y, z;
  vec3() = default;
  YM_HD explicit vec3(float s) : x(s), y(s), z(s) {}
  YM_HD vec3(float a, float b, float c) : x(a), y(b), z(c) {}
  YM_HD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
  YM_HD float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

YM_HD vec3 operator+(vec3 a, vec3 b) { return vec3(a.x + b.x, a.y + b.y, a.z + b.z); }
YM_HD vec3 operator-(vec3 a, vec3 b) { return vec3(a.x - b.x, a.y - b.y, a.z - b.z); }
YM_HD vec3 operator*(vec3 a, vec3 b) { return vec3(a.x * b.x, a.y * b.y, a.z * b.z); }
YM_HD vec3 operator/(vec3 a, vec3 b) { return vec3(a.x / b.x, a.y / b.y, a.z / b.z); }
YM_HD vec3 operator*(vec3 a, float s) { return vec3(a.x * s, a.y * s, a.z * s); }
YM_HD vec3 operator*(float s, vec3 a) { return vec3(s * a.x, s * a.y, s * a.z); }
YM_HD vec3 operator/(vec3 a, float s) { return vec3(a.x / s, a.y / s, a.z / s); }
YM_HD vec3 operator+(vec3 a, float s) { return vec3(a.x + s, a.y + s, a.z + s); }
YM_HD vec3 operator-(vec3 a, float s) { return vec3(a.x - s, a.y - s, a.z - s); }
YM_HD vec3 operator-(float s, vec3 a) { return vec3(s - a.x, s - a.y, s - a.z); }
YM_HD vec3 operator-(vec3 a) { return vec3(-a.x, -a.y, -a.z); }
YM_HD vec3& operator+=(vec3& a, vec3 b) { a = a + b; return a; }
YM_HD vec3& operator-=(vec3& a, vec3 b) { a = a - b; return a; }
YM_HD vec3& operator*=(vec3& a, vec3 b) { a = a * b; return a; }
YM_HD vec3& operator*=(vec3& a, float s) { a = a * s; return a; }
YM_HD vec3& operator/=(vec3& a, float s) { a = a / s; return a; }

YM_HD float dot(vec3 a, vec3 b) {
  const vec3 t = a * b;
  return t.x + t.y + t.z;
}
YM_HD vec3 cross(vec3 a, vec3 b) {
  return vec3(a.y * b.z - b.y * a.z, a.z * b.x - b.z * a.x, a.x * b.y - b.x * a.y);
}
YM_HD float length(vec3 v) { return sqrtf(dot(v, v)); }
YM_HD vec3 normalize(vec3 v) { return v * (1.0f / sqrtf(dot(v, v))); }
YM_HD vec3 vabs(vec3 v) { return vec3(fabsf(v.x), fabsf(v.y), fabsf(v.z)); }
YM_HD vec3 vmin(vec3 a, vec3 b) { return vec3(gmin(a.x, b.x), gmin(a.y, b.y), gmin(a.z, b.z)); }
YM_HD vec3 vmax(vec3 a, vec3 b) { return vec3(gmax(a.x, b.x), gmax(a.y, b.y), gmax(a.z, b.z)); }
YM_HD vec3 vclamp(vec3 v, vec3 lo, vec3 hi) { return vmin(vmax(v, lo), hi); }
YM_HD vec3 vsqrt(vec3 v) { return vec3(sqrtf(v.x), sqrtf(v.y), sqrtf(v.z)); }
YM_HD vec3 vexp(vec3 v) { return vec3(expf(v.x), expf(v.y), expf(v.z)); }
YM_HD vec3 vlog(vec3 v) { return vec3(logf(v.x), logf(v.y), logf(v.z)); }
YM_HD float max_component(vec3 v) { return gmax(v.x, gmax(v.y, v.z)); }
YM_HD int max_dimension(vec3 v) {
  int d = 0;
  if (v[1] > v[d]) d = 1;
  if (v[2] > v[d]) d = 2;
  return d;
}
// glm::mix(x, y, a) with scalar a: x + a * (y - x).
YM_HD vec3 mix(vec3 x, vec3 y, float a) { return x + a * (y - x); }
// glm::mix with per-channel weights.
YM_HD vec3 mix(vec3 x, vec3 y, vec3 a) { return x + a * (y - x); }
// The reference's own LinearLerp (src/MathCommon.h:56): (1 - w) * x + y * w.
YM_HD vec3 linear_lerp(vec3 x, vec3 y, float w) { return (1.0f - w) * x + y * w; }
// RGBToLuminance (src/MathCommon.h:146): the middle weight is a double literal,
// so the sum is formed in double and rounded back to float.
YM_HD float luminance(vec3 c) {
  return (float)((double)(0.2126f * c.x) + 0.7152 * (double)c.y + (double)(0.0722f * c.z));
}
YM_HD bool same_hemisphere(vec3 a, vec3 b) { return a.z * b.z > 0.0f; }

// Column-major 4x4 matrix, m[c] is column c (glm layout).
struct mat4 {
  float m[4][4];
};

// glm mat4 * vec4, w = 1 (points): ((c0*x + c1*y) + (c2*z + c3*1)).
YM_HD vec3 xform_point_glm(const mat4& M, vec3 p) {
  vec3 r;
  for (int i = 0; i < 3; ++i) {
    const float a0 = M.m[0][i] * p.x + M.m[1][i] * p.y;
    const float a1 = M.m[2][i] * p.z + M.m[3][i] * 1.0f;
    r[i] = a0 + a1;
  }
  return r;
}
// glm mat4 * vec4, w = 0 (directions): ((c0*x + c1*y) + (c2*z + c3*0)).
YM_HD vec3 xform_dir_glm(const mat4& M, vec3 v) {
  vec3 r;
  for (int i = 0; i < 3; ++i) {
    const float a0 = M.m[0][i] * v.x + M.m[1][i] * v.y;
    const float a1 = M.m[2][i] * v.z + M.m[3][i] * 0.0f;
    r[i] = a0 + a1;
  }
  return r;
}
// glm::transpose(M) * vec4(v, 0): row i of M dotted with v, summed as
// ((r0 + r1) + (r2 + r3*0)) in glm's column-product order.
YM_HD vec3 xform_transpose_dir_glm(const mat4& M, vec3 v) {
  vec3 r;
  for (int i = 0; i < 3; ++i) {
    const float a0 = M.m[i][0] * v.x + M.m[i][1] * v.y;
    const float a1 = M.m[i][2] * v.z + M.m[i][3] * 0.0f;
    r[i] = a0 + a1;
  }
  return r;
}
// TransformVector, src/MathCommon.h:181 (left-to-right sums).
YM_HD vec3 transform_vector(const mat4& M, vec3 v) {
  return vec3(M.m[0][0] * v.x + M.m[1][0] * v.y + M.m[2][0] * v.z,
              M.m[0][1] * v.x + M.m[1][1] * v.y + M.m[2][1] * v.z,
              M.m[0][2] * v.x + M.m[1][2] * v.y + M.m[2][2] * v.z);
}
// TransposeTransformVector, src/MathCommon.h:190.
YM_HD vec3 transpose_transform_vector(const mat4& M, vec3 v) {
  return vec3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z,
              M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z,
              M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z);
}
// TransformPosition with optional error bound, src/MathCommon.h:199-217.
YM_HD vec3 transform_position(const mat4& M, vec3 p, vec3* err = nullptr) {
  vec3 r(M.m[0][0] * p.x + M.m[1][0] * p.y + M.m[2][0] * p.z + M.m[3][0],
         M.m[0][1] * p.x + M.m[1][1] * p.y + M.m[2][1] * p.z + M.m[3][1],
         M.m[0][2] * p.x + M.m[1][2] * p.y + M.m[2][2] * p.z + M.m[3][2]);
  if (err) {
    const float xs = fabsf(M.m[0][0] * p.x) + fabsf(M.m[1][0] * p.y) + fabsf(M.m[2][0] * p.z) + fabsf(M.m[3][0]);
    const float ys = fabsf(M.m[0][1] * p.x) + fabsf(M.m[1][1] * p.y) + fabsf(M.m[2][1] * p.z) + fabsf(M.m[3][1]);
    const float zs = fabsf(M.m[0][2] * p.x) + fabsf(M.m[1][2] * p.y) + fabsf(M.m[2][2] * p.z) + fabsf(M.m[3][2]);
    const vec3 e = *err;
    const float xe = fabsf(M.m[0][0]) * e.x + fabsf(M.m[1][0]) * e.y + fabsf(M.m[2][0]) * e.z;
    const float ye = fabsf(M.m[0][1]) * e.x + fabsf(M.m[1][1]) * e.y + fabsf(M.m[2][1]) * e.z;
    const float ze = fabsf(M.m[0][2]) * e.x + fabsf(M.m[1][2]) * e.y + fabsf(M.m[2][2]) * e.z;
    *err = (error_gamma(3) + 1.0f) * vec3(xe, ye, ze) + error_gamma(3) * vec3(xs, ys, zs);
  }
  return r;
}

// glm::inverse of a 3x3 (glm/detail/func_matrix.inl:272-294), columns c0,c1,c2.
struct mat3 {
  float m[3][3];
};
YM_HD mat3 inverse3(const mat3& a) {
  const float (*m)[3] = a.m;
  const float det = +m[0][0] * (m[1][1] * m[2][2] - m[2][1] * m[1][2])
                    - m[1][0] * (m[0][1] * m[2][2] - m[2][1] * m[0][2])
                    + m[2][0] * (m[0][1] * m[1][2] - m[1][1] * m[0][2]);
  const float inv_det = 1.0f / det;
  mat3 r;
  r.m[0][0] = +(m[1][1] * m[2][2] - m[2][1] * m[1][2]) * inv_det;
  r.m[1][0] = -(m[1][0] * m[2][2] - m[2][0] * m[1][2]) * inv_det;
  r.m[2][0] = +(m[1][0] * m[2][1] - m[2][0] * m[1][1]) * inv_det;
  r.m[0][1] = -(m[0][1] * m[2][2] - m[2][1] * m[0][2]) * inv_det;
  r.m[1][1] = +(m[0][0] * m[2][2] - m[2][0] * m[0][2]) * inv_det;
  r.m[2][1] = -(m[0][0] * m[2][1] - m[2][0] * m[0][1]) * inv_det;
  r.m[0][2] = +(m[0][1] * m[1][2] - m[1][1] * m[0][2]) * inv_det;
  r.m[1][2] = -(m[0][0] * m[1][2] - m[1][0] * m[0][2]) * inv_det;
  r.m[2][2] = +(m[0][0] * m[1][1] - m[1][0] * m[0][1]) * inv_det;
  return r;
}
// glm mat3 * vec3 (glm/detail/type_mat3x3.inl:428-434).
YM_HD vec3 mul3(const mat3& m, vec3 v) {
  return vec3(m.m[0][0] * v.x + m.m[1][0] * v.y + m.m[2][0] * v.z,
              m.m[0][1] * v.x + m.m[1][1] * v.y + m.m[2][1] * v.z,
              m.m[0][2] * v.x + m.m[1][2] * v.y + m.m[2][2] * v.z);
}

// OffsetRayOrigin, src/ShadingUtilities.cuh:993-1011.
YM_HD vec3 offset_ray_origin(vec3 p, vec3 p_err, vec3 dir, vec3 ng) {
  const float d = dot(vabs(ng), p_err);
  vec3 off = d * ng;
  if (dot(dir, ng) < 0.0f) off = -off;
  vec3 po = p + off;
  for (int a = 0; a <= 2; ++a) {
    if (off[a] > 0.0f) po[a] = next_float_up(po[a]);
    else if (off[a] < 0.0f) po[a] = next_float_down(po[a]);
  }
  return po;
}

// OrthogonalBasis, src/MathCommon.h:86-101 (N is normalised in place).
YM_HD void orthogonal_basis(vec3& N, vec3& T, vec3& B) {
  N = normalize(N);
  if (fabsf(N.z) > fabsf(N.x)) {
    const float l = sqrtf(gmax(1.f - N.x * N.x, 0.0f));
    const float r = 1.f / l;
    B = vec3(0.f, N.z * r, -N.y * r);
  } else {
    const float l = sqrtf(gmax(1.f - N.z * N.z, 0.0f));
    const float r = 1.f / l;
    B = vec3(N.y * r, -N.x * r, 0.f);
  }
  T = cross(B, N);
}

}  // namespace ym
