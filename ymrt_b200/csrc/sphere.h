// Analytic spheres: the reference's Sphere geometry (a radius, centred on the
// object-space origin; src/GeometryDefines.h:521-526) as the traversal, the
// hit reconstruction, the sphere shape lights and the camera set-up test it.
//
// Both solves reproduce the reference's arithmetic bit for bit, including its
// mixed precision (a double division in the object test, a double
// discriminant in the light solve), so t, the hit point and the back-face flag
// are the reference's bits. Host and device code share these functions.
#pragma once

#include "ymrt_math.h"

namespace ym {

struct SphereHit {
  float t;  // accepted distance (TMIN <= t <= t_max)
  vec3 p;   // object-space hit point, projected onto the sphere
  int back; // the ray leaves the sphere at p
};

// ExtraHitInfo of a sphere test: the first crossing at or beyond TMIN (or the
// far one), whether or not it lies within t_max; feeds the nearby-hit list.
struct SphereExtra {
  bool hit;
  float t;
  int back;
};

// IntersectSphereObject (src/ShadingUtilities.cuh:219-276) for an object-space
// ray o + t d (d not normalised) and a sphere of `radius` at the origin.
YM_HD bool sphere_intersect(float radius, vec3 o, vec3 d, float t_max, SphereHit* h, SphereExtra* x) {
  const float a = d.x * d.x + d.y * d.y + d.z * d.z;
  const float b = 2.0f * (d.x * o.x + d.y * o.y + d.z * o.z);
  const float c = o.x * o.x + o.y * o.y + o.z * o.z - radius * radius;
  const float disc = b * b - 4.0f * a * c;
  x->hit = false;
  if (disc < 0) return false;
  const float sq = sqrtf(disc);
  // The reference divides in double, (-b - sq) / (2.0 * a), and rounds the
  // quotient to float. Both operands are floats (2a is exact in either
  // precision), and double carries more than 2 * 24 + 2 significand bits, so
  // that double rounding equals one correctly rounded float division
  // (Figueroa, "When is double rounding innocuous?", 1995): the float
  // division below yields the same bits without double-precision code in the
  // traversal loop.
  const float two_a = 2.0f * a;
  const float t1 = (-b - sq) / two_a;
  const float t2 = (-b + sq) / two_a;
  x->hit = true;
  x->t = t1 >= kTMin ? t1 : t2;
  x->back = dot(d, normalize(o + d * x->t)) > 0.0f;
  if (t1 > t_max || t2 < kTMin) return false;
  float t = t1;
  if (t < kTMin) {
    t = t2;
    if (t > t_max) return false;
  }
  vec3 p = o + d * t;
  const float dist = length(p);
  p = dist > kFloatEps ? p * radius / dist : vec3(0.0f);
  h->t = t;
  h->p = p;
  h->back = dot(d, p / radius) > 0.0f;
  return true;
}

// RayIntersectSphere (src/Light.h:42-62): both roots of |o + t d| = radius.
// Returns false when the ray misses or both roots lie behind the origin.
// Unlike the reference, a negative discriminant still yields the roots of
// the clamped (zero) discriminant, so callers that use t0 after a miss (the
// sphere light sampler on a grazing cone direction) read a defined value.
YM_HD bool sphere_solve(vec3 o, vec3 d, float radius, float* t0, float* t1) {
  const float a = d.x * d.x + d.y * d.y + d.z * d.z;
  const float b = 2.0f * (d.x * o.x + d.y * o.y + d.z * o.z);
  const float c = o.x * o.x + o.y * o.y + o.z * o.z - radius * radius;
  const float disc = (float)((double)(b * b) - 4.0 * (double)a * (double)c);
  const float sq = disc < 0.0f ? 0.0f : sqrtf(disc);
  const float ia = 1.0f / a;
  *t0 = (-b - sq) * 0.5f * ia;
  *t1 = (-b + sq) * 0.5f * ia;
  if (disc < 0.0f) return false;
  return !(*t1 < 1E-10f);
}

// GetTranslate (src/MathCommon.h:193-196): the transform's fourth column.
YM_HD vec3 get_translate(const mat4& M) { return vec3(M.m[3][0], M.m[3][1], M.m[3][2]); }

}  // namespace ym
