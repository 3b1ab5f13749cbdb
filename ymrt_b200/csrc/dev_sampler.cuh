// Halton sampling on the device: the reference's pixel-to-index enumerator
// (src/HaltonEnumerator.h:11-115) and its randomly permuted radical inverse
// (src/RandomSampler.cuh:416-508). Integer work is bit-exact; the float steps
// are the reference's, in its order.
#pragma once

#include "ymrt_scene.h"

namespace ym {

// First 1000 primes and their prefix sums (offset of each prime's digit
// permutation in the table), uploaded before each launch sequence.
__constant__ uint32_t c_primes[kHaltonDims];
__constant__ uint32_t c_prime_sums[kHaltonDims];

// Evaluation order of the reference's multi-draw argument lists
// (e.g. SampleLi(..., random(), random(), ...) at src/Shading.cu:325): the
// device front end evaluates call arguments left to right, so the first
// argument receives the first draw.
constexpr bool kDrawLeftToRight = true;

struct HaltonState {
  uint64_t index;
  uint32_t dim;
};

__device__ __forceinline__ uint64_t halton2_inverse(uint64_t index, uint64_t digits) {
  uint64_t r = 0;
  for (uint64_t i = 0; i < digits; ++i) {
    r = r * 2 + (index % 2);
    index /= 2;
  }
  return r;
}
__device__ __forceinline__ uint64_t halton3_inverse(uint64_t index, uint64_t digits) {
  uint64_t r = 0;
  for (uint64_t i = 0; i < digits; ++i) {
    r = r * 3 + (index % 3);
    index /= 3;
  }
  return r;
}

// HaltonEnumerator::GetIndex, src/HaltonEnumerator.h:43-48.
__device__ __forceinline__ uint64_t halton_index(const DeviceScene& S, int px, int py, int ith_sample) {
  const uint64_t ix = halton2_inverse((uint64_t)px, (uint64_t)S.halton_exp2);
  const uint64_t iy = halton3_inverse((uint64_t)py, (uint64_t)S.halton_exp3);
  const uint64_t off = (ix * (uint64_t)S.halton_mx + iy * (uint64_t)S.halton_my) % (uint64_t)S.halton_increment;
  return off + (uint64_t)ith_sample * (uint64_t)S.halton_increment;
}

// RadicalInversion with a digit permutation, src/RandomSampler.cuh:462-480.
// Indices below 2^32 (every sample of a 4K frame at 64 spp) take the 32-bit
// division path; the digits, and therefore the result, are identical.
__device__ __forceinline__ float radical_inverse_perm(uint64_t index, uint32_t base, const uint32_t* __restrict__ perm) {
  const float inv_base = 1.0f / float(base);
  uint64_t radical_sum = 0;
  float base_multiply = 1.0f;
  if (index <= 0xFFFFFFFFull) {
    uint32_t idx = (uint32_t)index;
    while (idx) {
      const uint32_t next = idx / base;
      const uint32_t digit = idx - next * base;
      radical_sum = radical_sum * base + __ldg(perm + digit);
      base_multiply *= inv_base;
      idx = next;
    }
  } else {
    while (index) {
      const uint64_t next = index / base;
      const uint64_t digit = index - next * base;
      radical_sum = radical_sum * base + __ldg(perm + digit);
      base_multiply *= inv_base;
      index = next;
    }
  }
  const float postfix_zero = (float)__ldg(perm) * base_multiply * inv_base / (1.0f - inv_base);
  return gmax(0.000001f, gmin(__ull2float_rn(radical_sum) * base_multiply + postfix_zero, 0.999999f));
}

// HaltonSampler::Random1D, src/RandomSampler.cuh:430-439.
__device__ __forceinline__ float halton_next(HaltonState& s, const uint32_t* __restrict__ table) {
  const uint32_t d = s.dim;
  const float r = radical_inverse_perm(s.index, c_primes[d], table + c_prime_sums[d]);
  ++s.dim;
  if (s.dim >= (uint32_t)kHaltonDims) s.dim = 2;
  return r;
}

// Two / three draws bound to argument positions in the reference's order.
__device__ __forceinline__ void halton_next2(HaltonState& s, const uint32_t* t, float* a0, float* a1) {
  if (kDrawLeftToRight) {
    *a0 = halton_next(s, t);
    *a1 = halton_next(s, t);
  } else {
    *a1 = halton_next(s, t);
    *a0 = halton_next(s, t);
  }
}
__device__ __forceinline__ void halton_next3(HaltonState& s, const uint32_t* t, float* a0, float* a1, float* a2) {
  if (kDrawLeftToRight) {
    *a0 = halton_next(s, t);
    *a1 = halton_next(s, t);
    *a2 = halton_next(s, t);
  } else {
    *a2 = halton_next(s, t);
    *a1 = halton_next(s, t);
    *a0 = halton_next(s, t);
  }
}

// RadicalInversion2 / RadicalInversion3 (un-permuted), src/RandomSampler.cuh:481-507.
__device__ __forceinline__ float radical_inverse_2(uint64_t index) {
  const float inv_base = 1.0f / float(2u);
  uint64_t radical_sum = 0;
  float base_multiply = 1.0f;
  while (index) {
    const uint64_t next = index / 2u;
    const uint64_t digit = index - next * 2u;
    radical_sum = radical_sum * 2u + digit;
    base_multiply *= inv_base;
    index = next;
  }
  return gmax(0.000001f, gmin(__ull2float_rn(radical_sum) * base_multiply, 0.999999f));
}
__device__ __forceinline__ float radical_inverse_3(uint64_t index) {
  const float inv_base = 1.0f / float(3u);
  uint64_t radical_sum = 0;
  float base_multiply = 1.0f;
  while (index) {
    const uint64_t next = index / 3u;
    const uint64_t digit = index - next * 3u;
    radical_sum = radical_sum * 3u + digit;
    base_multiply *= inv_base;
    index = next;
  }
  return gmax(0.000001f, gmin(__ull2float_rn(radical_sum) * base_multiply, 0.999999f));
}

}  // namespace ym
