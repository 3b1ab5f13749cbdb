// Sampling on the device: the reference's Halton pixel-to-index enumerator
// (src/HaltonEnumerator.h:11-115) and randomly permuted radical inverse
// (src/RandomSampler.cuh:416-508), its PCG hash sampler (:380-413) and its
// Owen-scrambled Sobol sampler (:510-615). Integer work is bit-exact; the
// float steps are the reference's, in its order.
#pragma once

#include "ymrt_scene.h"

namespace ym {

// First 1000 primes and their prefix sums (offset of each prime's digit
// permutation in the table), uploaded before each launch sequence.
static __constant__ uint32_t c_primes[kHaltonDims];
static __constant__ uint32_t c_prime_sums[kHaltonDims];

// Evaluation order of the reference's multi-draw argument lists
// (e.g. SampleLi(..., random(), random(), ...) at src/Shading.cu:325): the
// device front end evaluates call arguments left to right, so the first
// argument receives the first draw.
constexpr bool kDrawLeftToRight = true;

// Per-path sampler state (the reference's 32-byte RandomSampler union, kept
// in 16 bytes), by DeviceScene::sampler_type:
//   Halton (1): index = global Halton sample index, dim = next dimension
//   PCG (0):    index = pixel | sample-in-pixel << 32, dim, aux = frame - 1
//   Sobol (2):  index = sample (frame - 1) * spp + sample-in-pixel | pixel << 32, dim
struct PathSampler {
  uint64_t index;
  uint32_t dim;
  uint32_t aux;
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
__device__ __forceinline__ float halton_draw(PathSampler& s, const uint32_t* __restrict__ table) {
  const uint32_t d = s.dim;
  const float r = radical_inverse_perm(s.index, c_primes[d], table + c_prime_sums[d]);
  ++s.dim;
  if (s.dim >= (uint32_t)kHaltonDims) s.dim = 2;
  return r;
}

// The 4-D PCG hash of Jarzynski and Olano, "Hash Functions for GPU
// Rendering" (JCGT 9(3), 2020), as the reference's pcg4d uses it
// (src/RandomSampler.cuh:354-378): an LCG step on each lane, two rounds of
// lane mixing around a xorshift.
__device__ __forceinline__ uint4 pcg4d(uint4 v) {
  v.x = v.x * 1664525u + 1013904223u;
  v.y = v.y * 1664525u + 1013904223u;
  v.z = v.z * 1664525u + 1013904223u;
  v.w = v.w * 1664525u + 1013904223u;
  v.x += v.y * v.w;
  v.y += v.z * v.x;
  v.z += v.x * v.y;
  v.w += v.y * v.z;
  v.x ^= v.x >> 16u;
  v.y ^= v.y >> 16u;
  v.z ^= v.z >> 16u;
  v.w ^= v.w >> 16u;
  v.x += v.y * v.w;
  v.y += v.z * v.x;
  v.z += v.x * v.y;
  v.w += v.y * v.z;
  return v;
}

// PCGSampler::Random1D (src/RandomSampler.cuh:400-405): hash of (pixel,
// dimension, sample in pixel, frame), first lane over 2^32.
__device__ __forceinline__ float pcg_draw(PathSampler& s) {
  const uint4 h = pcg4d(make_uint4((uint32_t)s.index, s.dim, (uint32_t)(s.index >> 32), s.aux));
  ++s.dim;
  return (float)h.x / 4294967296.0f;
}

// Two-word xxHash32 mix (Collet's xxHash primes), the form of the reference's
// XxHash32(uvec2) (src/RandomSampler.cuh:277-286).
__device__ __forceinline__ uint32_t xxhash32_2(uint32_t x, uint32_t y) {
  const uint32_t P2 = 2246822519u, P3 = 3266489917u, P4 = 668265263u, P5 = 374761393u;
  uint32_t h = y + P5 + x * P3;
  h = P4 * ((h << 17) | (h >> 15));
  h = P2 * (h ^ (h >> 15));
  h = P3 * (h ^ (h >> 13));
  return h ^ (h >> 16);
}

// Hash-based Owen scrambling of a 32-bit Sobol sample (the Laine-Karras-style
// nested permutation with the multipliers pbrt-v4 uses), seeded per
// (dimension, pixel) as the reference does (src/RandomSampler.cuh:584-596).
__device__ __forceinline__ uint32_t owen_scramble(uint32_t v, uint32_t dim, uint32_t pixel) {
  const uint32_t seed = xxhash32_2(dim, pixel);
  v = __brev(v);
  v ^= v * 0x3d20adeau;
  v += seed;
  v *= (seed >> 16) | 1u;
  v ^= v * 0x05526c56u;
  v ^= v * 0x53a22864u;
  return __brev(v);
}

// SobolSampler::Random1D / SobolSample (src/RandomSampler.cuh:533-612): the
// Gray-code-ordered Sobol point of the sample in this dimension (generator
// matrices are an input: 32 columns per dimension), Owen-scrambled, clamped.
__device__ __forceinline__ float sobol_draw(PathSampler& s, const uint32_t* __restrict__ matrices) {
  const uint32_t dim = s.dim;
  const uint32_t* m = matrices + (size_t)dim * 32u;
  const uint32_t index = (uint32_t)s.index;
  uint32_t v = 0;
  for (uint32_t i = index ^ (index >> 1), j = 0; i; i >>= 1, ++j)
    if (i & 1u) v ^= __ldg(m + j);
  v = owen_scramble(v, dim, (uint32_t)(s.index >> 32));
  const float r = gmax(0.000001f, gmin(float(v) / float(0xFFFFFFFFu), 0.999999f));
  ++s.dim;
  if (s.dim >= 4096u) s.dim = 1;  // the reference wraps here (and prints a warning)
  return r;
}

// RandomSampler::Random1D (src/RandomSampler.cuh:681-697).
__device__ __forceinline__ float sample1d(PathSampler& s, const DeviceScene& S) {
  if (S.sampler_type == kSamplerHalton) return halton_draw(s, S.halton_perm);
  if (S.sampler_type == kSamplerPcg) return pcg_draw(s);
  return sobol_draw(s, S.sobol_matrices);
}

// Two / three draws bound to argument positions in the reference's order.
__device__ __forceinline__ void sample2d(PathSampler& s, const DeviceScene& S, float* a0, float* a1) {
  if (kDrawLeftToRight) {
    *a0 = sample1d(s, S);
    *a1 = sample1d(s, S);
  } else {
    *a1 = sample1d(s, S);
    *a0 = sample1d(s, S);
  }
}
__device__ __forceinline__ void sample3d(PathSampler& s, const DeviceScene& S, float* a0, float* a1, float* a2) {
  if (kDrawLeftToRight) {
    *a0 = sample1d(s, S);
    *a1 = sample1d(s, S);
    *a2 = sample1d(s, S);
  } else {
    *a2 = sample1d(s, S);
    *a1 = sample1d(s, S);
    *a0 = sample1d(s, S);
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
