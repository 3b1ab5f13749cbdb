// Force-included prelude for building the YMRT reference sources as host C++
// (g++), so that the oracle can run the reference's own stage kernels on the
// CPU. Test infrastructure only: nothing in the ymrt_b200 product includes it.
//
// What it supplies, and why:
//  * MSVC-only helpers the reference calls (_aligned_malloc/_aligned_free).
//  * Standard headers the reference gets transitively under MSVC.
//  * Host definitions of the CUDA built-in variables (threadIdx, blockIdx,
//    blockDim, gridDim): the oracle harness sets them per emulated thread.
//  * Host atomics with the signatures of CUDA's atomicAdd/atomicExch, so the
//    stage kernels' queue counters and per-pixel float accumulation are
//    thread-safe when the harness runs blocks on several host threads.
#pragma once
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <cstdint>
#include <cmath>
#include <math.h>  // global float overloads (::pow(float, float)), as CUDA provides
#include <cassert>
#include <algorithm>
#include <functional>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <unordered_map>
#include <unordered_set>
#include <vector>
#include <string>

#include <vector_types.h>

using std::isinf;
using std::isnan;

inline void* _aligned_malloc(size_t size, size_t alignment) {
  if (alignment < sizeof(void*)) alignment = sizeof(void*);
  size_t rounded = (size + alignment - 1) / alignment * alignment;
  return std::aligned_alloc(alignment, rounded ? rounded : alignment);
}
inline void _aligned_free(void* p) { std::free(p); }

// CUDA built-in index variables, one copy per host thread.
#define __DEVICE_LAUNCH_PARAMETERS_H__ 1
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

inline int atomicAdd(int* address, int val) {
  return __atomic_fetch_add(address, val, __ATOMIC_RELAXED);
}
inline unsigned int atomicAdd(unsigned int* address, unsigned int val) {
  return __atomic_fetch_add(address, val, __ATOMIC_RELAXED);
}
inline float atomicAdd(float* address, float val) {
  float expected;
  __atomic_load(address, &expected, __ATOMIC_RELAXED);
  float desired;
  do {
    desired = expected + val;
  } while (!__atomic_compare_exchange(address, &expected, &desired, false,
                                      __ATOMIC_RELAXED, __ATOMIC_RELAXED));
  return expected;
}
inline int atomicExch(int* address, int val) {
  return __atomic_exchange_n(address, val, __ATOMIC_RELAXED);
}
inline float atomicExch(float* address, float val) {
  float old;
  __atomic_exchange(address, &val, &old, __ATOMIC_RELAXED);
  return old;
}
