// Force-included prelude for building the YMRT reference sources for the
// device (nvcc for src/Shading.cu, g++ for the host-side scene module), so
// that the reference's own wavefront kernels run on the GPU as a baseline.
// Test and baseline infrastructure only: nothing in the ymrt_b200 product
// includes it.
//
// It supplies the MSVC-only helpers the reference calls
// (_aligned_malloc/_aligned_free) and the standard headers the reference gets
// transitively under MSVC.
#pragma once
#include <cstdlib>
#include <cstring>
#include <cstdio>
#include <cstdint>
#include <cmath>
#include <math.h>
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
#include <stdexcept>
#include <sstream>
#include <iostream>

inline void* _aligned_malloc(size_t size, size_t alignment) {
  if (alignment < sizeof(void*)) alignment = sizeof(void*);
  size_t rounded = (size + alignment - 1) / alignment * alignment;
  return std::aligned_alloc(alignment, rounded ? rounded : alignment);
}
inline void _aligned_free(void* p) { std::free(p); }
