// Where a bounded device loop gave up (YMRT_DEVERR_ITER), with the state of
// the ray it was following: the first such event since the record was last
// cleared is kept, later ones only set the error bit. Read and cleared by
// ymrt_debug_bound_record; every kernel of this library that has a bounded
// loop writes here.
#pragma once

#include "ymrt_scene.h"

namespace ym {

constexpr uint32_t kBoundShadowCrossings = 1;  // trace_tr: boundary crossings of one shadow ray
constexpr uint32_t kBoundDeltaTracking = 2;    // free-flight sampling steps in a heterogeneous medium
constexpr uint32_t kBoundRatioTracking = 3;    // transmittance steps in a heterogeneous medium
constexpr uint32_t kBoundWaves = 4;            // waves of one frame
constexpr uint32_t kBoundEditorBoundaries = 5; // editor-view pass-through boundaries of one camera ray
constexpr uint32_t kBoundTextureWalk = 6;      // steps of one texture-graph walk

struct BoundRecord {
  uint32_t taken;      // nonzero once written
  uint32_t site;       // kBound*
  uint32_t count;      // iterations made when the bound was reached
  uint32_t last_inst, last_tri;  // surface the ray leaves (trace_tr)
  float o[3], d[3];    // the ray at that moment (world space)
  float tmax;          // its remaining length
  float extra[4];      // tracking: majorant rgb and the sampled channel
  RayTransfer transfer;  // the ray's nested-media stack
};
static_assert(sizeof(BoundRecord) % 4 == 0, "BoundRecord is read as 32-bit words");
constexpr int kBoundRecordWords = (int)(sizeof(BoundRecord) / 4);

static __device__ BoundRecord g_bound;

static __device__ __noinline__ void note_bound(uint32_t site, uint32_t count, vec3 o, vec3 d, float tmax, uint32_t last_inst,
                                        uint32_t last_tri, const RayTransfer* rt, vec3 majorant = vec3(0.0f),
                                        int channel = -1) {
  if (atomicCAS(&g_bound.taken, 0u, 2u) != 0u) return;
  g_bound.site = site;
  g_bound.count = count;
  g_bound.last_inst = last_inst;
  g_bound.last_tri = last_tri;
  g_bound.o[0] = o.x; g_bound.o[1] = o.y; g_bound.o[2] = o.z;
  g_bound.d[0] = d.x; g_bound.d[1] = d.y; g_bound.d[2] = d.z;
  g_bound.tmax = tmax;
  g_bound.extra[0] = majorant.x;
  g_bound.extra[1] = majorant.y;
  g_bound.extra[2] = majorant.z;
  g_bound.extra[3] = (float)channel;
  if (rt) {
    g_bound.transfer = *rt;
  } else {
    g_bound.transfer.record_count = 0;
    g_bound.transfer.max_priority_record_index = -1;
  }
  __threadfence();
  atomicExch(&g_bound.taken, 1u);
}

}  // namespace ym
