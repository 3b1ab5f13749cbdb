// Scenes of the current batch in constant memory. Each job names a slot;
// kernels bind `const DeviceScene& S = c_scenes[slot]`, so scene fields are
// read through the constant cache (uniform across a warp when its lanes
// render the same scene, which wave generation makes the common case).
#pragma once

#include "ymrt_scene.h"

namespace ym {

constexpr int kMaxBatchScenes = 64;  // distinct (scene, sampler) pairs per batch launch
static __constant__ DeviceScene c_scenes[kMaxBatchScenes];

}  // namespace ym
