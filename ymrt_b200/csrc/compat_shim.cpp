// libymrt_compat.so: the reference's seventeen launcher symbols
// (src/core/RenderModule.cpp:14-46; defined in src/Shading.cu:1067-1165,
// 1333-1632, 1727, 1903, 2304, 2375, 2467-2515), forwarding to ymrt_compat_*
// in libymrt.so.
//
// The names and argument lists must be the reference's so that its
// RenderModule links against this library unchanged. C++ references are
// passed as pointers by the x86-64 calling convention, so each `T&` argument
// is received here as a pointer; the reference's structs are not needed
// except RayCounterData, whose two pointers this library fills (same member
// order as src/SceneDefines.h:120-124). The queue structs (ShadingRayData,
// HitData, ShadowRayData) are opaque: ymrt_b200 keeps its own queues.
//
// Like the reference's launchers (CUDA_CHECK, src/Helper.h:91-101), these
// report a failure by throwing std::runtime_error.
#include <stdexcept>
#include <string>

#include "../../include/ymrt_compat.h"

namespace {

struct RayCounterData {  // src/SceneDefines.h:120-124
  void* ray_counter_device;
  void* ray_counter_host;
};

void check(int rc, const char* where) {
  if (rc != YMRT_OK) {
    const char* msg = ymrt_last_error(nullptr);
    throw std::runtime_error(std::string(where) + ": " + (msg ? msg : "error") + " (" + std::to_string(rc) + ")");
  }
}

}  // namespace

extern "C" {

void AllocateRayCounter(RayCounterData* data) {
  check(ymrt_compat_alloc_counter(&data->ray_counter_host, &data->ray_counter_device), "AllocateRayCounter");
}

void ReleaseRayCounter(RayCounterData* data) {
  check(ymrt_compat_free_counter(data->ray_counter_host, data->ray_counter_device), "ReleaseRayCounter");
  data->ray_counter_host = nullptr;
  data->ray_counter_device = nullptr;
}

// ymrt_b200 keeps its own path queues: the reference's are not allocated.
void AllocateShadingRayData(void*) {}
void ReleaseShadingRayData(void*) {}
void AllocateHitData(void*) {}
void ReleaseHitData(void*) {}
void AllocateShadowRayData(void*) {}
void ReleaseShadowRayData(void*) {}

void RayGenerationPathTracing(int current_frame_index, const ymrt_render_setting* render_setting, void* scene_device,
                              void* halton_enumerator_device, void* ray_counter_device, uint32_t next_tile_index,
                              uint32_t tile_count_this_batch, uint32_t width, uint32_t height, uint32_t tile_count_x,
                              uint32_t tile_count_y, void* shading_ray_data, void* stream) {
  (void)scene_device;
  (void)halton_enumerator_device;
  (void)shading_ray_data;
  check(ymrt_compat_generate(current_frame_index, render_setting, ray_counter_device, next_tile_index,
                             tile_count_this_batch, width, height, tile_count_x, tile_count_y, stream),
        "RayGenerationPathTracing");
}

void RayTracePathTracing(int current_frame_index, const ymrt_render_setting* render_setting, void* scene_device,
                         void* ray_counter_device, void* ray_counter_host, uint32_t width, uint32_t height,
                         float* noise_image, void* shading_ray_data, void* hit_data, void* stream) {
  (void)scene_device;
  (void)ray_counter_host;
  (void)shading_ray_data;
  (void)hit_data;
  check(ymrt_compat_trace(current_frame_index, render_setting, ray_counter_device, width, height, noise_image, stream),
        "RayTracePathTracing");
}

void RayShadingPathTracing(int current_frame_index, const ymrt_render_setting* render_setting, void* scene_device,
                           void* ray_counter_device, void* ray_counter_host, uint32_t width, uint32_t height,
                           float* noise_image, void* shading_ray_data, void* hit_data, void* shadow_ray_data,
                           void* stream) {
  (void)scene_device;
  (void)ray_counter_host;
  (void)shading_ray_data;
  (void)hit_data;
  (void)shadow_ray_data;
  check(ymrt_compat_shade(current_frame_index, render_setting, ray_counter_device, width, height, noise_image, stream),
        "RayShadingPathTracing");
}

void RayGenerationEditorView(int current_frame_index, const ymrt_render_setting* render_setting, void* scene_device,
                             void* ray_counter_device, uint32_t next_tile_index, uint32_t tile_count_this_batch,
                             uint32_t width, uint32_t height, uint32_t tile_count_x, uint32_t tile_count_y,
                             void* shading_ray_data, void* stream) {
  (void)render_setting;
  (void)scene_device;
  (void)tile_count_this_batch;
  (void)tile_count_x;
  (void)tile_count_y;
  (void)shading_ray_data;
  check(ymrt_compat_editor_generate(current_frame_index, ray_counter_device, next_tile_index, width, height, stream),
        "RayGenerationEditorView");
}

void RayTraceEditorView(int current_frame_index, const ymrt_render_setting* render_setting, void* scene_device,
                        void* ray_counter_device, void* ray_counter_host, uint32_t width, uint32_t height,
                        float* beauty, uint32_t* primitive_index, void* shading_ray_data, void* hit_data,
                        void* stream) {
  (void)scene_device;
  (void)ray_counter_host;
  (void)shading_ray_data;
  (void)hit_data;
  check(ymrt_compat_editor_trace(current_frame_index, render_setting, ray_counter_device, width, height, beauty,
                                 primitive_index, stream),
        "RayTraceEditorView");
}

void RayShadingEditorView(int current_frame_index, const ymrt_render_setting* render_setting, void* scene_device,
                          void* ray_counter_device, void* ray_counter_host, uint32_t width, uint32_t height,
                          float* beauty, uint32_t* primitive_index, void* shading_ray_data, void* hit_data,
                          void* shadow_ray_data, void* stream) {
  (void)current_frame_index;
  (void)render_setting;
  (void)scene_device;
  (void)ray_counter_host;
  (void)width;
  (void)height;
  (void)beauty;
  (void)primitive_index;
  (void)shading_ray_data;
  (void)hit_data;
  (void)shadow_ray_data;
  check(ymrt_compat_editor_shade(ray_counter_device, stream), "RayShadingEditorView");
}

void PostProcessingEditorView(float* image, uint32_t* primitive_index, uint32_t width, uint32_t height,
                              uint32_t clicked_primitive_index, float gamma, float exposure, bool draw_selected_effect,
                              void* stream) {
  check(ymrt_compat_post_process(image, primitive_index, width, height, clicked_primitive_index, gamma, exposure,
                                 draw_selected_effect ? 1 : 0, stream),
        "PostProcessingEditorView");
}

void PostProcessingPathTracing(float* image, uint32_t width, uint32_t height, float gamma, float exposure, void* stream) {
  check(ymrt_compat_post_process(image, nullptr, width, height, 0xFFFFFFFFu, gamma, exposure, 0, stream),
        "PostProcessingPathTracing");
}

void AccumulateImagePathTracing(const float* noise_image, float* accumulated_image, uint32_t width, uint32_t height,
                                int frame_index, const int max_accumulate_frame, void* stream) {
  check(ymrt_compat_accumulate(noise_image, accumulated_image, width, height, frame_index, max_accumulate_frame, stream),
        "AccumulateImagePathTracing");
}

}  // extern "C"
