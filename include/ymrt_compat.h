/* ymrt_compat.h -- the reference's stage interface on top of ymrt_b200.
 *
 * The YMRT editor drives rendering through seventeen functions (four
 * Allocate / Release pairs, four path-tracing stage launchers, three
 * editor-view stage launchers and two post-processing calls)
 * declared in src/core/RenderModule.cpp:14-28, 36-42 and defined in src/Shading.cu
 * (AllocateRayCounter ... AccumulateImagePathTracing), called by the wave
 * loop of RenderModule::PathTracingExecuteTask
 * (src/core/RenderModule.cpp:494-653). libymrt_compat.so exports those seventeen
 * symbols with the same names and argument lists, so that RenderModule links
 * against it unchanged; each forwards to the entry points below (in
 * libymrt.so), which render with ymrt_b200's kernels.
 *
 * Protocol. The editor binds its ymrt context and scene once per scene
 * change (ymrt_compat_bind; a scene built from the same .ymtmp, or with
 * ymrt_scene_from_arrays from its SceneModule). Then, per frame, its loop
 * calls generation / trace / shading batch after batch: the first
 * generation call of a frame (tile 0) marks the frame; the trace call that
 * follows renders all of the frame's tiles into the noise image the loop
 * passes (ymrt_b200 plans its own waves) and clears the loop's device ray
 * counter, so the loop's remaining batches find no rays in flight and only
 * step through the tile indices. The queue arguments (ShadingRayData,
 * HitData, ShadowRayData) are not used and their Allocate / Release calls
 * allocate nothing; the ray counter is allocated as the reference does
 * (host copy and device copy).
 *
 * All calls are synchronous with respect to the caller's stream (they
 * synchronize it first) and return 0 or a negative YMRT_ERR_* code; the
 * reference-named wrappers throw std::runtime_error on an error, as the
 * reference's launchers do through CUDA_CHECK.
 */
#ifndef YMRT_COMPAT_H_
#define YMRT_COMPAT_H_

#include "ymrt.h"

#ifdef __cplusplus
extern "C" {
#endif

/* The context and scene the stage calls render with (replaces any earlier
 * binding; NULL scene unbinds). Call it after every scene change. */
int ymrt_compat_bind(ymrt_context* ctx, ymrt_scene* scene);

/* AllocateRayCounter / ReleaseRayCounter (src/Shading.cu:1067-1080): a
 * zeroed 12-byte RayCounter in host memory and a copy on the device. */
int ymrt_compat_alloc_counter(void** host_counter, void** device_counter);
int ymrt_compat_free_counter(void* host_counter, void* device_counter);

/* RayGenerationPathTracing (src/Shading.cu:1727). stream: a cudaStream_t. */
int ymrt_compat_generate(int frame_index, const ymrt_render_setting* setting, void* device_counter,
                         uint32_t next_tile, uint32_t tile_count, uint32_t width, uint32_t height,
                         uint32_t tiles_x, uint32_t tiles_y, void* stream);

/* RayTracePathTracing (src/Shading.cu:1903): renders the marked frame into
 * noise_rgba (width*height float4, device memory) and clears the device
 * counter. */
int ymrt_compat_trace(int frame_index, const ymrt_render_setting* setting, void* device_counter, uint32_t width,
                      uint32_t height, float* noise_rgba, void* stream);

/* RayShadingPathTracing (src/Shading.cu:2304): clears the device counter. */
int ymrt_compat_shade(int frame_index, const ymrt_render_setting* setting, void* device_counter, uint32_t width,
                      uint32_t height, float* noise_rgba, void* stream);

/* RayGenerationEditorView / RayTraceEditorView / RayShadingEditorView
 * (src/Shading.cu:1333, 1442, 1596): the same protocol for the editor view
 * (the first generation call marks the frame, the trace call renders the
 * whole view with ymrt_render_editor_view into the caller's beauty and
 * primitive-index buffers and clears the device counter). */
int ymrt_compat_editor_generate(int frame_index, void* device_counter, uint32_t next_tile, uint32_t width,
                                uint32_t height, void* stream);
int ymrt_compat_editor_trace(int frame_index, const ymrt_render_setting* setting, void* device_counter, uint32_t width,
                             uint32_t height, float* beauty_rgba, uint32_t* primitive_index, void* stream);
int ymrt_compat_editor_shade(void* device_counter, void* stream);

/* PostProcessingEditorView / PostProcessingPathTracing (src/Shading.cu:
 * 2467-2515), with ymrt_post_process on device buffers. */
int ymrt_compat_post_process(float* image_rgba, const uint32_t* primitive_index, uint32_t width, uint32_t height,
                             uint32_t selected, float gamma, float exposure, int outline, void* stream);

/* AccumulateImagePathTracing (src/Shading.cu:2375): the running mean, skipped
 * once max_frames (> 0) frames have been accumulated, as the reference. */
int ymrt_compat_accumulate(const float* noise_rgba, float* acc_rgba, uint32_t width, uint32_t height, int frame_index,
                           int max_frames, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* YMRT_COMPAT_H_ */
