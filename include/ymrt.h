/*
 * ymrt.h -- C ABI of the ymrt_b200 wavefront path tracer (sm_100a).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (0 = YMRT_OK, negative = YMRT_ERR_*). No exception or C++ type crosses
 * this boundary.
 *
 * What each entry point replaces in the YMRT reference (paths relative to
 * the reference project):
 *
 *   ymrt_scene_load_ymtmp   SceneParser::parsing_scene          src/core/YMParser.cpp:2330
 *                           + the scene preparation of
 *                           GuiModule::UpdateScene (BVH build,
 *                           shape-light table, camera)          src/core/GuiModule.cpp:116-282
 *   ymrt_scene_upload       GuiModule::UpdateScene device upload src/core/GuiModule.cpp:173-272
 *                           (UPLOAD_TO_GPU of every array)
 *   ymrt_render_forward     one progressive frame of
 *                           RenderModule::PathTracingExecuteTask src/core/RenderModule.cpp:494-653
 *                           i.e. the stage launchers
 *                           RayGenerationPathTracing            src/Shading.cu:1727
 *                           RayTracePathTracing                 src/Shading.cu:1903
 *                           RayShadingPathTracing               src/Shading.cu:2304
 *                           into the frame's noise image
 *   ymrt_accumulate         AccumulateImagePathTracing          src/Shading.cu:2375
 *   ymrt_debug_trace        TraceRay                            src/ShadingUtilities.cuh:310
 *   ymrt_debug_occluded     BVHTraverseShadow                   src/ShadingUtilities.cuh:563
 *   ymrt_debug_halton       HaltonEnumerator::GetIndex +        src/HaltonEnumerator.h:43
 *                           HaltonSampler::Random1D             src/RandomSampler.cuh:430
 *
 * Threading: a context owns one CUDA stream; use one context per host
 * thread. Scenes belong to the context they were uploaded with.
 */
#ifndef YMRT_H_
#define YMRT_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define YMRT_OK 0
#define YMRT_ERR_INVALID (-1)     /* bad argument */
#define YMRT_ERR_IO (-2)          /* file cannot be read */
#define YMRT_ERR_FORMAT (-3)      /* malformed .ymtmp */
#define YMRT_ERR_UNSUPPORTED (-4) /* valid input this build does not render */
#define YMRT_ERR_CUDA (-5)        /* CUDA runtime error (see ymrt_last_error) */
#define YMRT_ERR_OOM (-6)         /* device allocation failed */
#define YMRT_ERR_TIMEOUT (-7)     /* a bounded device loop gave up */
#define YMRT_ERR_OVERFLOW (-8)    /* a queue or stack limit was exceeded */
#define YMRT_ERR_NO_DEVICE (-9)   /* no CUDA device, or the kernels are missing */

typedef struct ymrt_context ymrt_context;
typedef struct ymrt_host_scene ymrt_host_scene;
typedef struct ymrt_scene ymrt_scene;

/* Byte-compatible with the reference's RenderSetting (src/SceneDefines.h:17-40). */
typedef struct ymrt_render_setting {
  int ssp;                 /* samples per pixel per frame */
  int ray_depth;           /* bounces before Russian roulette / termination */
  float gamma;             /* unused on this path (display only) */
  float exposure;          /* unused on this path (display only) */
  int max_frame_count;
  int sampler_type;        /* 0 PCG, 1 Halton, 2 Sobol (this build renders Halton) */
  int enable_shape_light;
  uint8_t enable_distant_light;
  uint8_t enable_volume_scattering;
  uint8_t enable_env_light;
  uint8_t enable_russian_roulette;
  uint8_t enable_indirect_clamp;
  uint8_t pad_[3];
  float indirect_limit;
} ymrt_render_setting;

/* Per-frame counters and timings filled by ymrt_render_forward. */
typedef struct ymrt_stats {
  uint64_t paths;            /* camera paths started */
  uint64_t extension_rays;   /* closest-hit queries */
  uint64_t shadow_rays;      /* any-hit (occlusion) queries */
  uint64_t waves;            /* extend/shade iterations */
  uint64_t node_visits;      /* wide-BVH nodes fetched by all queries */
  uint64_t triangle_tests;   /* triangles fetched and tested by all queries */
  uint64_t kernel_launches;  /* kernels launched for the frame */
  double ms_total;           /* device time of the frame (CUDA events) */
  double ms_generate;        /* per-kernel device time; filled when profiling is on */
  double ms_extend;          /* closest-hit kernel */
  double ms_shade;           /* shading kernel */
  uint32_t device_errors;    /* bit set of YMRT_DEVERR_* raised on the device */
  uint32_t tracking_bound_hits; /* delta / ratio tracking loops that stopped at the reference's
                                   MAX_FREE_PATH_LENGTH (2048 steps, src/VolumeEval.cuh:16, :144,
                                   :328), as the reference's do: not an error */
  uint64_t shadow_node_visits;     /* the part of node_visits made by occlusion queries */
  uint64_t shadow_triangle_tests;  /* the part of triangle_tests made by occlusion queries */
  double ms_sort;            /* hit listing by shading bucket (profiling on) */
  double ms_connect;         /* deferred shadow-ray kernel (profiling on) */
  uint64_t shaded_hits;      /* path vertices shaded (extension rays that hit) */
} ymrt_stats;

#define YMRT_DEVERR_STACK 1u     /* a traversal stack overflowed (entries were dropped) */
#define YMRT_DEVERR_QUEUE 2u     /* a path queue overflowed */
#define YMRT_DEVERR_ITER 4u      /* a bound of this library's own (shadow-ray boundary crossings, waves of a
                                    frame, editor-view boundaries) was reached; the render returns
                                    YMRT_ERR_OVERFLOW */

/* ---- contexts ---- */
int ymrt_create(int device_ordinal, ymrt_context** out);
void ymrt_destroy(ymrt_context* ctx);
/* Last error message of the context (or of the library when ctx is NULL). */
const char* ymrt_last_error(const ymrt_context* ctx);
/* Largest number of paths in flight (queue slots); 0 keeps the default. */
int ymrt_set_queue_capacity(ymrt_context* ctx, uint32_t paths);
/* When enabled, every stage launch is bracketed by CUDA events and the
 * per-stage times are reported in ymrt_stats (costs a little host time). */
int ymrt_set_profiling(ymrt_context* ctx, int enable);
/* Wave-loop options (no counterpart in the reference, whose stages have one
 * fixed form; results are the same either way up to the order of per-pixel
 * float additions):
 *   YMRT_OPT_SORT_HITS     (default 1) shade hits grouped by material lobes
 *   YMRT_OPT_DEFER_SHADOWS (default 1) queue surface shadow rays and trace
 *                          them in a separate kernel (not used with volume
 *                          scattering or the indirect clamp)
 *   YMRT_OPT_GRAPH_LOOP    (default 1) run the whole wave loop as one CUDA
 *                          graph (a device-side while loop) instead of one
 *                          host round trip per wave; off while profiling */
#define YMRT_OPT_SORT_HITS 1
#define YMRT_OPT_DEFER_SHADOWS 2
#define YMRT_OPT_GRAPH_LOOP 3
/*   YMRT_OPT_TRACE_BLOCK   (default 128) threads per block of the closest-hit
 *                          and shadow-ray kernels: 64, 128 or 256 */
#define YMRT_OPT_TRACE_BLOCK 4
/*   YMRT_OPT_SORT_RAYS     (default 1) trace each wave's continuing rays
 *                          grouped by origin cell and direction instead of
 *                          in the order shading left them (same hits) */
#define YMRT_OPT_SORT_RAYS 6
int ymrt_set_option(ymrt_context* ctx, int option, int value);
int ymrt_get_option(const ymrt_context* ctx, int option, int* value);

/* ---- scenes ---- */
/* Parses and prepares a scene on the host (no GPU needed). err may be NULL. */
int ymrt_scene_load_ymtmp(const char* path, int width, int height, ymrt_host_scene** out, char* err,
                          size_t err_len);
/* Scene build options (no counterpart in the reference, whose binary BVH has
 * one primitive per leaf). */
typedef struct ymrt_load_options {
  uint32_t max_leaf_triangles; /* wide-BVH leaf size, 1..4 (default 3); also instances per top-level leaf */
  uint32_t override_camera;    /* nonzero: the camera below replaces the file's Camera block (other views) */
  float camera_from[3], camera_look[3], camera_fov_deg;
  uint32_t reserved[7];
} ymrt_load_options;
int ymrt_scene_load_ymtmp_ex(const char* path, int width, int height, const ymrt_load_options* options,
                             ymrt_host_scene** out, char* err, size_t err_len);
void ymrt_host_scene_free(ymrt_host_scene* scene);

/* ---- scenes from memory ----
 * For a host that holds its scene in memory (the reference editor's
 * SceneModule arrays, src/core/SceneModule.h:288-326) instead of a .ymtmp
 * file: the same assets, already resolved to indices, prepared exactly as
 * ymrt_scene_load_ymtmp_ex prepares a parsed file (GuiModule::UpdateScene,
 * src/core/GuiModule.cpp:116-282). All arrays are host memory and are
 * copied; the caller keeps them. */
typedef struct ymrt_mesh_desc {
  /* Triangle mesh in creation order (as CreateMesh receives it,
   * src/core/SceneModule.cpp:239-262): the library orders the triangles as
   * the reference's mesh build does. 3 corner indices per triangle; one
   * position / normal (/ texcoord) index per corner. */
  const uint32_t* triangles;
  uint32_t triangle_count;
  const uint32_t* position_indices;
  const float* positions;          /* xyz */
  uint32_t position_count;
  const uint32_t* normal_indices;
  const float* normals;            /* xyz */
  uint32_t normal_count;
  const uint32_t* texcoord_indices; /* NULL: no texture coordinates */
  const float* texcoords;           /* uv */
  uint32_t texcoord_count;
  /* > 0: an analytic sphere of this radius (a Sphere block); the arrays are
   * then ignored. */
  float sphere_radius;
} ymrt_mesh_desc;

/* A texture node, in the words YMRT_QUERY_TEXTURES returns (20 per node):
 * type (src/Texture.h:16-28: 1 constant float, 2 constant rgb,
 * 3 checkerboard, 4 noise, 5 fBm, 6 turbulence, 7 marble, 8 wood,
 * 9 polka dot, 10 wave; 64 a density grid, which only
 * ymrt_scene_set_density_grid makes), the black and white input nodes
 * (0xFFFFFFFF: none; the solid nodes 3-10 require both), and the node's
 * parameters. Unused words are 0. Fields per type:
 *   constant float: value;  constant rgb: color;
 *   checkerboard: frequency;  noise: frequency, flags bit 0 (normalized);
 *   fBm, turbulence: frequency, lacunarity, gain, layer_count, amplitude, offset;
 *   marble: frequency, lacunarity, gain, layer_count, variation,
 *           flags bits 1-3 (x, y, z coordinate added to the phase);
 *   wood: frequency, variation;  polka dot: frequency, radius;
 *   wave: frequency, lacunarity, gain, layer_count (first fBm),
 *         frequency1, lacunarity1, gain1, layer_count1 (second fBm);
 *   image (type 0; ImageTexture, src/Texture.h:84-166): words 3-6 are
 *         int32 width, height, channels (1-4), wrap (0 repeat, 1 clamp);
 *         words 7-10 float scale_u, scale_v, offset_u, offset_v; word 15 the
 *         colour space its pixels were decoded from (0 sRGB, 1 linear). Its
 *         pixels are given with ymrt_host_scene_set_image. */
typedef struct ymrt_texture_desc {
  uint32_t type;
  uint32_t black, white;
  float value;
  float color[3];
  float frequency, lacunarity, gain;
  int32_t layer_count;
  float amplitude, offset;
  float variation, radius;
  uint32_t flags;
  float frequency1, lacunarity1, gain1;
  int32_t layer_count1;
} ymrt_texture_desc;

typedef struct ymrt_scene_desc {
  const float* transforms;          /* 16 floats per transform, column major (glm::mat4) */
  const float* inverse_transforms;  /* NULL: inverted here (glm's inverse) */
  const float* transform_scales;    /* xyz per transform (its Transform's own scale; sizes sphere lights); NULL: 1 */
  uint32_t transform_count;
  const ymrt_mesh_desc* geometries;
  uint32_t geometry_count;
  const void* instances;            /* PrimitiveInstance, 32 bytes each, creation order */
  uint32_t instance_count;
  const void* materials;            /* Material, 156 bytes each (src/Material.h) */
  uint32_t material_count;
  const void* volumes;              /* Volume, 36 bytes each (src/Volume.h) */
  uint32_t volume_count;
  const void* distant_lights;       /* DistantLight, 32 bytes each (src/Light.h:324-388) */
  uint32_t distant_light_count;
  const ymrt_texture_desc* textures;
  uint32_t texture_count;
  float camera_from[3], camera_look[3], camera_fov_deg;
} ymrt_scene_desc;

int ymrt_scene_from_arrays(const ymrt_scene_desc* desc, int width, int height, const ymrt_load_options* options,
                           ymrt_host_scene** out, char* err, size_t err_len);

/* Host-scene queries (for parity checks against the reference's own scene
 * preparation). Each copies into `out` (capacity `cap` elements) and returns
 * the element count, or a negative YMRT_ERR_*. */
#define YMRT_QUERY_COUNTS 0      /* uint64[8]: instances, meshes, triangles, instanced triangles, lights, blas nodes, tlas nodes, materials */
#define YMRT_QUERY_INSTANCES 1   /* uint32[6*n]: geometry, transform, material, volume, boundary, file index */
#define YMRT_QUERY_LIGHTS 2      /* float[4*n]: instance (bits), triangle (bits), power, area */
#define YMRT_QUERY_LIGHT_TABLE 3 /* float[n] */
#define YMRT_QUERY_TRANSFORMS 4  /* float[32*n]: object-to-world then world-to-object, column major */
#define YMRT_QUERY_CAMERA 5      /* float[14]: position, u, v, w, aspect, tan(fov/2) */
#define YMRT_QUERY_TRIANGLES 6   /* uint32[3*n] corner triples of mesh `index`, reference order */
#define YMRT_QUERY_MATERIALS 7   /* uint32[39*n]: the reference's Material struct words */
#define YMRT_QUERY_VOLUMES 8     /* uint32[9*n]: the reference's Volume struct words */
#define YMRT_QUERY_DISTANT_LIGHTS 9 /* uint32[8*n]: the reference's DistantLight struct words */
#define YMRT_QUERY_TEXTURES 10   /* uint32[20*n]: ymrt_texture_desc words per node */
#define YMRT_QUERY_GEOMETRIES 11 /* uint32[2*n]: kind (0 triangle mesh, 1 sphere), sphere radius (float bits) */
#define YMRT_QUERY_MESH_CORNERS 12 /* float[8*c] of mesh `index`, by corner: position, normal, uv (0 without texcoords) */
#define YMRT_QUERY_IMAGE_PIXELS 13 /* float[w*h*channels] of image node `index`: linear samples, bottom row first */
long long ymrt_host_scene_query(const ymrt_host_scene* scene, int what, int index, void* out, size_t cap);

/* Uploads a prepared scene. halton_perm: the concatenated digit permutations
 * of the first 1000 primes (3,682,913 uint32), the table the reference keeps
 * in Scene::sampler_data.halton_permute_table. */
int ymrt_scene_upload(ymrt_context* ctx, const ymrt_host_scene* scene, const uint32_t* halton_perm, size_t perm_len,
                      ymrt_scene** out);
/* Generator matrices of the Sobol sampler (RenderSetting::sampler_type 2):
 * 4096 dimensions x 32 columns, the reference's sobol_matrices32 table
 * (src/LowDiscrepancy.cpp:179), which its GuiModule::UpdateScene uploads
 * (src/core/GuiModule.cpp:256). Needed only for Sobol renders. */
int ymrt_scene_set_sobol_matrices(ymrt_scene* scene, const uint32_t* matrices, size_t count);
/* Scenes must be freed before the context they were uploaded to. */
void ymrt_scene_free(ymrt_scene* scene);

/* ---- transform edits ----
 * The reference's editor rebuilds its top-level BVH on the host after every
 * transform edit, reordering the instances by the build, then uploads the
 * whole scene again (GuiModule::UpdateScene, src/core/GuiModule.cpp:123-139;
 * TopBVH.cpp:34-198, the instance reorder at :171-191).
 *
 * ymrt_scene_set_transforms does it where the uploaded scene lives: it
 * replaces transforms first .. first+count-1 (16 floats each, column major,
 * object to world; world_to_object NULL: inverted here as glm inverts;
 * scales, 3 per transform, the Transform's own scale that sizes sphere
 * lights: NULL keeps them) and rebuilds on the device the instance world
 * boxes, the binary SAH build of them (which reorders the instances), the
 * wide top-level BVH, the shape-light table and the camera's nested-media
 * stack, bit for bit as ymrt_host_scene_set_transforms rebuilds a host scene.
 * The meshes' own trees are in object space and are kept. Instance indices
 * reported afterwards are the new order's (as in the reference). */
int ymrt_scene_set_transforms(ymrt_scene* scene, uint32_t first, uint32_t count, const float* object_to_world,
                              const float* world_to_object, const float* scales);
int ymrt_host_scene_set_transforms(ymrt_host_scene* scene, uint32_t first, uint32_t count,
                                   const float* object_to_world, const float* world_to_object, const float* scales);

/* Device contents of an uploaded scene's top level, to compare with a host
 * build: copies into `out` (cap_bytes) and returns the bytes, or the bytes
 * needed when out is NULL, or a negative YMRT_ERR_*. */
#define YMRT_SCENE_TLAS_NODES 1      /* wide top-level nodes, 80 bytes each */
#define YMRT_SCENE_TLAS_PRIMS 2      /* uint32 instance per top-level leaf slot */
#define YMRT_SCENE_INSTANCES 3       /* PrimitiveInstance, 32 bytes each, current order */
#define YMRT_SCENE_SHAPE_LIGHTS 4    /* ShapeLight, 16 bytes each */
#define YMRT_SCENE_LIGHT_TABLE 5     /* float power CDF */
#define YMRT_SCENE_INSTANCE_BUCKETS 6 /* uint8 shading bucket per instance */
#define YMRT_SCENE_CAMERA_MEDIA 7    /* the camera's RayTransfer, 104 bytes */
#define YMRT_SCENE_FILE_INDEX 8      /* uint32 file index of each instance */
long long ymrt_scene_download(const ymrt_scene* scene, int what, void* out, size_t cap_bytes);

/* ---- rendering ---- */
/* Renders one progressive frame (frame_index >= 1) of every tile into
 * out_rgba (width*height float4, linear radiance averaged over the frame's
 * samples, alpha = 1), like the reference's noise image. out_rgba is a device
 * pointer when out_on_device != 0, else host memory (copied back before
 * returning). stats may be NULL. */
int ymrt_render_forward(ymrt_scene* scene, const ymrt_render_setting* setting, int frame_index, float* out_rgba,
                        int out_on_device, ymrt_stats* stats);
/* Same, restricted to tiles [tile_begin, tile_end) of the 16x16 tiling. */
int ymrt_render_tiles(ymrt_scene* scene, const ymrt_render_setting* setting, int frame_index, int tile_begin,
                      int tile_end, float* out_rgba, int out_on_device, ymrt_stats* stats);

/* One render of a batch. */
typedef struct ymrt_job {
  ymrt_scene* scene;             /* uploaded scene (its resolution and camera) */
  ymrt_render_setting setting;
  int frame_index;               /* >= 1 */
  int tile_begin, tile_end;      /* 16x16 tiles to render; 0, 0 = all */
  float* out_rgba_device;        /* width*height*4 floats of device memory, overwritten */
  /* differentiable rendering (NULL otherwise): */
  float* path_radiance_device;   /* forward: receives each path's radiance (ymrt_job_path_count * 4 floats) */
  const float* dloss_device;     /* backward: dLoss/dImage, width*height*4 floats */
} ymrt_job;

/* Paths a job renders: tiles * 256 * spp (sizes path_radiance_device). */
unsigned long long ymrt_job_path_count(const ymrt_job* job);

/* Path-replay adjoint (no counterpart in the reference, which has no
 * backward pass): gradients of a loss with respect to every material's
 * diffuse albedo (rgb) and roughness (alpha_x = alpha_y), given dLoss/dImage
 * per job. The jobs must be the ones rendered (by ymrt_render_batch) with
 * path_radiance_device set, with unchanged scenes and settings: every path is
 * re-traced with its own samples. grads_device receives 4 floats per material
 * (n_materials materials, in the scene's material order), overwritten.
 * The indirect clamp is rejected. */
int ymrt_render_backward(ymrt_context* ctx, const ymrt_job* jobs, int n_jobs, float* grads_device,
                         uint32_t n_materials, ymrt_stats* stats);

/* What ymrt_render_backward_ex differentiates. Either target may be absent
 * (NULL). Material gradients: 4 floats per material as ymrt_render_backward.
 * Density-grid gradients (no counterpart in the reference): dLoss/d(value)
 * of the grid attached to texture node grid_texture
 * (ymrt_scene_set_density_grid), one float per grid value in the grid's
 * order, summed over every job; each job's scene must hold a grid of
 * grid_values values at that node, and the jobs must scatter in media. */
typedef struct ymrt_backward_targets {
  float* material_grads_device;
  uint32_t n_materials;
  uint32_t grid_texture;
  float* grid_grads_device;
  uint64_t grid_values;
  uint32_t reserved[4];
} ymrt_backward_targets;

/* ymrt_render_backward with material and/or density-grid targets; media
 * (volume scattering) are differentiated too: free-flight sampling and
 * shadow-ray transmittance contribute the grid's terms, with the tracking
 * decisions and the majorant held fixed. The outputs are overwritten. */
int ymrt_render_backward_ex(ymrt_context* ctx, const ymrt_job* jobs, int n_jobs, const ymrt_backward_targets* targets,
                            ymrt_stats* stats);

/* Material parameters a backward pass differentiates, 4 floats per material:
 * diffuse albedo r, g, b and roughness (stored as alpha_x and alpha_y). Light
 * materials are skipped (set) or read as zeros (get). */
int ymrt_scene_set_material_params(ymrt_scene* scene, uint32_t first, uint32_t count, const float* params);
/* Attaches a density grid to texture node `texture_index` (replacing that
 * node; no counterpart in the reference, whose texture graph has no grid): a
 * volume whose density texture is that node then reads the grid. values holds
 * nx*ny*nz floats in host memory, x fastest, sampled at cell centres of the
 * volume's object-space box [-0.5, 0.5]^3, read trilinearly with clamped
 * edges; store_half != 0 keeps them as float16 (rounded to nearest). The
 * node's upper bound, which sets the delta-tracking majorant, is the grid's
 * maximum. Values must be finite; calling it again replaces the grid. */
int ymrt_scene_set_density_grid(ymrt_scene* scene, uint32_t texture_index, int nx, int ny, int nz,
                                const float* values, int store_half);

int ymrt_scene_get_material_params(const ymrt_scene* scene, uint32_t first, uint32_t count, float* params);

/* Renders n_jobs renders (scenes, resolutions, spp and settings may all
 * differ; scenes must belong to ctx) together: their paths share the wave
 * queues, so small renders keep the GPU full. Same results as rendering each
 * job with ymrt_render_tiles. No counterpart in the reference, which renders
 * one frame per PathTracingExecuteTask. */
int ymrt_render_batch(ymrt_context* ctx, const ymrt_job* jobs, int n_jobs, ymrt_stats* stats);
/* Allocation-free variant of ymrt_render_tiles, for callers that cannot
 * allocate device memory while rendering (a host with a fixed up-front
 * memory budget or its own pool allocator, or code that must not let a
 * cudaMalloc synchronise the device mid-frame). It has no counterpart in the
 * reference. The path queues, hit records and counters live in one fixed
 * 32 MiB array that every device holds while the library is loaded; the
 * caller passes the scene and a device output image (width*height float4).
 * Limits: 256 * spp paths (one tile) must fit in the array, i.e.
 * spp <= ymrt_noalloc_max_paths() / 256; larger spp is rejected with
 * YMRT_ERR_INVALID. The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress), so make that first call before any stream
 * capture. All calls share the array: calls that overlap on the GPU race and
 * must be serialised by the caller. */
int ymrt_render_tiles_noalloc(ymrt_scene* scene, const ymrt_render_setting* setting, int frame_index, int tile_begin,
                              int tile_end, float* out_rgba_device, ymrt_stats* stats);
/* Path slots available to ymrt_render_tiles_noalloc. */
uint32_t ymrt_noalloc_max_paths(void);

/* Running mean over frames (device pointers): acc = (acc*(f-1) + noise) / f. */
int ymrt_accumulate(ymrt_scene* scene, const float* noise_rgba, float* acc_rgba, int frame_index);

/* ---- known-answer entry points (host buffers) ---- */
int ymrt_debug_trace(ymrt_scene* scene, int n, const float* origin, const float* dir, const uint32_t* last_hit,
                     uint32_t* inst, uint32_t* tri, float* t, float* bary, int* back, int* nearby);
/* Renders one frame of tiles [tile_begin, tile_end) like ymrt_render_tiles
 * (into out_rgba, a host array of width*height*4 floats; waves launched
 * from the host) and records, after every closest-hit stage, the vertex of
 * each path whose pixel has its bit set in watch_bits (host, one bit per
 * pixel index y*width+x): 24 words per vertex -- pixel, depth (1 = camera
 * ray), flags (1 hit, 2 volume scattering, 4 back face), instance, triangle,
 * t, origin[3], direction[3], barycentrics or scattering position[3],
 * throughput[3], light received so far[3], path index, 2 unused -- the
 * state the reference's trace stage holds at the same point
 * (Ray_trace_path_tracing, src/Shading.cu:1829-1854), so that paths can be
 * compared vertex by vertex. *n_records = vertices recorded;
 * YMRT_ERR_OVERFLOW when that exceeds `capacity` (the first `capacity` are
 * returned). */
int ymrt_debug_record_paths(ymrt_scene* scene, const ymrt_render_setting* setting, int frame_index, int tile_begin,
                            int tile_end, const uint32_t* watch_bits, uint32_t* records, int capacity,
                            int* n_records, float* out_rgba);
/* Value of texture node `texture_index` at n object-space points (3 floats
 * each; host buffers), as the media read it: known-answer checks of grid and
 * fBm nodes. */
int ymrt_debug_density(ymrt_scene* scene, uint32_t texture_index, int n, const float* points, float* out);
/* The shading frame at n given hits (instance, triangle, barycentrics (3),
 * back flag, ray direction (3); host buffers): out 22 floats per hit --
 * normal, tangent, bitangent, texture footprint du/dx dv/dx du/dy dv/dy, uv,
 * object-space position, dp/du, material index -- as the shade stage builds
 * it (FetchShadingData, Camera::TextureCoordinatesDifferential,
 * MaterialBSDF::InitShadingSpace): a known-answer check of normal and bump
 * mapping. */
int ymrt_debug_frame(ymrt_scene* scene, int n, const uint32_t* inst, const uint32_t* tri, const float* bary,
                     const int* back, const float* dir, float* out);

/* ---- editor view and post-processing ---- */

/* The editor's albedo / picking view (Ray_generation_editor_view,
 * Ray_trace_editor_view, Ray_shading_editor_view, src/Shading.cu:1276-1594)
 * of a width x height image from the scene's camera (aspect width/height):
 * per pixel one ray through the pixel centre, followed through pass-through
 * boundaries; the surface colour (diffuse albedo or its texture, a light's
 * colour x intensity, black for an invalid material) or, on a miss, the
 * background when setting->enable_env_light (else black) is ADDED to
 * beauty_rgba with alpha 1, and the first hit's instance unique_index is
 * written to primitive_index (a miss leaves it). device_buffers: 1 when both
 * buffers are device memory, 0 for host memory. */
int ymrt_render_editor_view(ymrt_scene* scene, const ymrt_render_setting* setting, uint32_t width, uint32_t height,
                            float* beauty_rgba, uint32_t* primitive_index, int device_buffers);

/* PostProcessingPathTracing / PostProcessingEditorView (src/Shading.cu:
 * 2396-2516): ACES tone mapping of exposure x colour, then 1/gamma, alpha 1;
 * with outline != 0 and selected != 0xFFFFFFFF, pixels whose 3x3
 * neighbourhood shows instance `selected` (primitive_index) partly turn red
 * and wholly get a 60% red tint. In place. */
int ymrt_post_process(ymrt_context* ctx, float* image_rgba, const uint32_t* primitive_index, uint32_t width,
                      uint32_t height, uint32_t selected, float gamma, float exposure, int outline,
                      int device_buffers);

/* SavePngImage (src/FileIO.cpp:167-194): writes a host image of width x
 * height float RGBA pixels, bottom row first (the order render output is in),
 * as an 8-bit RGBA PNG with each channel (uint8)(clamp(v, 0, 1) * 255 + 0.5).
 * The path's extension is replaced by .png and missing parent directories are
 * created. YMRT_ERR_INVALID for bad arguments, YMRT_ERR_IO when the file
 * cannot be written. No device is needed. */
int ymrt_save_png(const char* path, const float* rgba, int width, int height);

/* Pixels of image node `texture_index` of a host scene (from
 * ymrt_scene_from_arrays, or replacing a loaded image): count =
 * width * height * channels linear floats, channels interleaved, bottom row
 * first (the layout the reference's loader produces, src/FileIO.cpp:77-172). */
int ymrt_host_scene_set_image(ymrt_host_scene* scene, uint32_t texture_index, const float* pixels, size_t count);

/* Value (rgb) of texture node `texture_index` as a surface reads it, at n
 * points of 5 floats each: texture coordinates s, t and the object-space
 * position x, y, z (host buffers): known-answer checks of every node type. */
int ymrt_debug_texture(ymrt_scene* scene, uint32_t texture_index, int n, const float* coords, float* rgb);
/* Where a bounded device loop last gave up (the event behind
 * YMRT_DEVERR_ITER; no counterpart in the reference, whose loops have no
 * bound): the first such event on the context's device since the record was
 * last cleared, as 32-bit words -- taken (0: none, 1: written), site
 * (1 shadow-ray boundary crossings, 2 delta-tracking steps, 3 ratio-tracking
 * steps, 4 waves of a frame, 5 editor-view boundaries, 6 texture-graph walk),
 * the iteration count, the ray's last instance and triangle, origin (3
 * floats), direction (3), remaining length, the tracking majorant (3) and
 * channel, then its nested-media stack (max-priority index, record count,
 * 6 records of prim, ior, priority, volume). words receives up to n_words
 * words (42 in all); clear != 0 resets the record afterwards. */
int ymrt_debug_bound_record(ymrt_context* ctx, uint32_t* words, size_t n_words, int clear);
/* Fault injection for tests of the error paths (no counterpart in the
 * reference): the next `count` device allocations this library makes fail
 * as out of memory (the call that needs them returns YMRT_ERR_OOM and leaves
 * the context usable); 0 stops it. */
void ymrt_debug_fail_allocations(int count);
int ymrt_debug_occluded(ymrt_scene* scene, int n, const float* origin, const float* dir, const float* tmax,
                        int* occluded);
int ymrt_debug_halton(ymrt_scene* scene, int n, const int* px, const int* py, const int* sample, int n_dims,
                      uint64_t* index, float* offset, float* dims);

#ifdef __cplusplus
}
#endif

#endif /* YMRT_H_ */
