// Scene data shared by the host-side scene preparation and the sm_100a kernels.
//
// Records that cross the drop-in boundary keep the YMRT reference's byte
// layout (Material src/Material.h:9-359, Volume src/Volume.h:9-18,
// ShapeLight src/Light.h:80-86, PrimitiveInstance src/PrimtiveInstance.h:9-22,
// RenderSetting src/SceneDefines.h:17-40) so a caller holding the reference's
// arrays can pass them through unchanged. Everything the kernels traverse is
// this project's own layout: a compressed 8-wide BVH per mesh and one over the
// instances, triangles stored as three float4 vertices, geometry tables
// flattened into a few global arrays.
#pragma once

#include <cstdint>
#include <cstddef>

#include <vector_types.h>

#include "ymrt_math.h"

namespace ym {

constexpr int kMaxBoundaryRecord = 6;         // MAX_BOUNDARY_RECORD, src/Ray.h:12
constexpr int kMaxNearby = kMaxBoundaryRecord + 2;
constexpr int kMaxRayDepth = 64;              // MAX_RAY_DEPTH, src/SceneDefines.h:9
constexpr int kTileRes = 16;                  // TILE_X_RES / TILE_Y_RES
constexpr int kTilePixels = 256;
constexpr int kHaltonDims = 1000;             // PRIME_TABLE_SIZE, src/RandomSampler.cuh:12
constexpr int kMaxFreePath = 2048;            // MAX_FREE_PATH_LENGTH, src/VolumeEval.cuh:16

enum MaterialType : uint32_t { kDefaultMtl = 0, kLightMtl = 1 };

// DefaultMtl, src/Material.h:21-60 (152 bytes).
struct DefaultMtl {
  vec3 diffuse_albedo; uint32_t diffuse_albedo_tex;
  vec3 specular_albedo; uint32_t specular_albedo_tex;
  float alpha_x; uint32_t alpha_x_tex;
  float alpha_y; uint32_t alpha_y_tex;
  float specular_weight; uint32_t specular_weight_tex;
  float metalness; uint32_t metalness_tex;
  float transmission_weight; uint32_t transmission_weight_tex;
  float ior_n; uint32_t ior_priority;
  vec3 coat_albedo; uint32_t coat_albedo_tex;
  float coat_weight; uint32_t coat_weight_tex;
  float coat_thickness; uint32_t coat_thickness_tex;
  float coat_roughness_x; uint32_t coat_roughness_x_tex;
  float coat_roughness_y; uint32_t coat_roughness_y_tex;
  float coat_ior; uint32_t normal_mapping_tex;
  uint32_t bump_mapping_tex; uint32_t padding;
  uint32_t coat_normal_tex; uint32_t coat_normal_tex_type;
};
struct LightMtl {
  vec3 light_color;
  float intensity;
};
// Material, src/Material.h:200-207 (156 bytes).
struct Material {
  uint32_t material_type;
  union {
    DefaultMtl default_mtl;
    LightMtl light_mtl;
  };
};
static_assert(sizeof(DefaultMtl) == 152, "DefaultMtl layout");
static_assert(sizeof(Material) == 156, "Material layout");

// Volume, src/Volume.h:9-18 (36 bytes).
struct Volume {
  vec3 sigma_t;
  vec3 albedo;
  int density_texture_idx;
  uint32_t transform_idx;
  float g;
};
static_assert(sizeof(Volume) == 36, "Volume layout");

// ShapeLight, src/Light.h:80-86 (16 bytes): triangle `triangle_idx` (in the
// reference's post-build order) of instance `instance_idx`, or the whole
// sphere of a sphere instance (triangle_idx = EMPTY).
struct ShapeLight {
  uint32_t instance_idx;
  uint32_t triangle_idx;
  float power;
  float area;
};

// DistantLight, src/Light.h:324-388 (32 bytes): a cone of directions around
// the light transform's -y axis.
struct DistantLight {
  vec3 light_color;
  uint32_t transform_idx;
  float intensity;
  float cos_theta_max;
  float theta_max;
  float padding;
};
static_assert(sizeof(DistantLight) == 32, "DistantLight layout");

// PrimitiveInstance, src/PrimtiveInstance.h:9-22 (32 bytes).
struct Instance {
  uint32_t geometry_idx;
  uint32_t transform_idx;
  uint32_t transform_count;
  uint32_t material_idx;
  int inner_volume_idx;
  int treat_as_boundary;
  uint32_t unique_index;
  int padding;
};
static_assert(sizeof(Instance) == 32, "Instance layout");

// RenderSetting, src/SceneDefines.h:17-40 (40 bytes, x86-64 and device).
struct RenderSetting {
  int ssp;
  int ray_depth;
  float gamma;
  float exposure;
  int max_frame_count;
  int sampler_type;
  int enable_shape_light;
  bool enable_distant_light;
  bool enable_volume_scattering;
  bool enable_env_light;
  bool enable_russian_roulette;
  bool enable_indirect_clamp;
  float indirect_limit;
};
static_assert(sizeof(RenderSetting) == 40, "RenderSetting layout");

// Texture nodes (src/Texture.h:16-28, 84-690): images, constants and the
// solid (procedural) nodes, each solid node with a black and a white input
// node whose results it blends or selects. Children are texture indices
// (kEmpty: absent, reads as black). An image node holds its pixels (mip 0
// only, as the reference loads them) as floats, rows bottom-up, channels
// interleaved.
//
// kTexGrid is this project's density grid (the reference's texture graph has
// no grid node; a caller attaches one with ymrt_scene_set_density_grid): an
// nx x ny x nz lattice of values spanning the volume's object-space box
// [-0.5, 0.5]^3 with samples at cell centres, read trilinearly with clamped
// edges, stored as float32 or float16. `value` holds its maximum (the node's
// upper bound).
enum TextureType : uint32_t {
  kTexImage = 0, kTexConstFloat = 1, kTexConstRgb = 2, kTexChecker = 3, kTexNoise = 4, kTexFbm = 5,
  kTexTurbulence = 6, kTexMarble = 7, kTexWood = 8, kTexPolkaDot = 9, kTexWave = 10,
  kTexGrid = 64,
};
// Texture::flags bits.
constexpr uint32_t kTexNormalized = 1;  // noise: remapped from [-1, 1] to [0, 1]
constexpr uint32_t kTexTurbX = 2, kTexTurbY = 4, kTexTurbZ = 8;  // marble: coordinates added to the phase
constexpr int kTextureStack = 8;         // nodes on one evaluation path (the reference's texture_stack_size)
struct Texture {
  uint32_t type;
  uint32_t child[2];   // black / white inputs (kEmpty when absent)
  float value;         // constant float (grid: the maximum value)
  vec3 color;          // constant rgb
  float frequency, lacunarity, gain, amplitude, offset;  // checker .. wave (wave: its first fBm)
  int layer_count;
  uint32_t flags;      // kTexNormalized, kTexTurb*
  float variation;     // marble, wood
  float radius;        // polka dot
  float frequency1, lacunarity1, gain1;                  // wave: its second fBm
  int layer_count1;
  int grid_n[3];       // grid: lattice size x, y, z
  int grid_half;       // grid: values are float16 (else float32)
  const void* grid;    // grid: device values, x fastest
  int width, height, channels, wrap;             // image: size, samples per pixel, kWrap*
  float scale_u, scale_v, offset_u, offset_v;    // image: texture-coordinate transform
  uint32_t color_space;                          // image: kImageSrgb / kImageLinear (applied at load)
  const float* image;                            // image: device pixels
};
constexpr int kWrapRepeat = 0, kWrapClamp = 1;      // WARP_MODE_*, src/Texture.h:30-34
constexpr uint32_t kImageSrgb = 0, kImageLinear = 1;  // src/Texture.h:36-41

// Ray-transfer stack of nested media, src/Ray.h:106-260 (RayTransfer).
struct BoundaryRecord {
  uint32_t prim_idx;
  float ior;
  uint32_t ior_priority;
  int vol_idx;
};
struct RayTransfer {
  int max_priority_record_index;
  int record_count;
  BoundaryRecord records[kMaxBoundaryRecord];
};

// Pinhole camera (the reference's Camera, src/Camera.h:14-332, reduced to the
// fields ray generation reads) plus the media the camera sits in.
struct CameraDesc {
  vec3 position, u, v, w;
  float aspect_ratio;
  float tan_half_fov;
  RayTransfer transfer;
};

// ---- acceleration structures (this project's layout) ----

// One node of the compressed 8-wide BVH: 80 bytes, read as five 16-byte
// loads. Child boxes are quantised to 8 bits per bound on a per-node grid
// origin + q * 2^e (rounded outwards, so every decoded box contains the
// exact one). imask bit i set: child i is an internal node at
// child_base + meta[i]. Otherwise meta[i] = (count << 5) | offset: a leaf of
// `count` primitives at prim_base + offset (count 0: empty slot).
struct alignas(16) WideNode {
  float ox, oy, oz;
  uint8_t ex, ey, ez, imask;
  uint32_t child_base;
  uint32_t prim_base;
  uint8_t meta[8];
  uint8_t qlo_x[8], qlo_y[8], qlo_z[8];
  uint8_t qhi_x[8], qhi_y[8], qhi_z[8];
};
static_assert(sizeof(WideNode) == 80, "WideNode is five 16-byte words");

// GeometryData::geometry_type (src/GeometryDefines.h:10-14).
constexpr uint32_t kGeoMesh = 0, kGeoSphere = 1;

// Scene features the kernels are specialised on (template argument kF): a
// batch whose scenes hold no sphere geometry, no density grid or no textured
// surface (and no solid texture node beyond constants and fBm) runs
// instantiations without that code, so its register allocation is the same
// as if the feature did not exist.
constexpr uint32_t kFeatSpheres = 1, kFeatGrids = 2, kFeatTextures = 4, kFeatAll = 7;

// Per-geometry tables (offsets into the flattened global arrays). A sphere
// (kind kGeoSphere) is centred on its object-space origin and has no
// triangles or bottom-level nodes.
struct GeometryDesc {
  uint32_t tri_offset;      // into tri_corners (reference post-build triangle order)
  uint32_t tri_count;
  uint32_t corner_offset;   // into pos_idx / nrm_idx / uv_idx
  uint32_t pos_offset;      // into positions
  uint32_t nrm_offset;      // into normals
  int32_t uv_offset;        // into texcoords, -1 when the mesh has none
  uint32_t node_offset;     // root of the mesh's wide BVH in blas_nodes
  uint32_t wtri_offset;     // into wtris (wide-BVH triangle order)
  vec3 bbox_min, bbox_max;  // root box (object space)
  uint32_t kind;            // kGeoMesh or kGeoSphere
  float radius;             // sphere radius (Sphere::radius)
};

// Everything the kernels read, as device pointers.
// RenderSetting::sampler_type values (src/RandomSampler.cuh:617-620).
constexpr uint32_t kSamplerPcg = 0, kSamplerHalton = 1, kSamplerSobol = 2;

struct DeviceScene {
  // instances
  uint32_t instance_count;
  const Instance* instances;
  const mat4* transforms;
  const mat4* i_transforms;
  uint32_t transform_count;
  const uint8_t* inst_bucket;   // shading bucket of a hit on each instance
  // top-level BVH over instances
  const WideNode* tlas_nodes;
  const uint32_t* tlas_prims;   // instance index per TLAS leaf slot
  // meshes
  uint32_t geometry_count;
  const GeometryDesc* geometries;
  uint32_t sphere_count;        // sphere geometries (0: the traversal skips sphere tests)
  uint32_t grid_count;          // density-grid texture nodes
  uint32_t textured;            // materials read textures, or solid nodes beyond constants and fBm exist
  const WideNode* blas_nodes;
  const float4* wtris;          // 3 per triangle: v0, v1, v2 (w of v0 = triangle id bits)
  const uint32_t* tri_corners;  // 3 per triangle (Triangle id0,id1,id2)
  const uint32_t* pos_idx;
  const uint32_t* nrm_idx;
  const uint32_t* uv_idx;
  const float* positions;       // xyz
  const float* normals;         // xyz
  const float* texcoords;       // uv
  // materials, lights, media
  uint32_t material_count;
  const Material* materials;
  uint32_t distant_light_count;
  const DistantLight* distant_lights;
  uint32_t shape_light_count;
  const ShapeLight* shape_lights;
  const float* shape_light_table;
  uint32_t volume_count;
  const Volume* volumes;
  uint32_t texture_count;
  const Texture* textures;
  // sampler
  uint32_t sampler_type;            // RenderSetting::sampler_type of the current render
  const uint32_t* halton_perm;
  const uint32_t* sobol_matrices;   // 4096 dimensions x 32 columns (input; null until set)
  // camera
  CameraDesc camera;
  int width, height;
  // Halton enumerator (src/HaltonEnumerator.h:13-38)
  float halton_x_scale, halton_y_scale;
  int halton_mx, halton_my, halton_exp2, halton_exp3, halton_increment;
};

}  // namespace ym
