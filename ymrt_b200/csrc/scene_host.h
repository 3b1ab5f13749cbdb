// Host-side scene preparation for ymrt_b200.
//
// Reads YMRT's .ymtmp text format, builds the transforms, orders triangles and
// instances exactly as the reference's BVH builders do (so every triangle,
// instance and shape-light index a kernel reports is the index the reference
// reports), collapses those binary trees into compressed 8-wide BVHs, and
// flattens everything into the arrays the kernels read.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include <vector_types.h>

#include "bvh_build.h"
#include "ymrt_scene.h"

struct ymrt_scene_desc;
struct ymrt_texture_desc;

namespace ym {

// One geometry: a triangle mesh, or (kind kGeoSphere) an analytic sphere of
// `radius` with no triangles.
struct HostMesh {
  std::string name;
  uint32_t kind = kGeoMesh;
  float radius = 0.0f;
  std::vector<uint32_t> tris;      // corner triples (id0, id1, id2), reference post-build order
  std::vector<uint32_t> pos_idx, nrm_idx, uv_idx;
  std::vector<float> pos, nrm, uv;
  BBox root_box;                   // root box of the reference's mesh BVH
};

struct HostScene {
  // camera as written in the file
  vec3 cam_from{0.0f, 0.0f, 10.0f}, cam_look{0.0f, 0.0f, 4.0f};
  float cam_fov_deg = 45.0f;

  std::vector<mat4> transforms, i_transforms;
  std::vector<vec3> transform_scales;       // each Transform block's own (clamped) scale
  std::vector<HostMesh> meshes;
  std::vector<Instance> instances;          // after prepare(): reference order
  std::vector<uint32_t> instance_file_index;  // after prepare(): file index of each instance
  std::vector<Material> materials;
  std::vector<Texture> textures;
  std::map<uint32_t, std::vector<float>> images;  // pixels of each image node (Texture::image is set at upload)
  std::vector<Volume> volumes;
  std::vector<DistantLight> distant_lights;
  std::vector<ShapeLight> shape_lights;
  std::vector<float> shape_light_table;
  CameraDesc camera{};
  int width = 0, height = 0;
  uint32_t max_leaf_prims = 3;  // wide-BVH leaf size (1..4), a build option

  // flattened device-side arrays (filled by prepare())
  std::vector<GeometryDesc> geo_desc;
  std::vector<WideNode> blas_nodes, tlas_nodes;
  std::vector<float4> wtris;
  std::vector<uint32_t> tlas_prims;
  std::vector<uint32_t> tri_corners, all_pos_idx, all_nrm_idx, all_uv_idx;
  std::vector<float> all_pos, all_nrm, all_uv;
  size_t triangle_count_instanced = 0;
};

// Parses a .ymtmp file. Returns 0 or a negative YMRT_ERR_* code with a message.
int load_ymtmp(const std::string& path, HostScene* scene, std::string* error);

// Fills a scene from in-memory arrays (ymrt_scene_desc, include/ymrt.h):
// the same assets load_ymtmp produces, already resolved to indices. Returns 0
// or a negative YMRT_ERR_* code with a message.
int load_arrays(const ymrt_scene_desc* desc, HostScene* scene, std::string* error);

// Builds BVHs, orders instances/triangles/lights like the reference, sets up
// the rendering camera for a width x height image and flattens the arrays.
int prepare_scene(HostScene* scene, int width, int height, std::string* error);

// The top level of a prepared scene rebuilt from its current instance
// order: instance boxes, the reference's binary SAH build of them (the new
// instance order), the wide top-level BVH and the shape-light table.
int build_top_level(HostScene* scene, std::string* error);

// Replaces transforms first .. first+count-1 of a prepared scene (16 floats
// each, column major; world_to_object NULL: inverted here; scales NULL: kept)
// and rebuilds the top level and the camera's nested-media stack, as the
// reference's editor does after a transform edit.
int set_transforms(HostScene* scene, uint32_t first, uint32_t count, const float* object_to_world,
                   const float* world_to_object, const float* scales, std::string* error);

// The direction of the ray Camera::InitCameraRayTransfer casts from the
// camera (through the image centre) to find the media it sits in.
vec3 camera_media_ray(const CameraDesc& cam);

// Texture nodes in the words of ymrt_texture_desc (include/ymrt.h).
constexpr int kTextureWords = 20;
void texture_words(const Texture& t, uint32_t words[kTextureWords]);
int texture_from_desc(const ymrt_texture_desc& desc, Texture* t, std::string* error);

// Checks the texture graph a scene's materials and media read: indices in
// range, both inputs of every solid node present, no cycle, and no path of
// more than kTextureStack nodes (the evaluation stack). Returns 0 or
// `code` with a message.
int check_textures(const HostScene& scene, int code, std::string* error);

// Loads a PNG as the pixels of an image node (LoadImageTexture,
// src/FileIO.cpp:77-172: samples scaled by 1/255 or 1/65535, then decoded
// from sRGB unless the colour space is linear; mip 0 only; repeat wrap,
// unit scale, zero offset). Returns 0; YMRT_ERR_IO when the file cannot be
// read or decoded (the reference then leaves the node out); or
// YMRT_ERR_UNSUPPORTED for an image format other than PNG.
int load_image_texture(const std::string& path, uint32_t color_space, Texture* t, std::vector<float>* pixels,
                       std::string* error);

// The reference's sRGB decode of one sample (SRGBToLinear, src/MathCommon.h:136-139).
float srgb_to_linear(float s);

// glm-order transform helpers (exposed for tests through the C-ABI).
mat4 compose_transform(vec3 translate, vec3 scale, vec3 rotate_deg);
mat4 mat4_mul(const mat4& a, const mat4& b);
mat4 mat4_inverse(const mat4& m);

}  // namespace ym
