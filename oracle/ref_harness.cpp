// Headless host driver for the YMRT reference (the oracle).
//
// TEST INFRASTRUCTURE ONLY. Built by oracle/build_ref.py into
// oracle/_ref/libymrt_ref.so from the reference sources where they lie; only
// tests/, __graft_entry__.smoke() and bench.py's CPU-baseline/reference legs
// load it. The ymrt_b200 product never links or calls it.
//
// What it does: loads a .ymtmp scene with the reference's own parser and scene
// module (src/core/YMParser.cpp:2330 SceneParser::parsing_scene), prepares the
// scene exactly as the reference editor does before rendering
// (src/core/GuiModule.cpp:116-282 GuiModule::UpdateScene: top-level BVH build
// with instance reordering, shape-light table, camera ray-transfer), and runs
// the reference's three wavefront stage kernels (src/Shading.cu:1634
// Ray_generation_path_tracing, :1765 Ray_trace_path_tracing, :1953
// Ray_shading_path_tracing) as host functions with the wave protocol of
// src/core/RenderModule.cpp:494-653 (PathTracingExecuteTask). Blocks of each
// emulated launch are spread over host threads; threadIdx/blockIdx are
// thread_local.
//
// The wave capacity is a parameter (the reference uses 1 Mi rays). Each
// path's result is independent of how paths are packed into waves, so the
// per-pixel output equals the reference's up to the order of the per-pixel
// float additions when spp > 1.
#include YMRT_SHADING_SOURCE

#include "core/SceneModule.h"
#include "FileIO.h"
#include "core/YMParser.h"

#include <atomic>
#include <cstring>
#include <chrono>
#include <thread>

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

#include "ref_prepare.h"

using namespace YMRT;

namespace {

struct Queues {
  std::vector<Ray> s_ray;
  std::vector<glm::vec3> s_light, s_tp;
  std::vector<int> s_px, s_py, s_depth, s_never, s_cam, s_psi;
  std::vector<RandomSampler> s_sampler;
  std::vector<RayTransfer> s_transfer;

  std::vector<HitRecord> h_rec;
  std::vector<int> h_nearby_count;
  std::vector<uint32_t> h_nearby_prim;
  std::vector<float> h_nearby_t;
  std::vector<int> h_nearby_back;
  std::vector<float> h_vol_w;
  std::vector<Ray> h_ray;
  std::vector<glm::vec3> h_light, h_tp;
  std::vector<int> h_px, h_py, h_depth, h_never, h_cam, h_psi;
  std::vector<RandomSampler> h_sampler;
  std::vector<RayTransfer> h_transfer;

  void Resize(size_t n) {
    const size_t nb = MAX_BOUNDARY_RECORD + 2;
    s_ray.resize(n); s_light.resize(n); s_tp.resize(n); s_px.resize(n); s_py.resize(n);
    s_depth.resize(n); s_never.resize(n); s_cam.resize(n); s_psi.resize(n);
    s_sampler.resize(n); s_transfer.resize(n);
    h_rec.resize(n); h_nearby_count.resize(n); h_nearby_prim.resize(n * nb); h_nearby_t.resize(n * nb);
    h_nearby_back.resize(n * nb); h_vol_w.resize(n * MAX_BOUNDARY_RECORD);
    h_ray.resize(n); h_light.resize(n); h_tp.resize(n); h_px.resize(n); h_py.resize(n);
    h_depth.resize(n); h_never.resize(n); h_cam.resize(n); h_psi.resize(n);
    h_sampler.resize(n); h_transfer.resize(n);
  }
};

struct RefContext {
  std::shared_ptr<SceneModule> module;
  Scene scene{};
  RenderSetting setting;
  int width = 0, height = 0;
  std::vector<uint32_t> instance_old_index;
  Queues q;
  size_t capacity = 0;
  double last_render_seconds = 0.0;
};

// Runs `body` once per emulated CUDA thread of a 1-D launch of `count` threads
// in blocks of `block`, spreading whole blocks over `n_threads` host threads.
template <typename F>
void Launch(uint32_t count, uint32_t block, int n_threads, const F& body) {
  if (count == 0) return;
  const uint32_t n_blocks = (count + block - 1) / block;
  std::atomic<uint32_t> next_block(0);
  auto worker = [&]() {
    blockDim = dim3(block, 1, 1);
    gridDim = dim3(n_blocks, 1, 1);
    for (;;) {
      const uint32_t b = next_block.fetch_add(1);
      if (b >= n_blocks) break;
      blockIdx = make_uint3(b, 0, 0);
      for (uint32_t t = 0; t < block; ++t) {
        threadIdx = make_uint3(t, 0, 0);
        body();
      }
    }
  };
  if (n_threads <= 1 || n_blocks == 1) {
    worker();
    return;
  }
  std::vector<std::thread> pool;
  const int n = std::min<int>(n_threads, (int)n_blocks);
  for (int i = 0; i < n; ++i) pool.emplace_back(worker);
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

// Settings block passed from Python; mirrors the fields of the reference's
// RenderSetting (src/SceneDefines.h:17-40) that the stage kernels read.
struct YmrefSettings {
  int spp;
  int ray_depth;
  int sampler_type;
  int enable_shape_light;
  int enable_distant_light;
  int enable_volume_scattering;
  int enable_env_light;
  int enable_russian_roulette;
  int enable_indirect_clamp;
  float indirect_limit;
};

size_t ymref_halton_table_size() {
  size_t total = 0;
  for (uint32_t i = 0; i < prime_count; ++i) total += primes[i];
  return total;
}

void* ymref_scene_load(const char* path, const uint32_t* halton_perm, size_t perm_len, int width, int height) {
  if (perm_len != ymref_halton_table_size() || width <= 0 || height <= 0) return nullptr;
  auto ctx = new RefContext();
  ctx->module = std::make_shared<SceneModule>();
  SceneParser parser;
  if (!parser.parsing_scene(path, ctx->module)) {
    delete ctx;
    return nullptr;
  }
  GuiModule::PrepareScene(*ctx->module, halton_perm, perm_len, width, height, &ctx->instance_old_index);
  ctx->scene = GuiModule::HostScene(*ctx->module);
  ctx->scene.render_setting = &ctx->setting;
  ctx->width = width;
  ctx->height = height;
  return ctx;
}

void ymref_scene_free(void* handle) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& grids = ymrt_oracle_grids();
  for (size_t i = grids.size(); i-- > 0;)
    if (grids[i].node >= ctx->scene.textures && grids[i].node < ctx->scene.textures + ctx->scene.texture_count)
      grids.erase(grids.begin() + i);
  delete ctx;
}

void ymref_set_settings(void* handle, const YmrefSettings* s) {
  auto ctx = static_cast<RefContext*>(handle);
  RenderSetting& r = ctx->setting;
  r.ssp = s->spp;
  r.ray_depth = s->ray_depth;
  r.sampler_type = s->sampler_type;
  r.enable_shape_light = s->enable_shape_light;
  r.enable_distant_light = s->enable_distant_light != 0;
  r.enable_volume_scattering = s->enable_volume_scattering != 0;
  r.enable_env_light = s->enable_env_light != 0;
  r.enable_russian_roulette = s->enable_russian_roulette != 0;
  r.enable_indirect_clamp = s->enable_indirect_clamp != 0;
  r.indirect_limit = s->indirect_limit;
}

// Scene facts after the reference's preparation, for comparing host-side scene
// preparation (instance order, triangle order, light table) with ymrt_b200.
int ymref_scene_counts(void* handle, uint32_t* out /* [instances, geometries, lights, transforms, materials] */) {
  auto ctx = static_cast<RefContext*>(handle);
  out[0] = ctx->scene.primitive_instance_count;
  out[1] = ctx->scene.geometry_count;
  out[2] = ctx->scene.shape_light_count;
  out[3] = ctx->scene.transform_count;
  out[4] = ctx->scene.material_count;
  return 0;
}

// Per instance (reference order): geometry, transform, material, volume,
// boundary flag, and the instance's index in file order.
int ymref_instances(void* handle, uint32_t* out /* 6 per instance */) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& inst = GuiModule::Instances(*ctx->module);
  for (size_t i = 0; i < inst.size(); ++i) {
    out[6 * i + 0] = inst[i].geometry_idx;
    out[6 * i + 1] = inst[i].transform_idx;
    out[6 * i + 2] = inst[i].material_idx;
    out[6 * i + 3] = (uint32_t)inst[i].inner_volume_idx;
    out[6 * i + 4] = (uint32_t)inst[i].treat_as_boundary;
    out[6 * i + 5] = ctx->instance_old_index[i];
  }
  return 0;
}

// Triangle count of a mesh geometry (or -1).
int64_t ymref_geometry_triangle_count(void* handle, uint32_t g) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& geo = GuiModule::Geometries(*ctx->module);
  if (g >= geo.size() || geo[g].geometry_type != TRIANGLE_MESH) return -1;
  return geo[g].triangle_mesh.triangle_count;
}

// The geometry's triangles after the reference's bottom-level BVH build
// (src/BottomBVH.cpp:155-161 reorders them): three corner indices each.
int ymref_geometry_triangles(void* handle, uint32_t g, uint32_t* out) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& geo = GuiModule::Geometries(*ctx->module);
  if (g >= geo.size() || geo[g].geometry_type != TRIANGLE_MESH) return -1;
  const Triangle* tris = geo[g].triangle_mesh.GetTrianglesHost();
  for (int64_t i = 0; i < geo[g].triangle_mesh.triangle_count; ++i) {
    out[3 * i + 0] = tris[i].id0;
    out[3 * i + 1] = tris[i].id1;
    out[3 * i + 2] = tris[i].id2;
  }
  return 0;
}

// Geometry type (GEOMETRY_TYPE: 0 triangle mesh, 1 sphere) and, for a
// sphere, its radius; -1 for an index out of range.
int ymref_geometry_kind(void* handle, uint32_t g, float* radius) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& geo = GuiModule::Geometries(*ctx->module);
  if (g >= geo.size()) return -1;
  *radius = geo[g].geometry_type == SPHERE ? geo[g].sphere.radius : 0.0f;
  return (int)geo[g].geometry_type;
}

// Per corner of a mesh geometry (3 per triangle, corner-index order):
// position, normal and texcoord (0, 0 when the mesh has none), 8 floats.
int ymref_mesh_corners(void* handle, uint32_t g, float* out) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& geo = GuiModule::Geometries(*ctx->module);
  if (g >= geo.size() || geo[g].geometry_type != TRIANGLE_MESH) return -1;
  const TriangleMesh& m = geo[g].triangle_mesh;
  const uint32_t* pi = m.GetPositionIndicesHost();
  const glm::vec3* p = m.GetPositionsHost();
  const uint32_t* ni = m.GetNormalIndicesHost();
  const glm::vec3* n = m.GetNormalsHost();
  const bool has_uv = m.texcoord_idx_offset != -1 && m.texcoord_offset != -1;
  const uint32_t* ti = has_uv ? m.GetTexcoordIndicesHost() : nullptr;
  const glm::vec2* t = has_uv ? m.GetTexcoordsHost() : nullptr;
  for (int64_t c = 0; c < 3 * m.triangle_count; ++c) {
    float* o = out + 8 * c;
    const glm::vec3 q = p[pi[c]], r = n[ni[c]];
    o[0] = q.x; o[1] = q.y; o[2] = q.z;
    o[3] = r.x; o[4] = r.y; o[5] = r.z;
    o[6] = has_uv ? t[ti[c]].x : 0.0f;
    o[7] = has_uv ? t[ti[c]].y : 0.0f;
  }
  return 0;
}

// Shape lights (instance, triangle, power, area) and the power CDF table.
int ymref_lights(void* handle, uint32_t* ids /* 2 per light */, float* power_area /* 2 per light */,
                 float* table) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& lights = GuiModule::Lights(*ctx->module);
  auto& tab = GuiModule::LightTable(*ctx->module);
  for (size_t i = 0; i < lights.size(); ++i) {
    ids[2 * i] = lights[i].instance_idx;
    ids[2 * i + 1] = lights[i].triangle_idx;
    power_area[2 * i] = lights[i].power;
    power_area[2 * i + 1] = lights[i].area;
    table[i] = tab[i];
  }
  return 0;
}

// Object-to-world and world-to-object matrices, 16 floats each, column major.
int ymref_transforms(void* handle, float* fwd, float* inv) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& t = GuiModule::Transforms(*ctx->module);
  auto& it = GuiModule::InvTransforms(*ctx->module);
  std::memcpy(fwd, t.data(), t.size() * sizeof(glm::mat4));
  std::memcpy(inv, it.data(), it.size() * sizeof(glm::mat4));
  return 0;
}

// Scene records as the reference's scene module holds them. what: 0 materials
// (raw Material words), 1 volumes (raw Volume words), 2 distant lights (raw
// DistantLight words), 3 textures (20 words per node, the layout of
// ymrt_texture_desc: type, black/white inputs, constant value, constant rgb,
// frequency, lacunarity, gain, layer count, amplitude, offset, variation,
// radius, flags (1 normalized, 2/4/8 marble x/y/z), and the wave's second
// frequency, lacunarity, gain, layer count). Returns the number of 32-bit
// words (written when out has room).
int ymref_scene_records(void* handle, int what, uint32_t* out, int cap) {
  auto ctx = static_cast<RefContext*>(handle);
  std::vector<uint32_t> w;
  auto raw = [&](const void* p, size_t bytes) {
    const size_t n = bytes / 4;
    const size_t at = w.size();
    w.resize(at + n);
    std::memcpy(w.data() + at, p, n * 4);
  };
  auto f = [](float v) { uint32_t u; std::memcpy(&u, &v, 4); return u; };
  switch (what) {
    case 0: for (auto& m : GuiModule::Materials(*ctx->module)) raw(&m, sizeof(m)); break;
    case 1: for (auto& v : GuiModule::Volumes(*ctx->module)) raw(&v, sizeof(v)); break;
    case 2: for (auto& d : GuiModule::DistantLights(*ctx->module)) raw(&d, sizeof(d)); break;
    case 3:
      for (auto& t : GuiModule::Textures(*ctx->module)) {
        uint32_t r[20] = {t.texture_type, EMPTY_UINT32, EMPTY_UINT32};
        if (t.GetChildCount() == 2) {
          r[1] = t.GetChildTextureIndex(0);
          r[2] = t.GetChildTextureIndex(1);
        }
        auto fbm = [&](float freq, float lac, float gain, int layers) {
          r[7] = f(freq); r[8] = f(lac); r[9] = f(gain); r[10] = (uint32_t)layers;
        };
        switch (t.texture_type) {
          case IMAGE_TEXTURE: {
            const auto& im = t.image_texture;
            r[3] = (uint32_t)im.width; r[4] = (uint32_t)im.height; r[5] = (uint32_t)im.channel_count;
            r[6] = (uint32_t)im.warp_mode;
            r[7] = f(im.scale_u); r[8] = f(im.scale_v); r[9] = f(im.offset_u); r[10] = f(im.offset_v);
            r[15] = (uint32_t)im.color_space;
            break;
          }
          case CONSTANT_TEXTURE_FLOAT: r[3] = f(t.constant_texture_float.value); break;
          case CONSTANT_TEXTURE_RGB:
            r[4] = f(t.constant_texture_rgb.color.x); r[5] = f(t.constant_texture_rgb.color.y);
            r[6] = f(t.constant_texture_rgb.color.z);
            break;
          case SOLID_TEXTURE_CHECKERBOARD: r[7] = f(t.checker_board_texture.frequency); break;
          case SOLID_TEXTURE_NOISE:
            r[7] = f(t.noise_texture.frequency);
            r[15] = t.noise_texture.normalized ? 1u : 0u;
            break;
          case SOLID_TEXTURE_FBM: {
            const auto& n = t.noise_texture_fbm;
            fbm(n.frequency, n.lacunarity, n.gain, n.layer_count);
            r[11] = f(n.amplitude); r[12] = f(n.offset);
            break;
          }
          case SOLID_TEXTURE_TURBULENCE: {
            const auto& n = t.noise_texture_turbulence;
            fbm(n.frequency, n.lacunarity, n.gain, n.layer_count);
            r[11] = f(n.amplitude); r[12] = f(n.offset);
            break;
          }
          case SOLID_TEXTURE_MARBLE: {
            const auto& n = t.noise_texture_marble;
            fbm(n.frequency, n.lacunarity, n.gain, n.layer_count);
            r[13] = f(n.variation);
            r[15] = (n.x_turb ? 2u : 0u) | (n.y_turb ? 4u : 0u) | (n.z_turb ? 8u : 0u);
            break;
          }
          case SOLID_TEXTURE_WOOD:
            r[7] = f(t.noise_texture_wood.frequency); r[13] = f(t.noise_texture_wood.variation);
            break;
          case SOLID_TEXTURE_POLKA_DOT:
            r[7] = f(t.noise_texture_polka_dot.frequency); r[14] = f(t.noise_texture_polka_dot.radius);
            break;
          case SOLID_TEXTURE_WAVE: {
            const auto& n = t.noise_texture_wave;
            fbm(n.freq_0, n.lacunarity_0, n.gain_0, n.layer_count_0);
            r[16] = f(n.freq_1); r[17] = f(n.lacunarity_1); r[18] = f(n.gain_1); r[19] = (uint32_t)n.layer_count_1;
            break;
          }
          default: break;
        }
        w.insert(w.end(), r, r + 20);
      }
      break;
    default: return -1;
  }
  if (out && cap >= (int)w.size()) std::memcpy(out, w.data(), w.size() * 4);
  return (int)w.size();
}

// Pixels of image node `tex` as the reference holds them (32x32 tiles,
// src/FileIO.cpp:126-171), reassembled into rows (bottom row first, as
// loaded): width * height * channels floats. Returns the count, or -1.
long long ymref_image_pixels(void* handle, uint32_t tex, float* out, long long cap) {
  auto ctx = static_cast<RefContext*>(handle);
  const auto& textures = GuiModule::Textures(*ctx->module);
  if (tex >= textures.size() || textures[tex].texture_type != IMAGE_TEXTURE) return -1;
  const ImageTexture& im = textures[tex].image_texture;
  const long long n = (long long)im.width * im.height * im.channel_count;
  if (!out || cap < n) return n;
  const auto& tiles = GuiModule::ImageTiles(*ctx->module);
  const int tiles_x = (im.width + TEX_TILE_RES_X - 1) / TEX_TILE_RES_X;
  for (int y = 0; y < im.height; ++y)
    for (int x = 0; x < im.width; ++x) {
      const ImageTile& tile = tiles[im.tile_offset + (y / TEX_TILE_RES_Y) * tiles_x + x / TEX_TILE_RES_X];
      const float* d = static_cast<const float*>(tile.host_data) +
                       ((y % TEX_TILE_RES_Y) * TEX_TILE_RES_X + x % TEX_TILE_RES_X) * im.channel_count;
      for (int c = 0; c < im.channel_count; ++c) out[((long long)y * im.width + x) * im.channel_count + c] = d[c];
    }
  return n;
}

// SavePngImage (src/FileIO.cpp:167-194) of a width x height RGBA image (rows
// bottom first, as the renderer holds them). Returns 1 on success, 0 when the
// reference's function reports failure.
int ymref_save_png(const char* path, const float* rgba, int width, int height) {
  std::vector<glm::vec4> image(width > 0 && height > 0 ? (size_t)width * height : 0);
  for (size_t k = 0; k < image.size(); ++k)
    image[k] = glm::vec4(rgba[4 * k], rgba[4 * k + 1], rgba[4 * k + 2], rgba[4 * k + 3]);
  return SavePngImage(path ? std::string(path) : std::string(), image, width, height) ? 1 : 0;
}

// TextureEval (src/TextureEval.cuh:419-481) of texture node `tex` at n
// points of 5 floats (texture coordinates s, t, object-space x, y, z; the
// world position is set to the object position, which no procedural node
// reads): rgb out. Returns 0, or -1 for an unknown node.
int ymref_texture_eval(void* handle, uint32_t tex, int n, const float* coords, float* rgb) {
  auto ctx = static_cast<RefContext*>(handle);
  const auto& textures = GuiModule::Textures(*ctx->module);
  if (tex >= textures.size()) return -1;
  ImageTileCache cache;
  cache.image_tiles_host = GuiModule::ImageTiles(*ctx->module).data();
  for (int i = 0; i < n; ++i) {
    const float* c = coords + 5 * (size_t)i;
    const glm::vec3 p(c[2], c[3], c[4]);
    const TextureCoordinate tc(glm::vec2(c[0], c[1]), p, p);
    const glm::vec3 v = TextureEval(textures[tex], textures.data(), cache, tc);
    rgb[3 * i] = v.x;
    rgb[3 * i + 1] = v.y;
    rgb[3 * i + 2] = v.z;
  }
  return 0;
}

// Depth (root = 1) of the reference's binary BVHs: out[g] for mesh g, then
// out[geometry_count] for the top-level tree. The reference's traversals keep
// at most depth + 1 entries on a 32-entry stack (src/ShadingUtilities.cuh:147).
}  // extern "C"
namespace {
template <typename Node>
uint32_t binary_depth(const Node* nodes, size_t count) {
  if (!nodes || count == 0) return 0;
  std::vector<std::pair<uint32_t, uint32_t>> todo{{0u, 1u}};
  uint32_t best = 0;
  while (!todo.empty()) {
    auto [n, d] = todo.back();
    todo.pop_back();
    best = std::max(best, d);
    if (n >= count) return 0xFFFFFFFFu;
    if (nodes[n].internal.left != EMPTY_UINT32) continue;  // leaf
    todo.push_back({n + 1, d + 1});
    todo.push_back({nodes[n].internal.right, d + 1});
  }
  return best;
}
}  // namespace
extern "C" {

int ymref_bvh_depths(void* handle, uint32_t* out) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& geo = GuiModule::Geometries(*ctx->module);
  for (size_t g = 0; g < geo.size(); ++g) {
    out[g] = 0;
    if (geo[g].geometry_type != TRIANGLE_MESH) continue;
    const auto& tm = geo[g].triangle_mesh;
    const size_t n = (size_t)std::max<int64_t>(2 * tm.triangle_count - 1, 1);
    out[g] = binary_depth(tm.GetNodesHost(), n);
  }
  auto& top = GuiModule::TopNodes(*ctx->module);
  out[geo.size()] = binary_depth(top.data(), top.size());
  return (int)geo.size() + 1;
}

// The Sobol generator matrices the reference links (src/LowDiscrepancy.cpp:179,
// 4096 dimensions x 32 columns); returns the word count.
size_t ymref_sobol_matrices(uint32_t* out, size_t cap) {
  const size_t n = (size_t)4096 * 32;
  if (out && cap >= n) std::memcpy(out, sobol_matrices32, n * sizeof(uint32_t));
  return n;
}

// The rendering camera after preparation, as raw bytes of the reference's
// Camera struct (176 bytes on x86-64).
int ymref_camera_bytes(void* handle, uint8_t* out, int out_len) {
  auto ctx = static_cast<RefContext*>(handle);
  if (out_len < (int)sizeof(Camera)) return -(int)sizeof(Camera);
  std::memcpy(out, &GuiModule::Cameras(*ctx->module)[RENDERING_CAMERA_INDEX], sizeof(Camera));
  return (int)sizeof(Camera);
}

// Closest-hit queries through the reference's TraceRay
// (src/ShadingUtilities.cuh:310). Rays are built with the reference's Ray
// constructor (which normalises the direction). Outputs per ray: instance,
// triangle, t, barycentrics (3), back-face flag, nearby-hit count.
int ymref_trace(void* handle, int n, const float* origin, const float* dir, const uint32_t* last_hit /* 2 per ray or null */,
                uint32_t* inst, uint32_t* tri, float* t, float* bary, int* back, int* nearby) {
  auto ctx = static_cast<RefContext*>(handle);
  for (int i = 0; i < n; ++i) {
    Ray ray(glm::vec3(origin[3 * i], origin[3 * i + 1], origin[3 * i + 2]),
            glm::vec3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]),
            last_hit ? last_hit[2 * i] : EMPTY_UINT32, last_hit ? last_hit[2 * i + 1] : EMPTY_UINT32);
    HitRecord rec;
    int nearby_count = 0;
    NearbyHit nearby_hits[MAX_BOUNDARY_RECORD + 2];
    const bool hit = TraceRay(ctx->scene, ray, &rec, &nearby_count, nearby_hits);
    inst[i] = hit ? rec.hit_instance_idx : EMPTY_UINT32;
    tri[i] = hit ? rec.hit_triangle_idx : EMPTY_UINT32;
    t[i] = hit ? rec.hit_t : TMAX;
    bary[3 * i] = rec.hit_barycentric.x;
    bary[3 * i + 1] = rec.hit_barycentric.y;
    bary[3 * i + 2] = rec.hit_barycentric.z;
    back[i] = rec.hit_back;
    nearby[i] = nearby_count;
  }
  return 0;
}

// The shading frame the reference's shade stage builds at a hit
// (src/Shading.cu:2128-2188: FetchShadingData, the pixel's texture-coordinate
// footprint, MaterialBSDF::InitShadingSpace with normal / bump maps). Per
// hit: instance, triangle, barycentrics (3), back flag and ray direction (3)
// in; out 22 floats: normal, tangent, bitangent (9), du/dx, dv/dx, du/dy,
// dv/dy (4), uv (2), object-space position (3), shading dp/du (3) and the
// hit's material index as a float (1).
int ymref_shading_frame(void* handle, int n, const uint32_t* inst, const uint32_t* tri, const float* bary,
                        const int* back, const float* dir, float* out) {
  auto ctx = static_cast<RefContext*>(handle);
  const Scene& scene = ctx->scene;
  ImageTileCache cache;
  cache.image_tiles_host = GuiModule::ImageTiles(*ctx->module).data();
  for (int i = 0; i < n; ++i) {
    float* o = out + 22 * (size_t)i;
    for (int k = 0; k < 22; ++k) o[k] = 0.0f;
    HitRecord rec;
    rec.hit_instance_idx = inst[i];
    rec.hit_triangle_idx = tri[i];
    rec.hit_barycentric = glm::vec3(bary[3 * i], bary[3 * i + 1], bary[3 * i + 2]);
    rec.hit_back = back[i];
    Ray ray(glm::vec3(0.0f), glm::vec3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]));
    glm::vec3 p(0.0f), perr(0.0f), pobj(0.0f), ns(0.0f), ng(0.0f), dpdu(0.0f), dpdv(0.0f);
    glm::vec2 uv(0.0f);
    FetchShadingData(scene, rec, &p, &perr, &pobj, &ns, &ng, &uv, &dpdu, &dpdv);
    const glm::vec4 d = scene.camera->TextureCoordinatesDifferential(ray, p, ns, ng, dpdu, dpdv, ctx->width,
                                                                     ctx->height, 0.25f, 0.25f);
    const auto& prim = scene.primitive_instances[rec.hit_instance_idx];
    const auto& material = scene.materials[prim.material_idx];
    MaterialBSDF bsdf;
    const TextureCoordinate tc(uv, p, pobj, d);
    bsdf.InitShadingSpace(material, rec.hit_back, ray, ng, ns, dpdu, dpdv, scene.transforms[prim.transform_idx],
                          scene.i_transforms[prim.transform_idx], scene.textures, cache, tc);
    const float v[22] = {bsdf.normal.x, bsdf.normal.y, bsdf.normal.z, bsdf.tangent.x, bsdf.tangent.y,
                         bsdf.tangent.z, bsdf.bitangent.x, bsdf.bitangent.y, bsdf.bitangent.z, d.x, d.y, d.z, d.w,
                         uv.x, uv.y, pobj.x, pobj.y, pobj.z, dpdu.x, dpdu.y, dpdu.z, (float)prim.material_idx};
    for (int k = 0; k < 22; ++k) o[k] = v[k];
  }
  return 0;
}

// Any-hit occlusion through the reference's BVHTraverseShadow
// (src/ShadingUtilities.cuh:563) with ray.t = tmax.
int ymref_occluded(void* handle, int n, const float* origin, const float* dir, const float* tmax, int* occluded) {
  auto ctx = static_cast<RefContext*>(handle);
  for (int i = 0; i < n; ++i) {
    Ray ray(glm::vec3(origin[3 * i], origin[3 * i + 1], origin[3 * i + 2]),
            glm::vec3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]));
    ray.t = tmax[i];
    HitRecord rec;
    occluded[i] = BVHTraverseShadow(ctx->scene, ray, &rec) ? 1 : 0;
  }
  return 0;
}

// The boundary crossings of one shadow ray as the reference's TraceTr
// follows them (src/VolumeEval.cuh:420-468: TraceVolume, the nested-media
// update BoundaryTransitionBunch and OffsetRayOrigin), without the
// transmittance estimates, which do not move the ray. The ray starts at
// origin / dir (already offset) leaving last_inst / last_tri, with `tmax` of
// its length left and the nested-media stack `transfer` (the reference's
// RayTransfer as 32-bit words: max-priority index, record count, then 6
// records of prim, ior bits, priority, volume). At most max_steps crossings;
// per crossing 8 words: instance, triangle, t bits, back flag, nearby count,
// stack record count after it, and the distance traced so far (bits).
// Returns the number of crossings (the walk ends when the ray passes tmax or
// hits nothing). Float build only.
#ifndef YMREF_FP64
int ymref_boundary_walk(void* handle, const float* origin, const float* dir, float tmax, uint32_t last_inst,
                        uint32_t last_tri, const uint32_t* transfer, int max_steps, uint32_t* out) {
  auto ctx = static_cast<RefContext*>(handle);
  const Scene& scene = ctx->scene;
  RayTransfer rt;
  rt.max_priority_record_index = (int)transfer[0];
  rt.record_count = (int)transfer[1];
  for (int r = 0; r < rt.record_count && r < MAX_BOUNDARY_RECORD; ++r) {
    const uint32_t* w = transfer + 2 + 4 * r;
    float ior;
    std::memcpy(&ior, w + 1, 4);
    rt.boundary_records[r] = BoundaryRecord(w[0], ior, w[2], (int)w[3]);
  }
  Ray tr_ray(glm::vec3(origin[0], origin[1], origin[2]), glm::vec3(dir[0], dir[1], dir[2]), last_inst, last_tri);
  float traced = TMIN;
  int n = 0;
  while (traced < tmax && n < max_steps) {
    HitRecord rec;
    int nearby_count = 0;
    NearbyHit nearby[MAX_BOUNDARY_RECORD + 2];
    if (!TraceVolume(scene, tr_ray, &rec, &nearby_count, nearby)) break;
    traced += rec.hit_t;
    glm::vec3 p(0.0f), perr(0.0f), ng(0.0f);
    FetchGeometryNormal(scene, rec, &p, &perr, &ng);
    BoundaryTransitionBunch(rt, scene.primitive_instances, scene.materials, nearby, nearby_count);
    tr_ray = Ray(OffsetRayOrigin(p, perr, tr_ray.direction, ng), tr_ray.direction, rec.hit_instance_idx,
                 rec.hit_triangle_idx);
    uint32_t* o = out + 8 * (size_t)n;
    o[0] = rec.hit_instance_idx;
    o[1] = rec.hit_triangle_idx;
    std::memcpy(o + 2, &rec.hit_t, 4);
    o[3] = rec.hit_back ? 1u : 0u;
    o[4] = (uint32_t)nearby_count;
    o[5] = (uint32_t)rt.record_count;
    std::memcpy(o + 6, &traced, 4);
    o[7] = 0;
    ++n;
  }
  return n;
}
#endif

// Replaces the density node `tex` of the scene with a 3-D grid of nx*ny*nz
// values (x fastest) over the object-space box [-0.5, 0.5]^3 (this project's
// grid node; the reference has none): media read it trilinearly with clamped
// edges and track against its maximum (oracle/build_ref.py, _MEDIA_HOOKS).
// Calling it again for the same node replaces the grid.
int ymref_set_density_grid(void* handle, uint32_t tex, int nx, int ny, int nz, const float* values) {
  auto ctx = static_cast<RefContext*>(handle);
  if (tex >= ctx->scene.texture_count || nx < 1 || ny < 1 || nz < 1) return -1;
  const Texture* node = &ctx->scene.textures[tex];
  auto& grids = ymrt_oracle_grids();
  for (size_t i = 0; i < grids.size(); ++i)
    if (grids[i].node == node) {
      grids.erase(grids.begin() + i);
      break;
    }
  YmrtOracleGrid g;
  g.node = node;
  g.n[0] = nx;
  g.n[1] = ny;
  g.n[2] = nz;
  g.v.assign(values, values + (size_t)nx * ny * nz);
  g.vmax = 0.0f;
  for (const auto v : g.v) g.vmax = std::max(g.vmax, v);
  grids.push_back(std::move(g));
  return 0;
}

// A transform edit as the reference's editor applies it: transforms
// first .. first+count-1 replaced (16 floats each, column major, object to
// world; the inverse by glm::inverse; scales, 3 per transform, the
// TransformState scale that sizes sphere lights, when not null), then
// GuiModule::UpdateScene's rebuild (src/core/GuiModule.cpp:123-170).
int ymref_set_transforms(void* handle, uint32_t first, uint32_t count, const float* mats, const float* scales) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& T = GuiModule::Transforms(*ctx->module);
  auto& I = GuiModule::InvTransforms(*ctx->module);
  auto& S = GuiModule::TransformStates(*ctx->module);
  if (first > T.size() || count > T.size() - first) return -1;
  for (uint32_t k = 0; k < count; ++k) {
    glm::mat4 m;
    std::memcpy(&m, mats + 16 * (size_t)k, sizeof(m));
    T[first + k] = m;
    I[first + k] = glm::inverse(m);
    if (scales) S[first + k].scale_xyz = glm::vec3(scales[3 * k], scales[3 * k + 1], scales[3 * k + 2]);
  }
  GuiModule::RebuildAfterTransformEdit(*ctx->module, &ctx->instance_old_index);
  ctx->scene = GuiModule::HostScene(*ctx->module);
  ctx->scene.render_setting = &ctx->setting;  // as ymref_scene_load sets it
  return 0;
}

// Material parameters as ymrt_scene_set_material_params sets them (this
// project's editing entry; the reference edits materials through its GUI):
// for each default material in [first, first+count), 4 values -- diffuse
// albedo r, g, b and roughness, written to both alphas; other materials are
// left as they are. Returns 0, or -1 when the range is out of bounds.
int ymref_set_material_params(void* handle, uint32_t first, uint32_t count, const float* params) {
  auto ctx = static_cast<RefContext*>(handle);
  auto& M = GuiModule::Materials(*ctx->module);
  if (first > M.size() || count > M.size() - first) return -1;
  for (uint32_t k = 0; k < count; ++k) {
    Material& m = M[first + k];
    if (m.material_type != DEFAULT_MTL) continue;
    const float* q = params + 4 * (size_t)k;
    m.default_mtl.diffuse_albedo = glm::vec3(q[0], q[1], q[2]);
    m.default_mtl.alpha_x = q[3];
    m.default_mtl.alpha_y = q[3];
  }
  return 0;  // edited in place: the scene's material array is the module's
}

// The materials' (diffuse albedo r, g, b, alpha_x, lambertian) as 5 floats
// each, zeros for other material types; lambertian is 1 for a default
// material whose only lobe is the diffuse one (no specular, metal,
// transmission or coat weight, no texture on those or on the albedo).
int ymref_get_material_params(void* handle, uint32_t first, uint32_t count, float* out) {
  auto ctx = static_cast<RefContext*>(handle);
  const auto& M = GuiModule::Materials(*ctx->module);
  if (first > M.size() || count > M.size() - first) return -1;
  for (uint32_t k = 0; k < count; ++k) {
    const Material& m = M[first + k];
    float* q = out + 5 * (size_t)k;
    for (int c = 0; c < 5; ++c) q[c] = 0.0f;
    if (m.material_type != DEFAULT_MTL) continue;
    const auto& d = m.default_mtl;
    q[0] = d.diffuse_albedo.x;
    q[1] = d.diffuse_albedo.y;
    q[2] = d.diffuse_albedo.z;
    q[3] = d.alpha_x;
    const bool untextured = d.diffuse_albedo_tex == EMPTY_UINT32 && d.specular_weight_tex == EMPTY_UINT32 &&
                            d.metalness_tex == EMPTY_UINT32 && d.transmission_weight_tex == EMPTY_UINT32 &&
                            d.coat_weight_tex == EMPTY_UINT32;
    q[4] = (untextured && d.specular_weight == 0.0f && d.metalness == 0.0f && d.transmission_weight == 0.0f &&
            d.coat_weight == 0.0f) ? 1.0f : 0.0f;
  }
  return 0;
}

// A medium's density as the build-time copy of VolumeEval.cuh reads it
// (the grid node when one is attached to `tex`, else the reference's
// TextureEval), at n object-space points (3 floats each).
int ymref_density(void* handle, uint32_t tex, int n, const float* points, float* out) {
  auto ctx = static_cast<RefContext*>(handle);
  if (tex >= ctx->scene.texture_count) return -1;
  ImageTileCache cache;
  cache.image_tiles_host = GuiModule::ImageTiles(*ctx->module).data();
  const Texture& t = ctx->scene.textures[tex];
  for (int i = 0; i < n; ++i) {
    const glm::vec3 p(points[3 * i], points[3 * i + 1], points[3 * i + 2]);
    const TextureCoordinate tc(glm::vec2(0.0f), p, p);
    out[i] = ymrt_oracle_density(t, ctx->scene.textures, cache, tc).x;
  }
  return 0;
}

// Tracking loops (delta and ratio tracking) that reached the reference's
// MAX_FREE_PATH_LENGTH bound since the last reset, over every render.
unsigned long long ymref_tracking_caps(int reset) {
  return reset ? ymrt_oracle_tracking_caps().exchange(0) : ymrt_oracle_tracking_caps().load();
}

#if defined(YMRT_ORACLE_RECORDING) && !defined(YMREF_FP64)
// Path-vertex recording (parity build only): during the renders that follow,
// the trace stage writes the vertex of every path of a watched pixel (one bit
// per pixel in watch_bits, which must stay valid) into out, `capacity`
// records of 24 words (YmrtOracleVertex). watch_bits == nullptr stops it.
// Resets the count.
void ymref_set_recorder(void* handle, const uint32_t* watch_bits, void* out, int capacity) {
  auto ctx = static_cast<RefContext*>(handle);
  YmrtOracleRecorder& q = ymrt_oracle_recorder();
  q.out = nullptr;
  q.watch = watch_bits;
  q.n_pixels = watch_bits ? (uint32_t)(ctx->width * ctx->height) : 0u;
  q.capacity = watch_bits ? (uint32_t)std::max(capacity, 0) : 0u;
  q.count.store(0);
  q.out = watch_bits ? static_cast<YmrtOracleVertex*>(out) : nullptr;
}
// Vertices recorded since the recorder was set (those past its capacity are
// counted, not written).
uint32_t ymref_recorded(void) { return ymrt_oracle_recorder().count.load(); }
#endif

#if defined(YMRT_ORACLE_EVENTS)
// Radiance-event recording (parity builds, float and double): during the
// renders that follow, every radiance term the stages add and every surface
// scattering event of a watched pixel (one bit per pixel in watch_bits, which
// must stay valid; null: every pixel) is written to out (YmrtOracleEvent, 48
// bytes), up to `capacity`; out == nullptr stops it. Resets the count.
void ymref_set_events(void* handle, void* out, int capacity, const uint32_t* watch_bits) {
  auto ctx = static_cast<RefContext*>(handle);
  YmrtOracleEvents& q = ymrt_oracle_events();
  q.out = nullptr;
  q.capacity = out ? (uint32_t)std::max(capacity, 0) : 0u;
  q.watch = watch_bits;
  q.n_pixels = (uint32_t)(ctx->width * ctx->height);
  q.count.store(0);
  q.out = static_cast<YmrtOracleEvent*>(out);
}
// Events since the recorder was set (those past its capacity are counted, not
// written).
uint32_t ymref_events_recorded(void) { return ymrt_oracle_events().count.load(); }
#endif

// Halton sampler known-answer values: for each (px, py, sample) the global
// sample index (src/HaltonEnumerator.h:43 GetIndex), the pixel offset as the
// ray-generation stage computes it (src/Shading.cu:1698-1704) and the first
// n_dims scrambled dimensions starting at dimension 2
// (src/RandomSampler.cuh:430 Random1D).
int ymref_halton(void* handle, int n, const int* px, const int* py, const int* sample, int n_dims,
                 uint64_t* index, float* offset, float* dims) {
  auto ctx = static_cast<RefContext*>(handle);
  HaltonEnumerator he(ctx->width, ctx->height);
  for (int i = 0; i < n; ++i) {
    const uint64_t sample_index = he.GetIndex(px[i], py[i], sample[i]);
    index[i] = sample_index;
    RandomSampler sampler;
    sampler.InitHaltonSampler(sample_index, 2, ctx->scene.sampler_data.halton_permute_table);
    glm::vec2 pixel_offset = sampler.SamplePixelOffset();
    pixel_offset.x = he.ScaleX(pixel_offset.x) - float(px[i]);
    pixel_offset.y = he.ScaleY(pixel_offset.y) - float(py[i]);
    pixel_offset = glm::clamp(pixel_offset, glm::vec2(0.000001f), glm::vec2(0.999999f));
    offset[2 * i] = pixel_offset.x;
    offset[2 * i + 1] = pixel_offset.y;
    for (int d = 0; d < n_dims; ++d) dims[(size_t)i * n_dims + d] = sampler.Random1D();
  }
  return 0;
}

// One progressive frame of the path-tracing view over tiles
// [tile_begin, tile_end) (tile_end <= 0 means all tiles), accumulated into
// out_rgba (width*height*4 floats, zeroed here) exactly as the reference's
// noise image. Returns 0, or -1 on bad arguments.
int ymref_render_frame(void* handle, int frame_index, int tile_begin, int tile_end, int wave_capacity,
                       int n_threads, float* out_rgba) {
  auto ctx = static_cast<RefContext*>(handle);
  const RenderSetting& rs = ctx->setting;
  const uint32_t spp = (uint32_t)std::max(rs.ssp, 1);
  const uint32_t w = ctx->width, h = ctx->height;
  const uint32_t tiles_x = (w + TILE_X_RES - 1) / TILE_X_RES;
  const uint32_t tiles_y = (h + TILE_Y_RES - 1) / TILE_Y_RES;
  const uint32_t total_tiles = tiles_x * tiles_y;
  const uint32_t t_end = tile_end <= 0 ? total_tiles : std::min<uint32_t>(tile_end, total_tiles);
  const uint32_t rays_per_tile = TILE_PIXEL_COUNT * spp;
  if (frame_index < 1 || wave_capacity < (int)rays_per_tile || tile_begin < 0) return -1;
  const size_t cap = (size_t)wave_capacity;
  if (ctx->capacity < cap) {
    ctx->q.Resize(cap);
    ctx->capacity = cap;
  }
  Queues& q = ctx->q;
  std::memset(out_rgba, 0, sizeof(float) * 4 * w * h);
  glm::vec4* noise = reinterpret_cast<glm::vec4*>(out_rgba);
  HaltonEnumerator halton(w, h);
  RayCounter counter{0, 0, 0};
  RayCounter host_counter{0, 0, 0};
  const Scene* scene = &ctx->scene;
  uint32_t next_tile = (uint32_t)tile_begin;
  const auto t0 = std::chrono::steady_clock::now();

  while (host_counter.shading_ray_counter > 0 || next_tile < t_end) {
    const uint32_t tiles_this_batch =
        std::min<uint32_t>((uint32_t)((cap - host_counter.shading_ray_counter) / rays_per_tile), t_end - next_tile);
    const uint32_t gen_count = tiles_this_batch * rays_per_tile;
    counter.shading_ray_counter = host_counter.shading_ray_counter;
    Launch(gen_count, STAGE_RAY_GEN_BLOCK_SIZE, n_threads, [&]() {
      Ray_generation_path_tracing(frame_index, scene, &halton, &counter, next_tile, gen_count, spp, w, h, tiles_x,
                                  tiles_y, q.s_ray.data(), q.s_light.data(), q.s_tp.data(), q.s_px.data(),
                                  q.s_py.data(), q.s_depth.data(), q.s_never.data(), q.s_cam.data(),
                                  q.s_psi.data(), q.s_sampler.data(), q.s_transfer.data());
    });
    next_tile += tiles_this_batch;
    host_counter.shading_ray_counter += gen_count;

    counter = host_counter;
    const uint32_t trace_count = host_counter.shading_ray_counter;
    Launch(trace_count, STAGE_RAY_TRACE_BLOCK_SIZE, n_threads, [&]() {
      Ray_trace_path_tracing(frame_index, scene, &counter, trace_count, w, h, noise, q.s_ray.data(), q.s_light.data(),
                             q.s_tp.data(), q.s_px.data(), q.s_py.data(), q.s_depth.data(), q.s_never.data(),
                             q.s_cam.data(), q.s_psi.data(), q.s_sampler.data(), q.s_transfer.data(), q.h_rec.data(),
                             q.h_nearby_count.data(), q.h_nearby_prim.data(), q.h_nearby_t.data(),
                             q.h_nearby_back.data(), q.h_vol_w.data(), q.h_ray.data(), q.h_light.data(),
                             q.h_tp.data(), q.h_px.data(), q.h_py.data(), q.h_depth.data(), q.h_never.data(),
                             q.h_cam.data(), q.h_psi.data(), q.h_sampler.data(), q.h_transfer.data());
    });
    host_counter = counter;
    host_counter.shading_ray_counter = 0;

    counter = host_counter;
    const uint32_t shade_count = host_counter.hit_counter;
    Launch(shade_count, STAGE_RAY_SHADING_BLOCK_SIZE, n_threads, [&]() {
      Ray_shading_path_tracing(frame_index, scene, &counter, shade_count, w, h, noise, q.s_ray.data(),
                               q.s_light.data(), q.s_tp.data(), q.s_px.data(), q.s_py.data(), q.s_depth.data(),
                               q.s_never.data(), q.s_cam.data(), q.s_psi.data(), q.s_sampler.data(),
                               q.s_transfer.data(), q.h_rec.data(), q.h_nearby_count.data(), q.h_nearby_prim.data(),
                               q.h_nearby_t.data(), q.h_nearby_back.data(), q.h_vol_w.data(), q.h_ray.data(),
                               q.h_light.data(), q.h_tp.data(), q.h_px.data(), q.h_py.data(), q.h_depth.data(),
                               q.h_never.data(), q.h_cam.data(), q.h_psi.data(), q.h_sampler.data(),
                               q.h_transfer.data());
    });
    host_counter = counter;
    host_counter.hit_counter = 0;
    if (host_counter.shading_ray_counter > cap) return -2;  // queue overflow
  }
  ctx->last_render_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return 0;
}

// The editor view (src/Shading.cu:1276-1594) over all tiles with the
// stages' own queue protocol, the editor camera set to the rendering camera
// (as the editor sizes it to its viewport). Adds into beauty (width*height*4)
// and writes primitive_index (width*height) as the stages do; neither is
// cleared here. Returns 0, or -1 / -2 on bad arguments / queue overflow.
int ymref_render_editor_view(void* handle, int wave_capacity, int n_threads, float* beauty, uint32_t* primitive_index) {
  auto ctx = static_cast<RefContext*>(handle);
  const uint32_t w = ctx->width, h = ctx->height;
  const uint32_t tiles_x = (w + TILE_X_RES - 1) / TILE_X_RES;
  const uint32_t tiles_y = (h + TILE_Y_RES - 1) / TILE_Y_RES;
  const uint32_t total_tiles = tiles_x * tiles_y;
  if (wave_capacity < (int)TILE_PIXEL_COUNT) return -1;
  const size_t cap = (size_t)wave_capacity;
  if (ctx->capacity < cap) {
    ctx->q.Resize(cap);
    ctx->capacity = cap;
  }
  Camera* cams = GuiModule::Cameras(*ctx->module);
  std::memcpy(&cams[EDITOR_CAMERA_INDEX], &cams[RENDERING_CAMERA_INDEX], sizeof(Camera));
  Queues& q = ctx->q;
  glm::vec4* img = reinterpret_cast<glm::vec4*>(beauty);
  RayCounter counter{0, 0, 0}, host_counter{0, 0, 0};
  const Scene* scene = &ctx->scene;
  uint32_t next_tile = 0;
  while (host_counter.shading_ray_counter > 0 || next_tile < total_tiles) {
    const uint32_t tiles_this_batch = std::min<uint32_t>(
        (uint32_t)((cap - host_counter.shading_ray_counter) / TILE_PIXEL_COUNT), total_tiles - next_tile);
    const uint32_t gen_count = tiles_this_batch * TILE_PIXEL_COUNT;
    counter.shading_ray_counter = host_counter.shading_ray_counter;
    Launch(gen_count, STAGE_RAY_GEN_BLOCK_SIZE, n_threads, [&]() {
      Ray_generation_editor_view(1, scene, &counter, next_tile, gen_count, w, h, tiles_x, tiles_y, q.s_ray.data(),
                                 q.s_px.data(), q.s_py.data(), q.s_cam.data(), q.s_transfer.data());
    });
    next_tile += tiles_this_batch;
    host_counter.shading_ray_counter += gen_count;
    counter = host_counter;
    const uint32_t trace_count = host_counter.shading_ray_counter;
    Launch(trace_count, STAGE_RAY_TRACE_BLOCK_SIZE, n_threads, [&]() {
      Ray_trace_editor_view(1, scene, &counter, trace_count, w, h, img, primitive_index, q.s_ray.data(), q.s_px.data(),
                            q.s_py.data(), q.s_cam.data(), q.s_transfer.data(), q.h_rec.data(),
                            q.h_nearby_count.data(), q.h_nearby_prim.data(), q.h_nearby_t.data(),
                            q.h_nearby_back.data(), q.h_ray.data(), q.h_px.data(), q.h_py.data(), q.h_cam.data(),
                            q.h_transfer.data());
    });
    host_counter = counter;
    host_counter.shading_ray_counter = 0;
    counter = host_counter;
    const uint32_t shade_count = host_counter.hit_counter;
    Launch(shade_count, STAGE_RAY_SHADING_BLOCK_SIZE, n_threads, [&]() {
      Ray_shading_editor_view(1, scene, &counter, shade_count, w, h, img, primitive_index, q.s_ray.data(),
                              q.s_px.data(), q.s_py.data(), q.s_cam.data(), q.s_transfer.data(), q.h_rec.data(),
                              q.h_nearby_count.data(), q.h_nearby_prim.data(), q.h_nearby_t.data(),
                              q.h_nearby_back.data(), q.h_ray.data(), q.h_px.data(), q.h_py.data(), q.h_cam.data(),
                              q.h_transfer.data());
    });
    host_counter = counter;
    host_counter.hit_counter = 0;
    if (host_counter.shading_ray_counter > cap) return -2;
  }
  return 0;
}

// Gamma_correction_common and Draw_outline (src/Shading.cu:2396-2466) over
// an image in place, as PostProcessingEditorView runs them.
void ymref_post_process(float* image, const uint32_t* primitive_index, int width, int height, uint32_t selected,
                        float gamma, float exposure, int outline) {
  glm::vec4* img = reinterpret_cast<glm::vec4*>(image);
  auto grid = [&](auto body) {
    blockDim = dim3(32, 32, 1);
    gridDim = dim3((width + 31) / 32, (height + 31) / 32, 1);
    for (uint32_t by = 0; by < gridDim.y; ++by)
      for (uint32_t bx = 0; bx < gridDim.x; ++bx)
        for (uint32_t ty = 0; ty < 32; ++ty)
          for (uint32_t tx = 0; tx < 32; ++tx) {
            blockIdx = make_uint3(bx, by, 0);
            threadIdx = make_uint3(tx, ty, 0);
            body();
          }
  };
  grid([&]() { Gamma_correction_common(img, gamma, exposure, (uint32_t)width, (uint32_t)height); });
  if (outline && selected != EMPTY_UINT32)
    grid([&]() { Draw_outline(img, primitive_index, (uint32_t)width, (uint32_t)height, selected); });
}

double ymref_last_render_seconds(void* handle) { return static_cast<RefContext*>(handle)->last_render_seconds; }

// Closest-hit (TraceRay) and occlusion (BVHTraverseShadow) queries made by the
// stage kernels since the last reset (counted by oracle/build_ref.py's copy).
void ymref_query_counts(unsigned long long* out, int reset) {
  out[0] = ymrt_oracle_trace_queries.load();
  out[1] = ymrt_oracle_shadow_queries.load();
  if (reset) {
    ymrt_oracle_trace_queries.store(0);
    ymrt_oracle_shadow_queries.store(0);
  }
}

// Running mean over frames, src/Shading.cu:2354 Accumulate_image_path_tracing.
void ymref_accumulate(const float* noise, float* acc, int width, int height, int frame_index) {
  for (int y = 0; y < height; ++y)
    for (int x = 0; x < width; ++x) {
      blockIdx = make_uint3(0, 0, 0);
      blockDim = dim3(1, 1, 1);
      threadIdx = make_uint3(x, y, 0);
      Accumulate_image_path_tracing(reinterpret_cast<const glm::vec4*>(noise), reinterpret_cast<glm::vec4*>(acc),
                                    width, height, frame_index);
    }
}

}  // extern "C"
