// Wavefront path-tracing kernels for sm_100a.
//
// One frame is a sequence of waves over a fixed pool of path slots:
//   generate -> camera paths for whole 16x16 tiles appended behind the paths
//               still alive (Ray_generation_path_tracing, src/Shading.cu:1634);
//   extend   -> closest hit for every live path; misses are accumulated and
//               retired (Ray_trace_path_tracing, src/Shading.cu:1765);
//   shade    -> hit reconstruction, next-event estimation with both shadow
//               rays traced in place, BSDF continuation; surviving paths are
//               compacted into the other pool with one atomic per warp
//               (Ray_shading_path_tracing, src/Shading.cu:1953).
// Path state is structure-of-arrays (float4 / uint2 per field) so every
// field of a wave is read and written with coalesced 16-byte accesses.
//
// Per-path arithmetic follows the reference step for step (see dev_*.cuh),
// so each path's radiance equals the reference's; only the per-pixel sum of
// several samples depends on the order in which their atomics land.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include <cooperative_groups.h>


#include "wave_device.cuh"

namespace ym {

// Walks the wave's new paths (ctl->gen of them, written after the ctl->live
// continuing ones) with a grid-stride loop.
__global__ void __launch_bounds__(256) k_generate(PathPool P, const WaveControl* __restrict__ ctl,
                                                  const JobDesc* __restrict__ jobs, uint32_t n_jobs) {
  const uint32_t gen = ctl->gen, live = ctl->live;
  const unsigned long long cursor = ctl->gen_cursor;
  for (uint32_t tid = blockIdx.x * blockDim.x + threadIdx.x; tid < gen; tid += gridDim.x * blockDim.x)
    generate_path(P, live, tid, cursor, jobs, n_jobs);
}

__device__ __forceinline__ void generate_path(const PathPool& P, uint32_t base, uint32_t tid,
                                              unsigned long long path_cursor, const JobDesc* __restrict__ jobs,
                                              uint32_t n_jobs) {
  const uint32_t i = base + tid;
  const unsigned long long g = path_cursor + tid;
  const uint32_t job = find_job(jobs, n_jobs, g);
  const JobDesc& J = jobs[job];
  const DeviceScene& S = c_scenes[J.scene_slot];
  const uint32_t spp = J.spp;
  const int frame_index = J.frame_index;
  const uint32_t local_path = (uint32_t)(g - J.path_begin);
  const uint32_t per_tile = (uint32_t)kTilePixels * spp;
  const uint32_t tile = local_path / per_tile + J.tile_begin;
  const uint32_t tile_y = tile / J.tiles_x;
  const uint32_t tile_x = tile - J.tiles_x * tile_y;
  const uint32_t local = local_path - (tile - J.tile_begin) * per_tile;
  const uint32_t tile_pixel = local / spp;
  const uint32_t pixel_sample = local - tile_pixel * spp;
  const uint32_t tpy = tile_pixel / kTileRes;
  const uint32_t tpx = tile_pixel - tpy * kTileRes;
  const uint32_t px = tile_x * kTileRes + tpx;
  const uint32_t py = tile_y * kTileRes + tpy;
  if (!(px < (uint32_t)S.width && py < (uint32_t)S.height)) {
    P.pixel_flags[i] = make_uint2(kEmpty, kFlagDead);
    return;
  }
  const uint32_t pixel = py * (uint32_t)S.width + px;
  // Sampler set-up and pixel jitter, src/Shading.cu:1690-1711.
  PathSampler hs{0, 0u, 0u};
  float ox = 0.5f, oy = 0.5f;
  if (S.sampler_type == kSamplerHalton) {
    const uint64_t sample_index =
        halton_index(S, (int)px, (int)py, (frame_index - 1) * J.setting.ssp + (int)pixel_sample);
    hs = PathSampler{sample_index, 2u, 0u};
    ox = radical_inverse_2(sample_index);
    oy = radical_inverse_3(sample_index);
    ox = ox * S.halton_x_scale - float(px);
    oy = oy * S.halton_y_scale - float(py);
    ox = gmin(gmax(ox, 0.000001f), 0.999999f);
    oy = gmin(gmax(oy, 0.000001f), 0.999999f);
  } else if (S.sampler_type == kSamplerPcg) {
    hs = PathSampler{(uint64_t)pixel | ((uint64_t)pixel_sample << 32), 0u, (uint32_t)(frame_index - 1)};
    sample2d(hs, S, &ox, &oy);
  } else {
    const uint32_t sample = (uint32_t)(frame_index - 1) * (uint32_t)J.setting.ssp + pixel_sample;
    hs = PathSampler{(uint64_t)sample | ((uint64_t)pixel << 32), 1u, 0u};
    sample2d(hs, S, &ox, &oy);
  }
  // Camera::GenerateRay (src/Camera.h:164-170) + Ray's normalising constructor.
  const CameraDesc& cam = S.camera;
  const float ndc_x = float(px + ox) / float(S.width);
  const float ndc_y = float(py + oy) / float(S.height);
  const float h = 2.0f * cam.tan_half_fov;
  const float w = h * cam.aspect_ratio;
  const vec3 dir = normalize(-cam.w + (ndc_x - 0.5f) * w * cam.u + (ndc_y - 0.5f) * h * cam.v);
  store_path(P, i, cam.position, dir, vec3(1.0f), vec3(0.0f), pixel, flags_pack(1, true, true, job), kEmpty, kEmpty,
             hs, local_path);
  if (cam.transfer.record_count > 0) P.transfer[i] = cam.transfer;
  P.transfer_count[i] = (uint8_t)cam.transfer.record_count;
}

// Lists the slots holding hits bucket by bucket (a counting sort: the
// buckets' counts from k_extend give each bucket's start) and ends the paths
// whose ray left the scene: the background when the environment light is on
// (the miss branch of Ray_trace_path_tracing, src/Shading.cu:1855-1864), then
// the path's radiance into its pixel (not in the adjoint pass, whose jobs
// carry dLoss/dImage and only replay their paths). Misses are not listed.
// Debug recording: the vertex each watched path of job 0 reached in this
// wave's closest-hit stage (launched after k_extend only when a recorder is
// set; the render's kernels are unchanged).
__global__ void __launch_bounds__(256) k_record_vertices(PathPool P, const WaveControl* __restrict__ ctl, HitPool H,
                                                         const JobDesc* __restrict__ jobs, PathRecorder R) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ctl->count) return;
  const uint2 pf = P.pixel_flags[i];
  if ((pf.y & kFlagDead) || (pf.y >> kFlagJobShift) != 0u || pf.x >= R.n_pixels) return;
  if (!((R.watch[pf.x >> 5] >> (pf.x & 31u)) & 1u)) return;
  const uint32_t k = atomicAdd(R.count, 1u);
  if (k >= R.capacity) return;
  const uint4 ids = H.ids[i];
  const bool volume = (ids.z & 2u) != 0u, hit = ids.x != kEmpty || volume;
  VertexRecord v{};
  v.pixel = pf.x;
  v.depth = pf.y & kFlagDepthMask;
  v.flags = (hit ? kVertexHit : 0u) | (volume ? kVertexVolume : 0u) | ((ids.z & 1u) ? kVertexBack : 0u);
  v.inst = ids.x;
  v.tri = ids.y;
  const float4 o = P.ray_o[i], d = P.ray_d[i], tp = P.throughput[i], rad = P.radiance[i];
  const float4 bt = hit ? H.bary_t[i] : make_float4(1.0f, 1.0f, 1.0f, kTMax);
  v.t = bt.w;
  v.o[0] = o.x; v.o[1] = o.y; v.o[2] = o.z;
  v.d[0] = d.x; v.d[1] = d.y; v.d[2] = d.z;
  v.bary[0] = bt.x; v.bary[1] = bt.y; v.bary[2] = bt.z;
  v.throughput[0] = tp.x; v.throughput[1] = tp.y; v.throughput[2] = tp.z;
  v.radiance[0] = rad.x; v.radiance[1] = rad.y; v.radiance[2] = rad.z;
  v.path = P.path_id[i];
  (void)jobs;
  R.out[k] = v;
}

__global__ void __launch_bounds__(256) k_sort_hits(const WaveControl* __restrict__ ctl, HitPool H, PathPool P,
                                                   const JobDesc* __restrict__ jobs, WaveCounters* counters,
                                                   const uint32_t* __restrict__ ray_order) {
  __shared__ uint32_t s_start[kShadeBuckets];
  const uint32_t count = ctl->count;
  const uint32_t live = ray_order ? ctl->live : 0u;
  if (blockIdx.x * blockDim.x >= count) return;  // (uniform per block)
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int b = 0; b < kShadeBuckets; ++b) {
      s_start[b] = acc;
      acc += counters->bucket_count[b];
    }
  }
  __syncthreads();
  for (uint32_t warp_base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); warp_base < count;
       warp_base += gridDim.x * blockDim.x) {
  // slots in the order they were traced (continuing rays grouped), so that
  // each bucket lists its hits in that order too
  const uint32_t j = warp_base + (threadIdx.x & 31u);
  uint32_t i = j;
  if (j < live && ray_order[j] < live) i = ray_order[j];
  uint32_t b = j < count ? (uint32_t)H.bucket[i] : (uint32_t)kBucketNone;
  if (b == kBucketMiss) {
    const uint2 pf = P.pixel_flags[i];
    const JobDesc& J = jobs[pf.y >> kFlagJobShift];
    const float4 r4 = P.radiance[i];
    vec3 rad(r4.x, r4.y, r4.z);
    if (J.setting.enable_env_light) {
      const float4 t4 = P.throughput[i], d4 = P.ray_d[i];
      rad += indirect_clamp(J.setting, vec3(t4.x, t4.y, t4.z) * background(vec3(d4.x, d4.y, d4.z)),
                            (int)(pf.y & kFlagDepthMask));
    }
    if (!J.dloss) finish_path(J, pf.x, P.path_id[i], rad, 1.0f / gmax(J.setting.ssp, 1));  // (adjoint: replayed only)
    b = kBucketNone;
  }
  const bool has = b != kBucketNone;
  const uint32_t act = __ballot_sync(0xFFFFFFFFu, has);
  if (has) {
    const int lane = threadIdx.x & 31;
    const uint32_t peers = __match_any_sync(act, b);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&counters->bucket_fill[b], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    H.order[s_start[b] + base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = i;
  }
  }
}

// ----------------------------------------------------------- accumulate ---

__global__ void k_accumulate(const float4* noise, float4* acc, uint32_t n, int frame_index) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (frame_index == 1) {
    acc[i] = noise[i];
  } else {
    const float4 a = acc[i], z = noise[i];
    const float f1 = float(frame_index - 1), f = float(frame_index);
    acc[i] = make_float4((a.x * f1 + z.x) / f, (a.y * f1 + z.y) / f, (a.z * f1 + z.z) / f, (a.w * f1 + z.w) / f);
  }
}

// ---------------------------------------------------- known-answer tests ---

__global__ void __launch_bounds__(kTraceBlock) k_debug_trace(uint32_t slot, int n, const float* origin, const float* dir,
                                                             const uint32_t* last_hit, uint32_t* inst, uint32_t* tri,
                                                             float* t, float* bary, int* back, int* nearby,
                                                             uint32_t* errors) {
  YM_TRAVERSAL_SHARED(s_stack);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  TraversalStack st;
  st.bind(s_stack_entries, s_stack_t);
  const vec3 o(origin[3 * i], origin[3 * i + 1], origin[3 * i + 2]);
  const vec3 d = normalize(vec3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]));
  ClosestHit ch;
  uint32_t tests = 0, nodes = 0;
  const bool hit = trace_closest(slot, st, o, d, kTMax, last_hit ? last_hit[2 * i] : kEmpty,
                                 last_hit ? last_hit[2 * i + 1] : kEmpty, false, &ch, &tests, &nodes);
  inst[i] = hit ? ch.inst : kEmpty;
  tri[i] = hit ? ch.tri : kEmpty;
  t[i] = hit ? ch.t : kTMax;
  bary[3 * i] = hit ? ch.b0 : 1.0f;
  bary[3 * i + 1] = hit ? ch.b1 : 1.0f;
  bary[3 * i + 2] = hit ? ch.b2 : 1.0f;
  back[i] = hit ? ch.back : 0;
  nearby[i] = hit ? ch.nearby_count : 0;
  if (st.overflow) atomicOr(errors, (uint32_t)kDevErrStack);
}

__global__ void __launch_bounds__(kTraceBlock) k_debug_occluded(uint32_t slot, int n, const float* origin, const float* dir,
                                                                const float* tmax, int* occluded, uint32_t* errors) {
  YM_TRAVERSAL_SHARED(s_stack);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  TraversalStack st;
  st.bind(s_stack_entries, s_stack_t);
  const vec3 o(origin[3 * i], origin[3 * i + 1], origin[3 * i + 2]);
  const vec3 d = normalize(vec3(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]));
  uint32_t tests = 0, nodes = 0;
  occluded[i] = trace_occluded(slot, st, o, d, tmax[i], &tests, &nodes) ? 1 : 0;
  if (st.overflow) atomicOr(errors, (uint32_t)kDevErrStack);
}

__global__ void k_debug_density(uint32_t slot, int n, uint32_t tex, const float* p, float* out, uint32_t* errors) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DeviceScene& S = c_scenes[slot];
  out[i] = texture_eval(S.textures, tex, vec3(p[3 * i], p[3 * i + 1], p[3 * i + 2]), errors).x;
}

// ---------------------------------------------------------- editor view ---
//
// The editor's picking / albedo view (Ray_generation_editor_view,
// Ray_trace_editor_view, Ray_shading_editor_view, src/Shading.cu:1276-1594)
// fused into one thread per pixel: a camera ray through the pixel centre,
// closest hits followed through pass-through boundaries (medium stack
// updated as the shade stage does), then the hit surface's colour
// (MaterialSurfaceCol, src/BSDF.cuh:883-898: diffuse albedo or its texture;
// a light's colour times intensity; black for an invalid material) or the
// background (environment light on) / black on a miss, added to `beauty`
// with alpha 1. The camera ray's first hit writes the instance's
// unique_index into `primitive_index` (a miss leaves it). At most
// kEditorPassThroughs boundaries are followed; a ray still passing after
// that sets kDevErrIter and adds nothing.
constexpr int kEditorPassThroughs = 64;

__global__ void __launch_bounds__(kTraceBlock) k_editor_view(int slot, int width, int height, float aspect,
                                                             int env_light, float4* beauty, uint32_t* primitive_index,
                                                             uint32_t* errors) {
  YM_TRAVERSAL_SHARED(s_stack);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= width * height) return;
  const int px = i % width, py = i / width;
  const DeviceScene& S = c_scenes[slot];
  const CameraDesc& cam = S.camera;
  const float ndc_x = float(px + 0.5f) / float(width);
  const float ndc_y = float(py + 0.5f) / float(height);
  const float h = 2.0f * cam.tan_half_fov;
  const float w = h * aspect;
  vec3 o = cam.position;
  vec3 d = normalize(-cam.w + (ndc_x - 0.5f) * w * cam.u + (ndc_y - 0.5f) * h * cam.v);
  RayTransfer rt = cam.transfer;
  uint32_t last_inst = kEmpty, last_tri = kEmpty;
  TraversalStack st;
  st.bind(s_stack_entries, s_stack_t);
  uint32_t tests = 0, nodes = 0;
  vec3 col(0.0f);
  bool done = false;
  for (int pass = 0; pass <= kEditorPassThroughs && !done; ++pass) {
    ClosestHit ch;
    if (!trace_closest(slot, st, o, d, kTMax, last_inst, last_tri, false, &ch, &tests, &nodes)) {
      col = env_light ? background(d) : vec3(0.0f);
      done = true;
      break;
    }
    if (pass == 0) atomicExch(&primitive_index[i], S.instances[ch.inst].unique_index);
    const vec3 bary(ch.b0, ch.b1, ch.b2);
    const Instance inst = S.instances[ch.inst];
    if (!(inst.material_idx < S.material_count)) {
      done = true;
      break;
    }
    if (inst.treat_as_boundary) {
      if (pass == kEditorPassThroughs) break;
      vec3 p, p_err, ng;
      fetch_geometry_normal<kFeatAll>(S, ch.inst, ch.tri, bary, &p, &p_err, &ng);
      boundary_transition(S, rt, ch.nearby, ch.nearby_count, errors);
      o = offset_ray_origin(p, p_err, d, ng);
      d = normalize(d);  // the reference's Ray constructor normalises again
      last_inst = ch.inst;
      last_tri = ch.tri;
      continue;
    }
    const Material& mat = S.materials[inst.material_idx];
    if (mat.material_type == kLightMtl) {
      col = mat.light_mtl.light_color * mat.light_mtl.intensity;
    } else if (mat.material_type == kDefaultMtl) {
      const DefaultMtl& m = mat.default_mtl;
      if (m.diffuse_albedo_tex != kEmpty) {
        const SurfacePoint sp = fetch_surface<kFeatAll>(S, ch.inst, ch.tri, bary);
        col = surface_texture(S.textures, m.diffuse_albedo_tex, TexCoord{sp.u, sp.v, sp.p_obj}, errors);
      } else {
        col = m.diffuse_albedo;
      }
    }
    done = true;
  }
  if (st.overflow) atomicOr(errors, (uint32_t)kDevErrStack);
  if (!done) {
    atomicOr(errors, (uint32_t)kDevErrIter);
    note_bound(kBoundEditorBoundaries, kEditorPassThroughs, o, d, kTMax, last_inst, last_tri, &rt);
    return;
  }
  atomicAdd(&beauty[i].x, col.x);
  atomicAdd(&beauty[i].y, col.y);
  atomicAdd(&beauty[i].z, col.z);
  atomicAdd(&beauty[i].w, 1.0f);
}

// Gamma_correction_common (src/Shading.cu:2396-2425): ACES tone mapping of
// the exposed colour, then 1/gamma, alpha 1.
__global__ void k_tonemap(float4* image, int width, int height, float gamma, float exposure) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= width || y >= height) return;
  const size_t k = (size_t)y * width + x;
  const float4 c = image[k];
  vec3 col(c.x, c.y, c.z);
  const float a = 2.51f, b = 0.03f, cc = 2.43f, dd = 0.59f, e = 0.14f;
  col *= exposure;
  col = (col * (a * col + b)) / (col * (cc * col + dd) + e);
  const float g = 1.0f / gamma;
  image[k] = make_float4(powf(col.x, g), powf(col.y, g), powf(col.z, g), 1.0f);
}

// Draw_outline (src/Shading.cu:2426-2466): pixels whose 3x3 neighbourhood
// (clipped to the image) shows the selected instance partly become red,
// wholly a 60% tint towards (0.9, 0.2, 0.2); alpha 1.
__global__ void k_outline(float4* image, const uint32_t* primitive_index, int width, int height, uint32_t selected) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= width || y >= height) return;
  int hits = 0, total = 0;
  for (int dx = -1; dx <= 1; ++dx)
    for (int dy = -1; dy <= 1; ++dy) {
      const int sx = x + dx, sy = y + dy;
      if (sx < 0 || sx >= width || sy < 0 || sy >= height) continue;
      ++total;
      if (primitive_index[(size_t)sy * width + sx] == selected) ++hits;
    }
  const size_t k = (size_t)y * width + x;
  const float4 c = image[k];
  vec3 r(c.x, c.y, c.z);
  if (hits == total) r = mix(r, vec3(0.9f, 0.2f, 0.2f), 0.6f);
  else if (hits != 0) r = vec3(1.0f, 0.0f, 0.0f);
  image[k] = make_float4(r.x, r.y, r.z, 1.0f);
}

// The shading frame k_shade builds at given hits of scene slot 0 (the
// layout of the oracle's shading-frame probe): normal, tangent, bitangent,
// texture footprint, uv, object-space position, dp/du, material index.
__global__ void k_debug_frame(uint32_t slot, int n, const uint32_t* inst, const uint32_t* tri, const float* bary, const int* back,
                              const float* dir, float* out, uint32_t* errors) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DeviceScene& S = c_scenes[slot];
  float* o = out + 22 * (size_t)i;
  for (int k = 0; k < 22; ++k) o[k] = 0.0f;
  if (inst[i] >= S.instance_count) return;
  const vec3 rd(dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]);
  const SurfacePoint sp = fetch_surface<kFeatAll>(S, inst[i], tri[i], vec3(bary[3 * i], bary[3 * i + 1], bary[3 * i + 2]));
  const Instance in = S.instances[inst[i]];
  if (in.material_idx >= S.material_count) return;
  const Material& mat = S.materials[in.material_idx];
  float d[4];
  tex_differentials(S.camera, sp.p, sp.ns, sp.ng, sp.dpdu, sp.dpdv, S.width, S.height, 0.25f, 0.25f, d);
  LayeredBsdf B;
  const TexCoord tc{sp.u, sp.v, sp.p_obj};
  if (mat.material_type == kDefaultMtl && material_textured(mat.default_mtl))
    init_shading_frame_mapped(B, mat.default_mtl, back[i], rd, sp, S.i_transforms[in.transform_idx], S, tc, errors);
  else
    init_shading_frame(B, back[i], rd, sp.ng, sp.ns, sp.dpdu, sp.dpdv);
  const float v[22] = {B.n.x, B.n.y, B.n.z, B.t.x, B.t.y, B.t.z, B.b.x, B.b.y, B.b.z, d[0], d[1], d[2], d[3],
                       sp.u, sp.v, sp.p_obj.x, sp.p_obj.y, sp.p_obj.z, sp.dpdu.x, sp.dpdu.y, sp.dpdu.z,
                       (float)in.material_idx};
  for (int k = 0; k < 22; ++k) o[k] = v[k];
}

// Texture node `tex` of scene slot 0 at points (s, t, x, y, z): rgb out.
__global__ void k_debug_texture(uint32_t slot, int n, uint32_t tex, const float* c, float* out, uint32_t* errors) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DeviceScene& S = c_scenes[slot];
  const TexCoord tc{c[5 * i], c[5 * i + 1], vec3(c[5 * i + 2], c[5 * i + 3], c[5 * i + 4])};
  const vec3 r = surface_texture(S.textures, tex, tc, errors);
  out[3 * i] = r.x;
  out[3 * i + 1] = r.y;
  out[3 * i + 2] = r.z;
}

__global__ void k_debug_halton(uint32_t slot, int n, const int* px, const int* py, const int* sample, int n_dims, uint64_t* index,
                               float* offset, float* dims) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const DeviceScene& S = c_scenes[slot];
  const uint64_t idx = halton_index(S, px[i], py[i], sample[i]);
  index[i] = idx;
  float ox = radical_inverse_2(idx), oy = radical_inverse_3(idx);
  ox = ox * S.halton_x_scale - float(px[i]);
  oy = oy * S.halton_y_scale - float(py[i]);
  offset[2 * i] = gmin(gmax(ox, 0.000001f), 0.999999f);
  offset[2 * i + 1] = gmin(gmax(oy, 0.000001f), 0.999999f);
  PathSampler hs{idx, 2u, 0u};
  for (int d = 0; d < n_dims; ++d) dims[(size_t)i * n_dims + d] = halton_draw(hs, S.halton_perm);
}

// ------------------------------------------------------------ launchers ---

cudaError_t upload_constants(const DeviceScene* scenes, const uint32_t* slots, uint32_t n, const uint32_t* primes,
                             const uint32_t* prime_sums, cudaStream_t stream) {
  cudaError_t e = upload_slots_here(scenes, slots, n, primes, prime_sums, stream);
  if (e == cudaSuccess) e = upload_slots_media(scenes, slots, n, primes, prime_sums, stream);
  if (e == cudaSuccess) e = upload_slots_adjoint(scenes, slots, n, primes, prime_sums, stream);
  return e;
}

// ---------------------------------------------------------- wave control ---

// Start of a wave: the continuing paths left by the previous wave, the new
// paths to generate (as many as fit), and the per-wave counters cleared.
__global__ void k_plan(WaveControl* ctl, WaveCounters* counters) {
  __shared__ uint32_t s_live;
  if (threadIdx.x == 0) s_live = counters->next_count;
  __syncthreads();
  uint32_t* words = reinterpret_cast<uint32_t*>(counters);
  for (uint32_t k = threadIdx.x; k < (uint32_t)(kWaveClearBytes / sizeof(uint32_t)); k += blockDim.x) words[k] = 0u;
  if (threadIdx.x == 0) {
    const uint32_t live = ctl->more ? s_live : 0u;
    const unsigned long long left = ctl->more ? ctl->total - ctl->cursor : 0ull;
    const uint32_t room = ctl->capacity > live ? ctl->capacity - live : 0u;
    const uint32_t gen = (uint32_t)(left < (unsigned long long)room ? left : (unsigned long long)room);
    ctl->live = live;
    ctl->gen = gen;
    ctl->count = live + gen;
    ctl->gen_cursor = ctl->cursor;
    ctl->cursor += gen;
  }
}

// ------------------------------------------- continuing rays, grouped ---
//
// Continuing rays leave surfaces all over the scene in scattered directions;
// k_shade writes them in shading order (grouped by material). Traced in that
// order, the 32 lanes of a warp walk unrelated parts of the BVH. Before the
// closest-hit stage, the wave's continuing slots are grouped by a key of the
// ray's origin cell (an 8x8x8 grid over the scene's top-level bounds, Morton
// order) and its direction (cube face and quadrant, 24 values) with one
// counting sort (k_ray_hist, k_ray_scan_*, k_ray_scatter), and k_extend takes
// them in that order. The hits are written to the rays' own slots, so nothing
// after the closest-hit stage sees the order.

__device__ __forceinline__ uint32_t spread3(uint32_t v) {  // bits 0, 1, 2, ... -> bits 0, 3, 6, ...
  uint32_t r = 0;
  for (uint32_t b = 0; b < kRayCellBits; ++b) r |= ((v >> b) & 1u) << (3 * b);
  return r;
}

__device__ __forceinline__ uint32_t face_square(float u, float major) {  // u / |major| in [-1, 1] -> 0..kRayDirSplit-1
  const float f = (u / major + 1.0f) * (0.5f * (float)kRayDirSplit);
  return f > 0.0f ? min((uint32_t)f, kRayDirSplit - 1u) : 0u;
}

__device__ __forceinline__ uint32_t ray_group_key(const DeviceScene& S, float4 o, float4 d) {
  // the scene's bounds: the top-level root's grid, origin + [0, 255] * 2^e
  const uint4 w0 = __ldg(reinterpret_cast<const uint4*>(S.tlas_nodes));
  const float lo[3] = {__uint_as_float(w0.x), __uint_as_float(w0.y), __uint_as_float(w0.z)};
  const float ext[3] = {255.0f * __uint_as_float((w0.w & 0xFFu) << 23),
                        255.0f * __uint_as_float(((w0.w >> 8) & 0xFFu) << 23),
                        255.0f * __uint_as_float(((w0.w >> 16) & 0xFFu) << 23)};
  const float p[3] = {o.x, o.y, o.z};
  constexpr float kCells = (float)(1u << kRayCellBits);
  uint32_t cell[3];
  for (int a = 0; a < 3; ++a) {
    const float f = (p[a] - lo[a]) / ext[a] * kCells;
    cell[a] = f > 0.0f ? min((uint32_t)f, (1u << kRayCellBits) - 1u) : 0u;
  }
  const uint32_t morton = spread3(cell[0]) | (spread3(cell[1]) << 1) | (spread3(cell[2]) << 2);
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  uint32_t face, su, sv;
  if (ax >= ay && ax >= az) {
    face = d.x < 0.0f ? 1u : 0u;
    su = face_square(d.y, ax);
    sv = face_square(d.z, ax);
  } else if (ay >= az) {
    face = d.y < 0.0f ? 3u : 2u;
    su = face_square(d.x, ay);
    sv = face_square(d.z, ay);
  } else {
    face = d.z < 0.0f ? 5u : 4u;
    su = face_square(d.x, az);
    sv = face_square(d.y, az);
  }
  return morton * kRayDirs + (face * kRayDirSplit + su) * kRayDirSplit + sv;  // < kRayBins
}

__global__ void __launch_bounds__(256) k_ray_hist(PathPool P, const WaveControl* __restrict__ ctl, HitPool H,
                                                  const JobDesc* __restrict__ jobs) {
  const uint32_t live = ctl->live;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < live; i += gridDim.x * blockDim.x) {
    const uint2 pf = P.pixel_flags[i];
    const uint32_t key = ray_group_key(c_scenes[jobs[pf.y >> kFlagJobShift].scene_slot], P.ray_o[i], P.ray_d[i]);
    H.ray_key[i] = key;
    atomicAdd(&H.ray_bins[key], 1u);
  }
}

// Exclusive prefix sums of the kRayBins counts, in two steps: each
// 1024-bin block's own prefix sums into the offsets and its total into
// partial[block] (clearing the counts for the next wave), then the block
// totals' prefix sums (one block); k_ray_scatter adds the two.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t s_warp[32];
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (uint32_t off = 1; off < 32; off <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
    if (lane >= off) x += y;
  }
  if (lane == 31) s_warp[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const uint32_t n_warps = blockDim.x >> 5;
    uint32_t w = lane < n_warps ? s_warp[lane] : 0u;
    for (uint32_t off = 1; off < 32; off <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, w, off);
      if (lane >= off) w += y;
    }
    s_warp[lane] = w;  // inclusive totals of warps 0..lane
  }
  __syncthreads();
  *total = s_warp[(blockDim.x >> 5) - 1];
  return x - v + (warp > 0 ? s_warp[warp - 1] : 0u);
}

__global__ void __launch_bounds__(1024) k_ray_scan_blocks(HitPool H) {
  const uint32_t k = blockIdx.x * 1024u + threadIdx.x;
  const uint32_t v = k < kRayBins ? H.ray_bins[k] : 0u;
  uint32_t total;
  const uint32_t x = block_exclusive_scan(v, &total);
  if (k < kRayBins) {
    H.ray_bins[kRayBins + k] = x;
    H.ray_bins[k] = 0u;
  }
  if (threadIdx.x == 0) H.ray_bins[2 * kRayBins + blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_ray_scan_partials(HitPool H) {
  const uint32_t k = threadIdx.x;
  const uint32_t v = k < kRayScanBlocks ? H.ray_bins[2 * kRayBins + k] : 0u;
  uint32_t total;
  const uint32_t x = block_exclusive_scan(v, &total);
  if (k < kRayScanBlocks) H.ray_bins[2 * kRayBins + k] = x;
}

__global__ void __launch_bounds__(256) k_ray_scatter(const WaveControl* __restrict__ ctl, HitPool H) {
  const uint32_t live = ctl->live;
  for (uint32_t warp_base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); warp_base < live;
       warp_base += gridDim.x * blockDim.x) {
    const uint32_t i = warp_base + (threadIdx.x & 31u);
    const bool has = i < live;
    const uint32_t key = has ? (uint32_t)H.ray_key[i] : 0u;
    const uint32_t act = __ballot_sync(0xFFFFFFFFu, has);
    if (!has) continue;
    // lanes with the same key take consecutive positions, in slot order
    const int lane = threadIdx.x & 31;
    const uint32_t peers = __match_any_sync(act, key);
    const int leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader)
      base = H.ray_bins[2 * kRayBins + (key >> 10)] + atomicAdd(&H.ray_bins[kRayBins + key], (uint32_t)__popc(peers));
    base = __shfl_sync(peers, base, leader);
    H.ray_order[base + (uint32_t)__popc(peers & ((1u << lane) - 1u))] = i;
  }
}

// End of a wave: totals, and whether another wave is needed (the loop is
// bounded by max_waves, after which YMRT_DEVERR_ITER is raised).
__global__ void k_finish(WaveControl* ctl, WaveCounters* counters, unsigned long long graph_condition) {
  if (threadIdx.x != 0) return;
  if (!ctl->more) {
    if (graph_condition) cudaGraphSetConditional((cudaGraphConditionalHandle)graph_condition, 0u);
    return;
  }
  ctl->hits += counters->hit_count;
  ctl->waves += 1;
  bool more = counters->next_count > 0 || ctl->cursor < ctl->total;
  if (more && ctl->waves >= ctl->max_waves) {
    atomicOr(&counters->errors, (uint32_t)kDevErrIter);
    note_bound(kBoundWaves, ctl->waves, vec3(0.0f), vec3(0.0f), 0.0f, kEmpty, kEmpty, nullptr);
    more = false;
  }
  if (!more) counters->next_count = 0;
  ctl->more = more ? 1u : 0u;
  if (graph_condition) cudaGraphSetConditional((cudaGraphConditionalHandle)graph_condition, more ? 1u : 0u);
}

namespace {

// Persistent grid size (resident blocks per SM x SMs) of k_connect, which
// walks its queue grid-stride; the per-path kernels get one thread per slot.
struct PersistentGrids {
  int device = -1;
  uint32_t connect[3] = {0, 0, 0};  // k_connect blocks for 64-, 128- and 256-thread blocks
};
PersistentGrids g_grids;

template <typename K>
uint32_t grid_for(K kernel, int block, int sms) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
  return (uint32_t)(per_sm * sms);
}

// Surface (no media, no adjoint) extend and shade launches for scene
// features kF: instantiated on the sphere and texture bits (grids are media),
// so a batch runs one of four instantiations of each. The media and adjoint
// kernels are instantiated in wave_media.cu and wave_adjoint.cu.
template <uint32_t kF>
void launch_extend_surface(const WaveArgs& w) {
  const auto k = k_extend<false, kF & kFeatSpheres>;
  k<<<w.trace_blocks, w.trace_block, traversal_shared_bytes(w.trace_block), w.stream>>>(w.A, w.ctl, w.H, w.jobs, w.counters, nullptr,
                                                                   kEmpty, w.ray_order);
}

template <uint32_t kF>
void launch_shade_surface(const ShadowQueue* defer, const WaveArgs& w) {
  constexpr uint32_t kS = surface_features(kF);
  const ShadowQueue none{};
  if (defer)
    k_shade<false, true, false, kS><<<w.blocks, kTraceBlock, 0, w.stream>>>(w.A, w.ctl, w.H, w.B, w.jobs, w.counters,
                                                                            *defer);
  else
    k_shade<false, false, false, kS><<<w.blocks, kTraceBlock, 0, w.stream>>>(w.A, w.ctl, w.H, w.B, w.jobs,
                                                                             w.counters, none);
}

}  // namespace

void prepare_persistent_grids() {
  int dev = 0;
  cudaGetDevice(&dev);
  if (g_grids.device == dev) return;
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  PersistentGrids g;
  g.device = dev;
  for (int b = 0; b < 3; ++b) {
    const int block = 64 << b;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_connect<0>, block, occluded_shared_bytes(block)) !=
            cudaSuccess || per_sm < 1)
      per_sm = 1;
    g.connect[b] = (uint32_t)(per_sm * sms);
  }
  allow_trace_shared(k_extend<false, 0>);
  allow_trace_shared(k_extend<false, kFeatSpheres>);
  prepare_media_kernels();
  prepare_adjoint_kernels();
  g_grids = g;
}

uint32_t launch_wave(const PathPool& A, const PathPool& B, const HitPool& H, WaveControl* ctl, const JobDesc* jobs,
                     uint32_t n_jobs, WaveCounters* counters, const WaveOptions& opt, cudaEvent_t* ev,
                     cudaStream_t stream, unsigned long long graph_condition) {
  prepare_persistent_grids();
  const PersistentGrids& g = g_grids;
  const bool adjoint = opt.adjoint;
  const ShadowQueue* defer = (!opt.volumes && opt.defer_shadows && !adjoint) ? &opt.shadow_queue : nullptr;
  const bool sort_hits = opt.sort_hits;
  HitPool Hs = H;
  if (!sort_hits) Hs.order = nullptr;
  const uint32_t feat = opt.features & kFeatAll;
  // The per-path kernels get one thread per pool slot (blocks past the
  // wave's count return at once), so the hardware block scheduler balances
  // the uneven per-ray work; k_connect walks its queue with a GPU-sized grid.
  const uint32_t cap = std::max(opt.capacity, 1u);
  const uint32_t blocks_256 = (cap + 255) / 256, blocks_trace = (cap + kTraceBlock - 1) / kTraceBlock;
  // continuing rays grouped before tracing (the pool must have the key arrays)
  const bool sort_rays = opt.sort_rays && H.ray_key && H.ray_bins && H.ray_order;
  k_plan<<<1, 128, 0, stream>>>(ctl, counters);
  if (sort_rays) {
    // (the counts are zero: cleared when allocated, at the start of every
    // frame and by each wave's k_ray_scan_blocks)
    k_ray_hist<<<blocks_256, 256, 0, stream>>>(A, ctl, H, jobs);
    k_ray_scan_blocks<<<kRayScanBlocks, 1024, 0, stream>>>(H);
    k_ray_scan_partials<<<1, 1024, 0, stream>>>(H);
    k_ray_scatter<<<blocks_256, 256, 0, stream>>>(ctl, H);
  }
  if (ev) cudaEventRecord(ev[0], stream);
  k_generate<<<blocks_256, 256, 0, stream>>>(A, ctl, jobs, n_jobs);
  if (ev) cudaEventRecord(ev[1], stream);
  const uint32_t tb = (opt.trace_block == 64 || opt.trace_block == 256) ? opt.trace_block : (uint32_t)kTraceBlock;
  const WaveArgs w{A, B, Hs, ctl, jobs, counters, blocks_trace, stream, tb, (cap + tb - 1) / tb,
                   sort_rays ? H.ray_order : nullptr};
  if (adjoint && opt.volumes) {
    launch_adjoint_extend_media(w, opt);
  } else if (opt.volumes) {
    launch_media_extend(feat, w);
  } else {
    switch (feat & kFeatSpheres) {
      case 0: launch_extend_surface<0>(w); break;
      default: launch_extend_surface<kFeatSpheres>(w); break;
    }
  }
  if (opt.recorder.out) k_record_vertices<<<blocks_256, 256, 0, stream>>>(A, ctl, H, jobs, opt.recorder);
  if (ev) cudaEventRecord(ev[2], stream);
  if (sort_hits) k_sort_hits<<<blocks_256, 256, 0, stream>>>(ctl, Hs, A, jobs, counters, w.ray_order);
  if (ev) cudaEventRecord(ev[3], stream);
  if (adjoint) {
    launch_adjoint_shade(opt.volumes, feat, w, opt);
  } else if (opt.volumes) {
    launch_media_shade(feat, w);
  } else {
    switch (surface_features(feat)) {
      case 0: launch_shade_surface<0>(defer, w); break;
      case kFeatSpheres: launch_shade_surface<kFeatSpheres>(defer, w); break;
      case kFeatTextures: launch_shade_surface<kFeatTextures>(defer, w); break;
      default: launch_shade_surface<kFeatSpheres | kFeatTextures>(defer, w); break;
    }
  }
  if (ev) cudaEventRecord(ev[4], stream);
  const uint32_t conn_grid = g.connect[tb == 64 ? 0 : (tb == 128 ? 1 : 2)];
  if (defer && (feat & kFeatSpheres))
    k_connect<kFeatSpheres><<<conn_grid, tb, occluded_shared_bytes(tb), stream>>>(*defer, jobs, counters);
  else if (defer)
    k_connect<0><<<conn_grid, tb, occluded_shared_bytes(tb), stream>>>(*defer, jobs, counters);
  if (ev) cudaEventRecord(ev[5], stream);
  k_finish<<<1, 32, 0, stream>>>(ctl, counters, graph_condition);
  return 5u + (sort_hits ? 1u : 0u) + (defer ? 1u : 0u) + (sort_rays ? 4u : 0u);
}

cudaError_t read_bound_record(uint32_t* words, int n_words, bool clear, cudaStream_t stream) {
  // the first record taken in any translation unit
  BoundRecord r[3];
  cudaError_t e = read_bound_here(&r[0], clear, stream);
  if (e == cudaSuccess) e = read_bound_media(&r[1], clear, stream);
  if (e == cudaSuccess) e = read_bound_adjoint(&r[2], clear, stream);
  if (e != cudaSuccess) return e;
  int k = 0;
  while (k < 2 && r[k].taken != 1u) ++k;
  std::memcpy(words, &r[k], sizeof(uint32_t) * (size_t)std::min(n_words, kBoundRecordWords));
  return cudaSuccess;
}

void launch_accumulate(const float4* noise, float4* acc, uint32_t n, int frame_index, cudaStream_t stream) {
  if (n == 0) return;
  k_accumulate<<<(n + 255) / 256, 256, 0, stream>>>(noise, acc, n, frame_index);
}

void launch_debug_trace(uint32_t slot, int n, const float* o, const float* d, const uint32_t* lh, uint32_t* inst, uint32_t* tri,
                        float* t, float* bary, int* back, int* nearby, uint32_t* errors, cudaStream_t stream) {
  if (n <= 0) return;
  k_debug_trace<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, stream>>>(slot, n, o, d, lh, inst, tri, t, bary, back,
                                                                                 nearby, errors);
}

void launch_debug_density(uint32_t slot, int n, uint32_t tex, const float* p, float* out, uint32_t* err, cudaStream_t stream) {
  if (n <= 0) return;
  k_debug_density<<<(n + 255) / 256, 256, 0, stream>>>(slot, n, tex, p, out, err);
}

void launch_editor_view(int slot, int width, int height, int env_light, float4* beauty, uint32_t* primitive_index,
                        uint32_t* errors, cudaStream_t stream) {
  const int n = width * height;
  if (n <= 0) return;
  k_editor_view<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, stream>>>(
      slot, width, height, float(width) / float(height), env_light, beauty, primitive_index, errors);
}

void launch_post_process(float4* image, const uint32_t* primitive_index, int width, int height, uint32_t selected,
                         float gamma, float exposure, bool outline, cudaStream_t stream) {
  if (width <= 0 || height <= 0) return;
  const dim3 block(32, 8), grid((width + 31) / 32, (height + 7) / 8);
  k_tonemap<<<grid, block, 0, stream>>>(image, width, height, gamma, exposure);
  if (outline) k_outline<<<grid, block, 0, stream>>>(image, primitive_index, width, height, selected);
}

void launch_debug_frame(uint32_t slot, int n, const uint32_t* inst, const uint32_t* tri, const float* bary, const int* back,
                        const float* dir, float* out, uint32_t* err, cudaStream_t stream) {
  if (n <= 0) return;
  k_debug_frame<<<(n + 127) / 128, 128, 0, stream>>>(slot, n, inst, tri, bary, back, dir, out, err);
}

void launch_debug_texture(uint32_t slot, int n, uint32_t tex, const float* c, float* out, uint32_t* err, cudaStream_t stream) {
  if (n <= 0) return;
  k_debug_texture<<<(n + 255) / 256, 256, 0, stream>>>(slot, n, tex, c, out, err);
}

void launch_debug_occluded(uint32_t slot, int n, const float* o, const float* d, const float* tmax, int* occ, uint32_t* errors,
                           cudaStream_t stream) {
  if (n <= 0) return;
  k_debug_occluded<<<(n + kTraceBlock - 1) / kTraceBlock, kTraceBlock, 0, stream>>>(slot, n, o, d, tmax, occ, errors);
}

void launch_debug_halton(uint32_t slot, int n, const int* px, const int* py, const int* sample, int n_dims, uint64_t* index,
                         float* offset, float* dims, cudaStream_t stream) {
  if (n <= 0) return;
  k_debug_halton<<<(n + 127) / 128, 128, 0, stream>>>(slot, n, px, py, sample, n_dims, index, offset, dims);
}

}  // namespace ym
