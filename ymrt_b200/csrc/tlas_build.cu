// Top-level rebuild on the device after transform edits (ymrt_scene_set_transforms).
//
// The reference rebuilds its top-level BVH on the host at every scene edit
// and reorders the instance array by the build (GuiModule::UpdateScene,
// src/core/GuiModule.cpp:123-139; TopBVH.cpp:34-198, dst_indices_map at
// :171-191), which also reorders the shape-light table; the whole scene is
// then uploaded again. Here the uploaded scene is rebuilt where it lives:
//   k_tlas_items    instance world boxes (one thread per instance)
//   k_tlas_binary   the binary SAH build, level by level in one block: each
//                   frontier node is split by one thread (the nodes' item
//                   ranges are disjoint), one thread numbers the children in
//                   node order as the host builder does
//   k_tlas_wide     the wide collapse (one thread, depth first)
//   k_tlas_reorder  instances, shading buckets and file indices into the
//                   build's order
//   k_light_count / k_light_offsets / k_light_fill / k_light_table
//                   the shape-light table in the new order
//   k_camera_inside / k_camera_stack
//                   the camera's nested-media stack
// Every step is bvh_build.h's, the code the host preparation runs, so the
// device-built top level equals a host rebuild bit for bit.
#include <cuda_runtime.h>

#include "bvh_build.h"
#include "kernels.h"
#include "sphere.h"

namespace ym {

namespace {

__global__ void k_tlas_items(TlasBuild b) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  const Instance inst = b.instances[i];
  const GeometryDesc& g = b.geometries[inst.geometry_idx];
  BBox root;
  root.pmin = g.bbox_min;
  root.pmax = g.bbox_max;
  BuildItem it;
  it.box = box_transform(root, b.transforms[inst.transform_idx]);
  it.center = box_center(it.box);
  it.idx = i;
  b.items[i] = it;
}

constexpr int kBinaryThreads = 512;

__global__ void __launch_bounds__(kBinaryThreads) k_tlas_binary(TlasBuild b) {
  __shared__ uint32_t s_start, s_total;
  if (threadIdx.x == 0) {
    BinNode root;
    root.offset = 0;
    root.count = b.n;
    root.left = root.right = kEmpty;
    b.nodes[0] = root;
    b.mid[0] = 0;
    s_start = 0;
    s_total = 1;
  }
  __syncthreads();
  for (;;) {
    const uint32_t start = s_start, total = s_total;
    if (total == start) break;
    for (uint32_t ni = start + threadIdx.x; ni < total; ni += blockDim.x) {
      BinNode node = b.nodes[ni];
      uint32_t left_count = 0;
      const int kind = split_node(node, b.items + node.offset, b.mid[ni] != 0, &left_count);
      node.left = node.right = kEmpty;
      b.nodes[ni] = node;
      b.split_kind[ni] = (uint8_t)kind;
      b.split_left[ni] = left_count;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      // children numbered in node order, two per split node (the host's order)
      uint32_t t = total;
      for (uint32_t ni = start; ni < total; ++ni) {
        const int kind = b.split_kind[ni];
        if (kind == kSplitLeaf) continue;
        BinNode& node = b.nodes[ni];
        const uint32_t lc = b.split_left[ni];
        node.left = t;
        node.right = t + 1;
        BinNode l, r;
        l.offset = node.offset;
        l.count = lc;
        r.offset = node.offset + lc;
        r.count = node.count - lc;
        l.left = l.right = r.left = r.right = kEmpty;
        b.nodes[t] = l;
        b.nodes[t + 1] = r;
        b.mid[t] = b.mid[t + 1] = kind == kSplitMid ? 1 : 0;
        t += 2;
      }
      s_start = total;
      s_total = t;
    }
    __syncthreads();
  }
}

__global__ void k_tlas_wide(TlasBuild b, uint32_t max_leaf) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t n_nodes = 1, n_prims = 0;
  build_wide_into(b.nodes, max_leaf, b.wide, 0, &n_nodes, b.prims, &n_prims, b.stack);
  b.counts[0] = n_nodes;
  b.counts[1] = n_prims;
}

__global__ void k_tlas_reorder(TlasBuild b) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  const uint32_t src = b.items[i].idx;
  b.instances_out[i] = b.instances[src];
  b.bucket_out[i] = b.bucket[src];
  b.file_index_out[i] = b.file_index[src];
}

// SceneModule::LoadShapeLight (src/core/SceneModule.cpp:1203-1304), in the
// new instance order: one entry per triangle of a light mesh, one per light
// sphere.
__device__ __forceinline__ uint32_t light_entries(const TlasBuild& b, const Instance& inst) {
  if (!(inst.material_idx < b.material_count) || b.materials[inst.material_idx].material_type != kLightMtl) return 0u;
  const GeometryDesc& g = b.geometries[inst.geometry_idx];
  return g.kind == kGeoSphere ? 1u : g.tri_count;
}

__global__ void k_light_count(TlasBuild b) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= b.n) return;
  b.light_offsets[i] = light_entries(b, b.instances_out[i]);
}

__global__ void k_light_offsets(TlasBuild b) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  uint32_t acc = 0;
  for (uint32_t i = 0; i < b.n; ++i) {
    const uint32_t c = b.light_offsets[i];
    b.light_offsets[i] = acc;
    acc += c;
  }
  b.counts[2] = acc;
}

__global__ void k_light_fill(TlasBuild b) {
  const uint32_t pi = blockIdx.x * blockDim.x + threadIdx.x;
  if (pi >= b.n || b.counts[2] != b.light_count) return;  // (a different light count is reported by the host)
  const Instance inst = b.instances_out[pi];
  const uint32_t n = light_entries(b, inst);
  if (n == 0) return;
  const Material& mat = b.materials[inst.material_idx];
  const mat4& otw = b.transforms[inst.transform_idx];
  const vec3 c = mat.light_mtl.light_color;
  const float irradiance = (c.x + c.y + c.z) * mat.light_mtl.intensity * kPi;
  const GeometryDesc& g = b.geometries[inst.geometry_idx];
  ShapeLight* out = b.lights + b.light_offsets[pi];
  if (g.kind == kGeoSphere) {
    // the transform's own scale stretches the sphere into an ellipsoid;
    // its area is approximated as (4/3) pi (ab + bc + ca)
    const vec3 sc = b.transform_scales[inst.transform_idx];
    const float a = g.radius * sc.x, bb = g.radius * sc.y, c3 = g.radius * sc.z;
    const float area = (4.0f / 3.0f) * kPi * (a * bb + bb * c3 + c3 * a);
    out[0] = ShapeLight{pi, kEmpty, irradiance * area, area};
    return;
  }
  for (uint32_t t = 0; t < n; ++t) {
    const uint32_t* tc = b.tri_corners + 3 * (size_t)(g.tri_offset + t);
    vec3 p[3];
    for (int k = 0; k < 3; ++k) {
      const uint32_t vi = b.pos_idx[g.corner_offset + tc[k]];
      const float* q = b.positions + 3 * (size_t)(g.pos_offset + vi);
      p[k] = transform_position(otw, vec3(q[0], q[1], q[2]));
    }
    const float area = length(cross(p[1] - p[0], p[2] - p[0]));
    out[t] = ShapeLight{pi, t, irradiance * area, 0.5f * area};
  }
}

// The power CDF, summed in light order as the host does.
__global__ void k_light_table(TlasBuild b) {
  if (threadIdx.x != 0 || blockIdx.x != 0 || b.counts[2] != b.light_count) return;
  float total = 0.0f;
  for (uint32_t i = 0; i < b.light_count; ++i) {
    total += b.lights[i].power;
    b.light_table[i] = total;
  }
  const float rcp = safe_rcp(total);
  for (uint32_t i = 0; i < b.light_count; ++i) b.light_table[i] = total == 0.0f ? 0.0f : (b.light_table[i] * rcp);
}

// Camera::InitCameraRayTransfer (src/Camera.cpp:15-78): an instance encloses
// the camera when a ray from it hits the instance forwards and backwards.
// One block per instance, its threads over the mesh's triangles (each test's
// answer is the host's; only whether any triangle is hit matters).
constexpr int kCameraThreads = 256;

__global__ void __launch_bounds__(kCameraThreads) k_camera_inside(TlasBuild b, vec3 cam_pos, vec3 cam_dir) {
  const uint32_t i = blockIdx.x;
  if (i >= b.n) return;
  const Instance inst = b.instances_out[i];
  const mat4& wto = b.i_transforms[inst.transform_idx];
  const vec3 o = xform_point_glm(wto, cam_pos);
  const vec3 d = xform_dir_glm(wto, cam_dir), nd = xform_dir_glm(wto, -cam_dir);
  const GeometryDesc& g = b.geometries[inst.geometry_idx];
  bool fwd = false, bwd = false;
  if (g.kind == kGeoSphere) {
    if (threadIdx.x == 0) {
      SphereHit h;
      SphereExtra x;
      fwd = sphere_intersect(g.radius, o, d, kTMax, &h, &x);
      bwd = sphere_intersect(g.radius, o, nd, kTMax, &h, &x);
    }
  } else {
    for (uint32_t t = threadIdx.x; t < g.tri_count && !(fwd && bwd); t += blockDim.x) {
      const uint32_t* tc = b.tri_corners + 3 * (size_t)(g.tri_offset + t);
      vec3 p[3];
      for (int k = 0; k < 3; ++k) {
        const uint32_t vi = b.pos_idx[g.corner_offset + tc[k]];
        const float* q = b.positions + 3 * (size_t)(g.pos_offset + vi);
        p[k] = vec3(q[0], q[1], q[2]);
      }
      float th;
      if (!fwd) fwd = watertight_hit(p[0], p[1], p[2], o, d, kTMax, &th);
      if (!bwd) bwd = watertight_hit(p[0], p[1], p[2], o, nd, kTMax, &th);
    }
  }
  const int any_fwd = __syncthreads_or(fwd ? 1 : 0);
  const int any_bwd = __syncthreads_or(bwd ? 1 : 0);
  if (threadIdx.x == 0) b.inside[i] = (any_fwd && any_bwd) ? 1 : 0;
}

__global__ void k_camera_stack(TlasBuild b) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  RayTransfer rt{};  // records past record_count stay zero, as on the host
  rt.max_priority_record_index = -1;
  rt.record_count = 0;
  for (uint32_t i = 0; i < b.n; ++i) {
    if (!b.inside[i]) continue;
    if (rt.record_count == kMaxBoundaryRecord) break;
    const Instance inst = b.instances_out[i];
    const bool dm = inst.material_idx < b.material_count && b.materials[inst.material_idx].material_type == kDefaultMtl;
    const float ior = dm ? b.materials[inst.material_idx].default_mtl.ior_n : 1.0f;
    const uint32_t prio = dm ? b.materials[inst.material_idx].default_mtl.ior_priority : 0u;
    BoundaryRecord& r = rt.records[rt.record_count++];
    r.prim_idx = i;
    r.ior = ior;
    r.ior_priority = prio;
    r.vol_idx = inst.inner_volume_idx;
    if (rt.record_count == 1 || prio >= rt.records[rt.max_priority_record_index].ior_priority)
      rt.max_priority_record_index = rt.record_count - 1;
  }
  *b.camera_transfer = rt;
}

}  // namespace

void launch_tlas_rebuild(const TlasBuild& b, uint32_t max_leaf, vec3 cam_pos, vec3 cam_dir, cudaStream_t stream) {
  if (b.n == 0) return;
  const uint32_t blocks = (b.n + 127) / 128;
  k_tlas_items<<<blocks, 128, 0, stream>>>(b);
  k_tlas_binary<<<1, kBinaryThreads, 0, stream>>>(b);
  k_tlas_wide<<<1, 32, 0, stream>>>(b, max_leaf);
  k_tlas_reorder<<<blocks, 128, 0, stream>>>(b);
  k_light_count<<<blocks, 128, 0, stream>>>(b);
  k_light_offsets<<<1, 32, 0, stream>>>(b);
  k_light_fill<<<blocks, 128, 0, stream>>>(b);
  k_light_table<<<1, 32, 0, stream>>>(b);
  k_camera_inside<<<b.n, kCameraThreads, 0, stream>>>(b, cam_pos, cam_dir);
  k_camera_stack<<<1, 32, 0, stream>>>(b);
}

}  // namespace ym
