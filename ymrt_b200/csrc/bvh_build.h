// BVH construction steps shared by the host scene preparation (scene_host.cpp)
// and the device top-level rebuild (tlas_build.cu): the same source, compiled
// by g++ with -ffp-contract=off and by nvcc with -fmad=false, so that both
// produce the same trees bit for bit.
//
// The binary builder is the reference's top-down SAH builder
// (src/BottomBVH.cpp:34-166, src/BottomBVH.h:40-190, src/TopBVH.cpp:34-198):
// 24 bins per axis, a median split (heap selection) when SAH declines or
// partitioning fails, one primitive per leaf, nodes numbered level by level.
// Its partitioning and selection steps are reproduced step for step, because
// the resulting primitive order defines the triangle and instance indices
// (and the shape-light order) that every result is reported in. The wide
// collapse and the quantised 8-wide node format are this project's.
#pragma once

#include <cstdint>
#include <cmath>

#include "ymrt_scene.h"

namespace ym {

struct BBox {
  vec3 pmax{kFloatMin, kFloatMin, kFloatMin};
  vec3 pmin{kFloatMax, kFloatMax, kFloatMax};
};

template <typename T>
YM_HD void bvh_swap(T& a, T& b) {
  const T t = a;
  a = b;
  b = t;
}

// BBox3 helpers, src/BoundingBox.h:10-140.
YM_HD BBox box_extend(const BBox& b, vec3 p) {
  BBox r;
  r.pmin = vec3(gmin(b.pmin.x, p.x), gmin(b.pmin.y, p.y), gmin(b.pmin.z, p.z));
  r.pmax = vec3(gmax(b.pmax.x, p.x), gmax(b.pmax.y, p.y), gmax(b.pmax.z, p.z));
  return r;
}
YM_HD BBox box_union(const BBox& a, const BBox& b) {
  BBox r;
  r.pmin = vec3(gmin(a.pmin.x, b.pmin.x), gmin(a.pmin.y, b.pmin.y), gmin(a.pmin.z, b.pmin.z));
  r.pmax = vec3(gmax(a.pmax.x, b.pmax.x), gmax(a.pmax.y, b.pmax.y), gmax(a.pmax.z, b.pmax.z));
  return r;
}
YM_HD BBox bound_fix(const BBox& in) {
  const float eps = 0.0005f;
  BBox b = in;
  for (int i = 0; i < 3; ++i) {
    if (b.pmax[i] < b.pmin[i]) {
      const float t = b.pmax[i];
      b.pmax[i] = b.pmin[i];
      b.pmin[i] = t;
    }
    if (fabsf(b.pmax[i] - b.pmin[i]) < 2.0f * eps) {
      b.pmax[i] += eps;
      b.pmin[i] -= eps;
    }
  }
  return b;
}
YM_HD float box_area(const BBox& b) {
  const vec3 e = b.pmax - b.pmin;
  return 2.f * (e.x * e.y + e.y * e.z + e.x * e.z);
}
YM_HD int box_longest_axis(const BBox& b) {
  const vec3 d = b.pmax - b.pmin;
  int a = 0;
  if (d[1] > d[a]) a = 1;
  if (d[2] > d[a]) a = 2;
  return a;
}
YM_HD vec3 box_center(const BBox& b) { return (b.pmax + b.pmin) * 0.5f; }
// The world box of an instance: its mesh's root box through the transform
// (BBox3 transformed corner by corner, then fixed for flat extents).
YM_HD BBox box_transform(const BBox& b, const mat4& M) {
  BBox r;
  for (int i = 0; i < 8; ++i) {
    const vec3 c((i & 1) ? b.pmax.x : b.pmin.x, (i & 2) ? b.pmax.y : b.pmin.y, (i & 4) ? b.pmax.z : b.pmin.z);
    r = box_extend(r, xform_point_glm(M, c));
  }
  return bound_fix(r);
}

// Watertight ray/triangle test, the reference's IntersectTri
// (src/ShadingUtilities.cuh:54-134), for the camera's media set-up on the host
// and on the device: whether the ray hits within [TMIN, tmax].
YM_HD bool watertight_hit(vec3 p0, vec3 p1, vec3 p2, vec3 o, vec3 d, float tmax, float* t_out) {
  p0 = p0 - o;
  p1 = p1 - o;
  p2 = p2 - o;
  const int kz = max_dimension(vabs(d));
  int kx = kz + 1;
  if (kx == 3) kx = 0;
  int ky = kx + 1;
  if (ky == 3) ky = 0;
  const vec3 dd(d[kx], d[ky], d[kz]);
  p0 = vec3(p0[kx], p0[ky], p0[kz]);
  p1 = vec3(p1[kx], p1[ky], p1[kz]);
  p2 = vec3(p2[kx], p2[ky], p2[kz]);
  const float sx = -dd.x / dd.z, sy = -dd.y / dd.z, sz = 1.f / dd.z;
  p0.x += sx * p0.z;
  p0.y += sy * p0.z;
  p1.x += sx * p1.z;
  p1.y += sy * p1.z;
  p2.x += sx * p2.z;
  p2.y += sy * p2.z;
  const float e0 = p1.x * p2.y - p1.y * p2.x;
  const float e1 = p2.x * p0.y - p2.y * p0.x;
  const float e2 = p0.x * p1.y - p0.y * p1.x;
  if ((e0 < 0 || e1 < 0 || e2 < 0) && (e0 > 0 || e1 > 0 || e2 > 0)) return false;
  const float den = e0 + e1 + e2;
  if (den == 0) return false;
  p0.z *= sz;
  p1.z *= sz;
  p2.z *= sz;
  const float inv = 1.0f / den;
  float t = e0 * p0.z + e1 * p1.z + e2 * p2.z;
  t *= inv;
  if (t < kTMin || t > tmax) return false;
  *t_out = t;
  return true;
}

// ------------------------------------------------------- binary builder ---

struct BuildItem {
  BBox box;
  vec3 center;
  uint32_t idx;
};

struct BinNode {
  BBox box;
  uint32_t left, right;   // children (kEmpty: a leaf)
  uint32_t offset, count; // the node's items
};

YM_HD void heap_down(BuildItem* t, uint32_t i, uint32_t right, int axis) {
  for (;;) {
    const uint32_t lc = 2 * i + 1, rc = 2 * i + 2;
    if (!(lc <= right)) return;
    uint32_t target = lc;
    if (rc <= right && t[rc].center[axis] > t[lc].center[axis]) target = rc;
    if (t[i].center[axis] > t[target].center[axis]) return;
    bvh_swap(t[i], t[target]);
    i = target;
  }
}

// Heap selection of the median along `axis` (the reference's FindMidElement).
YM_HD uint32_t find_mid_element(BuildItem* t, uint32_t count, int axis) {
  const uint32_t n_th = (count - 1) / 2;
  uint32_t n_pass = count - n_th;
  for (uint32_t i = count / 2 - 1; i != kEmpty; --i) heap_down(t, i, count - 1, axis);
  for (uint32_t i = count - 1; i > 0 && n_pass > 0; --i, --n_pass) {
    bvh_swap(t[0], t[i]);
    heap_down(t, 0, i - 1, axis);
  }
  return n_th;
}

YM_HD uint32_t partition_items(BuildItem* t, uint32_t count, float pivot, int axis) {
  uint32_t left = 0, right = count - 1;
  while (left <= right && right != kEmpty) {
    if (t[left].center[axis] <= pivot) ++left;
    else bvh_swap(t[left], t[right--]);
  }
  return right;
}

constexpr int kSahBins = 24;

YM_HD bool eval_sah(const BuildItem* prims, uint32_t count, const BBox& cb, float parent_cost, float* split_pos,
                    int* split_axis) {
  int best_axis = -1;
  float best_pos = 0.0f, best_cost = 1E36f;
  struct Bin {
    uint32_t count;
    BBox box;
  };
  bool valid[3] = {true, true, true};
  vec3 ext = cb.pmax - cb.pmin;
  for (int a = 0; a < 3; ++a)
    if (ext[a] < kFloatEps) {
      valid[a] = false;
      ext[a] = kFloatEps;
    }
  Bin bins[kSahBins][3];
  for (int b = 0; b < kSahBins; ++b)
    for (int a = 0; a < 3; ++a) {
      bins[b][a].count = 0;
      bins[b][a].box = BBox();
    }
  const vec3 i_ext = vec3(1.0f) / ext;
  const vec3 bin_len = vmax(cb.pmax - cb.pmin, vec3(0.0f)) / float(kSahBins);
  for (uint32_t i = 0; i < count; ++i) {
    const vec3 ndc = (prims[i].center - cb.pmin) * i_ext;
    for (int a = 0; a < 3; ++a) {
      const int b = gmax(gmin((int)(ndc[a] * kSahBins), kSahBins - 1), 0);
      bins[b][a].count++;
      bins[b][a].box = box_union(bins[b][a].box, prims[i].box);
    }
  }
  for (int a = 0; a < 3; ++a) {
    if (!valid[a]) continue;
    float la[kSahBins - 1], ra[kSahBins - 1];
    uint32_t lc[kSahBins - 1], rc[kSahBins - 1];
    BBox lb, rb;
    uint32_t lcount = 0, rcount = 0;
    for (int i = 0; i < kSahBins - 1; ++i) {
      lcount += bins[i][a].count;
      lb = box_union(lb, bins[i][a].box);
      lc[i] = lcount;
      la[i] = box_area(lb);
      rcount += bins[kSahBins - 1 - i][a].count;
      rb = box_union(rb, bins[kSahBins - 1 - i][a].box);
      rc[kSahBins - 2 - i] = rcount;
      ra[kSahBins - 2 - i] = box_area(rb);
    }
    for (int i = 0; i < kSahBins - 1; ++i) {
      const float cost = lc[i] * la[i] + rc[i] * ra[i];
      if (cost <= 0.0f) continue;
      if (cost < best_cost) {
        best_cost = cost;
        best_axis = a;
        best_pos = cb.pmin[a] + float(i + 1) * bin_len[a];
      }
    }
  }
  if (best_axis == -1 || best_cost >= parent_cost) return false;
  *split_axis = best_axis;
  *split_pos = best_pos;
  return true;
}

// How one node of the level-by-level build divides.
constexpr int kSplitLeaf = 0;  // one item: a leaf
constexpr int kSplitSah = 1;   // SAH split: the children go on with SAH
constexpr int kSplitMid = 2;   // median split: the children split at their medians too

// Bounds the node's items (node.box), decides how it divides and reorders
// its items in place (partition or median selection); *left_count receives
// the left child's item count. mid_split: the node is the child of a median
// split. The caller numbers the children.
YM_HD int split_node(BinNode& node, BuildItem* its, bool mid_split, uint32_t* left_count) {
  BBox nb, cb;
  for (uint32_t i = 0; i < node.count; ++i) {
    nb = box_union(nb, its[i].box);
    cb = box_extend(cb, its[i].center);
  }
  node.box = nb;
  if (node.count <= 1) return kSplitLeaf;
  auto mid = [&]() {
    *left_count = find_mid_element(its, node.count, box_longest_axis(nb)) + 1;
    return kSplitMid;
  };
  if (mid_split) return mid();
  const float parent_cost = node.count * box_area(node.box);
  int axis = 0;
  float pos = 0.0f;
  if (!eval_sah(its, node.count, cb, parent_cost, &pos, &axis)) return mid();
  const uint32_t split = partition_items(its, node.count, pos, axis);
  if (split == kEmpty || split == node.count - 1) return mid();
  *left_count = split + 1;
  return kSplitSah;
}

// ------------------------------------------------------- wide collapse ---

constexpr int kWide = 8;

// The node grid exponent: the smallest e (stored + 127) with
// extent / 2^e <= 250 (margin for outward rounding), exact.
YM_HD uint8_t quant_exp(float extent) {
  int e = -126;
  if (extent > 0.0f) {
    int ex = 0;
    const float m = frexpf(extent / 250.0f, &ex);  // extent / 250 = m * 2^ex, m in [0.5, 1)
    e = (m == 0.5f) ? ex - 1 : ex;
  }
  e = gmax(-126, gmin(127, e));
  return (uint8_t)(e + 127);
}
YM_HD float exp_scale(uint8_t be) { return u2f((uint32_t)be << 23); }

// Grows a box by a relative margin so float rounding in the slab test can
// never reject a ray that touches the exact box.
YM_HD BBox pad_box(const BBox& b) {
  BBox r = b;
  for (int a = 0; a < 3; ++a) {
    const float m = 2e-6f * gmax(fabsf(b.pmin[a]), fabsf(b.pmax[a])) + 1e-30f;
    r.pmin[a] = b.pmin[a] - m;
    r.pmax[a] = b.pmax[a] + m;
  }
  return r;
}

// Fills wide node out[slot] from binary node `root`: its children are the
// binary descendants reached by opening, largest surface area first, any
// internal node of more than max_leaf items until there are 8. Leaf children
// (a binary leaf, or a subtree of at most max_leaf items) append their item
// positions to prim_order; internal children get consecutive wide slots from
// *n_nodes on and are returned in `internal` (binary nodes, child order).
// Returns the number of internal children.
YM_HD int collapse_node(const BinNode* B, uint32_t root, uint32_t max_leaf, WideNode* out, uint32_t slot,
                        uint32_t* n_nodes, uint32_t* prim_order, uint32_t* n_prims, uint32_t internal[kWide]) {
  uint32_t cand[kWide];
  int n_cand = 0;
  if (B[root].left == kEmpty) {
    cand[n_cand++] = root;  // single-leaf tree
  } else {
    cand[n_cand++] = B[root].left;
    cand[n_cand++] = B[root].right;
    while (n_cand < kWide) {
      int best = -1;
      float best_area = -1.0f;
      for (int i = 0; i < n_cand; ++i) {
        const BinNode& c = B[cand[i]];
        if (c.left == kEmpty || c.count <= max_leaf) continue;
        const float a = box_area(c.box);
        if (a > best_area) {
          best_area = a;
          best = i;
        }
      }
      if (best < 0) break;
      const uint32_t e = cand[best];
      for (int i = n_cand; i > best + 1; --i) cand[i] = cand[i - 1];
      cand[best] = B[e].left;
      cand[best + 1] = B[e].right;
      ++n_cand;
    }
  }
  WideNode node;
  uint8_t* raw = reinterpret_cast<uint8_t*>(&node);
  for (int k = 0; k < (int)sizeof(WideNode); ++k) raw[k] = 0;
  BBox all, boxes[kWide];
  for (int i = 0; i < n_cand; ++i) {
    boxes[i] = pad_box(B[cand[i]].box);
    all = box_union(all, boxes[i]);
  }
  node.ox = all.pmin.x;
  node.oy = all.pmin.y;
  node.oz = all.pmin.z;
  node.ex = quant_exp(all.pmax.x - all.pmin.x);
  node.ey = quant_exp(all.pmax.y - all.pmin.y);
  node.ez = quant_exp(all.pmax.z - all.pmin.z);
  node.prim_base = *n_prims;
  int n_internal = 0;
  for (int i = 0; i < n_cand; ++i) {
    const BinNode& c = B[cand[i]];
    if (c.left == kEmpty || c.count <= max_leaf) {
      const uint32_t off = *n_prims - node.prim_base;
      for (uint32_t k = 0; k < c.count; ++k) prim_order[(*n_prims)++] = c.offset + k;
      node.meta[i] = (uint8_t)((c.count << 5) | off);
    } else {
      node.imask |= (uint8_t)(1u << i);
      node.meta[i] = (uint8_t)n_internal;
      internal[n_internal++] = cand[i];
    }
  }
  // Quantise every child box on the node grid origin + q * 2^e, decoding
  // exactly as the kernel does (one fmaf) and rounding outwards; widen the
  // grid step if a bound does not fit in 8 bits.
  const float org[3] = {node.ox, node.oy, node.oz};
  uint8_t* exps[3] = {&node.ex, &node.ey, &node.ez};
  uint8_t* qlo[3] = {node.qlo_x, node.qlo_y, node.qlo_z};
  uint8_t* qhi[3] = {node.qhi_x, node.qhi_y, node.qhi_z};
  for (int a = 0; a < 3; ++a) {
    for (;;) {
      const float sc = exp_scale(*exps[a]);
      bool ok = true;
      for (int i = 0; i < n_cand && ok; ++i) {
        int lo = (int)floorf((boxes[i].pmin[a] - org[a]) / sc);
        int hi = (int)ceilf((boxes[i].pmax[a] - org[a]) / sc);
        lo = gmax(0, gmin(255, lo));
        hi = gmax(0, gmin(255, hi));
        while (lo > 0 && fmaf((float)lo, sc, org[a]) > boxes[i].pmin[a]) --lo;
        while (hi < 255 && fmaf((float)hi, sc, org[a]) < boxes[i].pmax[a]) ++hi;
        if (fmaf((float)lo, sc, org[a]) > boxes[i].pmin[a] || fmaf((float)hi, sc, org[a]) < boxes[i].pmax[a])
          ok = false;
        qlo[a][i] = (uint8_t)lo;
        qhi[a][i] = (uint8_t)hi;
      }
      if (ok || *exps[a] >= 254) break;
      ++*exps[a];
    }
  }
  node.child_base = *n_nodes;
  *n_nodes += (uint32_t)n_internal;
  out[slot] = node;
  return n_internal;
}

// The whole collapse of a binary tree (root 0) into out[root_slot] and the
// slots after *n_nodes, depth first in child order (the node numbering and
// the prim_order sequence follow that order). stack: room for 2 words per
// pending node (at most 7 per level of the binary tree plus one).
YM_HD void build_wide_into(const BinNode* B, uint32_t max_leaf, WideNode* out, uint32_t root_slot, uint32_t* n_nodes,
                           uint32_t* prim_order, uint32_t* n_prims, uint32_t* stack) {
  int sp = 0;
  stack[sp++] = 0;
  stack[sp++] = root_slot;
  while (sp > 0) {
    const uint32_t slot = stack[--sp];
    const uint32_t bin = stack[--sp];
    uint32_t internal[kWide];
    const uint32_t base = *n_nodes;
    const int n = collapse_node(B, bin, max_leaf, out, slot, n_nodes, prim_order, n_prims, internal);
    for (int k = n - 1; k >= 0; --k) {  // the first child's subtree first
      stack[sp++] = internal[k];
      stack[sp++] = base + (uint32_t)k;
    }
  }
}

}  // namespace ym
