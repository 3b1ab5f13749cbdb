// Host-side scene preparation: .ymtmp loading, transforms, BVH ordering,
// wide-BVH construction, shape-light table, camera. See scene_host.h.
//
// Built with -ffp-contract=off: the transform matrices, triangle boxes and
// light powers are rounded exactly as the reference computes them, because
// the kernels' intersection results depend on those bits.
#include "scene_host.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <functional>
#include <new>
#include <sstream>
#include <type_traits>
#include <unordered_map>

#include "../../include/ymrt.h"
#include "image_decode.h"
#include "png_decode.h"
#include "sphere.h"

namespace ym {

// ------------------------------------------------------------- matrices ---
// glm 0.9.8 operation order (glm/detail/type_mat4x4.inl, glm/gtc/matrix_transform.inl,
// glm/detail/func_matrix.inl), as used by InitTransformMatrix (src/Transform.h:39-66).

namespace {
struct v4 {
  float x, y, z, w;
};
inline v4 operator*(v4 a, float s) { return {a.x * s, a.y * s, a.z * s, a.w * s}; }
inline v4 operator*(v4 a, v4 b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
inline v4 operator+(v4 a, v4 b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline v4 operator-(v4 a, v4 b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline v4 col(const mat4& m, int c) { return {m.m[c][0], m.m[c][1], m.m[c][2], m.m[c][3]}; }
inline void set_col(mat4& m, int c, v4 v) {
  m.m[c][0] = v.x; m.m[c][1] = v.y; m.m[c][2] = v.z; m.m[c][3] = v.w;
}
inline mat4 identity() {
  mat4 r{};
  for (int i = 0; i < 4; ++i) r.m[i][i] = 1.0f;
  return r;
}
inline float radians(float deg) { return deg * static_cast<float>(0.01745329251994329576923690768489); }

mat4 translate(const mat4& m, vec3 v) {
  mat4 r = m;
  set_col(r, 3, col(m, 0) * v.x + col(m, 1) * v.y + col(m, 2) * v.z + col(m, 3));
  return r;
}
mat4 scale(const mat4& m, vec3 v) {
  mat4 r;
  set_col(r, 0, col(m, 0) * v.x);
  set_col(r, 1, col(m, 1) * v.y);
  set_col(r, 2, col(m, 2) * v.z);
  set_col(r, 3, col(m, 3));
  return r;
}
mat4 rotate(const mat4& m, float angle, vec3 axis_in) {
  const float c = std::cos(angle);
  const float s = std::sin(angle);
  const vec3 axis = normalize(axis_in);
  const vec3 temp = (1.0f - c) * axis;
  float R[3][3];
  R[0][0] = c + temp.x * axis.x;
  R[0][1] = temp.x * axis.y + s * axis.z;
  R[0][2] = temp.x * axis.z - s * axis.y;
  R[1][0] = temp.y * axis.x - s * axis.z;
  R[1][1] = c + temp.y * axis.y;
  R[1][2] = temp.y * axis.z + s * axis.x;
  R[2][0] = temp.z * axis.x + s * axis.y;
  R[2][1] = temp.z * axis.y - s * axis.x;
  R[2][2] = c + temp.z * axis.z;
  mat4 r;
  for (int i = 0; i < 3; ++i) set_col(r, i, col(m, 0) * R[i][0] + col(m, 1) * R[i][1] + col(m, 2) * R[i][2]);
  set_col(r, 3, col(m, 3));
  return r;
}
}  // namespace

mat4 mat4_mul(const mat4& a, const mat4& b) {
  mat4 r;
  for (int j = 0; j < 4; ++j) {
    const v4 bj = col(b, j);
    set_col(r, j, col(a, 0) * bj.x + col(a, 1) * bj.y + col(a, 2) * bj.z + col(a, 3) * bj.w);
  }
  return r;
}

mat4 mat4_inverse(const mat4& M) {
  const float (*m)[4] = M.m;
  const float c00 = m[2][2] * m[3][3] - m[3][2] * m[2][3];
  const float c02 = m[1][2] * m[3][3] - m[3][2] * m[1][3];
  const float c03 = m[1][2] * m[2][3] - m[2][2] * m[1][3];
  const float c04 = m[2][1] * m[3][3] - m[3][1] * m[2][3];
  const float c06 = m[1][1] * m[3][3] - m[3][1] * m[1][3];
  const float c07 = m[1][1] * m[2][3] - m[2][1] * m[1][3];
  const float c08 = m[2][1] * m[3][2] - m[3][1] * m[2][2];
  const float c10 = m[1][1] * m[3][2] - m[3][1] * m[1][2];
  const float c11 = m[1][1] * m[2][2] - m[2][1] * m[1][2];
  const float c12 = m[2][0] * m[3][3] - m[3][0] * m[2][3];
  const float c14 = m[1][0] * m[3][3] - m[3][0] * m[1][3];
  const float c15 = m[1][0] * m[2][3] - m[2][0] * m[1][3];
  const float c16 = m[2][0] * m[3][2] - m[3][0] * m[2][2];
  const float c18 = m[1][0] * m[3][2] - m[3][0] * m[1][2];
  const float c19 = m[1][0] * m[2][2] - m[2][0] * m[1][2];
  const float c20 = m[2][0] * m[3][1] - m[3][0] * m[2][1];
  const float c22 = m[1][0] * m[3][1] - m[3][0] * m[1][1];
  const float c23 = m[1][0] * m[2][1] - m[2][0] * m[1][1];
  const v4 f0{c00, c00, c02, c03}, f1{c04, c04, c06, c07}, f2{c08, c08, c10, c11};
  const v4 f3{c12, c12, c14, c15}, f4{c16, c16, c18, c19}, f5{c20, c20, c22, c23};
  const v4 e0{m[1][0], m[0][0], m[0][0], m[0][0]};
  const v4 e1{m[1][1], m[0][1], m[0][1], m[0][1]};
  const v4 e2{m[1][2], m[0][2], m[0][2], m[0][2]};
  const v4 e3{m[1][3], m[0][3], m[0][3], m[0][3]};
  const v4 i0 = e1 * f0 - e2 * f1 + e3 * f2;
  const v4 i1 = e0 * f0 - e2 * f3 + e3 * f4;
  const v4 i2 = e0 * f1 - e1 * f3 + e3 * f5;
  const v4 i3 = e0 * f2 - e1 * f4 + e2 * f5;
  const v4 sa{+1, -1, +1, -1}, sb{-1, +1, -1, +1};
  mat4 inv;
  set_col(inv, 0, i0 * sa);
  set_col(inv, 1, i1 * sb);
  set_col(inv, 2, i2 * sa);
  set_col(inv, 3, i3 * sb);
  const v4 row0{inv.m[0][0], inv.m[1][0], inv.m[2][0], inv.m[3][0]};
  const v4 d0 = col(M, 0) * row0;
  const float d1 = (d0.x + d0.y) + (d0.z + d0.w);
  const float one_over_det = 1.0f / d1;
  mat4 r;
  for (int c = 0; c < 4; ++c) set_col(r, c, col(inv, c) * one_over_det);
  return r;
}

mat4 compose_transform(vec3 t, vec3 s, vec3 r_deg) {
  const mat4 I = identity();
  mat4 m = translate(I, t);
  m = mat4_mul(m, rotate(I, radians(r_deg.z), vec3(0.0f, 0.0f, 1.0f)));
  m = mat4_mul(m, rotate(I, radians(r_deg.y), vec3(0.0f, 1.0f, 0.0f)));
  m = mat4_mul(m, rotate(I, radians(r_deg.x), vec3(1.0f, 0.0f, 0.0f)));
  m = mat4_mul(m, scale(I, s));
  return m;
}

// --------------------------------------------------- BVH construction ---
// The binary SAH build and the wide collapse are bvh_build.h (shared with the
// device top-level rebuild); these drive them over host vectors.

namespace {

// Builds the binary tree; reorders `items` in place. Returns the nodes in
// build (level by level) order, root at 0.
std::vector<BinNode> build_binary(std::vector<BuildItem>& items) {
  const uint32_t n = (uint32_t)items.size();
  std::vector<BinNode> nodes;
  if (n == 0) return nodes;
  nodes.resize(2 * n - 1);
  std::vector<char> mid_split(2 * n - 1, 0);
  nodes[0].offset = 0;
  nodes[0].count = n;
  uint32_t start = 0, total = 1;
  while (total - start > 0) {
    const uint32_t process = total - start;
    for (uint32_t ni = start; ni < start + process; ++ni) {
      BinNode& node = nodes[ni];
      uint32_t left_count = 0;
      const int kind = split_node(node, items.data() + node.offset, mid_split[ni] != 0, &left_count);
      if (kind == kSplitLeaf) {
        node.left = node.right = kEmpty;
        continue;
      }
      const uint32_t l = total;
      total += 2;
      node.left = l;
      node.right = l + 1;
      nodes[l].offset = node.offset;
      nodes[l].count = left_count;
      nodes[l + 1].offset = node.offset + left_count;
      nodes[l + 1].count = node.count - left_count;
      mid_split[l] = mid_split[l + 1] = kind == kSplitMid ? 1 : 0;
    }
    start += process;
  }
  nodes.resize(total);
  return nodes;
}

// Builds the wide BVH for a binary tree; appends nodes to `out` (root first)
// and the primitive order of the leaves to `prim_order`.
uint32_t build_wide(const std::vector<BinNode>& bin, std::vector<WideNode>* out, std::vector<uint32_t>* prim_order,
                    uint32_t max_leaf) {
  const uint32_t root = (uint32_t)out->size();
  uint32_t n_nodes = root + 1;
  uint32_t n_prims = (uint32_t)prim_order->size();
  out->resize(root + std::max<size_t>(bin.size(), 1));
  prim_order->resize(n_prims + bin[0].count);
  std::vector<uint32_t> stack(2 * (7 * bin.size() + 2));
  build_wide_into(bin.data(), max_leaf, out->data(), root, &n_nodes, prim_order->data(), &n_prims, stack.data());
  out->resize(n_nodes);
  prim_order->resize(n_prims);
  return root;
}

// ------------------------------------------------------------- parsing ---

struct Statement {
  size_t line;
  bool bracket;
  std::string left, right;
};

bool valid_char(char c) {
  return std::isalpha((unsigned char)c) || std::isdigit((unsigned char)c) || c == '=' || c == '<' || c == '>' ||
         c == ',' || c == '.' || c == '"' || c == '(' || c == ')' || c == '#' || c == '_' || c == ';' || c == '[' ||
         c == ']' || c == '+' || c == '-' || c == '\\' || c == '/' || c == ':';
}

bool parse_vec(const std::string& s, vec3* v) {
  if (s.size() < 2 || s.front() != '<' || s.back() != '>') return false;
  int n = 0;
  size_t start = 1;
  for (size_t end = 1; end < s.size(); ++end) {
    if (s[end] != ',' && s[end] != '>') continue;
    if (n >= 3) return false;
    (*v)[n++] = std::stof(s.substr(start, end - start));
    start = end + 1;
  }
  return n == 3;
}
template <typename T, typename F>
bool parse_array(const std::string& s, std::vector<T>* out, F conv) {
  if (s.size() < 2 || s.front() != '[' || s.back() != ']') return false;
  size_t start = 1;
  for (size_t end = 1; end < s.size(); ++end) {
    if (s[end] != ',' && s[end] != ']') continue;
    if (end > start) out->push_back(conv(s.substr(start, end - start)));
    start = end + 1;
  }
  return true;
}
std::string unquote(const std::string& s) {
  if (s.size() >= 2 && s.front() == '"' && s.back() == '"') return s.substr(1, s.size() - 2);
  return s;
}

// The built-in unit cube of a Cube block (GeometryData::InitCube,
// src/GeometryDefines.h:274-520): [-0.5, 0.5]^3 as 12 triangles over 36
// unshared corners, faces in the order -z, +z, -x, +x, -y, +y. Each face lists
// its six corners by the signs of its two in-plane coordinates, in the order
// the reference writes them (the bottom-level build orders triangles from
// these, so the order is part of the format); the normal is the face's, and
// uv = (first in-plane coordinate > 0, second > 0, each flipped as marked).
HostMesh make_unit_cube(const std::string& name) {
  struct Face {
    int axis;           // normal axis
    float sign;         // normal direction
    int a, b;           // in-plane axes
    const char* corners;  // six sign pairs of (a, b)
    bool flip_v;        // v = (b < 0) instead of (b > 0)
  };
  static const Face faces[6] = {
      {2, -1.0f, 0, 1, "--+++-++---+", true},     {2, 1.0f, 0, 1, "--+-++++-+--", false},
      {0, -1.0f, 1, 2, "+++------+++", true},     {0, 1.0f, 1, 2, "++--+---++-+", false},
      {1, -1.0f, 0, 2, "--+-++++-+--", false},    {1, 1.0f, 0, 2, "--+++-++---+", true},
  };
  HostMesh m;
  m.name = name;
  for (const Face& f : faces) {
    for (int k = 0; k < 6; ++k) {
      const bool pa = f.corners[2 * k] == '+', pb = f.corners[2 * k + 1] == '+';
      float p[3], n[3] = {0.0f, 0.0f, 0.0f};
      p[f.axis] = 0.5f * f.sign;
      p[f.a] = pa ? 0.5f : -0.5f;
      p[f.b] = pb ? 0.5f : -0.5f;
      n[f.axis] = f.sign;
      const uint32_t c = (uint32_t)m.pos.size() / 3;
      m.pos.insert(m.pos.end(), p, p + 3);
      m.nrm.insert(m.nrm.end(), n, n + 3);
      m.uv.push_back(pa ? 1.0f : 0.0f);
      m.uv.push_back((pb != f.flip_v) ? 1.0f : 0.0f);
      m.tris.push_back(c);
      m.pos_idx.push_back(c);
      m.nrm_idx.push_back(c);
      m.uv_idx.push_back(c);
    }
  }
  return m;
}

}  // namespace

int load_ymtmp(const std::string& path, HostScene* scene, std::string* error) {
  auto fail = [&](int code, const std::string& msg) {
    if (error) *error = msg;
    return code;
  };
  if (path.size() < 6 || path.substr(path.size() - 6) != ".ymtmp")
    return fail(YMRT_ERR_FORMAT, "scene file must have the .ymtmp extension: " + path);
  std::ifstream f(path, std::ios::binary);
  if (!f) return fail(YMRT_ERR_IO, "cannot open " + path);
  std::stringstream ss;
  ss << f.rdbuf();
  const std::string text = ss.str();

  // Strip comments (to end of line) and characters the format ignores, then
  // split into ';'-terminated statements.
  std::vector<Statement> stmts;
  {
    std::string cur;
    size_t line = 1, stmt_line = 1;
    bool in_comment = false;
    for (char c : text) {
      if (c == '\n') {
        ++line;
        in_comment = false;
        continue;
      }
      if (in_comment) continue;
      if (c == '#') {
        in_comment = true;
        continue;
      }
      if (!valid_char(c)) continue;
      if (cur.empty()) stmt_line = line;
      if (c == ';') {
        if (!cur.empty()) {
          Statement st;
          st.line = stmt_line;
          const size_t eq = cur.find('=');
          if (eq == std::string::npos) {
            st.bracket = true;
            st.left = cur;
          } else {
            st.bracket = false;
            st.left = cur.substr(0, eq);
            st.right = cur.substr(eq + 1);
          }
          stmts.push_back(std::move(st));
        }
        cur.clear();
        continue;
      }
      cur.push_back(c);
    }
  }

  std::unordered_map<std::string, uint32_t> names;
  auto bad = [&](const Statement& st, const std::string& msg) {
    return fail(YMRT_ERR_FORMAT, path + ":" + std::to_string(st.line) + ": " + msg);
  };
  auto lookup = [&](const std::string& v, uint32_t* idx) -> bool {
    auto it = names.find(unquote(v));
    if (it == names.end()) return false;
    *idx = it->second;
    return true;
  };

  size_t i = 0;
  while (i < stmts.size()) {
    const Statement& open = stmts[i];
    if (!open.bracket || open.left.rfind("Begin(", 0) != 0 || open.left.back() != ')')
      return bad(open, "expected Begin(Type)");
    const std::string type = open.left.substr(6, open.left.size() - 7);
    size_t j = i + 1;
    while (j < stmts.size() && !(stmts[j].bracket && stmts[j].left == "End(" + type + ")")) {
      if (stmts[j].bracket) return bad(stmts[j], "unexpected " + stmts[j].left + " inside " + type);
      ++j;
    }
    if (j >= stmts.size()) return bad(open, "missing End(" + type + ")");
    std::string name;
    std::unordered_map<std::string, std::string> attrs;
    for (size_t k = i + 1; k < j; ++k) {
      // is_valid_statement (src/core/YMParser.cpp:680-720): attribute names
      // are letters and '_' only (so NoiseTextureWave's freq_0 .. layer_count_1
      // can never be given in a file)
      for (char c : stmts[k].left)
        if (!(std::isalpha((unsigned char)c) || c == '_')) return bad(stmts[k], "illegal statement " + stmts[k].left);
      if (stmts[k].left == "name") name = unquote(stmts[k].right);
      else attrs[stmts[k].left] = stmts[k].right;
    }
    auto get_f = [&](const char* key, float def) { return attrs.count(key) ? std::stof(attrs[key]) : def; };
    auto get_v = [&](const char* key, vec3 def) {
      vec3 v = def;
      if (attrs.count(key)) parse_vec(attrs[key], &v);
      return v;
    };
    auto get_ref = [&](const char* key, uint32_t* idx) -> int {
      *idx = kEmpty;
      if (!attrs.count(key)) return 0;
      if (!lookup(attrs[key], idx)) return bad(open, std::string("unknown name for ") + key + ": " + attrs[key]);
      return 0;
    };
    if (type != "Camera") {
      if (name.empty()) return bad(open, type + " requires a name");
      if (names.count(name)) return bad(open, "name already declared: " + name);
    }
    int rc = 0;
    if (type == "Camera") {
      scene->cam_from = get_v("from", vec3(0.0f, 0.0f, 10.0f));
      scene->cam_look = get_v("look", vec3(0.0f, 0.0f, 4.0f));
      scene->cam_fov_deg = gmax(get_f("fov", 45.0f), 0.01f);
    } else if (type == "Transform") {
      const vec3 t = get_v("translate", vec3(0.0f));
      const vec3 s = vmax(vec3(0.0001f), get_v("scale", vec3(1.0f)));
      const vec3 r = vclamp(get_v("rotate", vec3(0.0f)), vec3(0.0f), vec3(360.0f));
      uint32_t parent = kEmpty;
      if ((rc = get_ref("parent_transform_index", &parent))) return rc;
      mat4 m = compose_transform(t, s, r);
      if (parent != kEmpty) m = mat4_mul(scene->transforms[parent], m);
      names[name] = (uint32_t)scene->transforms.size();
      scene->transforms.push_back(m);
      scene->i_transforms.push_back(mat4_inverse(m));
      scene->transform_scales.push_back(s);
    } else if (type == "Mesh") {
      HostMesh mesh;
      mesh.name = name;
      auto to_u = [](const std::string& s) { return (uint32_t)std::stoi(s); };
      auto to_f = [](const std::string& s) { return std::stof(s); };
      std::vector<uint32_t> tris;
      if (attrs.count("mesh_triangles")) parse_array(attrs["mesh_triangles"], &tris, to_u);
      if (attrs.count("mesh_position_indices")) parse_array(attrs["mesh_position_indices"], &mesh.pos_idx, to_u);
      if (attrs.count("mesh_positions")) parse_array(attrs["mesh_positions"], &mesh.pos, to_f);
      if (attrs.count("mesh_normal_indices")) parse_array(attrs["mesh_normal_indices"], &mesh.nrm_idx, to_u);
      if (attrs.count("mesh_normals")) parse_array(attrs["mesh_normals"], &mesh.nrm, to_f);
      if (attrs.count("mesh_texcoord_indices")) parse_array(attrs["mesh_texcoord_indices"], &mesh.uv_idx, to_u);
      if (attrs.count("mesh_texcoords")) parse_array(attrs["mesh_texcoords"], &mesh.uv, to_f);
      const size_t nt = tris.size() / 3;
      tris.resize(nt * 3);
      if (nt == 0) return bad(open, "mesh has no triangles");
      if (mesh.pos_idx.size() != nt * 3) return bad(open, "mesh's position indices number is wrong");
      if (mesh.nrm_idx.size() != nt * 3) return bad(open, "mesh's normal indices number is wrong");
      if (!mesh.uv_idx.empty() && mesh.uv_idx.size() != nt * 3) return bad(open, "mesh's texcoord indices number is wrong");
      if (mesh.nrm.empty() || mesh.pos.empty()) return bad(open, "mesh requires position and normal arrays");
      if (mesh.uv_idx.empty() || mesh.uv.empty()) {
        mesh.uv_idx.clear();
        mesh.uv.clear();
      }
      const size_t np = mesh.pos.size() / 3, nn = mesh.nrm.size() / 3, nu = mesh.uv.size() / 2;
      for (size_t k = 0; k < nt * 3; ++k) {
        if (tris[k] >= nt * 3) return bad(open, "triangle corner index out of range");
        if (mesh.pos_idx[k] >= np || mesh.nrm_idx[k] >= nn) return bad(open, "vertex index out of range");
        if (!mesh.uv_idx.empty() && mesh.uv_idx[k] >= nu) return bad(open, "texcoord index out of range");
      }
      mesh.tris = std::move(tris);
      names[name] = (uint32_t)scene->meshes.size();
      scene->meshes.push_back(std::move(mesh));
    } else if (type == "Cube") {
      // CreateCube (src/core/SceneModule.cpp:263-277)
      names[name] = (uint32_t)scene->meshes.size();
      scene->meshes.push_back(make_unit_cube(name));
    } else if (type == "Sphere") {
      // read_sphere_attributes / CreateSphere (src/core/YMParser.cpp:1155-1187,
      // src/core/SceneModule.cpp:278-292)
      HostMesh sphere;
      sphere.name = name;
      sphere.kind = kGeoSphere;
      sphere.radius = attrs.count("radius") ? gmax(0.0001f, std::stof(attrs["radius"])) : 1.0f;
      names[name] = (uint32_t)scene->meshes.size();
      scene->meshes.push_back(std::move(sphere));
    } else if (type == "PrimitiveInstance") {
      Instance inst{};
      uint32_t g, t, m, v;
      if ((rc = get_ref("geometry_index", &g)) || (rc = get_ref("transform_index", &t)) ||
          (rc = get_ref("material_index", &m)) || (rc = get_ref("inner_volume_index", &v)))
        return rc;
      if (g == kEmpty) return bad(open, "primitive instance requires a geometry");
      if (t == kEmpty) return bad(open, "primitive instance requires a transform");
      if (m == kEmpty) return bad(open, "primitive instance requires a material");
      inst.geometry_idx = g;
      inst.transform_idx = t;
      inst.transform_count = 1;
      inst.material_idx = m;
      inst.inner_volume_idx = (int)v;
      inst.treat_as_boundary = attrs.count("treat_as_boundary") && attrs["treat_as_boundary"] == "true";
      inst.unique_index = (uint32_t)scene->instances.size();
      names[name] = inst.unique_index;
      scene->instances.push_back(inst);
    } else if (type == "DefaultMaterial") {
      Material mat;
      std::memset(&mat, 0, sizeof(mat));
      mat.material_type = kDefaultMtl;
      DefaultMtl& d = mat.default_mtl;
      d.diffuse_albedo = vmax(get_v("diffuse_albedo", vec3(0.5f)), vec3(0.0f));
      d.specular_albedo = vmax(get_v("specular_albedo", vec3(1.0f)), vec3(0.0f));
      d.alpha_x = gclamp(get_f("roughness_x", 0.2f), 0.0f, 1.0f);
      d.alpha_y = gclamp(get_f("roughness_y", 0.2f), 0.0f, 1.0f);
      d.ior_n = gmax(0.0001f, get_f("ior_n", 1.3f));
      d.metalness = gclamp(get_f("metalness", 0.0f), 0.0f, 1.0f);
      d.specular_weight = gclamp(get_f("specular_weight", 1.0f), 0.0f, 1.0f);
      d.transmission_weight = gclamp(get_f("transmission_weight", 0.0f), 0.0f, 1.0f);
      d.ior_priority = attrs.count("ior_priority") ? (uint32_t)gmax(0, std::stoi(attrs["ior_priority"])) : 0u;
      d.coat_albedo = vmax(get_v("coat_albedo", vec3(1.0f)), vec3(0.0f));
      d.coat_weight = gclamp(get_f("coat_weight", 0.0f), 0.0f, 1.0f);
      d.coat_thickness = gmax(get_f("coat_thickness", 1.0f), 0.0f);
      d.coat_ior = gmax(get_f("coat_ior", 1.6f), 0.0001f);
      d.coat_roughness_x = gclamp(get_f("coat_roughness_x", 0.2f), 0.0f, 1.0f);
      d.coat_roughness_y = gclamp(get_f("coat_roughness_y", 0.2f), 0.0f, 1.0f);
      const char* tex_keys[] = {"diffuse_albedo_tex", "alpha_x_tex", "specular_albedo_tex", "alpha_y_tex",
                                "specular_weight_tex", "metalness_tex", "transmission_weight_tex",
                                "normal_mapping_tex", "bump_mapping_tex", "coat_albedo_tex", "coat_weight_tex",
                                "coat_thickness_tex", "coat_roughness_x_tex", "coat_roughness_y_tex",
                                "coat_normal_tex"};
      uint32_t* tex_fields[] = {&d.diffuse_albedo_tex, &d.alpha_x_tex, &d.specular_albedo_tex, &d.alpha_y_tex,
                                &d.specular_weight_tex, &d.metalness_tex, &d.transmission_weight_tex,
                                &d.normal_mapping_tex, &d.bump_mapping_tex, &d.coat_albedo_tex, &d.coat_weight_tex,
                                &d.coat_thickness_tex, &d.coat_roughness_x_tex, &d.coat_roughness_y_tex,
                                &d.coat_normal_tex};
      for (int k = 0; k < 15; ++k)
        if ((rc = get_ref(tex_keys[k], tex_fields[k]))) return rc;
      d.coat_normal_tex_type = attrs.count("coat_normal_tex_type") ? (uint32_t)std::stoi(attrs["coat_normal_tex_type"]) : 1u;
      names[name] = (uint32_t)scene->materials.size();
      scene->materials.push_back(mat);
    } else if (type == "LightMaterial") {
      Material mat;
      std::memset(&mat, 0, sizeof(mat));
      mat.material_type = kLightMtl;
      mat.light_mtl.light_color = vmax(get_v("light_color", vec3(1.0f)), vec3(0.0f));
      mat.light_mtl.intensity = gmax(get_f("intensity", 1.0f), 0.0f);
      names[name] = (uint32_t)scene->materials.size();
      scene->materials.push_back(mat);
    } else if (type == "ConstantTextureFloat" || type == "ConstantTextureRgb" || type == "CheckerBoardTexture" ||
               type == "NoiseTexture" || type == "NoiseTextureFBM" || type == "NoiseTextureTurbulence" ||
               type == "NoiseTextureMarble" || type == "NoiseTextureWood" || type == "NoiseTexturePolkaDot" ||
               type == "NoiseTextureWave") {
      // read_*_texture_attributes (src/core/YMParser.cpp:1560-2118): the
      // readers' defaults and clamps. Attributes a reader has no case for
      // are dropped (the fBm, turbulence and marble readers have none for
      // "lacunarity", so theirs stays 2).
      Texture tex;
      std::memset(&tex, 0, sizeof(tex));
      tex.child[0] = tex.child[1] = kEmpty;
      auto get_i = [&](const char* k, int def) { return attrs.count(k) ? std::stoi(attrs[k]) : def; };
      auto get_b = [&](const char* k, bool def) { return attrs.count(k) ? attrs[k] == "true" : def; };
      if (type == "ConstantTextureFloat") {
        tex.type = kTexConstFloat;
        tex.value = get_f("value", 0.0f);
      } else if (type == "ConstantTextureRgb") {
        tex.type = kTexConstRgb;
        tex.color = get_v("color", vec3(0.0f));
      } else {
        if ((rc = get_ref("texture_black_idx", &tex.child[0])) || (rc = get_ref("texture_white_idx", &tex.child[1])))
          return rc;
        if (tex.child[0] == kEmpty || tex.child[1] == kEmpty) return bad(open, type + " requires black and white inputs");
        if (type == "CheckerBoardTexture") {
          tex.type = kTexChecker;
          tex.frequency = gmax(get_f("frequency", 4.0f), 0.001f);
        } else if (type == "NoiseTexture") {
          tex.type = kTexNoise;
          tex.frequency = gmax(get_f("frequency", 1.0f), 0.001f);
          tex.flags = get_b("normalized", true) ? kTexNormalized : 0u;
        } else if (type == "NoiseTextureFBM" || type == "NoiseTextureTurbulence") {
          tex.type = type == "NoiseTextureFBM" ? kTexFbm : kTexTurbulence;
          tex.frequency = gmax(0.001f, get_f("frequency", 16.0f));
          tex.lacunarity = 2.0f;
          tex.gain = get_f("gain", 0.5f);
          tex.layer_count = get_i("layer_count", 4);
          tex.amplitude = get_f("amplitude", 1.0f);
          tex.offset = get_f("offset", 0.0f);
        } else if (type == "NoiseTextureMarble") {
          tex.type = kTexMarble;
          tex.frequency = get_f("frequency", 16.0f);
          tex.lacunarity = 2.0f;
          tex.gain = get_f("gain", 0.5f);
          tex.layer_count = get_i("layer_count", 4);
          tex.variation = get_f("variation", 10.0f);
          tex.flags = (get_b("x_turb", true) ? kTexTurbX : 0u) | (get_b("y_turb", true) ? kTexTurbY : 0u) |
                      (get_b("z_turb", true) ? kTexTurbZ : 0u);
        } else if (type == "NoiseTextureWood") {
          tex.type = kTexWood;
          tex.frequency = gmax(0.001f, get_f("frequency", 2.0f));
          tex.variation = get_f("variation", 10.0f);
        } else if (type == "NoiseTexturePolkaDot") {
          tex.type = kTexPolkaDot;
          tex.frequency = get_f("frequency", 8.0f);
          tex.radius = get_f("radius", 0.35f);
        } else {
          // the reader's defaults (its numbered attributes are illegal statements)
          tex.type = kTexWave;
          tex.frequency = 0.1f;
          tex.lacunarity = 2.0f;
          tex.gain = 0.5f;
          tex.layer_count = 2;
          tex.frequency1 = 2.0f;
          tex.lacunarity1 = 2.0f;
          tex.gain1 = 0.5f;
          tex.layer_count1 = 4;
        }
      }
      names[name] = (uint32_t)scene->textures.size();
      scene->textures.push_back(tex);
    } else if (type == "ImageTexture") {
      // read_image_texture_attributes (src/core/YMParser.cpp:1509-1557): the
      // file lies in the folder texture_<stem>_<extension> beside the scene
      // file; a file that does not load leaves the name without a node
      // (CreateImageTexture returns EMPTY, src/core/SceneModule.cpp:665-670).
      const std::string file = attrs.count("texture_file_name") ? unquote(attrs["texture_file_name"]) : "";
      const std::string cs = attrs.count("color_space") ? unquote(attrs["color_space"]) : "";
      if (file.empty()) return bad(open, "image texture requires a file name");
      const size_t slash = path.find_last_of('/');
      const std::string dir = slash == std::string::npos ? "" : path.substr(0, slash + 1);
      const std::string fname = slash == std::string::npos ? path : path.substr(slash + 1);
      const size_t dot = fname.find_last_of('.');
      const std::string folder = dir + "texture_" + fname.substr(0, dot) + "_" + fname.substr(dot + 1);
      Texture tex;
      std::vector<float> pixels;
      std::string why;
      const int irc = load_image_texture(folder + "/" + file, (cs.empty() || cs == "SRGB") ? kImageSrgb : kImageLinear,
                                         &tex, &pixels, &why);
      if (irc == YMRT_ERR_UNSUPPORTED) return fail(irc, why);
      if (irc != YMRT_OK) {
        names[name] = kEmpty;
      } else {
        names[name] = (uint32_t)scene->textures.size();
        scene->images[(uint32_t)scene->textures.size()] = std::move(pixels);
        scene->textures.push_back(tex);
      }
    } else if (type == "DistantLight") {
      DistantLight dl{};
      dl.light_color = vmax(get_v("light_color", vec3(1.0f)), vec3(0.0f));
      if ((rc = get_ref("transform_index", &dl.transform_idx))) return rc;
      if (dl.transform_idx == kEmpty) return bad(open, "distant light requires a transform");
      dl.intensity = gmax(get_f("intensity", 1.0f), 0.0f);
      dl.theta_max = gmax(0.0f, get_f("theta_max", 5.0f));
      dl.cos_theta_max = std::cos(dl.theta_max * static_cast<float>(0.01745329251994329576923690768489));
      names[name] = (uint32_t)scene->distant_lights.size();
      scene->distant_lights.push_back(dl);
    } else if (type == "Volume") {
      Volume vol{};
      uint32_t t, tex;
      if ((rc = get_ref("transform_index", &t)) || (rc = get_ref("density_texture_index", &tex))) return rc;
      if (t == kEmpty) return bad(open, "volume requires a transform");
      vol.transform_idx = t;
      vol.sigma_t = vmax(vec3(0.0f), get_v("sigma_t", vec3(0.05f)));
      vol.albedo = vmax(vec3(0.0f), get_v("albedo", vec3(1.0f)));
      vol.g = gclamp(get_f("g", 0.0f), 0.0f, 1.0f);
      vol.density_texture_idx = (int)tex;
      names[name] = (uint32_t)scene->volumes.size();
      scene->volumes.push_back(vol);
    } else {
      return bad(open, "unknown block type " + type);
    }
    i = j + 1;
  }
  for (const Instance& inst : scene->instances) {
    if (inst.geometry_idx >= scene->meshes.size() || inst.transform_idx >= scene->transforms.size() ||
        inst.material_idx >= scene->materials.size())
      return fail(YMRT_ERR_FORMAT, "instance refers to an asset of the wrong type");
    if (inst.inner_volume_idx != -1 && (uint32_t)inst.inner_volume_idx >= scene->volumes.size())
      return fail(YMRT_ERR_FORMAT, "instance refers to an unknown volume");
  }
  std::string why;
  if (const int rc = check_textures(*scene, YMRT_ERR_FORMAT, &why)) return fail(rc, why);
  return YMRT_OK;
}

// ------------------------------------------------------- texture nodes ---

static_assert(sizeof(ymrt_texture_desc) == kTextureWords * 4, "ymrt_texture_desc is 20 words");

float srgb_to_linear(float s) {
  return s > 0.04045 ? (float)std::pow((s + 0.055) / 1.055, (double)2.4f) : (s / 12.92f);
}

int load_image_texture(const std::string& path, uint32_t color_space, Texture* t, std::vector<float>* pixels,
                       std::string* error) {
  std::vector<uint8_t> bytes;
  {
    std::ifstream f(path, std::ios::binary);
    if (!f) {
      if (error) *error = "cannot open " + path;
      return YMRT_ERR_IO;
    }
    bytes.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
  }
  PngImage img;
  try {
    const ImageFormat fmt = sniff_image(bytes.data(), bytes.size());
    if (fmt == ImageFormat::kPng) {
      if (!decode_png(bytes.data(), bytes.size(), &img, error)) {
        if (error) *error = path + ": " + *error;
        return YMRT_ERR_IO;
      }
    } else {
      Image8 im;
      bool unsupported = false, ok = false;
      std::string msg;
      if (fmt == ImageFormat::kJpeg) ok = decode_jpeg(bytes.data(), bytes.size(), &im, &msg, &unsupported);
      else if (fmt == ImageFormat::kHdr) ok = decode_hdr(bytes.data(), bytes.size(), &im, &msg);
      else if (fmt == ImageFormat::kBmp) ok = decode_bmp(bytes.data(), bytes.size(), &im, &msg, &unsupported);
      else if (fmt == ImageFormat::kTga) ok = decode_tga(bytes.data(), bytes.size(), &im, &msg, &unsupported);
      else {
        unsupported = true;
        msg = "unknown image format";
      }
      if (!ok) {
        if (error) *error = path + ": " + msg;
        return unsupported ? YMRT_ERR_UNSUPPORTED : YMRT_ERR_IO;
      }
      img.width = im.width;
      img.height = im.height;
      img.channels = im.channels;
      img.sixteen = false;
      img.samples.assign(im.samples.begin(), im.samples.end());
    }
  } catch (const std::bad_alloc&) {
    if (error) *error = path + ": out of memory decoding the image";
    return YMRT_ERR_IO;
  }
  std::memset(t, 0, sizeof(*t));
  t->type = kTexImage;
  t->child[0] = t->child[1] = kEmpty;
  t->width = img.width;
  t->height = img.height;
  t->channels = img.channels;
  t->wrap = kWrapRepeat;
  t->scale_u = t->scale_v = 1.0f;
  t->offset_u = t->offset_v = 0.0f;
  t->color_space = color_space;
  const float inv = img.sixteen ? 1.0f / 65535.0f : 1.0f / 255.0f;
  pixels->resize(img.samples.size());
  for (size_t i = 0; i < img.samples.size(); ++i) {
    const float v = float((int)img.samples[i]) * inv;
    (*pixels)[i] = color_space == kImageSrgb ? srgb_to_linear(v) : v;
  }
  return YMRT_OK;
}

void texture_words(const Texture& t, uint32_t r[kTextureWords]) {
  for (int k = 0; k < kTextureWords; ++k) r[k] = 0;
  r[0] = t.type;
  r[1] = t.child[0];
  r[2] = t.child[1];
  r[3] = f2u(t.value);
  r[4] = f2u(t.color.x);
  r[5] = f2u(t.color.y);
  r[6] = f2u(t.color.z);
  r[7] = f2u(t.frequency);
  r[8] = f2u(t.lacunarity);
  r[9] = f2u(t.gain);
  r[10] = (uint32_t)t.layer_count;
  r[11] = f2u(t.amplitude);
  r[12] = f2u(t.offset);
  r[13] = f2u(t.variation);
  r[14] = f2u(t.radius);
  r[15] = t.flags;
  r[16] = f2u(t.frequency1);
  r[17] = f2u(t.lacunarity1);
  r[18] = f2u(t.gain1);
  r[19] = (uint32_t)t.layer_count1;
  if (t.type == kTexGrid) {  // the lattice is not part of the node's words
    r[1] = r[2] = kEmpty;
  }
  if (t.type == kTexImage) {
    for (int k = 3; k < kTextureWords; ++k) r[k] = 0;
    r[3] = (uint32_t)t.width;
    r[4] = (uint32_t)t.height;
    r[5] = (uint32_t)t.channels;
    r[6] = (uint32_t)t.wrap;
    r[7] = f2u(t.scale_u);
    r[8] = f2u(t.scale_v);
    r[9] = f2u(t.offset_u);
    r[10] = f2u(t.offset_v);
    r[15] = t.color_space;
  }
}

int texture_from_desc(const ymrt_texture_desc& d, Texture* t, std::string* error) {
  std::memset(t, 0, sizeof(*t));
  t->type = d.type;
  t->child[0] = t->child[1] = kEmpty;
  if (d.type == kTexConstFloat) {
    t->value = d.value;
    return YMRT_OK;
  }
  if (d.type == kTexConstRgb) {
    t->color = vec3(d.color[0], d.color[1], d.color[2]);
    return YMRT_OK;
  }
  if (d.type == kTexImage) {  // words: width, height, channels, wrap, scale u/v, offset u/v, colour space
    uint32_t w[kTextureWords];
    std::memcpy(w, &d, sizeof(w));
    t->width = (int)w[3];
    t->height = (int)w[4];
    t->channels = (int)w[5];
    t->wrap = (int)w[6];
    std::memcpy(&t->scale_u, &w[7], 4);
    std::memcpy(&t->scale_v, &w[8], 4);
    std::memcpy(&t->offset_u, &w[9], 4);
    std::memcpy(&t->offset_v, &w[10], 4);
    t->color_space = w[15];
    if (t->width < 1 || t->height < 1 || t->channels < 1 || t->channels > 4 ||
        (t->wrap != kWrapRepeat && t->wrap != kWrapClamp)) {
      if (error) *error = "image node: size, channel count (1-4) or wrap mode (0 repeat, 1 clamp) out of range";
      return YMRT_ERR_INVALID;
    }
    return YMRT_OK;  // pixels: ymrt_host_scene_set_image
  }
  if (d.type < kTexChecker || d.type > kTexWave) {
    if (error) *error = "node type " + std::to_string(d.type) + " is not supported (constant and solid nodes are)";
    return YMRT_ERR_UNSUPPORTED;
  }
  t->child[0] = d.black;
  t->child[1] = d.white;
  t->frequency = d.frequency;
  t->lacunarity = d.lacunarity;
  t->gain = d.gain;
  t->layer_count = d.layer_count;
  t->amplitude = d.amplitude;
  t->offset = d.offset;
  t->variation = d.variation;
  t->radius = d.radius;
  t->flags = d.flags & (kTexNormalized | kTexTurbX | kTexTurbY | kTexTurbZ);
  t->frequency1 = d.frequency1;
  t->lacunarity1 = d.lacunarity1;
  t->gain1 = d.gain1;
  t->layer_count1 = d.layer_count1;
  return YMRT_OK;
}

int check_textures(const HostScene& s, int code, std::string* error) {
  const size_t n = s.textures.size();
  auto fail = [&](const std::string& msg) {
    if (error) *error = msg;
    return code;
  };
  for (size_t k = 0; k < n; ++k) {
    const Texture& t = s.textures[k];
    if (t.type < kTexChecker || t.type > kTexWave) continue;
    if (t.child[0] >= n || t.child[1] >= n)
      return fail("texture " + std::to_string(k) + " requires black and white inputs");
  }
  // longest path (in nodes) from each node; 0 = not yet visited, -1 = on the path
  std::vector<int> depth(n, 0);
  std::function<int(uint32_t)> walk = [&](uint32_t k) -> int {
    if (depth[k] > 0) return depth[k];
    if (depth[k] < 0) return -1;
    depth[k] = -1;
    int d = 1;
    const Texture& t = s.textures[k];
    if (t.type >= kTexChecker && t.type <= kTexWave)
      for (int c = 0; c < 2; ++c) {
        const int dc = walk(t.child[c]);
        if (dc < 0) return -1;
        d = std::max(d, dc + 1);
      }
    depth[k] = d;
    return d;
  };
  // the graphs the renderer evaluates: from material references and media densities
  auto root = [&](uint32_t k) -> int {
    const int d = walk(k);
    if (d < 0) return fail("the texture graph has a cycle through node " + std::to_string(k));
    if (d > kTextureStack)
      return fail("texture " + std::to_string(k) + " is " + std::to_string(d) + " nodes deep (at most " +
                  std::to_string(kTextureStack) + " are evaluated)");
    return YMRT_OK;
  };
  for (size_t m = 0; m < s.materials.size(); ++m) {
    const Material& mat = s.materials[m];
    if (mat.material_type != kDefaultMtl) continue;
    const DefaultMtl& d = mat.default_mtl;
    const uint32_t refs[] = {d.diffuse_albedo_tex, d.alpha_x_tex, d.specular_albedo_tex, d.alpha_y_tex,
                             d.specular_weight_tex, d.metalness_tex, d.transmission_weight_tex, d.normal_mapping_tex,
                             d.bump_mapping_tex, d.coat_albedo_tex, d.coat_weight_tex, d.coat_thickness_tex,
                             d.coat_roughness_x_tex, d.coat_roughness_y_tex};
    for (uint32_t r : refs) {
      if (r == kEmpty) continue;
      if (r >= n) return fail("material " + std::to_string(m) + " refers to an unknown texture");
      if (const int rc = root(r)) return rc;
    }
  }
  for (const Volume& v : s.volumes)
    if (v.density_texture_idx >= 0 && (size_t)v.density_texture_idx < n)
      if (const int rc = root((uint32_t)v.density_texture_idx)) return rc;
  return YMRT_OK;
}

// ------------------------------------------------------- from arrays ---

int load_arrays(const ymrt_scene_desc* d, HostScene* scene, std::string* error) {
  auto fail = [&](int code, const std::string& msg) {
    if (error) *error = msg;
    return code;
  };
  if (!d) return fail(YMRT_ERR_INVALID, "null scene description");
  // transforms
  if (d->transform_count > 0 && !d->transforms) return fail(YMRT_ERR_INVALID, "transforms missing");
  for (uint32_t t = 0; t < d->transform_count; ++t) {
    mat4 m, mi;
    std::memcpy(&m.m[0][0], d->transforms + 16 * (size_t)t, sizeof(float) * 16);
    if (d->inverse_transforms) std::memcpy(&mi.m[0][0], d->inverse_transforms + 16 * (size_t)t, sizeof(float) * 16);
    else mi = mat4_inverse(m);
    scene->transforms.push_back(m);
    scene->i_transforms.push_back(mi);
    const float* sc = d->transform_scales ? d->transform_scales + 3 * (size_t)t : nullptr;
    scene->transform_scales.push_back(sc ? vmax(vec3(0.0001f), vec3(sc[0], sc[1], sc[2])) : vec3(1.0f));
  }
  // geometries
  if (d->geometry_count > 0 && !d->geometries) return fail(YMRT_ERR_INVALID, "geometries missing");
  for (uint32_t g = 0; g < d->geometry_count; ++g) {
    const ymrt_mesh_desc& md = d->geometries[g];
    HostMesh m;
    m.name = "geometry " + std::to_string(g);
    if (md.sphere_radius > 0.0f) {
      m.kind = kGeoSphere;
      m.radius = gmax(0.0001f, md.sphere_radius);
      scene->meshes.push_back(std::move(m));
      continue;
    }
    const size_t nt = md.triangle_count, nc = 3 * nt;
    if (nt == 0 || !md.triangles || !md.position_indices || !md.positions || !md.normal_indices || !md.normals)
      return fail(YMRT_ERR_INVALID, m.name + ": a mesh needs triangles, positions and normals with their indices");
    m.tris.assign(md.triangles, md.triangles + nc);
    m.pos_idx.assign(md.position_indices, md.position_indices + nc);
    m.nrm_idx.assign(md.normal_indices, md.normal_indices + nc);
    m.pos.assign(md.positions, md.positions + 3 * (size_t)md.position_count);
    m.nrm.assign(md.normals, md.normals + 3 * (size_t)md.normal_count);
    if (md.texcoord_indices && md.texcoords && md.texcoord_count > 0) {
      m.uv_idx.assign(md.texcoord_indices, md.texcoord_indices + nc);
      m.uv.assign(md.texcoords, md.texcoords + 2 * (size_t)md.texcoord_count);
    }
    for (size_t k = 0; k < nc; ++k) {
      if (m.tris[k] >= nc) return fail(YMRT_ERR_INVALID, m.name + ": triangle corner index out of range");
      if (m.pos_idx[k] >= md.position_count || m.nrm_idx[k] >= md.normal_count)
        return fail(YMRT_ERR_INVALID, m.name + ": vertex index out of range");
      if (!m.uv_idx.empty() && m.uv_idx[k] >= md.texcoord_count)
        return fail(YMRT_ERR_INVALID, m.name + ": texcoord index out of range");
    }
    scene->meshes.push_back(std::move(m));
  }
  // textures
  if (d->texture_count > 0 && !d->textures) return fail(YMRT_ERR_INVALID, "textures missing");
  for (uint32_t k = 0; k < d->texture_count; ++k) {
    Texture tex;
    std::string why;
    const int rc = texture_from_desc(d->textures[k], &tex, &why);
    if (rc) return fail(rc, "texture " + std::to_string(k) + ": " + why);
    scene->textures.push_back(tex);
  }
  // materials, volumes, distant lights: the reference's own layouts
  auto take = [&](const void* src, uint32_t n, auto* out) -> bool {
    using T = typename std::remove_pointer<decltype(out)>::type::value_type;
    if (n > 0 && !src) return false;
    out->resize(n);
    if (n) std::memcpy(out->data(), src, sizeof(T) * n);
    return true;
  };
  if (!take(d->materials, d->material_count, &scene->materials)) return fail(YMRT_ERR_INVALID, "materials missing");
  if (!take(d->volumes, d->volume_count, &scene->volumes)) return fail(YMRT_ERR_INVALID, "volumes missing");
  if (!take(d->distant_lights, d->distant_light_count, &scene->distant_lights))
    return fail(YMRT_ERR_INVALID, "distant lights missing");
  if (!take(d->instances, d->instance_count, &scene->instances)) return fail(YMRT_ERR_INVALID, "instances missing");
  for (const Material& m : scene->materials)
    if (m.material_type != kDefaultMtl && m.material_type != kLightMtl)
      return fail(YMRT_ERR_UNSUPPORTED, "material type " + std::to_string(m.material_type) + " is not supported");
  for (const Volume& v : scene->volumes) {
    if (v.transform_idx >= scene->transforms.size()) return fail(YMRT_ERR_INVALID, "volume refers to an unknown transform");
    if (v.density_texture_idx != -1 && (uint32_t)v.density_texture_idx >= scene->textures.size())
      return fail(YMRT_ERR_INVALID, "volume refers to an unknown texture");
  }
  for (const DistantLight& l : scene->distant_lights)
    if (l.transform_idx >= scene->transforms.size())
      return fail(YMRT_ERR_INVALID, "distant light refers to an unknown transform");
  for (const Instance& inst : scene->instances) {
    if (inst.geometry_idx >= scene->meshes.size() || inst.transform_idx >= scene->transforms.size() ||
        inst.material_idx >= scene->materials.size())
      return fail(YMRT_ERR_INVALID, "instance refers to an unknown asset");
    if (inst.inner_volume_idx != -1 && (uint32_t)inst.inner_volume_idx >= scene->volumes.size())
      return fail(YMRT_ERR_INVALID, "instance refers to an unknown volume");
  }
  {
    std::string why;
    const int rc = check_textures(*scene, YMRT_ERR_INVALID, &why);
    if (rc) return fail(rc, why);
  }
  scene->cam_from = vec3(d->camera_from[0], d->camera_from[1], d->camera_from[2]);
  scene->cam_look = vec3(d->camera_look[0], d->camera_look[1], d->camera_look[2]);
  scene->cam_fov_deg = gmax(d->camera_fov_deg, 0.01f);
  return YMRT_OK;
}

// ---------------------------------------------------------- preparation ---

namespace {

}  // namespace

vec3 camera_media_ray(const CameraDesc& cam) {
  const float height = 2.0f * cam.tan_half_fov;
  const float width = height * cam.aspect_ratio;
  const vec3 dir = -cam.w + (0.5f - 0.5f) * width * cam.u + (0.5f - 0.5f) * height * cam.v;
  return normalize(dir);
}

namespace {

// Camera::InitCameraRayTransfer (src/Camera.cpp:15-78): instances the
// camera sits inside (a ray from the camera hits them both forwards and
// backwards) are pushed on the camera's ray-transfer stack.
void init_camera_transfer(HostScene* s) {
  RayTransfer& rt = s->camera.transfer;
  rt = RayTransfer{};  // records past record_count are zero
  rt.max_priority_record_index = -1;
  rt.record_count = 0;
  const CameraDesc& cam = s->camera;
  const vec3 dir = camera_media_ray(cam);
  auto hits_geometry = [&](uint32_t inst_idx, vec3 o_world, vec3 d_world) {
    const Instance& inst = s->instances[inst_idx];
    const mat4& wto = s->i_transforms[inst.transform_idx];
    const vec3 o = xform_point_glm(wto, o_world), d = xform_dir_glm(wto, d_world);
    const HostMesh& m = s->meshes[inst.geometry_idx];
    if (m.kind == kGeoSphere) {
      SphereHit h;
      SphereExtra x;
      return sphere_intersect(m.radius, o, d, kTMax, &h, &x);
    }
    for (size_t t = 0; t < m.tris.size() / 3; ++t) {
      vec3 p[3];
      for (int k = 0; k < 3; ++k) {
        const uint32_t vi = m.pos_idx[m.tris[3 * t + k]];
        p[k] = vec3(m.pos[3 * vi], m.pos[3 * vi + 1], m.pos[3 * vi + 2]);
      }
      float th;
      if (watertight_hit(p[0], p[1], p[2], o, d, kTMax, &th)) return true;
    }
    return false;
  };
  std::vector<uint32_t> inside;
  for (uint32_t i = 0; i < s->instances.size(); ++i)
    if (hits_geometry(i, cam.position, dir) && hits_geometry(i, cam.position, -dir)) inside.push_back(i);
  for (uint32_t i : inside) {
    if (rt.record_count == kMaxBoundaryRecord) break;
    const Instance& inst = s->instances[i];
    const bool dm = inst.material_idx < s->materials.size() && s->materials[inst.material_idx].material_type == kDefaultMtl;
    const float ior = dm ? s->materials[inst.material_idx].default_mtl.ior_n : 1.0f;
    const uint32_t prio = dm ? s->materials[inst.material_idx].default_mtl.ior_priority : 0u;
    BoundaryRecord& r = rt.records[rt.record_count++];
    r.prim_idx = i;
    r.ior = ior;
    r.ior_priority = prio;
    r.vol_idx = inst.inner_volume_idx;
    if (rt.record_count == 1 || prio >= rt.records[rt.max_priority_record_index].ior_priority)
      rt.max_priority_record_index = rt.record_count - 1;
  }
}

}  // namespace

// The top level: instance world boxes, the reference's binary SAH build of
// them (which fixes the instance order), the wide top-level BVH, and the
// shape-light table in the new instance order. prepare_scene runs it after
// the meshes are built; set_transforms runs it again after an edit, starting
// from the current instance order as the reference's editor does
// (GuiModule::UpdateScene, src/core/GuiModule.cpp:123-139).
int build_top_level(HostScene* s, std::string* error) {
  const uint32_t ni = (uint32_t)s->instances.size();
  if (ni == 0) {
    if (error) *error = "scene has no instances";
    return YMRT_ERR_INVALID;
  }
  std::vector<BuildItem> items(ni);
  for (uint32_t i = 0; i < ni; ++i) {
    const Instance& inst = s->instances[i];
    items[i].box = box_transform(s->meshes[inst.geometry_idx].root_box, s->transforms[inst.transform_idx]);
    items[i].center = box_center(items[i].box);
    items[i].idx = i;
  }
  std::vector<BinNode> tbin = build_binary(items);
  std::vector<Instance> reordered(ni);
  std::vector<uint32_t> file_index(ni);
  const bool ordered_before = s->instance_file_index.size() == ni;
  for (uint32_t i = 0; i < ni; ++i) {
    reordered[i] = s->instances[items[i].idx];
    file_index[i] = ordered_before ? s->instance_file_index[items[i].idx] : items[i].idx;
  }
  s->instances.swap(reordered);
  s->instance_file_index.swap(file_index);
  s->tlas_nodes.clear();
  s->tlas_prims.clear();
  build_wide(tbin, &s->tlas_nodes, &s->tlas_prims, s->max_leaf_prims);
  s->triangle_count_instanced = 0;
  for (const Instance& inst : s->instances) s->triangle_count_instanced += s->meshes[inst.geometry_idx].tris.size() / 3;

  // Shape lights: SceneModule::LoadShapeLight (src/core/SceneModule.cpp:1203-1304).
  s->shape_lights.clear();
  s->shape_light_table.clear();
  for (uint32_t pi = 0; pi < ni; ++pi) {
    const Instance& inst = s->instances[pi];
    const Material& mat = s->materials[inst.material_idx];
    if (mat.material_type != kLightMtl) continue;
    const mat4& otw = s->transforms[inst.transform_idx];
    const vec3 c = mat.light_mtl.light_color;
    const float irradiance = (c.x + c.y + c.z) * mat.light_mtl.intensity * kPi;
    const HostMesh& m = s->meshes[inst.geometry_idx];
    if (m.kind == kGeoSphere) {
      // the transform's own scale stretches the sphere into an ellipsoid;
      // its area is approximated as (4/3) pi (ab + bc + ca)
      const vec3 sc = s->transform_scales[inst.transform_idx];
      const float a = m.radius * sc.x, b = m.radius * sc.y, c3 = m.radius * sc.z;
      const float area = (4.0f / 3.0f) * kPi * (a * b + b * c3 + c3 * a);
      s->shape_lights.push_back(ShapeLight{pi, kEmpty, irradiance * area, area});
      continue;
    }
    for (uint32_t t = 0; t < m.tris.size() / 3; ++t) {
      vec3 p[3];
      for (int k = 0; k < 3; ++k) {
        const uint32_t vi = m.pos_idx[m.tris[3 * t + k]];
        p[k] = transform_position(otw, vec3(m.pos[3 * vi], m.pos[3 * vi + 1], m.pos[3 * vi + 2]));
      }
      const float area = length(cross(p[1] - p[0], p[2] - p[0]));
      s->shape_lights.push_back(ShapeLight{pi, t, irradiance * area, 0.5f * area});
    }
  }
  {
    float total = 0.0f;
    s->shape_light_table.resize(s->shape_lights.size());
    for (size_t i = 0; i < s->shape_lights.size(); ++i) {
      total += s->shape_lights[i].power;
      s->shape_light_table[i] = total;
    }
    const float rcp = safe_rcp(total);
    for (float& v : s->shape_light_table) v = total == 0.0f ? 0.0f : (v * rcp);
  }

  return YMRT_OK;
}

int set_transforms(HostScene* s, uint32_t first, uint32_t count, const float* object_to_world,
                   const float* world_to_object, const float* scales, std::string* error) {
  if (!object_to_world || first > s->transforms.size() || count > s->transforms.size() - first) {
    if (error) *error = "transform range out of bounds";
    return YMRT_ERR_INVALID;
  }
  for (uint32_t k = 0; k < count; ++k) {
    mat4 m, mi;
    std::memcpy(&m, object_to_world + 16 * (size_t)k, sizeof(mat4));
    if (world_to_object) std::memcpy(&mi, world_to_object + 16 * (size_t)k, sizeof(mat4));
    else mi = mat4_inverse(m);
    s->transforms[first + k] = m;
    s->i_transforms[first + k] = mi;
    if (scales) {
      const float* sc = scales + 3 * (size_t)k;
      s->transform_scales[first + k] = vmax(vec3(0.0001f), vec3(sc[0], sc[1], sc[2]));
    }
  }
  const int rc = build_top_level(s, error);
  if (rc != YMRT_OK) return rc;
  init_camera_transfer(s);
  return YMRT_OK;
}

int prepare_scene(HostScene* s, int width, int height, std::string* error) {
  if (width <= 0 || height <= 0) {
    if (error) *error = "image size must be positive";
    return YMRT_ERR_INVALID;
  }
  s->width = width;
  s->height = height;

  // Bottom level: per mesh, the reference's build order, then a wide BVH.
  s->geo_desc.clear();
  s->blas_nodes.clear();
  s->wtris.clear();
  s->tri_corners.clear();
  s->all_pos_idx.clear(); s->all_nrm_idx.clear(); s->all_uv_idx.clear();
  s->all_pos.clear(); s->all_nrm.clear(); s->all_uv.clear();
  for (HostMesh& m : s->meshes) {
    if (m.kind == kGeoSphere) {
      // GetSphereObjectBound (src/GeometryUtilities.h:19-25); no triangles
      BBox b;
      b.pmin = vec3(-m.radius);
      b.pmax = vec3(m.radius);
      m.root_box = bound_fix(b);
      GeometryDesc gd{};
      gd.tri_offset = (uint32_t)(s->tri_corners.size() / 3);
      gd.corner_offset = (uint32_t)s->all_pos_idx.size();
      gd.pos_offset = (uint32_t)(s->all_pos.size() / 3);
      gd.nrm_offset = (uint32_t)(s->all_nrm.size() / 3);
      gd.uv_offset = -1;
      gd.wtri_offset = (uint32_t)(s->wtris.size() / 3);
      gd.bbox_min = m.root_box.pmin;
      gd.bbox_max = m.root_box.pmax;
      gd.kind = kGeoSphere;
      gd.radius = m.radius;
      s->geo_desc.push_back(gd);
      continue;
    }
    const uint32_t nt = (uint32_t)(m.tris.size() / 3);
    auto P = [&](uint32_t corner) {
      const uint32_t vi = m.pos_idx[corner];
      return vec3(m.pos[3 * vi], m.pos[3 * vi + 1], m.pos[3 * vi + 2]);
    };
    std::vector<BuildItem> items(nt);
    for (uint32_t t = 0; t < nt; ++t) {
      const vec3 p0 = P(m.tris[3 * t]), p1 = P(m.tris[3 * t + 1]), p2 = P(m.tris[3 * t + 2]);
      BBox b;
      b = box_extend(b, p0);
      b = box_extend(b, p1);
      b = box_extend(b, p2);
      items[t].box = bound_fix(b);
      items[t].center = (p0 + p1 + p2) / 3.f;
      items[t].idx = t;
    }
    std::vector<BinNode> bin = build_binary(items);
    std::vector<uint32_t> reordered(nt * 3);
    for (uint32_t t = 0; t < nt; ++t)
      for (int k = 0; k < 3; ++k) reordered[3 * t + k] = m.tris[3 * items[t].idx + k];
    m.tris.swap(reordered);
    m.root_box = bin[0].box;

    GeometryDesc gd{};
    gd.tri_offset = (uint32_t)(s->tri_corners.size() / 3);
    gd.tri_count = nt;
    gd.corner_offset = (uint32_t)s->all_pos_idx.size();
    gd.pos_offset = (uint32_t)(s->all_pos.size() / 3);
    gd.nrm_offset = (uint32_t)(s->all_nrm.size() / 3);
    gd.uv_offset = m.uv.empty() ? -1 : (int32_t)(s->all_uv.size() / 2);
    gd.bbox_min = m.root_box.pmin;
    gd.bbox_max = m.root_box.pmax;
    gd.kind = kGeoMesh;
    s->tri_corners.insert(s->tri_corners.end(), m.tris.begin(), m.tris.end());
    s->all_pos_idx.insert(s->all_pos_idx.end(), m.pos_idx.begin(), m.pos_idx.end());
    s->all_nrm_idx.insert(s->all_nrm_idx.end(), m.nrm_idx.begin(), m.nrm_idx.end());
    if (!m.uv.empty()) s->all_uv_idx.insert(s->all_uv_idx.end(), m.uv_idx.begin(), m.uv_idx.end());
    else s->all_uv_idx.resize(s->all_pos_idx.size(), 0);
    s->all_pos.insert(s->all_pos.end(), m.pos.begin(), m.pos.end());
    s->all_nrm.insert(s->all_nrm.end(), m.nrm.begin(), m.nrm.end());
    s->all_uv.insert(s->all_uv.end(), m.uv.begin(), m.uv.end());

    std::vector<uint32_t> order;
    gd.node_offset = build_wide(bin, &s->blas_nodes, &order, s->max_leaf_prims);
    // the wide builder numbered nodes relative to the whole array already;
    // prim_base values are relative to this mesh's triangle block.
    gd.wtri_offset = (uint32_t)(s->wtris.size() / 3);
    for (uint32_t pos : order) {
      // `pos` is a position in the reordered triangle array == triangle id
      const vec3 p0 = P(m.tris[3 * pos]), p1 = P(m.tris[3 * pos + 1]), p2 = P(m.tris[3 * pos + 2]);
      s->wtris.push_back(float4{p0.x, p0.y, p0.z, u2f(pos)});
      s->wtris.push_back(float4{p1.x, p1.y, p1.z, 0.0f});
      s->wtris.push_back(float4{p2.x, p2.y, p2.z, 0.0f});
    }
    s->geo_desc.push_back(gd);
  }

  int rc = build_top_level(s, error);
  if (rc != YMRT_OK) return rc;

  // Camera: SceneParser -> Camera::SetFov/SetPosition/SetDir (src/Camera.h:32,
  // 235-238, 301-311), then the rendering camera's aspect ratio.
  {
    CameraDesc& cam = s->camera;
    const float fov = s->cam_fov_deg * static_cast<float>(0.01745329251994329576923690768489);
    cam.tan_half_fov = std::tan(0.5f * fov);
    cam.position = s->cam_from;
    vec3 w = s->cam_from - s->cam_look;
    w = w * safe_rcp(length(w));
    const vec3 up(0.0f, 1.0f, 0.0f);
    double mu[3], mv[3];
    mu[0] = (double)up.y * (double)w.z - (double)up.z * (double)w.y;
    mu[1] = -((double)up.x * (double)w.z - (double)up.z * (double)w.x);
    mu[2] = (double)up.x * (double)w.y - (double)up.y * (double)w.x;
    const vec3 u = vec3((float)mu[0], (float)mu[1], (float)mu[2]) *
                   safe_rcp((float)std::sqrt(mu[0] * mu[0] + mu[1] * mu[1] + mu[2] * mu[2]));
    mv[0] = (double)w.y * (double)u.z - (double)w.z * (double)u.y;
    mv[1] = -((double)w.x * (double)u.z - (double)w.z * (double)u.x);
    mv[2] = (double)w.x * (double)u.y - (double)w.y * (double)u.x;
    const vec3 v = vec3((float)mv[0], (float)mv[1], (float)mv[2]) *
                   safe_rcp((float)std::sqrt(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]));
    cam.w = w;
    cam.u = u;
    cam.v = v;
    cam.aspect_ratio = float(width) / float(height);
    init_camera_transfer(s);
  }
  return YMRT_OK;
}

}  // namespace ym
