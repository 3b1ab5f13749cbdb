"""Build recipe for the oracle: the YMRT reference compiled for the host.

TEST INFRASTRUCTURE ONLY. Compiles the reference's own sources where they lie
(``<reference>/src``) with g++ into ``oracle/_ref/libymrt_ref.so``
(git-ignored, but shipped with the repository snapshot to GPU machines). The
reference's CMake build is not used: the hot-path sources compile directly
once a few MSVC/CUDA-runtime stand-ins are provided (``oracle/shims``,
``oracle/ref_stubs.cpp``). ``oracle/ref_harness.cpp`` is this project's
headless driver around the reference's stage kernels.

The reference root is taken from ``YMRT_REFERENCE_ROOT`` or ``--reference``.

Floating point: ``-ffp-contract=off`` (no fused multiply-add), SSE2 scalar
float, IEEE division and square root; glm is forced to its scalar code path.
That is the same arithmetic the ymrt_b200 kernels use (they are built with
``-fmad=false``), so both evaluate each reference expression in source order.

Sampler argument order: where the reference passes several ``random()`` calls
as arguments of one call (e.g. ``src/Shading.cu:325, 370``), C++ leaves their
evaluation order unspecified. With ``arg_order="ltr"`` the build writes a copy
of ``src/Shading.cu`` into ``oracle/_ref/gen/`` in which those argument lists
are drawn left to right (the order nvcc's device front end uses); with
``"native"`` the file is compiled unchanged (g++ on x86-64 evaluates them
right to left). Nothing else in the file is changed.

The same build-time copy also counts the stage kernels' closest-hit and
occlusion queries, and reads the maximum-priority record of the nested-media
stack directly where the reference reads it through a dangling reference
(see ``_COUNTERS``).

Usage: ``python oracle/build_ref.py --reference <checkout> [--arg-order ltr|native] [--force] [--gpu]``.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# The reference checkout this recipe compiles: YMRT_REFERENCE_ROOT, or
# --reference on the command line (set_reference). Without it only the
# prebuilt libraries under oracle/_ref are used.
REF = os.environ.get("YMRT_REFERENCE_ROOT", "")


def set_reference(root: str) -> None:
    global REF
    REF = root


def reference_root() -> str:
    """The reference checkout: REF, else the one the prebuilt oracle was last
    built from (recorded in oracle/_ref/reference_root), else ""."""
    if REF:
        return REF
    try:
        with open(os.path.join(OUT, "reference_root")) as f:
            return f.read().strip()
    except OSError:
        return ""


def _record_root() -> None:
    with open(os.path.join(OUT, "reference_root"), "w") as f:
        f.write(REF)
OUT = os.path.join(HERE, "_ref")
LIB = os.path.join(OUT, "libymrt_ref.so")

HOST_SOURCES = [
    "src/BottomBVH.cpp",
    "src/TopBVH.cpp",
    "src/Camera.cpp",
    "src/core/SceneModule.cpp",
    "src/core/YMParser.cpp",
    "src/FileIO.cpp",
    "src/LowDiscrepancy.cpp",
]

CXXFLAGS = [
    "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-DNDEBUG", "-DGLM_FORCE_PURE",
    "-fPIC", "-w", "-pthread",
]


def _includes():
    return [
        "-include", os.path.join(HERE, "shims", "ymrt_ref_prelude.h"),
        "-I" + os.path.join(HERE, "shims"),
        "-I" + REF, "-I" + os.path.join(REF, "src"), "-I" + os.path.join(REF, "src", "core"),
        "-I" + os.path.join(REF, "external", "glm"),
        "-I" + os.path.join(REF, "external", "glad", "include"),
        "-I" + os.path.join(REF, "external", "image_lib"),
        "-I" + os.path.join(REF, "external", "assimp-5.1.0", "include"),
        "-I/usr/local/cuda/include",
    ]


# The library binds its own symbols (-Bsymbolic): its CUDA-runtime stand-ins
# must win over a real libcudart that the host process (e.g. torch) may have
# loaded globally.

# Call arguments made of several sampler draws, e.g. "random(), random()" or
# "ray_sampler.Random1D(), ray_sampler.Random1D(), ray_sampler.Random1D()".
_DRAW = r"(random\(\)|[A-Za-z_][A-Za-z_0-9]*\.Random1D\(\))"
_RUN = re.compile(_DRAW + r"(?:\s*,\s*" + _DRAW + r")+")


def _sequence_draws(text: str) -> tuple[str, int]:
    """Rewrites each run of sampler draws inside an argument list so that the
    draws happen left to right whatever order the compiler evaluates
    arguments in: the first-evaluated draw of the run fills a small buffer in
    source order, each argument then reads its own slot."""
    count = 0

    def repl(m: re.Match) -> str:
        nonlocal count
        parts = [p.strip() for p in m.group(0).split(",")]
        n = len(parts)
        if n < 2 or len(set(parts)) != 1:
            return m.group(0)
        count += 1
        draw = parts[0]
        fn = "[&]()->float{ return " + draw + "; }"
        return ", ".join(f"ymrt_oracle_draw_in_order({fn}, {n}, {k})" for k in range(n))

    return _RUN.sub(repl, text), count


_HELPER = r'''
// ---- inserted by oracle/build_ref.py: left-to-right sampler draws ----
#include <cstddef>
namespace {
struct YmrtOracleDrawBuffer { float v[8]; int pending = 0; };
thread_local YmrtOracleDrawBuffer ymrt_oracle_draw_buffer;
template <typename Draw>
inline float ymrt_oracle_draw_in_order(Draw draw, int n, int k) {
  YmrtOracleDrawBuffer& b = ymrt_oracle_draw_buffer;
  if (b.pending == 0) { for (int i = 0; i < n; ++i) b.v[i] = draw(); b.pending = n; }
  --b.pending;
  return b.v[k];
}
}  // namespace
// ---- end of insertion ----
'''


# Ray counting: the build-time copy routes the stage kernels' calls of the
# reference's closest-hit and occlusion queries (TraceRay,
# BVHTraverseShadow) through counting wrappers, so the reference's Mrays/s is
# computed from the same query counts as ymrt_b200's.
_COUNTERS = r'''
// ---- inserted by oracle/build_ref.py: query counters ----
#include <atomic>
std::atomic<unsigned long long> ymrt_oracle_trace_queries{0};
std::atomic<unsigned long long> ymrt_oracle_shadow_queries{0};
template <typename... A>
inline bool ymrt_oracle_counted_trace(A&&... a) {
  ymrt_oracle_trace_queries.fetch_add(1, std::memory_order_relaxed);
  return YMRT::TraceRay(std::forward<A>(a)...);
}
template <typename... A>
inline bool ymrt_oracle_counted_shadow(A&&... a) {
  ymrt_oracle_shadow_queries.fetch_add(1, std::memory_order_relaxed);
  return YMRT::BVHTraverseShadow(std::forward<A>(a)...);
}
// RayTransfer::GetMaxPriorityRecord (src/Ray.h:148-151) returns a reference
// bound to a temporary copy of the selected record (its conditional operator
// has a prvalue branch); g++ compiles reading through that dangling reference
// into a null dereference. The priority the expression copies is read here
// directly, which is the value the device build reads.
inline uint32_t ymrt_oracle_max_priority(const YMRT::RayTransfer& rt) {
  return rt.max_priority_record_index != -1 ? rt.boundary_records[rt.max_priority_record_index].ior_priority
                                            : YMRT::BoundaryRecord().ior_priority;
}
// ---- end of insertion ----
'''


# Path-vertex recording, for parity diagnostics (the host parity build only:
# the timing build stays as the reference wrote it, and the device builds
# read the same vertices from the hit queue the trace stage writes, in
# oracle/ref_gpu_harness.cu, without touching the reference's kernels).
# After the trace stage's closest hit and volume free flight
# (src/Shading.cu:1829-1854), the vertex of each watched pixel's path (the
# ray, what it hit, the throughput and the light received so far) is written
# to a record array, so that a path can be compared vertex by vertex with
# ymrt_b200's (ymrt_debug_record_paths, the same 24-word layout).
_RECORD_FILL = r'''
struct YmrtOracleVertex {
  uint32_t pixel, depth, flags, inst, tri;
  float t, o[3], d[3], bary[3], tp[3], light[3];
  uint32_t path, pad[2];
};
template <typename R, typename H, typename V>
YMRT_ORACLE_FN void ymrt_oracle_fill(YmrtOracleVertex& v, uint32_t pixel, int depth, int sample, const R& ray, bool hit,
                                     const H& rec, const V& tp, const V& light) {
  v.pixel = pixel;
  v.depth = (uint32_t)depth;
  v.flags = (hit ? 1u : 0u) | (rec.volume_hit ? 2u : 0u) | (rec.hit_back ? 4u : 0u);
  v.inst = rec.hit_instance_idx;
  v.tri = rec.hit_triangle_idx;
  v.t = rec.hit_t;
  for (int c = 0; c < 3; ++c) {
    v.o[c] = ray.origin[c];
    v.d[c] = ray.direction[c];
    v.bary[c] = rec.hit_barycentric[c];
    v.tp[c] = tp[c];
    v.light[c] = light[c];
  }
  v.path = (uint32_t)sample;
  v.pad[0] = v.pad[1] = 0u;
}
'''
_RECORD_HOST = ("\n// ---- inserted by oracle/build_ref.py: path-vertex recording ----\n#define YMRT_ORACLE_RECORDING 1\n"
                "#define YMRT_ORACLE_FN inline\n" +
                _RECORD_FILL + r'''
struct YmrtOracleRecorder {
  const uint32_t* watch = nullptr;
  uint32_t n_pixels = 0;
  YmrtOracleVertex* out = nullptr;
  uint32_t capacity = 0;
  std::atomic<uint32_t> count{0};
};
inline YmrtOracleRecorder& ymrt_oracle_recorder() {
  static YmrtOracleRecorder r;
  return r;
}
template <typename R, typename H, typename V>
inline void ymrt_oracle_record(uint32_t pixel, int depth, int sample, const R& ray, bool hit, const H& rec, const V& tp,
                               const V& light) {
  YmrtOracleRecorder& q = ymrt_oracle_recorder();
  if (!q.out || pixel >= q.n_pixels || !((q.watch[pixel >> 5] >> (pixel & 31u)) & 1u)) return;
  const uint32_t k = q.count.fetch_add(1u, std::memory_order_relaxed);
  if (k < q.capacity) ymrt_oracle_fill(q.out[k], pixel, depth, sample, ray, hit, rec, tp, light);
}
// ---- end of insertion ----
''')
# Radiance-event recording, for the double-precision albedo adjoint
# (oracle/adjoint64.py; parity builds only). Every term a path adds to its
# received light in the stage kernels (src/Shading.cu:1857 background,
# 2084/2088 next-event estimation at a volume vertex, 2183 a light seen
# before any scattering, 2218/2237 next-event estimation at a surface
# vertex) is recorded with its pixel, sample, depth, kind and (surface
# next-event estimation) the vertex's material, and so is every surface
# scattering event (src/Shading.cu:2265, after the BSDF weight multiplies the
# throughput) with its material. Values are stored in double whatever the
# build's precision. Nothing the stages compute changes: the hooks return
# their argument.
_EVENT_HOST = r'''
// ---- inserted by oracle/build_ref.py: radiance-event recording ----
#define YMRT_ORACLE_EVENTS 1
struct YmrtOracleEvent {
  uint32_t pixel, sample, depth;
  int32_t kind, material;  // kind: 0 surface scattering, 1 surface NEE, 2 volume NEE, 3 background, 4 light seen
  uint32_t pad;
  double value[3];
};
struct YmrtOracleEvents {
  YmrtOracleEvent* out = nullptr;
  uint32_t capacity = 0;
  const uint32_t* watch = nullptr;  // one bit per pixel (null: every pixel)
  uint32_t n_pixels = 0;
  std::atomic<uint32_t> count{0};
};
inline YmrtOracleEvents& ymrt_oracle_events() {
  static YmrtOracleEvents e;
  return e;
}
inline void ymrt_oracle_event(int kind, uint32_t pixel, int sample, int depth, int material, double r, double g,
                              double b) {
  YmrtOracleEvents& q = ymrt_oracle_events();
  if (!q.out) return;
  if (q.watch && (pixel >= q.n_pixels || !((q.watch[pixel >> 5] >> (pixel & 31u)) & 1u))) return;
  const uint32_t k = q.count.fetch_add(1u, std::memory_order_relaxed);
  if (k >= q.capacity) return;
  YmrtOracleEvent& e = q.out[k];
  e.pixel = pixel;
  e.sample = (uint32_t)sample;
  e.depth = (uint32_t)depth;
  e.kind = kind;
  e.material = material;
  e.pad = 0u;
  e.value[0] = r;
  e.value[1] = g;
  e.value[2] = b;
}
template <typename V>
inline V ymrt_oracle_contrib(int kind, uint32_t pixel, int sample, int depth, int material, const V& x) {
  ymrt_oracle_event(kind, pixel, sample, depth, material, (double)x[0], (double)x[1], (double)x[2]);
  return x;
}
inline void ymrt_oracle_scatter(uint32_t pixel, int sample, int depth, int material) {
  ymrt_oracle_event(0, pixel, sample, depth, material, 0.0, 0.0, 0.0);
}
// ---- end of insertion ----
'''
_SCATTER_SITE = "ray_throughput *= bsdf_weight;"
_SCATTER_CALL = ("ray_throughput *= bsdf_weight;\n\t\t"
                 "ymrt_oracle_scatter(pixel_index, pixel_sample_index, ray_depth, (int)material_index);")


def _event_sites(body: str) -> tuple[str, int, int]:
    """Wraps each indirect_light_clamp(...) term added to ray_received_light
    in ymrt_oracle_contrib (kind from the term's contents) and records the
    surface scattering site. Returns (body, terms wrapped, scatter sites)."""
    spans = []
    for m in re.finditer(r"\bindirect_light_clamp\(", body):
        start = body.rfind(";", 0, m.start())
        if "ray_received_light +=" not in body[start:m.start()]:
            continue  # the legacy kernel's `L +=` terms and the definition
        depth_level, k = 0, m.end() - 1
        while True:
            c = body[k]
            if c == "(":
                depth_level += 1
            elif c == ")":
                depth_level -= 1
                if depth_level == 0:
                    break
            k += 1
        inner = body[m.start():k + 1]
        if "EvalVolume" in inner:
            args = "2, pixel_index, pixel_sample_index, ray_depth, -1"
        elif "Background(" in inner:
            args = ("3, pixel_index, shading_ray_data_pixel_sample_index[ray_index], "
                    "shading_ray_data_ray_depth[ray_index], -1")
        elif "light_mtl" in inner:
            args = "4, pixel_index, pixel_sample_index, ray_depth, -1"
        elif "EvalDistantLight(" in inner or "EvalShapeLight(" in inner:
            args = "1, pixel_index, pixel_sample_index, ray_depth, (int)material_index"
        else:
            raise RuntimeError(f"Shading.cu: unclassified radiance term {inner[:80]!r}")
        spans.append((m.start(), k + 1, args))
    for a, b, args in reversed(spans):
        body = body[:a] + f"ymrt_oracle_contrib({args}, " + body[a:b] + ")" + body[b:]
    n_scatter = body.count(_SCATTER_SITE)
    body = body.replace(_SCATTER_SITE, _SCATTER_CALL)
    return body, len(spans), n_scatter


_RECORD_CALL = ("ymrt_oracle_record(pixel_index, shading_ray_data_ray_depth[ray_index], "
                "shading_ray_data_pixel_sample_index[ray_index], ray, hit_something, hit_record, ray_throughput, "
                "ray_received_light);\n\t\t")


# Material::FetchIOR (src/Material.h:262-277) writes the IOR priority only
# for default materials; for a light material its callers go on with an
# uninitialised priority (src/Shading.cu:694-697, 2146-2151,
# src/ShadingUtilities.cuh:969-974, src/VolumeEval.cuh:460-461,
# src/Camera.cpp:71-73), pushing it onto the nested-media stack when a light
# lies within two ulps of a boundary hit. The parity builds declare those
# variables zero-initialised (priority 0 for lights, the value ymrt_b200
# uses), so that the oracle's results do not depend on leftover register or
# stack contents. The timing build and the reference's default device build
# keep the code as written.
_PRIORITY_DECL = re.compile(r"\buint32_t\s+(mtl_ior_priority|material_ior_priority)\s*;")


def _init_priorities(text: str) -> tuple[str, int]:
    return _PRIORITY_DECL.subn(r"uint32_t \1 = 0u;", text)


# Files besides Shading.cu that hold FetchIOR calls; the parity builds compile
# copies of them (in the directory of the Shading.cu copy, so that its quoted
# includes find them first), with the priorities initialised.
_PRIORITY_FILES = {"ShadingUtilities.cuh": 1, "Camera.cpp": 1}


def _priority_copies(gen_dir: str) -> None:
    for name, expect in _PRIORITY_FILES.items():
        src = os.path.join(REF, "src", name)
        with open(src, "r", encoding="utf-8", errors="replace") as f:
            text, n = _init_priorities(f.read())
        if n != expect:
            raise RuntimeError(f"{name}: {n} FetchIOR priority declarations (expected {expect})")
        with open(os.path.join(gen_dir, name), "w") as f:
            f.write(f'#line 1 "{src}"\n' + text)


def _host_sources(gen_dir: str) -> list:
    """HOST_SOURCES with Camera.cpp taken from the parity copy in gen_dir."""
    return [os.path.join(gen_dir, "Camera.cpp") if s == "src/Camera.cpp" else os.path.join(REF, s)
            for s in HOST_SOURCES]


def _record_site(body: str) -> str:
    """Inserts the recording call into Ray_trace_path_tracing, before its
    miss branch (after the volume block)."""
    k = body.index("__global__ void Ray_trace_path_tracing(")
    j = body.index("if (!hit_something) {", k)
    return body[:j] + _RECORD_CALL + body[j:]


def shading_source(arg_order: str, counted: bool = True, gen_name: str = "gen") -> str:
    """Writes the build-time copy of src/Shading.cu (and its sampler and
    media headers) into oracle/_ref/<gen_name>. counted=False leaves the
    TraceRay / BVHTraverseShadow calls as the reference wrote them (the
    counters are still defined, never incremented): the timing build."""
    src = os.path.join(REF, "src", "Shading.cu")
    with open(src, "r", encoding="utf-8", errors="replace") as f:
        text = f.read()
    n = 0
    if arg_order == "ltr":
        text, n = _sequence_draws(text)
    # counting wrappers go after the includes, before the first namespace block
    first_ns = text.index("namespace YMRT")
    head, body = text[:first_ns], text[first_ns:]
    n_trace = n_shadow = 0
    if counted:
        body, n_trace = re.subn(r"\bTraceRay\(", "ymrt_oracle_counted_trace(", body)
        body, n_shadow = re.subn(r"\bBVHTraverseShadow\(", "ymrt_oracle_counted_shadow(", body)
    body, n_prio = re.subn(r"\b(\w+)\.GetMaxPriorityRecord\(\)\.ior_priority", r"ymrt_oracle_max_priority(\1)", body)
    n_init = n_terms = n_scatter = 0
    if counted:
        body = _record_site(body)
        body, n_init = _init_priorities(body)
        if n_init != 2:
            raise RuntimeError(f"Shading.cu: {n_init} FetchIOR priority declarations (expected 2)")
        body, n_terms, n_scatter = _event_sites(body)
        if (n_terms, n_scatter) != (6, 1):
            raise RuntimeError(f"Shading.cu: {n_terms} radiance terms and {n_scatter} scattering sites (expected 6, 1)")
    line_of_body = head.count("\n") + 1
    gen_dir = os.path.join(OUT, gen_name)
    os.makedirs(gen_dir, exist_ok=True)
    dst = os.path.join(gen_dir, "Shading.cu")
    out = (_HELPER + f'#line 1 "{src}"\n' + head + _COUNTERS + (_RECORD_HOST + _EVENT_HOST if counted else "") +
           f'#line {line_of_body} "{src}"\n' + body)
    with open(dst, "w") as f:
        f.write(out)
    n_pairs = _sampler_headers(arg_order, gen_dir, parity=counted)
    if counted:
        _priority_copies(gen_dir)
    with open(os.path.join(gen_dir, "Shading.cu.sites"), "w") as f:
        f.write(f"{n} argument lists sequenced, {n_trace} TraceRay and {n_shadow} BVHTraverseShadow calls counted, "
                f"{n_prio} GetMaxPriorityRecord reads made direct, {n_init} IOR priorities initialised, "
                f"{n_terms} radiance terms and {n_scatter} scattering sites recorded, "
                f"{n_pairs} two-draw constructors in RandomSampler.cuh sequenced\n")
    return dst


_PAIR = re.compile(r"return glm::vec2\(Random1D\(\), Random1D\(\)\);")


def _sampler_headers(arg_order: str, gen_dir: str, parity: bool = True) -> int:
    """The PCG and Sobol samplers' Random2D / SamplePixelOffset build a vec2
    from two Random1D() calls (src/RandomSampler.cuh:401-405, 544-548); the
    build-time copy of the header draws them first then second, as the
    device build evaluates them. VolumeEval.cuh, the header's only other
    includer, is copied beside it so that it picks the copy up."""
    src_dir = os.path.join(REF, "src")
    with open(os.path.join(src_dir, "RandomSampler.cuh"), "r", encoding="utf-8", errors="replace") as f:
        text = f.read()
    n = 0
    if arg_order == "ltr":
        text, n = _PAIR.subn("{ const float ymrt_first = Random1D(); const float ymrt_second = Random1D(); "
                             "return glm::vec2(ymrt_first, ymrt_second); }", text)
    with open(os.path.join(gen_dir, "RandomSampler.cuh"), "w") as f:
        f.write(f'#line 1 "{os.path.join(src_dir, "RandomSampler.cuh")}"\n' + text)
    with open(os.path.join(src_dir, "VolumeEval.cuh"), "r", encoding="utf-8", errors="replace") as f:
        vol = f.read()
    vol = _media_hooks(vol)
    if parity:
        vol, n_init = _init_priorities(vol)
        if n_init != 1:
            raise RuntimeError(f"VolumeEval.cuh: {n_init} FetchIOR priority declarations (expected 1)")
    with open(os.path.join(gen_dir, "VolumeEval.cuh"), "w") as f:
        f.write(f'#line 1 "{os.path.join(src_dir, "VolumeEval.cuh")}"\n' + vol)
    return n


# Media hooks in the build-time copy of VolumeEval.cuh (no change to the
# estimators): a medium's density node may be replaced by a 3-D density grid
# (this project's grid node, which the reference lacks: trilinear over cell
# centres of the object-space box [-0.5, 0.5]^3 with clamped edges, upper
# bound = the grid's maximum, in the same operand order as ymrt_b200's
# grid_eval), and the two "Max iteration reached" messages of the tracking
# loops (MAX_FREE_PATH_LENGTH steps, src/VolumeEval.cuh:144, 328) are counted
# instead of printed, so tests can compare how often each side reaches that
# bound.
_MEDIA_HOOKS = r'''
// ---- inserted by oracle/build_ref.py: density grids, tracking-bound counts ----
struct YmrtOracleGrid {
  const Texture* node;
  int n[3];
  std::vector<float> v;
  float vmax;
};
inline std::vector<YmrtOracleGrid>& ymrt_oracle_grids() {
  static std::vector<YmrtOracleGrid> g;
  return g;
}
inline std::atomic<unsigned long long>& ymrt_oracle_tracking_caps() {
  static std::atomic<unsigned long long> c{0};
  return c;
}
inline const YmrtOracleGrid* ymrt_oracle_find_grid(const Texture& t) {
  for (const YmrtOracleGrid& g : ymrt_oracle_grids())
    if (g.node == &t) return &g;
  return nullptr;
}
inline void ymrt_oracle_grid_axis(float p, int n, int* i0, int* i1, float* w) {
  const float g = (p + 0.5f) * (float)n - 0.5f;
  if (!(g > 0.0f)) { *i0 = *i1 = 0; *w = 0.0f; }
  else if (!(g < (float)(n - 1))) { *i0 = *i1 = n - 1; *w = 0.0f; }
  else { const float fl = std::floor(g); *i0 = (int)fl; *i1 = *i0 + 1; *w = g - fl; }
}
inline float ymrt_oracle_lerp(float a, float b, float w) { return a + w * (b - a); }
inline float ymrt_oracle_grid_eval(const YmrtOracleGrid& G, const glm::vec3& p) {
  int x0, x1, y0, y1, z0, z1;
  float wx, wy, wz;
  ymrt_oracle_grid_axis(p.x, G.n[0], &x0, &x1, &wx);
  ymrt_oracle_grid_axis(p.y, G.n[1], &y0, &y1, &wy);
  ymrt_oracle_grid_axis(p.z, G.n[2], &z0, &z1, &wz);
  auto at = [&](int x, int y, int z) { return G.v[((size_t)z * G.n[1] + y) * G.n[0] + x]; };
  const float c00 = ymrt_oracle_lerp(at(x0, y0, z0), at(x1, y0, z0), wx);
  const float c10 = ymrt_oracle_lerp(at(x0, y1, z0), at(x1, y1, z0), wx);
  const float c01 = ymrt_oracle_lerp(at(x0, y0, z1), at(x1, y0, z1), wx);
  const float c11 = ymrt_oracle_lerp(at(x0, y1, z1), at(x1, y1, z1), wx);
  return ymrt_oracle_lerp(ymrt_oracle_lerp(c00, c10, wy), ymrt_oracle_lerp(c01, c11, wy), wz);
}
inline glm::vec3 ymrt_oracle_density(const Texture& t, const Texture* textures, const ImageTileCache& cache,
                                     const TextureCoordinate& tc) {
  if (const YmrtOracleGrid* g = ymrt_oracle_find_grid(t)) return glm::vec3(ymrt_oracle_grid_eval(*g, tc.p_object));
  return TextureEval(t, textures, cache, tc);
}
inline float ymrt_oracle_upper_bound(const Texture& t, const glm::vec3& o, const glm::vec3& d, float t_max) {
  if (const YmrtOracleGrid* g = ymrt_oracle_find_grid(t)) return g->vmax;
  return t.GetUpperBound(o, d, t_max);
}
// ---- end of insertion ----
'''


def _media_hooks(text: str) -> str:
    i = text.index("namespace YMRT {") + len("namespace YMRT {")
    line = text[:i].count("\n") + 2
    text = (text[:i] + _MEDIA_HOOKS + f'#line {line}\n' + text[i:])
    text, a = re.subn(r"\bTextureEval\(density_texture,", "ymrt_oracle_density(density_texture,", text)
    text, b = re.subn(r"scene\.textures\[vol\.density_texture_idx\]\.GetUpperBound\(",
                      "ymrt_oracle_upper_bound(scene.textures[vol.density_texture_idx], ", text)
    text, c = re.subn(r'printf\("Max iteration reached at (SampleTrHeterogeneous|EvalTrHeterogeneous)!\\n"\);',
                      "ymrt_oracle_tracking_caps().fetch_add(1, std::memory_order_relaxed);", text)
    if (a, b, c) != (2, 2, 2):
        raise RuntimeError(f"VolumeEval.cuh hooks: {a} density, {b} bound, {c} cap sites (expected 2 each)")
    return "#include <atomic>\n#include <cmath>\n#include <vector>\n" + text


# ---------------------------------------------------------------------------
# The reference's own kernels built for the device (sm_100a), as a baseline.

GPU_LIB = os.path.join(OUT, "libymrt_refgpu.so")
# Same kernels compiled without FMA contraction and with IEEE division and
# square root (the flags ymrt_b200 is built with), for per-sample comparison.
GPU_LIB_EXACT = os.path.join(OUT, "libymrt_refgpu_exact.so")
EXACT_FLAGS = ["-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false"]

_GPU_FIX = r'''
// ---- inserted by oracle/build_ref.py: direct priority read ----
// RayTransfer::GetMaxPriorityRecord (src/Ray.h:148-151) returns a reference
// bound to a temporary copy of the selected record; the priority it yields is
// read here directly instead of through that reference.
__host__ __device__ inline uint32_t ymrt_oracle_max_priority(const YMRT::RayTransfer& rt) {
  return rt.max_priority_record_index != -1 ? rt.boundary_records[rt.max_priority_record_index].ior_priority
                                            : YMRT::BoundaryRecord().ior_priority;
}
// ---- end of insertion ----
'''


def shading_source_gpu(exact: bool = False) -> str:
    """Build-time copy of src/Shading.cu for the device build, in a
    directory of its own (oracle/_ref/gen_gpu, or gen_gpu_exact), so that it
    includes the reference's own headers: the GetMaxPriorityRecord reads are
    rewritten; argument order and everything else stay as the reference
    wrote them. exact=True (the parity build) also initialises the IOR
    priorities FetchIOR leaves unset, here and in copies of VolumeEval.cuh,
    ShadingUtilities.cuh and Camera.cpp beside it."""
    src = os.path.join(REF, "src", "Shading.cu")
    with open(src, "r", encoding="utf-8", errors="replace") as f:
        text = f.read()
    first_ns = text.index("namespace YMRT")
    head, body = text[:first_ns], text[first_ns:]
    body, n_prio = re.subn(r"\b(\w+)\.GetMaxPriorityRecord\(\)\.ior_priority", r"ymrt_oracle_max_priority(\1)", body)
    # nvcc does not macro-expand the argument of "#pragma unroll" (MSVC's
    # conforming preprocessor does): write the values, MAX_BOUNDARY_RECORD = 6.
    body, n_unroll = re.subn(r"#pragma unroll \(MAX_BOUNDARY_RECORD \+ 2\)", "#pragma unroll 8", body)
    body, n_unroll6 = re.subn(r"#pragma unroll MAX_BOUNDARY_RECORD\b", "#pragma unroll 6", body)
    n_unroll += n_unroll6
    n_init = 0
    gen_dir = os.path.join(OUT, "gen_gpu_exact" if exact else "gen_gpu")
    os.makedirs(gen_dir, exist_ok=True)
    if exact:
        body, n_init = _init_priorities(body)
        if n_init != 2:
            raise RuntimeError(f"Shading.cu: {n_init} FetchIOR priority declarations (expected 2)")
        vsrc = os.path.join(REF, "src", "VolumeEval.cuh")
        with open(vsrc, "r", encoding="utf-8", errors="replace") as f:
            vol, nv = _init_priorities(f.read())
        if nv != 1:
            raise RuntimeError(f"VolumeEval.cuh: {nv} FetchIOR priority declarations (expected 1)")
        with open(os.path.join(gen_dir, "VolumeEval.cuh"), "w") as f:
            f.write(f'#line 1 "{vsrc}"\n' + vol)
        _priority_copies(gen_dir)
    line_of_body = head.count("\n") + 1
    dst = os.path.join(gen_dir, "Shading_gpu.cu")
    with open(dst, "w") as f:
        f.write(f'#line 1 "{src}"\n' + head + _GPU_FIX + f'#line {line_of_body} "{src}"\n' + body)
    with open(dst + ".sites", "w") as f:
        f.write(f"{n_prio} GetMaxPriorityRecord reads made direct, {n_init} IOR priorities initialised, "
                f"{n_unroll} unroll counts written as literals\n")
    return dst


NVCC_GPU_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-DNDEBUG", "-DGLM_FORCE_PURE",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-w", "-lineinfo",
]


def _gpu_includes():
    inc = _includes()
    inc[1] = os.path.join(HERE, "shims", "ymrt_ref_gpu_prelude.h")  # replace the host prelude
    return inc


def _gpu_stamp(exact: bool) -> str:
    h = hashlib.sha256()
    h.update(" ".join(CXXFLAGS + NVCC_GPU_FLAGS + (EXACT_FLAGS if exact else [])).encode())
    for rel in HOST_SOURCES + ["src/Shading.cu"]:
        h.update(str(os.path.getmtime(os.path.join(REF, rel))).encode())
    for rel in ["ref_gpu_harness.cu", "ref_prepare.h", "ref_stubs.cpp", "build_ref.py", "shims/ymrt_ref_gpu_prelude.h",
                "shims/ppl.h"]:
        with open(os.path.join(HERE, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def build_gpu(force: bool = False, jobs: int = 8, exact: bool = False) -> str:
    """Builds oracle/_ref/libymrt_refgpu.so: the reference's stage kernels for
    sm_100a (nvcc's default floating-point flags, as the reference's CMake
    build uses) plus its host-side scene module, driven by ref_gpu_harness.cu.
    exact=True builds libymrt_refgpu_exact.so with EXACT_FLAGS instead."""
    lib = GPU_LIB_EXACT if exact else GPU_LIB
    if not os.path.isdir(os.path.join(REF, "src")):
        if os.path.exists(lib):
            return lib
        raise FileNotFoundError(f"reference sources not found at {REF} and no prebuilt {lib}")
    os.makedirs(OUT, exist_ok=True)
    stamp_file = os.path.join(OUT, "stamp_gpu_exact" if exact else "stamp_gpu")
    stamp = _gpu_stamp(exact)
    if not force and os.path.exists(lib) and os.path.exists(stamp_file):
        with open(stamp_file) as f:
            if f.read().strip() == stamp:
                return lib
    obj_dir = os.path.join(OUT, "obj_gpu_exact" if exact else "obj_gpu")
    os.makedirs(obj_dir, exist_ok=True)
    shading = shading_source_gpu(exact)
    cmds, objs = [], []
    sources = _host_sources(os.path.dirname(shading)) if exact else [os.path.join(REF, s) for s in HOST_SOURCES]
    for src in sources:
        obj = os.path.join(obj_dir, os.path.basename(src) + ".o")
        cmds.append(["g++"] + CXXFLAGS + _gpu_includes() + ["-c", src, "-o", obj])
        objs.append(obj)
    obj = os.path.join(obj_dir, "ref_stubs.o")
    cmds.append(["g++"] + CXXFLAGS + ["-DYMRT_ORACLE_REAL_CUDA"] + _gpu_includes() +
                ["-c", os.path.join(HERE, "ref_stubs.cpp"), "-o", obj])
    objs.append(obj)
    obj = os.path.join(obj_dir, "ref_gpu_harness.o")
    cmds.append(["nvcc"] + NVCC_GPU_FLAGS + (EXACT_FLAGS if exact else []) +
                [f'-DYMRT_SHADING_SOURCE="{shading}"'] + _gpu_includes() +
                ["-c", os.path.join(HERE, "ref_gpu_harness.cu"), "-o", obj])
    objs.append(obj)
    procs = []
    for cmd in cmds:
        procs.append((cmd[-3], subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        while len([p for _, p in procs if p.poll() is None]) >= jobs:
            procs[0][1].wait()
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"device oracle build failed for {src}:\n{out.decode(errors='replace')[-4000:]}")
    vs = os.path.join(obj_dir, "exports.map")
    with open(vs, "w") as f:
        f.write("{ global: ymrefgpu_*; local: *; };\n")
    tmp = lib + ".tmp"
    cmd = ["nvcc", "-shared", "-cudart", "static", "-gencode", "arch=compute_100a,code=sm_100a", "-o", tmp] + objs + [
        "-Xlinker", "-Bsymbolic", "-Xlinker", "--version-script=" + vs, "-Xlinker", "--no-undefined", "-lpthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("device oracle link failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, lib)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    return lib


def _stamp(arg_order: str) -> str:
    h = hashlib.sha256()
    h.update(arg_order.encode())
    h.update(" ".join(CXXFLAGS).encode())
    for rel in HOST_SOURCES + ["src/Shading.cu"]:
        p = os.path.join(REF, rel)
        h.update(str(os.path.getmtime(p)).encode())
    for rel in ["ref_harness.cpp", "ref_prepare.h", "ref_stubs.cpp", "build_ref.py", "shims/ymrt_ref_prelude.h",
                "shims/ppl.h"]:
        with open(os.path.join(HERE, rel), "rb") as f:
            h.update(f.read())
    return h.hexdigest()


def build(arg_order: str = "ltr", force: bool = False, jobs: int = 8) -> str:
    if not os.path.isdir(os.path.join(REF, "src")):
        if os.path.exists(LIB):
            return LIB
        raise FileNotFoundError(f"reference sources not found at {REF} and no prebuilt {LIB}")
    os.makedirs(OUT, exist_ok=True)
    _record_root()
    stamp_file = os.path.join(OUT, "stamp")
    stamp = _stamp(arg_order)
    if not force and os.path.exists(LIB) and os.path.exists(stamp_file):
        with open(stamp_file) as f:
            if f.read().strip() == stamp:
                return LIB
    objs = []
    procs = []
    obj_dir = os.path.join(OUT, "obj")
    os.makedirs(obj_dir, exist_ok=True)
    shading = shading_source(arg_order)
    jobs_list = [(s, os.path.join(obj_dir, os.path.basename(s) + ".o"), [])
                 for s in _host_sources(os.path.dirname(shading))]
    jobs_list.append((os.path.join(HERE, "ref_harness.cpp"), os.path.join(obj_dir, "ref_harness.o"),
                      [f'-DYMRT_SHADING_SOURCE="{shading}"']))
    jobs_list.append((os.path.join(HERE, "ref_stubs.cpp"), os.path.join(obj_dir, "ref_stubs.o"), []))
    for src, obj, extra in jobs_list:
        cmd = ["g++"] + CXXFLAGS + extra + _includes() + ["-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
        while len([p for _, p in procs if p.poll() is None]) >= jobs:
            procs[0][1].wait()
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"oracle build failed for {src}:\n{out.decode(errors='replace')[-4000:]}")
    tmp = LIB + ".tmp"
    cmd = ["g++", "-shared", "-pthread", "-o", tmp] + objs + ["-Wl,--no-undefined", "-Wl,-Bsymbolic"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle link failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, LIB)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    return LIB


# ---------------------------------------------------------------------------
# Timing build: the CPU baseline. The same sources (draws in the device's
# order, the priority read made direct so the host build does not crash) with
# g++ -O3 and an -march instruction set, glm's SIMD paths allowed, contraction
# left at g++'s default, and no query counters in the stage kernels (shared
# atomic counters would slow every query); the query count of a timed sample
# comes from a run of the counted build on the same sample. The library is
# built for two instruction sets (x86-64-v4: AVX-512; x86-64-v3: AVX2 + FMA)
# because it is built here and run on another machine; oracle/ref.py loads
# the widest one that machine supports.

TIMING_ISAS = ("x86-64-v4", "x86-64-v3")
TIMING_CXXFLAGS = ["-std=c++17", "-O3", "-DNDEBUG", "-fPIC", "-w", "-pthread"]


def timing_lib_path(isa: str) -> str:
    return os.path.join(OUT, f"libymrt_ref_fast_{isa.replace('x86-64-', '')}.so")


def build_timing(isa: str = "x86-64-v4", force: bool = False, jobs: int = 8) -> str:
    lib = timing_lib_path(isa)
    if not os.path.isdir(os.path.join(REF, "src")):
        if os.path.exists(lib):
            return lib
        raise FileNotFoundError(f"reference sources not found at {REF} and no prebuilt {lib}")
    os.makedirs(OUT, exist_ok=True)
    tag = isa.replace("x86-64-", "")
    stamp_file = os.path.join(OUT, f"stamp_fast_{tag}")
    h = hashlib.sha256(_stamp("ltr").encode())
    h.update(" ".join(TIMING_CXXFLAGS + [isa]).encode())
    stamp = h.hexdigest()
    if not force and os.path.exists(lib) and os.path.exists(stamp_file):
        with open(stamp_file) as f:
            if f.read().strip() == stamp:
                return lib
    obj_dir = os.path.join(OUT, f"obj_fast_{tag}")
    os.makedirs(obj_dir, exist_ok=True)
    shading = shading_source("ltr", counted=False, gen_name="gen_fast")
    flags = TIMING_CXXFLAGS + [f"-march={isa}"]
    jobs_list = [(os.path.join(REF, s), os.path.join(obj_dir, os.path.basename(s) + ".o"), []) for s in HOST_SOURCES]
    jobs_list.append((os.path.join(HERE, "ref_harness.cpp"), os.path.join(obj_dir, "ref_harness.o"),
                      [f'-DYMRT_SHADING_SOURCE="{shading}"']))
    jobs_list.append((os.path.join(HERE, "ref_stubs.cpp"), os.path.join(obj_dir, "ref_stubs.o"), []))
    procs, objs = [], []
    for src, obj, extra in jobs_list:
        cmd = ["g++"] + flags + extra + _includes() + ["-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
        while len([p for _, p in procs if p.poll() is None]) >= jobs:
            procs[0][1].wait()
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"timing build failed for {src}:\n{out.decode(errors='replace')[-4000:]}")
    tmp = lib + ".tmp"
    r = subprocess.run(["g++", "-shared", "-pthread", "-o", tmp] + objs + ["-Wl,--no-undefined", "-Wl,-Bsymbolic"],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("timing build link failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, lib)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    return lib


# ---------------------------------------------------------------------------
# FP64 oracle: the same reference sources and harness with every float
# computation done in double precision, for the converged-image error of the
# float renderers (the reference's and ymrt_b200's) at equal spp.
#
# The build-time copy (oracle/_ref/gen64) is made by rewriting tokens, not by
# editing the algorithm: ``float`` becomes ``double``; glm's float vector and
# matrix types become their double counterparts; float literals lose their
# ``f`` suffix (so glm's templates see one scalar type); the two places that
# reinterpret a float's bits (NextFloatUp/NextFloatDown, src/MathCommon.h:263-
# 297, and Ray::SetInvalid/Invalid, src/Ray.h:36-52) are rewritten for a
# 64-bit double (std::nextafter, an all-ones 64-bit pattern). The scene is
# still parsed with std::stof, so both precisions see the same geometry. The
# sampler draws, the light selection and every estimator step are the
# reference's; only rounding differs.

LIB64 = os.path.join(OUT, "libymrt_ref64.so")
_CODE_EXT = (".h", ".cuh", ".cu", ".cpp", ".hpp")
_FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)[fF](?![\w.])")
_NEXT_UP = re.compile(r"inline double NextFloatUp\(double f\)\s*\{.*?return UintToFloat\(ui\);\s*\}", re.S)
_NEXT_DOWN = re.compile(r"inline double NextFloatDown\(double f\)\s*\{.*?return UintToFloat\(ui\);\s*\}", re.S)
_BITS32 = re.compile(r"uint32_t& ui = \*\(\(uint32_t\*\)\(&f\)\);(\s*)ui = 0xFFFFFFFF;")
_CHECK32 = re.compile(r"uint32_t& ui = \*\(\(uint32_t\*\)\(&f\)\);(\s*)return ui == 0xFFFFFFFF;")


def to_fp64(text: str) -> tuple[str, dict]:
    """The token rewrite described above; returns the text and per-rule counts."""
    n = {}
    text, n["float"] = re.subn(r"\bfloat\b", "double", text)
    text, n["glm types"] = re.subn(r"\bglm::(vec|mat)([234])\b", r"glm::d\1\2", text)
    text, n["literals"] = _FLOAT_LIT.subn(r"\1", text)
    text, a = _NEXT_UP.subn("inline double NextFloatUp(double f) { return std::isinf(f) && f > 0.0 ? f : "
                            "std::nextafter(f == -0.0 ? 0.0 : f, INFINITY); }", text)
    text, b = _NEXT_DOWN.subn("inline double NextFloatDown(double f) { return std::isinf(f) && f < 0.0 ? f : "
                              "std::nextafter(f == 0.0 ? -0.0 : f, -INFINITY); }", text)
    n["next float"] = a + b
    text, a = _BITS32.subn(r"uint64_t& ui = *((uint64_t*)(&f));\1ui = 0xFFFFFFFFFFFFFFFFull;", text)
    text, b = _CHECK32.subn(r"uint64_t& ui = *((uint64_t*)(&f));\1return ui == 0xFFFFFFFFFFFFFFFFull;", text)
    n["invalid bits"] = a + b
    return text, n


def _fp64_tree() -> str:
    """Writes oracle/_ref/gen64: the rewritten reference src/ tree (with the
    sequenced Shading.cu / RandomSampler.cuh / VolumeEval.cuh of the float
    oracle in place of the originals), the harness and its shims."""
    shading_source("ltr")  # the float oracle's sequenced copies, rewritten below
    gen = os.path.join(OUT, "gen")
    root = os.path.join(OUT, "gen64")
    src_root = os.path.join(REF, "src")
    totals = {}
    for d, _, files in os.walk(src_root):
        for name in files:
            if not name.endswith(_CODE_EXT):
                continue
            rel = os.path.relpath(os.path.join(d, name), src_root)
            origin = os.path.join(d, name)
            if rel in ("Shading.cu", "RandomSampler.cuh", "VolumeEval.cuh") + tuple(_PRIORITY_FILES):
                origin = os.path.join(gen, rel)
            with open(origin, "r", encoding="utf-8", errors="replace") as f:
                text, n = to_fp64(f.read())
            for k, v in n.items():
                totals[k] = totals.get(k, 0) + v
            dst = os.path.join(root, "src", rel)
            os.makedirs(os.path.dirname(dst), exist_ok=True)
            with open(dst, "w") as f:
                f.write(text)
    for rel in ("ref_harness.cpp", "ref_prepare.h", "ref_stubs.cpp", os.path.join("shims", "ymrt_ref_prelude.h"),
                os.path.join("shims", "ppl.h")):
        with open(os.path.join(HERE, rel)) as f:
            text, _ = to_fp64(f.read())
        dst = os.path.join(root, rel)
        os.makedirs(os.path.dirname(dst), exist_ok=True)
        with open(dst, "w") as f:
            f.write(text)
    with open(os.path.join(root, "rewrites.txt"), "w") as f:
        f.write(", ".join(f"{k}: {v}" for k, v in sorted(totals.items())) + "\n")
    return root


def _fp64_includes(root: str):
    return [
        "-include", os.path.join(root, "shims", "ymrt_ref_prelude.h"),
        "-I" + os.path.join(root, "shims"), "-I" + os.path.join(HERE, "shims"),
        "-I" + root, "-I" + os.path.join(root, "src"), "-I" + os.path.join(root, "src", "core"),
        "-I" + os.path.join(REF, "external", "glm"),
        "-I" + os.path.join(REF, "external", "glad", "include"),
        "-I" + os.path.join(REF, "external", "image_lib"),
        "-I" + os.path.join(REF, "external", "assimp-5.1.0", "include"),
        "-I/usr/local/cuda/include",
    ]


def build_fp64(force: bool = False, jobs: int = 8) -> str:
    """Builds oracle/_ref/libymrt_ref64.so (exports ymref_*, with double in
    place of float in every signature)."""
    if not os.path.isdir(os.path.join(REF, "src")):
        if os.path.exists(LIB64):
            return LIB64
        raise FileNotFoundError(f"reference sources not found at {REF} and no prebuilt {LIB64}")
    os.makedirs(OUT, exist_ok=True)
    stamp_file = os.path.join(OUT, "stamp64")
    stamp = _stamp("fp64")
    if not force and os.path.exists(LIB64) and os.path.exists(stamp_file):
        with open(stamp_file) as f:
            if f.read().strip() == stamp:
                return LIB64
    root = _fp64_tree()
    obj_dir = os.path.join(OUT, "obj64")
    os.makedirs(obj_dir, exist_ok=True)
    inc = _fp64_includes(root)
    jobs_list = [(os.path.join(root, s), os.path.join(obj_dir, os.path.basename(s) + ".o"), []) for s in HOST_SOURCES]
    jobs_list.append((os.path.join(root, "ref_harness.cpp"), os.path.join(obj_dir, "ref_harness.o"),
                      [f'-DYMRT_SHADING_SOURCE="{os.path.join(root, "src", "Shading.cu")}"']))
    jobs_list.append((os.path.join(root, "ref_stubs.cpp"), os.path.join(obj_dir, "ref_stubs.o"), []))
    procs, objs = [], []
    for src, obj, extra in jobs_list:
        # assimp's material getters are called with the (now double) colour
        # arrays of the model importer; its double-precision mode types them
        cmd = ["g++"] + CXXFLAGS + ["-DASSIMP_DOUBLE_PRECISION", "-DYMREF_FP64"] + extra + inc + ["-c", src, "-o", obj]
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
        objs.append(obj)
        while len([p for _, p in procs if p.poll() is None]) >= jobs:
            procs[0][1].wait()
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"fp64 oracle build failed for {src}:\n{out.decode(errors='replace')[-6000:]}")
    tmp = LIB64 + ".tmp"
    cmd = ["g++", "-shared", "-pthread", "-o", tmp] + objs + ["-Wl,--no-undefined", "-Wl,-Bsymbolic"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("fp64 oracle link failed:\n" + r.stdout[-4000:] + r.stderr[-4000:])
    os.replace(tmp, LIB64)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    return LIB64


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--arg-order", choices=["ltr", "native"], default="ltr")
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--gpu", action="store_true", help="also build the reference's kernels for sm_100a")
    ap.add_argument("--reference", default=None, help="the reference checkout (default: $YMRT_REFERENCE_ROOT)")
    a = ap.parse_args(argv)
    if a.reference:
        set_reference(a.reference)
    print(build(a.arg_order, a.force))
    print(build_fp64(a.force))
    for isa in TIMING_ISAS:
        print(build_timing(isa, a.force))
    if a.gpu:
        print(build_gpu(a.force))
        print(build_gpu(a.force, exact=True))


if __name__ == "__main__":
    sys.exit(main())
