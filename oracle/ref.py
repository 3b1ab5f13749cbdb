"""ctypes front end of the oracle (the YMRT reference built for the host).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, never by the ymrt_b200 product.
See oracle/build_ref.py for how the library is built and oracle/ref_harness.cpp
for what each entry point runs in the reference.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libymrt_ref.so")
LIB64_PATH = os.path.join(HERE, "_ref", "libymrt_ref64.so")

_lib = None
_lib64 = None


class Settings(ctypes.Structure):
    _fields_ = [
        ("spp", ctypes.c_int), ("ray_depth", ctypes.c_int), ("sampler_type", ctypes.c_int),
        ("enable_shape_light", ctypes.c_int), ("enable_distant_light", ctypes.c_int),
        ("enable_volume_scattering", ctypes.c_int), ("enable_env_light", ctypes.c_int),
        ("enable_russian_roulette", ctypes.c_int), ("enable_indirect_clamp", ctypes.c_int),
        ("indirect_limit", ctypes.c_float),
    ]


class Settings64(ctypes.Structure):
    _fields_ = [(n, t) for n, t in Settings._fields_[:-1]] + [("indirect_limit", ctypes.c_double)]


# One radiance event of the parity builds' event recorder (YmrtOracleEvent):
# kind 0 surface scattering (material: the vertex's), 1 next-event estimation
# at a surface vertex (material: the vertex's), 2 next-event estimation at a
# volume vertex, 3 background, 4 a light seen before any scattering; value:
# the term added to the path's light (0 for scattering), in double.
EVENT_DTYPE = np.dtype([("pixel", "<u4"), ("sample", "<u4"), ("depth", "<u4"), ("kind", "<i4"), ("material", "<i4"),
                        ("pad", "<u4"), ("value", "<f8", 3)])
assert EVENT_DTYPE.itemsize == 48
# One path vertex as the trace stage leaves it (24 words; the layout the
# build-time recording hook writes and ymrt_debug_record_paths returns).
VERTEX_DTYPE = np.dtype([("pixel", "<u4"), ("depth", "<u4"), ("flags", "<u4"), ("inst", "<u4"), ("tri", "<u4"),
                         ("t", "<f4"), ("o", "<f4", 3), ("d", "<f4", 3), ("bary", "<f4", 3), ("tp", "<f4", 3),
                         ("light", "<f4", 3), ("path", "<u4"), ("pad", "<u4", 2)])
assert VERTEX_DTYPE.itemsize == 96


def watch_bits(pixels, n_pixels: int) -> np.ndarray:
    """One bit per pixel index, set for the given pixels."""
    bits = np.zeros((n_pixels + 31) // 32, np.uint32)
    px = np.asarray(pixels, np.int64).ravel()
    np.bitwise_or.at(bits, px >> 5, (np.uint32(1) << (px & 31).astype(np.uint32)))
    return bits


def available() -> bool:
    return os.path.exists(LIB_PATH)


def _bind(L, settings_type):
    vp, i, u64 = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint64
    L.ymref_halton_table_size.restype = ctypes.c_size_t
    L.ymref_scene_load.restype = vp
    L.ymref_scene_load.argtypes = [ctypes.c_char_p, vp, ctypes.c_size_t, i, i]
    L.ymref_scene_free.argtypes = [vp]
    L.ymref_set_settings.argtypes = [vp, ctypes.POINTER(settings_type)]
    for name in ("ymref_scene_counts", "ymref_instances", "ymref_transforms"):
        getattr(L, name).argtypes = [vp, vp] if name != "ymref_transforms" else [vp, vp, vp]
    L.ymref_geometry_triangle_count.restype = ctypes.c_int64
    L.ymref_geometry_triangle_count.argtypes = [vp, ctypes.c_uint32]
    L.ymref_geometry_triangles.argtypes = [vp, ctypes.c_uint32, vp]
    L.ymref_geometry_kind.argtypes = [vp, ctypes.c_uint32, vp]
    L.ymref_mesh_corners.argtypes = [vp, ctypes.c_uint32, vp]
    L.ymref_lights.argtypes = [vp, vp, vp, vp]
    L.ymref_camera_bytes.argtypes = [vp, vp, i]
    L.ymref_scene_records.argtypes = [vp, i, vp, i]
    L.ymref_texture_eval.argtypes = [vp, ctypes.c_uint32, i, vp, vp]
    L.ymref_render_editor_view.argtypes = [vp, i, i, vp, vp]
    L.ymref_post_process.argtypes = [vp, vp, i, i, ctypes.c_uint32, ctypes.c_float, ctypes.c_float, i]
    L.ymref_shading_frame.argtypes = [vp, i, vp, vp, vp, vp, vp, vp]
    L.ymref_image_pixels.restype = ctypes.c_longlong
    if hasattr(L, "ymref_set_events"):
        L.ymref_set_events.argtypes = [vp, vp, i, vp]
        L.ymref_events_recorded.restype = ctypes.c_uint32
    if hasattr(L, "ymref_save_png"):
        L.ymref_save_png.argtypes = [ctypes.c_char_p, vp, i, i]
    L.ymref_image_pixels.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_longlong]
    L.ymref_bvh_depths.argtypes = [vp, vp]
    L.ymref_sobol_matrices.restype = ctypes.c_size_t
    L.ymref_sobol_matrices.argtypes = [vp, ctypes.c_size_t]
    L.ymref_trace.argtypes = [vp, i, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ymref_occluded.argtypes = [vp, i, vp, vp, vp, vp]
    L.ymref_set_density_grid.argtypes = [vp, ctypes.c_uint32, i, i, i, vp]
    L.ymref_density.argtypes = [vp, ctypes.c_uint32, i, vp, vp]
    L.ymref_set_transforms.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
    L.ymref_set_material_params.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp]
    L.ymref_get_material_params.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp]
    L.ymref_tracking_caps.restype = ctypes.c_ulonglong
    L.ymref_tracking_caps.argtypes = [i]
    if hasattr(L, "ymref_set_recorder"):
        L.ymref_set_recorder.argtypes = [vp, vp, vp, i]
        L.ymref_recorded.restype = ctypes.c_uint32
    if hasattr(L, "ymref_boundary_walk"):
        L.ymref_boundary_walk.argtypes = [vp, vp, vp, ctypes.c_float, ctypes.c_uint32, ctypes.c_uint32, vp, i, vp]
    L.ymref_halton.argtypes = [vp, i, vp, vp, vp, i, vp, vp, vp]
    L.ymref_render_frame.argtypes = [vp, i, i, i, i, i, vp]
    L.ymref_last_render_seconds.restype = ctypes.c_double
    L.ymref_last_render_seconds.argtypes = [vp]
    L.ymref_accumulate.argtypes = [vp, vp, i, i, i]
    L.ymref_query_counts.argtypes = [vp, i]


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build_ref  # noqa: F401  (only when sources are present)
            build_ref.build()
        L = ctypes.CDLL(LIB_PATH)
        _bind(L, Settings)
        _lib = L
    return _lib


_lib_fast = None


def _cpu_flags() -> set:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    return set(line.split(":", 1)[1].split())
    except OSError:
        pass
    return set()


def lib_fast():
    """The timing build of the reference (build_ref.build_timing) for the
    widest instruction set this machine runs, with its name; None when
    neither is built."""
    global _lib_fast
    if _lib_fast is None:
        from . import build_ref
        flags = _cpu_flags()
        isas = [i for i in build_ref.TIMING_ISAS
                if i != "x86-64-v4" or {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl"} <= flags]
        for isa in isas:
            path = build_ref.timing_lib_path(isa)
            if not os.path.exists(path):
                try:
                    build_ref.build_timing(isa)
                except Exception:  # noqa: BLE001 - no sources here: try the next one
                    continue
            L = ctypes.CDLL(path)
            _bind(L, Settings)
            _lib_fast = (L, isa)
            break
    return _lib_fast


def available64() -> bool:
    return os.path.exists(LIB64_PATH)


def lib64():
    """The FP64 build of the oracle (every float of the reference and the
    harness computed in double; see build_ref.build_fp64)."""
    global _lib64
    if _lib64 is None:
        if not os.path.exists(LIB64_PATH):
            from . import build_ref  # noqa: F401  (only when sources are present)
            build_ref.build_fp64()
        L = ctypes.CDLL(LIB64_PATH)
        _bind(L, Settings64)
        _lib64 = L
    return _lib64


def _p(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def sobol_matrices() -> np.ndarray:
    """The reference's Sobol generator matrices (4096 x 32 uint32)."""
    n = lib().ymref_sobol_matrices(None, 0)
    out = np.zeros(n, np.uint32)
    lib().ymref_sobol_matrices(_p(out), n)
    return out


class RefScene:
    """One scene loaded and prepared by the reference's own scene module."""

    def __init__(self, path: str, halton_perm: np.ndarray, width: int, height: int, fp64: bool = False,
                 fast: bool = False):
        """fp64: load it into the FP64 build (renders return float64 images).
        fast: into the timing build (no query counters; see lib_fast)."""
        if fast:
            lf = lib_fast()
            if lf is None:
                raise RuntimeError("the timing build of the reference is not available")
            L, self.isa = lf
        else:
            L = lib64() if fp64 else lib()
        self._L = L
        self._f = np.float64 if fp64 else np.float32
        self._settings = Settings64 if fp64 else Settings
        perm = np.ascontiguousarray(halton_perm, dtype=np.uint32)
        self.width, self.height = width, height
        self.h = L.ymref_scene_load(path.encode(), _p(perm), perm.size, width, height)
        if not self.h:
            raise RuntimeError(f"reference failed to load {path}")
        self._perm = perm

    def close(self):
        if self.h:
            self._L.ymref_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_settings(self, spp=1, ray_depth=8, sampler_type=1, shape_light=1, distant_light=0, volume=0,
                     env_light=0, russian_roulette=0, indirect_clamp=0, indirect_limit=10.0):
        s = self._settings(spp, ray_depth, sampler_type, shape_light, distant_light, volume, env_light,
                     russian_roulette, indirect_clamp, indirect_limit)
        self._L.ymref_set_settings(self.h, ctypes.byref(s))

    def counts(self) -> dict:
        out = np.zeros(5, np.uint32)
        self._L.ymref_scene_counts(self.h, _p(out))
        return dict(zip(["instances", "geometries", "lights", "transforms", "materials"], out.tolist()))

    def instances(self) -> np.ndarray:
        n = self.counts()["instances"]
        out = np.zeros((n, 6), np.uint32)
        self._L.ymref_instances(self.h, _p(out))
        return out

    def geometry_triangles(self, g: int) -> np.ndarray:
        n = self._L.ymref_geometry_triangle_count(self.h, g)
        out = np.zeros((max(n, 0), 3), np.uint32)
        if n > 0:
            self._L.ymref_geometry_triangles(self.h, g, _p(out))
        return out

    def geometries(self) -> np.ndarray:
        """(type, radius) per geometry: type 0 a triangle mesh, 1 a sphere."""
        n = self.counts()["geometries"]
        out = np.zeros((n, 2), self._f)
        r = np.zeros(1, self._f)
        for g in range(n):
            out[g, 0] = self._L.ymref_geometry_kind(self.h, g, _p(r))
            out[g, 1] = r[0]
        return out

    def mesh_corners(self, g: int) -> np.ndarray:
        n = self._L.ymref_geometry_triangle_count(self.h, g)
        out = np.zeros((3 * max(n, 0), 8), self._f)
        if n > 0:
            self._L.ymref_mesh_corners(self.h, g, _p(out))
        return out

    def lights(self):
        n = self.counts()["lights"]
        ids = np.zeros((n, 2), np.uint32)
        pa = np.zeros((n, 2), self._f)
        tab = np.zeros(n, self._f)
        self._L.ymref_lights(self.h, _p(ids), _p(pa), _p(tab))
        return ids, pa, tab

    def transforms(self):
        n = self.counts()["transforms"]
        fwd = np.zeros((n, 16), self._f)
        inv = np.zeros((n, 16), self._f)
        self._L.ymref_transforms(self.h, _p(fwd), _p(inv))
        return fwd, inv

    def camera_bytes(self) -> bytes:
        buf = np.zeros(512, np.uint8)
        n = self._L.ymref_camera_bytes(self.h, _p(buf), buf.size)
        return buf[:n].tobytes()

    def bvh_depths(self) -> np.ndarray:
        """Depth of each mesh's binary BVH, then of the top-level BVH."""
        out = np.zeros(self.counts()["geometries"] + 1, np.uint32)
        self._L.ymref_bvh_depths(self.h, _p(out))
        return out

    def records(self, kind: str) -> np.ndarray:
        """Materials, volumes, distant lights (raw 32-bit words of the
        reference structs) or textures (20 words each, the layout of
        ymrt_texture_desc), one row per record."""
        what = {"materials": 0, "volumes": 1, "distant_lights": 2, "textures": 3}[kind]
        width = {"materials": 39, "volumes": 9, "distant_lights": 8, "textures": 20}[kind]
        n = self._L.ymref_scene_records(self.h, what, None, 0)
        out = np.zeros(max(n, 0), np.uint32)
        if n > 0:
            self._L.ymref_scene_records(self.h, what, _p(out), out.size)
        return out.reshape(-1, width)

    def shading_frame(self, inst, tri, bary, back, dirs) -> np.ndarray:
        """The reference's shading frame at given hits: (n, 22) floats (normal,
        tangent, bitangent, texture footprint du/dx dv/dx du/dy dv/dy, uv,
        object-space position, dp/du, material index)."""
        n = len(inst)
        out = np.zeros((n, 22), self._f)
        self._L.ymref_shading_frame(self.h, n, _p(np.ascontiguousarray(inst, np.uint32)),
                                    _p(np.ascontiguousarray(tri, np.uint32)), _p(np.ascontiguousarray(bary, self._f)),
                                    _p(np.ascontiguousarray(back, np.int32)), _p(np.ascontiguousarray(dirs, self._f)),
                                    _p(out))
        return out

    def editor_view(self, wave_capacity: int = 1 << 20, threads: int = 0):
        """The reference's editor view: (beauty (H, W, 4), primitive index (H, W))
        from zeroed beauty and an all-EMPTY primitive index."""
        beauty = np.zeros((self.height, self.width, 4), self._f)
        prim = np.full((self.height, self.width), 0xFFFFFFFF, np.uint32)
        rc = self._L.ymref_render_editor_view(self.h, wave_capacity, threads or (os.cpu_count() or 1), _p(beauty),
                                              _p(prim))
        if rc != 0:
            raise RuntimeError(f"ymref_render_editor_view failed ({rc})")
        return beauty, prim

    def image_pixels(self, tex: int) -> np.ndarray:
        """Pixels of image node `tex` as the reference loaded them (linear
        samples, bottom row first, channels interleaved), flat."""
        n = self._L.ymref_image_pixels(self.h, tex, None, 0)
        if n < 0:
            raise ValueError("not an image node")
        out = np.zeros(n, self._f)
        self._L.ymref_image_pixels(self.h, tex, _p(out), n)
        return out

    def texture(self, tex: int, st, points) -> np.ndarray:
        """The reference's TextureEval of node `tex` at texture coordinates
        st (n, 2) and object-space points (n, 3): rgb (n, 3)."""
        st = np.asarray(st, self._f).reshape(-1, 2)
        p = np.asarray(points, self._f).reshape(-1, 3)
        c = np.ascontiguousarray(np.concatenate([st, p], axis=1), self._f)
        out = np.zeros((c.shape[0], 3), self._f)
        if self._L.ymref_texture_eval(self.h, tex, c.shape[0], _p(c), _p(out)) != 0:
            raise ValueError("unknown texture node")
        return out

    def trace(self, origins, dirs, last_hit=None) -> dict:
        o = np.ascontiguousarray(origins, self._f)
        d = np.ascontiguousarray(dirs, self._f)
        n = o.shape[0]
        lh = None if last_hit is None else np.ascontiguousarray(last_hit, np.uint32)
        inst = np.zeros(n, np.uint32)
        tri = np.zeros(n, np.uint32)
        t = np.zeros(n, self._f)
        bary = np.zeros((n, 3), self._f)
        back = np.zeros(n, np.int32)
        nearby = np.zeros(n, np.int32)
        self._L.ymref_trace(self.h, n, _p(o), _p(d), None if lh is None else _p(lh), _p(inst), _p(tri), _p(t),
                          _p(bary), _p(back), _p(nearby))
        return {"inst": inst, "tri": tri, "t": t, "bary": bary, "back": back, "nearby": nearby}

    def occluded(self, origins, dirs, tmax) -> np.ndarray:
        o = np.ascontiguousarray(origins, self._f)
        d = np.ascontiguousarray(dirs, self._f)
        tm = np.ascontiguousarray(tmax, self._f)
        out = np.zeros(o.shape[0], np.int32)
        self._L.ymref_occluded(self.h, o.shape[0], _p(o), _p(d), _p(tm), _p(out))
        return out

    def set_density_grid(self, texture_index: int, values) -> None:
        """Replaces density node `texture_index` with a 3-D grid (values of
        shape (nz, ny, nx), x fastest), as ymrt_scene_set_density_grid does;
        pass the values the device stores (float16-rounded for a half grid)."""
        v = np.ascontiguousarray(values, self._f)
        nz, ny, nx = v.shape
        assert self._L.ymref_set_density_grid(self.h, texture_index, nx, ny, nz, _p(v)) == 0

    def set_transforms(self, first: int, object_to_world, scales=None) -> None:
        """A transform edit and the reference editor's rebuild after it
        (top level, instance order, lights, camera media)."""
        m = np.ascontiguousarray(object_to_world, self._f).reshape(-1, 16)
        sc = None if scales is None else np.ascontiguousarray(scales, self._f).reshape(-1, 3)
        assert self._L.ymref_set_transforms(self.h, first, m.shape[0], _p(m), None if sc is None else _p(sc)) == 0

    def material_params(self) -> tuple[np.ndarray, np.ndarray]:
        """((materials, 4) diffuse albedo rgb and alpha_x of each default
        material, zeros for others; (materials,) bool: the material is
        Lambertian, its diffuse lobe alone)."""
        n = int(self.counts()["materials"])
        out = np.zeros((n, 5), self._f)
        if self._L.ymref_get_material_params(self.h, 0, n, _p(out)) != 0:
            raise ValueError("material range out of bounds")
        return out[:, :4].copy(), out[:, 4] != 0

    def set_material_params(self, params, first: int = 0) -> None:
        """(materials, 4): diffuse albedo rgb and roughness of each default
        material, as ymrt_b200's Scene.set_material_params takes them."""
        p = np.ascontiguousarray(params, self._f).reshape(-1, 4)
        if self._L.ymref_set_material_params(self.h, first, p.shape[0], _p(p)) != 0:
            raise ValueError("material range out of bounds")

    def density(self, texture_index: int, points) -> np.ndarray:
        """A medium's density node (or attached grid) at object-space points
        (n, 3), as the tracking loops read it."""
        p = np.ascontiguousarray(points, self._f).reshape(-1, 3)
        out = np.zeros(p.shape[0], self._f)
        assert self._L.ymref_density(self.h, texture_index, p.shape[0], _p(p), _p(out)) == 0
        return out

    def tracking_caps(self, reset: bool = True) -> int:
        """Tracking loops that reached MAX_FREE_PATH_LENGTH steps (all scenes
        of this library) since the last reset."""
        return int(self._L.ymref_tracking_caps(int(reset)))

    def boundary_walk(self, origin, direction, tmax, last_inst, last_tri, transfer_words, max_steps=1024) -> np.ndarray:
        """Boundary crossings of one shadow ray as the reference's TraceTr
        follows them: one row per crossing (instance, triangle, t, back,
        nearby count, stack records after it, distance traced)."""
        o = np.ascontiguousarray(origin, np.float32)
        d = np.ascontiguousarray(direction, np.float32)
        tw = np.ascontiguousarray(transfer_words, np.uint32)
        out = np.zeros((max_steps, 8), np.uint32)
        n = self._L.ymref_boundary_walk(self.h, _p(o), _p(d), float(tmax), last_inst, last_tri, _p(tw), max_steps,
                                        _p(out))
        return out[:n]

    def halton(self, px, py, sample, n_dims: int):
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        sm = np.ascontiguousarray(sample, np.int32)
        n = px.size
        idx = np.zeros(n, np.uint64)
        off = np.zeros((n, 2), self._f)
        dims = np.zeros((n, n_dims), self._f)
        self._L.ymref_halton(self.h, n, _p(px), _p(py), _p(sm), n_dims, _p(idx), _p(off), _p(dims))
        return idx, off, dims

    def render_frame(self, frame_index: int = 1, tile_begin: int = 0, tile_end: int = 0,
                     wave_capacity: int = 1 << 18, threads: int | None = None) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), self._f)
        threads = threads or os.cpu_count() or 1
        rc = self._L.ymref_render_frame(self.h, frame_index, tile_begin, tile_end, wave_capacity, threads, _p(out))
        if rc != 0:
            raise RuntimeError(f"reference render failed ({rc})")
        return out

    def last_render_seconds(self) -> float:
        return self._L.ymref_last_render_seconds(self.h)

    def record_events(self, frame_index: int = 1, tile_begin: int = 0, tile_end: int = 0, capacity: int = 1 << 22,
                      pixels=None, threads: int | None = None):
        """Renders a frame while recording its radiance events (EVENT_DTYPE:
        every term added to a path's light and every surface scattering
        event) of the given pixel indices (None: all); returns (events,
        image). Parity builds, float or double."""
        if not hasattr(self._L, "ymref_set_events"):
            raise RuntimeError("event recording needs a parity build")
        out = np.zeros(capacity, EVENT_DTYPE)
        watch = None if pixels is None else watch_bits(pixels, self.width * self.height)
        self._L.ymref_set_events(self.h, _p(out), capacity, None if watch is None else _p(watch))
        try:
            img = self.render_frame(frame_index, tile_begin, tile_end, threads=threads)
            n = int(self._L.ymref_events_recorded())
        finally:
            self._L.ymref_set_events(self.h, None, 0, None)
        if n > capacity:
            raise RuntimeError(f"{n} events recorded, capacity {capacity}")
        return out[:n].copy(), img

    def record_paths(self, pixels, frame_index: int = 1, tile_begin: int = 0, tile_end: int = 0,
                     capacity: int = 1 << 16, threads: int | None = None):
        """Renders a frame while recording the path vertices of the given
        pixel indices (the trace stage's ray, hit, throughput and received
        light at each depth); returns (records as VERTEX_DTYPE, image)."""
        if self._f is not np.float32 or not hasattr(self._L, "ymref_set_recorder"):
            raise RuntimeError("path recording needs the float parity build")
        watch = watch_bits(pixels, self.width * self.height)
        out = np.zeros(capacity, VERTEX_DTYPE)
        self._L.ymref_set_recorder(self.h, _p(watch), _p(out), capacity)
        try:
            img = self.render_frame(frame_index, tile_begin, tile_end, threads=threads)
            n = int(self._L.ymref_recorded())
        finally:
            self._L.ymref_set_recorder(self.h, None, None, 0)
        if n > capacity:
            raise RuntimeError(f"{n} vertices recorded, capacity {capacity}")
        return out[:n].copy(), img


def save_png(path: str, image) -> bool:
    """The reference's SavePngImage of an (H, W, 4) float image, bottom row
    first (float oracle)."""
    img = np.ascontiguousarray(image, np.float32)
    return lib().ymref_save_png(os.fsencode(path), _p(img), img.shape[1], img.shape[0]) == 1


def post_process(image, primitive_index, selected: int, gamma: float, exposure: float, outline: bool):
    """The reference's tone mapping (and outline) of an (H, W, 4) float32
    image, returned as a new array."""
    img = np.ascontiguousarray(image, np.float32).copy()
    prim = np.ascontiguousarray(primitive_index, np.uint32)
    lib().ymref_post_process(_p(img), _p(prim), img.shape[1], img.shape[0], selected, gamma, exposure, int(outline))
    return img


def query_counts(reset: bool = True) -> tuple[int, int]:
    """(closest-hit queries, occlusion queries) made by the reference's stage
    kernels since the last reset, across all scenes."""
    out = np.zeros(2, np.uint64)
    lib().ymref_query_counts(_p(out), int(reset))
    return int(out[0]), int(out[1])


# ---------------------------------------------------------------------------
# The reference's own wavefront kernels rebuilt for the device (sm_100a),
# driven by oracle/ref_gpu_harness.cu. Two builds: nvcc's default
# floating-point flags (the reference's own build; the timing baseline) and
# "exact" (no FMA contraction, IEEE division/square root -- the flags
# ymrt_b200 uses), for per-sample comparison.

GPU_LIB_PATHS = {False: os.path.join(HERE, "_ref", "libymrt_refgpu.so"),
                 True: os.path.join(HERE, "_ref", "libymrt_refgpu_exact.so")}
_gpu_libs = {}


def gpu_available(exact: bool = False) -> bool:
    return os.path.exists(GPU_LIB_PATHS[exact])


def gpu_lib(exact: bool = False):
    if exact not in _gpu_libs:
        path = GPU_LIB_PATHS[exact]
        if not os.path.exists(path):
            from . import build_ref
            build_ref.build_gpu(exact=exact)
        L = ctypes.CDLL(path)
        vp, i = ctypes.c_void_p, ctypes.c_int
        L.ymrefgpu_scene_load.restype = vp
        L.ymrefgpu_scene_load.argtypes = [ctypes.c_char_p, vp, ctypes.c_size_t, i, i, i]
        L.ymrefgpu_scene_free.argtypes = [vp]
        L.ymrefgpu_set_settings.argtypes = [vp, ctypes.POINTER(Settings)]
        L.ymrefgpu_render_frame.argtypes = [vp, i, i, i, vp]
        L.ymrefgpu_last_error.restype = ctypes.c_char_p
        L.ymrefgpu_last_error.argtypes = [vp]
        L.ymrefgpu_set_profiling.argtypes = [vp, i]
        L.ymrefgpu_last_stage_ms.restype = ctypes.c_uint32
        L.ymrefgpu_last_stage_ms.argtypes = [vp, vp]
        for name in ("ymrefgpu_last_render_ms", "ymrefgpu_last_wall_ms"):
            getattr(L, name).restype = ctypes.c_double
            getattr(L, name).argtypes = [vp]
        if hasattr(L, "ymrefgpu_set_recorder"):
            L.ymrefgpu_set_recorder.argtypes = [vp, vp, i]
            L.ymrefgpu_read_records.argtypes = [vp, vp, i]
        _gpu_libs[exact] = L
    return _gpu_libs[exact]


class RefGpuScene:
    """A scene rendered by the reference's own CUDA kernels on `device`."""

    def __init__(self, path: str, halton_perm: np.ndarray, width: int, height: int, device: int = 0,
                 exact: bool = False):
        self.L = gpu_lib(exact)
        perm = np.ascontiguousarray(halton_perm, dtype=np.uint32)
        self.width, self.height = width, height
        self.h = self.L.ymrefgpu_scene_load(path.encode(), _p(perm), perm.size, width, height, device)
        if not self.h:
            raise RuntimeError(f"reference (device build) failed to load {path}")

    def set_settings(self, spp=1, ray_depth=8, sampler_type=1, shape_light=1, distant_light=0, volume=0,
                     env_light=0, russian_roulette=0, indirect_clamp=0, indirect_limit=10.0):
        s = Settings(spp, ray_depth, sampler_type, shape_light, distant_light, volume, env_light,
                     russian_roulette, indirect_clamp, indirect_limit)
        if self.L.ymrefgpu_set_settings(self.h, ctypes.byref(s)) != 0:
            raise RuntimeError("ymrefgpu_set_settings failed")

    def render_frame(self, frame_index: int, tile_begin: int = 0, tile_end: int = 0, copy_out: bool = True):
        out = np.zeros((self.height, self.width, 4), np.float32) if copy_out else None
        rc = self.L.ymrefgpu_render_frame(self.h, frame_index, tile_begin, tile_end,
                                          _p(out) if copy_out else None)
        if rc != 0:
            raise RuntimeError("reference device render failed: " + self.L.ymrefgpu_last_error(self.h).decode())
        return out

    def last_render_ms(self) -> float:
        return self.L.ymrefgpu_last_render_ms(self.h)

    def last_wall_ms(self) -> float:
        return self.L.ymrefgpu_last_wall_ms(self.h)

    def set_profiling(self, on: bool):
        self.L.ymrefgpu_set_profiling(self.h, int(on))

    def record_paths(self, pixels, frame_index: int = 1, tile_begin: int = 0, tile_end: int = 0,
                     capacity: int = 1 << 16):
        """As RefScene.record_paths, on the device: the harness reads the
        hit queue the reference's trace stage writes, so only vertices that
        hit something are recorded (the reference's kernels are unchanged)."""
        watch = watch_bits(pixels, self.width * self.height)
        if self.L.ymrefgpu_set_recorder(self.h, _p(watch), capacity) != 0:
            raise RuntimeError("ymrefgpu_set_recorder failed")
        try:
            img = self.render_frame(frame_index, tile_begin, tile_end)
            out = np.zeros(capacity, VERTEX_DTYPE)
            n = self.L.ymrefgpu_read_records(self.h, _p(out), capacity)
        finally:
            self.L.ymrefgpu_set_recorder(self.h, None, 0)
        if n < 0 or n > capacity:
            raise RuntimeError(f"recording failed or overflowed ({n} of {capacity})")
        return out[:n].copy(), img

    def last_stage_ms(self) -> dict:
        out = np.zeros(3, np.float64)
        waves = self.L.ymrefgpu_last_stage_ms(self.h, _p(out))
        return {"generate": float(out[0]), "trace": float(out[1]), "shade": float(out[2]), "waves": int(waves)}

    def close(self):
        if self.h:
            self.L.ymrefgpu_scene_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
