"""ymrt_b200: a B200-native (sm_100a) wavefront path tracer behind YMRT's
scene format and stage interface.

Python front end over the C ABI in ``include/ymrt.h`` (``libymrt.so``, built
in-tree by ``ymrt_b200.build``). It mirrors the reference's host side
(src/core/RenderModule.cpp, src/core/SceneModule.cpp): load a ``.ymtmp``
scene, upload it, render progressive frames into a float4 noise image and
accumulate them. There is no CPU rendering path: without a CUDA device or
without the built library every render call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

__all__ = [
    "RenderSetting", "Stats", "YmrtError", "Context", "HostScene", "Scene", "library", "default_setting",
    "HALTON_TABLE_SIZE",
]

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libymrt.so")
HALTON_TABLE_SIZE = 3682913  # sum of the first 1000 primes
TEXTURE_WORDS = 20  # 32-bit words of a ymrt_texture_desc

YMRT_OK = 0
ERRORS = {
    -1: "invalid argument", -2: "i/o error", -3: "malformed scene", -4: "unsupported", -5: "CUDA error",
    -6: "out of memory", -7: "timeout", -8: "overflow", -9: "no CUDA device",
}

QUERY_COUNTS, QUERY_INSTANCES, QUERY_LIGHTS, QUERY_LIGHT_TABLE = 0, 1, 2, 3
QUERY_TRANSFORMS, QUERY_CAMERA, QUERY_TRIANGLES = 4, 5, 6
QUERY_MATERIALS, QUERY_VOLUMES, QUERY_DISTANT_LIGHTS, QUERY_TEXTURES = 7, 8, 9, 10
QUERY_GEOMETRIES, QUERY_MESH_CORNERS, QUERY_IMAGE_PIXELS = 11, 12, 13


class YmrtError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}): {message}")
        self.code = code


class RenderSetting(ctypes.Structure):
    """Byte-compatible with the reference's RenderSetting (src/SceneDefines.h:17-40)."""
    _fields_ = [
        ("ssp", ctypes.c_int), ("ray_depth", ctypes.c_int), ("gamma", ctypes.c_float),
        ("exposure", ctypes.c_float), ("max_frame_count", ctypes.c_int), ("sampler_type", ctypes.c_int),
        ("enable_shape_light", ctypes.c_int), ("enable_distant_light", ctypes.c_uint8),
        ("enable_volume_scattering", ctypes.c_uint8), ("enable_env_light", ctypes.c_uint8),
        ("enable_russian_roulette", ctypes.c_uint8), ("enable_indirect_clamp", ctypes.c_uint8),
        ("pad_", ctypes.c_uint8 * 3), ("indirect_limit", ctypes.c_float),
    ]


assert ctypes.sizeof(RenderSetting) == 40


def default_setting(spp=1, ray_depth=8, shape_light=True, distant_light=False, volume=False, env_light=False,
                    russian_roulette=False, indirect_clamp=False, indirect_limit=10.0, sampler_type=1) -> RenderSetting:
    s = RenderSetting()
    s.ssp, s.ray_depth, s.gamma, s.exposure, s.max_frame_count = spp, ray_depth, 2.2, 1.0, -1
    s.sampler_type = sampler_type
    s.enable_shape_light = int(shape_light)
    s.enable_distant_light, s.enable_volume_scattering, s.enable_env_light = int(distant_light), int(volume), int(env_light)
    s.enable_russian_roulette, s.enable_indirect_clamp, s.indirect_limit = int(russian_roulette), int(indirect_clamp), indirect_limit
    return s


class LoadOptions(ctypes.Structure):
    _fields_ = [("max_leaf_triangles", ctypes.c_uint32), ("override_camera", ctypes.c_uint32),
                ("camera_from", ctypes.c_float * 3), ("camera_look", ctypes.c_float * 3),
                ("camera_fov_deg", ctypes.c_float), ("reserved", ctypes.c_uint32 * 7)]


class Job(ctypes.Structure):
    _fields_ = [("scene", ctypes.c_void_p), ("setting", RenderSetting), ("frame_index", ctypes.c_int),
                ("tile_begin", ctypes.c_int), ("tile_end", ctypes.c_int), ("out_rgba_device", ctypes.c_void_p),
                ("path_radiance_device", ctypes.c_void_p), ("dloss_device", ctypes.c_void_p)]


# One path vertex as the closest-hit stage leaves it (ymrt_debug_record_paths).
VERTEX_DTYPE = np.dtype([("pixel", "<u4"), ("depth", "<u4"), ("flags", "<u4"), ("inst", "<u4"), ("tri", "<u4"),
                         ("t", "<f4"), ("o", "<f4", 3), ("d", "<f4", 3), ("bary", "<f4", 3), ("tp", "<f4", 3),
                         ("light", "<f4", 3), ("path", "<u4"), ("pad", "<u4", 2)])
VERTEX_HIT, VERTEX_VOLUME, VERTEX_BACK = 1, 2, 4


class Stats(ctypes.Structure):
    _fields_ = [
        ("paths", ctypes.c_uint64), ("extension_rays", ctypes.c_uint64), ("shadow_rays", ctypes.c_uint64),
        ("waves", ctypes.c_uint64), ("node_visits", ctypes.c_uint64), ("triangle_tests", ctypes.c_uint64),
        ("kernel_launches", ctypes.c_uint64), ("ms_total", ctypes.c_double), ("ms_generate", ctypes.c_double),
        ("ms_extend", ctypes.c_double), ("ms_shade", ctypes.c_double), ("device_errors", ctypes.c_uint32),
        ("tracking_bound_hits", ctypes.c_uint32), ("shadow_node_visits", ctypes.c_uint64),
        ("shadow_triangle_tests", ctypes.c_uint64), ("ms_sort", ctypes.c_double), ("ms_connect", ctypes.c_double),
        ("shaded_hits", ctypes.c_uint64),
    ]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_ if not k.endswith("_")}


_lib = None


def library():
    """Loads libymrt.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise YmrtError(-9, f"{LIB_PATH} is missing; run `python -m ymrt_b200.build`")
    L = ctypes.CDLL(LIB_PATH)
    vp, i, sz = ctypes.c_void_p, ctypes.c_int, ctypes.c_size_t
    L.ymrt_create.argtypes = [i, ctypes.POINTER(vp)]
    L.ymrt_destroy.argtypes = [vp]
    L.ymrt_last_error.restype = ctypes.c_char_p
    L.ymrt_last_error.argtypes = [vp]
    L.ymrt_set_queue_capacity.argtypes = [vp, ctypes.c_uint32]
    L.ymrt_set_profiling.argtypes = [vp, i]
    L.ymrt_set_option.argtypes = [vp, i, i]
    L.ymrt_get_option.argtypes = [vp, i, ctypes.POINTER(i)]
    L.ymrt_scene_load_ymtmp.argtypes = [ctypes.c_char_p, i, i, ctypes.POINTER(vp), ctypes.c_char_p, sz]
    L.ymrt_scene_load_ymtmp_ex.argtypes = [ctypes.c_char_p, i, i, ctypes.POINTER(LoadOptions), ctypes.POINTER(vp),
                                           ctypes.c_char_p, sz]
    L.ymrt_host_scene_free.argtypes = [vp]
    L.ymrt_scene_from_arrays.argtypes = [ctypes.POINTER(SceneDesc), i, i, ctypes.POINTER(LoadOptions), ctypes.POINTER(vp),
                                         ctypes.c_char_p, sz]
    L.ymrt_host_scene_query.restype = ctypes.c_longlong
    L.ymrt_host_scene_query.argtypes = [vp, i, i, vp, sz]
    L.ymrt_scene_upload.argtypes = [vp, vp, vp, sz, ctypes.POINTER(vp)]
    L.ymrt_scene_free.argtypes = [vp]
    L.ymrt_scene_set_sobol_matrices.argtypes = [vp, vp, sz]
    L.ymrt_render_batch.argtypes = [vp, ctypes.POINTER(Job), i, ctypes.POINTER(Stats)]
    L.ymrt_render_backward.argtypes = [vp, ctypes.POINTER(Job), i, vp, ctypes.c_uint32, ctypes.POINTER(Stats)]
    L.ymrt_render_backward_ex.argtypes = [vp, ctypes.POINTER(Job), i, ctypes.POINTER(BackwardTargets),
                                          ctypes.POINTER(Stats)]
    L.ymrt_job_path_count.restype = ctypes.c_ulonglong
    L.ymrt_job_path_count.argtypes = [ctypes.POINTER(Job)]
    L.ymrt_scene_set_material_params.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp]
    L.ymrt_scene_get_material_params.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp]
    L.ymrt_scene_set_density_grid.argtypes = [vp, ctypes.c_uint32, i, i, i, vp, i]
    L.ymrt_debug_density.argtypes = [vp, ctypes.c_uint32, i, vp, vp]
    L.ymrt_debug_texture.argtypes = [vp, ctypes.c_uint32, i, vp, vp]
    L.ymrt_host_scene_set_image.argtypes = [vp, ctypes.c_uint32, vp, ctypes.c_size_t]
    L.ymrt_debug_frame.argtypes = [vp, i, vp, vp, vp, vp, vp, vp]
    L.ymrt_render_editor_view.argtypes = [vp, ctypes.POINTER(RenderSetting), ctypes.c_uint32, ctypes.c_uint32, vp, vp, i]
    L.ymrt_post_process.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_float,
                                    ctypes.c_float, i, i]
    L.ymrt_save_png.argtypes = [ctypes.c_char_p, vp, i, i]
    L.ymrt_render_forward.argtypes = [vp, ctypes.POINTER(RenderSetting), i, vp, i, ctypes.POINTER(Stats)]
    L.ymrt_render_tiles.argtypes = [vp, ctypes.POINTER(RenderSetting), i, i, i, vp, i, ctypes.POINTER(Stats)]
    L.ymrt_accumulate.argtypes = [vp, vp, vp, i]
    L.ymrt_debug_trace.argtypes = [vp, i, vp, vp, vp, vp, vp, vp, vp, vp, vp]
    L.ymrt_debug_record_paths.argtypes = [vp, ctypes.POINTER(RenderSetting), i, i, i, vp, vp, i, ctypes.POINTER(i), vp]
    L.ymrt_debug_occluded.argtypes = [vp, i, vp, vp, vp, vp]
    L.ymrt_debug_halton.argtypes = [vp, i, vp, vp, vp, i, vp, vp, vp]
    L.ymrt_debug_bound_record.argtypes = [vp, vp, sz, i]
    L.ymrt_debug_fail_allocations.argtypes = [i]
    L.ymrt_debug_fail_allocations.restype = None
    L.ymrt_scene_set_transforms.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp]
    L.ymrt_host_scene_set_transforms.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, vp, vp, vp]
    L.ymrt_scene_download.restype = ctypes.c_longlong
    L.ymrt_scene_download.argtypes = [vp, i, vp, sz]
    _lib = L
    return L


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


def _check(rc: int, ctx=None):
    if rc != YMRT_OK:
        msg = library().ymrt_last_error(ctx).decode(errors="replace")
        raise YmrtError(rc, msg)


OPTIONS = {"sort_hits": 1, "defer_shadows": 2, "graph_loop": 3, "trace_block": 4, "sort_rays": 6}


class Context:
    """One CUDA device + stream (the reference's RenderModule path-tracing stream)."""

    def __init__(self, device: int = 0, queue_capacity: int = 0, profiling: bool = False, **options):
        import weakref
        self.h = ctypes.c_void_p()
        self._scenes = weakref.WeakSet()  # scenes made on this context: freed before it
        _check(library().ymrt_create(device, ctypes.byref(self.h)))
        if queue_capacity:
            library().ymrt_set_queue_capacity(self.h, queue_capacity)
        if profiling:
            library().ymrt_set_profiling(self.h, 1)
        for name, value in options.items():
            self.set_option(name, value)

    def set_option(self, name: str, value) -> None:
        """Wave-loop options: sort_hits, defer_shadows, graph_loop (see include/ymrt.h)."""
        _check(library().ymrt_set_option(self.h, OPTIONS[name], int(value)))

    def get_option(self, name: str) -> int:
        v = ctypes.c_int()
        _check(library().ymrt_get_option(self.h, OPTIONS[name], ctypes.byref(v)))
        return v.value

    BOUND_SITES = {1: "shadow-ray boundary crossings", 2: "delta-tracking steps", 3: "ratio-tracking steps",
                   4: "waves of a frame", 5: "editor-view boundaries", 6: "texture-graph walk"}

    def bound_record(self, clear: bool = True) -> dict | None:
        """Where a bounded device loop last gave up (YMRT_DEVERR_ITER) on this
        context's device, with the ray it was following; None when none did."""
        w = np.zeros(64, np.uint32)
        _check(library().ymrt_debug_bound_record(self.h, _p(w), w.size, int(clear)), self.h)
        if w[0] == 0:
            return None
        f = w.view(np.float32)
        rec = np.array(w[18:18 + 24]).reshape(6, 4)
        return {"site": int(w[1]), "what": self.BOUND_SITES.get(int(w[1]), "?"), "count": int(w[2]),
                "last_inst": int(w[3]), "last_tri": int(w[4]), "o": f[5:8].copy(), "d": f[8:11].copy(),
                "tmax": float(f[11]), "majorant": f[12:15].copy(), "channel": float(f[15]),
                "max_priority_index": int(w[16].view(np.int32)), "record_count": int(w[17].view(np.int32)),
                "records": [(int(r[0]), float(r[1:2].view(np.float32)[0]), int(r[2]), int(r[3:4].view(np.int32)[0]))
                            for r in rec[:max(0, min(6, int(w[17].view(np.int32))))]]}

    def close(self):
        if self.h:
            for sc in list(self._scenes):
                sc.close()
            library().ymrt_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MeshDesc(ctypes.Structure):
    _fields_ = [("triangles", ctypes.c_void_p), ("triangle_count", ctypes.c_uint32),
                ("position_indices", ctypes.c_void_p), ("positions", ctypes.c_void_p), ("position_count", ctypes.c_uint32),
                ("normal_indices", ctypes.c_void_p), ("normals", ctypes.c_void_p), ("normal_count", ctypes.c_uint32),
                ("texcoord_indices", ctypes.c_void_p), ("texcoords", ctypes.c_void_p), ("texcoord_count", ctypes.c_uint32),
                ("sphere_radius", ctypes.c_float)]


class SceneDesc(ctypes.Structure):
    _fields_ = [("transforms", ctypes.c_void_p), ("inverse_transforms", ctypes.c_void_p),
                ("transform_scales", ctypes.c_void_p), ("transform_count", ctypes.c_uint32),
                ("geometries", ctypes.POINTER(MeshDesc)), ("geometry_count", ctypes.c_uint32),
                ("instances", ctypes.c_void_p), ("instance_count", ctypes.c_uint32),
                ("materials", ctypes.c_void_p), ("material_count", ctypes.c_uint32),
                ("volumes", ctypes.c_void_p), ("volume_count", ctypes.c_uint32),
                ("distant_lights", ctypes.c_void_p), ("distant_light_count", ctypes.c_uint32),
                ("textures", ctypes.c_void_p), ("texture_count", ctypes.c_uint32),
                ("camera_from", ctypes.c_float * 3), ("camera_look", ctypes.c_float * 3), ("camera_fov_deg", ctypes.c_float)]


class HostScene:
    """A parsed and prepared .ymtmp scene (no GPU involved)."""

    def __init__(self, path: str, width: int, height: int, max_leaf_triangles: int = 3, camera=None):
        """camera: optional (from, look, fov_degrees) replacing the file's camera."""
        self.h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        opts = LoadOptions()
        opts.max_leaf_triangles = max_leaf_triangles
        if camera is not None:
            frm, look, fov = camera
            opts.override_camera = 1
            opts.camera_from[:] = [float(x) for x in frm]
            opts.camera_look[:] = [float(x) for x in look]
            opts.camera_fov_deg = float(fov)
        rc = library().ymrt_scene_load_ymtmp_ex(path.encode(), width, height, ctypes.byref(opts), ctypes.byref(self.h),
                                                err, len(err))
        if rc != YMRT_OK:
            raise YmrtError(rc, err.value.decode(errors="replace"))
        self.width, self.height = width, height

    @classmethod
    def from_arrays(cls, width: int, height: int, transforms, geometries, instances, materials, camera,
                    volumes=None, distant_lights=None, textures=None, inverse_transforms=None, transform_scales=None,
                    max_leaf_triangles: int = 3) -> "HostScene":
        """A scene from in-memory arrays (ymrt_scene_from_arrays):
        transforms (n, 16) float32 column major; geometries: dicts with
        triangles (n, 3), position_indices, positions (m, 3), normal_indices,
        normals, optional texcoord_indices / texcoords, or {"sphere_radius": r};
        instances / materials / volumes / distant_lights: the reference's
        structs as uint32 words ((n, 8), (n, 39), (n, 9), (n, 8)); textures:
        (n, 20) words as records("textures") returns (ymrt_texture_desc); camera:
        (from, look, fov)."""
        keep = []

        def arr(a, dtype, cols=None):
            if a is None:
                return None, 0
            v = np.ascontiguousarray(a, dtype=dtype)
            if cols:
                v = v.reshape(-1, cols)
            keep.append(v)
            return v.ctypes.data_as(ctypes.c_void_p), (v.shape[0] if v.ndim > 1 else v.size)

        d = SceneDesc()
        d.transforms, d.transform_count = arr(transforms, np.float32, 16)
        d.inverse_transforms, _ = arr(inverse_transforms, np.float32, 16)
        d.transform_scales, _ = arr(transform_scales, np.float32, 3)
        meshes = (MeshDesc * max(len(geometries), 1))()
        for k, g in enumerate(geometries):
            m = meshes[k]
            if g.get("sphere_radius"):
                m.sphere_radius = float(g["sphere_radius"])
                continue
            m.triangles, m.triangle_count = arr(g["triangles"], np.uint32, 3)
            m.position_indices, _ = arr(g["position_indices"], np.uint32)
            m.positions, m.position_count = arr(g["positions"], np.float32, 3)
            m.normal_indices, _ = arr(g["normal_indices"], np.uint32)
            m.normals, m.normal_count = arr(g["normals"], np.float32, 3)
            if g.get("texcoords") is not None:
                m.texcoord_indices, _ = arr(g["texcoord_indices"], np.uint32)
                m.texcoords, m.texcoord_count = arr(g["texcoords"], np.float32, 2)
        keep.append(meshes)
        d.geometries, d.geometry_count = meshes, len(geometries)
        d.instances, d.instance_count = arr(instances, np.uint32, 8)
        d.materials, d.material_count = arr(materials, np.uint32, 39)
        d.volumes, d.volume_count = arr(volumes, np.uint32, 9)
        d.distant_lights, d.distant_light_count = arr(distant_lights, np.uint32, 8)
        d.textures, d.texture_count = arr(textures, np.uint32, TEXTURE_WORDS)
        frm, look, fov = camera
        d.camera_from[:] = [float(x) for x in frm]
        d.camera_look[:] = [float(x) for x in look]
        d.camera_fov_deg = float(fov)
        opts = LoadOptions()
        opts.max_leaf_triangles = max_leaf_triangles
        self = cls.__new__(cls)
        self.h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(1024)
        rc = library().ymrt_scene_from_arrays(ctypes.byref(d), width, height, ctypes.byref(opts), ctypes.byref(self.h),
                                              err, len(err))
        if rc != YMRT_OK:
            raise YmrtError(rc, err.value.decode(errors="replace"))
        self.width, self.height = width, height
        return self

    def close(self):
        if self.h:
            library().ymrt_host_scene_free(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _query(self, what, dtype, index=0):
        L = library()
        n = L.ymrt_host_scene_query(self.h, what, index, None, 0)
        if n < 0:
            raise YmrtError(int(n), "query failed")
        out = np.zeros(int(n), dtype=dtype)
        if n:
            L.ymrt_host_scene_query(self.h, what, index, _p(out), int(n))
        return out

    def counts(self) -> dict:
        c = self._query(QUERY_COUNTS, np.uint64)
        keys = ["instances", "meshes", "triangles", "instanced_triangles", "lights", "blas_nodes", "tlas_nodes", "materials"]
        return dict(zip(keys, (int(x) for x in c)))

    def instances(self) -> np.ndarray:
        return self._query(QUERY_INSTANCES, np.uint32).reshape(-1, 6)

    def lights(self):
        raw = self._query(QUERY_LIGHTS, np.float32).reshape(-1, 4)
        ids = raw[:, :2].copy().view(np.uint32)
        return ids, raw[:, 2:].copy(), self._query(QUERY_LIGHT_TABLE, np.float32)

    def set_transforms(self, first: int, object_to_world, scales=None) -> None:
        """Replaces transforms first.. of this prepared scene and rebuilds its
        top level on the host (ymrt_host_scene_set_transforms)."""
        m = np.ascontiguousarray(object_to_world, np.float32).reshape(-1, 16)
        sc = None if scales is None else np.ascontiguousarray(scales, np.float32).reshape(-1, 3)
        _check(library().ymrt_host_scene_set_transforms(self.h, first, m.shape[0], _p(m), None, _p(sc)))

    def transforms(self):
        t = self._query(QUERY_TRANSFORMS, np.float32).reshape(-1, 32)
        return t[:, :16].copy(), t[:, 16:].copy()

    def camera(self) -> np.ndarray:
        return self._query(QUERY_CAMERA, np.float32)

    def triangles(self, mesh: int) -> np.ndarray:
        return self._query(QUERY_TRIANGLES, np.uint32, mesh).reshape(-1, 3)

    def geometries(self) -> np.ndarray:
        """(kind, radius) per geometry: kind 0 a triangle mesh, 1 a sphere."""
        g = self._query(QUERY_GEOMETRIES, np.uint32).reshape(-1, 2)
        return np.stack([g[:, 0].astype(np.float32), g[:, 1].view(np.float32)], axis=1)

    def mesh_corners(self, mesh: int) -> np.ndarray:
        """Per corner of a mesh: position, normal, uv (8 floats; uv 0 without texcoords)."""
        return self._query(QUERY_MESH_CORNERS, np.float32, mesh).reshape(-1, 8)

    def image_pixels(self, texture_index: int) -> np.ndarray:
        """Pixels of an image node: linear samples, bottom row first, channels interleaved (flat)."""
        return self._query(QUERY_IMAGE_PIXELS, np.float32, texture_index)

    def set_image(self, texture_index: int, pixels) -> None:
        """Pixels of image node `texture_index` (width * height * channels
        linear floats, bottom row first): for scenes from arrays."""
        p = np.ascontiguousarray(pixels, np.float32).reshape(-1)
        _check(library().ymrt_host_scene_set_image(self.h, texture_index, _p(p), p.size))

    def records(self, kind: str) -> np.ndarray:
        """Materials, volumes, distant lights (32-bit words of the reference's
        structs) or textures (TEXTURE_WORDS words each: ymrt_texture_desc), one
        row per record."""
        what, width = {"materials": (QUERY_MATERIALS, 39), "volumes": (QUERY_VOLUMES, 9),
                       "distant_lights": (QUERY_DISTANT_LIGHTS, 8), "textures": (QUERY_TEXTURES, TEXTURE_WORDS)}[kind]
        return self._query(what, np.uint32).reshape(-1, width)


class Scene:
    """A scene resident on the device of a Context."""

    def __init__(self, ctx: Context, host: HostScene, halton_perm: np.ndarray):
        self.ctx = ctx
        self.width, self.height = host.width, host.height
        perm = np.ascontiguousarray(halton_perm, dtype=np.uint32)
        self.h = ctypes.c_void_p()
        _check(library().ymrt_scene_upload(ctx.h, host.h, _p(perm), perm.size, ctypes.byref(self.h)), ctx.h)
        self.host = host
        ctx._scenes.add(self)

    def material_params(self) -> np.ndarray:
        """(materials, 4) float32: diffuse albedo r, g, b and roughness per
        material (zeros for light materials)."""
        n = int(self.host.counts()["materials"])
        out = np.zeros((n, 4), np.float32)
        _check(library().ymrt_scene_get_material_params(self.h, 0, n, _p(out)), self.ctx.h)
        return out

    def set_material_params(self, params: np.ndarray, first: int = 0) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1, 4)
        _check(library().ymrt_scene_set_material_params(self.h, first, p.shape[0], _p(p)), self.ctx.h)

    SCENE_PARTS = {"tlas_nodes": (1, np.uint8), "tlas_prims": (2, np.uint32), "instances": (3, np.uint32),
                   "shape_lights": (4, np.uint32), "light_table": (5, np.float32), "instance_buckets": (6, np.uint8),
                   "camera_media": (7, np.uint32), "file_index": (8, np.uint32)}

    def set_transforms(self, first: int, object_to_world, scales=None) -> None:
        """Replaces transforms first.. (object-to-world 4x4 matrices, as
        (count, 4, 4) arrays indexed [column][row] like glm) and rebuilds the
        top level on the device (ymrt_scene_set_transforms)."""
        m = np.ascontiguousarray(object_to_world, np.float32).reshape(-1, 16)
        sc = None if scales is None else np.ascontiguousarray(scales, np.float32).reshape(-1, 3)
        _check(library().ymrt_scene_set_transforms(self.h, first, m.shape[0], _p(m), None, _p(sc)), self.ctx.h)

    def download(self, part: str) -> np.ndarray:
        """Device contents of the scene's top level (ymrt_scene_download)."""
        what, dt = self.SCENE_PARTS[part]
        n = library().ymrt_scene_download(self.h, what, None, 0)
        _check(0 if n >= 0 else int(n), self.ctx.h)
        out = np.zeros(max(int(n), 1) // np.dtype(dt).itemsize, dt)
        got = library().ymrt_scene_download(self.h, what, _p(out), out.nbytes)
        _check(0 if got >= 0 else int(got), self.ctx.h)
        return out[: int(n) // np.dtype(dt).itemsize]

    def set_density_grid(self, texture_index: int, values: np.ndarray, half: bool = False) -> None:
        """Attaches a density grid to texture node `texture_index`: values has
        shape (nz, ny, nx) over the volume's object-space box [-0.5, 0.5]^3."""
        v = np.ascontiguousarray(values, dtype=np.float32)
        if v.ndim != 3:
            raise ValueError("density grid must be a (nz, ny, nx) array")
        nz, ny, nx = v.shape
        _check(library().ymrt_scene_set_density_grid(self.h, texture_index, nx, ny, nz, _p(v), int(half)), self.ctx.h)

    def editor_view(self, setting: "RenderSetting"):
        """The editor's albedo / picking view at the scene's size: (beauty
        (H, W, 4), primitive index (H, W), 0xFFFFFFFF where nothing was hit)."""
        beauty = np.zeros((self.height, self.width, 4), np.float32)
        prim = np.full((self.height, self.width), 0xFFFFFFFF, np.uint32)
        _check(library().ymrt_render_editor_view(self.h, ctypes.byref(setting), self.width, self.height, _p(beauty),
                                                 _p(prim), 0), self.ctx.h)
        return beauty, prim

    def shading_frame(self, inst, tri, bary, back, dirs) -> np.ndarray:
        """The shading frame at given hits: (n, 22) floats (normal, tangent,
        bitangent, texture footprint, uv, object-space position, dp/du,
        material index)."""
        n = len(inst)
        out = np.zeros((n, 22), np.float32)
        args = [np.ascontiguousarray(inst, np.uint32), np.ascontiguousarray(tri, np.uint32),
                np.ascontiguousarray(bary, np.float32), np.ascontiguousarray(back, np.int32),
                np.ascontiguousarray(dirs, np.float32)]
        _check(library().ymrt_debug_frame(self.h, n, *[_p(a) for a in args], _p(out)), self.ctx.h)
        return out

    def texture(self, texture_index: int, st, points) -> np.ndarray:
        """rgb of texture node `texture_index` as a surface reads it, at
        texture coordinates st (n, 2) and object-space points (n, 3)."""
        st = np.asarray(st, np.float32).reshape(-1, 2)
        p = np.asarray(points, np.float32).reshape(-1, 3)
        if st.shape[0] != p.shape[0]:
            raise ValueError("st and points must have the same length")
        c = np.ascontiguousarray(np.concatenate([st, p], axis=1), np.float32)
        out = np.zeros((c.shape[0], 3), np.float32)
        _check(library().ymrt_debug_texture(self.h, texture_index, c.shape[0], _p(c), _p(out)), self.ctx.h)
        return out

    def density(self, texture_index: int, points) -> np.ndarray:
        """Texture node `texture_index` at object-space points (n, 3), on the device."""
        p = np.ascontiguousarray(points, np.float32).reshape(-1, 3)
        out = np.zeros(p.shape[0], np.float32)
        _check(library().ymrt_debug_density(self.h, texture_index, p.shape[0], _p(p), _p(out)), self.ctx.h)
        return out

    def set_sobol_matrices(self, matrices: np.ndarray) -> None:
        """Generator matrices for the Sobol sampler (4096 x 32 uint32)."""
        m = np.ascontiguousarray(matrices, dtype=np.uint32)
        _check(library().ymrt_scene_set_sobol_matrices(self.h, _p(m), m.size), self.ctx.h)

    def close(self):
        # a scene outlives its context only as a handle: the context's close()
        # freed it already
        if self.h and self.ctx.h:
            library().ymrt_scene_free(self.h)
        self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def render(self, setting: RenderSetting, frame_index: int = 1, out=None, tile_begin: int = 0, tile_end: int = 0):
        """Renders one frame. `out`: None (returns a new host array), a host
        numpy float32 (H, W, 4) array, or a torch CUDA tensor of that shape."""
        stats = Stats()
        on_device = 0
        if out is None:
            out = np.zeros((self.height, self.width, 4), np.float32)
        if isinstance(out, np.ndarray):
            assert out.dtype == np.float32 and out.flags.c_contiguous and out.size == self.width * self.height * 4
            ptr = _p(out)
        else:  # torch tensor on the device
            assert out.is_cuda and out.is_contiguous() and out.numel() == self.width * self.height * 4
            ptr = ctypes.c_void_p(out.data_ptr())
            on_device = 1
        rc = library().ymrt_render_tiles(self.h, ctypes.byref(setting), frame_index, tile_begin, tile_end, ptr,
                                         on_device, ctypes.byref(stats))
        _check(rc, self.ctx.h)
        return out, stats

    def record_paths(self, setting: RenderSetting, pixels, frame_index: int = 1, tile_begin: int = 0,
                     tile_end: int = 0, capacity: int = 1 << 16):
        """Renders a frame (waves launched from the host) while recording,
        after each closest-hit stage, the vertex of every path of the given
        pixel indices: ray, hit, throughput and light received so far
        (ymrt_debug_record_paths). Returns (records as VERTEX_DTYPE, image)."""
        n_pix = self.width * self.height
        watch = np.zeros((n_pix + 31) // 32, np.uint32)
        px = np.asarray(pixels, np.int64).ravel()
        np.bitwise_or.at(watch, px >> 5, (np.uint32(1) << (px & 31).astype(np.uint32)))
        out = np.zeros(capacity, VERTEX_DTYPE)
        img = np.zeros((self.height, self.width, 4), np.float32)
        n = ctypes.c_int(0)
        _check(library().ymrt_debug_record_paths(self.h, ctypes.byref(setting), frame_index, tile_begin, tile_end,
                                                 _p(watch), _p(out), capacity, ctypes.byref(n), _p(img)), self.ctx.h)
        return out[:n.value].copy(), img

    def trace(self, origins, dirs, last_hit=None) -> dict:
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(dirs, np.float32)
        n = o.shape[0]
        lh = None if last_hit is None else np.ascontiguousarray(last_hit, np.uint32)
        inst, tri = np.zeros(n, np.uint32), np.zeros(n, np.uint32)
        t, bary = np.zeros(n, np.float32), np.zeros((n, 3), np.float32)
        back, nearby = np.zeros(n, np.int32), np.zeros(n, np.int32)
        _check(library().ymrt_debug_trace(self.h, n, _p(o), _p(d), _p(lh), _p(inst), _p(tri), _p(t), _p(bary),
                                          _p(back), _p(nearby)), self.ctx.h)
        return {"inst": inst, "tri": tri, "t": t, "bary": bary, "back": back, "nearby": nearby}

    def occluded(self, origins, dirs, tmax) -> np.ndarray:
        o = np.ascontiguousarray(origins, np.float32)
        d = np.ascontiguousarray(dirs, np.float32)
        tm = np.ascontiguousarray(tmax, np.float32)
        out = np.zeros(o.shape[0], np.int32)
        _check(library().ymrt_debug_occluded(self.h, o.shape[0], _p(o), _p(d), _p(tm), _p(out)), self.ctx.h)
        return out

    def halton(self, px, py, sample, n_dims: int):
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        sm = np.ascontiguousarray(sample, np.int32)
        n = px.size
        idx = np.zeros(n, np.uint64)
        off = np.zeros((n, 2), np.float32)
        dims = np.zeros((n, max(n_dims, 1)), np.float32)
        _check(library().ymrt_debug_halton(self.h, n, _p(px), _p(py), _p(sm), n_dims, _p(idx), _p(off), _p(dims)),
               self.ctx.h)
        return idx, off, dims[:, :n_dims]


def _jobs(renders, records=None, dlosses=None):
    jobs = (Job * len(renders))()
    for k, r in enumerate(renders):
        scene, setting, frame, out = r[:4]
        tb, te = (r[4], r[5]) if len(r) > 4 else (0, 0)
        assert out.is_cuda and out.dtype.is_floating_point and out.is_contiguous()
        assert out.numel() == scene.width * scene.height * 4
        jobs[k].scene = scene.h.value if isinstance(scene.h, ctypes.c_void_p) else scene.h
        jobs[k].setting = setting
        jobs[k].frame_index = frame
        jobs[k].tile_begin, jobs[k].tile_end = tb, te
        jobs[k].out_rgba_device = out.data_ptr()
        if records is not None:
            jobs[k].path_radiance_device = records[k].data_ptr()
        if dlosses is not None:
            jobs[k].dloss_device = dlosses[k].data_ptr()
    return jobs


def render_batch(ctx: Context, renders, records=None) -> Stats:
    """Renders several (scene, setting, frame_index, out, tile_begin, tile_end)
    tuples in one batch; each `out` is a torch CUDA float32 tensor of its
    scene's (H, W, 4) shape and receives that render. `records` (optional,
    one CUDA float32 tensor of path_count(render) x 4 per render) receive
    each path's radiance, for a later backward pass."""
    jobs = _jobs(renders, records)
    stats = Stats()
    _check(library().ymrt_render_batch(ctx.h, jobs, len(renders), ctypes.byref(stats)), ctx.h)
    return stats


def path_count(render) -> int:
    """Paths the render (as render_batch takes it) traces."""
    return int(library().ymrt_job_path_count(ctypes.byref(_jobs([render])[0])))


class BackwardTargets(ctypes.Structure):
    _fields_ = [("material_grads_device", ctypes.c_void_p), ("n_materials", ctypes.c_uint32),
                ("grid_texture", ctypes.c_uint32), ("grid_grads_device", ctypes.c_void_p),
                ("grid_values", ctypes.c_uint64), ("reserved", ctypes.c_uint32 * 4)]


def post_process(ctx: Context, image, primitive_index=None, selected: int = 0xFFFFFFFF, gamma: float = 2.2,
                 exposure: float = 1.0, outline: bool = False) -> np.ndarray:
    """ACES tone mapping and gamma (and the selection outline) of an (H, W, 4)
    float32 host image; returns a new array."""
    img = np.ascontiguousarray(image, np.float32).copy()
    prim = None if primitive_index is None else np.ascontiguousarray(primitive_index, np.uint32)
    _check(library().ymrt_post_process(ctx.h, _p(img), None if prim is None else _p(prim), img.shape[1], img.shape[0],
                                       selected, gamma, exposure, int(outline), 0), ctx.h)
    return img


def save_png(path: str, image) -> None:
    """Writes an (H, W, 4) float host image, bottom row first, as an 8-bit
    RGBA PNG the way the reference's SavePngImage does (the extension becomes
    .png; channels clamped to [0, 1], scaled by 255 and rounded)."""
    img = np.ascontiguousarray(image, np.float32)
    if img.ndim != 3 or img.shape[2] != 4:
        raise ValueError("save_png: image must be (height, width, 4)")
    rc = library().ymrt_save_png(os.fsencode(path), _p(img), img.shape[1], img.shape[0])
    if rc != YMRT_OK:
        raise YmrtError(rc, f"save_png: cannot write {path}")


def render_backward_ex(ctx: Context, renders, records, dlosses, material_grads=None, grid_texture=None,
                       grid_grads=None) -> Stats:
    """render_backward with optional targets: `material_grads` (CUDA float32,
    (materials, 4)) and/or `grid_grads` (CUDA float32, one value per value of
    the density grid attached to texture node `grid_texture`, in the grid's
    (nz, ny, nx) order). Media are differentiated."""
    jobs = _jobs(renders, records, dlosses)
    t = BackwardTargets()
    t.grid_texture = 0xFFFFFFFF
    if material_grads is not None:
        assert material_grads.is_cuda and material_grads.dtype.is_floating_point and material_grads.is_contiguous()
        t.material_grads_device, t.n_materials = material_grads.data_ptr(), material_grads.shape[0]
    if grid_grads is not None:
        assert grid_grads.is_cuda and grid_grads.is_contiguous() and grid_texture is not None
        t.grid_texture, t.grid_grads_device, t.grid_values = grid_texture, grid_grads.data_ptr(), grid_grads.numel()
    stats = Stats()
    _check(library().ymrt_render_backward_ex(ctx.h, jobs, len(renders), ctypes.byref(t), ctypes.byref(stats)), ctx.h)
    return stats


def render_backward(ctx: Context, renders, records, dlosses, grads) -> Stats:
    """Path-replay adjoint of render_batch(ctx, renders, records): `dlosses`
    holds dLoss/dImage per render (CUDA float32, (H, W, 4)); `grads` (CUDA
    float32, (materials, 4)) receives dLoss/d(albedo rgb, roughness) per
    material."""
    jobs = _jobs(renders, records, dlosses)
    stats = Stats()
    assert grads.is_cuda and grads.dtype.is_floating_point and grads.is_contiguous()
    _check(library().ymrt_render_backward(ctx.h, jobs, len(renders), grads.data_ptr(), grads.shape[0],
                                          ctypes.byref(stats)), ctx.h)
    return stats

