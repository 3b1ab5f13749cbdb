"""Failure paths, each made on purpose without faulting the GPU: every one
returns its negative status, fills the frame's statistics, traps nothing and
leaves the context usable.

* An allocation that fails (host-side injection, ymrt_debug_fail_allocations)
  returns YMRT_ERR_OOM; the next call succeeds.
* Seven nested media boundaries overflow the six-record nested-media stack
  (MAX_BOUNDARY_RECORD, src/Ray.h:12): the record is dropped, as the
  reference drops it (RayTransfer::PushRecord, src/Ray.h:181-186, which
  prints a warning), and the call returns YMRT_ERR_OVERFLOW with
  YMRT_DEVERR_STACK; the image still equals the reference's.
* A shadow ray through more than 4 x 64 medium boundaries (130 index-matched
  slabs between the floor and the light) reaches this library's own bound
  on boundary crossings: YMRT_ERR_OVERFLOW with YMRT_DEVERR_ITER, and the
  bound record names the site.
* A medium whose majorant (sigma_t 5000 over a grid that is nearly empty)
  makes delta tracking run past MAX_FREE_PATH_LENGTH stops there as the
  reference does: not an error; the stopped loops are counted and equal the
  reference's count, and the images agree per sample.
"""
import ctypes

import numpy as np
import pytest

import ymrt_b200 as Y
from ymrt_b200 import scenes

pytestmark = pytest.mark.gpu


def render_raw(sc: Y.Scene, setting, frame=1):
    """rc, stats and image of one frame, without raising."""
    st = Y.Stats()
    img = np.zeros((sc.height, sc.width, 4), np.float32)
    rc = Y.library().ymrt_render_tiles(sc.h, ctypes.byref(setting), frame, 0, 0,
                                        img.ctypes.data_as(ctypes.c_void_p), 0, ctypes.byref(st))
    return rc, st, img


def _write(tmp_path, s, name):
    path = str(tmp_path / f"{name}.ymtmp")
    scenes.write_scene(s, path)
    return path


def test_allocation_failure_returns_oom(cornell_path, halton_perm):
    ctx = Y.Context(0)
    sc = Y.Scene(ctx, Y.HostScene(cornell_path, 64, 64), halton_perm)
    setting = Y.default_setting(spp=1, ray_depth=8)
    want, _ = sc.render(setting, 1)
    Y.library().ymrt_set_queue_capacity(ctx.h, 1 << 22)  # the next render allocates larger queues
    Y.library().ymrt_debug_fail_allocations(1)
    rc, _, _ = render_raw(sc, setting, 1)
    Y.library().ymrt_debug_fail_allocations(0)
    assert rc == -6, rc  # YMRT_ERR_OOM
    assert b"allocating" in Y.library().ymrt_last_error(ctx.h)
    got, st = sc.render(setting, 1)  # the context is still usable
    assert st.device_errors == 0
    np.testing.assert_allclose(got, want, rtol=1e-5, atol=1e-7)
    sc.close()
    ctx.close()


def nested_boxes_scene(n_boxes=7):
    s = scenes.cornell_scene(0)
    s.materials.append(("DefaultMaterial", "nest_material", {"ior_n": 1.0}))
    for k in range(n_boxes):
        size = 1.9 - 0.12 * k
        s.transforms.append((f"nest_t{k}", (0.0, 0.0, 0.0), (size, size, size), (0, 0, 0)))
        s.instances.append((f"nest_{k}", "Geo_Box", f"nest_t{k}", "nest_material", None, True))
    return s


def test_nested_media_stack_overflow(tmp_path, halton_perm, ctx, oracle):
    path = _write(tmp_path, nested_boxes_scene(), "nested")
    sc = Y.Scene(ctx, Y.HostScene(path, 64, 64), halton_perm)
    rc, st, img = render_raw(sc, Y.default_setting(spp=1, ray_depth=8))
    assert rc == -8, rc  # YMRT_ERR_OVERFLOW
    assert st.device_errors & 1  # YMRT_DEVERR_STACK
    assert st.paths == 64 * 64
    ref = oracle.RefScene(path, halton_perm, 64, 64)
    ref.set_settings(spp=1, ray_depth=8)
    want = ref.render_frame(1)
    ref.close()
    diff = np.abs(img[..., :3] - want[..., :3])
    bad = np.any(diff > 1e-5 * np.maximum(np.abs(img[..., :3]), np.abs(want[..., :3])) + 1e-7, axis=-1)
    assert bad.mean() <= 5e-3, bad.sum()
    sc.close()


def slabs_scene(n_slabs=130):
    s = scenes.cornell_scene(0)
    s.volumes.append(("fog", "fog_t", (0.05, 0.05, 0.05), (0.8, 0.8, 0.8), 0.0, None))
    s.transforms.append(("fog_t", (0.0, 0.0, 0.0), (1.98, 1.98, 1.98), (0, 0, 0)))
    s.materials.append(("DefaultMaterial", "slab_material", {"ior_n": 1.0}))
    s.instances.append(("fog_box", "Geo_Box", "fog_t", "slab_material", "fog", True))
    for k in range(n_slabs):
        y = -0.95 + 1.9 * (k + 0.5) / n_slabs
        s.transforms.append((f"slab_t{k}", (0.0, y, 0.0), (1.5, 0.004, 1.5), (0, 0, 0)))
        s.instances.append((f"slab_{k}", "Geo_Box", f"slab_t{k}", "slab_material", None, True))
    return s


def test_shadow_ray_crossing_bound(tmp_path, halton_perm, ctx):
    path = _write(tmp_path, slabs_scene(), "slabs")
    sc = Y.Scene(ctx, Y.HostScene(path, 32, 32), halton_perm)
    ctx.bound_record(clear=True)
    rc, st, _ = render_raw(sc, Y.default_setting(spp=1, ray_depth=4, volume=True))
    assert rc == -8, rc  # YMRT_ERR_OVERFLOW
    assert st.device_errors & 4  # YMRT_DEVERR_ITER
    rec = ctx.bound_record(clear=True)
    assert rec is not None and rec["site"] == 1, rec  # shadow-ray boundary crossings
    assert rec["count"] == 256
    sc.close()


def dense_majorant_scene():
    s = scenes.cornell_scene(0)
    s.textures.append(("ConstantTextureFloat", "smoke_density", {"value": 1.0}))
    s.transforms.append(("smoke_t", (0.3, 0.2, 0.0), (0.7, 0.7, 0.7), (0, 0, 0)))
    s.volumes.append(("smoke", "smoke_t", (5000.0, 5000.0, 5000.0), (0.9, 0.9, 0.9), 0.0, "smoke_density"))
    s.materials.append(("DefaultMaterial", "smoke_boundary", {"ior_n": 1.0}))
    s.instances.append(("smoke_box", "Geo_Box", "smoke_t", "smoke_boundary", "smoke", True))
    return s


def test_tracking_bound_is_the_references(tmp_path, halton_perm, ctx, oracle):
    path = _write(tmp_path, dense_majorant_scene(), "majorant")
    grid = np.full((8, 8, 8), 1e-6, np.float32)
    grid[0, 0, 0] = 1.0  # majorant 5000 per unit, density almost nowhere
    sc = Y.Scene(ctx, Y.HostScene(path, 48, 48), halton_perm)
    sc.set_density_grid(0, grid)
    ref = oracle.RefScene(path, halton_perm, 48, 48)
    ref.set_density_grid(0, grid)
    setting = Y.default_setting(spp=1, ray_depth=4, volume=True)
    ref.set_settings(spp=1, ray_depth=4, volume=1)
    rc, st, img = render_raw(sc, setting)
    ref.tracking_caps(reset=True)
    want = ref.render_frame(1)
    caps = ref.tracking_caps(reset=True)
    ref.close()
    assert rc == 0, Y.library().ymrt_last_error(ctx.h)
    assert st.device_errors == 0
    assert st.tracking_bound_hits > 0 and caps > 0
    assert abs(int(st.tracking_bound_hits) - caps) <= max(2, caps // 100), (st.tracking_bound_hits, caps)
    diff = np.abs(img[..., :3] - want[..., :3])
    bad = np.any(diff > 1e-5 * np.maximum(np.abs(img[..., :3]), np.abs(want[..., :3])) + 1e-7, axis=-1)
    assert bad.mean() <= 1e-2, bad.sum()
    sc.close()
