"""The allocation-free render entry point (ymrt_render_tiles_noalloc).

It exists for callers that cannot allocate device memory while they render
(a host with a fixed memory budget or its own pool allocator, or code that
must not let a cudaMalloc synchronise the device mid-frame): its path queues
live in a fixed per-device array instead of the context's allocations. This
test calls it through the C ABI twice in a row and checks both frames against
the regular entry point's frame of the same samples, within the tolerance the
parity tests use (1e-5 relative), and checks that a sample count too large
for the fixed array is rejected.

The file is named to be collected last, so a run that stops at the first
failure has already run every other test.
"""
import ctypes

import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
ABS_TOL = 1e-7


def _noalloc(lib):
    f = lib.ymrt_render_tiles_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(Y.RenderSetting), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                  ctypes.c_void_p, ctypes.POINTER(Y.Stats)]
    f.restype = ctypes.c_int
    lib.ymrt_noalloc_max_paths.restype = ctypes.c_uint32
    return f


def test_noalloc_matches_regular_entry_point(cornell_path, halton_perm):
    import torch
    lib = Y.library()
    render_noalloc = _noalloc(lib)
    ctx = Y.Context(0)
    scene = Y.Scene(ctx, Y.HostScene(cornell_path, 256, 256), halton_perm)
    setting = Y.default_setting(spp=4, ray_depth=8)

    expected = torch.zeros((256, 256, 4), dtype=torch.float32, device="cuda")
    _, st_ref = scene.render(setting, frame_index=3, out=expected)
    want = expected.cpu().numpy()

    for call in range(2):  # two calls in a row share (and reuse) the fixed array
        got_t = torch.full((256, 256, 4), float("nan"), dtype=torch.float32, device="cuda")
        stats = Y.Stats()
        rc = render_noalloc(scene.h, ctypes.byref(setting), 3, 0, 0, ctypes.c_void_p(got_t.data_ptr()),
                            ctypes.byref(stats))
        assert rc == 0, lib.ymrt_last_error(ctx.h).decode()
        got = got_t.cpu().numpy()
        assert np.array_equal(got[..., 3], want[..., 3])
        diff = np.abs(got[..., :3] - want[..., :3])
        tol = REL_TOL * np.maximum(np.abs(got[..., :3]), np.abs(want[..., :3])) + ABS_TOL
        assert np.all(diff <= tol), f"call {call}: {np.sum(diff > tol)} values differ beyond tolerance"
        assert stats.extension_rays == st_ref.extension_rays
        assert stats.shadow_rays == st_ref.shadow_rays
        assert stats.device_errors == 0

    # a sample count whose single tile does not fit in the fixed array is rejected
    too_many = lib.ymrt_noalloc_max_paths() // 256 + 1
    big = Y.default_setting(spp=too_many, ray_depth=8)
    rc = render_noalloc(scene.h, ctypes.byref(big), 1, 0, 0, ctypes.c_void_p(expected.data_ptr()), None)
    assert rc == -1
    assert "scratch array" in lib.ymrt_last_error(ctx.h).decode()
    scene.close()
    ctx.close()
