"""ymrt_debug_record_paths: recording leaves the render as it is (up to the
order of a pixel's float additions: shadow rays are traced in the shading
stage while recording), and each watched path is recorded vertex after
vertex, each ray starting where the previous one hit; against the host
oracle the first difference along a path is a last-bit one. (Against the
reference's device build every recorded vertex is equal bit for bit:
test_gpu_refcuda.py.)"""
import numpy as np
import pytest

import divergence as D
import ymrt_b200 as Y

pytestmark = pytest.mark.gpu


def test_recorded_paths_follow_the_render(ctx, cornell_path, halton_perm, oracle):
    ours = Y.Scene(ctx, Y.HostScene(cornell_path, 128, 128), halton_perm)
    ref = oracle.RefScene(cornell_path, halton_perm, 128, 128)
    ref.set_settings(spp=1, ray_depth=8)
    s = Y.default_setting(spp=1, ray_depth=8)
    plain, _ = ours.render(s, 2)
    pixels = np.arange(0, 128 * 128, 97)
    rec, img = ours.record_paths(s, pixels, 2)
    assert np.allclose(img, plain, rtol=1e-5, atol=1e-7)
    assert set(rec["pixel"].tolist()) == set(pixels.tolist())
    for p in pixels[:40]:
        v = rec[rec["pixel"] == p]
        assert v["depth"][0] == 1 and np.all(np.diff(v["depth"].astype(np.int64)) == 1)
        for k in range(len(v) - 1):
            hit = v[k]["o"].astype(np.float64) + v[k]["d"].astype(np.float64) * float(v[k]["t"])
            assert np.abs(hit - v[k + 1]["o"]).max() < 1e-3 * (1.0 + np.abs(hit).max())
    # against the host oracle the same paths differ at most in last bits
    # (its math library), except where they take another branch
    rrec, _ = ref.record_paths(pixels, 2)
    far = 0
    for p in pixels:
        a, b = rec[rec["pixel"] == p], rrec[rrec["pixel"] == p]
        for x, y in zip(a, b):
            f = D.first_difference(x, y)
            if f is not None:
                far += f[0] != "last_bit"
                break
    assert far <= 3
    ours.close()
    ref.close()
