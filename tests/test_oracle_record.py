"""The oracle's path-vertex recording hook (used to classify per-sample
divergences): recording changes nothing in the render, every watched pixel
gets its vertices in wave order with depths from 1 up (a crossing of an
index-matched medium boundary continues at the same depth), and each
vertex's ray starts where the previous one hit."""
import numpy as np
import pytest


@pytest.mark.parametrize("scene", ["cornell", "spheres"])
def test_recording_follows_each_watched_path(scene, scene_dir, halton_perm, oracle):
    from ymrt_b200 import scenes
    path = scenes.scene_path(scene, 0, scene_dir)
    r = oracle.RefScene(path, halton_perm, 64, 64)
    r.set_settings(spp=1, ray_depth=8)
    plain = r.render_frame(2)
    pixels = [0, 37, 100, 2080, 2081, 4095]
    rec, img = r.record_paths(pixels, 2)
    assert np.array_equal(plain.view(np.uint32), img.view(np.uint32))
    assert set(rec["pixel"].tolist()) == set(pixels)
    for p in pixels:
        v = rec[rec["pixel"] == p]
        depth = v["depth"].astype(np.int64)
        assert depth[0] == 1 and np.all(np.diff(depth) >= 0) and np.all(np.diff(depth) <= 1)
        for k in range(len(v) - 1):
            assert v[k]["flags"] & 1  # a path continues only after a hit
            hit_point = v[k]["o"].astype(np.float64) + v[k]["d"].astype(np.float64) * float(v[k]["t"])
            assert np.abs(hit_point - v[k + 1]["o"]).max() < 1e-3 * (1.0 + np.abs(hit_point).max())
    r.close()
