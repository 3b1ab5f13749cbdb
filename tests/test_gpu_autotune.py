"""The autotuner on the GPU: it measures every point of a small space and the
configuration it picks renders the same image as the defaults."""
import numpy as np
import pytest

import ymrt_b200 as Y
from ymrt_b200 import autotune

pytestmark = pytest.mark.gpu


def test_tune_scene_and_apply(cornell_path, halton_perm, tmp_path):
    import torch
    setting = Y.default_setting(spp=4, ray_depth=8)
    space = {"queue_capacity": [1 << 16, 1 << 18], "sort_hits": [0, 1], "defer_shadows": [1],
             "max_leaf_triangles": [2, 4]}
    cache = str(tmp_path / "tune.json")
    r = autotune.tune_scene(cornell_path, 128, 128, setting, halton_perm, space=space, cache_file=cache)
    assert len(r["table"]) == 8 and all(t["ms"] and t["ms"] > 0 for t in r["table"])
    assert r["ms"] == min(t["ms"] for t in r["table"])
    assert autotune.tune_scene(cornell_path, 128, 128, setting, halton_perm, space=space, cache_file=cache) == r

    ctx = Y.Context(0)
    ref_img, _ = Y.Scene(ctx, Y.HostScene(cornell_path, 128, 128), halton_perm).render(setting, 2)
    autotune.apply(ctx, r["best"])
    scene = Y.Scene(ctx, Y.HostScene(cornell_path, 128, 128, max_leaf_triangles=r["best"]["max_leaf_triangles"]),
                    halton_perm)
    img, st = scene.render(setting, 2)
    assert st.device_errors == 0
    assert np.array_equal(img[..., 3], ref_img[..., 3])
    diff = np.abs(img[..., :3] - ref_img[..., :3])
    bad = np.any(diff > 1e-5 * np.maximum(np.abs(img[..., :3]), np.abs(ref_img[..., :3])) + 1e-7, axis=-1)
    assert bad.mean() <= 2e-3  # (a different leaf size may resolve an exact-t tie the other way)
    scene.close()
    ctx.close()
