"""Transform edits rebuilt on the device (ymrt_scene_set_transforms) against
the same edits rebuilt on the host (ymrt_host_scene_set_transforms, itself
pinned to the reference editor's rebuild in tests/test_transform_edit.py).

After each edit the device's top-level nodes, leaf instances, instance
order, shading buckets, file indices, shape lights, light table and camera
media stack equal those of the host-edited scene uploaded afresh, byte for
byte, and both render the same frame.
"""
import time

import numpy as np
import pytest

import ymrt_b200 as Y
from test_transform_edit import edit_matrices

pytestmark = pytest.mark.gpu

PARTS = ["tlas_nodes", "tlas_prims", "instances", "instance_buckets", "file_index", "shape_lights", "light_table",
         "camera_media"]


@pytest.mark.parametrize("name,size", [("cornell", (128, 128)), ("volumetric", (128, 128)),
                                       ("spheres", (128, 128)), ("instanced", (320, 180))])
def test_device_rebuild_equals_host_rebuild(ctx, name, size, scene_dir, halton_perm):
    from ymrt_b200 import scenes
    path = scenes.scene_path(name, 0, scene_dir)
    host = Y.HostScene(path, *size)
    dev = Y.Scene(ctx, host, halton_perm)
    n_t = host.transforms()[0].shape[0]
    volume = name in ("volumetric", "spheres")
    setting = Y.default_setting(spp=1, ray_depth=8, volume=volume)
    t_dev = t_host = 0.0
    for step, first in enumerate([0, n_t // 2, max(0, n_t - 3)]):
        count = min(3, n_t - first)
        m, s = edit_matrices(200 + step, count, host, first)
        t = time.perf_counter()
        dev.set_transforms(first, m, s)
        t_dev += time.perf_counter() - t
        t = time.perf_counter()
        host.set_transforms(first, m, s)
        fresh = Y.Scene(ctx, host, halton_perm)
        t_host += time.perf_counter() - t
        for part in PARTS:
            a, b = dev.download(part), fresh.download(part)
            assert a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8)), f"edit {step}: {part}"
        ia, _ = dev.render(setting, step + 1)
        ib, _ = fresh.render(setting, step + 1)
        np.testing.assert_allclose(ia, ib, rtol=1e-5, atol=1e-7, err_msg=f"edit {step}: image")
        fresh.close()
    print(f"{name}: device rebuild {t_dev / 3 * 1e3:.2f} ms per edit, host rebuild + upload {t_host / 3 * 1e3:.2f} ms")
    dev.close()
