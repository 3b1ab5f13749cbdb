"""Continuing rays traced grouped by origin cell and direction
(YMRT_OPT_SORT_RAYS, one of the choices ymrt_b200.autotune tunes): the
grouping changes only the order in which slots are traced, so with it on and
off a frame traces the same rays through the same nodes (equal ray, node
and triangle counts) and renders the same image up to the order of a pixel's
float additions; on surfaces and in media, on several waves of paths."""
import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scene,volume", [("instanced", False), ("volumetric", True), ("spheres", False)])
def test_grouped_rays_render_alike(scene, volume, scene_dir, halton_perm):
    from ymrt_b200 import scenes
    path = scenes.scene_path(scene, 0, scene_dir)
    ctx = Y.Context(0, queue_capacity=1 << 16)  # several waves, so most paths continue from an earlier one
    sc = Y.Scene(ctx, Y.HostScene(path, 320, 240), halton_perm)
    setting = Y.default_setting(spp=4, ray_depth=8, volume=volume)
    out = {}
    for on in (1, 0):
        ctx.set_option("sort_rays", on)
        assert ctx.get_option("sort_rays") == on
        img, st = sc.render(setting, 3)
        assert st.device_errors == 0 and st.waves > 4
        out[on] = (img, st.as_dict())
    a, b = out[1][1], out[0][1]
    for k in ("paths", "extension_rays", "shadow_rays", "node_visits", "triangle_tests", "shadow_node_visits"):
        assert a[k] == b[k], (k, a[k], b[k])
    np.testing.assert_allclose(out[1][0], out[0][0], rtol=1e-5, atol=1e-7)
    sc.close()
    ctx.close()
