"""Block shape of the closest-hit and shadow-ray kernels (YMRT_OPT_TRACE_BLOCK,
one of the choices ymrt_b200.autotune tunes): 64-, 128- and 256-thread blocks
render the same frame (one path per pixel: equal up to the order of a
pixel's float additions), with media and without."""
import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scene,volume", [("instanced", False), ("volumetric", True)])
def test_block_shapes_render_alike(scene, volume, scene_dir, halton_perm):
    from ymrt_b200 import scenes
    path = scenes.scene_path(scene, 0, scene_dir)
    ctx = Y.Context(0)
    sc = Y.Scene(ctx, Y.HostScene(path, 320, 240), halton_perm)
    setting = Y.default_setting(spp=1, ray_depth=8, volume=volume)
    images = {}
    for tb in (128, 64, 256):
        ctx.set_option("trace_block", tb)
        assert ctx.get_option("trace_block") == tb
        images[tb], st = sc.render(setting, 3)
        assert st.device_errors == 0
    for tb in (64, 256):
        np.testing.assert_allclose(images[tb], images[128], rtol=1e-5, atol=1e-7, err_msg=f"{tb} threads")
    with pytest.raises(Y.YmrtError):
        ctx.set_option("trace_block", 96)
    sc.close()
    ctx.close()
