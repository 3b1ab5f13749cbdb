"""GPU parity for the editor view and post-processing.

The editor's albedo / picking view (ymrt_render_editor_view) against the
reference's three editor stages run by the oracle with the same camera:
the primitive-index image must be equal (up to exact ties), and the colour
image equal (bit for bit where no texture is read; within 1e-5 relative on
textured surfaces, where marble's sinf and the spheres' acosf / atan2f may
round differently on the device). The spheres
scene's camera sits inside a medium boundary sphere, so every camera ray
passes through a boundary first. Tone mapping (ACES, 1/gamma; powf on the
device against the host's) and the selection outline against the
reference's Gamma_correction_common and Draw_outline.
"""
import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["cornell", "spheres", "textured", "imaged"])
@pytest.mark.parametrize("env", [False, True])
def test_editor_view_matches_reference(ctx, scene_dir, halton_perm, oracle, name, env):
    from ymrt_b200 import scenes
    path = scenes.scene_path(name, 0, scene_dir)
    w, h = 200, 150
    ours = Y.Scene(ctx, Y.HostScene(path, w, h), halton_perm)
    ref = oracle.RefScene(path, halton_perm, w, h)
    ref.set_settings(spp=1, ray_depth=8, env_light=int(env))
    a, pa = ours.editor_view(Y.default_setting(spp=1, env_light=env))
    b, pb = ref.editor_view()
    # an exact tie (equal t on two instances where they meet) may resolve to the other instance: the
    # reference keeps the later hit of its binary traversal order, an 8-wide traversal visits in another
    # order (seen: one pixel of the textured scene, on the floor / wall seam)
    assert (pa != pb).sum() <= (0 if name in ("cornell", "spheres") else 2)
    assert (pa != 0xFFFFFFFF).mean() > 0.5
    assert np.array_equal(a[..., 3], b[..., 3])
    if name in ("cornell", "spheres"):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    else:
        bad = ~np.isclose(a, b, rtol=1e-5, atol=1e-7).all(axis=-1)
        assert bad.mean() <= 1e-3, bad.sum()
    ours.close()
    ref.close()


def test_post_process_matches_reference(ctx, oracle):
    rng = np.random.default_rng(3)
    h, w = 61, 83
    img = rng.uniform(0.0, 4.0, (h, w, 4)).astype(np.float32)
    prim = rng.integers(0, 4, (h, w)).astype(np.uint32)
    for selected, outline, gamma, exposure in ((0xFFFFFFFF, False, 2.2, 1.0), (2, True, 2.2, 0.8), (1, True, 1.8, 1.5)):
        a = Y.post_process(ctx, img, prim, selected, gamma, exposure, outline)
        b = oracle.post_process(img, prim, selected, gamma, exposure, outline)
        assert np.array_equal(a[..., 3], b[..., 3])
        assert np.allclose(a, b, rtol=2e-6, atol=1e-7), np.abs(a - b).max()
        if outline:
            red = np.all(b[..., :3] == np.float32([1.0, 0.0, 0.0]), axis=-1)
            assert red.any() and np.array_equal(red, np.all(a[..., :3] == np.float32([1.0, 0.0, 0.0]), axis=-1))
