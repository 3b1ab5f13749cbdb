"""GPU parity for texture nodes, textured materials and normal / bump maps.

Every node of the generated ``textured`` scene is evaluated on the device
(ymrt_debug_texture) at seeded texture coordinates and object-space points
and compared with the reference's TextureEval run by the oracle: equal bit
for bit for the nodes built from arithmetic and floor (constants, noise, fBm,
turbulence, wood, polka dot, wave), and within a few ulp for the nodes that
take a sine (checkerboard: its sign only; marble), where CUDA's sinf and the
host's sinf may round differently. Whole frames of the textured scene (every
solid node on material parameters, a normal map, a bump map, a noise-density
medium) must agree with the oracle within 1e-5 relative radiance per pixel,
with the same ray counts. In the adjoint pass a textured parameter's constant
receives no gradient.
"""
import numpy as np
import pytest

import divergence as D
import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

W = H = 256


@pytest.fixture(scope="module")
def textured_path(scene_dir):
    from ymrt_b200 import scenes
    return scenes.scene_path("textured", 0, scene_dir)


@pytest.fixture(scope="module")
def textured(ctx, textured_path, halton_perm, oracle):
    ours = Y.Scene(ctx, Y.HostScene(textured_path, W, H), halton_perm)
    ref = oracle.RefScene(textured_path, halton_perm, W, H)
    yield ours, ref
    ours.close()
    ref.close()


def test_texture_nodes_match_reference(textured, textured_path):
    ours, ref = textured
    rec = Y.HostScene(textured_path, 16, 16).records("textures")

    def subtree(k):  # node types of k and everything below it
        t = {int(rec[k, 0])}
        if 3 <= rec[k, 0] <= 10:
            t |= subtree(int(rec[k, 1])) | subtree(int(rec[k, 2]))
        return t

    rng = np.random.default_rng(23)
    n = 20000
    st = rng.uniform(-2.0, 5.0, (n, 2)).astype(np.float32)
    p = rng.uniform(-1.5, 1.5, (n, 3)).astype(np.float32)
    for k in range(rec.shape[0]):
        a = ours.texture(k, st, p)
        b = ref.texture(k, st, p)
        sub = subtree(k)
        close = np.isclose(a, b, rtol=4e-6, atol=4e-7).all(axis=1)
        if 3 in sub:  # a checkerboard selects by the sign of a product of sines
            assert (~close).mean() <= 1e-4, (k, (~close).mean())
        elif 7 in sub:  # marble: sinf of the phase
            assert close.all(), (k, np.abs(a - b).max())
        else:
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (k, sub, np.abs(a - b).max())


@pytest.mark.parametrize("volume", [0, 1])
@pytest.mark.parametrize("frame", [1, 2])
def test_per_sample_radiance_textured(textured, oracle, volume, frame):
    ours, ref = textured
    s = Y.default_setting(spp=1, ray_depth=8, volume=bool(volume))
    ref.set_settings(spp=1, ray_depth=8, volume=volume)
    oracle.query_counts(reset=True)
    a, stats = ours.render(s, frame)
    b = ref.render_frame(frame)
    ext, shadow = oracle.query_counts(reset=True)
    assert np.array_equal(a[..., 3], b[..., 3])
    assert a[..., :3].mean() > 0.01
    D.check_against_host(f"textured_v{volume}_f{frame}", ours, ref, s, frame, a, b)
    assert stats.device_errors == 0
    assert abs(int(stats.extension_rays) - ext) <= 0.01 * ext
    assert abs(int(stats.shadow_rays) - shadow) <= 0.01 * shadow


def test_textured_parameters_get_no_gradient(ctx, textured_path, halton_perm):
    """Material gradients (albedo rgb, roughness) of the textured scene: the
    floor's albedo comes from a checkerboard, so its albedo constant has no
    effect and gets exactly zero, and so does the back wall's roughness
    (noise); the untextured ceiling's albedo gets a gradient."""
    import torch
    from diff_harness import MultiViewRenderer
    scene = Y.Scene(ctx, Y.HostScene(textured_path, 64, 64), halton_perm)
    r = MultiViewRenderer(ctx, [scene], Y.default_setting(spp=4, ray_depth=6), frame_index=1)
    r.forward()
    rng = np.random.default_rng(5)
    w = [torch.as_tensor(rng.uniform(0.0, 1.0, tuple(img.shape)).astype(np.float32), device="cuda")
         for img in r.images]
    g = r.backward(w).cpu().numpy()
    floor, ceiling, back = 0, 1, 2  # material order of the Cornell-like room
    assert np.all(g[floor, :3] == 0.0)
    assert g[back, 3] == 0.0
    assert np.any(g[ceiling, :3] != 0.0)
    scene.close()


@pytest.fixture(scope="module")
def imaged(ctx, scene_dir, halton_perm, oracle):
    from ymrt_b200 import scenes
    path = scenes.scene_path("imaged", 0, scene_dir)
    ours = Y.Scene(ctx, Y.HostScene(path, W, H), halton_perm)
    ref = oracle.RefScene(path, halton_perm, W, H)
    yield ours, ref, Y.HostScene(path, 16, 16).records("textures")
    ours.close()
    ref.close()


def test_image_nodes_match_reference(imaged):
    """Bilinear image fetches (repeat wrap, negative and >1 coordinates,
    1-4 channels) equal the reference's EvalTexImage bit for bit."""
    ours, ref, rec = imaged
    rng = np.random.default_rng(31)
    n = 20000
    st = rng.uniform(-3.0, 4.0, (n, 2)).astype(np.float32)
    p = rng.uniform(-1.0, 1.0, (n, 3)).astype(np.float32)
    for k in range(rec.shape[0]):
        a, b = ours.texture(k, st, p), ref.texture(k, st, p)
        if rec[k, 0] == 3:  # the checkerboard of two images: its selection may flip where the sines' product is ~0
            assert np.mean(np.any(a != b, axis=1)) <= 1e-4, k
        else:
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (k, np.abs(a - b).max())


@pytest.mark.parametrize("frame", [1, 2])
def test_per_sample_radiance_imaged(imaged, oracle, frame):
    """One-sample frames of the image scene. Its bump map (a 2-bit image
    differenced over a 0.0005 texture-coordinate step) turns last-place
    differences of a path's earlier directions (sampling's sinf / cosf on the
    device against the host's) into larger normal differences, so more
    pixels pass 1e-5 than in the other scenes, and a few paths take another
    branch (the frames themselves are pinned bit for bit by
    test_shading_frames_match_reference). Every differing pixel is replayed
    and classified (tests/divergence.py), their number bounded by the count
    observed; at most 0.2% of the pixels beyond 1e-3, and the image means
    within 2e-4."""
    ours, ref, _ = imaged
    s = Y.default_setting(spp=1, ray_depth=8)
    ref.set_settings(spp=1, ray_depth=8)
    oracle.query_counts(reset=True)
    a, stats = ours.render(s, frame)
    b = ref.render_frame(frame)
    ext, shadow = oracle.query_counts(reset=True)
    assert np.array_equal(a[..., 3], b[..., 3])
    assert a[..., :3].mean() > 0.01
    D.check_against_host(f"imaged_f{frame}", ours, ref, s, frame, a, b)
    diff = np.abs(a[..., :3] - b[..., :3]) / np.maximum(np.maximum(np.abs(a[..., :3]), np.abs(b[..., :3])), 1e-6)
    assert np.mean(np.any(diff > 1e-3, axis=-1)) <= 2e-3
    assert abs(float(a[..., :3].mean()) - float(b[..., :3].mean())) <= 2e-4 * float(b[..., :3].mean())
    assert stats.device_errors == 0
    assert abs(int(stats.extension_rays) - ext) <= 0.01 * ext
    assert abs(int(stats.shadow_rays) - shadow) <= 0.01 * shadow


@pytest.mark.parametrize("scene_name", ["imaged", "textured"])
def test_shading_frames_match_reference(ctx, scene_dir, halton_perm, oracle, scene_name):
    """Normal, tangent and bitangent after normal / bump mapping, the texture
    footprint, object-space position and dp/du at 20,000 hits: equal to the
    reference's FetchShadingData + TextureCoordinatesDifferential +
    InitShadingSpace bit for bit. Texture coordinates too, except on spheres,
    whose angles come from acosf / atan2f (CUDA's and the host's may differ in
    the last place)."""
    from ymrt_b200 import scenes
    path = scenes.scene_path(scene_name, 0, scene_dir)
    ours = Y.Scene(ctx, Y.HostScene(path, W, H), halton_perm)
    ref = oracle.RefScene(path, halton_perm, W, H)
    rng = np.random.default_rng(41)
    n = 20000
    o = rng.uniform(-0.9, 0.9, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    hit = ref.trace(o, d)
    m = hit["inst"] != 0xFFFFFFFF
    args = (hit["inst"][m], hit["tri"][m], hit["bary"][m], hit["back"][m], d[m])
    a = ours.shading_frame(*args)
    b = ref.shading_frame(*args)
    names = ["n"] * 3 + ["t"] * 3 + ["b"] * 3 + ["footprint"] * 4 + ["uv"] * 2 + ["p_obj"] * 3 + ["dpdu"] * 3 + ["mat"]
    for c in range(22):
        bad = a[:, c].view(np.uint32) != b[:, c].view(np.uint32)
        if names[c] == "uv":
            bad &= ~np.isclose(a[:, c], b[:, c], rtol=1e-6, atol=1e-7)
        assert not bad.any(), (names[c], c, int(bad.sum()), a[bad][:3, c], b[bad][:3, c], a[bad][:3, 21])
    ours.close()
    ref.close()
