"""GPU parity for the analytic shapes: Sphere and Cube blocks.

The spheres scene is the Cornell-like room with a built-in unit cube, a
smooth dielectric sphere (transmission 1, IOR 1.55), a rough conductor
sphere, a small emissive sphere (a sphere shape light, sampled by the cone it
subtends) and a medium-filled boundary sphere that encloses the camera.
Closest-hit and any-hit queries must equal the oracle's bit for bit (t, the
object-space hit point a sphere hit carries in the barycentric slots, the
back-face flag); one-sample-per-pixel frames must agree within 1e-5 relative
radiance per pixel, with and without the medium.
"""
import numpy as np
import pytest

import divergence as D
import ymrt_b200 as Y
from test_gpu_parity import _trace_case

pytestmark = pytest.mark.gpu

W = H = 256


@pytest.fixture(scope="module")
def spheres_path(scene_dir):
    from ymrt_b200 import scenes
    return scenes.scene_path("spheres", 0, scene_dir)


@pytest.fixture(scope="module")
def spheres(ctx, spheres_path, halton_perm, oracle):
    ours = Y.Scene(ctx, Y.HostScene(spheres_path, W, H), halton_perm)
    ref = oracle.RefScene(spheres_path, halton_perm, W, H)
    yield ours, ref
    ours.close()
    ref.close()


def test_trace_kat_spheres(spheres):
    hits, _ = _trace_case(spheres, 20000, 13)
    assert hits > 10000


def test_occlusion_kat_spheres(spheres):
    ours, ref = spheres
    rng = np.random.default_rng(17)
    n = 20000
    o = rng.uniform(-0.95, 0.95, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    tmax = rng.uniform(0.05, 3.0, n).astype(np.float32)
    a = ours.occluded(o, d, tmax)
    b = ref.occluded(o, d, tmax)
    assert np.array_equal(a, b), f"occlusion differs on {np.sum(a != b)} rays"
    assert 0 < a.sum() < n


@pytest.mark.parametrize("volume", [0, 1])
@pytest.mark.parametrize("frame", [1, 2])
def test_per_sample_radiance_spheres(spheres, oracle, volume, frame):
    ours, ref = spheres
    s = Y.default_setting(spp=1, ray_depth=8, volume=bool(volume))
    ref.set_settings(spp=1, ray_depth=8, volume=volume)
    oracle.query_counts(reset=True)
    a, stats = ours.render(s, frame)
    b = ref.render_frame(frame)
    ext, shadow = oracle.query_counts(reset=True)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_host(f"spheres_v{volume}_f{frame}", ours, ref, s, frame, a, b)
    assert stats.device_errors == 0
    assert abs(int(stats.extension_rays) - ext) <= 0.01 * ext
    assert abs(int(stats.shadow_rays) - shadow) <= 0.01 * shadow


def test_converged_spheres_16spp(spheres):
    ours, ref = spheres
    s = Y.default_setting(spp=16, ray_depth=8)
    ref.set_settings(spp=16, ray_depth=8)
    a, _ = ours.render(s, 1)
    b = ref.render_frame(1)
    rmse = float(np.sqrt(np.mean((a[..., :3] - b[..., :3]) ** 2)))
    assert rmse <= 1e-3, rmse
    # the sphere light is visible and lit: the frame is not just background
    assert float(a[..., :3].max()) > 1.0


@pytest.mark.parametrize("sort_hits,defer_shadows", [(1, 1), (0, 0)])
def test_wave_options_spheres(ctx, spheres, sort_hits, defer_shadows):
    ours, ref = spheres
    before = {k: ctx.get_option(k) for k in ("sort_hits", "defer_shadows")}
    try:
        ctx.set_option("sort_hits", sort_hits)
        ctx.set_option("defer_shadows", defer_shadows)
        s = Y.default_setting(spp=1, ray_depth=8)
        ref.set_settings(spp=1, ray_depth=8)
        a, _ = ours.render(s, 3)
        b = ref.render_frame(3)
        D.check_against_host("spheres_v0_f3", ours, ref, s, 3, a, b)
    finally:
        for k, v in before.items():
            ctx.set_option(k, v)
