"""GPU parity for participating media and distant lights.

The volumetric scene is the Cornell-like box filled with a homogeneous,
forward-scattering fog volume (a boundary box with priority 0) that contains
a heterogeneous smoke box (fBm density, priority 1), lit by the ceiling quad
and by a sun (a distant light with a 5 degree cone) shining in through the
open front. Each setting renders one path per pixel through the C ABI and
through the oracle (the reference built for the host) with identical Halton
tables; radiance must agree within 1e-5 relative per pixel. Free-flight
sampling and ratio tracking evaluate expf/logf many times per path, so a
path whose transcendental differs in its last bit between CUDA and glibc may
take a different branch: every differing pixel is replayed and classified,
and their number is bounded by the count observed (tests/divergence.py).
"""
import numpy as np
import pytest

import divergence as D
import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

W = H = 256


@pytest.fixture(scope="module")
def volumetric(ctx, volumetric_path, halton_perm, oracle):
    ours = Y.Scene(ctx, Y.HostScene(volumetric_path, W, H), halton_perm)
    ref = oracle.RefScene(volumetric_path, halton_perm, W, H)
    yield ours, ref
    ours.close()
    ref.close()


@pytest.mark.parametrize("distant,volume", [(1, 0), (0, 1), (1, 1)])
@pytest.mark.parametrize("frame", [1, 2])
def test_per_sample_radiance_volumetric(volumetric, oracle, distant, volume, frame):
    ours, ref = volumetric
    s = Y.default_setting(spp=1, ray_depth=8, distant_light=bool(distant), volume=bool(volume))
    ref.set_settings(spp=1, ray_depth=8, distant_light=distant, volume=volume)
    oracle.query_counts(reset=True)
    a, stats = ours.render(s, frame)
    b = ref.render_frame(frame)
    ext, shadow = oracle.query_counts(reset=True)
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_host(f"volumetric_d{distant}v{volume}_f{frame}", ours, ref, s, frame, a, b)
    assert stats.device_errors == 0
    # ray counts follow the same paths: equal up to the few diverged ones
    assert abs(int(stats.extension_rays) - ext) <= 0.01 * ext
    assert abs(int(stats.shadow_rays) - shadow) <= 0.01 * shadow


def test_converged_volumetric_16spp(volumetric):
    ours, ref = volumetric
    s = Y.default_setting(spp=16, ray_depth=8, distant_light=True, volume=True)
    ref.set_settings(spp=16, ray_depth=8, distant_light=1, volume=1)
    a, stats = ours.render(s, 1)
    b = ref.render_frame(1)
    rmse = float(np.sqrt(np.mean((a[..., :3] - b[..., :3]) ** 2)))
    assert rmse <= 1e-3, rmse
    assert np.allclose(a[..., 3], 1.0, atol=1e-6)
    assert stats.device_errors == 0


def test_volumes_off_matches_surface_kernels(volumetric):
    """With volume scattering off, the volumetric scene renders exactly like a
    scene of the same surfaces: the media's boundary boxes are passed through
    (index-matched) and only change the nested-media stack."""
    ours, ref = volumetric
    s = Y.default_setting(spp=1, ray_depth=8)
    ref.set_settings(spp=1, ray_depth=8)
    a, _ = ours.render(s, 3)
    b = ref.render_frame(3)
    D.check_against_host("volumetric_d0v0_f3", ours, ref, s, 3, a, b)
