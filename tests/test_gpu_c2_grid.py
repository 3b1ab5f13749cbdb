"""The volumetric configuration with its density grid (C2 as configured:
1280x720, 32 spp, depth 16, the fog box and a smoke box whose density is a
128^3 float16 grid of 4-octave fBm scaled to a maximum sigma_t of 2.0).

The reference has no grid node, so the oracle's media read the same grid
values through a grid node of this project's (oracle/build_ref.py,
_MEDIA_HOOKS: trilinear over cell centres, clamped edges, majorant = the
grid's maximum). The grid is the reference's own fBm node (TextureEval, run
by the oracle) sampled at the cell centres and rounded to float16, the values
the device stores.

A path that leaves the smoke box while its nested-media stack still holds
the box (a grazing entry at an edge whose exit crossing falls below TMIN)
free-flies to infinity through the grid's clamped edge, where the density is
near zero: its delta-tracking loop then stops at the reference's
MAX_FREE_PATH_LENGTH (2048 steps) and reports a failed sample, as the
reference's does (src/VolumeEval.cuh:144). That is counted in
ymrt_stats.tracking_bound_hits, not raised: the reference's own host build
reaches the bound on the same frame (4 loops in frame 1, 3 in frame 2 of the
whole 1280x720 frame).
"""
import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

W, H = 1280, 720
GRID_N = 128
TILES = (1700, 1740)  # 40 of the frame's 3600 16x16 tiles, across the smoke box
REL_TOL, ABS_TOL = 1e-5, 1e-7


@pytest.fixture(scope="module")
def grid_values(volumetric_path, halton_perm, oracle):
    """The smoke's fBm node (texture 2) at the grid's cell centres, scaled to
    a maximum of 1 and rounded to float16 (float32 array, x fastest)."""
    ref = oracle.RefScene(volumetric_path, halton_perm, W, H)
    c = (np.arange(GRID_N, dtype=np.float32) + np.float32(0.5)) / np.float32(GRID_N) - np.float32(0.5)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    pts = np.stack([x, y, z], axis=-1).reshape(-1, 3)
    v = ref.texture(2, np.zeros((pts.shape[0], 2), np.float32), pts)[:, 0].reshape(GRID_N, GRID_N, GRID_N)
    ref.close()
    v = np.maximum(v, 0.0)
    return (v / max(float(v.max()), 1e-12)).astype(np.float16).astype(np.float32)


@pytest.fixture(scope="module")
def c2(ctx, volumetric_path, halton_perm, grid_values):
    ours = Y.Scene(ctx, Y.HostScene(volumetric_path, W, H), halton_perm)
    ours.set_density_grid(2, grid_values, half=True)
    yield ours
    ours.close()


def _ref(oracle, path, perm, grid, fp64=False):
    r = oracle.RefScene(path, perm, W, H, fp64=fp64)
    r.set_density_grid(2, grid)
    return r


def _setting(spp):
    return Y.default_setting(spp=spp, ray_depth=16, volume=True)


def test_grid_read_equals_oracle(c2, volumetric_path, halton_perm, oracle, grid_values):
    """The device's grid read (ymrt_debug_density) equals the oracle's grid
    node bit for bit at points inside and outside the box."""
    rng = np.random.default_rng(11)
    pts = rng.uniform(-0.7, 0.7, (20000, 3)).astype(np.float32)
    ref = _ref(oracle, volumetric_path, halton_perm, grid_values)
    want = ref.density(2, pts)
    ref.close()
    assert np.array_equal(c2.density(2, pts), want)


def test_c2_frame_has_no_device_errors(c2):
    """The whole C2 frame renders without a device error; tracking loops that
    stop at the reference's 2048-step bound are counted, a handful per frame
    as in the reference's own run."""
    for frame in (1, 2):
        img, stats = c2.render(_setting(32), frame)  # raises on a device error
        assert stats.device_errors == 0
        assert stats.paths == W * H * 32
        print(f"C2 frame {frame}: {stats.extension_rays + stats.shadow_rays} rays, "
              f"{stats.tracking_bound_hits} tracking loops at the 2048-step bound")
        assert stats.tracking_bound_hits <= 32
        assert np.all(np.isfinite(img)) and np.allclose(img[..., 3], 1.0, atol=1e-5)


@pytest.mark.parametrize("frame", [1, 2])
def test_c2_per_sample_band(c2, volumetric_path, halton_perm, oracle, grid_values, frame):
    """One path per pixel over a band of tiles through the smoke box: radiance
    within 1e-5 relative per pixel against the reference's own estimator on
    the same grid, equal coverage, equal ray and tracking-bound counts up to
    the few paths a last-bit transcendental difference sends another way."""
    ref = _ref(oracle, volumetric_path, halton_perm, grid_values)
    ref.set_settings(spp=1, ray_depth=16, volume=1)
    oracle.query_counts(reset=True)
    ref.tracking_caps(reset=True)
    b = ref.render_frame(frame, *TILES)
    ext, shadow = oracle.query_counts(reset=True)
    caps = ref.tracking_caps(reset=True)
    ref.close()
    a, stats = c2.render(_setting(1), frame, tile_begin=TILES[0], tile_end=TILES[1])
    assert np.array_equal(a[..., 3], b[..., 3])
    diff = np.abs(a[..., :3] - b[..., :3])
    bad = np.any(diff > REL_TOL * np.maximum(np.abs(a[..., :3]), np.abs(b[..., :3])) + ABS_TOL, axis=-1)
    n_pix = int((b[..., 3] > 0).sum())
    print(f"frame {frame}: {int(bad.sum())} of {n_pix} pixels beyond 1e-5 relative; tracking bound "
          f"{stats.tracking_bound_hits} (reference {caps})")
    assert bad.sum() <= 5e-3 * n_pix
    assert stats.device_errors == 0
    assert abs(int(stats.extension_rays) - ext) <= 0.01 * ext
    assert abs(int(stats.shadow_rays) - shadow) <= 0.01 * shadow
    assert abs(int(stats.tracking_bound_hits) - caps) <= 1


def test_c2_converged_band_vs_fp64(c2, volumetric_path, halton_perm, oracle, grid_values):
    """32 spp on the band: RMSE against the FP64 oracle (same grid values)
    within 1e-3, or no further than the reference's float code (x1.5)."""
    if not oracle.available64():
        pytest.skip("FP64 oracle unavailable")
    f32 = _ref(oracle, volumetric_path, halton_perm, grid_values)
    f64 = _ref(oracle, volumetric_path, halton_perm, grid_values, fp64=True)
    for r in (f32, f64):
        r.set_settings(spp=32, ray_depth=16, volume=1)
    b = f32.render_frame(1, *TILES)
    c = f64.render_frame(1, *TILES)
    f32.close()
    f64.close()
    a, stats = c2.render(_setting(32), 1, tile_begin=TILES[0], tile_end=TILES[1])
    cov = c[..., 3] > 0
    assert np.array_equal(a[..., 3] > 0, cov)
    rmse_ours = float(np.sqrt(np.mean((a[..., :3][cov].astype(np.float64) - c[..., :3][cov]) ** 2)))
    rmse_ref = float(np.sqrt(np.mean((b[..., :3][cov].astype(np.float64) - c[..., :3][cov]) ** 2)))
    print(f"C2 grid band: RMSE vs FP64 ymrt_b200 {rmse_ours:.3e}, reference float {rmse_ref:.3e}")
    assert stats.device_errors == 0
    assert rmse_ours <= max(1e-3, 1.5 * rmse_ref), (rmse_ours, rmse_ref)
