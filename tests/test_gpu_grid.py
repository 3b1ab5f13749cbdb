"""Density grids (kTexGrid): the lattice read, and media rendered through it.

The reference's texture graph has no grid node, so the grid is pinned three
ways: its trilinear read against a numpy restatement of the same float32
arithmetic (bit for bit), a constant grid against the reference's constant
density texture per sample (the oracle renders the constant), and a grid
sampled from the scene's fBm node against that node in a converged image.
"""
import numpy as np
import pytest

import divergence as D
import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

FBM = 2  # texture index of the smoke's density node in the volumetric scenes


def trilinear(grid: np.ndarray, p: np.ndarray) -> np.ndarray:
    """The device's grid read in float32: cell-centred samples over
    [-0.5, 0.5]^3, clamped edges, lerp a + w * (b - a) along x, y, z."""
    f = np.float32
    nz, ny, nx = grid.shape
    idx, wts = [], []
    for a, n in enumerate((nx, ny, nz)):
        g = (p[:, a].astype(f) + f(0.5)) * f(n) - f(0.5)
        lo = np.zeros(len(g), np.int64)
        hi = np.zeros(len(g), np.int64)
        w = np.zeros(len(g), f)
        inside = (g > 0) & (g < f(n - 1))
        fl = np.floor(g[inside])
        lo[inside] = fl.astype(np.int64)
        hi[inside] = lo[inside] + 1
        w[inside] = (g[inside] - fl).astype(f)
        top = ~(g > 0) & ~inside
        lo[top], hi[top] = 0, 0
        high = (g >= f(n - 1))
        lo[high], hi[high] = n - 1, n - 1
        idx.append((lo, hi))
        wts.append(w)
    (x0, x1), (y0, y1), (z0, z1) = idx
    wx, wy, wz = wts
    G = grid.astype(f)

    def lerp(a, b, w):
        return (a + w * (b - a)).astype(f)

    c00 = lerp(G[z0, y0, x0], G[z0, y0, x1], wx)
    c10 = lerp(G[z0, y1, x0], G[z0, y1, x1], wx)
    c01 = lerp(G[z1, y0, x0], G[z1, y0, x1], wx)
    c11 = lerp(G[z1, y1, x0], G[z1, y1, x1], wx)
    return lerp(lerp(c00, c10, wy), lerp(c01, c11, wy), wz)


@pytest.fixture(scope="module")
def vol_scene(ctx, scene_dir, halton_perm):
    from ymrt_b200 import scenes
    path = scenes.scene_path("volumetric", 0, scene_dir)
    s = Y.Scene(ctx, Y.HostScene(path, 128, 128), halton_perm)
    yield s
    s.close()


@pytest.mark.parametrize("half", [False, True])
def test_grid_read_matches_trilinear(vol_scene, half):
    rng = np.random.default_rng(5)
    grid = rng.uniform(0.0, 2.0, (9, 13, 17)).astype(np.float32)  # nz, ny, nx: not a cube
    vol_scene.set_density_grid(FBM, grid, half=half)
    want_grid = grid.astype(np.float16).astype(np.float32) if half else grid
    pts = rng.uniform(-0.7, 0.7, (20000, 3)).astype(np.float32)  # inside and outside the box
    pts[:16] = [[-0.5, -0.5, -0.5], [0.5, 0.5, 0.5], [0.0, 0.0, 0.0], [-0.5 + 0.5 / 17, 0.0, 0.0]] * 4
    got = vol_scene.density(FBM, pts)
    want = trilinear(want_grid, pts)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), np.abs(got - want).max()
    # cell centres read back the stored values (up to the float32 rounding of
    # the centre coordinates themselves)
    k = rng.integers(0, [17, 13, 9], (500, 3))
    centres = ((k + 0.5) / np.array([17, 13, 9]) - 0.5).astype(np.float32)
    assert np.allclose(vol_scene.density(FBM, centres), want_grid[k[:, 2], k[:, 1], k[:, 0]], rtol=0, atol=1e-5)


def test_grid_rejects_bad_input(vol_scene):
    with pytest.raises(Y.YmrtError):
        vol_scene.set_density_grid(99, np.ones((2, 2, 2), np.float32))
    bad = np.ones((2, 2, 2), np.float32)
    bad[1, 1, 1] = np.nan
    with pytest.raises(Y.YmrtError):
        vol_scene.set_density_grid(FBM, bad)


@pytest.mark.parametrize("half", [False, True])
@pytest.mark.parametrize("frame", [1, 2])
def test_constant_grid_renders_as_constant_density(ctx, scene_dir, halton_perm, oracle, half, frame):
    """A grid of 0.5s in place of the fBm node against the reference's scene
    whose node is the constant 0.5: same density at every point, same upper
    bound, so the same paths."""
    from ymrt_b200 import scenes
    path = scenes.scene_path("volumetric", 0, scene_dir)
    const_path = scenes.scene_path("volumetric_const", 0, scene_dir)
    ours = Y.Scene(ctx, Y.HostScene(path, 128, 128), halton_perm)
    ours.set_density_grid(FBM, np.full((8, 8, 8), 0.5, np.float32), half=half)
    ref = oracle.RefScene(const_path, halton_perm, 128, 128)
    s = Y.default_setting(spp=1, ray_depth=8, distant_light=True, volume=True)
    ref.set_settings(spp=1, ray_depth=8, distant_light=1, volume=1)
    a, st = ours.render(s, frame)
    b = ref.render_frame(frame)
    assert st.device_errors == 0
    assert np.array_equal(a[..., 3], b[..., 3])
    D.check_against_host(f"grid_const_h{int(half)}_f{frame}", ours, ref, s, frame, a, b)
    ours.close()
    ref.close()


def test_fbm_grid_converges_to_fbm_node(ctx, scene_dir, halton_perm):
    """A 128^3 float16 grid sampled from the smoke's fBm node renders close
    to the procedural node itself. The two media have different majorants
    (the grid's maximum against the fBm node's analytic bound), so the same
    samples take different tracking decisions: the images are independent
    64-spp estimates, compared as 8x8-pixel block means."""
    from ymrt_b200 import scenes
    path = scenes.scene_path("volumetric", 0, scene_dir)
    proc = Y.Scene(ctx, Y.HostScene(path, 128, 128), halton_perm)
    grid_scene = Y.Scene(ctx, Y.HostScene(path, 128, 128), halton_perm)
    lattice = (np.arange(128, dtype=np.float32) + 0.5) / 128 - 0.5
    z, y, x = np.meshgrid(lattice, lattice, lattice, indexing="ij")
    vals = proc.density(FBM, np.stack([x, y, z], -1).reshape(-1, 3)).reshape(128, 128, 128)
    grid_scene.set_density_grid(FBM, vals, half=True)
    s = Y.default_setting(spp=64, ray_depth=8, distant_light=True, volume=True)
    a, sa = proc.render(s, 1)
    b, sb = grid_scene.render(s, 1)
    proc.close()
    grid_scene.close()
    assert sa.device_errors == 0 and sb.device_errors == 0
    blocks_a = a[..., :3].reshape(16, 8, 16, 8, 3).mean(axis=(1, 3))
    blocks_b = b[..., :3].reshape(16, 8, 16, 8, 3).mean(axis=(1, 3))
    rmse = float(np.sqrt(np.mean((blocks_a - blocks_b) ** 2)))
    mean = float(np.mean(a[..., :3]))
    print(f"fBm node vs 128^3 fp16 grid of it, 64 spp, 8x8 block means: RMSE {rmse:.3e} "
          f"(mean radiance {mean:.3f}, means {mean:.4f} / {float(np.mean(b[..., :3])):.4f})")
    assert rmse <= 0.02 * mean, (rmse, mean)
    assert abs(float(np.mean(b[..., :3])) - mean) <= 0.01 * mean
