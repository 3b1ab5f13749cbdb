"""The oracle's density-grid node (this project's addition to the reference,
oracle/build_ref.py _MEDIA_HOOKS) against a numpy float32 restatement of the
grid read: trilinear over cell centres of the object-space box
[-0.5, 0.5]^3 with clamped edges, in the operand order of ymrt_b200's
grid_eval; and the node's majorant and the tracking-bound counter."""
import numpy as np
import pytest


def grid_read(g, pts):
    """numpy float32 restatement of the grid read (g: (nz, ny, nx))."""
    n = g.shape[::-1]
    half = np.float32(0.5)
    lo, hi, w = [], [], []
    for a in range(3):
        gg = ((pts[:, a] + half) * np.float32(n[a]) - half).astype(np.float32)
        inside = (gg > 0) & (gg < np.float32(n[a] - 1))
        fl = np.floor(gg)
        l = np.where(inside, fl, np.where(~(gg > 0), 0, n[a] - 1)).astype(np.int64)
        lo.append(l)
        hi.append(np.where(inside, l + 1, l))
        w.append(np.where(inside, (gg - fl).astype(np.float32), np.float32(0)))

    def lerp(a, b, t):
        return (a + t * (b - a)).astype(np.float32)

    (x0, y0, z0), (x1, y1, z1) = lo, hi
    c00 = lerp(g[z0, y0, x0], g[z0, y0, x1], w[0])
    c10 = lerp(g[z0, y1, x0], g[z0, y1, x1], w[0])
    c01 = lerp(g[z1, y0, x0], g[z1, y0, x1], w[0])
    c11 = lerp(g[z1, y1, x0], g[z1, y1, x1], w[0])
    return lerp(lerp(c00, c10, w[1]), lerp(c01, c11, w[1]), w[2])


def test_oracle_grid_node(volumetric_path, halton_perm, oracle):
    rng = np.random.default_rng(3)
    g = rng.uniform(0.0, 2.0, (5, 6, 8)).astype(np.float32)
    pts = rng.uniform(-0.8, 0.8, (5000, 3)).astype(np.float32)
    ref = oracle.RefScene(volumetric_path, halton_perm, 64, 64)
    fbm = ref.density(2, pts)
    ref.set_density_grid(2, g)
    got = ref.density(2, pts)
    ref.close()
    assert np.array_equal(got, grid_read(g, pts))
    assert not np.array_equal(fbm, got)  # the node was replaced
    # scene freed: a new scene of the same file reads the fBm node again
    ref2 = oracle.RefScene(volumetric_path, halton_perm, 64, 64)
    assert np.array_equal(ref2.density(2, pts), fbm)
    ref2.close()


def test_oracle_tracking_bound_counter(volumetric_path, halton_perm, oracle):
    """The counter of tracking loops stopped at MAX_FREE_PATH_LENGTH reads
    and resets (its counts on the C2 frame are checked against the device's
    in tests/test_gpu_c2_grid.py)."""
    ref = oracle.RefScene(volumetric_path, halton_perm, 32, 32)
    ref.set_density_grid(2, np.full((4, 4, 4), 1.0, np.float32))
    ref.set_settings(spp=1, ray_depth=8, volume=1)
    ref.tracking_caps(reset=True)
    ref.render_frame(1)
    assert ref.tracking_caps(reset=True) >= 0
    assert ref.tracking_caps(reset=False) == 0
    ref.close()
