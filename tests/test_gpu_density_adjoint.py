"""The path-replay adjoint through participating media (ymrt_render_backward_ex).

The volumetric scene's smoke density is a seeded float32 16^3 grid of values
in [0.2, 0.6] with one cell at 1.0; the loss is linear in the image,
sum(w * image) with fixed random weights w, so dLoss/dImage = w.

* Density grid: the adjoint's dLoss/d(grid value), summed over the cells
  weighted by their values, is the derivative of the loss with respect to
  scaling them all (but the maximum); it is compared with central finite
  differences of
  the forward render with the same samples. Tracking decisions (real or null
  collision) move with the density, so per sample set the two are different
  unbiased estimates: they must agree within three standard errors (over
  eight sample sets) plus 3%.
* Material albedo with media on: the walls are Lambertian, sampling does not
  depend on albedo, so the adjoint equals the finite difference to 1%.
"""
import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

FBM = 2      # texture index of the smoke's density node
N = 16       # grid cells per axis
SIZE = 128   # image width and height
SPP = 64


@pytest.fixture(scope="module")
def media(ctx, scene_dir, halton_perm):
    from ymrt_b200 import scenes
    path = scenes.scene_path("volumetric", 0, scene_dir)
    scene = Y.Scene(ctx, Y.HostScene(path, SIZE, SIZE), halton_perm)
    rng = np.random.default_rng(3)
    grid = rng.uniform(0.2, 0.6, (N, N, N)).astype(np.float32)
    grid[0, 0, 0] = 1.0  # the maximum (the majorant's factor), away from the differentiated cells
    scene.set_density_grid(FBM, grid)
    yield scene, grid
    scene.close()


def _setting():
    return Y.default_setting(spp=SPP, ray_depth=8, distant_light=True, volume=True)


def _forward(ctx, scene, frame, record=False):
    import torch
    out = torch.zeros((SIZE, SIZE, 4), dtype=torch.float32, device="cuda")
    render = (scene, _setting(), frame, out, 0, 0)
    rec = None
    if record:
        rec = torch.zeros((Y.path_count(render), 4), dtype=torch.float32, device="cuda")
    st = Y.render_batch(ctx, [render], [rec] if record else None)
    assert st.device_errors == 0
    return render, out, rec


def _loss(img, w):
    return float((img[..., :3].double() * w[..., :3].double()).sum().item())


def _weights(seed):
    import torch
    rng = np.random.default_rng(seed)
    return torch.as_tensor(rng.uniform(0.0, 1.0, (SIZE, SIZE, 4)).astype(np.float32), device="cuda")


REGIONS = {
    "all": (slice(None), slice(None), slice(None)),
    "front_half": (slice(N // 2, None), slice(None), slice(None)),   # z >= 0 in the smoke's frame
    "left_half": (slice(None), slice(None), slice(0, N // 2)),       # x < 0
}


@pytest.mark.parametrize("region", sorted(REGIONS))
def test_density_grid_gradient_matches_finite_differences(ctx, media, region):
    import torch
    scene, grid = media
    # the region's cells but the maximum: scaled by 1 +- eps they stay below
    # it, so the majorant does not move
    blk = np.zeros(grid.shape, bool)
    blk[REGIONS[region]] = True
    blk[0, 0, 0] = False
    assert grid[blk].max() * 1.1 < grid.max()
    eps = 0.05
    adj, fd = [], []
    for frame in range(1, 9):
        w = _weights(100 + frame)
        scene.set_density_grid(FBM, grid)
        render, out, rec = _forward(ctx, scene, frame, record=True)
        gg = torch.zeros(N * N * N, dtype=torch.float32, device="cuda")
        st = Y.render_backward_ex(ctx, [render], [rec], [w], grid_texture=FBM, grid_grads=gg)
        assert st.device_errors == 0
        g = gg.cpu().numpy().reshape(N, N, N)
        adj.append(float((g[blk].astype(np.float64) * grid[blk]).sum()))
        ls = []
        for sgn in (+1, -1):
            pert = grid.copy()
            pert[blk] *= np.float32(1 + sgn * eps)
            scene.set_density_grid(FBM, pert)
            _, img, _ = _forward(ctx, scene, frame)
            ls.append(_loss(img, w))
        fd.append((ls[0] - ls[1]) / (2 * eps))
    scene.set_density_grid(FBM, grid)
    adj, fd = np.array(adj), np.array(fd)
    d = adj - fd
    se = d.std(ddof=1) / np.sqrt(len(d))
    print(f"{region}: grid-scale derivative over {len(d)} sample sets: adjoint {adj.mean():.5g} +- {adj.std(ddof=1):.3g}, "
          f"finite differences {fd.mean():.5g} +- {fd.std(ddof=1):.3g}, difference {d.mean():.4g} (SE {se:.3g})")
    assert abs(adj.mean()) > 0
    assert abs(d.mean()) <= 3 * se + 0.03 * abs(fd.mean()), (adj, fd)


def test_albedo_gradient_with_media_matches_finite_differences(ctx, media):
    import torch
    scene, grid = media
    n_mat = scene.material_params().shape[0]
    params = scene.material_params()
    w = _weights(7)
    render, out, rec = _forward(ctx, scene, 1, record=True)
    grads = torch.zeros((n_mat, 4), dtype=torch.float32, device="cuda")
    st = Y.render_backward_ex(ctx, [render], [rec], [w], material_grads=grads)
    assert st.device_errors == 0
    g = grads.cpu().numpy()
    eps = 0.05
    checked = 0
    for m in range(5):  # the five Lambertian walls
        for k in range(3):
            lo, hi = params.copy(), params.copy()
            lo[m, k] -= eps
            hi[m, k] += eps
            scene.set_material_params(hi)
            _, a, _ = _forward(ctx, scene, 1)
            scene.set_material_params(lo)
            _, b, _ = _forward(ctx, scene, 1)
            scene.set_material_params(params)
            fd = (_loss(a, w) - _loss(b, w)) / (2 * eps)
            assert abs(g[m, k] - fd) <= 0.01 * abs(fd) + 1e-3, (m, k, g[m, k], fd)
            checked += 1
    assert checked == 15
