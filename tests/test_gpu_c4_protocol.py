"""C4's gradient checks as the differentiable-rendering workload states
them: central finite differences with eps = 1e-3 on seeded random
parameters drawn from material albedo, material roughness and single cells
of a 64^3 density grid, and a double-precision reference on a 64x64 image.

The loss is linear in the image, sum(w * image) with fixed random weights w
(so dLoss/dImage = w), computed in double.

* Albedo (the volumetric scene: Lambertian walls seen through a fog box and
  an fBm smoke box, media and sun on, 64x64, 16 spp): sampling does not
  depend on albedo, so each render is a polynomial in it. ymrt_render_backward
  is compared with central differences (eps 1e-3) of the reference's own
  renderer built in double (the FP64 oracle, same samples) on eight seeded
  (material, channel) pairs: each within 1%.
* Roughness (the glossy scene's conductor and plastic boxes): sampled
  directions move with roughness, so per sample set the adjoint (directions
  held fixed) and the finite difference (directions moved) are two
  different unbiased estimates of the derivative of the expectation: their
  means over 400 sample sets must agree within three standard errors plus
  1% (at eps 1e-3 the finite difference's visibility jumps leave it a
  standard error of a few percent).
* Single cells of a 64^3 grid in place of the smoke's density (values in
  [0.2, 0.6], maximum 1.0 in a corner cell so the majorant does not move):
  four seeded cells among the 200 with the largest gradient. Tracking
  decisions (real or null collision) flip with the density, so a finite
  difference with the same samples is a rare large jump: its variance per
  sample set grows as 1/eps, and at eps 1e-3 a few hundred sets see almost
  none of the jumps. The cells are therefore differenced with a step of
  0.05 (the expectation is smooth in a cell's value, and the central
  difference's bias is second order), and the means over sample sets are
  compared (three standard errors plus 1%). At this size one cell's
  derivative still carries a standard error of 30-50% of its value after a
  few hundred sets, so this bound checks unbiasedness, not 1%.
"""
import os

import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

EPS = 1e-3
SIZE = 64


def _weights(seed, size=SIZE):
    import torch
    rng = np.random.default_rng(seed)
    return torch.as_tensor(rng.uniform(0.0, 1.0, (size, size, 4)).astype(np.float32), device="cuda")


def _loss(img, w):
    import torch
    if isinstance(img, np.ndarray):
        img = torch.as_tensor(img)
    return float((img[..., :3].double().cpu() * w[..., :3].double().cpu()).sum().item())


class _Renderer:
    def __init__(self, ctx, scene, setting, n_grid=0, grid_tex=None):
        self.ctx, self.scene, self.setting = ctx, scene, setting
        self.n_grid, self.grid_tex = n_grid, grid_tex

    def forward(self, frame, record=False):
        import torch
        out = torch.zeros((self.scene.height, self.scene.width, 4), dtype=torch.float32, device="cuda")
        render = (self.scene, self.setting, frame, out, 0, 0)
        rec = torch.zeros((Y.path_count(render), 4), dtype=torch.float32, device="cuda") if record else None
        st = Y.render_batch(self.ctx, [render], [rec] if record else None)
        assert st.device_errors == 0
        return render, out, rec

    def adjoint(self, frame, w):
        import torch
        render, out, rec = self.forward(frame, True)
        n_mat = self.scene.material_params().shape[0]
        mg = torch.zeros((n_mat, 4), dtype=torch.float32, device="cuda")
        kw = dict(material_grads=mg)
        gg = None
        if self.n_grid:
            gg = torch.zeros(self.n_grid, dtype=torch.float32, device="cuda")
            kw.update(grid_texture=self.grid_tex, grid_grads=gg)
        st = Y.render_backward_ex(self.ctx, [render], [rec], [w], **kw)
        assert st.device_errors == 0
        return mg.cpu().numpy(), (gg.cpu().numpy() if gg is not None else None)


def test_albedo_gradients_match_the_fp64_reference(ctx, volumetric_path, halton_perm, oracle):
    if not oracle.available64():
        pytest.skip("FP64 oracle not built")
    setting_kw = dict(spp=16, ray_depth=8, distant_light=True, volume=True)
    scene = Y.Scene(ctx, Y.HostScene(volumetric_path, SIZE, SIZE), halton_perm)
    ref = oracle.RefScene(volumetric_path, halton_perm, SIZE, SIZE, fp64=True)
    ref.set_settings(spp=16, ray_depth=8, distant_light=1, volume=1)
    r = _Renderer(ctx, scene, Y.default_setting(**setting_kw))
    params = scene.material_params()
    w = _weights(21)
    g, _ = r.adjoint(1, w)
    lambertian = [m for m in range(params.shape[0]) if params[m, :3].sum() > 0 and m < 5]
    rng = np.random.default_rng(8)
    picks = [(int(rng.choice(lambertian)), int(rng.integers(0, 3))) for _ in range(8)]
    wn = w.cpu().numpy().astype(np.float64)
    base = params.astype(np.float64)
    for m, k in picks:
        ls = []
        for sgn in (+1, -1):
            p = base.copy()
            p[m, k] += sgn * EPS
            ref.set_material_params(p)
            img = ref.render_frame(1)
            ls.append(float((img[..., :3] * wn[..., :3]).sum()))
        ref.set_material_params(base)
        fd = (ls[0] - ls[1]) / (2 * EPS)
        print(f"albedo m{m} c{k}: adjoint {g[m, k]:.6g}, FP64 reference central difference {fd:.6g}")
        assert abs(g[m, k] - fd) <= 0.01 * abs(fd), (m, k, g[m, k], fd)
    scene.close()
    ref.close()


def test_albedo_gradients_match_the_fp64_host_adjoint_on_a_crop(ctx, volumetric_path, halton_perm, oracle):
    """ymrt_render_backward on a 512x512 view (16 spp, media and sun on)
    with dLoss/dImage nonzero only on a 64x64 crop, against the host adjoint
    in double precision (oracle/adjoint64.py) over the FP64 oracle's
    radiance terms of the same samples, for every Lambertian (material,
    channel) pair: each within 1%."""
    import torch
    from oracle import adjoint64
    if not oracle.available64():
        pytest.skip("FP64 oracle not built")
    view, crop, x0, y0, spp = 512, 64, 224, 192, 16
    scene = Y.Scene(ctx, Y.HostScene(volumetric_path, view, view), halton_perm)
    r = _Renderer(ctx, scene, Y.default_setting(spp=spp, ray_depth=8, distant_light=True, volume=True))
    rng = np.random.default_rng(33)
    w = np.zeros((view, view, 4), np.float32)
    w[y0:y0 + crop, x0:x0 + crop] = rng.uniform(0.0, 1.0, (crop, crop, 4))
    g, _ = r.adjoint(1, torch.as_tensor(w, device="cuda"))
    ref = oracle.RefScene(volumetric_path, halton_perm, view, view, fp64=True)
    ref.set_settings(spp=spp, ray_depth=8, distant_light=1, volume=1)
    params, lam = ref.material_params()
    tiles_x = view // 16
    ys, xs = np.mgrid[y0:y0 + crop, x0:x0 + crop]
    ev, _ = ref.record_events(1, tile_begin=(y0 // 16) * tiles_x, tile_end=((y0 + crop) // 16) * tiles_x,
                              pixels=(ys * view + xs).ravel())
    h = adjoint64.albedo_adjoint(ev, w.astype(np.float64), params, np.flatnonzero(lam), spp)
    worst = 0.0
    for m in np.flatnonzero(lam):
        for k in range(3):
            rel = abs(g[m, k] - h[m, k]) / abs(h[m, k])
            worst = max(worst, rel)
            assert rel <= 0.01, (m, k, g[m, k], h[m, k])
    print(f"{len(np.flatnonzero(lam)) * 3} albedo gradients against the FP64 host adjoint: worst relative "
          f"difference {worst:.2e}")
    ref.close()
    scene.close()


def test_albedo_gradients_match_float_finite_differences_at_1e3(ctx, volumetric_path, halton_perm):
    """The same eight pairs against central differences (eps 1e-3) of
    ymrt_b200's own forward render with the same samples."""
    scene = Y.Scene(ctx, Y.HostScene(volumetric_path, SIZE, SIZE), halton_perm)
    r = _Renderer(ctx, scene, Y.default_setting(spp=16, ray_depth=8, distant_light=True, volume=True))
    params = scene.material_params()
    w = _weights(21)
    g, _ = r.adjoint(1, w)
    lambertian = [m for m in range(params.shape[0]) if params[m, :3].sum() > 0 and m < 5]
    rng = np.random.default_rng(8)
    for _ in range(8):
        m, k = int(rng.choice(lambertian)), int(rng.integers(0, 3))
        ls = []
        for sgn in (+1, -1):
            p = params.copy()
            p[m, k] += sgn * EPS
            scene.set_material_params(p)
            ls.append(_loss(r.forward(1)[1], w))
        scene.set_material_params(params)
        fd = (ls[0] - ls[1]) / (2 * EPS)
        assert abs(g[m, k] - fd) <= 0.01 * abs(fd), (m, k, g[m, k], fd)
    scene.close()


def _mean_test(a, d, name):
    a, d = np.asarray(a, np.float64), np.asarray(d, np.float64)
    se = np.sqrt(a.var(ddof=1) / len(a) + d.var(ddof=1) / len(d))
    print(f"{name}: adjoint {a.mean():.5g} (SE {a.std(ddof=1) / np.sqrt(len(a)):.3g}), finite differences "
          f"{d.mean():.5g} (SE {d.std(ddof=1) / np.sqrt(len(d)):.3g}) over {len(a)} sample sets")
    assert abs(a.mean() - d.mean()) <= 3.0 * se + 0.01 * abs(d.mean()), (name, a.mean(), d.mean(), se)


def test_roughness_gradients_fd_of_expectation(ctx, scene_dir, halton_perm):
    from ymrt_b200 import scenes
    path = scenes.scene_path("glossy", 0, scene_dir)
    scene = Y.Scene(ctx, Y.HostScene(path, SIZE, SIZE), halton_perm)
    r = _Renderer(ctx, scene, Y.default_setting(spp=32, ray_depth=8))
    params = scene.material_params()
    rough = [m for m in range(params.shape[0]) if params[m, 3] > 0.2]
    assert len(rough) == 2
    w = _weights(11)
    for m in rough:
        a, d = [], []
        for frame in range(1, 401):
            g, _ = r.adjoint(frame, w)
            a.append(g[m, 3])
            ls = []
            for sgn in (+1, -1):
                p = params.copy()
                p[m, 3] += sgn * EPS
                scene.set_material_params(p)
                ls.append(_loss(r.forward(frame)[1], w))
            scene.set_material_params(params)
            d.append((ls[0] - ls[1]) / (2 * EPS))
        _mean_test(a, d, f"roughness of material {m}")
    scene.close()


def test_single_grid_cells_fd_of_expectation(ctx, volumetric_path, halton_perm):
    N, FBM = 64, 2
    sets = int(os.environ.get("YMRT_C4_CELL_SETS", "160"))
    scene = Y.Scene(ctx, Y.HostScene(volumetric_path, SIZE, SIZE), halton_perm)
    rng = np.random.default_rng(3)
    grid = rng.uniform(0.2, 0.6, (N, N, N)).astype(np.float32)
    grid[0, 0, 0] = 1.0
    scene.set_density_grid(FBM, grid)
    r = _Renderer(ctx, scene, Y.default_setting(spp=64, ray_depth=8, distant_light=True, volume=True), N ** 3, FBM)
    w = _weights(11)
    acc = np.zeros(N ** 3)
    for frame in range(1, 17):
        acc += r.adjoint(frame, w)[1]
    top = np.argsort(-np.abs(acc))[:200]
    cells = np.random.default_rng(5).choice(top, 4, replace=False)
    for c in cells:
        a, d = [], []
        for frame in range(1, sets + 1):
            a.append(r.adjoint(frame, w)[1][c])
            ls = []
            for sgn in (+1, -1):
                pert = grid.copy()
                pert.ravel()[c] += sgn * 0.05
                scene.set_density_grid(FBM, pert)
                ls.append(_loss(r.forward(frame)[1], w))
            scene.set_density_grid(FBM, grid)
            d.append((ls[0] - ls[1]) / (2 * 0.05))
        _mean_test(a, d, f"grid cell {np.unravel_index(c, (N, N, N))}")
    scene.close()
