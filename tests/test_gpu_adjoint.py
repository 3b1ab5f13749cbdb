"""Path-replay adjoint (ymrt_render_backward) against central finite
differences of the forward render with the same samples.

The loss is linear in the image, sum(w * image) with fixed random weights w,
so dLoss/dImage = w and the finite difference is of the rendered estimator
itself. Lambertian albedos (the Cornell-like scene): sampling does not depend
on albedo, so the estimator is a polynomial in it and the two must agree to
1%. Roughness (the glossy scene's conductor and plastic boxes): sampled
directions move with roughness, so agreement is to 5%.
"""
import numpy as np
import pytest

import ymrt_b200 as Y
from diff_harness import MultiViewRenderer, RenderFunction

pytestmark = pytest.mark.gpu


def _setup(ctx, path, halton_perm, size, spp, views=1):
    scenes = [Y.Scene(ctx, Y.HostScene(path, size, size), halton_perm) for _ in range(views)]
    return MultiViewRenderer(ctx, scenes, Y.default_setting(spp=spp, ray_depth=8), frame_index=1)


def _loss(images, w):
    return float(sum((img[..., :3].double() * wk[..., :3].double()).sum().item() for img, wk in zip(images, w)))


def _fd(renderer, params, m, k, eps, w):
    lo, hi = params.copy(), params.copy()
    lo[m, k] -= eps
    hi[m, k] += eps
    renderer.set_params(hi)
    l_hi = _loss(renderer.forward(), w)
    renderer.set_params(lo)
    l_lo = _loss(renderer.forward(), w)
    renderer.set_params(params)
    return (l_hi - l_lo) / (2 * eps)


def _adjoint(renderer, params, w):
    import torch
    renderer.set_params(params)
    renderer.forward()
    return renderer.backward([torch.as_tensor(wk, device="cuda") for wk in w]).cpu().numpy()


def _weights(renderer, seed):
    import torch
    rng = np.random.default_rng(seed)
    return [torch.as_tensor(rng.uniform(0.0, 1.0, tuple(img.shape)).astype(np.float32), device="cuda")
            for img in renderer.images]


def test_record_holds_each_paths_radiance(ctx, cornell_path, halton_perm):
    import torch
    r = _setup(ctx, cornell_path, halton_perm, 64, 4)
    img = r.forward()[0].cpu().numpy()
    rec = r.records[0].cpu().numpy()[:, :3]
    # path index -> pixel: 16x16 tiles in order, 256 * spp paths per tile, spp per pixel
    spp, W = 4, 64
    idx = np.arange(rec.shape[0])
    tile, local = idx // (256 * spp), idx % (256 * spp)
    tp = local // spp
    px = (tile % (W // 16)) * 16 + tp % 16
    py = (tile // (W // 16)) * 16 + tp // 16
    acc = np.zeros((64, 64, 3), np.float64)
    np.add.at(acc, (py, px), rec / spp)
    assert np.allclose(acc, img[..., :3], rtol=1e-5, atol=1e-6)
    for s in r.scenes:
        s.close()


def test_albedo_gradients_match_finite_differences(ctx, cornell_path, halton_perm):
    r = _setup(ctx, cornell_path, halton_perm, 96, 16)
    params = r.scenes[0].material_params()
    w = _weights(r, 7)
    g = _adjoint(r, params, w)
    checked = 0
    for m in range(params.shape[0]):
        if params[m].sum() == 0.0:
            continue  # the light material
        for k in range(3):
            fd = _fd(r, params, m, k, 1e-2, w)
            if abs(fd) < 1e-3 * np.abs(g[:, :3]).max():
                continue
            assert abs(g[m, k] - fd) <= 0.01 * abs(fd), (m, k, g[m, k], fd)
            checked += 1
    assert checked >= 6
    for s in r.scenes:
        s.close()


def test_roughness_gradients_match_finite_differences(ctx, scene_dir, halton_perm):
    """Roughness moves the sampled directions, so a finite difference with
    the same random numbers and the adjoint (which holds directions fixed)
    are two different unbiased estimates of the same derivative: compare
    their means over independent sample sets (frames) within three standard
    errors plus 2%."""
    from ymrt_b200 import scenes
    path = scenes.scene_path("glossy", 0, scene_dir)
    r = _setup(ctx, path, halton_perm, 96, 32)
    params = r.scenes[0].material_params()
    w = _weights(r, 11)
    rough = [m for m in range(params.shape[0]) if params[m, 3] > 0.2]  # the two boxes
    assert len(rough) == 2
    frames = [1, 2, 3, 4]
    g = {m: [] for m in rough}
    fd = {m: [] for m in rough}
    for f in frames:
        for rr in r.renders:
            rr[2] = f
        ga = _adjoint(r, params, w)
        for m in rough:
            g[m].append(ga[m, 3])
            fd[m].append(_fd(r, params, m, 3, 1e-2, w))
    for m in rough:
        a, b = np.array(g[m], np.float64), np.array(fd[m], np.float64)
        se = np.sqrt(a.var(ddof=1) / len(a) + b.var(ddof=1) / len(b))
        assert abs(a.mean() - b.mean()) <= 3.0 * se + 0.02 * abs(b.mean()), (m, a, b)
    for s in r.scenes:
        s.close()


def test_autograd_function_two_views(ctx, cornell_path, halton_perm):
    import torch
    from ymrt_b200 import scenes
    views = [Y.Scene(ctx, Y.HostScene(cornell_path, 64, 64, camera=scenes.orbit_view("cornell", 0, v, 4)), halton_perm)
             for v in (0, 3)]
    r = MultiViewRenderer(ctx, views, Y.default_setting(spp=8, ray_depth=8))
    base = views[0].material_params()
    target_params = base.copy()
    target_params[:, :3] = np.clip(target_params[:, :3] + 0.1, 0, 1)
    target_params[base.sum(1) == 0] = 0
    r.set_params(target_params)
    target = torch.stack(r.forward()).detach()
    params = torch.tensor(base, requires_grad=True)
    images = RenderFunction.apply(params, r)
    loss = ((images[..., :3] - target[..., :3]) ** 2).sum()
    loss.backward()
    g = params.grad.numpy()
    # brightening the albedos lowers the loss: the gradient points down on the walls
    walls = [m for m in range(base.shape[0]) if base[m].sum() > 0]
    assert np.all(g[walls, :3].sum(1) < 0)
    for s in views:
        s.close()
