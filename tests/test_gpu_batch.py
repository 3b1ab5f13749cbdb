"""Batched rendering (ymrt_render_batch): several renders -- different
scenes, resolutions, sample counts, samplers and settings -- share the wave
queues of one batch. Each render must equal the same render made alone,
up to the order of per-pixel float additions."""
import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu

REL_TOL = 1e-5
ABS_TOL = 1e-7


def _close(a, b):
    diff = np.abs(a - b)
    return np.all(diff <= REL_TOL * np.maximum(np.abs(a), np.abs(b)) + ABS_TOL)


def test_batch_equals_single_renders(ctx, cornell_path, volumetric_path, instanced_path, halton_perm, oracle):
    import torch
    cases = [
        (Y.Scene(ctx, Y.HostScene(cornell_path, 256, 256), halton_perm), Y.default_setting(spp=4, ray_depth=8), 1, 0, 0),
        (Y.Scene(ctx, Y.HostScene(cornell_path, 96, 64), halton_perm), Y.default_setting(spp=2, ray_depth=8), 3, 0, 0),
        (Y.Scene(ctx, Y.HostScene(volumetric_path, 128, 128), halton_perm),
         Y.default_setting(spp=2, ray_depth=8, volume=True, distant_light=True), 2, 0, 0),
        (Y.Scene(ctx, Y.HostScene(instanced_path, 640, 480), halton_perm), Y.default_setting(spp=3, ray_depth=12),
         1, 400, 700),
        (Y.Scene(ctx, Y.HostScene(cornell_path, 128, 128), halton_perm),
         Y.default_setting(spp=2, ray_depth=8, sampler_type=0), 5, 0, 0),
    ]
    singles, outs = [], []
    for scene, setting, frame, tb, te in cases:
        single = torch.zeros((scene.height, scene.width, 4), dtype=torch.float32, device="cuda")
        scene.render(setting, frame, out=single, tile_begin=tb, tile_end=te)
        singles.append(single.cpu().numpy())
        outs.append(torch.full((scene.height, scene.width, 4), float("nan"), dtype=torch.float32, device="cuda"))
    stats = Y.render_batch(ctx, [(c[0], c[1], c[2], o, c[3], c[4]) for c, o in zip(cases, outs)])
    assert stats.device_errors == 0
    for k, (o, want) in enumerate(zip(outs, singles)):
        got = o.cpu().numpy()
        assert np.array_equal(got[..., 3], want[..., 3]), f"render {k}: sample counts differ"
        assert _close(got[..., :3], want[..., :3]), f"render {k}: radiance differs"
    for c in cases:
        c[0].close()


def test_batch_beyond_scene_slots(ctx, cornell_path, halton_perm):
    """70 small renders of 68 distinct scenes: more (scene, sampler) pairs
    than the 64 constant-memory scene slots, so the batch runs as two groups
    of jobs; every render must still equal the same render made alone."""
    import torch
    sizes = [(32 + 16 * (k % 6), 32 + 16 * (k // 6 % 4)) for k in range(68)]
    scenes = [Y.Scene(ctx, Y.HostScene(cornell_path, w, h), halton_perm) for w, h in sizes]
    cases = [(scenes[k % 68], Y.default_setting(spp=1 + k % 3, ray_depth=6), 1 + k % 2) for k in range(70)]
    singles, outs = [], []
    for scene, setting, frame in cases:
        single = torch.zeros((scene.height, scene.width, 4), dtype=torch.float32, device="cuda")
        scene.render(setting, frame, out=single)
        singles.append(single.cpu().numpy())
        outs.append(torch.full((scene.height, scene.width, 4), float("nan"), dtype=torch.float32, device="cuda"))
    stats = Y.render_batch(ctx, [(c[0], c[1], c[2], o) for c, o in zip(cases, outs)])
    assert stats.device_errors == 0
    for k, (o, want) in enumerate(zip(outs, singles)):
        got = o.cpu().numpy()
        assert np.array_equal(got[..., 3], want[..., 3]), f"render {k}: sample counts differ"
        assert _close(got[..., :3], want[..., :3]), f"render {k}: radiance differs"
    for s in scenes:
        s.close()
