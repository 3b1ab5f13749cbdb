"""Transform edits on the host against the reference editor's rebuild.

The reference's editor, after a transform edit, rebuilds its top-level BVH
from the current instance order (which reorders the instances again),
rebuilds the shape-light list and re-derives the camera's media
(GuiModule::UpdateScene, src/core/GuiModule.cpp:123-170). The oracle runs
exactly that on the reference's scene module (oracle/ref_prepare.h
RebuildAfterTransformEdit); ymrt_host_scene_set_transforms must give the
same instance order, transforms and light table bit for bit, edit after
edit. (tests/test_gpu_transform_edit.py checks the device rebuild against
this host rebuild.)
"""
import numpy as np
import pytest

import ymrt_b200 as Y


def edit_matrices(seed, n, host: Y.HostScene, first):
    """n object-to-world matrices near the current ones: each moved, turned
    about y and rescaled a little (column-major 4x4, [column][row])."""
    rng = np.random.default_rng(seed)
    fwd, _ = host.transforms()
    out, scales = [], []
    for k in range(n):
        m = fwd[first + k].reshape(4, 4).astype(np.float64)
        a = rng.uniform(-0.6, 0.6)
        s = rng.uniform(0.8, 1.25, 3)
        rot = np.array([[np.cos(a), 0, -np.sin(a), 0], [0, 1, 0, 0], [np.sin(a), 0, np.cos(a), 0], [0, 0, 0, 1]])
        scale = np.diag([s[0], s[1], s[2], 1.0])
        e = rot @ scale  # applied in object space: m' = m * e (column-major: columns are basis vectors)
        mm = (e.T @ m)   # [col][row] layout: (M E)^T = E^T M^T
        mm[3, :3] += rng.uniform(-0.3, 0.3, 3)
        out.append(mm.astype(np.float32))
        scales.append(s.astype(np.float32))
    return np.stack(out), np.stack(scales)


@pytest.mark.parametrize("name,size", [("cornell", (128, 128)), ("volumetric", (128, 128)),
                                       ("spheres", (128, 128)), ("instanced", (320, 180))])
def test_host_edit_matches_reference_editor(name, size, scene_dir, halton_perm, oracle):
    from ymrt_b200 import scenes
    path = scenes.scene_path(name, 0, scene_dir)
    ours = Y.HostScene(path, *size)
    ref = oracle.RefScene(path, halton_perm, *size)
    n_t = ours.transforms()[0].shape[0]
    for step, first in enumerate([0, n_t // 2, max(0, n_t - 3)]):
        count = min(3, n_t - first)
        m, s = edit_matrices(100 + step, count, ours, first)
        ours.set_transforms(first, m, s)
        ref.set_transforms(first, m, s)
        assert np.array_equal(ours.instances(), ref.instances()), f"edit {step}: instance order"
        fa, ia = ours.transforms()
        fb, ib = ref.transforms()
        assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32))
        assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32))
        la, lb = ours.lights(), ref.lights()
        assert np.array_equal(la[0], lb[0]), f"edit {step}: light list"
        assert np.array_equal(la[1].view(np.uint32), lb[1].view(np.uint32)), f"edit {step}: light power / area"
        assert np.array_equal(la[2].view(np.uint32), lb[2].view(np.uint32)), f"edit {step}: light table"
    ref.close()


def test_edit_rejects_out_of_range(cornell_path):
    h = Y.HostScene(cornell_path, 64, 64)
    n_t = h.transforms()[0].shape[0]
    with pytest.raises(Y.YmrtError):
        h.set_transforms(n_t, np.eye(4, dtype=np.float32)[None])
