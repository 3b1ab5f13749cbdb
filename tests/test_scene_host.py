"""Host-side scene preparation against the reference's own scene module.

The instance order, per-mesh triangle order, transforms, shape-light table and
camera must equal the reference's bit for bit: they define every index and
light selection the renderer reports.
"""
import os

import numpy as np
import pytest

import ymrt_b200 as Y


def _meaningful(kind, rec):
    """Zeroes the words of a record that the reference leaves uninitialised:
    DefaultMtl's padding word, the tail of a light material's union and
    DistantLight's padding word."""
    rec = rec.copy()
    if kind == "materials":
        default = rec[:, 0] == 0
        rec[default, 36] = 0
        rec[~default, 5:] = 0
    elif kind == "distant_lights":
        rec[:, 7] = 0
    return rec


@pytest.mark.parametrize("name,size", [("cornell", (256, 256)), ("instanced", (1920, 1080)),
                                       ("volumetric", (256, 256)), ("spheres", (256, 256)), ("textured", (256, 256))])
def test_scene_preparation_matches_reference(name, size, scene_dir, halton_perm, oracle):
    from ymrt_b200 import scenes
    path = scenes.scene_path(name, 0, scene_dir)
    ours = Y.HostScene(path, *size)
    ref = oracle.RefScene(path, halton_perm, *size)
    assert np.array_equal(ours.instances(), ref.instances())
    fa, ia = ours.transforms()
    fb, ib = ref.transforms()
    assert np.array_equal(fa.view(np.uint32), fb.view(np.uint32))
    assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32))
    la, lb = ours.lights(), ref.lights()
    assert np.array_equal(la[0], lb[0])
    assert np.array_equal(la[1].view(np.uint32), lb[1].view(np.uint32))
    assert np.array_equal(la[2].view(np.uint32), lb[2].view(np.uint32))
    for kind in ("materials", "volumes", "distant_lights", "textures"):
        a, b = _meaningful(kind, ours.records(kind)), _meaningful(kind, ref.records(kind))
        assert np.array_equal(a, b), kind
    assert np.array_equal(ours.geometries().view(np.uint32), ref.geometries().view(np.uint32))
    for g in range(ref.counts()["geometries"]):
        assert np.array_equal(ours.triangles(g), ref.geometry_triangles(g)), f"mesh {g}"
        assert np.array_equal(ours.mesh_corners(g).view(np.uint32), ref.mesh_corners(g).view(np.uint32)), f"mesh {g}"
    # camera: position, u, v, w, aspect, tan(fov/2) against the reference Camera bytes
    cam = np.frombuffer(ref.camera_bytes(), dtype=np.float32)
    # Camera layout: m_width, m_height (ints), position, u, v, w, aspect, fov, lens, tan_half_fov
    pos_u_v_w = cam[2:14]
    assert np.array_equal(ours.camera()[:12].view(np.uint32), pos_u_v_w.view(np.uint32))
    assert ours.camera()[12] == cam[14] and ours.camera()[13] == cam[17]


def test_instanced_scene_size(instanced_path):
    c = Y.HostScene(instanced_path, 1920, 1080).counts()
    assert c["instances"] == 66
    assert 1_150_000 < c["instanced_triangles"] < 1_300_000
    assert c["lights"] == 4


def write(tmp_path, text, name="s.ymtmp"):
    p = os.path.join(tmp_path, name)
    with open(p, "w") as f:
        f.write(text)
    return p


def test_loader_rejects_bad_input(tmp_path):
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene(write(tmp_path, "Begin(Camera);\nEnd(Camera);\n", "x.txt"), 8, 8)
    assert e.value.code == -3
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene(os.path.join(tmp_path, "missing.ymtmp"), 8, 8)
    assert e.value.code == -2
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene(write(tmp_path, "Begin(Transform);\n\ttranslate = <0,0,0>;\n"), 8, 8)
    assert e.value.code == -3  # missing End
    with pytest.raises(Y.YmrtError) as e:  # an image texture needs a file name
        Y.HostScene(write(tmp_path, 'Begin(ImageTexture);\n\tname = "t";\nEnd(ImageTexture);\n'), 8, 8)
    assert e.value.code == -3
    with pytest.raises(Y.YmrtError) as e:  # a solid node needs both inputs (the reference's reader too)
        Y.HostScene(write(tmp_path, 'Begin(CheckerBoardTexture);\n\tname = "t";\nEnd(CheckerBoardTexture);\n'), 8, 8)
    assert e.value.code == -3
    with pytest.raises(Y.YmrtError) as e:  # instance referring to an undeclared name
        Y.HostScene(write(tmp_path, 'Begin(PrimitiveInstance);\n\tname = "i";\n\tgeometry_index = "g";\nEnd(PrimitiveInstance);\n'), 8, 8)
    assert e.value.code == -3
    with pytest.raises(Y.YmrtError) as e:  # scene without instances
        Y.HostScene(write(tmp_path, "Begin(Camera);\n\tfov = 30;\nEnd(Camera);\n"), 8, 8)
    assert e.value.code == -1


@pytest.mark.parametrize("name", ["cornell", "instanced", "volumetric", "spheres"])
def test_reference_bvh_depth_fits_its_stack(name, scene_dir, halton_perm, oracle):
    """The reference's traversals keep at most depth + 1 node indices on a
    32-entry stack with no bounds check in release builds
    (src/ShadingUtilities.cuh:147-212): its device kernels are only run on
    scenes whose binary BVHs are shallower than that."""
    from ymrt_b200 import scenes
    ref = oracle.RefScene(scenes.scene_path(name, 0, scene_dir), halton_perm, 64, 64)
    depths = ref.bvh_depths()
    assert depths.max() + 1 <= 32, depths


def test_loader_rejects_malformed_values(tmp_path):
    """Malformed values: a non-number in a vector, an unterminated block, a
    reference to an undeclared name; each is YMRT_ERR_FORMAT with a message
    naming the file, nothing thrown across the C ABI."""
    cases = [
        'Begin(Transform);\n\tname = "t";\n\ttranslate = <1,x,3>;\nEnd(Transform);\n',
        'Begin(Transform);\n\tname = "t";\n\ttranslate = <1,2,3>;\n',
        'Begin(PrimitiveInstance);\n\tname = "i";\n\tgeometry_index = "missing";\nEnd(PrimitiveInstance);\n',
    ]
    for k, text in enumerate(cases):
        with pytest.raises(Y.YmrtError) as e:
            Y.HostScene(write(tmp_path, text, f"bad{k}.ymtmp"), 8, 8)
        assert e.value.code == -3, (k, e.value)
