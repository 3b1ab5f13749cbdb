"""Scenes from in-memory arrays (ymrt_scene_from_arrays) against the same
scenes loaded from .ymtmp files.

A host that keeps its scene in memory hands over transforms, meshes,
instances, materials, media, distant lights and texture nodes already
resolved to indices. Given the same assets, the prepared scene must equal
the file's bit for bit (instance and triangle order, lights, transforms,
camera), and so must its renders.
"""
import numpy as np
import pytest

import ymrt_b200 as Y
from ymrt_b200 import scenes


def arrays_of(name, scene_dir, width, height):
    """The arrays a host holding the generated scene would pass: meshes in
    creation order, instances in creation order, and the assets the file
    load produced (materials, media, lights and texture nodes as the
    reference's structs; transform matrices as composed)."""
    model = scenes.SCENES[name](0)
    path = scenes.scene_path(name, 0, scene_dir)
    hs = Y.HostScene(path, width, height)
    fwd, inv = hs.transforms()
    scales = np.array([np.maximum(np.asarray(s, np.float32), np.float32(0.0001)) for _, _, s, _ in model.transforms],
                      np.float32)
    geometries = []
    kinds = hs.geometries()
    for g in range(kinds.shape[0]):
        if kinds[g, 0] == 1:
            geometries.append({"sphere_radius": float(kinds[g, 1])})
            continue
        corners = hs.mesh_corners(g)  # per corner: position, normal, uv (creation order)
        n = corners.shape[0]
        ident = np.arange(n, dtype=np.uint32)
        mesh = {"triangles": ident.reshape(-1, 3), "position_indices": ident, "positions": corners[:, 0:3],
                "normal_indices": ident, "normals": corners[:, 3:6]}
        if g >= len(model.meshes) or model.meshes[g].uv_idx is not None:  # meshes with texture coordinates
            mesh.update(texcoord_indices=ident, texcoords=corners[:, 6:8])
        geometries.append(mesh)
    inst = hs.instances()  # prepared order: geometry, transform, material, volume, boundary, file index
    order = np.argsort(inst[:, 5])
    created = np.zeros((inst.shape[0], 8), np.uint32)
    created[:, 0] = inst[order, 0]
    created[:, 1] = inst[order, 1]
    created[:, 2] = 1
    created[:, 3] = inst[order, 2]
    created[:, 4] = inst[order, 3]
    created[:, 5] = inst[order, 4]
    created[:, 6] = inst[order, 5]
    kw = dict(transforms=fwd, inverse_transforms=inv, transform_scales=scales, geometries=geometries,
              instances=created, materials=hs.records("materials"), volumes=hs.records("volumes"),
              distant_lights=hs.records("distant_lights"), textures=hs.records("textures"), camera=model.camera)
    return hs, kw


@pytest.mark.parametrize("name,size", [("cornell", (256, 256)), ("spheres", (256, 256)),
                                       ("volumetric", (128, 128)), ("textured", (128, 128))])
def test_arrays_prepare_like_the_file(name, size, scene_dir):
    hs, kw = arrays_of(name, scene_dir, *size)
    ha = Y.HostScene.from_arrays(size[0], size[1], **kw)
    assert np.array_equal(ha.instances(), hs.instances())
    for x, y in zip(ha.transforms(), hs.transforms()):
        assert np.array_equal(x.view(np.uint32), y.view(np.uint32))
    for x, y in zip(ha.lights(), hs.lights()):
        assert np.array_equal(np.asarray(x).view(np.uint32), np.asarray(y).view(np.uint32))
    for kind in ("materials", "volumes", "distant_lights", "textures"):
        assert np.array_equal(ha.records(kind), hs.records(kind)), kind
    assert np.array_equal(ha.geometries().view(np.uint32), hs.geometries().view(np.uint32))
    for g in range(hs.geometries().shape[0]):
        assert np.array_equal(ha.triangles(g), hs.triangles(g)), g
        assert np.array_equal(ha.mesh_corners(g).view(np.uint32), hs.mesh_corners(g).view(np.uint32))
    assert np.array_equal(ha.camera().view(np.uint32), hs.camera().view(np.uint32))
    assert ha.counts() == hs.counts()


def test_arrays_reject_bad_input(scene_dir):
    hs, kw = arrays_of("cornell", scene_dir, 64, 64)
    bad = dict(kw)
    inst = kw["instances"].copy()
    inst[0, 0] = 99  # unknown geometry
    bad["instances"] = inst
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene.from_arrays(64, 64, **bad)
    assert e.value.code == -1
    bad = dict(kw)
    tex = np.zeros((1, Y.TEXTURE_WORDS), np.uint32)
    tex[0, 0] = 11  # an unknown node type
    bad["textures"] = tex
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene.from_arrays(64, 64, **bad)
    assert e.value.code == -4
    bad = dict(kw)
    g = dict(kw["geometries"][0])
    g["position_indices"] = np.full_like(g["position_indices"], 10 ** 6)
    bad["geometries"] = [g] + kw["geometries"][1:]
    with pytest.raises(Y.YmrtError):
        Y.HostScene.from_arrays(64, 64, **bad)


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["spheres", "volumetric"])
def test_arrays_render_like_the_file(ctx, halton_perm, scene_dir, name):
    hs, kw = arrays_of(name, scene_dir, 128, 128)
    ha = Y.HostScene.from_arrays(128, 128, **kw)
    a_scene, b_scene = Y.Scene(ctx, hs, halton_perm), Y.Scene(ctx, ha, halton_perm)
    s = Y.default_setting(spp=2, ray_depth=8, distant_light=True, volume=True)
    a, sa = a_scene.render(s, 1)
    b, sb = b_scene.render(s, 1)
    a_scene.close()
    b_scene.close()
    assert sa.extension_rays == sb.extension_rays and sa.shadow_rays == sb.shadow_rays
    assert np.allclose(a, b, rtol=1e-6, atol=1e-7)
