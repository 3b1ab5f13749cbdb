"""Texture nodes on the host: the solid (procedural) node types of the
format, textured material parameters and normal / bump maps as the loader
reads them, against the reference's own scene module.

The generated ``textured`` scene holds every solid node type on material
parameters and a medium density; the reference's own test scene
(src/model/CornellBox_Test.ymtmp: checkerboard albedo, metalness and bump map
on its ground) is checked too where the reference checkout is present. Node
records (the 20 words of ymrt_texture_desc), materials, volumes and instances
must equal the reference's bit for bit. The texture-graph checks (missing
inputs, cycles, graphs deeper than the evaluation stack, image nodes) and the
reference parser's attribute-name rule are exercised on small inputs.
"""
import os

import numpy as np
import pytest

import ymrt_b200 as Y
from ymrt_b200 import scenes
from test_scene_arrays import arrays_of
from test_scene_host import _meaningful


def _compare_prepared(ours, ref):
    assert np.array_equal(ours.instances(), ref.instances())
    for kind in ("materials", "volumes", "distant_lights", "textures"):
        a, b = _meaningful(kind, ours.records(kind)), _meaningful(kind, ref.records(kind))
        assert np.array_equal(a, b), kind
    la, lb = ours.lights(), ref.lights()
    assert np.array_equal(la[0], lb[0])
    assert np.array_equal(la[1].view(np.uint32), lb[1].view(np.uint32))
    for g in range(ref.counts()["geometries"]):
        assert np.array_equal(ours.triangles(g), ref.geometry_triangles(g)), f"mesh {g}"
        assert np.array_equal(ours.mesh_corners(g).view(np.uint32), ref.mesh_corners(g).view(np.uint32)), f"mesh {g}"


def test_textured_scene_covers_every_solid_node(scene_dir):
    hs = Y.HostScene(scenes.scene_path("textured", 0, scene_dir), 64, 64)
    types = set(hs.records("textures")[:, 0].tolist())
    assert set(range(1, 11)) <= types, types
    mats = hs.records("materials")
    default = mats[mats[:, 0] == 0]
    # every texture reference of DefaultMtl is used by some material: the words of diffuse_albedo_tex,
    # specular_albedo_tex, alpha_x/y_tex, specular_weight_tex, metalness_tex, transmission_weight_tex,
    # coat_albedo_tex, coat_weight_tex, coat_thickness_tex, coat_roughness_x/y_tex, normal and bump maps
    slots = [4, 8, 10, 12, 14, 16, 18, 24, 26, 28, 30, 32, 34, 35]
    assert all((default[:, w] != 0xFFFFFFFF).any() for w in slots), [w for w in slots if (default[:, w] == 0xFFFFFFFF).all()]


def test_textured_scene_prepares_like_the_reference(scene_dir, halton_perm, oracle):
    path = scenes.scene_path("textured", 0, scene_dir)
    _compare_prepared(Y.HostScene(path, 256, 256), oracle.RefScene(path, halton_perm, 256, 256))


def test_reference_test_scene_prepares_like_the_reference(halton_perm, oracle):
    """src/model/CornellBox_Test.ymtmp, read where the reference checkout is."""
    from oracle import build_ref
    path = os.path.join(build_ref.reference_root(), "src", "model", "CornellBox_Test.ymtmp")
    if not os.path.exists(path):
        pytest.skip("reference checkout absent")
    ours = Y.HostScene(path, 320, 240)
    ref = oracle.RefScene(path, halton_perm, 320, 240)
    _compare_prepared(ours, ref)
    tex = ours.records("textures")
    assert (tex[:, 0] == 3).sum() == 3  # the checkerboard albedo, metalness and bump nodes


def test_texture_nodes_from_arrays(scene_dir):
    hs, kw = arrays_of("textured", scene_dir, 64, 64)
    ha = Y.HostScene.from_arrays(64, 64, **kw)
    assert np.array_equal(ha.records("textures"), hs.records("textures"))
    assert np.array_equal(ha.records("materials"), hs.records("materials"))


def _bad_textures(kw, textures, materials=None):
    bad = dict(kw)
    bad["textures"] = np.asarray(textures, np.uint32)
    if materials is not None:
        bad["materials"] = materials
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene.from_arrays(64, 64, **bad)
    return e.value.code


def _node(kind, black=0xFFFFFFFF, white=0xFFFFFFFF, freq=1.0):
    r = np.zeros(Y.TEXTURE_WORDS, np.uint32)
    r[0], r[1], r[2] = kind, black, white
    r[7] = np.float32(freq).view(np.uint32)
    return r


def test_texture_graph_checks(scene_dir):
    hs, kw = arrays_of("cornell", scene_dir, 64, 64)
    const = _node(1)
    # an unknown node type is not supported; an image node needs a size, 1-4 channels and a wrap mode
    assert _bad_textures(kw, [_node(11)]) == -4
    assert _bad_textures(kw, [_node(0)]) == -1
    # a solid node needs both inputs
    assert _bad_textures(kw, [const, _node(3, 0)]) == -1
    # a graph read by a material: a cycle, and a chain deeper than the 8-node evaluation stack
    mats = kw["materials"].copy()
    mats[0, 4] = 0  # DefaultMtl.diffuse_albedo_tex of material 0 (after the type word and the rgb albedo)
    cyc = [_node(3, 1, 1), _node(3, 0, 0)]
    assert _bad_textures(kw, cyc, mats) == -1
    deep = [_node(3, k + 1, k + 1) for k in range(8)] + [const]  # 9 nodes on the path from node 0
    assert _bad_textures(kw, deep, mats) == -1
    ok = dict(kw)
    ok["textures"] = np.asarray(deep[1:], np.uint32)  # 8 nodes (renumbered): accepted
    ok["textures"][:, 1:3] = np.where(ok["textures"][:, 1:3] != 0xFFFFFFFF, ok["textures"][:, 1:3] - 1, 0xFFFFFFFF)
    ok["materials"] = mats
    Y.HostScene.from_arrays(64, 64, **ok)
    # deep graphs nothing reads are accepted
    unused = dict(kw)
    unused["textures"] = np.asarray(deep, np.uint32)
    Y.HostScene.from_arrays(64, 64, **unused)
    # a material referring to a node that does not exist
    mats2 = kw["materials"].copy()
    mats2[0, 4] = 5
    assert _bad_textures(kw, [const], mats2) == -1


def test_wave_parameters_are_illegal_statements(tmp_path, halton_perm, oracle):
    """The reference's statement check allows letters and '_' in attribute
    names only (src/core/YMParser.cpp:700-705), so NoiseTextureWave's
    freq_0 .. layer_count_1 make a file unreadable; ours reads it the same."""
    s = scenes.cornell_scene(0)
    s.textures.append(("ConstantTextureFloat", "w0", {"value": 0.0}))
    s.textures.append(("ConstantTextureFloat", "w1", {"value": 1.0}))
    s.textures.append(("NoiseTextureWave", "wave", {"texture_black_idx": "w0", "texture_white_idx": "w1",
                                                    "freq_0": 0.5}))
    path = scenes.write_scene(s, str(tmp_path / "wave_params.ymtmp"))
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene(path, 32, 32)
    assert e.value.code == -3
    with pytest.raises(RuntimeError):
        oracle.RefScene(path, halton_perm, 32, 32)


# ---- image textures ----

def test_image_scene_prepares_like_the_reference(scene_dir, halton_perm, oracle):
    """PNG files of every kind the scene uses (8-bit RGB / RGBA interlaced,
    16-bit grey, 4-bit palette with transparency, 2-bit grey): node records
    and decoded pixels equal the reference's (its image library plus its
    sRGB decode) bit for bit; the image whose file is missing is left out
    as the reference leaves it out."""
    path = scenes.scene_path("imaged", 0, scene_dir)
    ours, ref = Y.HostScene(path, 128, 128), oracle.RefScene(path, halton_perm, 128, 128)
    _compare_prepared(ours, ref)
    tex = ours.records("textures")
    images = np.flatnonzero(tex[:, 0] == 0)
    assert len(images) == 10
    for k in images:
        assert np.array_equal(ours.image_pixels(int(k)).view(np.uint32), ref.image_pixels(int(k)).view(np.uint32)), k
    mats = ours.records("materials")
    assert mats[1, 4] == 0xFFFFFFFF  # the ceiling's image did not load: its albedo stays constant


def _png_cases():
    rng = np.random.default_rng(99)
    cases = []
    for ctype, depths in ((0, (1, 2, 4, 8, 16)), (2, (8, 16)), (3, (1, 2, 4, 8)), (4, (8, 16)), (6, (8, 16))):
        n = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}[ctype]
        for depth in depths:
            for interlace in (False, True):
                h, w = 13, 19
                top = (1 << depth) - 1 if ctype != 3 else min(15, (1 << depth) - 1)
                img = rng.integers(0, top + 1, (h, w, n)).astype(np.uint16)
                kw = dict(depth=depth, color_type=ctype, interlace=interlace, first_filter=depth % 5)
                if ctype == 3:
                    kw["palette"] = rng.integers(0, 256, (top + 1, 3))
                    kw["trns"] = bytes(rng.integers(0, 256, top + 1 - 1).tolist()) if interlace else None
                if ctype == 0 and depth == 8 and interlace:
                    kw["trns"] = bytes([0, int(img[0, 0, 0])])  # a grey colour key present in the image
                if ctype == 2 and depth == 16 and not interlace:
                    v = img[1, 2]
                    kw["trns"] = b"".join(int(x).to_bytes(2, "big") for x in v)
                cases.append((f"c{ctype}d{depth}{'i' if interlace else ''}", img, kw))
    return cases


@pytest.mark.parametrize("case", _png_cases(), ids=lambda c: c[0])
def test_png_decoding_matches_the_reference(case, tmp_path, halton_perm, oracle):
    name, img, kw = case
    s = scenes.cornell_scene(0)
    s.image_files["img.png"] = (img, kw)
    for cs in ("SRGB", "Linear"):
        s.textures.append(("ImageTexture", "img_" + cs, {"texture_file_name": "img.png", "color_space": cs}))
    path = scenes.write_scene(s, str(tmp_path / "png_case.ymtmp"))
    ours, ref = Y.HostScene(path, 32, 32), oracle.RefScene(path, halton_perm, 32, 32)
    assert np.array_equal(ours.records("textures"), ref.records("textures"))
    for k in (0, 1):
        a, b = ours.image_pixels(k), ref.image_pixels(k)
        assert a.size == b.size and np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, k)


def _image_cases():
    rng = np.random.default_rng(7)
    cases = []
    yy, xx = np.mgrid[0:53, 0:61]
    smooth = np.stack([128 + 100 * np.sin(xx / 7.0), 128 + 90 * np.cos(yy / 5.0), (xx * 3 + yy * 2) % 256], axis=-1)
    noisy = rng.integers(0, 256, (53, 61, 3))
    for name, img in (("smooth", smooth), ("noisy", noisy)):
        for sub in ("444", "422", "420"):
            for q, rst in ((75, 0), (30, 3), (95, 1)):
                cases.append((f"jpg_{name}_{sub}_q{q}_r{rst}", "img.jpg", np.clip(img, 0, 255).astype(np.uint8),
                              dict(quality=q, subsampling=sub, restart=rst)))
    cases.append(("jpg_grey", "img.jpg", smooth[..., 0].astype(np.uint8), dict(quality=80)))
    cases.append(("jpg_grey_restart", "img.jpg", noisy[..., 1].astype(np.uint8), dict(quality=60, restart=2)))
    cases.append(("jpg_adobe_rgb", "img.jpg", np.clip(smooth, 0, 255).astype(np.uint8), dict(adobe_rgb=True)))
    cases.append(("jpg_tiny", "img.jpg", noisy[:3, :5].astype(np.uint8), dict(subsampling="420")))
    hdr = np.exp(rng.normal(0.0, 2.0, (11, 37, 3)))
    hdr[2, 3] = 0.0
    cases.append(("hdr_rle", "img.hdr", hdr, dict(rle=True)))
    cases.append(("hdr_flat", "img.hdr", hdr, dict(rle=False)))
    cases.append(("hdr_narrow", "img.hdr", hdr[:, :5], dict(rle=True)))
    rgb = np.clip(smooth, 0, 255).astype(np.uint8)[:13, :23]
    alpha = ((np.arange(13)[:, None] * 19 + np.arange(23)[None, :] * 7) % 256).astype(np.uint8)
    rgba = np.concatenate([rgb, alpha[..., None]], axis=-1)
    pal = rng.integers(0, 256, (256, 3)).astype(np.uint8)
    idx = rng.integers(0, 256, (13, 23)).astype(np.uint8)
    cases += [
        ("bmp24", "img.bmp", rgb, {}),
        ("bmp24_top_down", "img.bmp", rgb, dict(top_down=True)),
        ("bmp24_core", "img.bmp", rgb, dict(header=12)),
        ("bmp32", "img.bmp", rgba, dict(bpp=32)),
        ("bmp32_alpha_zero", "img.bmp", np.concatenate([rgb, np.zeros_like(alpha)[..., None]], -1), dict(bpp=32)),
        ("bmp16_555", "img.bmp", rgb, dict(bpp=16)),
        ("bmp16_565", "img.bmp", rgb, dict(bpp=16, masks=(0xF800, 0x7E0, 0x1F, 0))),
        ("bmp16_565_h56", "img.bmp", rgb, dict(bpp=16, header=56, masks=(0xF800, 0x7E0, 0x1F, 0))),
        ("bmp16_4444_v4", "img.bmp", rgba, dict(bpp=16, header=108, masks=(0xF00, 0xF0, 0xF, 0xF000))),
        ("bmp32_rgb_v5", "img.bmp", rgb, dict(bpp=32, header=124, masks=(0xFF0000, 0xFF00, 0xFF, 0))),
        ("bmp32_2_10_v5", "img.bmp", rgba, dict(bpp=32, header=124, masks=(0x3F << 20, 0x7F << 10, 0x1F, 0x3 << 30))),
        ("bmp8", "img.bmp", idx, dict(bpp=8, palette=pal)),
        # a core header's palette is sized from (offset - 38) / 3: the library
        # reads 252 of 256 entries and leaves the rest undefined, so no index
        # above 251 is compared
        ("bmp8_core", "img.bmp", idx % 252, dict(bpp=8, header=12, palette=pal)),
        ("bmp4", "img.bmp", idx % 16, dict(bpp=4, palette=pal[:16])),
        ("bmp1", "img.bmp", idx % 2, dict(bpp=1, palette=pal[:2], top_down=True)),
        ("tga24", "img.tga", rgb, {}),
        ("tga24_top_down", "img.tga", rgb, dict(top_down=True, image_id=b"ymrt")),
        ("tga32_rle", "img.tga", rgba, dict(rle=True)),
        ("tga24_rle_runs", "img.tga", np.repeat(rgb[:, ::4], 4, axis=1)[:, :23], dict(rle=True, top_down=True)),
        ("tga_grey", "img.tga", rgb[..., 1], dict(image_type=3)),
        ("tga_grey_rle", "img.tga", (rgb[..., 0] // 32) * 32, dict(image_type=3, rle=True)),
        ("tga_grey_alpha", "img.tga", np.stack([rgb[..., 2], alpha], -1), dict(image_type=3)),
        ("tga16", "img.tga", rgb, dict(bpp=16)),
        ("tga15_rle", "img.tga", rgb, dict(bpp=15, rle=True)),
        ("tga_pal24", "img.tga", idx, dict(image_type=1, palette=pal)),
        ("tga_pal32_rle", "img.tga", idx % 8, dict(image_type=1, rle=True,
                                                    palette=np.concatenate([pal[:8], pal[:8, :1]], -1),
                                                    palette_bits=32)),
        ("tga_pal16_idx16", "img.tga", idx, dict(image_type=1, bpp=16, palette=pal, palette_bits=16)),
    ]
    return cases


@pytest.mark.parametrize("case", _image_cases(), ids=lambda c: c[0])
def test_image_formats_decode_like_the_reference(case, tmp_path, halton_perm, oracle):
    """JPEG (baseline; grey, RGB and YCbCr with 4:4:4 / 4:2:2 / 4:2:0
    chroma, restart markers, sizes that are not whole MCUs), Radiance HDR
    (run-length and flat scanlines), BMP (core, info, V4 and V5 headers;
    1/4/8-bit palettes, 24-bit, 16/32-bit default and bit-field layouts, an
    all-zero alpha, either row order) and TGA (true colour, grey, grey +
    alpha, 15/16-bit, colour-mapped; raw and run-length; either row order),
    each decoded as the reference's loader decodes it: the same linear
    samples bit for bit."""
    name, fname, img, kw = case
    s = scenes.cornell_scene(0)
    s.image_files[fname] = (img, kw)
    for cs in ("SRGB", "Linear"):
        s.textures.append(("ImageTexture", "img_" + cs, {"texture_file_name": fname, "color_space": cs}))
    path = scenes.write_scene(s, str(tmp_path / "img_case.ymtmp"))
    ours, ref = Y.HostScene(path, 32, 32), oracle.RefScene(path, halton_perm, 32, 32)
    assert np.array_equal(ours.records("textures"), ref.records("textures"))
    for k in (0, 1):
        a, b = ours.image_pixels(k), ref.image_pixels(k)
        assert a.size == b.size and np.array_equal(a.view(np.uint32), b.view(np.uint32)), (name, k)


def test_unsupported_image_formats(tmp_path):
    """Variants the reference's library reads and this build does not
    decode (a progressive JPEG; a BMP with an unknown header size, which the
    library does not take for a BMP either) are YMRT_ERR_UNSUPPORTED, not a
    silent constant."""
    s = scenes.cornell_scene(0)
    s.textures.append(("ImageTexture", "jpg", {"texture_file_name": "photo.jpg", "color_space": "SRGB"}))
    path = scenes.write_scene(s, str(tmp_path / "jpg_case.ymtmp"))
    folder = scenes.texture_folder(path)
    os.makedirs(folder, exist_ok=True)
    # SOI, then a progressive frame header (SOF2)
    with open(os.path.join(folder, "photo.jpg"), "wb") as f:
        f.write(b"\xff\xd8\xff\xc2\x00\x0b\x08\x00\x10\x00\x10\x01\x01\x11\x00" + bytes(16))
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene(path, 32, 32)
    assert e.value.code == -4
    with open(os.path.join(folder, "photo.jpg"), "wb") as f:
        f.write(b"BM" + bytes(64))
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene(path, 32, 32)
    assert e.value.code == -4


def test_image_nodes_from_arrays(scene_dir):
    path = scenes.scene_path("imaged", 0, scene_dir)
    hs = Y.HostScene(path, 64, 64)
    _, kw = arrays_of("cornell", scene_dir, 64, 64)
    tex = hs.records("textures")
    k = int(np.flatnonzero(tex[:, 0] == 0)[0])
    kw = dict(kw)
    kw["textures"] = tex[k:k + 1]
    ha = Y.HostScene.from_arrays(64, 64, **kw)
    assert np.array_equal(ha.records("textures"), tex[k:k + 1])
    with pytest.raises(Y.YmrtError):
        ha.set_image(0, np.zeros(5, np.float32))  # wrong sample count
    ha.set_image(0, hs.image_pixels(k))
    assert np.array_equal(ha.image_pixels(0), hs.image_pixels(k))
    bad = tex[k:k + 1].copy()
    bad[0, 5] = 7  # seven channels
    kw["textures"] = bad
    with pytest.raises(Y.YmrtError) as e:
        Y.HostScene.from_arrays(64, 64, **kw)
    assert e.value.code == -1


def test_corrupt_png_is_left_out_like_the_reference(tmp_path, halton_perm, oracle):
    """A truncated PNG fails to decode in both loaders; the node is left out
    and the material that names it keeps its constant albedo."""
    s = scenes.cornell_scene(0)
    s.image_files["broken.png"] = (np.full((8, 8, 3), 128, np.uint16), dict(depth=8, color_type=2))
    s.textures.append(("ImageTexture", "broken", {"texture_file_name": "broken.png", "color_space": "SRGB"}))
    mats = dict((name, i) for i, (_, name, _) in enumerate(s.materials))
    kind, name, attrs = s.materials[mats["back_material"]]
    s.materials[mats["back_material"]] = (kind, name, {**attrs, "diffuse_albedo_tex": "broken"})
    path = scenes.write_scene(s, str(tmp_path / "broken_png.ymtmp"))
    png = os.path.join(scenes.texture_folder(path), "broken.png")
    data = open(png, "rb").read()
    with open(png, "wb") as f:
        f.write(data[: len(data) // 2])
    ours, ref = Y.HostScene(path, 32, 32), oracle.RefScene(path, halton_perm, 32, 32)
    assert ours.records("textures").shape[0] == 0 == ref.records("textures").shape[0]
    assert np.array_equal(_meaningful("materials", ours.records("materials")),
                          _meaningful("materials", ref.records("materials")))


def test_malformed_pngs_are_left_out(tmp_path, halton_perm, oracle):
    """PNGs the reference's image library refuses (a tRNS chunk on an image
    with alpha, a palette tRNS longer than the palette, an oversized header)
    leave the node out here too."""
    import struct
    import zlib
    s = scenes.cornell_scene(0)
    cases = {"alpha_trns.png": (np.full((4, 4, 4), 9, np.uint16), dict(depth=8, color_type=6, trns=b"\0\1\0\2\0\3")),
             "long_trns.png": (np.zeros((4, 4), np.uint16), dict(depth=8, color_type=3, palette=[[1, 2, 3]],
                                                                  trns=b"\1\2"))}
    for fname, img in cases.items():
        s.image_files[fname] = img
        s.textures.append(("ImageTexture", fname[:-4], {"texture_file_name": fname, "color_space": "Linear"}))
    s.textures.append(("ImageTexture", "huge", {"texture_file_name": "huge.png", "color_space": "Linear"}))
    path = scenes.write_scene(s, str(tmp_path / "bad_pngs.ymtmp"))

    def chunk(kind, body):
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    huge = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", 1 << 24, 1 << 24, 8, 2, 0, 0, 0))
    huge += chunk(b"IDAT", zlib.compress(b"\0" * 64)) + chunk(b"IEND", b"")
    with open(os.path.join(scenes.texture_folder(path), "huge.png"), "wb") as f:
        f.write(huge)
    assert Y.HostScene(path, 32, 32).records("textures").shape[0] == 0
    assert oracle.RefScene(path, halton_perm, 32, 32).records("textures").shape[0] == 0
