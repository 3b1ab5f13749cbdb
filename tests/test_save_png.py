"""The PNG writer (ymrt_save_png) against the reference's SavePngImage
(src/FileIO.cpp:167-194, run from the oracle build): both files decode to
the same 8-bit RGBA pixels, rows in the same order, for values inside and
outside [0, 1] and at the rounding boundaries. The two files' bytes differ
(different deflate and row filters); the pixels are the contract."""
import struct
import zlib

import numpy as np
import pytest

import ymrt_b200 as Y


def _read_png(path):
    """RGBA8, non-interlaced PNG -> (H, W, 4) uint8, top row first."""
    data = open(path, "rb").read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, hdr = 8, b"", None
    while pos < len(data):
        n, kind = struct.unpack(">I4s", data[pos:pos + 8])
        body = data[pos + 8:pos + 8 + n]
        assert zlib.crc32(kind + body) == struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0]
        if kind == b"IHDR":
            hdr = struct.unpack(">IIBBBBB", body)
        elif kind == b"IDAT":
            idat += body
        pos += 12 + n
    w, h, depth, ctype, _, _, interlace = hdr
    assert (depth, ctype, interlace) == (8, 6, 0)
    raw = zlib.decompress(idat)
    stride, bpp = 4 * w, 4
    out = np.zeros((h, stride), np.int32)
    prev = np.zeros(stride, np.int32)
    for y in range(h):
        f = raw[y * (stride + 1)]
        line = np.frombuffer(raw, np.uint8, stride, y * (stride + 1) + 1).astype(np.int32)
        cur = np.zeros(stride, np.int32)
        for x in range(stride):
            a = cur[x - bpp] if x >= bpp else 0
            b = prev[x]
            c = prev[x - bpp] if x >= bpp else 0
            if f == 0:
                p = 0
            elif f == 1:
                p = a
            elif f == 2:
                p = b
            elif f == 3:
                p = (a + b) // 2
            else:
                q = a + b - c
                pa, pb, pc = abs(q - a), abs(q - b), abs(q - c)
                p = a if (pa <= pb and pa <= pc) else (b if pb <= pc else c)
            cur[x] = (line[x] + p) & 0xFF
        out[y] = cur
        prev = cur
    return out.reshape(h, w, 4).astype(np.uint8)


def _image(seed, h=23, w=37):
    rng = np.random.default_rng(seed)
    img = rng.uniform(-0.5, 1.5, (h, w, 4)).astype(np.float32)
    # values at and around the rounding boundaries (k + 0.5) / 255
    edges = ((np.arange(h * w * 4) % 256) + 0.5) / 255.0
    img.reshape(-1)[::3] = np.nextafter(edges[::3].astype(np.float32), np.float32(2))
    img[0, :4] = [0.0, 1.0, -0.0, 0.5]
    return img


def _expected(img):
    c = np.clip(img, np.float32(0), np.float32(1))
    return (c * np.float32(255) + np.float32(0.5)).astype(np.uint8)[::-1]


def test_written_png_decodes_to_the_quantised_image(tmp_path):
    img = _image(1)
    Y.save_png(str(tmp_path / "sub" / "dir" / "frame.exr"), img)
    out = tmp_path / "sub" / "dir" / "frame.png"  # extension replaced, directories created
    assert out.exists() and not (tmp_path / "sub" / "dir" / "frame.exr").exists()
    np.testing.assert_array_equal(_read_png(out), _expected(img))


def test_written_png_matches_the_reference_writer(tmp_path, oracle):
    for seed in (2, 3):
        img = _image(seed, 17 + seed, 41)
        Y.save_png(str(tmp_path / f"ours{seed}.png"), img)
        assert oracle.save_png(str(tmp_path / f"ref{seed}.png"), img)
        ours, ref = _read_png(tmp_path / f"ours{seed}.png"), _read_png(tmp_path / f"ref{seed}.png")
        np.testing.assert_array_equal(ours, ref)


def test_bad_arguments_are_rejected(tmp_path):
    with pytest.raises(ValueError):
        Y.save_png(str(tmp_path / "a.png"), np.zeros((4, 4, 3), np.float32))
    with pytest.raises(Y.YmrtError):
        Y.save_png(str(tmp_path / "a.png"), np.zeros((0, 4, 4), np.float32))
    with pytest.raises(Y.YmrtError):
        Y.save_png("", np.zeros((2, 2, 4), np.float32))
