"""Seeded synthetic scenes in YMRT's ``.ymtmp`` text format.

The reference publishes no benchmark scenes (its only scene file ships with
meshes that are missing from the checkout), so the workloads are generated
from seeds with numpy ``PCG64``:

* ``cornell``  -- Cornell-box-like: 5 wall quads, 2 boxes rotated by U[0,45]
  degrees about y, 1 emissive quad (radiance 15); Lambertian albedos
  U[0.1,0.9] per channel; every object one instance.
* ``instanced`` -- ~1.2 M instanced triangles: 64 instances of an icosphere
  (subdivision 5, 20,480 triangles), a 256x256 fBm heightfield (131,072
  triangles), a 64-segment torus and a box, each with a random affine
  transform; 32 materials (GGX conductors with roughness U[0.05,0.8],
  dielectrics with IOR 1.5 and roughness U[0,0.3], diffuse); 2 quad lights.
* ``volumetric`` -- the Cornell scene plus a homogeneous fog box
  (sigma_t 0.05, albedo 0.8, g 0.6) and a heterogeneous medium whose density is
  a procedural fBm texture (the reference's ``NoiseTextureFBM``).
* ``spheres`` -- the Cornell walls with the analytic shapes of the format: a
  built-in ``Cube`` block (rotated, diffuse), ``Sphere`` blocks as a smooth
  dielectric (IOR 1.55), a rough conductor, a small emissive sphere beside the
  ceiling quad light, and a medium-filled boundary sphere (sigma_t 0.02) large
  enough to enclose the camera.

The file layout follows the reference's parser (src/core/YMParser.cpp:2330,
block types :57-92, attribute sets :94-372). Every float is written as the
shortest decimal that round-trips its float32 value, so the reference parser
(``std::stof``) and this project's loader read identical bits.

The Halton permutation table (src/core/SceneModule.cpp:1412
``InitHaltonPermuteTable``) is seeded by ``std::random_device`` in the
reference; here it is an explicit seeded input shared by both sides.
"""
from __future__ import annotations

import math
import os

import numpy as np

__all__ = [
    "first_primes", "halton_permutations", "cornell_scene", "instanced_scene", "volumetric_scene", "spheres_scene",
    "write_scene", "SCENES",
]


def first_primes(n: int = 1000) -> np.ndarray:
    """The first ``n`` primes (the reference tabulates 1000, 2..7919)."""
    limit = 8000
    sieve = np.ones(limit, dtype=bool)
    sieve[:2] = False
    for i in range(2, int(limit ** 0.5) + 1):
        if sieve[i]:
            sieve[i * i::i] = False
    p = np.nonzero(sieve)[0][:n]
    assert len(p) == n
    return p.astype(np.uint32)


def halton_permutations(seed: int = 0x594D5254) -> np.ndarray:
    """Concatenated random digit permutations for the first 1000 primes, in
    prime order (permutation k occupies ``sum(primes[:k])`` onwards), as the
    reference's table is laid out."""
    rng = np.random.Generator(np.random.PCG64(seed))
    parts = [rng.permutation(int(p)).astype(np.uint32) for p in first_primes()]
    return np.concatenate(parts)


# ---------------------------------------------------------------- meshes ---

class Mesh:
    """Triangle mesh with one position index and one normal index per corner
    (and optionally one texture-coordinate index)."""

    def __init__(self, name, positions, pos_idx, normals, nrm_idx, uvs=None, uv_idx=None):
        self.name = name
        self.positions = np.asarray(positions, dtype=np.float32).reshape(-1, 3)
        self.pos_idx = np.asarray(pos_idx, dtype=np.uint32).reshape(-1)
        self.normals = np.asarray(normals, dtype=np.float32).reshape(-1, 3)
        self.nrm_idx = np.asarray(nrm_idx, dtype=np.uint32).reshape(-1)
        self.uvs = None if uvs is None else np.asarray(uvs, dtype=np.float32).reshape(-1, 2)
        self.uv_idx = None if uv_idx is None else np.asarray(uv_idx, dtype=np.uint32).reshape(-1)
        assert len(self.pos_idx) == len(self.nrm_idx) and len(self.pos_idx) % 3 == 0
        assert self.uv_idx is None or len(self.uv_idx) == len(self.pos_idx)

    @property
    def triangle_count(self) -> int:
        return len(self.pos_idx) // 3


def quad_mesh(name="Geo_Quad") -> Mesh:
    p = [[-0.5, 0, -0.5], [-0.5, 0, 0.5], [0.5, 0, 0.5], [0.5, 0, -0.5]]
    idx = [0, 1, 2, 0, 2, 3]
    return Mesh(name, p, idx, [[0, 1, 0]], [0] * 6)


def uv_quad_mesh(name="Geo_UVQuad", repeat=1.0) -> Mesh:
    """The quad with texture coordinates [0, repeat]^2 over its corners."""
    p = [[-0.5, 0, -0.5], [-0.5, 0, 0.5], [0.5, 0, 0.5], [0.5, 0, -0.5]]
    idx = [0, 1, 2, 0, 2, 3]
    uv = [[0, 0], [0, repeat], [repeat, repeat], [repeat, 0]]
    return Mesh(name, p, idx, [[0, 1, 0]], [0] * 6, uv, idx)


def box_mesh(name="Geo_Box") -> Mesh:
    faces = []  # (normal, u axis, v axis)
    for axis in range(3):
        for sign in (1.0, -1.0):
            n = np.zeros(3)
            n[axis] = sign
            u = np.zeros(3)
            u[(axis + 1) % 3] = 1.0
            v = np.cross(n, u)
            faces.append((n, u, v))
    pos, pidx, nrm, nidx = [], [], [], []
    for fi, (n, u, v) in enumerate(faces):
        c = 0.5 * n
        corners = [c - 0.5 * u - 0.5 * v, c + 0.5 * u - 0.5 * v, c + 0.5 * u + 0.5 * v, c - 0.5 * u + 0.5 * v]
        base = len(pos)
        pos.extend(corners)
        nrm.append(n)
        for tri in ((0, 1, 2), (0, 2, 3)):
            pidx.extend(base + k for k in tri)
            nidx.extend([fi] * 3)
    return Mesh(name, pos, pidx, nrm, nidx)


def icosphere_mesh(subdivisions=5, name="Geo_Icosphere") -> Mesh:
    t = (1.0 + 5.0 ** 0.5) / 2.0
    verts = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
             [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    verts = [list(np.asarray(v) / np.linalg.norm(v)) for v in verts]
    faces = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
             [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
             [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (min(a, b), max(a, b))
            if key not in cache:
                m = np.asarray(verts[a]) + np.asarray(verts[b])
                verts.append(list(m / np.linalg.norm(m)))
                cache[key] = len(verts) - 1
            return cache[key]

        nf = []
        for a, b, c in faces:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
        faces = nf
    v = np.asarray(verts, dtype=np.float64)
    idx = np.asarray(faces, dtype=np.uint32).reshape(-1)
    return Mesh(name, v, idx, v, idx)


def _fbm2(x, y, rng_perm, octaves=5):
    """Value-noise fBm on a 2-D grid (numpy), used for heightfield displacement."""
    total = np.zeros_like(x)
    amp, freq = 1.0, 1.0
    for _ in range(octaves):
        xi = np.floor(x * freq).astype(np.int64)
        yi = np.floor(y * freq).astype(np.int64)
        xf = x * freq - xi
        yf = y * freq - yi

        def h(ix, iy):
            return rng_perm[(rng_perm[ix & 255] + iy) & 255] / 255.0

        sx = xf * xf * (3 - 2 * xf)
        sy = yf * yf * (3 - 2 * yf)
        a = h(xi, yi) + sx * (h(xi + 1, yi) - h(xi, yi))
        b = h(xi, yi + 1) + sx * (h(xi + 1, yi + 1) - h(xi, yi + 1))
        total += amp * (a + sy * (b - a))
        amp *= 0.5
        freq *= 2.0
    return total


def heightfield_mesh(res=256, seed=1, name="Geo_Heightfield") -> Mesh:
    rng = np.random.Generator(np.random.PCG64(seed))
    perm = rng.permutation(256)
    n = res + 1
    g = np.linspace(-0.5, 0.5, n)
    x, z = np.meshgrid(g, g, indexing="xy")
    hgt = 0.25 * _fbm2((x + 0.5) * 6.0, (z + 0.5) * 6.0, perm)
    pos = np.stack([x, hgt, z], axis=-1).reshape(-1, 3)
    # smooth normals from central differences
    dx = np.gradient(hgt, g, axis=1)
    dz = np.gradient(hgt, g, axis=0)
    nrm = np.stack([-dx, np.ones_like(hgt), -dz], axis=-1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    nrm = nrm.reshape(-1, 3)
    i, j = np.meshgrid(np.arange(res), np.arange(res), indexing="xy")
    v00 = (j * n + i).reshape(-1)
    v10 = v00 + 1
    v01 = v00 + n
    v11 = v01 + 1
    tris = np.stack([v00, v01, v11, v00, v11, v10], axis=-1).reshape(-1)  # +y facing
    return Mesh(name, pos, tris, nrm, tris)


def torus_mesh(major=64, minor=32, r_major=0.35, r_minor=0.15, name="Geo_Torus") -> Mesh:
    u = np.arange(major) * (2 * math.pi / major)
    v = np.arange(minor) * (2 * math.pi / minor)
    uu, vv = np.meshgrid(u, v, indexing="ij")
    cx, cz = np.cos(uu), np.sin(uu)
    pos = np.stack([(r_major + r_minor * np.cos(vv)) * cx, r_minor * np.sin(vv),
                    (r_major + r_minor * np.cos(vv)) * cz], axis=-1).reshape(-1, 3)
    nrm = np.stack([np.cos(vv) * cx, np.sin(vv), np.cos(vv) * cz], axis=-1).reshape(-1, 3)
    i, j = np.meshgrid(np.arange(major), np.arange(minor), indexing="ij")
    a = (i * minor + j)
    b = (((i + 1) % major) * minor + j)
    c = (((i + 1) % major) * minor + (j + 1) % minor)
    d = (i * minor + (j + 1) % minor)
    tris = np.stack([a, d, c, a, c, b], axis=-1).reshape(-1)
    return Mesh(name, pos, tris, nrm, tris)


# ------------------------------------------------------------ scene model ---

class Scene:
    def __init__(self):
        self.camera = None  # (from, look, fov)
        self.meshes = []
        self.cubes = []       # names of built-in unit cubes (Cube blocks)
        self.spheres = []     # (name, radius) of analytic spheres (Sphere blocks)
        self.transforms = []  # (name, translate, scale, rotate_deg)
        self.materials = []   # (kind, name, dict)
        self.textures = []    # (kind, name, dict)
        self.volumes = []     # (name, transform, sigma_t, albedo, g, density_texture or None)
        self.instances = []   # (name, geometry, transform, material, volume or None, boundary)
        self.distant_lights = []  # (name, transform, color, intensity, theta_max_deg)
        self.image_files = {}  # file name -> (samples, write_png keyword arguments), written beside the scene

    @property
    def triangle_count(self) -> int:
        by_name = {m.name: m.triangle_count for m in self.meshes}
        by_name.update({c: 12 for c in self.cubes})
        by_name.update({n: 0 for n, _ in self.spheres})
        return sum(by_name[i[1]] for i in self.instances)


def _f(v) -> str:
    # shortest positional decimal that reads back as the same float32 (the
    # reference's parser accepts no exponent notation)
    return np.format_float_positional(np.float32(v), unique=True, trim="-")


def _vec(v) -> str:
    return "<" + ",".join(_f(x) for x in v) + ">"


def _arr(a, fmt) -> str:
    return "[" + ",".join(fmt(x) for x in a) + "]"


_ADAM7 = ((0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2))


def _png_rows(img: np.ndarray, depth: int) -> np.ndarray:
    """Samples (h, w, n) packed into scanline bytes (h, row bytes), big-endian."""
    h, w, n = img.shape
    if depth == 16:
        return img.astype(">u2").reshape(h, w * n).view(np.uint8).reshape(h, -1)
    if depth == 8:
        return img.astype(np.uint8).reshape(h, w * n)
    per = 8 // depth
    flat = img.reshape(h, w * n).astype(np.uint8)
    pad = (-flat.shape[1]) % per
    flat = np.pad(flat, ((0, 0), (0, pad)))
    flat = flat.reshape(h, -1, per)
    shifts = (8 - depth * (np.arange(per) + 1)).astype(np.uint8)
    return np.bitwise_or.reduce(flat << shifts, axis=2).astype(np.uint8)


def _png_filter(rows: np.ndarray, bpp: int, first_filter: int) -> bytes:
    """Filters each scanline (types cycling from first_filter) and prefixes
    its filter byte."""
    out = bytearray()
    prev = np.zeros(rows.shape[1], np.int32)
    for y in range(rows.shape[0]):
        x = rows[y].astype(np.int32)
        a = np.concatenate([np.zeros(bpp, np.int32), x[:-bpp]]) if x.size > bpp else np.zeros_like(x)
        c = np.concatenate([np.zeros(bpp, np.int32), prev[:-bpp]]) if x.size > bpp else np.zeros_like(x)
        b = prev
        t = (first_filter + y) % 5
        if t == 0:
            f = x
        elif t == 1:
            f = x - a
        elif t == 2:
            f = x - b
        elif t == 3:
            f = x - (a + b) // 2
        else:
            p = a + b - c
            pa, pb, pc = np.abs(p - a), np.abs(p - b), np.abs(p - c)
            f = x - np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))
        out.append(t)
        out += (f & 255).astype(np.uint8).tobytes()
        prev = x
    return bytes(out)


def write_png(path: str, samples, depth: int = 8, color_type: int = 2, palette=None, trns: bytes | None = None,
              interlace: bool = False, first_filter: int = 0) -> str:
    """Writes a PNG (this project's encoder, for test images): samples
    (h, w, n) in file order (top row first; palette images hold indices in
    one channel), any bit depth the colour type allows, optional Adam7
    interlacing, scanline filters cycling through all five types."""
    import struct
    import zlib
    img = np.asarray(samples)
    if img.ndim == 2:
        img = img[..., None]
    h, w, n = img.shape
    bpp = max(1, n * depth // 8)
    if interlace:
        data = b"".join(_png_filter(_png_rows(img[y0::dy, x0::dx], depth), bpp, first_filter)
                        for x0, y0, dx, dy in _ADAM7 if x0 < w and y0 < h)
    else:
        data = _png_filter(_png_rows(img, depth), bpp, first_filter)

    def chunk(kind: bytes, body: bytes) -> bytes:
        return struct.pack(">I", len(body)) + kind + body + struct.pack(">I", zlib.crc32(kind + body) & 0xFFFFFFFF)

    png = b"\x89PNG\r\n\x1a\n" + chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, color_type, 0, 0, int(interlace)))
    if palette is not None:
        png += chunk(b"PLTE", np.asarray(palette, np.uint8).tobytes())
    if trns is not None:
        png += chunk(b"tRNS", bytes(trns))
    png += chunk(b"IDAT", zlib.compress(data, 6)) + chunk(b"IEND", b"")
    with open(path, "wb") as f:
        f.write(png)
    return path


# Baseline JPEG writer (this project's encoder, for test images; ITU-T T.81
# Annex K example quantisation and Huffman tables).
_K_LUM_Q = [16, 11, 10, 16, 24, 40, 51, 61, 12, 12, 14, 19, 26, 58, 60, 55, 14, 13, 16, 24, 40, 57, 69, 56,
            14, 17, 22, 29, 51, 87, 80, 62, 18, 22, 37, 56, 68, 109, 103, 77, 24, 35, 55, 64, 81, 104, 113, 92,
            49, 64, 78, 87, 103, 121, 120, 101, 72, 92, 95, 98, 112, 100, 103, 99]
_K_CHR_Q = [17, 18, 24, 47, 99, 99, 99, 99, 18, 21, 26, 66, 99, 99, 99, 99, 24, 26, 56, 99, 99, 99, 99, 99,
            47, 66, 99, 99, 99, 99, 99, 99] + [99] * 32
_K_DC_LUM = ([0, 1, 5, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0, 0, 0], list(range(12)))
_K_DC_CHR = ([0, 3, 1, 1, 1, 1, 1, 1, 1, 1, 1, 0, 0, 0, 0, 0], list(range(12)))
_K_AC_LUM = ([0, 2, 1, 3, 3, 2, 4, 3, 5, 5, 4, 4, 0, 0, 1, 0x7d], bytes.fromhex(
    "01020300041105122131410613516107227114328191a1082342b1c11552d1f02433627282090a161718191a25262728292a3435363738"
    "393a434445464748494a535455565758595a636465666768696a737475767778797a838485868788898a92939495969798999aa2a3a4a5"
    "a6a7a8a9aab2b3b4b5b6b7b8b9bac2c3c4c5c6c7c8c9cad2d3d4d5d6d7d8d9dae1e2e3e4e5e6e7e8e9eaf1f2f3f4f5f6f7f8f9fa"))
_K_AC_CHR = ([0, 2, 1, 2, 4, 4, 3, 4, 7, 5, 4, 4, 0, 1, 2, 0x77], bytes.fromhex(
    "000102031104052131061241510761711322328108144291a1b1c109233352f0156272d10a162434e125f11718191a262728292a35363738"
    "393a434445464748494a535455565758595a636465666768696a737475767778797a82838485868788898a92939495969798999aa2a3a4a5"
    "a6a7a8a9aab2b3b4b5b6b7b8b9bac2c3c4c5c6c7c8c9cad2d3d4d5d6d7d8d9dae2e3e4e5e6e7e8e9eaf2f3f4f5f6f7f8f9fa"))
_ZIGZAG = [0, 1, 8, 16, 9, 2, 3, 10, 17, 24, 32, 25, 18, 11, 4, 5, 12, 19, 26, 33, 40, 48, 41, 34, 27, 20, 13, 6, 7, 14,
           21, 28, 35, 42, 49, 56, 57, 50, 43, 36, 29, 22, 15, 23, 30, 37, 44, 51, 58, 59, 52, 45, 38, 31, 39, 46, 53,
           60, 61, 54, 47, 55, 62, 63]


def _huff_codes(counts, symbols):
    codes, code, k = {}, 0, 0
    for length in range(1, 17):
        for _ in range(counts[length - 1]):
            codes[symbols[k]] = (code, length)
            code += 1
            k += 1
        code <<= 1
    return codes


class _BitWriter:
    def __init__(self):
        self.out = bytearray()
        self.acc = 0
        self.n = 0

    def put(self, value, length):
        for b in range(length - 1, -1, -1):
            self.acc = (self.acc << 1) | ((value >> b) & 1)
            self.n += 1
            if self.n == 8:
                self.out.append(self.acc)
                if self.acc == 0xFF:
                    self.out.append(0)
                self.acc = self.n = 0

    def flush(self):
        while self.n:
            self.put(1, 1)


def write_jpeg(path: str, samples, quality: int = 75, subsampling: str = "420", restart: int = 0,
               adobe_rgb: bool = False) -> str:
    """Writes a baseline JPEG (this project's encoder, for test images):
    samples (h, w) grey or (h, w, 3) RGB uint8, top row first; chroma
    subsampling "444", "422" or "420"; a restart marker every `restart` MCUs
    (0: none); adobe_rgb: store R, G, B without colour transform (Adobe APP14
    transform 0, no JFIF marker)."""
    import struct
    img = np.asarray(samples, np.float64)
    grey = img.ndim == 2
    h, w = img.shape[:2]
    scale = 5000 // quality if quality < 50 else 200 - 2 * quality
    def qtab(base):
        return [min(255, max(1, (b * scale + 50) // 100)) for b in base]
    ql, qc = qtab(_K_LUM_Q), qtab(_K_CHR_Q)
    if grey:
        planes = [img]
        sf = [(1, 1)]
    else:
        r, g, b = img[..., 0], img[..., 1], img[..., 2]
        if adobe_rgb:
            planes = [r, g, b]
            sf = [(1, 1)] * 3
        else:
            y = 0.299 * r + 0.587 * g + 0.114 * b
            cb = -0.168736 * r - 0.331264 * g + 0.5 * b + 128
            cr = 0.5 * r - 0.418688 * g - 0.081312 * b + 128
            hs, vs = {"444": (1, 1), "422": (2, 1), "420": (2, 2)}[subsampling]
            planes = [y, cb, cr]
            sf = [(hs, vs), (1, 1), (1, 1)]
    hmax, vmax = max(f[0] for f in sf), max(f[1] for f in sf)
    mx, my = -(-w // (8 * hmax)), -(-h // (8 * vmax))
    n_comp = len(planes)
    comp_planes = []
    for k, pl in enumerate(planes):
        ch, cv = sf[k]
        dx, dy = hmax // ch, vmax // cv
        pw, ph = mx * ch * 8, my * cv * 8
        full = np.pad(pl, ((0, my * vmax * 8 - h), (0, mx * hmax * 8 - w)), mode="edge")
        sub = full.reshape(ph, dy, pw, dx).mean(axis=(1, 3))
        comp_planes.append(sub - 128.0)
    # orthonormal 8-point DCT-II
    n = np.arange(8)
    C = np.cos((2 * n[None, :] + 1) * n[:, None] * np.pi / 16) * np.sqrt(2 / 8)
    C[0] /= np.sqrt(2)
    tabs = [ql] + [qc] * (n_comp - 1) if not adobe_rgb else [ql] * n_comp
    dc_codes = [_huff_codes(*_K_DC_LUM), _huff_codes(*_K_DC_CHR)]
    ac_codes = [_huff_codes(*_K_AC_LUM), _huff_codes(*_K_AC_CHR)]
    tsel = [0] + [1] * (n_comp - 1) if not adobe_rgb else [0] * n_comp
    bw = _BitWriter()
    pred = [0] * n_comp

    def bits_of(v):
        m = abs(v)
        nbits = m.bit_length()
        return nbits, (v if v >= 0 else v + (1 << nbits) - 1)

    def block(k, by, bx):
        blk = comp_planes[k][by * 8:by * 8 + 8, bx * 8:bx * 8 + 8]
        coef = C @ blk @ C.T
        zz = coef.reshape(64)[_ZIGZAG]
        qz = np.rint(zz / np.array(tabs[k], np.float64)).astype(int)
        diff = int(qz[0]) - pred[k]
        pred[k] = int(qz[0])
        nb, v = bits_of(diff)
        c, l = dc_codes[tsel[k]][nb]
        bw.put(c, l)
        if nb:
            bw.put(v, nb)
        run = 0
        for i in range(1, 64):
            a = int(qz[i])
            if a == 0:
                run += 1
                continue
            while run > 15:
                c, l = ac_codes[tsel[k]][0xF0]
                bw.put(c, l)
                run -= 16
            nb, v = bits_of(a)
            c, l = ac_codes[tsel[k]][(run << 4) | nb]
            bw.put(c, l)
            bw.put(v, nb)
            run = 0
        if run:
            c, l = ac_codes[tsel[k]][0x00]
            bw.put(c, l)

    data = bytearray()
    mcu, rst = 0, 0
    if n_comp == 1:
        units = [(0, by, bx) for by in range(-(-h // 8)) for bx in range(-(-w // 8))]
        groups = [[u] for u in units]
    else:
        groups = []
        for j in range(my):
            for i in range(mx):
                groups.append([(k, j * sf[k][1] + y, i * sf[k][0] + x) for k in range(n_comp)
                               for y in range(sf[k][1]) for x in range(sf[k][0])])
    for g in groups:
        if restart and mcu and mcu % restart == 0:
            bw.flush()
            data += bw.out + bytes([0xFF, 0xD0 + rst])
            bw.out = bytearray()
            rst = (rst + 1) & 7
            pred = [0] * n_comp
        for k, by, bx in g:
            block(k, by, bx)
        mcu += 1
    bw.flush()
    data += bw.out

    def seg(marker, body):
        return bytes([0xFF, marker]) + struct.pack(">H", len(body) + 2) + body

    out = b"\xff\xd8"
    if adobe_rgb:
        out += seg(0xEE, b"Adobe" + bytes([0, 100, 0, 0, 0, 0, 0]))
    else:
        out += seg(0xE0, b"JFIF\x00\x01\x01\x00\x00\x01\x00\x01\x00\x00")
    out += seg(0xDB, bytes([0]) + bytes(ql))
    if n_comp > 1 and not adobe_rgb:
        out += seg(0xDB, bytes([1]) + bytes(qc))
    out += seg(0xC0, struct.pack(">BHHB", 8, h, w, n_comp) + b"".join(
        bytes([k + 1, (sf[k][0] << 4) | sf[k][1], 0 if (k == 0 or adobe_rgb) else 1]) for k in range(n_comp)))
    for cls, tabsel, spec in ((0, 0, _K_DC_LUM), (1, 0, _K_AC_LUM), (0, 1, _K_DC_CHR), (1, 1, _K_AC_CHR)):
        if tabsel == 1 and (n_comp == 1 or adobe_rgb):
            continue
        out += seg(0xC4, bytes([(cls << 4) | tabsel]) + bytes(spec[0]) + bytes(spec[1]))
    if restart:
        out += seg(0xDD, struct.pack(">H", restart))
    out += seg(0xDA, bytes([n_comp]) + b"".join(
        bytes([k + 1, 0x00 if (k == 0 or adobe_rgb) else 0x11]) for k in range(n_comp)) + bytes([0, 63, 0]))
    out += bytes(data) + b"\xff\xd9"
    with open(path, "wb") as f:
        f.write(out)
    return path


def write_hdr(path: str, rgb, rle: bool = True) -> str:
    """Writes a Radiance RGBE file (this project's encoder, for test images):
    rgb (h, w, 3) float, top row first; per-channel run-length scanlines when
    rle (and 8 <= w < 32768), else flat pixels."""
    img = np.asarray(rgb, np.float64)
    h, w = img.shape[:2]
    m = img.max(axis=2)
    e = np.zeros((h, w), np.int64)
    mant = np.zeros((h, w), np.float64)
    nz = m > 1e-32
    mant[nz], e[nz] = np.frexp(m[nz])
    rgbe = np.zeros((h, w, 4), np.uint8)
    f = np.where(nz, mant * 256.0 / np.where(nz, m, 1.0), 0.0)
    rgbe[..., :3] = np.clip(np.floor(img * f[..., None]), 0, 255).astype(np.uint8)
    rgbe[..., 3] = np.where(nz, e + 128, 0).astype(np.uint8)
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        if not rle or w < 8 or w >= 32768:
            out += rgbe[y].tobytes()
            continue
        out += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            row = rgbe[y, :, c]
            i = 0
            while i < w:
                run = 1
                while i + run < w and run < 127 and row[i + run] == row[i]:
                    run += 1
                if run >= 3:
                    out += bytes([128 + run, int(row[i])])
                    i += run
                    continue
                j = i
                while j < w and j - i < 128 and not (j + 2 < w and row[j] == row[j + 1] == row[j + 2]):
                    j += 1
                out += bytes([j - i]) + row[i:j].tobytes()
                i = j
    with open(path, "wb") as f:
        f.write(bytes(out))
    return path


def write_bmp(path: str, samples, bpp: int = 24, header: int = 40, top_down: bool = False, masks=None,
              palette=None) -> str:
    """Writes a Windows bitmap (this project's encoder, for test images):
    samples (h, w, n) top row first, or (h, w) palette indices with palette
    (k, 3) RGB for bpp 1/4/8; header 12 (core), 40, 56, 108 or 124 bytes;
    masks (r, g, b, a) pack 16/32-bit pixels as BI_BITFIELDS (header 40/56:
    three masks after the header; 108/124: all four inside it), else the
    default layouts (16: 5-5-5, 32: B, G, R, A bytes)."""
    import struct
    img = np.asarray(samples, np.uint8)
    h, w = img.shape[:2]
    compress = 3 if masks is not None else 0
    dib = bytearray()
    if header == 12:
        dib += struct.pack("<IHHHH", 12, w, h, 1, bpp)
    else:
        dib += struct.pack("<IiiHHIIiiII", header, w, -h if top_down else h, 1, bpp, compress, 0, 2835, 2835, 0, 0)
        if header == 56:
            dib += struct.pack("<4I", *(masks or (0, 0, 0, 0)))
        elif header in (108, 124):
            dib += struct.pack("<4I", *(masks or (0, 0, 0, 0))) + struct.pack("<I", 0x73524742) + bytes(36 + 12)
            if header == 124:
                dib += bytes(16)
        if masks is not None and header in (40, 56):
            dib += struct.pack("<3I", *masks[:3])
    pal = b""
    if bpp < 16:
        k = np.asarray(palette, np.uint8)
        pal = b"".join(bytes([c[2], c[1], c[0]]) + (b"" if header == 12 else b"\0") for c in k)
    offset = 14 + len(dib) + len(pal)
    rows = []
    for y in (range(h) if top_down else range(h - 1, -1, -1)):
        r = img[y]
        if bpp < 16:
            idx = [int(v) for v in r]
            if bpp == 8:
                row = bytes(idx)
            else:
                per = 8 // bpp
                row = bytearray((w + per - 1) // per)
                for i, v in enumerate(idx):
                    row[i // per] |= v << (8 - bpp * (1 + i % per))
                row = bytes(row)
        elif bpp == 24:
            row = r[:, [2, 1, 0]].tobytes()
        else:
            m = masks or ((31 << 10, 31 << 5, 31, 0) if bpp == 16 else (0xFF0000, 0xFF00, 0xFF, 0xFF000000))
            px = np.zeros(w, np.uint64)
            for c, mask in enumerate(m):
                if not mask or c >= r.shape[1]:
                    continue
                low = (mask & -mask).bit_length() - 1
                bits = bin(mask).count("1")
                px |= ((r[:, c].astype(np.uint64) >> np.uint64(8 - bits)) << np.uint64(low))
            row = px.astype("<u2" if bpp == 16 else "<u4").tobytes()
        rows.append(row + bytes((-len(row)) % 4))
    body = b"".join(rows)
    out = b"BM" + struct.pack("<IHHI", offset + len(body), 0, 0, offset) + bytes(dib) + pal + body
    with open(path, "wb") as f:
        f.write(out)
    return path


def write_tga(path: str, samples, image_type: int = 2, bpp: int | None = None, rle: bool = False,
              top_down: bool = False, palette=None, palette_bits: int = 24, image_id: bytes = b"") -> str:
    """Writes a Truevision TGA (this project's encoder, for test images):
    samples (h, w, n) top row first, or (h, w) indices into palette (k, n)
    for image_type 1; true-colour pixels stored B, G, R(, A), 15/16-bit
    pixels as five bits per channel; rle packs run-length packets (runs and
    literal spans, which may cross rows)."""
    import struct
    img = np.asarray(samples, np.uint8)
    h, w = img.shape[:2]
    n = 1 if img.ndim == 2 else img.shape[2]
    if bpp is None:
        bpp = 8 if image_type == 1 else 8 * n

    def pixel_bytes(v, bits):
        v = np.atleast_1d(v)
        if bits in (15, 16) and len(v) == 3:
            p = ((int(v[0]) >> 3) << 10) | ((int(v[1]) >> 3) << 5) | (int(v[2]) >> 3)
            return struct.pack("<H", p)
        if len(v) >= 3:
            return bytes([v[2], v[1], v[0]]) + bytes(v[3:])
        return bytes(int(x) for x in v)

    pal = b""
    if image_type == 1:
        k = np.asarray(palette, np.uint8)
        pal = b"".join(pixel_bytes(c, palette_bits) for c in k)
        order = img if top_down else img[::-1]
        pixels = [struct.pack("<B" if bpp == 8 else "<H", int(i)) for i in order.reshape(-1)]
    else:
        order = img if top_down else img[::-1]
        flat = order.reshape(h * w, n)
        pixels = [pixel_bytes(p, bpp) for p in flat]
    if rle:
        data = bytearray()
        i = 0
        while i < len(pixels):
            run = 1
            while i + run < len(pixels) and run < 128 and pixels[i + run] == pixels[i]:
                run += 1
            if run >= 2:
                data += bytes([0x80 | (run - 1)]) + pixels[i]
                i += run
                continue
            j = i
            while j < len(pixels) and j - i < 128 and not (j + 1 < len(pixels) and pixels[j] == pixels[j + 1]):
                j += 1
            data += bytes([j - i - 1]) + b"".join(pixels[i:j])
            i = j
    else:
        data = b"".join(pixels)
    cmap = 1 if image_type == 1 else 0
    hdr = struct.pack("<BBBHHBHHHHBB", len(image_id), cmap, image_type + (8 if rle else 0), 0,
                      len(palette) if cmap else 0, palette_bits if cmap else 0, 0, 0, w, h, bpp,
                      0x20 if top_down else 0)
    with open(path, "wb") as f:
        f.write(hdr + image_id + pal + bytes(data))
    return path


def texture_folder(path: str) -> str:
    """Where a scene file's image textures lie: texture_<stem>_<extension>
    beside it (get_texture_folder_from_scene_file, src/core/YMParser.cpp:20-30)."""
    d, name = os.path.split(os.path.abspath(path))
    stem, ext = os.path.splitext(name)
    return os.path.join(d, f"texture_{stem}_{ext[1:]}")


def write_scene(scene: Scene, path: str) -> str:
    out = []
    if scene.image_files:
        folder = texture_folder(path)
        os.makedirs(folder, exist_ok=True)
        for fname, (samples, kw) in scene.image_files.items():
            writer = {".jpg": write_jpeg, ".jpeg": write_jpeg, ".hdr": write_hdr, ".bmp": write_bmp,
                      ".tga": write_tga}.get(os.path.splitext(fname)[1].lower(), write_png)
            writer(os.path.join(folder, fname), samples, **kw)
    frm, look, fov = scene.camera
    out.append(f"Begin(Camera);\n\tfov = {_f(fov)};\n\tfrom = {_vec(frm)};\n\tlook = {_vec(look)};\nEnd(Camera);\n")
    for m in scene.meshes:
        n = m.triangle_count
        corners = np.arange(3 * n, dtype=np.uint32)
        pos = m.positions.astype(np.float32).reshape(-1)
        nrm = m.normals.astype(np.float32).reshape(-1)
        out.append("Begin(Mesh);\n")
        out.append(f'\tname = "{m.name}";\n')
        out.append("\tmesh_triangles = " + _arr(corners.tolist(), str) + ";\n")
        out.append("\tmesh_position_indices = " + _arr(m.pos_idx.tolist(), str) + ";\n")
        out.append("\tmesh_positions = " + _arr(pos, _f) + ";\n")
        out.append("\tmesh_normal_indices = " + _arr(m.nrm_idx.tolist(), str) + ";\n")
        out.append("\tmesh_normals = " + _arr(nrm, _f) + ";\n")
        if m.uv_idx is not None:
            out.append("\tmesh_texcoord_indices = " + _arr(m.uv_idx.tolist(), str) + ";\n")
            out.append("\tmesh_texcoords = " + _arr(m.uvs.reshape(-1), _f) + ";\n")
        out.append("End(Mesh);\n")
    for name in scene.cubes:
        out.append(f'Begin(Cube);\n\tname = "{name}";\nEnd(Cube);\n')
    for name, radius in scene.spheres:
        out.append(f'Begin(Sphere);\n\tname = "{name}";\n\tradius = {_f(radius)};\nEnd(Sphere);\n')
    for name, t, s, r in scene.transforms:
        out.append(f'Begin(Transform);\n\tname = "{name}";\n\ttranslate = {_vec(t)};\n\tscale = {_vec(s)};\n'
                   f'\trotate = {_vec(r)};\nEnd(Transform);\n')
    for name, tr, color, intensity, theta_max in scene.distant_lights:
        out.append(f'Begin(DistantLight);\n\tname = "{name}";\n\ttransform_index = "{tr}";\n'
                   f"\tlight_color = {_vec(color)};\n\tintensity = {_f(intensity)};\n\ttheta_max = {_f(theta_max)};\n"
                   "End(DistantLight);\n")
    for kind, name, attrs in scene.textures:
        out.append(f"Begin({kind});\n\tname = \"{name}\";\n")
        for k, v in attrs.items():
            if isinstance(v, str):
                out.append(f'\t{k} = "{v}";\n')
            elif isinstance(v, (list, tuple, np.ndarray)):
                out.append(f"\t{k} = {_vec(v)};\n")
            elif isinstance(v, bool):
                out.append(f"\t{k} = {'true' if v else 'false'};\n")
            elif isinstance(v, int):
                out.append(f"\t{k} = {v};\n")
            else:
                out.append(f"\t{k} = {_f(v)};\n")
        out.append(f"End({kind});\n")
    for kind, name, attrs in scene.materials:
        out.append(f"Begin({kind});\n\tname = \"{name}\";\n")
        for k, v in attrs.items():
            if isinstance(v, str):  # a texture node's name
                out.append(f'\t{k} = "{v}";\n')
            elif isinstance(v, (list, tuple, np.ndarray)):
                out.append(f"\t{k} = {_vec(v)};\n")
            elif isinstance(v, int):
                out.append(f"\t{k} = {v};\n")
            else:
                out.append(f"\t{k} = {_f(v)};\n")
        out.append(f"End({kind});\n")
    for name, tr, sigma, albedo, g, dens in scene.volumes:
        out.append(f'Begin(Volume);\n\tname = "{name}";\n\ttransform_index = "{tr}";\n\tsigma_t = {_vec(sigma)};\n'
                   f"\talbedo = {_vec(albedo)};\n\tg = {_f(g)};\n")
        if dens is not None:
            out.append(f'\tdensity_texture_index = "{dens}";\n')
        out.append("End(Volume);\n")
    for name, geo, tr, mat, vol, boundary in scene.instances:
        out.append(f'Begin(PrimitiveInstance);\n\tname = "{name}";\n\tgeometry_index = "{geo}";\n'
                   f'\ttransform_index = "{tr}";\n\tmaterial_index = "{mat}";\n')
        if vol is not None:
            out.append(f'\tinner_volume_index = "{vol}";\n')
        out.append(f"\ttreat_as_boundary = {'true' if boundary else 'false'};\nEnd(PrimitiveInstance);\n")
    d = os.path.dirname(os.path.abspath(path))
    os.makedirs(d, exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        f.write("".join(out))
    os.replace(tmp, path)
    return path


def _lambert(rgb) -> dict:
    return {"diffuse_albedo": list(rgb), "specular_weight": 0.0, "metalness": 0.0, "transmission_weight": 0.0,
            "coat_weight": 0.0}


def cornell_scene(seed: int = 0) -> Scene:
    rng = np.random.Generator(np.random.PCG64(seed))
    s = Scene()
    s.camera = ((0.0, 0.0, 3.4), (0.0, 0.0, 0.0), 40.0)
    s.meshes = [quad_mesh(), box_mesh()]
    walls = [("floor", (0, -1, 0), (0, 0, 0)), ("ceiling", (0, 1, 0), (180, 0, 0)),
             ("back", (0, 0, -1), (90, 0, 0)), ("left", (-1, 0, 0), (0, 0, -90)),
             ("right", (1, 0, 0), (0, 0, 90))]
    for name, t, r in walls:
        s.transforms.append((name + "_transform", t, (2, 1, 2), r))
        s.materials.append(("DefaultMaterial", name + "_material", _lambert(rng.uniform(0.1, 0.9, 3))))
        s.instances.append((name, "Geo_Quad", name + "_transform", name + "_material", None, False))
    boxes = [("tall_box", (-0.35, -0.399, -0.3), (0.6, 1.2, 0.6)), ("short_box", (0.35, -0.699, 0.3), (0.6, 0.6, 0.6))]
    for name, t, sc in boxes:
        s.transforms.append((name + "_transform", t, sc, (0.0, float(rng.uniform(0, 45)), 0.0)))
        s.materials.append(("DefaultMaterial", name + "_material", _lambert(rng.uniform(0.1, 0.9, 3))))
        s.instances.append((name, "Geo_Box", name + "_transform", name + "_material", None, False))
    s.transforms.append(("light_transform", (0, 0.995, 0), (0.5, 1, 0.5), (180, 0, 0)))
    s.materials.append(("LightMaterial", "light_material", {"light_color": [1.0, 1.0, 1.0], "intensity": 15.0}))
    s.instances.append(("light", "Geo_Quad", "light_transform", "light_material", None, False))
    return s


def instanced_scene(seed: int = 0) -> Scene:
    rng = np.random.Generator(np.random.PCG64(seed))
    s = Scene()
    s.camera = ((0.0, 9.0, 24.0), (0.0, 1.5, 0.0), 45.0)
    sphere, hfield, torus, box = icosphere_mesh(5), heightfield_mesh(256, seed + 1), torus_mesh(), box_mesh()
    s.meshes = [sphere, hfield, torus, box, quad_mesh()]
    # 7 heightfields + 12 spheres + 16 tori + 29 boxes = 1,229,148 triangles in 64 instances
    kinds = ["Geo_Heightfield"] * 7 + ["Geo_Icosphere"] * 12 + ["Geo_Torus"] * 16 + ["Geo_Box"] * 29
    order = rng.permutation(len(kinds))
    closed = {"Geo_Icosphere", "Geo_Torus", "Geo_Box"}
    for m in range(32):
        kind = m % 3
        if kind == 0:
            r = float(rng.uniform(0.05, 0.8))
            attrs = {"diffuse_albedo": list(rng.uniform(0.4, 0.95, 3)), "specular_albedo": list(rng.uniform(0.5, 1.0, 3)),
                     "roughness_x": r, "roughness_y": r, "metalness": 1.0}
        elif kind == 1:
            r = float(rng.uniform(0.0, 0.3))
            attrs = {"diffuse_albedo": [0.5, 0.5, 0.5], "specular_albedo": list(rng.uniform(0.85, 1.0, 3)),
                     "roughness_x": r, "roughness_y": r, "ior_n": 1.5, "metalness": 0.0, "specular_weight": 1.0,
                     "transmission_weight": 1.0}
        else:
            attrs = _lambert(rng.uniform(0.1, 0.9, 3))
        s.materials.append(("DefaultMaterial", f"material_{m}", attrs))
    diffuse = [m for m in range(32) if m % 3 == 2]
    for i, k in enumerate(order):
        geo = kinds[k]
        if geo == "Geo_Heightfield":
            sc = rng.uniform(5.0, 9.0)
            scale = (sc, float(rng.uniform(2.0, 4.0)), sc)
            t = (float(rng.uniform(-8, 8)), float(rng.uniform(-1.0, 0.0)), float(rng.uniform(-8, 8)))
            rot = (0.0, float(rng.uniform(0, 360)), 0.0)
        else:
            sc = float(rng.uniform(0.6, 2.2))
            scale = (sc * float(rng.uniform(0.8, 1.25)), sc * float(rng.uniform(0.8, 1.25)), sc * float(rng.uniform(0.8, 1.25)))
            t = (float(rng.uniform(-9, 9)), float(rng.uniform(0.3, 4.0)), float(rng.uniform(-9, 9)))
            rot = tuple(float(x) for x in rng.uniform(0, 360, 3))
        mat = int(rng.integers(0, 32))
        if mat % 3 == 1 and geo not in closed:
            mat = diffuse[int(rng.integers(0, len(diffuse)))]
        s.transforms.append((f"t_{i}", t, scale, rot))
        s.instances.append((f"inst_{i}", geo, f"t_{i}", f"material_{mat}", None, False))
    for li, (lt, rot) in enumerate((((-5.0, 14.0, 2.0), (180, 0, 15)), ((6.0, 12.0, -4.0), (180, 0, -20)))):
        s.transforms.append((f"light_t_{li}", lt, (6.0, 1.0, 6.0), rot))
        s.materials.append(("LightMaterial", f"light_material_{li}", {"light_color": [1.0, 0.95, 0.9], "intensity": 12.0}))
        s.instances.append((f"light_{li}", "Geo_Quad", f"light_t_{li}", f"light_material_{li}", None, False))
    return s


def volumetric_scene(seed: int = 0) -> Scene:
    s = cornell_scene(seed)
    s.textures.append(("ConstantTextureFloat", "density_black", {"value": 0.0}))
    s.textures.append(("ConstantTextureFloat", "density_white", {"value": 1.0}))
    s.textures.append(("NoiseTextureFBM", "density_fbm", {
        "texture_black_idx": "density_black", "texture_white_idx": "density_white", "frequency": 4.0,
        "lacunarity": 2.0, "gain": 0.5, "layer_count": 4, "amplitude": 1.0, "offset": 0.0}))
    s.transforms.append(("fog_transform", (0.0, 0.0, 0.0), (1.98, 1.98, 1.98), (0, 0, 0)))
    s.volumes.append(("fog_volume", "fog_transform", (0.05, 0.05, 0.05), (0.8, 0.8, 0.8), 0.6, None))
    s.materials.append(("DefaultMaterial", "boundary_material", {"ior_n": 1.0}))
    s.instances.append(("fog_box", "Geo_Box", "fog_transform", "boundary_material", "fog_volume", True))
    s.transforms.append(("smoke_transform", (0.3, 0.2, 0.0), (0.7, 0.7, 0.7), (0, 0, 0)))
    s.volumes.append(("smoke_volume", "smoke_transform", (2.0, 2.0, 2.0), (0.9, 0.9, 0.9), 0.0, "density_fbm"))
    s.materials.append(("DefaultMaterial", "smoke_boundary_material", {"ior_n": 1.0, "ior_priority": 1}))
    s.instances.append(("smoke_box", "Geo_Box", "smoke_transform", "smoke_boundary_material", "smoke_volume", True))
    # a sun shining in through the open front of the box: the light's +y axis
    # maps to the direction light travels, so rotate it to point back into the box
    s.transforms.append(("sun_transform", (0.0, 0.0, 0.0), (1.0, 1.0, 1.0), (-110.0, 15.0, 0.0)))
    s.distant_lights.append(("sun", "sun_transform", (1.0, 0.95, 0.85), 3.0, 5.0))
    return s


def spheres_scene(seed: int = 0) -> Scene:
    rng = np.random.Generator(np.random.PCG64(seed))
    s = cornell_scene(seed)
    keep = {"tall_box", "short_box"}
    s.instances = [i for i in s.instances if i[0] not in keep]
    s.cubes = ["Geo_UnitCube"]
    s.spheres = [("Geo_Sphere", 1.0), ("Geo_SmallSphere", 0.5)]
    s.transforms.append(("cube_transform", (-0.4, -0.6, -0.35), (0.55, 0.8, 0.55), (0.0, float(rng.uniform(10, 40)), 0.0)))
    s.materials.append(("DefaultMaterial", "cube_material", _lambert(rng.uniform(0.2, 0.9, 3))))
    s.instances.append(("cube", "Geo_UnitCube", "cube_transform", "cube_material", None, False))
    s.transforms.append(("glass_transform", (0.4, -0.62, 0.25), (0.38, 0.38, 0.38), (0, 0, 0)))
    s.materials.append(("DefaultMaterial", "glass_material", {
        "diffuse_albedo": [0.5, 0.5, 0.5], "specular_albedo": [1.0, 1.0, 1.0], "roughness_x": 0.031,
        "roughness_y": 0.035, "ior_n": 1.55, "metalness": 0.0, "specular_weight": 1.0, "transmission_weight": 1.0}))
    s.instances.append(("glass_sphere", "Geo_Sphere", "glass_transform", "glass_material", None, False))
    s.transforms.append(("metal_transform", (-0.45, 0.45, -0.5), (0.5, 0.5, 0.5), (0, 30, 0)))
    s.materials.append(("DefaultMaterial", "metal_material", {
        "diffuse_albedo": list(rng.uniform(0.5, 0.95, 3)), "specular_albedo": [1.0, 1.0, 1.0],
        "roughness_x": 0.2, "roughness_y": 0.2, "metalness": 1.0}))
    s.instances.append(("metal_sphere", "Geo_SmallSphere", "metal_transform", "metal_material", None, False))
    s.transforms.append(("bulb_transform", (0.55, 0.7, -0.45), (0.12, 0.12, 0.12), (0, 0, 0)))
    s.materials.append(("LightMaterial", "bulb_material", {"light_color": [1.0, 0.8, 0.6], "intensity": 20.0}))
    s.instances.append(("bulb", "Geo_Sphere", "bulb_transform", "bulb_material", None, False))
    s.transforms.append(("air_transform", (0.0, 0.0, 0.5), (3.5, 3.5, 3.5), (0, 0, 0)))
    s.volumes.append(("air_volume", "air_transform", (0.02, 0.02, 0.02), (0.9, 0.9, 0.9), 0.3, None))
    s.materials.append(("DefaultMaterial", "air_boundary_material", {"ior_n": 1.0}))
    s.instances.append(("air", "Geo_Sphere", "air_transform", "air_boundary_material", "air_volume", True))
    return s


def instanced_fog_scene(seed: int = 0) -> Scene:
    """The instanced scene inside a box of heterogeneous fog (sigma_t 0.15,
    albedo 0.8, g 0.3) whose density node (texture 0, a constant 1 in the
    file) takes a density grid at run time: the differentiable media workload."""
    s = instanced_scene(seed)
    s.meshes = s.meshes + [box_mesh("Geo_FogBox")]
    s.textures.append(("ConstantTextureFloat", "fog_density", {"value": 1.0}))
    s.transforms.append(("fog_transform", (0.0, 2.0, 0.0), (20.0, 6.0, 20.0), (0, 0, 0)))
    s.volumes.append(("fog_volume", "fog_transform", (0.15, 0.15, 0.15), (0.8, 0.8, 0.8), 0.3, "fog_density"))
    s.materials.append(("DefaultMaterial", "fog_boundary_material", {"ior_n": 1.0}))
    s.instances.append(("fog_box", "Geo_FogBox", "fog_transform", "fog_boundary_material", "fog_volume", True))
    return s


def smooth_grid(n: int, seed: int = 0, lo: float = 0.2, hi: float = 1.0) -> np.ndarray:
    """A seeded smooth density grid of n^3 values in [lo, hi]: a sum of a few
    random low-frequency sinusoids, rescaled."""
    rng = np.random.Generator(np.random.PCG64(seed))
    c = (np.arange(n) + 0.5) / n
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    v = np.zeros((n, n, n))
    for _ in range(6):
        k = rng.uniform(1.0, 4.0, 3) * 2 * np.pi
        v += rng.uniform(0.5, 1.0) * np.sin(k[0] * x + k[1] * y + k[2] * z + rng.uniform(0, 2 * np.pi))
    v = (v - v.min()) / max(v.max() - v.min(), 1e-12)
    return (lo + (hi - lo) * v).astype(np.float32)


def volumetric_const_scene(seed: int = 0) -> Scene:
    """The volumetric scene with the smoke's fBm density replaced by the
    constant 0.5 (same node name and index): a density grid of 0.5s attached
    to that node must render exactly as this constant."""
    s = volumetric_scene(seed)
    s.textures = [t if t[1] != "density_fbm" else ("ConstantTextureFloat", "density_fbm", {"value": 0.5})
                  for t in s.textures]
    return s


def glossy_scene(seed: int = 0) -> Scene:
    """The Cornell-like scene with a rough GGX conductor tall box and a
    rough plastic-like (diffuse + specular) short box: every differentiated
    material parameter (albedo, roughness) affects the image."""
    s = cornell_scene(seed)
    rng = np.random.Generator(np.random.PCG64(seed + 1000))
    mats = dict((name, i) for i, (_, name, _) in enumerate(s.materials))
    s.materials[mats["tall_box_material"]] = ("DefaultMaterial", "tall_box_material", {
        "diffuse_albedo": list(rng.uniform(0.5, 0.9, 3)), "specular_albedo": list(rng.uniform(0.6, 1.0, 3)),
        "roughness_x": 0.35, "roughness_y": 0.35, "metalness": 1.0})
    s.materials[mats["short_box_material"]] = ("DefaultMaterial", "short_box_material", {
        "diffuse_albedo": list(rng.uniform(0.2, 0.8, 3)), "specular_albedo": [1.0, 1.0, 1.0],
        "roughness_x": 0.3, "roughness_y": 0.3, "metalness": 0.0, "specular_weight": 1.0, "ior_n": 1.5,
        "transmission_weight": 0.0})
    return s


def _const(s, name, v):
    if np.ndim(v) == 0:
        s.textures.append(("ConstantTextureFloat", name, {"value": float(v)}))
    else:
        s.textures.append(("ConstantTextureRgb", name, {"color": tuple(float(x) for x in v)}))
    return name


def _solid(s, kind, name, black, white, **attrs):
    s.textures.append((kind, name, {"texture_black_idx": black, "texture_white_idx": white, **attrs}))
    return name


def textured_scene(seed: int = 0) -> Scene:
    """The Cornell-like room with every solid texture node of the format on
    material parameters: a checkerboard floor (albedo, metalness and a bump
    map, as the reference's own test scene has), a marble back wall with
    noise-driven roughness, wood and wave side walls, a turbulence box with a
    normal map from rgb noise, a polka-dot unit cube (texture coordinates of
    the built-in cube), a coated sphere whose coat weight, thickness, albedo
    and roughness are textured, a polka-dot sphere (spherical texture
    coordinates), a textured-transmission glass sphere, a quad with its own
    texture coordinates and a three-level node graph, and a medium sphere
    whose density is normalised noise."""
    rng = np.random.Generator(np.random.PCG64(seed + 77))
    s = cornell_scene(seed)
    s.meshes.append(uv_quad_mesh(repeat=3.0))
    s.cubes = ["Geo_UnitCube"]
    s.spheres = [("Geo_Sphere", 1.0)]
    mats = dict((name, i) for i, (_, name, _) in enumerate(s.materials))

    def set_mat(name, attrs):
        s.materials[mats[name]] = ("DefaultMaterial", name, attrs)

    # floor: checkerboard albedo, metalness and bump (CornellBox_Test's ground)
    _solid(s, "CheckerBoardTexture", "floor_albedo", _const(s, "floor_dark", (0.1, 0.12, 0.15)),
           _const(s, "floor_light", (0.8, 0.75, 0.6)), frequency=12.0)
    _solid(s, "CheckerBoardTexture", "floor_metal", _const(s, "floor_metal_0", 0.0), _const(s, "floor_metal_1", 1.0),
           frequency=12.0)
    _solid(s, "CheckerBoardTexture", "floor_bump", _const(s, "floor_bump_0", 0.15), _const(s, "floor_bump_1", 0.35),
           frequency=40.0)
    set_mat("floor_material", {"diffuse_albedo": [0.5, 0.5, 0.5], "specular_albedo": [1.0, 1.0, 1.0],
                               "roughness_x": 0.25, "roughness_y": 0.25, "ior_n": 1.65, "metalness": 0.0,
                               "specular_weight": 1.0, "transmission_weight": 0.0,
                               "diffuse_albedo_tex": "floor_albedo", "metalness_tex": "floor_metal",
                               "bump_mapping_tex": "floor_bump"})
    # back wall: marble albedo, noise roughness (x and y), specular albedo from fBm
    _solid(s, "NoiseTextureMarble", "back_marble", _const(s, "marble_vein", (0.25, 0.2, 0.2)),
           _const(s, "marble_base", (0.9, 0.88, 0.85)), frequency=2.5, gain=0.55, layer_count=5, variation=6.0,
           x_turb=True, y_turb=False, z_turb=True)
    _solid(s, "NoiseTexture", "back_rough", _const(s, "rough_lo", 0.1), _const(s, "rough_hi", 0.6), frequency=5.0,
           normalized=True)
    _solid(s, "NoiseTextureFBM", "back_spec", _const(s, "spec_lo", (0.6, 0.6, 0.6)), _const(s, "spec_hi", (1, 1, 1)),
           frequency=3.0, gain=0.5, layer_count=3, amplitude=0.5, offset=0.5)
    set_mat("back_material", {"diffuse_albedo": [0.5, 0.5, 0.5], "roughness_x": 0.3, "roughness_y": 0.3,
                              "ior_n": 1.5, "specular_weight": 1.0, "diffuse_albedo_tex": "back_marble",
                              "alpha_x_tex": "back_rough", "alpha_y_tex": "back_rough",
                              "specular_albedo_tex": "back_spec"})
    # side walls: wood and wave albedo
    _solid(s, "NoiseTextureWood", "left_wood", _const(s, "wood_dark", (0.35, 0.2, 0.1)),
           _const(s, "wood_light", (0.75, 0.55, 0.3)), frequency=1.5, variation=8.0)
    set_mat("left_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "left_wood"})
    # (the reference's parser accepts no wave parameters: attribute names with digits are illegal)
    _solid(s, "NoiseTextureWave", "right_wave", _const(s, "wave_a", (0.1, 0.3, 0.6)), _const(s, "wave_b", (0.9, 0.8, 0.3)))
    set_mat("right_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "right_wave"})
    # tall box: turbulence albedo and a normal map from rgb noise
    _solid(s, "NoiseTextureTurbulence", "box_turb", _const(s, "turb_a", (0.2, 0.5, 0.3)),
           _const(s, "turb_b", (0.9, 0.9, 0.7)), frequency=4.0, gain=0.5, layer_count=4, amplitude=1.0, offset=0.0)
    _solid(s, "NoiseTexture", "box_normal", _const(s, "nrm_a", (0.4, 0.45, 1.0)), _const(s, "nrm_b", (0.6, 0.55, 1.0)),
           frequency=9.0, normalized=True)
    set_mat("tall_box_material", {**_lambert((0.5, 0.5, 0.5)), "specular_weight": 0.5, "roughness_x": 0.4,
                                  "roughness_y": 0.4, "diffuse_albedo_tex": "box_turb",
                                  "normal_mapping_tex": "box_normal"})
    # short box: metalness and specular weight from a three-level graph (checker of marble and wood)
    _solid(s, "NoiseTextureMarble", "graph_marble", _const(s, "g_m0", 0.0), _const(s, "g_m1", 1.0), frequency=4.0)
    _solid(s, "NoiseTextureWood", "graph_wood", _const(s, "g_w0", 0.2), _const(s, "g_w1", 0.9), frequency=3.0,
           variation=4.0)
    _solid(s, "CheckerBoardTexture", "graph_checker", "graph_marble", "graph_wood", frequency=9.0)
    set_mat("short_box_material", {"diffuse_albedo": [0.7, 0.5, 0.3], "specular_albedo": [1.0, 0.9, 0.8],
                                   "roughness_x": 0.3, "roughness_y": 0.3, "metalness_tex": "graph_checker",
                                   "specular_weight_tex": "graph_checker"})
    # the built-in cube: polka dots over its texture coordinates
    _solid(s, "NoiseTexturePolkaDot", "cube_dots", _const(s, "dots_bg", (0.85, 0.85, 0.8)),
           _const(s, "dots_fg", (0.7, 0.1, 0.1)), frequency=4.0, radius=0.3)
    s.transforms.append(("cube_transform", (0.55, 0.1, -0.55), (0.3, 0.3, 0.3), (20.0, 30.0, 0.0)))
    s.materials.append(("DefaultMaterial", "cube_material", {**_lambert((0.5, 0.5, 0.5)),
                                                             "diffuse_albedo_tex": "cube_dots"}))
    s.instances.append(("cube", "Geo_UnitCube", "cube_transform", "cube_material", None, False))
    # a quad with its own texture coordinates (3x repeat): polka dots and checker coat on the ceiling side
    _solid(s, "NoiseTexturePolkaDot", "quad_dots", _const(s, "qd_bg", (0.2, 0.6, 0.3)), _const(s, "qd_fg", (0.9, 0.9, 0.2)),
           frequency=2.0, radius=0.2)
    s.transforms.append(("uvquad_transform", (-0.6, 0.3, -0.8), (0.6, 1.0, 0.6), (70.0, 25.0, 0.0)))
    s.materials.append(("DefaultMaterial", "uvquad_material", {**_lambert((0.5, 0.5, 0.5)),
                                                               "diffuse_albedo_tex": "quad_dots"}))
    s.instances.append(("uvquad", "Geo_UVQuad", "uvquad_transform", "uvquad_material", None, False))
    # coated sphere: coat weight, thickness, albedo and roughness textured
    _solid(s, "CheckerBoardTexture", "coat_w", _const(s, "coat_w0", 0.2), _const(s, "coat_w1", 1.0), frequency=10.0)
    _solid(s, "NoiseTexture", "coat_t", _const(s, "coat_t0", 0.5), _const(s, "coat_t1", 2.0), frequency=3.0)
    _solid(s, "NoiseTextureFBM", "coat_a", _const(s, "coat_a0", (0.9, 0.5, 0.3)), _const(s, "coat_a1", (0.4, 0.6, 0.9)),
           frequency=2.0, gain=0.5, layer_count=2)
    _solid(s, "NoiseTexture", "coat_r", _const(s, "coat_r0", 0.05), _const(s, "coat_r1", 0.4), frequency=6.0,
           normalized=False)
    s.transforms.append(("coated_transform", (-0.1, -0.75, 0.45), (0.25, 0.25, 0.25), (0.0, 40.0, 0.0)))
    s.materials.append(("DefaultMaterial", "coated_material", {
        "diffuse_albedo": list(rng.uniform(0.3, 0.8, 3)), "roughness_x": 0.5, "roughness_y": 0.5, "ior_n": 1.5,
        "specular_weight": 0.0, "coat_ior": 1.6, "coat_weight_tex": "coat_w", "coat_thickness_tex": "coat_t",
        "coat_albedo_tex": "coat_a", "coat_roughness_x_tex": "coat_r", "coat_roughness_y_tex": "coat_r"}))
    s.instances.append(("coated_sphere", "Geo_Sphere", "coated_transform", "coated_material", None, False))
    # polka-dot sphere (texture coordinates from the sphere's angles)
    _solid(s, "NoiseTexturePolkaDot", "sphere_dots", _const(s, "sd_bg", (0.9, 0.9, 0.9)), _const(s, "sd_fg", (0.1, 0.2, 0.7)),
           frequency=6.0, radius=0.25)
    s.transforms.append(("dots_transform", (0.45, 0.55, 0.3), (0.2, 0.2, 0.2), (30.0, 0.0, 0.0)))
    s.materials.append(("DefaultMaterial", "dots_material", {**_lambert((0.5, 0.5, 0.5)),
                                                             "diffuse_albedo_tex": "sphere_dots"}))
    s.instances.append(("dots_sphere", "Geo_Sphere", "dots_transform", "dots_material", None, False))
    # glass sphere with textured transmission weight
    _solid(s, "CheckerBoardTexture", "glass_tw", _const(s, "glass_tw0", 0.3), _const(s, "glass_tw1", 1.0), frequency=8.0)
    s.transforms.append(("glass_transform", (0.35, -0.8, 0.55), (0.18, 0.18, 0.18), (0, 0, 0)))
    s.materials.append(("DefaultMaterial", "glass_material", {
        "diffuse_albedo": [0.6, 0.6, 0.6], "specular_albedo": [1.0, 1.0, 1.0], "roughness_x": 0.05,
        "roughness_y": 0.05, "ior_n": 1.5, "metalness": 0.0, "specular_weight": 1.0,
        "transmission_weight_tex": "glass_tw"}))
    s.instances.append(("glass_sphere", "Geo_Sphere", "glass_transform", "glass_material", None, False))
    # a medium sphere with normalised-noise density
    _solid(s, "NoiseTexture", "haze_density", _const(s, "haze_0", 0.0), _const(s, "haze_1", 1.0), frequency=3.0)
    s.transforms.append(("haze_transform", (-0.45, 0.45, 0.2), (0.35, 0.35, 0.35), (0, 0, 0)))
    s.volumes.append(("haze_volume", "haze_transform", (2.0, 2.0, 2.0), (0.8, 0.8, 0.8), 0.2, "haze_density"))
    s.materials.append(("DefaultMaterial", "haze_boundary_material", {"ior_n": 1.0}))
    s.instances.append(("haze", "Geo_Sphere", "haze_transform", "haze_boundary_material", "haze_volume", True))
    return s


def imaged_scene(seed: int = 0) -> Scene:
    """The Cornell-like room with image textures (PNG files in the scene's
    texture folder): an 8-bit sRGB RGB back wall, a floor whose albedo is an
    interlaced 8-bit RGBA image and whose roughness and metalness come from a
    16-bit linear grey image, a 4-bit palette image with transparency on the
    left wall, a 2-bit grey bump map on the right wall, an 8-bit linear
    normal map on the tall box, a checkerboard of two images on the short
    box, an image over the built-in cube's and a sphere's texture
    coordinates, a quad with 3x-repeating texture coordinates, and an image
    whose file is missing (its material keeps its constant albedo, as in the
    reference)."""
    rng = np.random.Generator(np.random.PCG64(seed + 4242))
    s = cornell_scene(seed)
    s.meshes.append(uv_quad_mesh(repeat=3.0))
    s.cubes = ["Geo_UnitCube"]
    s.spheres = [("Geo_Sphere", 1.0)]
    mats = dict((name, i) for i, (_, name, _) in enumerate(s.materials))

    def set_mat(name, attrs):
        s.materials[mats[name]] = ("DefaultMaterial", name, attrs)

    def image(name, fname, samples, color_space="SRGB", **png):
        s.image_files[fname] = (samples, png)
        s.textures.append(("ImageTexture", name, {"texture_file_name": fname, "color_space": color_space}))
        return name

    def smooth(h, w, n, scale=255):
        y, x = np.mgrid[0:h, 0:w]
        base = [np.sin(x * (0.21 + 0.05 * k) + y * (0.13 - 0.03 * k) + k) for k in range(n)]
        img = (np.stack(base, -1) * 0.35 + 0.5 + rng.uniform(-0.15, 0.15, (h, w, n)))
        return np.clip(np.rint(img * scale), 0, scale).astype(np.uint16)

    image("back_img", "back_wall.png", smooth(48, 64, 3), depth=8, color_type=2, first_filter=0)
    set_mat("back_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "back_img"})
    image("floor_albedo_img", "floor_albedo.png", smooth(40, 40, 4), depth=8, color_type=6, interlace=True,
          first_filter=2)
    image("floor_gray16", "floor_rough.png", smooth(33, 27, 1, 65535), color_space="Linear", depth=16,
          color_type=0, first_filter=4)
    set_mat("floor_material", {"diffuse_albedo": [0.5, 0.5, 0.5], "specular_albedo": [1.0, 1.0, 1.0],
                               "roughness_x": 0.3, "roughness_y": 0.3, "ior_n": 1.5, "specular_weight": 1.0,
                               "diffuse_albedo_tex": "floor_albedo_img", "alpha_x_tex": "floor_gray16",
                               "alpha_y_tex": "floor_gray16", "metalness_tex": "floor_gray16"})
    pal = rng.integers(20, 235, (16, 3))
    idx = (np.add.outer(np.arange(30) // 3, np.arange(50) // 5) % 16).astype(np.uint16)
    image("left_img", "left_palette.png", idx, depth=4, color_type=3, palette=pal,
          trns=bytes(rng.integers(0, 256, 10).tolist()), first_filter=1)
    set_mat("left_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "left_img"})
    image("right_bump", "right_bump.png", (smooth(32, 32, 1, 3)).astype(np.uint16), depth=2, color_type=0,
          first_filter=3)
    set_mat("right_material", {**_lambert((0.6, 0.6, 0.6)), "bump_mapping_tex": "right_bump"})
    nrm = np.stack([smooth(24, 24, 1, 255)[..., 0] // 4 + 96, smooth(24, 24, 1, 255)[..., 0] // 4 + 96,
                    np.full((24, 24), 250)], -1).astype(np.uint16)
    image("box_normal", "box_normal.png", nrm, color_space="Linear", depth=8, color_type=2, first_filter=2)
    set_mat("tall_box_material", {**_lambert((0.7, 0.6, 0.5)), "normal_mapping_tex": "box_normal"})
    image("chk_a", "checker_a.png", smooth(16, 16, 3), depth=8, color_type=2)
    image("chk_b", "checker_b.png", smooth(8, 12, 1), depth=8, color_type=0, first_filter=1)
    _solid(s, "CheckerBoardTexture", "short_checker", "chk_a", "chk_b", frequency=10.0)
    set_mat("short_box_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "short_checker"})
    image("cube_img", "cube.png", smooth(20, 30, 3), depth=8, color_type=2, first_filter=3)
    s.transforms.append(("cube_transform", (0.55, 0.1, -0.55), (0.3, 0.3, 0.3), (20.0, 30.0, 0.0)))
    s.materials.append(("DefaultMaterial", "cube_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "cube_img"}))
    s.instances.append(("cube", "Geo_UnitCube", "cube_transform", "cube_material", None, False))
    s.transforms.append(("ball_transform", (-0.45, 0.5, 0.2), (0.25, 0.25, 0.25), (30.0, 0.0, 0.0)))
    s.materials.append(("DefaultMaterial", "ball_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "cube_img"}))
    s.instances.append(("ball", "Geo_Sphere", "ball_transform", "ball_material", None, False))
    image("quad_img", "quad.png", smooth(10, 14, 3), depth=8, color_type=2, interlace=True)
    s.transforms.append(("uvquad_transform", (-0.6, 0.3, -0.8), (0.6, 1.0, 0.6), (70.0, 25.0, 0.0)))
    s.materials.append(("DefaultMaterial", "uvquad_material", {**_lambert((0.5, 0.5, 0.5)), "diffuse_albedo_tex": "quad_img"}))
    s.instances.append(("uvquad", "Geo_UVQuad", "uvquad_transform", "uvquad_material", None, False))
    s.textures.append(("ImageTexture", "missing_img", {"texture_file_name": "missing.png", "color_space": "SRGB"}))
    set_mat("ceiling_material", {**_lambert((0.7, 0.7, 0.7)), "diffuse_albedo_tex": "missing_img"})
    return s


def orbit_view(name: str, seed: int, k: int, n: int):
    """The k-th of n cameras (from, look, fov) on a 90-degree arc around the
    scene's look-at point, at the original camera's height and distance and
    centred on it (for HostScene(..., camera=...))."""
    frm, look, fov = SCENES[name](seed).camera
    dx, dz = frm[0] - look[0], frm[2] - look[2]
    r = float(np.hypot(dx, dz))
    a0 = float(np.arctan2(dx, dz))
    a = a0 + (k / max(n - 1, 1) - 0.5) * (np.pi / 2)
    return (float(look[0] + r * np.sin(a)), float(frm[1]), float(look[2] + r * np.cos(a))), tuple(look), fov


SCENES = {
    "cornell": cornell_scene,
    "glossy": glossy_scene,
    "instanced": instanced_scene,
    "instanced_fog": instanced_fog_scene,
    "spheres": spheres_scene,
    "textured": textured_scene,
    "imaged": imaged_scene,
    "volumetric": volumetric_scene,
    "volumetric_const": volumetric_const_scene,
}


def fbm_grid(scene, texture_index: int, n: int = 128) -> np.ndarray:
    """An n^3 lattice (cell centres of the object-space box [-0.5, 0.5]^3)
    of texture node `texture_index` of an uploaded scene (ymrt_b200.Scene),
    evaluated on the device and scaled so that its maximum is 1: the density
    grid of the media workload, whose volume's sigma_t is then the maximum
    extinction."""
    c = (np.arange(n, dtype=np.float32) + np.float32(0.5)) / np.float32(n) - np.float32(0.5)
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    pts = np.stack([x, y, z], axis=-1).reshape(-1, 3)
    v = scene.density(texture_index, pts).reshape(n, n, n)
    v = np.maximum(v, 0.0)
    return (v / max(float(v.max()), 1e-12)).astype(np.float32)


def scene_path(name: str, seed: int = 0, cache_dir: str | None = None) -> str:
    """Writes (once) and returns the path of a generated scene file."""
    cache_dir = cache_dir or os.environ.get("YMRT_SCENE_CACHE", os.path.join(os.path.dirname(__file__), "_scenes"))
    path = os.path.join(cache_dir, f"{name}_{seed}.ymtmp")
    if not os.path.exists(path):
        write_scene(SCENES[name](seed), path)
    return path
