"""The reference's stage interface (libymrt_compat.so) driven the way the
reference editor drives it.

tests/compat_driver.cpp declares the reference-named launchers with the
reference's argument kinds and runs the editor's wave-loop protocol (tile
batches of MAX_RAY_COUNT rays, counters copied between host and device)
for several frames with accumulation; it also renders the same frames
through the C ABI directly. The two accumulated images must agree within
the per-sample tolerance (the renders differ only in the order of
per-pixel float additions). The driver also runs the editor view through
the three editor-view launchers with the editor's own loop and both
post-processing launchers, against the direct C-ABI calls.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    import ymrt_b200 as Y
    Y.library()  # built
    lib_dir = os.path.join(ROOT, "ymrt_b200")
    if not os.path.exists(os.path.join(lib_dir, "libymrt_compat.so")):
        pytest.fail("libymrt_compat.so is missing: build with python -m ymrt_b200.build")
    if shutil.which("g++") is None:
        pytest.skip("no host compiler")
    out = str(tmp_path_factory.mktemp("compat") / "compat_driver")
    cmd = ["g++", "-O2", "-std=c++17", os.path.join(ROOT, "tests", "compat_driver.cpp"),
           "-I" + os.path.join(ROOT, "include"), "-I/usr/local/cuda/include", "-L" + lib_dir,
           "-l:libymrt_compat.so", "-l:libymrt.so", "-L/usr/local/cuda/lib64", "-lcudart",
           "-Wl,-rpath," + lib_dir + ":/usr/local/cuda/lib64", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    return out


@pytest.mark.parametrize("max_frames", [0, 2])
def test_reference_stage_protocol_matches_direct_render(driver, cornell_path, halton_perm, tmp_path, max_frames):
    w = h = 512  # 1024 tiles at 16 spp: four generation batches of 2^20 rays per frame
    frames = 3
    perm_file = tmp_path / "perm.u32"
    np.ascontiguousarray(halton_perm, np.uint32).tofile(perm_file)
    a_file, b_file = tmp_path / "compat.f32", tmp_path / "direct.f32"
    ea_file, eb_file = tmp_path / "editor_compat.bin", tmp_path / "editor_direct.bin"
    r = subprocess.run([driver, cornell_path, str(perm_file), str(w), str(h), "16", str(frames), str(max_frames),
                        str(a_file), str(b_file), str(ea_file), str(eb_file)], capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    assert "generation_calls %d" % (4 * frames) in r.stdout, r.stdout
    a = np.fromfile(a_file, np.float32).reshape(h, w, 4)
    b = np.fromfile(b_file, np.float32).reshape(h, w, 4)
    assert a[..., :3].mean() > 0.01
    assert np.allclose(a, b, rtol=1e-5, atol=1e-6), np.abs(a - b).max()
    # the editor view and post-processing through the reference-named launchers equal the direct calls
    n = w * h
    ea, eb = np.fromfile(ea_file, np.uint8), np.fromfile(eb_file, np.uint8)
    assert ea.size == eb.size == n * (16 + 4 + 16 + 16)
    assert np.array_equal(ea[:n * 20], eb[:n * 20])  # beauty and primitive index, bit for bit
    assert (ea[n * 16:n * 20].view(np.uint32) != 0xFFFFFFFF).mean() > 0.5
    assert np.array_equal(ea[n * 20:n * 36], eb[n * 20:n * 36])  # editor post-processing with the outline
    pa, pb = ea[n * 36:].view(np.float32), eb[n * 36:].view(np.float32)
    assert np.allclose(pa, pb, rtol=1e-5, atol=1e-6)  # path-traced image after tone mapping
