"""Builds ``ymrt_b200/libymrt.so`` in-tree for sm_100a.

Kernels and the C ABI are compiled by nvcc for ``sm_100a`` only; the host-side
scene preparation by g++. Floating point: ``-fmad=false``, IEEE division and
square root, no flush-to-zero on the device, ``-ffp-contract=off`` on the
host, so that every expression the path tracer shares with the reference is
rounded exactly as written (explicit ``fmaf`` is used where that does not
matter, e.g. BVH box tests).

Usage: ``python -m ymrt_b200.build [--force] [--verbose]``.
"""
from __future__ import annotations

import argparse
import hashlib
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libymrt.so")
# The reference's stage-launcher symbols, forwarding to libymrt.so (include/ymrt_compat.h).
COMPAT_LIB = os.path.join(HERE, "libymrt_compat.so")
COMPAT_SOURCE = "compat_shim.cpp"
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

NVCC_FLAGS = ARCH + [
    "-O3", "-lineinfo", "-std=c++17", "-fmad=false", "-prec-div=true", "-prec-sqrt=true", "-ftz=false",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-ffp-contract=off", "-I" + os.path.join(ROOT, "include"),
]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-ffp-contract=off", "-fno-fast-math", "-I/usr/local/cuda/include",
             "-I" + os.path.join(ROOT, "include")]

CU_SOURCES = ["kernels.cu", "wave_media.cu", "wave_adjoint.cu", "tlas_build.cu", "capi.cu"]
CXX_SOURCES = ["scene_host.cpp", "png_decode.cpp", "png_encode.cpp", "image_decode.cpp"]


def _stamp() -> str:
    h = hashlib.sha256()
    h.update(" ".join(NVCC_FLAGS + CXX_FLAGS).encode())
    for d in (CSRC, os.path.join(ROOT, "include")):
        for name in sorted(os.listdir(d)):
            p = os.path.join(d, name)
            if os.path.isfile(p):
                with open(p, "rb") as f:
                    h.update(name.encode())
                    h.update(f.read())
    return h.hexdigest()


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"command failed: {' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return r.stdout + r.stderr


def build(force: bool = False, verbose: bool = False, ptxas_report: bool = False) -> str:
    os.makedirs(OUT_DIR, exist_ok=True)
    stamp_file = os.path.join(OUT_DIR, "stamp")
    stamp = _stamp()
    if not force and os.path.exists(LIB) and os.path.exists(COMPAT_LIB) and os.path.exists(stamp_file):
        with open(stamp_file) as f:
            if f.read().strip() == stamp:
                return LIB
    objs, procs = [], []
    for src in CU_SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        extra = ["-Xptxas", "-v"] if ptxas_report else []
        cmd = [NVCC] + NVCC_FLAGS + extra + ["-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    for src in CXX_SOURCES:
        obj = os.path.join(OUT_DIR, src + ".o")
        cmd = ["g++"] + CXX_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
        procs.append((cmd, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)))
        objs.append(obj)
    reports = []
    for cmd, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            raise RuntimeError(f"build failed: {' '.join(cmd)}\n{out}")
        if verbose or ptxas_report:
            reports.append(out)
    tmp = LIB + ".tmp"
    # Export only the C ABI and bind internal references locally, so the
    # statically linked CUDA runtime never collides with another copy loaded
    # by the host process (torch, the oracle).
    vs = os.path.join(OUT_DIR, "exports.map")
    with open(vs, "w") as f:
        f.write("{ global: ymrt_*; local: *; };\n")
    _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", tmp] + objs +
         ["-lz", "-Xlinker", "-Bsymbolic", "-Xlinker", "--version-script=" + vs], verbose)
    os.replace(tmp, LIB)
    # libymrt_compat.so: host code only, linked against libymrt.so (found
    # beside it at run time), so that one CUDA runtime does all device work.
    cobj = os.path.join(OUT_DIR, COMPAT_SOURCE + ".o")
    _run(["g++"] + CXX_FLAGS + ["-c", os.path.join(CSRC, COMPAT_SOURCE), "-o", cobj], verbose)
    ctmp = COMPAT_LIB + ".tmp"
    _run(["g++", "-shared", "-o", ctmp, cobj, "-L" + HERE, "-l:libymrt.so", "-Wl,-rpath,$ORIGIN",
          "-Wl,--no-undefined"], verbose)
    os.replace(ctmp, COMPAT_LIB)
    with open(stamp_file, "w") as f:
        f.write(stamp)
    if reports:
        print("\n".join(reports))
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas", action="store_true", help="print the ptxas register/spill report")
    a = ap.parse_args(argv)
    print(build(a.force, a.verbose, a.ptxas))


if __name__ == "__main__":
    sys.exit(main())
