"""The FP64 oracle: the reference's algorithm with every float computed in
double (oracle/build_ref.py build_fp64), the yardstick for converged-image
error at equal spp.

Pinned against the float oracle on the Cornell-like scene: the same samples
drive both, so per pixel they differ by rounding only, except on the few
paths where rounding flips a branch.
"""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def ref64(oracle):
    if not oracle.available64():
        try:
            from oracle import build_ref
            build_ref.build_fp64()
        except Exception as e:  # reference sources absent and no prebuilt library
            pytest.skip(f"FP64 oracle unavailable: {e}")
    return oracle


def test_fp64_oracle_matches_float_oracle(ref64, cornell_path, halton_perm):
    a = ref64.RefScene(cornell_path, halton_perm, 96, 96)
    b = ref64.RefScene(cornell_path, halton_perm, 96, 96, fp64=True)
    for s in (a, b):
        s.set_settings(spp=4, ray_depth=8)
    fa, fb = a.render_frame(1), b.render_frame(1)
    a.close()
    b.close()
    assert fa.dtype == np.float32 and fb.dtype == np.float64
    assert np.array_equal(fa[..., 3].astype(np.float64), fb[..., 3])  # same paths per pixel
    d = fa[..., :3].astype(np.float64) - fb[..., :3]
    rmse = float(np.sqrt(np.mean(d ** 2)))
    assert rmse <= 1e-5, rmse
    rel = np.abs(d) / np.maximum(np.abs(fb[..., :3]), 1e-6)
    assert np.mean(np.any(rel > 1e-3, axis=-1)) <= 1e-3
    # the double build really computes in double: some pixels differ in low bits
    assert np.any(d != 0.0)
