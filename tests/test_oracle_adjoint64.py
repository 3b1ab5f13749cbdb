"""The double-precision host adjoint of material albedo (oracle/adjoint64.py)
pinned on the CPU: the FP64 oracle's recorded radiance terms sum to its
image, and the adjoint over them equals central differences of the same
FP64 render (eps 1e-3; the render is a polynomial in the albedos, so the
difference is exact up to its second-order term and double rounding)."""
import numpy as np
import pytest

from ymrt_b200 import scenes

SIZE, SPP = 64, 16


@pytest.fixture(scope="module")
def ref64(volumetric_path, halton_perm):
    from oracle import ref
    if not ref.available64():
        pytest.skip("FP64 oracle not built")
    r = ref.RefScene(volumetric_path, halton_perm, SIZE, SIZE, fp64=True)
    r.set_settings(spp=SPP, ray_depth=8, distant_light=1, volume=1)
    yield r
    r.close()


def test_recorded_terms_sum_to_the_image(ref64):
    ev, img = ref64.record_events(1)
    terms = ev["kind"] > 0
    acc = np.zeros((SIZE * SIZE, 3))
    np.add.at(acc, ev["pixel"][terms], ev["value"][terms])
    np.testing.assert_allclose(acc / SPP, img.reshape(-1, 4)[:, :3], rtol=0, atol=1e-12)
    # every kind the volumetric scene produces: scattering, surface and volume NEE, the light seen directly
    assert set(np.unique(ev["kind"])) >= {0, 1, 2, 4}


def test_host_adjoint_equals_fp64_central_differences(ref64):
    from oracle import adjoint64
    params, lam = ref64.material_params()
    lambertian = np.flatnonzero(lam)
    assert len(lambertian) == 7  # five walls, two boxes
    w = np.random.default_rng(21).uniform(0.0, 1.0, (SIZE, SIZE, 4))
    ev, _ = ref64.record_events(1)
    g = adjoint64.albedo_adjoint(ev, w, params, lambertian, SPP)
    assert np.all(g[~lam] == 0)
    eps = 1e-3
    rng = np.random.default_rng(8)
    for _ in range(4):
        m, k = int(rng.choice(lambertian)), int(rng.integers(0, 3))
        ls = []
        for sgn in (+1, -1):
            p = params.astype(np.float64).copy()
            p[m, k] += sgn * eps
            ref64.set_material_params(p)
            ls.append(float((ref64.render_frame(1)[..., :3] * w[..., :3]).sum()))
        ref64.set_material_params(params)
        fd = (ls[0] - ls[1]) / (2 * eps)
        assert abs(g[m, k] - fd) <= 1e-6 * abs(fd), (m, k, g[m, k], fd)
