"""The per-sample divergence classifier (tests/divergence.py) on made-up
vertex records: each class is named for the first field that differs."""
import numpy as np

import divergence as D
from oracle.ref import VERTEX_DTYPE


def _path(pixel, n):
    v = np.zeros(n, VERTEX_DTYPE)
    v["pixel"] = pixel
    v["depth"] = np.arange(1, n + 1)
    v["flags"] = 1
    v["inst"], v["tri"] = 3, 7
    v["t"] = 1.5
    v["o"] = [0.25, 0.5, 0.75]
    v["d"] = [0.0, 0.6, 0.8]
    v["bary"] = [0.2, 0.3, 0.5]
    v["tp"] = [0.5, 0.5, 0.5]
    v["light"] = [0.1, 0.2, 0.3]
    return v


def _classify(mutate, n=4, k=2):
    a, b = _path(9, n), _path(9, n)
    mutate(b[k])
    img = np.zeros((1, 16, 4), np.float32)
    counts, detail = D.classify([9], a, b, img, img)
    return detail[0][1], detail[0][2], detail[0][3]


def test_classes():
    def tie(v):
        v["tri"] = 8
    def last_bit(v):
        v["d"][1] = np.nextafter(np.float32(0.6), np.float32(1.0))
    def large(v):
        v["d"] = [0.8, 0.6, 0.0]
    def t(v):
        v["t"] = np.float32(1.5) + np.float32(1e-3)
    def miss(v):
        v["flags"] = 0
    def tp(v):
        v["tp"][0] = np.float32(0.5) * np.float32(1.000001)
    assert _classify(tie) == ("tie", 3, "primitive")
    assert _classify(last_bit) == ("last_bit", 3, "d")
    assert _classify(large) == ("other", 3, "d")
    assert _classify(t) == ("traversal", 3, "t")
    assert _classify(tp) == ("last_bit", 3, "tp")
    # a miss is dropped from the compared vertices: the paths differ in length
    assert _classify(miss)[0] == "other"


def test_equal_paths_fall_back_to_the_pixel():
    a, b = _path(5, 3), _path(5, 3)
    ia = np.zeros((1, 8, 4), np.float32)
    ib = ia.copy()
    ia[0, 5, 0], ib[0, 5, 0] = 1.0, np.float32(1.0) + np.float32(1e-6)
    counts, detail = D.classify([5], a, b, ia, ib)
    assert detail[0][1] == "final_last_bit"
    ib[0, 5, 0] = 2.0
    counts, detail = D.classify([5], a, b, ia, ib)
    assert detail[0][1] == "final_other"


def test_observed_bounds_have_a_margin():
    assert all(D.bound(k) >= v + 8 for k, v in D.OBSERVED.items())
