"""The boundary's threading contract (one context per host thread): renders
from two contexts on one device, run at the same time from two threads,
equal the same renders made one after the other. Scenes live in
constant-memory slots shared by every context on the device; each call
leases the slots it uses (the reference runs its editor view and path
tracer concurrently on two streams, src/core/RenderModule.cpp:93-143)."""
import threading

import numpy as np
import pytest

import ymrt_b200 as Y

pytestmark = pytest.mark.gpu


def test_two_contexts_render_concurrently(cornell_path, volumetric_path, halton_perm):
    jobs = [(cornell_path, 256, 256, Y.default_setting(spp=1, ray_depth=8)),
            (volumetric_path, 320, 240, Y.default_setting(spp=1, ray_depth=8, volume=True, distant_light=True))]
    ctxs = [Y.Context(0), Y.Context(0)]
    scs = [Y.Scene(c, Y.HostScene(p, w, h), halton_perm) for c, (p, w, h, _) in zip(ctxs, jobs)]
    frames = range(1, 9)
    # one path per pixel: a pixel's value depends on the order of its few
    # atomic additions (the path and its deferred shadow rays) only in the
    # last bits
    want = [[sc.render(s, f)[0] for f in frames] for sc, (_, _, _, s) in zip(scs, jobs)]
    got = [[None] * len(frames) for _ in jobs]
    errors = []
    start = threading.Barrier(2)

    def worker(k):
        try:
            start.wait()
            for i, f in enumerate(frames):
                got[k][i] = scs[k].render(jobs[k][3], f)[0]
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    assert not errors, errors
    for k in range(2):
        for i in range(len(frames)):
            np.testing.assert_allclose(got[k][i], want[k][i], rtol=1e-5, atol=1e-7, err_msg=f"job {k} frame {i}")
    for sc in scs:
        sc.close()
    for c in ctxs:
        c.close()
