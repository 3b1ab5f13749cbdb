"""Double-precision host adjoint of material albedo, over the oracle's
recorded radiance events.

TEST INFRASTRUCTURE ONLY (the checker of ymrt_render_backward's albedo
gradients; nothing in ymrt_b200 imports it).

The reference has no backward pass; this is this project's derivative of the
reference's own estimator, taken over the events its FP64 build records
(oracle/build_ref.py `_EVENT_HOST`). For a Lambertian material (a default
material whose only lobe is the diffuse one, src/BSDF.cuh:185-213), the
albedo enters a path only as a factor: each scattering at such a vertex
multiplies the throughput by its BSDF weight f cos / pdf = albedo
(DefaultMtlBSDF::SampleWi with one lobe, src/BSDF.cuh:633-679), and
next-event estimation at such a vertex evaluates f = albedo / pi
(src/BSDF.cuh:619-632); lobe selection and every pdf are independent of the
albedo. So every radiance term is a monomial in the albedos of the
Lambertian vertices before it (and, for next-event estimation at a surface,
of the vertex itself), and its derivative with respect to channel c of
albedo m is the term times n_m / albedo_m[c], n_m the number of those
factors that are material m. The adjoint of a loss sum(w * image) is then

    dL/dalbedo_m[c] = sum over terms  w[pixel, c] * term[c] * n_m / albedo_m[c] / spp

accumulated in double, with the same samples as the forward render.
"""
from __future__ import annotations

import numpy as np


def albedo_adjoint(events: np.ndarray, weights: np.ndarray, albedo: np.ndarray, lambertian, spp: int) -> np.ndarray:
    """dLoss/dAlbedo for the Lambertian materials (rows of `albedo` listed in
    `lambertian`; other rows are zero).

    events: the FP64 oracle's record_events output (oracle.ref.EVENT_DTYPE)
    for one frame; weights: (H*W, 3) or (H, W, >=3) dLoss/dImage; albedo:
    (M, >=3) the materials' albedos; spp: samples per pixel of the frame."""
    w = np.asarray(weights, np.float64)
    w = w.reshape(-1, w.shape[-1])[:, :3]
    alb = np.asarray(albedo, np.float64)[:, :3]
    n_mat = alb.shape[0]
    lam = np.zeros(n_mat, bool)
    lam[list(lambertian)] = True
    grad = np.zeros((n_mat, 3), np.float64)
    if len(events) == 0:
        return grad
    ev = np.asarray(events)
    # order each path's events by depth, its scattering event after the terms
    # added at the same vertex (the scattering raises the next vertex's depth)
    path = ev["pixel"].astype(np.int64) * (int(ev["sample"].max()) + 1) + ev["sample"].astype(np.int64)
    scatter = ev["kind"] == 0
    order = np.lexsort((scatter, ev["depth"], path))
    ev, path, scatter = ev[order], path[order], scatter[order]
    # factors before each event: running counts of scattering events per
    # material within the path, excluding the event itself
    mats = np.where(ev["material"] >= 0, ev["material"], n_mat)
    onehot = np.zeros((len(ev), n_mat + 1), np.int32)
    onehot[np.arange(len(ev)), mats] = scatter
    before = np.cumsum(onehot, axis=0) - onehot
    starts = np.flatnonzero(np.r_[True, path[1:] != path[:-1]])
    first = np.repeat(starts, np.diff(np.r_[starts, len(ev)]))
    counts = (before - before[first])[:, :n_mat].astype(np.float64)
    # next-event estimation at a surface vertex: its own albedo as well
    own = (ev["kind"] == 1) & (ev["material"] >= 0)
    counts[np.flatnonzero(own), ev["material"][own]] += 1.0
    terms = ~scatter
    contrib = w[ev["pixel"][terms]] * ev["value"][terms]  # (n_terms, 3)
    for m in np.flatnonzero(lam):
        grad[m] = (counts[terms, m][:, None] * contrib).sum(axis=0) / alb[m] / spp
    return grad
