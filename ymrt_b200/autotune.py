"""Autotuner for the renderer's wave loop and scene build.

Picks, by measuring on the GPU, the configuration that renders a workload
fastest: path-queue capacity (paths in flight per wave), material-sorted
shading on/off, continuing rays grouped by origin and direction on/off,
deferred shadow rays on/off, the block shape of the
closest-hit and shadow-ray kernels (threads per block), the CUDA-graph wave
loop on/off and the wide-BVH leaf size. The search is exhaustive over a
small space (the defaults below: 3 x 2 x 2 x 2 x 3 x 3 = 216 points, two
wave-loop kinds only when asked), each point timed on a sample of the
workload (a band of tiles from
the middle of the frame, large enough to fill several waves) after one
warm-up render; results are cached in a JSON file keyed by the workload.

The renderer's results do not depend on these choices beyond the order of
per-pixel float additions, so tuning changes speed only.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os
import time
from typing import Callable, Dict, Iterable, List, Optional

DEFAULT_SPACE: Dict[str, List[int]] = {
    "queue_capacity": [1 << 20, 1 << 21, 1 << 22],
    "sort_hits": [0, 1],
    "sort_rays": [0, 1],
    "defer_shadows": [0, 1],
    "trace_block": [64, 128, 256],
    "max_leaf_triangles": [2, 3, 4],
}

WAVE_OPTIONS = ("sort_hits", "sort_rays", "defer_shadows", "graph_loop", "trace_block")


def points(space: Dict[str, Iterable[int]]) -> List[Dict[str, int]]:
    """Every combination of the space's values, in a fixed order."""
    keys = sorted(space)
    return [dict(zip(keys, combo)) for combo in itertools.product(*(list(space[k]) for k in keys))]


def search(space: Dict[str, Iterable[int]], measure: Callable[[Dict[str, int]], float],
           repeats: int = 2) -> Dict[str, object]:
    """Times every point with `measure` (milliseconds; the best of `repeats`
    calls after one warm-up call) and returns the fastest point, its time and
    the whole table. Points whose measurement raises are recorded as failed
    and never chosen."""
    table = []
    best, best_ms = None, float("inf")
    for p in points(space):
        try:
            measure(p)  # warm-up: first-use allocations, graph capture
            ms = min(measure(p) for _ in range(max(1, repeats)))
        except Exception as e:  # noqa: BLE001 - a configuration the device rejects
            table.append({"config": p, "ms": None, "error": f"{type(e).__name__}: {e}"})
            continue
        table.append({"config": p, "ms": ms})
        if ms < best_ms:
            best, best_ms = p, ms
    if best is None:
        raise RuntimeError("autotune: no configuration could be measured")
    return {"best": best, "ms": best_ms, "table": table}


def apply(ctx, config: Dict[str, int]) -> None:
    """Sets a tuned configuration's context-level choices on `ctx` (the leaf
    size is a scene-build option: pass config['max_leaf_triangles'] to
    HostScene)."""
    from . import library
    if "queue_capacity" in config:
        library().ymrt_set_queue_capacity(ctx.h, int(config["queue_capacity"]))
    for k in WAVE_OPTIONS:
        if k in config:
            ctx.set_option(k, config[k])


def sample_tiles(width: int, height: int, spp: int, capacity: int, waves: int = 4):
    """A band of tiles from the middle of the frame holding about `waves`
    full waves of paths (the whole frame when it is smaller)."""
    tiles_x, tiles_y = (width + 15) // 16, (height + 15) // 16
    total = tiles_x * tiles_y
    want = max(1, (capacity * waves + 256 * spp - 1) // (256 * spp))
    if want >= total:
        return 0, 0
    begin = max(0, (total - want) // 2)
    return begin, begin + want


def _cache_key(path: str, width: int, height: int, setting, space) -> str:
    h = hashlib.sha256()
    with open(path, "rb") as f:
        h.update(f.read())
    fields = [width, height, setting.ssp, setting.ray_depth, setting.sampler_type, setting.enable_shape_light,
              setting.enable_distant_light, setting.enable_volume_scattering, setting.enable_env_light,
              setting.enable_russian_roulette, setting.enable_indirect_clamp]
    h.update(json.dumps([fields, {k: list(v) for k, v in sorted(space.items())}]).encode())
    return h.hexdigest()


def tune_scene(path: str, width: int, height: int, setting, halton_perm, device: int = 0,
               space: Optional[Dict[str, Iterable[int]]] = None, repeats: int = 2,
               cache_file: Optional[str] = None) -> Dict[str, object]:
    """Tunes the rendering of one .ymtmp scene at one resolution and setting.
    Returns {"best": config, "ms": sample time, "table": [...], "sample_tiles": (b, e)}."""
    import torch

    from . import Context, HostScene, Scene

    space = dict(space or DEFAULT_SPACE)
    key = _cache_key(path, width, height, setting, space)
    if cache_file and os.path.exists(cache_file):
        with open(cache_file) as f:
            cached = json.load(f)
        if key in cached:
            return cached[key]
    leaf_sizes = list(space.pop("max_leaf_triangles", [3]))
    ctx = Context(device)
    out = torch.zeros((height, width, 4), dtype=torch.float32, device=f"cuda:{device}")
    capacity = max(space.get("queue_capacity", [1 << 21]))
    tb, te = sample_tiles(width, height, max(setting.ssp, 1), capacity)
    scenes = {}

    def scene_for(leaf: int):
        if leaf not in scenes:
            scenes[leaf] = Scene(ctx, HostScene(path, width, height, max_leaf_triangles=leaf), halton_perm)
        return scenes[leaf]

    def measure(p: Dict[str, int]) -> float:
        apply(ctx, p)
        scene = scene_for(p["max_leaf_triangles"])
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        _, st = scene.render(setting, 1, out=out, tile_begin=tb, tile_end=te)
        wall = (time.perf_counter() - t0) * 1e3
        return st.ms_total if st.ms_total > 0 else wall

    try:
        space["max_leaf_triangles"] = leaf_sizes
        result = search(space, measure, repeats)
    finally:
        for sc in scenes.values():
            sc.close()
        ctx.close()
    result["sample_tiles"] = [tb, te]
    if cache_file:
        cached = {}
        if os.path.exists(cache_file):
            with open(cache_file) as f:
                cached = json.load(f)
        cached[key] = result
        tmp = cache_file + ".tmp"
        with open(tmp, "w") as f:
            json.dump(cached, f, indent=1)
        os.replace(tmp, cache_file)
    return result


def tune_batch(ctx, renders, space: Optional[Dict[str, Iterable[int]]] = None, repeats: int = 2) -> Dict[str, object]:
    """Tunes the context-level choices (queue capacity, sorting, deferral,
    block shape, graph loop) for a batch of renders as ymrt_b200.render_batch takes them;
    leaves the best configuration applied to `ctx`."""
    from . import render_batch

    space = dict(space or {k: v for k, v in DEFAULT_SPACE.items() if k != "max_leaf_triangles"})
    space.pop("max_leaf_triangles", None)

    def measure(p: Dict[str, int]) -> float:
        apply(ctx, p)
        return render_batch(ctx, renders).ms_total

    result = search(space, measure, repeats)
    apply(ctx, result["best"])
    return result
