"""Benchmark: Mrays/s of the ymrt_b200 path tracer on one B200 (or N replicas).

Workload (the reference's headline configuration that fits one GPU): the
seeded instanced scene of ~1.2 M triangles (64 instances of an icosphere, a
fBm heightfield, a torus and a box; 32 GGX conductor / dielectric / diffuse
materials; 2 quad lights), 1920x1080, 64 samples per pixel, maximum depth 12,
Halton sampler, shape-light next-event estimation. One step = one full frame.

Metric: Mrays/s = (closest-hit queries + occlusion queries) / time; the
reference performs the same queries on the same paths.

Arms:
  (default)          ymrt_b200 kernels. `value`: K frames with the scene
                     resident, timed with CUDA events between a barrier and a
                     synchronize on each side (max over ranks). `e2e`: through
                     the C ABI with the scene uploaded from host memory and the
                     image read back every step. `kernels` / `roofline`: one
                     profiled frame with events around every launch.
                     `ref_cuda`: the reference's own stage kernels rebuilt for
                     sm_100a on the same frame. `cpu_baseline`: the reference
                     built for the host on a bounded tile sample.
                     `rmse_vs_fp64`: the profiled frame against the FP64
                     oracle on a band of tiles, beside the reference's own
                     float error there.
  --impl reference   the reference's own path tracer compiled for the host
                     (oracle/_ref), all host threads, on a bounded tile
                     sample of the same frame.

Multi-GPU (torchrun, one rank per GPU): every rank renders its own frame of
the progressive sequence (frame index = step * N + rank + 1, so the ranks
draw disjoint Halton samples) and the frames are summed with one NCCL
all-reduce per step (weak scaling: the per-GPU work is fixed).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    "instanced": dict(scene="instanced", width=1920, height=1080, spp=64, depth=12),
    "cornell": dict(scene="cornell", width=256, height=256, spp=16, depth=8),
    # the Cornell-like scene with a homogeneous fog box and a procedural fBm
    # smoke box (the density-texture form the reference renders), delta tracking
    "volumetric": dict(scene="volumetric", width=1280, height=720, spp=32, depth=16, volume=True),
    # the same scene with the smoke's density as a 128^3 float16 grid sampled
    # from its fBm node (maximum sigma_t 2.0); the reference has no grid node,
    # so its arms render the procedural form of the same medium
    "volumetric_grid": dict(scene="volumetric", width=1280, height=720, spp=32, depth=16, volume=True, grid=128),
    # the Cornell-like scene with every solid texture node on material
    # parameters, a checkerboard bump map, an rgb-noise normal map and a
    # noise-density medium (the texture graph the reference evaluates per hit)
    "textured": dict(scene="textured", width=1280, height=720, spp=32, depth=12, volume=True),
}


class quiet_stdout:
    """Sends file descriptor 1 to /dev/null while the reference's own code
    runs (its scene loader reports progress on stdout), so that stdout
    carries only the one JSON line."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        devnull = os.open(os.devnull, os.O_WRONLY)
        os.dup2(devnull, 1)
        os.close(devnull)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)


def workload_config(wl, W, H, spp, world) -> dict:
    """The `config` both arms print (identical, so that their lines compare)."""
    return {"workload": f"{wl['scene']} {W}x{H} {spp}spp depth {wl['depth']}" +
                        (" (~1.2M instanced triangles)" if wl["scene"] == "instanced" else ""),
            "sampler": "halton", "lights": "shape lights, NEE with MIS",
            "media": (("fog box + smoke box with a 128^3 fp16 density grid (fBm, 4 octaves, max "
                       "sigma_t 2.0), delta tracking") if wl.get("grid") else
                      ("noise-density medium sphere, delta tracking" if wl["scene"] == "textured" else
                       "fog box + fBm smoke box, delta tracking")) if wl.get("volume") else "none",
            "parallelism": f"replica x{world}" + (" + allreduce of frames" if world > 1 else ""),
            "l2": "256 MB buffer written between steps; path queues (>1 GB) exceed L2"}


def dist_env():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def read_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for n, v in zip(names, parts[5:9]):
                    if v.lower() == "active":
                        reasons.add(n)
        os.unlink(self.path)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(torch_mod, buf):
    buf.add_(1.0)  # writes 256 MB (> 126 MB L2)


# Algorithmic bytes per unit (the path state each kernel must move; BVH nodes
# and triangles are counted separately: the unique scene geometry is a few MB
# and stays resident in L2).
EXT_STATE_BYTES_PER_RAY = 81       # reads ray o/d 32, pixel+flags 8, last hit 8; writes hit 16+16+1 (a miss: 40)
SHADE_STATE_BYTES_PER_HIT = 222    # reads path+hit state 125 B; writes the continuation 97 B
SHADOW_QUEUE_BYTES_PER_RAY = 48    # written by k_shade, read by k_connect
NODE_BYTES, TRI_BYTES = 80, 48     # one wide node; one triangle (3 float4)


def kernel_table(pst):
    """Per-kernel device time of the profiled frame with the algorithmic
    bytes of each launch (averaged over the frame's waves)."""
    waves = max(int(pst.waves), 1)
    ext_nodes = pst.node_visits - pst.shadow_node_visits
    ext_tris = pst.triangle_tests - pst.shadow_triangle_tests
    k = {
        "k_extend": dict(ms=pst.ms_extend, state=pst.extension_rays * EXT_STATE_BYTES_PER_RAY,
                         bvh=ext_nodes * NODE_BYTES + ext_tris * TRI_BYTES, units=pst.extension_rays, unit="rays"),
        "k_shade": dict(ms=pst.ms_shade, state=pst.shaded_hits * SHADE_STATE_BYTES_PER_HIT +
                        pst.shadow_rays * SHADOW_QUEUE_BYTES_PER_RAY, bvh=0, units=pst.shaded_hits, unit="hits"),
        "k_connect": dict(ms=pst.ms_connect, state=pst.shadow_rays * SHADOW_QUEUE_BYTES_PER_RAY,
                          bvh=pst.shadow_node_visits * NODE_BYTES + pst.shadow_triangle_tests * TRI_BYTES,
                          units=pst.shadow_rays, unit="shadow rays"),
        "k_sort_hits": dict(ms=pst.ms_sort, state=pst.extension_rays * 1 + pst.shaded_hits * 4, bvh=0,
                            units=pst.extension_rays, unit="slots"),
        "k_generate": dict(ms=pst.ms_generate, state=pst.paths * 97, bvh=0, units=pst.paths, unit="paths"),
    }
    out = {}
    for name, v in k.items():
        ms_launch = v["ms"] / waves
        out[name] = {"ms_per_frame": round(v["ms"], 3), "launches": waves, "ms_per_launch": round(ms_launch, 4),
                     "alg_state_bytes_per_launch": int(v["state"] / waves),
                     "bvh_bytes_per_launch": int(v["bvh"] / waves),
                     "units_per_launch": int(v["units"] / waves), "unit": v["unit"],
                     "state_gbs": round(v["state"] / waves / (ms_launch * 1e-3) / 1e9, 1) if ms_launch > 0 else None,
                     "bvh_l2_gbs": round(v["bvh"] / waves / (ms_launch * 1e-3) / 1e9, 1) if ms_launch > 0 else None}
    return out


def batch_renders(seed: int = 0, n: int = 64, small: bool = False):
    """The batched workload: n renders, each a Cornell-like or instanced
    scene variant (per-render scene seed), at a resolution drawn from
    {256x256, 512x512, 640x480, 1024x1024} and U{4..64} spp, all seeded.
    Instanced variants use two scene seeds (their BVH build dominates set-up).

    small=True: previews that each fill a small part of the GPU (2k-200k
    paths against a 2 Mi-path queue): n renders over a pool of 48 scenes
    (46 Cornell-like variants, each at one resolution of {64x64, 128x128,
    160x120, 256x256}, and the two instanced seeds at 128x128), U{1..8} spp."""
    rng = np.random.default_rng(seed)
    if small:
        res = [(64, 64), (128, 128), (160, 120), (256, 256)]
        pool = [("cornell", k, *res[k % len(res)]) for k in range(46)] + [("instanced", k, 128, 128) for k in range(2)]
        out = []
        for _ in range(n):
            kind, scene_seed, W, H = pool[int(rng.integers(0, len(pool)))]
            out.append({"scene": kind, "seed": scene_seed, "width": W, "height": H, "spp": int(rng.integers(1, 9)),
                        "depth": 12 if kind == "instanced" else 8})
        return out
    res = [(256, 256), (512, 512), (640, 480), (1024, 1024)]
    out = []
    for k in range(n):
        kind = "instanced" if rng.random() < 0.25 else "cornell"
        scene_seed = int(rng.integers(0, 2)) if kind == "instanced" else k
        W, H = res[int(rng.integers(0, len(res)))]
        spp = int(rng.integers(4, 65))
        out.append({"scene": kind, "seed": scene_seed, "width": W, "height": H, "spp": spp,
                    "depth": 12 if kind == "instanced" else 8})
    return out


def run_batch_workload(args):
    """64 renders in one batch (one CUDA-graph wave loop over all of them)
    against the same renders made one after another; workload batch_small:
    256 small previews (batch_renders(small=True)) the same way."""
    import torch
    import ymrt_b200 as Y
    from ymrt_b200 import scenes

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    perm = scenes.halton_permutations()
    small = args.workload == "batch_small"
    specs = batch_renders(seed=rank, n=256 if small else 64, small=small)
    ctx = Y.Context(local_rank)
    hosts, renders = {}, []
    for sp in specs:
        key = (sp["scene"], sp["seed"], sp["width"], sp["height"])
        if key not in hosts:
            hosts[key] = Y.Scene(ctx, Y.HostScene(scenes.scene_path(sp["scene"], sp["seed"]), sp["width"], sp["height"]),
                                 perm)
        out = torch.zeros((sp["height"], sp["width"], 4), dtype=torch.float32, device="cuda")
        renders.append([hosts[key], Y.default_setting(spp=sp["spp"], ray_depth=sp["depth"]), 1, out])
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def step(i):
        for r in renders:
            r[2] = i + 1
        st = Y.render_batch(ctx, renders)
        flush.add_(1.0)
        return st

    tuned = None
    if args.autotune:
        from ymrt_b200 import autotune
        r = autotune.tune_batch(ctx, renders, space={"queue_capacity": [1 << 21, 1 << 22], "sort_hits": [0, 1]},
                                repeats=1)
        tuned = {"best": r["best"], "table": [{"config": t["config"], "ms": t["ms"]} for t in r["table"]]}
    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    rays = launches = errors = 0
    for i in range(args.steps):
        st = step(args.warmup + i)
        rays += st.extension_rays + st.shadow_rays
        launches += st.kernel_launches
        errors |= st.device_errors
    ev1.record()
    torch.cuda.synchronize()
    clk = clocks.stop()
    elapsed = ev0.elapsed_time(ev1)
    # the same renders one after another (frame 1 of each)
    # (ms: the renders' own device times summed; loop_ms: CUDA events around
    # the whole loop, host calls between the renders included)
    seq_ms, seq_rays = 0.0, 0
    ev0.record()
    for sc, setting, _, out in renders:
        _, s1 = sc.render(setting, 1, out=out)
        seq_ms += s1.ms_total
        seq_rays += s1.extension_rays + s1.shadow_rays
    ev1.record()
    torch.cuda.synchronize()
    seq_loop_ms = ev0.elapsed_time(ev1)
    batch_ms = elapsed / args.steps
    paths = sum(sp["width"] * sp["height"] * sp["spp"] for sp in specs)
    result = {
        "metric": "Mrays/s", "value": round(rays / (elapsed * 1e-3) / 1e6, 2), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(batch_ms, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded .ymtmp scenes generated by ymrt_b200.scenes)",
        "config": {"workload": f"batch of {len(specs)} renders (Cornell-like and instanced variants, " +
                               ("64x64..256x256, 1-8 spp)" if small else "256x256..1024x1024, 4-64 spp)"),
                   "paths_per_step": paths,
                   "l2": "256 MB buffer written between steps"},
        "spp_per_s": round(paths / (batch_ms * 1e-3), 1),
        "sequential": {"ms": round(seq_ms, 3), "mrays_s": round(seq_rays / (seq_ms * 1e-3) / 1e6, 2),
                       "batch_speedup": round(seq_ms / batch_ms, 3), "loop_ms": round(seq_loop_ms, 3),
                       "batch_speedup_loop": round(seq_loop_ms / batch_ms, 3)},
        "gpu_launches": int(launches), "device_errors": int(errors), "clocks": clk,
        "autotuned": tuned,
        "renders": specs,
    }
    for sc in hosts.values():
        sc.close()
    ctx.close()
    return result if rank == 0 else None


def run_diff_workload(args, media=False):
    """Differentiable batched render: 16 views of the instanced scene (32
    materials) at 512x512, 16 spp, forward with path records and the
    path-replay backward of an L2 loss against a target rendered with
    perturbed albedos and roughnesses. Reports the forward and backward
    device times and their ratio. media=True: the scene sits in a box of fog
    whose density is a 64^3 float32 grid, the target's grid is scaled per cell
    by U[0.5, 1.5], and the backward pass also returns dLoss/d(grid)."""
    import torch
    import ymrt_b200 as Y
    from ymrt_b200 import scenes

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    perm = scenes.halton_permutations()
    n_views, size, spp = 16, 512, 16
    ctx = Y.Context(local_rank)
    name = "instanced_fog" if media else "instanced"
    path = scenes.scene_path(name, 0)
    views = [Y.Scene(ctx, Y.HostScene(path, size, size, camera=scenes.orbit_view(name, 0, v, n_views)), perm)
             for v in range(n_views)]
    setting = Y.default_setting(spp=spp, ray_depth=12, volume=media)
    grid_n, fog_tex = 64, 0
    grid = scenes.smooth_grid(grid_n, 5) if media else None
    if media:
        target_grid = (grid * np.random.default_rng(4).uniform(0.5, 1.5, grid.shape)).astype(np.float32)
        for v in views:
            v.set_density_grid(fog_tex, target_grid)
    images = [torch.zeros((size, size, 4), dtype=torch.float32, device="cuda") for _ in views]
    renders = [[v, setting, 1, img] for v, img in zip(views, images)]
    records = [torch.zeros((Y.path_count(r), 4), dtype=torch.float32, device="cuda") for r in renders]
    params = views[0].material_params()
    rng = np.random.default_rng(3)
    target_params = params.copy()
    live = params.sum(1) > 0
    target_params[live, :3] = np.clip(params[live, :3] + rng.uniform(-0.2, 0.2, (live.sum(), 3)), 0.0, 1.0)
    target_params[live, 3] = np.clip(params[live, 3] + rng.uniform(-0.1, 0.1, live.sum()), 0.01, 0.99)
    for v in views:
        v.set_material_params(target_params)
    Y.render_batch(ctx, renders)
    targets = [img.clone() for img in images]
    for v in views:
        v.set_material_params(params)
        if media:
            v.set_density_grid(fog_tex, grid)
    grads = torch.zeros((params.shape[0], 4), dtype=torch.float32, device="cuda")
    grid_grads = torch.zeros(grid_n ** 3, dtype=torch.float32, device="cuda") if media else None
    fwd_ms, bwd_ms, plain_ms = [], [], []
    for i in range(args.warmup + args.steps):
        for r in renders:
            r[2] = i + 1
        st_plain = Y.render_batch(ctx, renders)  # the plain forward (no records, deferred shadow rays)
        st_f = Y.render_batch(ctx, renders, records)
        dl = [2.0 * (img - t) for img, t in zip(images, targets)]
        if media:
            st_b = Y.render_backward_ex(ctx, renders, records, dl, material_grads=grads, grid_texture=fog_tex,
                                        grid_grads=grid_grads)
        else:
            st_b = Y.render_backward(ctx, renders, records, dl, grads)
        if i >= args.warmup:
            plain_ms.append(st_plain.ms_total)
            fwd_ms.append(st_f.ms_total)
            bwd_ms.append(st_b.ms_total)
        errors = st_f.device_errors | st_b.device_errors
    # per-stage device times of one profiled forward (recorded) and backward
    Y.library().ymrt_set_profiling(ctx.h, 1)
    st_pf = Y.render_batch(ctx, renders, records)
    if media:
        st_pb = Y.render_backward_ex(ctx, renders, records, dl, material_grads=grads, grid_texture=fog_tex,
                                     grid_grads=grid_grads)
    else:
        st_pb = Y.render_backward(ctx, renders, records, dl, grads)
    Y.library().ymrt_set_profiling(ctx.h, 0)

    def stages(st):
        return {k: round(getattr(st, "ms_" + k), 2) for k in ("generate", "extend", "sort", "shade", "connect")}

    g = grads.cpu().numpy()
    plain, fwd, bwd = float(np.mean(plain_ms)), float(np.mean(fwd_ms)), float(np.mean(bwd_ms))
    rays = st_f.extension_rays + st_f.shadow_rays
    result = {
        "metric": "Mrays/s", "value": round(rays / (fwd * 1e-3) / 1e6, 2), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(fwd + bwd, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded .ymtmp scene generated by ymrt_b200.scenes, 16 orbit views)",
        "config": {"workload": f"differentiable: {n_views} views {size}x{size} {spp}spp depth 12 of the instanced "
                               "scene" + (" in a fog box with a 64^3 float32 density grid" if media else "") +
                               ", L2 loss against perturbed-parameter target",
                   "params": "32 materials x (albedo rgb, roughness)" + (" + 64^3 density grid" if media else "")},
        "forward_plain_ms": round(plain, 3), "forward_recorded_ms": round(fwd, 3), "backward_ms": round(bwd, 3),
        "backward_over_plain_forward": round(bwd / plain, 3),
        "stage_ms": {"forward_recorded": stages(st_pf), "backward": stages(st_pb)},
        "grad_norm": float(np.linalg.norm(g)), "device_errors": int(errors),
    }
    if media:
        result["grid_grad_norm"] = float(torch.linalg.vector_norm(grid_grads).item())
    for v in views:
        v.close()
    ctx.close()
    return result if rank == 0 else None


def run_ours(args):
    import torch
    import ymrt_b200 as Y
    from ymrt_b200 import scenes

    from ymrt_b200 import distributed as D
    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        D.init("nccl", timeout_s=120)
    wl = WORKLOADS[args.workload]
    W, H = wl["width"], wl["height"]
    spp = args.spp or wl["spp"]
    perm = scenes.halton_permutations()
    path = scenes.scene_path(wl["scene"], 0)
    ctx = Y.Context(local_rank, queue_capacity=args.queue, profiling=False)
    if args.no_graph_loop:
        ctx.set_option("graph_loop", 0)
    for item in args.option:
        name, value = item.split("=")
        ctx.set_option(name, int(value))
    # host scene preparation (parse, the reference's binary SAH builds, wide
    # collapse, light table), timed apart from the frames: the reference's
    # editor does it once per scene edit, not per frame
    t_prep = time.perf_counter()
    host = Y.HostScene(path, W, H)
    prep_ms = (time.perf_counter() - t_prep) * 1e3
    scene = Y.Scene(ctx, host, perm)
    grid = None
    if wl.get("grid"):
        grid = scenes.fbm_grid(scene, 2, wl["grid"])
        scene.set_density_grid(2, grid, half=True)
    setting = Y.default_setting(spp=spp, ray_depth=wl["depth"], volume=wl.get("volume", False))
    image = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def step(i):
        _, st = scene.render(setting, frame_index=D.frame_index(i, rank, world), out=image)
        D.combine_frames(image, world, mean=False)  # one all-reduce of the ranks' frames per step
        flush_l2(torch, flush)
        return st

    for i in range(args.warmup):
        step(i)

    # Timed region: K steps between a barrier + synchronize on each side,
    # timed with CUDA events on this stream (render() returns after its own
    # stream finished, so the events bracket every kernel of the K frames).
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    rays = ext = shadow = launches = 0
    frame_ms = 0.0
    errors = 0
    for i in range(args.steps):
        st = step(args.warmup + i)
        rays += st.extension_rays + st.shadow_rays
        ext += st.extension_rays
        shadow += st.shadow_rays
        frame_ms += st.ms_total
        launches += st.kernel_launches
        errors |= st.device_errors
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    elapsed_ms = ev0.elapsed_time(ev1)

    # Per-kernel device times from one profiled frame (events around each launch).
    lib = Y.library()
    lib.ymrt_set_profiling(ctx.h, 1)
    _, pst = scene.render(setting, frame_index=10_000 + rank, out=image)
    lib.ymrt_set_profiling(ctx.h, 0)
    profiled_image = image.cpu().numpy() if rank == 0 else None

    # End to end through the C ABI: upload the scene from host memory, render,
    # read the image back into pinned host memory -- every step.
    host_img = torch.zeros((H, W, 4), dtype=torch.float32).pin_memory().numpy()
    e2e_rays, e2e_wall, e2e_upload, e2e_render_dev = 0, 0.0, 0.0, 0.0
    for i in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t = time.perf_counter()
        sc2 = Y.Scene(ctx, host, perm)
        if grid is not None:
            sc2.set_density_grid(2, grid, half=True)
        t_up = time.perf_counter()
        _, st = sc2.render(setting, frame_index=20_000 + i * world + rank, out=host_img)
        t_end = time.perf_counter()
        e2e_wall += t_end - t
        e2e_upload += t_up - t
        e2e_render_dev += st.ms_total * 1e-3
        e2e_rays += st.extension_rays + st.shadow_rays
        sc2.close()
    scene_bytes = scene_upload_bytes(host, perm) + (grid.size * 2 if grid is not None else 0)

    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([rays, elapsed_ms, e2e_rays, e2e_wall], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        rays_all, ms_max = t[0].item(), tmax[1].item()
        e2e_rays_all, e2e_wall_max = t[2].item(), tmax[3].item()
    else:
        rays_all, ms_max = rays, elapsed_ms
        e2e_rays_all, e2e_wall_max = e2e_rays, e2e_wall

    result = None
    if rank == 0:
        hbm_peak, peak_kind = read_peaks()
        kernels = kernel_table(pst)
        dominant = max(kernels, key=lambda n: kernels[n]["ms_per_frame"])
        dk = kernels[dominant]
        achieved = dk["state_gbs"] or 0.0
        value = rays_all / (ms_max * 1e-3) / 1e6
        result = {
            "metric": "Mrays/s", "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded .ymtmp scene generated by ymrt_b200.scenes)",
            "config": workload_config(wl, W, H, spp, world),
            "wave_options": {name: ctx.get_option(name) for name in Y.OPTIONS},
            "spp_per_s": round(W * H * spp * world * args.steps / (ms_max * 1e-3), 1),
            "rays": {"extension": ext, "shadow": shadow, "per_step": rays // max(args.steps, 1)},
            "frame_ms_device": round(frame_ms / args.steps, 3),
            "gpu_launches": int(launches),
            "device_errors": int(errors),
            "kernels": kernels,
            "roofline": {"bound": "hbm", "kernel": dominant, "achieved": achieved, "peak": hbm_peak,
                         "peak_kind": peak_kind, "unit": "GB/s", "frac": round(achieved / hbm_peak, 4),
                         "traffic": read_traffic(dominant, dk),
                         "alg_bytes_per_launch": dk["alg_state_bytes_per_launch"],
                         "l2_bvh_gbs": dk["bvh_l2_gbs"]},
            "e2e": {"value": round(e2e_rays_all / e2e_wall_max / 1e6, 2) if e2e_wall_max > 0 else None,
                    "unit": "Mrays/s", "h2d_bytes_per_step": int(scene_bytes), "d2h_bytes_per_step": int(W * H * 16),
                    "scene_prepare_host_ms": round(prep_ms, 2),
                    "ms_per_step": {"scene_upload": round(e2e_upload * 1e3 / max(1, min(args.steps, 3)), 2),
                                    "render_device": round(e2e_render_dev * 1e3 / max(1, min(args.steps, 3)), 2),
                                    "total": round(e2e_wall * 1e3 / max(1, min(args.steps, 3)), 2)}},
            "clocks": clk,
        }
        with quiet_stdout():
            if not args.no_ref_cuda:
                result["ref_cuda"] = ref_cuda_timing(path, perm, W, H, spp, wl["depth"], pst, volume=wl.get("volume", False))
            if not args.no_cpu_baseline:
                result["cpu_baseline"] = cpu_baseline(path, perm, W, H, spp, wl["depth"], budget_s=args.cpu_budget,
                                                      volume=wl.get("volume", False))
            if not args.no_fp64:
                result["rmse_vs_fp64"] = fp64_check(path, perm, W, H, spp, wl["depth"], 10_000, profiled_image,
                                                    volume=wl.get("volume", False))
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    scene.close()
    ctx.close()
    return result


def fp64_check(path, perm, W, H, spp, depth, frame, image, volume=False, n_tiles=40):
    """Image error of the profiled frame against the FP64 oracle (the
    reference's algorithm computed in double, oracle/_ref/libymrt_ref64.so)
    on the same samples, over a band of tiles through the middle of the frame,
    beside the error of the reference's own float arithmetic (the float
    oracle) on the same band."""
    try:
        from oracle import ref
        if not (ref.available() and ref.available64()):
            return {"unavailable": "oracle/_ref/libymrt_ref64.so not built"}
        total = ((W + 15) // 16) * ((H + 15) // 16)
        tb = max(0, total // 2 - n_tiles // 2)
        te = min(total, tb + n_tiles)
        imgs = []
        for fp64 in (True, False):
            r = ref.RefScene(path, perm, W, H, fp64=fp64)
            r.set_settings(spp=spp, ray_depth=depth, volume=int(volume))
            imgs.append(r.render_frame(frame, tb, te))
            r.close()
        c, b = imgs
        cov = c[..., 3] > 0
        ours = np.sqrt(np.mean((image[..., :3][cov].astype(np.float64) - c[..., :3][cov]) ** 2))
        theirs = np.sqrt(np.mean((b[..., :3][cov].astype(np.float64) - c[..., :3][cov]) ** 2))
    except Exception as e:  # noqa: BLE001 - reported, not fatal for our own measurement
        return {"unavailable": f"{type(e).__name__}: {e}"}
    return {"rmse": float(f"{ours:.4g}"), "rmse_reference_float": float(f"{theirs:.4g}"), "pixels": int(cov.sum()),
            "spp": spp, "sample": f"tiles {tb}..{te - 1} (16x16 each) of frame {frame}, same samples on all three"}


def ref_cuda_timing(path, perm, W, H, spp, depth, pst, frames=5, volume=False):
    """The reference's own wavefront kernels rebuilt for sm_100a
    (oracle/_ref/libymrt_refgpu.so, nvcc default floating-point flags), on
    the same frame: device time of its wave loop, the median of `frames`
    frames after one warm-up, with the SM clocks sampled while they run. Its
    paths are the same samples, so its query count is ours for the same frame
    index."""
    try:
        from oracle import ref
        if not ref.gpu_available(exact=False):
            return {"unavailable": "oracle/_ref/libymrt_refgpu.so not built"}
        rg = ref.RefGpuScene(path, perm, W, H)
        rg.set_settings(spp=spp, ray_depth=depth, volume=int(volume))
        rg.render_frame(10_000, copy_out=False)  # warm-up (same frame as the profiled one)
        clocks = ClockSampler(int(os.environ.get("LOCAL_RANK", "0")))
        clocks.start()
        ms = []
        for _ in range(frames):
            rg.render_frame(10_000, copy_out=False)
            ms.append(rg.last_render_ms())
        clk = clocks.stop()
        rg.set_profiling(True)
        rg.render_frame(10_000, copy_out=False)
        stages = rg.last_stage_ms()
        rg.close()
    except Exception as e:  # noqa: BLE001 - reported, not fatal for our own measurement
        return {"unavailable": f"{type(e).__name__}: {e}"}
    rays = pst.extension_rays + pst.shadow_rays
    med = float(np.median(ms))
    return {"value": round(rays / (med * 1e-3) / 1e6, 2), "unit": "Mrays/s", "ms_per_frame": round(med, 2),
            "frames": frames, "ms_min_max": [round(min(ms), 2), round(max(ms), 2)], "clocks": clk,
            "stage_ms": {k: round(v, 2) if isinstance(v, float) else v for k, v in stages.items()},
            "build": "reference src/Shading.cu stage kernels, nvcc -O3 sm_100a default FP flags, MAX_RAY_COUNT 1Mi",
            "rays_per_frame": int(rays)}


def read_traffic(kernel, dk):
    """DRAM bytes per launch of `kernel` from the committed ncu summary
    (profiles/traffic.json: bytes per unit from one capture), scaled to this
    frame's units per launch."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            t = json.load(f)[kernel]
        return {"bytes_per_launch": int(t["dram_bytes_per_unit"] * dk["units_per_launch"]),
                "dram_bytes_per_unit": t["dram_bytes_per_unit"], "unit": t["unit"], "source": t["source"]}
    except Exception:
        return None


def scene_upload_bytes(host, perm) -> int:
    c = host.counts()
    # instance/transform/node/triangle arrays plus the Halton table
    return int(c["instances"] * (32 + 128) + c["blas_nodes"] * 80 + c["tlas_nodes"] * 80 + c["triangles"] * (48 + 12 + 24)
               + perm.nbytes)


def _reference_sample(path, perm, W, H, spp, depth, budget_s, threads, volume):
    """The bounded tile sample the CPU legs time: tiles from the middle of
    frame 1, as many as the timing build renders in about budget_s on
    `threads` host threads. Returns the timing-build scene (settings made),
    the tile range and the closest-hit + occlusion queries the reference makes
    on it (counted by the counted build on the same tiles, untimed)."""
    from oracle import ref
    rs = ref.RefScene(path, perm, W, H, fast=True)
    rs.set_settings(spp=spp, ray_depth=depth, volume=int(volume))
    tiles_x, tiles_y = (W + 15) // 16, (H + 15) // 16
    total = tiles_x * tiles_y
    mid = (tiles_y // 2) * tiles_x
    # calibrate on growing samples from the same first tile (tiles differ in
    # cost across the frame) until one takes an eighth of the budget
    n = max(threads // 4, 1)
    while True:
        rs.render_frame(1, mid, mid + n, wave_capacity=256 * spp * min(n, 64), threads=threads)
        t1 = rs.last_render_seconds()
        if t1 >= budget_s / 8 or mid + n >= total:
            break
        n = min(total - mid, max(n + 1, int(n * min(8.0, budget_s / 8 / max(t1, 1e-3)))))
    n_tiles = int(max(1, min(total - mid, n * budget_s / max(t1, 1e-3))))
    counted = ref.RefScene(path, perm, W, H)
    counted.set_settings(spp=spp, ray_depth=depth, volume=int(volume))
    ref.query_counts(True)
    counted.render_frame(1, mid, mid + n_tiles, wave_capacity=256 * spp * min(n_tiles, 64), threads=threads)
    tq, sq = ref.query_counts(True)
    counted.close()
    return rs, (mid, mid + n_tiles), tq + sq, total


def cpu_baseline(path, perm, W, H, spp, depth, budget_s=10.0, threads=None, volume=False):
    """The reference's own path tracer built for the host (its timing build:
    g++ -O3 -march, no query counters), on a bounded tile sample of the same
    frame, all host threads."""
    threads = threads or os.cpu_count() or 1
    rs, (tb, te), rays, _ = _reference_sample(path, perm, W, H, spp, depth, budget_s, threads, volume)
    rs.render_frame(1, tb, te, wave_capacity=256 * spp * min(te - tb, 64), threads=threads)
    secs = rs.last_render_seconds()
    isa = rs.isa
    rs.close()
    n_tiles = te - tb
    return {"value": round(rays / secs / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "build": f"g++ -O3 -march={isa} (oracle/build_ref.py build_timing)",
            "sample": f"{n_tiles} tiles (16x16 px, {n_tiles * 256 * spp} paths at {spp} spp) from the middle of frame 1, "
                      f"{secs:.1f} s; queries counted by the counted build on the same tiles", "rays": rays}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return None
    from ymrt_b200 import scenes
    wl = WORKLOADS[args.workload]
    W, H = wl["width"], wl["height"]
    spp = args.spp or wl["spp"]
    perm = scenes.halton_permutations()
    path = scenes.scene_path(wl["scene"], 0)
    threads = os.cpu_count() or 1
    # each step a sample of about cpu_budget seconds, the whole run about two minutes at most
    budget = min(args.cpu_budget, 120.0 / (args.warmup + args.steps))
    rs, (tb, te), rays_per_step, total_tiles = _reference_sample(path, perm, W, H, spp, wl["depth"], budget,
                                                                 threads, wl.get("volume", False))
    secs = 0.0
    for i in range(args.warmup + args.steps):
        # every step renders the same sample (frame 1 of those tiles), whose
        # queries the counted build counted
        rs.render_frame(1, tb, te, wave_capacity=256 * spp * min(te - tb, 64), threads=threads)
        if i >= args.warmup:
            secs += rs.last_render_seconds()
    isa = rs.isa
    rs.close()
    rays = rays_per_step * args.steps
    value = rays / secs / 1e6
    n_tiles = te - tb
    sample = (f"{n_tiles} of {total_tiles} tiles per step ({n_tiles * 256 * spp} paths at {spp} spp, frame 1), "
              f"{threads} host threads, g++ -O3 -march={isa}")
    return {
        "impl": "reference", "metric": "Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded .ymtmp scene generated by ymrt_b200.scenes)",
        "config": workload_config(wl, W, H, spp, world),
        "cpu_baseline": {"value": round(value, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 3), "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=sorted(WORKLOADS) + ["batch", "batch_small", "diff", "diff_media"], default="instanced")
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--queue", type=int, default=0, help="path queue capacity (0 = library default)")
    ap.add_argument("--cpu-budget", type=float, default=10.0, help="seconds of CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip timing the reference's own CUDA kernels")
    ap.add_argument("--no-fp64", action="store_true", help="skip the image check against the FP64 oracle")
    ap.add_argument("--no-graph-loop", action="store_true",
                    help="launch the wave loop from the host instead of as one CUDA graph (for per-kernel profilers)")
    ap.add_argument("--option", action="append", default=[], metavar="NAME=VALUE",
                    help="wave option for the instanced-style workloads (ymrt_b200.OPTIONS), e.g. extend_refill=0")
    ap.add_argument("--autotune", action="store_true", help="batch workload: tune the wave options first")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        with quiet_stdout():
            res = run_reference(args)
    elif args.workload in ("batch", "batch_small"):
        res = run_batch_workload(args)
    elif args.workload in ("diff", "diff_media"):
        res = run_diff_workload(args, media=args.workload == "diff_media")
    else:
        res = run_ours(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
