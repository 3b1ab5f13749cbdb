"""Benchmark: Mrays/s of the ymrt_b200 path tracer on one B200 (or N replicas).

Workload (the reference's headline configuration that fits one GPU): the
seeded instanced scene of ~1.2 M triangles (64 instances of an icosphere, a
fBm heightfield, a torus and a box; 32 GGX conductor / dielectric / diffuse
materials; 2 quad lights), 1920x1080, 64 samples per pixel, maximum depth 12,
Halton sampler, shape-light next-event estimation. One step = one full frame.

Metric: Mrays/s = (closest-hit queries + occlusion queries) / frame time; the
reference performs the same queries on the same paths (its counts are taken
from the instrumented oracle build in the reference arm).

Arms:
  (default)          ymrt_b200 kernels; `value` timed on the device with the
                     scene resident; `e2e` through the C ABI with the scene
                     uploaded from host memory and the image read back every step.
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
}


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


def run_ours(args):
    import torch
    import ymrt_b200 as Y
    from ymrt_b200 import scenes

    rank, world, local_rank = dist_env()
    torch.cuda.set_device(local_rank)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    wl = WORKLOADS[args.workload]
    W, H = wl["width"], wl["height"]
    spp = args.spp or wl["spp"]
    perm = scenes.halton_permutations()
    path = scenes.scene_path(wl["scene"], 0)
    ctx = Y.Context(local_rank, queue_capacity=args.queue, profiling=False)
    host = Y.HostScene(path, W, H)
    scene = Y.Scene(ctx, host, perm)
    setting = Y.default_setting(spp=spp, ray_depth=wl["depth"])
    image = torch.zeros((H, W, 4), dtype=torch.float32, device="cuda")
    flush = torch.zeros(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def step(i):
        _, st = scene.render(setting, frame_index=i * world + rank + 1, out=image)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(image)
        flush_l2(torch, flush)
        return st

    for i in range(args.warmup):
        step(i)
    torch.cuda.synchronize()
    barrier()
    clocks = ClockSampler(local_rank)
    clocks.start()
    t0 = time.perf_counter()
    rays = 0
    dev_ms = 0.0
    launches = 0
    node_visits = tri_tests = ext = shadow = 0
    errors = 0
    for i in range(args.steps):
        st = step(args.warmup + i)
        rays += st.extension_rays + st.shadow_rays
        ext += st.extension_rays
        shadow += st.shadow_rays
        node_visits += st.node_visits
        tri_tests += st.triangle_tests
        dev_ms += st.ms_total
        launches += st.kernel_launches
        errors |= st.device_errors
    torch.cuda.synchronize()
    barrier()
    wall = time.perf_counter() - t0
    clk = clocks.stop()

    # Per-stage device times from one profiled frame (events around each launch).
    lib = Y.library()
    lib.ymrt_set_profiling(ctx.h, 1)
    _, pst = scene.render(setting, frame_index=10_000 + rank, out=image)
    lib.ymrt_set_profiling(ctx.h, 0)

    # End to end through the C ABI: upload the scene from host memory, render,
    # read the image back -- every step.
    host_img = np.zeros((H, W, 4), np.float32)
    e2e_rays, e2e_wall = 0, 0.0
    h2d = None
    for i in range(max(1, min(args.steps, 3))):
        torch.cuda.synchronize()
        t = time.perf_counter()
        sc2 = Y.Scene(ctx, host, perm)
        _, st = sc2.render(setting, frame_index=20_000 + i * world + rank, out=host_img)
        e2e_wall += time.perf_counter() - t
        e2e_rays += st.extension_rays + st.shadow_rays
        sc2.close()
        if h2d is None:
            c = host.counts()
            h2d = None
    scene_bytes = scene_upload_bytes(host, perm)

    out = {"rays": rays, "dev_ms": dev_ms, "wall": wall, "ext": ext, "shadow": shadow}
    if world > 1:
        import torch.distributed as dist
        t = torch.tensor([rays, dev_ms, wall, e2e_rays, e2e_wall], dtype=torch.float64, device="cuda")
        tmax = t.clone()
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        dist.all_reduce(tmax, op=dist.ReduceOp.MAX)
        rays_all, dev_ms_max, wall_max = t[0].item(), tmax[1].item(), tmax[2].item()
        e2e_rays_all, e2e_wall_max = t[3].item(), tmax[4].item()
    else:
        rays_all, dev_ms_max, wall_max = rays, dev_ms, wall
        e2e_rays_all, e2e_wall_max = e2e_rays, e2e_wall

    result = None
    if rank == 0:
        hbm_peak, peak_kind = read_peaks()
        # Roofline of the dominant kernel (the shade stage: next-event shadow
        # traversals plus BSDF work). Algorithmic bytes per path-vertex:
        # traversal fetches (80 B per wide node, 48 B per triangle) plus the
        # path/hit state the stage reads and writes.
        dominant = "k_shade" if pst.ms_shade >= pst.ms_extend else "k_extend"
        frac_nodes = 1.0
        state_ext = 32 + 8 + 8 + 16 + 32  # ray, pixel/flags, last hit, sampler; hit record written
        state_shade = 32 + 32 + 8 + 8 + 16 + 32 + 104 * 0  # path state read + hit read (+ continuation write below)
        alg_bytes = pst.node_visits * 80 + pst.triangle_tests * 48 + pst.extension_rays * (state_ext + state_shade + 96)
        ms_kernels = pst.ms_extend + pst.ms_shade + pst.ms_generate
        achieved = alg_bytes / (ms_kernels * 1e-3) / 1e9 if ms_kernels > 0 else 0.0
        value = rays_all / (dev_ms_max * 1e-3) / 1e6
        result = {
            "metric": "Mrays/s", "value": round(value, 2), "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(dev_ms_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded .ymtmp scene generated by ymrt_b200.scenes)",
            "config": {"workload": f"{wl['scene']} {W}x{H} {spp}spp depth {wl['depth']} (~1.2M instanced triangles)"
                       if wl["scene"] == "instanced" else f"{wl['scene']} {W}x{H} {spp}spp depth {wl['depth']}",
                       "sampler": "halton", "lights": "shape lights, NEE with MIS",
                       "parallelism": f"replica x{world}" + (" + allreduce of frames" if world > 1 else ""),
                       "l2": "256 MB buffer written between steps; path queues (>1 GB) exceed L2"},
            "spp_per_s": round(W * H * spp * world / (dev_ms_max * 1e-3 / args.steps) / args.steps * args.steps, 1),
            "rays": {"extension": ext, "shadow": shadow, "per_step": rays // max(args.steps, 1)},
            "wall_s": round(wall_max, 3),
            "gpu_launches": int(launches),
            "device_errors": int(errors),
            "stage_ms": {"generate": round(pst.ms_generate, 2), "extend": round(pst.ms_extend, 2),
                         "shade": round(pst.ms_shade, 2), "frame": round(pst.ms_total, 2), "waves": int(pst.waves)},
            "roofline": {"bound": "hbm", "kernels": "k_extend+k_shade+k_generate", "dominant": dominant,
                         "achieved": round(achieved, 1), "peak": hbm_peak, "peak_kind": peak_kind, "unit": "GB/s",
                         "frac": round(achieved / hbm_peak, 4), "traffic": read_traffic(pst),
                         "alg_bytes_per_frame": int(alg_bytes)},
            "e2e": {"value": round(e2e_rays_all / e2e_wall_max / 1e6, 2) if e2e_wall_max > 0 else None,
                    "unit": "Mrays/s", "h2d_bytes_per_step": int(scene_bytes), "d2h_bytes_per_step": int(W * H * 16)},
            "clocks": clk,
        }
        if not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(path, perm, W, H, spp, wl["depth"], budget_s=args.cpu_budget)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    scene.close()
    ctx.close()
    return result


def read_traffic(pst):
    """DRAM bytes per frame from the committed ncu summary, scaled to this frame."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            t = json.load(f)
        return {"bytes_per_path_vertex": t["bytes_per_path_vertex"],
                "bytes_per_frame": int(t["bytes_per_path_vertex"] * pst.extension_rays), "source": t["source"]}
    except Exception:
        return None


def scene_upload_bytes(host, perm) -> int:
    c = host.counts()
    # instance/transform/node/triangle arrays plus the Halton table
    return int(c["instances"] * (32 + 128) + c["blas_nodes"] * 80 + c["tlas_nodes"] * 80 + c["triangles"] * (48 + 12 + 24)
               + perm.nbytes)


def cpu_baseline(path, perm, W, H, spp, depth, budget_s=15.0, threads=None):
    """The reference's own path tracer built for the host, on a bounded tile
    sample of the same frame (all host threads)."""
    from oracle import ref
    threads = threads or os.cpu_count() or 1
    rs = ref.RefScene(path, perm, W, H)
    rs.set_settings(spp=spp, ray_depth=depth)
    tiles_x, tiles_y = (W + 15) // 16, (H + 15) // 16
    mid = (tiles_y // 2) * tiles_x
    # calibrate on a few tiles, then size the sample to the budget
    n = max(threads // 4, 1)
    ref.query_counts(True)
    rs.render_frame(1, mid, mid + n, wave_capacity=256 * spp * max(n, 1), threads=threads)
    t1 = rs.last_render_seconds()
    ref.query_counts(True)
    n_tiles = int(max(1, min(tiles_x * tiles_y - mid, n * budget_s / max(t1, 1e-3))))
    rs.render_frame(1, mid, mid + n_tiles, wave_capacity=256 * spp * min(n_tiles, 64), threads=threads)
    secs = rs.last_render_seconds()
    tq, sq = ref.query_counts(True)
    rs.close()
    return {"value": round((tq + sq) / secs / 1e6, 3), "unit": "Mrays/s", "cores": threads, "kind": "reference",
            "sample": f"{n_tiles} tiles (16x16 px, {n_tiles * 256 * spp} paths at {spp} spp) from the middle of the frame, "
                      f"{secs:.1f} s", "rays": tq + sq}


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
    from oracle import ref
    threads = os.cpu_count() or 1
    rs = ref.RefScene(path, perm, W, H)
    rs.set_settings(spp=spp, ray_depth=wl["depth"])
    tiles_x, tiles_y = (W + 15) // 16, (H + 15) // 16
    total_tiles = tiles_x * tiles_y
    mid = (tiles_y // 2) * tiles_x
    n = max(threads // 4, 1)
    ref.query_counts(True)
    rs.render_frame(1, mid, mid + n, wave_capacity=256 * spp * n, threads=threads)
    t1 = rs.last_render_seconds()
    n_tiles = int(max(1, min(total_tiles - mid, n * args.cpu_budget / max(t1, 1e-3))))
    rays = 0
    secs = 0.0
    for i in range(args.warmup + args.steps):
        ref.query_counts(True)
        rs.render_frame(i + 1, mid, mid + n_tiles, wave_capacity=256 * spp * min(n_tiles, 64), threads=threads)
        tq, sq = ref.query_counts(True)
        if i >= args.warmup:
            rays += tq + sq
            secs += rs.last_render_seconds()
    rs.close()
    value = rays / secs / 1e6
    sample = f"{n_tiles} of {total_tiles} tiles per step ({n_tiles * 256 * spp} paths at {spp} spp)"
    return {
        "impl": "reference", "metric": "Mrays/s", "value": round(value, 3), "unit": "Mrays/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(secs / args.steps * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded .ymtmp scene generated by ymrt_b200.scenes)",
        "config": {"workload": f"{wl['scene']} {W}x{H} {spp}spp depth {wl['depth']}", "sampler": "halton",
                   "parallelism": f"{threads} host threads"},
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
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="instanced")
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--queue", type=int, default=0, help="path queue capacity (0 = library default)")
    ap.add_argument("--cpu-budget", type=float, default=12.0, help="seconds of CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args(argv)
    if args.warmup < 3:
        args.warmup = 3
    res = run_reference(args) if args.impl == "reference" else run_ours(args)
    if res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()
