"""Multi-GPU host logic on CPU: two gloo ranks (one process each), the same
steps bench.py takes with NCCL on GPUs."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from ymrt_b200 import distributed as D


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _frame(frame: int, shape=(8, 6, 4)) -> torch.Tensor:
    # a stand-in for a rendered frame: deterministic per frame index
    rng = np.random.default_rng(frame)
    return torch.as_tensor(rng.uniform(0.0, 1.0, shape).astype(np.float32))


def _worker(rank, world, port, steps, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    D.init("gloo", timeout_s=60)
    import torch.distributed as dist
    r, w, lr = D.env()
    assert (r, w, lr) == (rank, world, rank)
    frames = [D.frame_index(s, rank, world) for s in range(steps)]
    acc = torch.zeros((8, 6, 4))
    for f in frames:
        img = _frame(f)
        D.combine_frames(img, world)  # mean of the ranks' frames for this step
        acc += img
    t_max = D.max_over_ranks(10.0 + rank)
    n_sum = D.sum_over_ranks(1.0)
    dist.barrier()
    if rank == 0:
        np.save(os.path.join(out_dir, "acc.npy"), (acc / steps).numpy())
        np.save(os.path.join(out_dir, "meta.npy"), np.array([t_max, n_sum]))
    np.save(os.path.join(out_dir, f"frames_{rank}.npy"), np.array(frames))
    dist.destroy_process_group()


def test_two_ranks_render_disjoint_frames_and_combine_to_their_mean(tmp_path):
    world, steps = 2, 3
    mp.spawn(_worker, args=(world, _free_port(), steps, str(tmp_path)), nprocs=world, join=True)
    frames = sorted(np.concatenate([np.load(tmp_path / f"frames_{r}.npy") for r in range(world)]).tolist())
    assert frames == list(range(1, world * steps + 1))  # every progressive frame once
    want = torch.stack([_frame(f) for f in frames]).mean(0).numpy()
    assert np.allclose(np.load(tmp_path / "acc.npy"), want, rtol=1e-6, atol=1e-7)
    t_max, n_sum = np.load(tmp_path / "meta.npy")
    assert t_max == 11.0 and n_sum == 2.0


def test_single_process_needs_no_group():
    img = _frame(1)
    before = img.clone()
    D.combine_frames(img, 1)
    assert torch.equal(img, before)
    assert D.max_over_ranks(3.5) == 3.5
    assert D.frame_index(4, 0, 1) == 5
