"""Frames of one trajectory spread over the GPUs of a node.

Every (frame, subsystem) evaluation is independent, so the frames are split
into contiguous ranges, one per rank (one process per GPU), each rank runs
its range through its own BindingSystem, and the per-frame rows are gathered
back in frame order.  The statistics of binding.rs:704-743 are then taken
over the gathered rows in that order, so they do not depend on the number of
ranks.  torch.distributed is the plumbing (NCCL between GPUs, gloo on CPU);
the gather moves 13 doubles per frame.
"""
from __future__ import annotations

import numpy as np


def frame_range(n_frames: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of a rank's frames: contiguous blocks, the first
    n_frames % world ranks take one frame more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_frames, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def gather_rows(local: np.ndarray, n_frames: int, group=None) -> np.ndarray:
    """All-gather the (rows, k) float64 blocks of every rank into (n_frames, k)
    in rank (= frame) order."""
    import torch
    import torch.distributed as dist

    world = dist.get_world_size(group)
    local = np.ascontiguousarray(local, dtype=np.float64)
    k = local.shape[1]
    counts = [frame_range(n_frames, r, world)[1] - frame_range(n_frames, r, world)[0] for r in range(world)]
    if local.shape[0] != counts[dist.get_rank(group)]:
        raise ValueError("local rows do not match this rank's frame range")
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else torch.device("cpu")
    m = max(counts)
    buf = torch.zeros((m, k), dtype=torch.float64, device=dev)
    if local.shape[0]:
        buf[: local.shape[0]] = torch.from_numpy(local).to(dev)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather(parts, buf, group=group)
    return np.concatenate([parts[r][: counts[r]].cpu().numpy() for r in range(world)], axis=0)


def binding_frames_sharded(system, frames_f32_A, group=None) -> np.ndarray:
    """(F, 13) frame energies of all F frames, each rank evaluating its range
    with ``system`` (a BindingSystem on that rank's GPU); every rank receives
    the full array."""
    import torch.distributed as dist

    F = frames_f32_A.shape[0]
    a, b = frame_range(F, dist.get_rank(group), dist.get_world_size(group))
    local = system.run(frames_f32_A[a:b]) if b > a else np.zeros((0, 13))
    return gather_rows(local, F, group)


def statistics(rows: np.ndarray) -> dict:
    """Means and sample standard deviations (n - 1) of the four binding terms
    and the standard error of the total, over (F, 13) frame rows in frame
    order, with the reference's summation order (binding.rs:704-743)."""
    rows = np.asarray(rows, dtype=np.float64)
    n = rows.shape[0]
    if n == 0:
        raise ValueError("No frames found in trajectory")
    out = {}
    for name, col in (("delta_mm", 9), ("delta_polar", 10), ("delta_sa", 11), ("delta_total", 12)):
        vals = rows[:, col].tolist()
        mean = 0.0
        for v in vals:
            mean += v
        mean /= n
        if n <= 1:
            std = 0.0
        else:
            var = 0.0
            for v in vals:
                var += (v - mean) * (v - mean)
            std = float(np.sqrt(var / (n - 1)))
        out["mean_" + name] = mean
        out["std_" + name] = std
    out["sem_delta_total"] = out["std_delta_total"] / float(np.sqrt(n))
    return out
