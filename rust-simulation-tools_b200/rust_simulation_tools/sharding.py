"""Frames of one trajectory spread over the GPUs of a node.

Every (frame, subsystem) evaluation is independent, so the frames are split
into contiguous ranges, one per rank (one process per GPU), each rank runs
its range through its own BindingSystem, and the per-frame rows are merged
back in frame order on the host.  The statistics of binding.rs:704-743 are
then taken over the merged rows in that order, so they do not depend on the
number of ranks.

The module carries no transport of its own: the caller hands in an
``allgather(obj) -> list`` callable that returns every rank's object in rank
order (13 doubles per frame cross it).  With torch.distributed that is::

    def allgather(obj):
        out = [None] * dist.get_world_size()
        dist.all_gather_object(out, obj)
        return out

with mpi4py ``comm.allgather``; in one process ``lambda obj: [obj]``.
"""
from __future__ import annotations

from typing import Callable, Sequence

import numpy as np


def frame_range(n_frames: int, rank: int, world: int) -> tuple[int, int]:
    """[start, stop) of a rank's frames: contiguous blocks, the first
    n_frames % world ranks take one frame more."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(n_frames, world)
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def merge_rows(blocks: Sequence[np.ndarray], n_frames: int) -> np.ndarray:
    """The (n_frames, k) rows of all ranks in frame order, from the per-rank
    (rows, k) blocks listed in rank order; each block must hold exactly its
    rank's frame range."""
    world = len(blocks)
    if world < 1:
        raise ValueError("no rank blocks to merge")
    out = []
    for r, b in enumerate(blocks):
        a, e = frame_range(n_frames, r, world)
        b = np.asarray(b, dtype=np.float64)
        if b.ndim != 2 or b.shape[0] != e - a:
            raise ValueError(f"rank {r} sent a block of shape {b.shape} for frames [{a}, {e})")
        out.append(b)
    return np.concatenate(out, axis=0)


def gather_rows(local: np.ndarray, n_frames: int, rank: int, world: int,
                allgather: Callable[[object], list]) -> np.ndarray:
    """Every rank's (rows, k) float64 block, exchanged through ``allgather``
    and merged into (n_frames, k) in frame order."""
    a, b = frame_range(n_frames, rank, world)
    local = np.ascontiguousarray(local, dtype=np.float64)
    if local.shape[0] != b - a:
        raise ValueError("local rows do not match this rank's frame range")
    blocks = allgather(local)
    if len(blocks) != world:
        raise ValueError(f"allgather returned {len(blocks)} blocks for {world} ranks")
    return merge_rows(blocks, n_frames)


def binding_frames_sharded(system, frames_f32_A, rank: int, world: int,
                           allgather: Callable[[object], list]) -> np.ndarray:
    """(F, 13) frame energies of all F frames, each rank evaluating its range
    with ``system`` (a BindingSystem on that rank's GPU); every rank receives
    the full array."""
    F = frames_f32_A.shape[0]
    a, b = frame_range(F, rank, world)
    local = system.run(frames_f32_A[a:b]) if b > a else np.zeros((0, 13))
    return gather_rows(local, F, rank, world, allgather)


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
