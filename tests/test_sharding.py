"""Frames of one trajectory split over ranks and gathered back (two gloo
ranks on CPU): contiguous ranges, rows gathered in frame order, statistics
independent of the number of ranks and equal to the in-process C++ path's
formulas (binding.rs:704-743)."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def fake_rows(a, b):
    # stand-in for BindingSystem.run on frames a..b-1: deterministic per frame
    f = np.arange(a, b, dtype=np.float64)[:, None]
    return np.sin(f * 0.37 + np.arange(13)[None, :]) * 10.0 + f


def _rank(rank, world, port, n_frames, out_dir):
    import torch.distributed as dist

    from rust_simulation_tools import sharding as SH

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        a, b = SH.frame_range(n_frames, rank, world)
        rows = SH.gather_rows(fake_rows(a, b), n_frames)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"), rows)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_frames", [7, 8, 1])
def test_gather_over_two_gloo_ranks(tmp_path, n_frames):
    import torch.multiprocessing as mp

    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, n_frames, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    want = fake_rows(0, n_frames)
    for r in range(2):
        np.testing.assert_array_equal(np.load(tmp_path / f"rank{r}.npy"), want)


def test_frame_ranges_cover_once():
    from rust_simulation_tools.sharding import frame_range

    for F in range(0, 20):
        for W in range(1, 6):
            seen = []
            for r in range(W):
                a, b = frame_range(F, r, W)
                seen.extend(range(a, b))
            assert seen == list(range(F))
    with pytest.raises(ValueError):
        frame_range(4, 2, 2)


def test_statistics_formulas():
    from rust_simulation_tools.sharding import statistics

    rows = fake_rows(0, 9)
    st = statistics(rows)
    d = rows[:, 12]
    assert abs(st["mean_delta_total"] - d.mean()) < 1e-12
    assert abs(st["std_delta_total"] - d.std(ddof=1)) < 1e-12
    assert abs(st["sem_delta_total"] - d.std(ddof=1) / 3.0) < 1e-12
    assert statistics(rows[:1])["std_delta_mm"] == 0.0
    with pytest.raises(ValueError):
        statistics(rows[:0])
