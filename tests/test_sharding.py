"""Frames of one trajectory split over ranks and merged back on the host
(two gloo ranks on CPU): contiguous ranges, rows merged in frame order,
statistics independent of the number of ranks and equal to the reference's
formulas (binding.rs:704-743).  Each rank evaluates its own frames of a small
synthetic system with the CPU restatement (the GPU engine's rows go through
the same merge in tests/test_gpu_gbsa.py)."""
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


def _system(tmp_dir):
    from rust_simulation_tools import synthetic as S

    s = S.make_system(60, 8, seed=71)
    fr = S.make_frames(s, 7, seed=72)
    prm = os.path.join(tmp_dir, "shard.prmtop")
    if not os.path.exists(prm):
        S.write_prmtop(s, prm)
    return s, fr, prm


def _oracle_rows(prm, s, fr):
    import oracle as O

    O.set_threads(1)
    top = O.Topology.load(prm)
    x = (fr.astype(np.float64) * 0.1) * 10.0
    return O.binding_frames(top, x, s.receptor_residues, s.ligand_residues,
                            gb=O.gb_params("obc2", solvent_dielectric=78.5), sa=O.sa_params(n_points=120))


def _rank(rank, world, port, n_frames, out_dir):
    import datetime

    import torch.distributed as dist

    from rust_simulation_tools import sharding as SH

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        s, fr, prm = _system(out_dir)
        fr = fr[:n_frames]
        a, b = SH.frame_range(n_frames, rank, world)
        local = _oracle_rows(prm, s, fr[a:b]) if b > a else np.zeros((0, 13))

        def allgather(obj):
            out = [None] * world
            dist.all_gather_object(out, obj)
            return out

        rows = SH.gather_rows(local, n_frames, rank, world, allgather)
        np.save(os.path.join(out_dir, f"rank{rank}_{n_frames}.npy"), rows)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_frames", [7, 4, 1])
def test_gather_over_two_gloo_ranks(tmp_path, n_frames):
    import torch.multiprocessing as mp

    from rust_simulation_tools import sharding as SH

    s, fr, prm = _system(str(tmp_path))
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_rank, args=(r, 2, port, n_frames, str(tmp_path))) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    want = _oracle_rows(prm, s, fr[:n_frames])
    for r in range(2):
        got = np.load(tmp_path / f"rank{r}_{n_frames}.npy")
        np.testing.assert_array_equal(got, want)
        assert SH.statistics(got) == SH.statistics(want)


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


def test_merge_rejects_wrong_block_sizes():
    from rust_simulation_tools.sharding import merge_rows

    rows = np.arange(5 * 13, dtype=np.float64).reshape(5, 13)
    np.testing.assert_array_equal(merge_rows([rows[:3], rows[3:]], 5), rows)
    with pytest.raises(ValueError):
        merge_rows([rows[:2], rows[2:]], 5)
    with pytest.raises(ValueError):
        merge_rows([], 5)


def test_statistics_formulas():
    from rust_simulation_tools.sharding import statistics

    f = np.arange(9, dtype=np.float64)[:, None]
    rows = np.sin(f * 0.37 + np.arange(13)[None, :]) * 10.0 + f
    st = statistics(rows)
    d = rows[:, 12]
    assert abs(st["mean_delta_total"] - d.mean()) < 1e-12
    assert abs(st["std_delta_total"] - d.std(ddof=1)) < 1e-12
    assert abs(st["sem_delta_total"] - d.std(ddof=1) / 3.0) < 1e-12
    assert statistics(rows[:1])["std_delta_mm"] == 0.0
    with pytest.raises(ValueError):
        statistics(rows[:0])
