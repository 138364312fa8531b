"""Failure semantics of the serving loop and the PB solver (GPU, no fault):
cancellation of queued and running requests, wait time-outs, unknown request
ids, requests too large for the device refused with RSTG_ERR_NOMEM
(MemoryError), and a PB solve capped before convergence that still returns an
energy with converged = false (pb_energy.rs:408-422 warns and returns the
energy of the last iterate)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rst():
    import rust_simulation_tools as r

    if r.device_count() < 1:
        pytest.skip("no CUDA device")
    return r


@pytest.fixture(scope="module")
def systems(rst, tmp_path_factory):
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("fail")
    out = []
    for k, (nr, nl, nf) in enumerate(((5000, 50, 96), (300, 20, 3), (200, 12, 2))):
        s = S.make_system(nr, nl, seed=90 + k)
        fr = S.make_frames(s, nf, seed=95 + k)
        prm = str(d / f"s{k}.prmtop")
        S.write_prmtop(s, prm)
        top = rst.read_prmtop(prm)
        out.append((s, fr, top, rst.BindingSystem(top, s.receptor_residues, s.ligand_residues)))
    return out


def test_cancel_queued_and_running_requests(rst, systems):
    from rust_simulation_tools._native import RequestCancelled

    (s0, f0, _, big), (s1, f1, _, mid), (s2, f2, _, small) = systems
    alone = small.run(f2)
    srv = rst.Server(max_inflight=1)
    try:
        a = srv.submit(big, f0)    # runs first (one slot)
        b = srv.submit(mid, f1)    # queued behind it
        c = srv.submit(small, f2)  # queued
        srv.cancel(b)              # queued: removed at once
        srv.cancel(a)              # running: its results are discarded when it ends
        with pytest.raises(RequestCancelled):
            srv.wait(b, 60000)
        with pytest.raises(RequestCancelled):
            srv.wait(a, 600000)
        np.testing.assert_array_equal(srv.wait(c, 600000), alone)
        assert srv.stats()["completed"] == 1
    finally:
        srv.close()


def test_wait_times_out_and_unknown_ids_fail(rst, systems):
    (s0, f0, _, big), _, _ = systems
    srv = rst.Server(max_inflight=1)
    try:
        a = srv.submit(big, f0)
        with pytest.raises(TimeoutError):
            srv.wait(a, 0)
        assert srv.poll(a) is None or srv.poll(a).shape == (f0.shape[0], 13)
        out = srv.wait(a, 600000)  # a time-out leaves the request running
        assert out.shape == (f0.shape[0], 13) and np.all(np.isfinite(out))
        srv._keep[12345] = (big, 1)
        with pytest.raises(ValueError, match="unknown request id"):
            srv.wait(12345, 0)
    finally:
        srv.close()


def test_request_too_large_for_the_device_is_refused(rst, systems):
    # a 0.05 A PB grid around a 220-atom complex needs far more than the device holds
    _, (s1, f1, top, _), _ = systems
    p = rst.PbParams(grid_spacing=0.05, grid_buffer=10.0, fillratio=0.0)
    huge = rst.BindingSystem(top, s1.receptor_residues, s1.ligand_residues, pb_params=p)
    srv = rst.Server(max_inflight=2)
    try:
        with pytest.raises(MemoryError):
            srv.submit(huge, f1[:1])
    finally:
        srv.close()
    with pytest.raises(MemoryError):
        huge.run(f1[:1])


def test_pb_iteration_cap_returns_unconverged_energy(rst, systems):
    _, (s1, f1, top, _), _ = systems
    x_nm = (f1[0].astype(np.float64) * 0.1)
    capped = rst.compute_pb_energy(top, x_nm, rst.PbParams(grid_spacing=0.7, grid_buffer=4.0, fillratio=0.0,
                                                           max_iterations=1))
    full = rst.compute_pb_energy(top, x_nm, rst.PbParams(grid_spacing=0.7, grid_buffer=4.0, fillratio=0.0))
    assert capped.diag["converged"] == [False, False]
    assert capped.diag["iterations"] == [1, 1]
    assert np.isfinite(capped.total) and capped.total != full.total
    assert full.diag["converged"] == [True, True]
    # the batched engine applies the same cap: one V-cycle per grid, an energy all the same
    p = rst.PbParams(grid_spacing=0.7, grid_buffer=4.0, fillratio=0.0, max_iterations=1)
    b = rst.BindingSystem(top, s1.receptor_residues, s1.ligand_residues, pb_params=p)
    out = b.run(f1[:1])
    assert np.all(np.isfinite(out)) and b.pb_stats()["cycles"] >= 1
