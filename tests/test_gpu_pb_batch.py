"""GPU parity of the batched mixed-precision PB engine (fused BindingSystem
with PbParams).

Tolerances:
  * per-frame binding terms within 1e-3 kcal/mol of the CPU restatement
    (accurate receptor x ligand MM differences), subsystem PB energies within
    1e-6 relative;
  * on the 3,040-atom PB workload the CPU restatement takes about a minute
    per frame, so the batched engine is compared with the plain FP64 GPU
    form there, which tests/test_gpu_pb.py pins to the restatement (grid maps
    bit for bit, energies within 1e-8 relative): polar terms within 1e-3;
  * a frame gives identical bits alone and inside a larger batch.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FRAME = ("complex_mm", "complex_polar", "complex_sa", "receptor_mm", "receptor_polar", "receptor_sa",
         "ligand_mm", "ligand_polar", "ligand_sa", "delta_mm", "delta_polar", "delta_sa", "delta_total")


@pytest.fixture(scope="module")
def rst():
    import rust_simulation_tools as r

    if r.device_count() < 1:
        pytest.skip("no CUDA device")
    return r


def dcd_coords(fr):
    return (fr.astype(np.float64) * 0.1) * 10.0


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.fixture(scope="module")
def small(tmp_path_factory):
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("pbb")
    s = S.make_system(40, 6, seed=51)
    fr = S.make_frames(s, 3, seed=52)
    S.write_prmtop(s, str(d / "s.prmtop"))
    return s, fr, str(d / "s.prmtop")


@pytest.mark.parametrize("fill,spacing,buffer", [(0.0, 0.6, 4.0), (4.0, 0.6, 4.0), (0.0, 1.0, 2.0)])
def test_pb_fused_matches_restatement(rst, oracle, small, fill, spacing, buffer):
    # (0.0, 1.0, 2.0): grids of at most 8 points per side take the plain SOR path
    s, fr, prm = small
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    p = rst.PbParams(grid_spacing=spacing, grid_buffer=buffer, fillratio=fill)
    op = oracle.pb_params(grid_spacing=spacing, grid_buffer=buffer, fillratio=fill)
    sysf = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p, mode="fused")
    out = sysf.run(fr)
    for f in range(len(fr)):
        acc = oracle.binding_frame(otop, dcd_coords(fr[f]), s.receptor_residues, s.ligand_residues, pb=op,
                                   accurate=True)
        for k in (9, 10, 11, 12):
            assert abs(out[f, k] - acc[FRAME[k]]) < 1e-3, (f, FRAME[k], out[f, k], acc[FRAME[k]])
        for k in (1, 4, 7):
            assert rel(out[f, k], acc[FRAME[k]]) < 1e-6, (f, FRAME[k], out[f, k], acc[FRAME[k]])
        assert abs(out[f, 12] - (out[f, 9] + out[f, 10] + out[f, 11])) < 1e-9
    st = sysf.pb_stats()
    assert st["grids"] == len(fr) * 6 * (2 if fill > 0 else 1)
    if spacing == 1.0:
        assert st["fp64_fallbacks"] > 0  # SOR grids are counted there


@pytest.fixture(scope="module")
def w3(tmp_path_factory):
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("w3")
    s, fr = S.workload(3, n_frames=2)
    S.write_prmtop(s, str(d / "w3.prmtop"))
    return s, fr, str(d / "w3.prmtop")


@pytest.mark.parametrize("buffer,fill", [(12.0, 0.0), (10.0, 4.0)])
def test_pb_fused_matches_plain_on_workload(rst, w3, buffer, fill):
    # frame 0: the complex and receptor solvated grids stop at the 200-cycle
    # cap unconverged; frame 1: the complex V-cycles diverge and SOR follows
    s, fr, prm = w3
    top = rst.read_prmtop(prm)
    p = rst.PbParams(grid_buffer=buffer, fillratio=fill)
    fused = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p, mode="fused").run(fr)
    plain = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p, mode="plain").run(fr)
    for k in (1, 4, 7, 10):
        np.testing.assert_allclose(fused[:, k], plain[:, k], rtol=0, atol=1e-3, err_msg=FRAME[k])
    np.testing.assert_allclose(fused[:, 11], plain[:, 11], rtol=0, atol=1e-9)


def test_pb_fused_frame_alone_equals_batch(rst, small):
    s, fr, prm = small
    top = rst.read_prmtop(prm)
    p = rst.PbParams(grid_spacing=0.6, grid_buffer=4.0, fillratio=4.0)
    a = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p).run(fr)
    one = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p)
    one.set_pb_batch(1)
    b = np.concatenate([one.run(fr[f:f + 1]) for f in range(len(fr))])
    np.testing.assert_array_equal(a, b)


def test_server_mixes_pb_and_gb_requests(rst, small):
    # PB and GB requests interleaved in one serving loop: each result is the
    # same bits as the request run alone
    s, fr, prm = small
    top = rst.read_prmtop(prm)
    pbs = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues,
                            pb_params=rst.PbParams(grid_spacing=0.6, grid_buffer=4.0, fillratio=4.0))
    gbs = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues)
    alone_p, alone_g = pbs.run(fr), gbs.run(fr)
    srv = rst.Server(max_inflight=3)
    ids = [srv.submit(pbs, fr), srv.submit(gbs, fr), srv.submit(pbs, fr[1:]), srv.submit(gbs, fr[:2])]
    res = [srv.wait(i, 600000) for i in ids]
    st = srv.stats()
    srv.close()
    np.testing.assert_array_equal(res[0], alone_p)
    np.testing.assert_array_equal(res[1], alone_g)
    np.testing.assert_array_equal(res[2], alone_p[1:])
    np.testing.assert_array_equal(res[3], alone_g[:2])
    assert st["completed"] == 4


def test_server_evicts_pb_systems_under_budget(rst, small):
    # a budget smaller than any request: one request at a time, each admission
    # releases the idle system's resident batch buffers (PB pools included);
    # results keep their bits when the systems come back
    s, fr, prm = small
    top = rst.read_prmtop(prm)
    pbs = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues,
                            pb_params=rst.PbParams(grid_spacing=0.6, grid_buffer=4.0))
    gbs = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues)
    alone_p, alone_g = pbs.run(fr), gbs.run(fr)
    srv = rst.Server(memory_budget_bytes=1, max_inflight=2)
    ids = [srv.submit(pbs, fr), srv.submit(gbs, fr), srv.submit(pbs, fr[:2]), srv.submit(gbs, fr)]
    res = [srv.wait(i, 600000) for i in ids]
    srv.close()
    np.testing.assert_array_equal(res[0], alone_p)
    np.testing.assert_array_equal(res[1], alone_g)
    np.testing.assert_array_equal(res[2], alone_p[:2])
    np.testing.assert_array_equal(res[3], alone_g)


def test_system_outlives_server_after_growing_buffers(rst, small):
    # buffers a system allocates while a server runs its request belong to a
    # server slot stream; destroying the system after the server must be safe
    import gc

    s, fr, prm = small
    top = rst.read_prmtop(prm)
    for kw in (dict(pb_params=rst.PbParams(grid_spacing=0.6, grid_buffer=4.0)), {}):
        sysx = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, **kw)
        one = sysx.run(fr[:1])
        srv = rst.Server(max_inflight=2)
        rid = srv.submit(sysx, fr)  # three frames: per-batch buffers grow on the slot stream
        got = srv.wait(rid, 600000)
        srv.close()
        np.testing.assert_array_equal(got[:1], one)
        del sysx, srv
        gc.collect()
