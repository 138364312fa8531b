"""The oracle's converged PB solves (CPU only): three solvers of different
kind -- Jacobi-preconditioned CG, flexible CG with a consistent V-cycle,
and defect correction with that V-cycle (the GPU engine's relative-residual
iteration, here in FP64) -- reach the same solution of the same discrete
system, so the converged energy does not depend on the solver; and the
reference's own schedule, which stops on an absolute RMS residual, lands
close to it on a small grid where its V-cycles do converge."""
import numpy as np


def _system(tmp_path):
    from rust_simulation_tools import synthetic as S

    s = S.make_system(40, 6, seed=51)
    fr = S.make_frames(s, 1, seed=52)
    prm = str(tmp_path / "s.prmtop")
    S.write_prmtop(s, prm)
    return s, (fr[0].astype(np.float64) * 0.1) * 10.0, prm


def test_converged_solvers_agree(tmp_path, oracle):
    s, x, prm = _system(tmp_path)
    top = oracle.Topology.load(prm)
    base = dict(grid_spacing=0.6, grid_buffer=4.0, fillratio=0.0)
    e = {}
    for m in (0, 1, 2):
        e[m], d = oracle.pb_energy(top, x, oracle.pb_params(**base, converged_rel_tol=1e-11, converged_method=m))
        assert d["converged"] == [1, 1], (m, d)
        assert max(d["residual"]) < 1e-11
    assert abs(e[1] - e[0]) < 1e-8 * abs(e[0]) and abs(e[2] - e[0]) < 1e-8 * abs(e[0]), e
    ref, d = oracle.pb_energy(top, x, oracle.pb_params(**base))
    assert d["converged"] == [1, 1]
    assert abs(ref - e[0]) < 1e-4 * abs(e[0]), (ref, e[0])


def test_relative_stop_tightens_monotonically(tmp_path, oracle):
    s, x, prm = _system(tmp_path)
    top = oracle.Topology.load(prm)
    base = dict(grid_spacing=0.6, grid_buffer=4.0, fillratio=0.0, converged_method=2)
    exact, _ = oracle.pb_energy(top, x, oracle.pb_params(**base, converged_rel_tol=1e-12))
    errs, its = [], []
    for tol in (1e-4, 1e-6, 1e-8):
        e, d = oracle.pb_energy(top, x, oracle.pb_params(**base, converged_rel_tol=tol))
        errs.append(abs(e - exact))
        its.append(sum(d["iterations"]))
    assert errs[0] >= errs[1] >= errs[2] and its[0] <= its[1] <= its[2], (errs, its)
