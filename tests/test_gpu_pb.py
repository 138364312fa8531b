"""GPU parity of the Poisson-Boltzmann path against the CPU restatement.

Grid set-up maps are compared point by point: charge density, SES inside
flags, face dielectrics and kappa-bar^2 bit for bit, the Debye-Hueckel
boundary potential to 1e-12 relative (its exp() comes from a different
math library).  Energies of converged solves agree to 1e-8 relative: the
V-cycle arithmetic is the reference's, so the GPU and CPU potentials differ
only through those boundary values and reduction order.
"""
import math

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
def pbsys(tmp_path_factory):
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("pb")
    s = S.make_system(40, 6, seed=51)
    fr = S.make_frames(s, 2, seed=52)
    S.write_prmtop(s, str(d / "s.prmtop"))
    return s, fr, str(d / "s.prmtop")


def gpu_maps(rst, x, q, r, params, ein, eout, ionic):
    import ctypes as C

    from rust_simulation_tools import _native as N

    x = np.ascontiguousarray(x, dtype=np.float64)
    q = np.ascontiguousarray(q, dtype=np.float64)
    r = np.ascontiguousarray(r, dtype=np.float64)
    dims = np.zeros(3, np.int64)
    org = np.zeros(3)
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int64))
    args = (N.ctx(), dp(x), len(q), dp(q), dp(r), C.byref(params._c), ein, eout, int(ionic), ip(dims), dp(org))
    N.check(N.lib.rstg_pb_grid_maps(*args, None, None, None, None, None, None, None))
    n = int(np.prod(dims))
    m = {k: np.zeros(n) for k in ("charge", "ex", "ey", "ez", "k2", "boundary")}
    inside = np.zeros(n, np.uint8)
    N.check(N.lib.rstg_pb_grid_maps(*args, dp(m["charge"]), inside.ctypes.data_as(C.POINTER(C.c_uint8)), dp(m["ex"]),
                                    dp(m["ey"]), dp(m["ez"]), dp(m["k2"]), dp(m["boundary"])))
    m["inside"], m["dims"], m["origin"] = inside, dims, org
    return m


@pytest.mark.parametrize("probe,ionic", [(1.4, True), (1.4, False), (0.0, True)])
def test_pb_maps_match_restatement(rst, oracle, pbsys, probe, ionic):
    s, fr, prm = pbsys
    x = (fr[0].astype(np.float64) * 0.1) * 10.0
    q, r = s.charges_e, s.radii
    params = rst.PbParams(grid_spacing=0.6, grid_buffer=4.0, probe_radius=probe)
    kap = oracle.kappa(0.15, 80.0, 300.0)
    eout = 80.0 if ionic else 1.0
    g = gpu_maps(rst, x, q, r, params, 1.0, eout, ionic)
    o = oracle.pb_maps(x, q, r, 0.6, 4.0, probe, 2.0, 1.0, eout, kap, 80.0, ionic)
    np.testing.assert_array_equal(g["dims"], o["dims"])
    np.testing.assert_array_equal(g["origin"], o["origin"])
    np.testing.assert_array_equal(g["charge"], o["charge"])
    if eout != 1.0:
        np.testing.assert_array_equal(g["inside"], o["inside"])
    for k in ("ex", "ey", "ez", "k2"):
        np.testing.assert_array_equal(g[k], o[k])
    np.testing.assert_allclose(g["boundary"], o["boundary"], rtol=1e-12, atol=1e-300)


@pytest.mark.parametrize("fillratio", [0.0, 4.0])
def test_pb_energy_matches_restatement(rst, oracle, pbsys, fillratio):
    s, fr, prm = pbsys
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = (fr[1].astype(np.float64) * 0.1) * 10.0
    p = rst.PbParams(grid_spacing=0.6, grid_buffer=4.0, fillratio=fillratio)
    e = rst.compute_pb_energy(top, x / 10.0, p)
    ref, diag = oracle.pb_energy(otop, (x / 10.0) * 10.0,
                                 oracle.pb_params(grid_spacing=0.6, grid_buffer=4.0, fillratio=fillratio))
    assert abs(e.total - ref) <= 1e-8 * abs(ref), (e.total, ref)
    assert e.diag["dims"] == diag["dims"]
    assert e.diag["iterations"] == diag["iterations"]
    assert all(e.diag["converged"])


def test_pb_born_ion_known_answer(rst):
    # pb_energy.rs:529-570: within 15 % of -0.5 (1 - 1/80) 332.0522 / 2
    ion = rst.AmberTopology.from_arrays([18.2223], [2.0], screen=[0.8])
    p = rst.PbParams(grid_spacing=0.25, grid_buffer=15.0, solute_dielectric=1.0, solvent_dielectric=80.0,
                     salt_concentration=0.0, probe_radius=0.0, ion_radius=0.0, tolerance=1e-8, max_iterations=20000)
    e = rst.compute_pb_energy(ion, np.zeros((1, 3)), p)
    ana = -0.5 * (1.0 - 1.0 / 80.0) * 332.0522 / 2.0
    assert abs((e.total - ana) / ana) < 0.15


def test_pb_small_grid_uses_plain_sor(rst, oracle):
    # min grid dimension <= 8: Chebyshev SOR (pb_solver.rs:1044-1059)
    x = np.array([[0.0, 0.0, 0.0], [1.2, 0.3, -0.4]])
    q, r = [0.5, -0.3], [1.7, 1.5]
    top = rst.AmberTopology.from_arrays(np.array(q) * 18.2223, r, screen=[0.8, 0.8])
    p = rst.PbParams(grid_spacing=1.0, grid_buffer=2.0, fillratio=0.0, tolerance=1e-8)
    e = rst.compute_pb_energy(top, x / 10.0, p)
    ref = oracle.pb_energy_raw(x, q, r, oracle.pb_params(grid_spacing=1.0, grid_buffer=2.0, fillratio=0.0,
                                                         tolerance=1e-8))
    assert max(e.diag["dims"]) <= 8
    assert abs(e.total - ref) <= 1e-8 * abs(ref)


def test_pb_solute_residues_strips(rst, pbsys):
    s, fr, prm = pbsys
    top = rst.read_prmtop(prm)
    x = (fr[0].astype(np.float64) * 0.1) * 10.0
    p = rst.PbParams(grid_spacing=0.7, grid_buffer=4.0, fillratio=0.0)
    rec = s.receptor_residues
    whole = rst.compute_pb_energy(rst.extract_subtopology(top, top.get_atom_indices(rec)),
                                  x[top.get_atom_indices(rec)] / 10.0, p)
    stripped = rst.compute_pb_energy(top, x / 10.0, p, solute_residues=rec)
    assert whole.total == stripped.total


def test_pb_binding_frame_matches_restatement(rst, oracle, pbsys):
    s, fr, prm = pbsys
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = (fr[0].astype(np.float64) * 0.1) * 10.0
    p = rst.PbParams(grid_spacing=0.7, grid_buffer=4.0, fillratio=0.0)
    f = rst.compute_binding_energy_single_frame(top, x / 10.0, s.receptor_residues, s.ligand_residues, pb_params=p)
    ref = oracle.binding_frame(otop, (x / 10.0) * 10.0, s.receptor_residues, s.ligand_residues,
                               pb=oracle.pb_params(grid_spacing=0.7, grid_buffer=4.0, fillratio=0.0))
    for k in ("complex_polar", "receptor_polar", "ligand_polar"):
        assert abs(getattr(f, k) - ref[k]) <= 1e-8 * abs(ref[k]), k
    assert abs(f.delta_polar - (f.complex_polar - f.receptor_polar - f.ligand_polar)) < 1e-9
