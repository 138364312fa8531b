"""Pins the CPU restatement against every known-answer test the reference
holds for this path (crates/mmpbsa/src/*.rs #[cfg(test)] modules,
crates/core/src/sasa.rs tests, tests/test_sasa.py) plus the reference's own
consistency identities (tests/test_mmpbsa.py)."""
import math

import numpy as np
import pytest


def test_kappa_known_answer(oracle):
    # gb_energy.rs:394-402: kappa(0.15 M, 78.3, 300 K) = 0.127315 +- 0.001
    assert abs(oracle.kappa(0.15, 78.3, 300.0) - 0.127315) < 0.001
    # gb_energy.rs:405-408
    assert oracle.kappa(0.0, 78.3, 300.0) == 0.0
    assert oracle.kappa(-1.0, 78.3, 300.0) == 0.0


def test_single_ion_gb(oracle):
    # gb_energy.rs:451-494
    t = oracle.Topology.from_arrays([18.2223], [1.5], screen=[0.8])
    e, R = oracle.gb_energy(t, np.zeros((1, 3)), oracle.gb_params("obc1", salt=0.0, offset=0.09))
    rho = 1.5 - 0.09
    assert abs(R[0] - rho) < 1e-10
    assert abs(e - (-0.5 * (1.0 - 1.0 / 78.3) * 18.2223 ** 2 / rho)) < 0.01


def test_bond_energy(oracle):
    # mm_energy.rs:316-340
    t = oracle.Topology.from_arrays([0.0, 0.0], [1.5, 1.5], bonds=[(0, 1, 0)], bond_k=[300.0], bond_req=[1.5],
                                    num_excluded=[1, 0], excluded_list=[1], type_idx=[0, 0], nb_index=[1])
    e = oracle.mm_energy(t, np.array([[0.0, 0.0, 0.0], [2.0, 0.0, 0.0]]))
    assert abs(e[0] - 75.0) < 1e-10


def test_angle_energy(oracle):
    # mm_energy.rs:342-365
    t = oracle.Topology.from_arrays([0.0] * 3, [1.5] * 3, angles=[(0, 1, 2, 0)], angle_k=[50.0],
                                    angle_teq=[math.pi], num_excluded=[2, 1, 0], excluded_list=[1, 2, 2],
                                    type_idx=[0, 0, 0], nb_index=[1])
    e = oracle.mm_energy(t, np.array([[1.0, 0.0, 0.0], [0.0, 0.0, 0.0], [0.0, 1.0, 0.0]]))
    assert abs(e[1] - 50.0 * (math.pi / 2) ** 2) < 1e-10


def test_dihedral_energy_range(oracle):
    # mm_energy.rs:367-399
    t = oracle.Topology.from_arrays([0.0] * 4, [1.5] * 4, dihedrals=[(0, 1, 2, 3, 0, 0)], dih_pk=[2.0],
                                    dih_pn=[2.0], dih_phase=[math.pi], num_excluded=[3, 2, 1, 0],
                                    excluded_list=[1, 2, 3, 2, 3, 3], type_idx=[0] * 4, nb_index=[1])
    e = oracle.mm_energy(t, np.array([[1.0, 1.0, 0.0], [0, 0, 0], [1.0, 0, 0], [2.0, 1.0, 0]], dtype=float))
    assert 0.0 <= e[2] < 10.0


def test_single_atom_sasa(oracle):
    # sa_energy.rs:82-141 (2 %) and sasa.rs:386-397 (5 % at 1000 points)
    t = oracle.Topology.from_arrays([0.0], [1.7], screen=[0.72])
    e, tot, per = oracle.sa_energy(t, np.zeros((1, 3)), oracle.sa_params())
    exp = 4.0 * math.pi * 3.1 ** 2
    assert abs(tot - exp) / exp < 0.02
    assert abs(e - 0.0072 * exp) < 0.1
    s = oracle.sasa_raw(np.zeros((1, 3)), [1.5], 1.4, 1000)
    assert abs(s[0] - 4 * math.pi * 2.9 ** 2) / (4 * math.pi * 2.9 ** 2) < 0.05


def test_sasa_python_suite_cases(oracle):
    # tests/test_sasa.py: distant atoms, occlusion, buried centre, probe monotonicity
    single = 4 * np.pi * 3.1 ** 2
    far = oracle.sasa_raw(np.array([[0, 0, 0], [100.0, 0, 0]]), [1.7, 1.7], 1.4, 960)
    assert abs(far.sum() - 2 * single) / (2 * single) < 0.05
    close = oracle.sasa_raw(np.array([[0, 0, 0], [3.0, 0, 0]]), [1.7, 1.7], 1.4, 960)
    assert close.sum() < 2 * single * 0.95
    c = np.array([[0, 0, 0], [3.5, 0, 0], [-3.5, 0, 0], [0, 3.5, 0], [0, -3.5, 0], [0, 0, 3.5], [0, 0, -3.5]])
    b = oracle.sasa_raw(c.astype(float), [1.7] * 7, 1.4, 960)
    assert b[0] < b[1:].mean()
    vals = [oracle.sasa_raw(np.zeros((1, 3)), [1.5], p, 960)[0] for p in (0.0, 1.0, 1.4, 2.0)]
    assert all(vals[i] < vals[i + 1] for i in range(3))


def test_fibonacci_unit_norm(oracle):
    # sasa.rs:411-425
    p = oracle.fibonacci(100)
    assert p.shape == (100, 3)
    assert np.all(np.abs(np.linalg.norm(p, axis=1) - 1.0) < 1e-10)


def test_charge_conservation(oracle):
    # pb_grid.rs:1013-1025
    assert abs(oracle.charge_total(np.array([[5.0, 5.0, 5.0]]), [1.0], 1.0, 5.0) - 1.0) < 1e-10


def test_restrict_prolong_constant(oracle):
    # pb_solver.rs:1260-1283
    c, f = oracle.restrict_prolong_constant(3.0)
    assert np.all(np.abs(c - 3.0) < 1e-12)
    assert np.all(np.abs(f - 3.0) < 0.5)


def test_born_ion_pb(oracle):
    # pb_energy.rs:529-570: within 15 % of -0.5 (1 - 1/80) 332.0522 / 2
    p = oracle.pb_params(grid_spacing=0.25, grid_buffer=15.0, solute_dielectric=1.0, solvent_dielectric=80.0,
                         salt=0.0, probe=0.0, ion_radius=0.0, tolerance=1e-8, max_iterations=20000)
    e = oracle.pb_energy_raw(np.zeros((1, 3)), [1.0], [2.0], p)
    ana = -0.5 * (1.0 - 1.0 / 80.0) * 332.0522 / 2.0
    assert abs((e - ana) / ana) < 0.15


def test_binding_identities(oracle, small_system):
    # tests/test_mmpbsa.py:220-279: delta = C - R - L and total = sum of terms
    s, fr, prm, _ = small_system
    top = oracle.Topology.load(prm)
    f = oracle.binding_frame(top, fr[0].astype(float), s.receptor_residues, s.ligand_residues)
    for k in ("mm", "polar", "sa"):
        assert abs(f["delta_" + k] - (f["complex_" + k] - f["receptor_" + k] - f["ligand_" + k])) < 1e-4
    assert abs(f["delta_total"] - (f["delta_mm"] + f["delta_polar"] + f["delta_sa"])) < 1e-4


def test_decomposition_sums_to_exact_delta(oracle, small_system):
    # per-residue terms add up to the exact binding difference (no bonded terms)
    s, fr, prm, _ = small_system
    top = oracle.Topology.load(prm)
    x = fr[1].astype(float)
    gb = oracle.gb_params("obc2", solvent_dielectric=78.5)
    sa = oracle.sa_params(n_points=960)
    ro, lo = oracle.decompose(top, x, s.receptor_residues, s.ligand_residues, gb, sa, accurate=True)
    f = oracle.binding_frame(top, x, s.receptor_residues, s.ligand_residues, gb=gb, sa=sa, accurate=True)
    assert abs(ro.sum() + lo.sum() - f["delta_total"]) < 1e-6


def test_prmtop_dcd_roundtrip(oracle, small_system):
    s, fr, prm, dcd = small_system
    top = oracle.Topology.load(prm)
    assert top.n_atoms == s.n_atoms and top.n_residues == len(s.residue_labels)
    a = top.arrays()
    np.testing.assert_allclose(a["charges_amber"], s.charges_e * 18.2223, rtol=1e-7)
    np.testing.assert_array_equal(a["type_idx"], s.type_idx)
    nm = oracle.read_dcd_nm(dcd)
    assert nm.shape == fr.shape
    np.testing.assert_allclose(nm * 10.0, fr, atol=1e-5)


def test_reimage_known_answer():
    """reimage_complex (binding.rs:234-308) by hand: a three-atom chain torn
    across the x faces of a 10 A cell is unwrapped along its bonds from atom
    0, and a lone atom whose centre sits more than half a cell from the
    chain's centre moves by one cell edge towards it."""
    import oracle as O

    x = [[9.5, 5.0, 5.0], [0.25, 5.0, 5.0], [1.0, 5.0, 5.0], [0.5, 5.0, 9.75]]
    out = O.reimage_complex(x, [(0, 1), (1, 2)], [10.0, 10.0, 10.0])
    # 0.25 - 9.5 < -5: +10; 1.0 - 10.25 < -5: +10; centre (9.5 + 10.25 + 11) / 3
    # = 10.25 vs 0.5 on x: +10; z: 9.75 - 5 < 5 stays
    want = [[9.5, 5.0, 5.0], [10.25, 5.0, 5.0], [11.0, 5.0, 5.0], [10.5, 5.0, 9.75]]
    assert out.tolist() == want
    # a component found later keeps its own start; no bonds, one atom: unchanged
    assert O.reimage_complex([[3.0, 4.0, 5.0]], [], [10.0, 10.0, 10.0]).tolist() == [[3.0, 4.0, 5.0]]
