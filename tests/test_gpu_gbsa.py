"""GPU parity of the MM-GBSA path against the CPU restatement.

Tolerances:
  * plain FP64 form vs the reference-faithful restatement: relative 1e-10 on
    every energy, 1e-12 on Born radii, per-atom SASA bit-identical;
  * fused mixed-precision form vs the accurate restatement: per-frame
    binding terms within 1e-3 kcal/mol, per-residue terms within 1e-4
    kcal/mol, sub-system totals within 1e-6 relative;
  * SASA binding differences come from identical accessible-point counts, so
    they agree to rounding (1e-9 kcal/mol).
"""
import math

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


@pytest.fixture(scope="module")
def sysdata(tmp_path_factory):
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("gb")
    s = S.make_system(300, 24, seed=21)
    fr = S.make_frames(s, 4, seed=22)
    S.write_prmtop(s, str(d / "s.prmtop"))
    S.write_dcd(fr, str(d / "s.dcd"))
    return s, fr, str(d / "s.prmtop"), str(d / "s.dcd")


def dcd_coords(fr):
    return (fr.astype(np.float64) * 0.1) * 10.0


def rel(a, b):
    return abs(a - b) / max(1.0, abs(b))


@pytest.mark.parametrize("model,salt,name", [(0, 0.15, "hct"), (1, 0.0, "obc1"), (2, 0.15, "obc2")])
def test_gb_plain_matches_restatement(rst, oracle, sysdata, model, salt, name):
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = dcd_coords(fr[0])
    g = rst.compute_gb_energy(top, x / 10.0, rst.GbParams(model=model, salt_concentration=salt))
    e, R = oracle.gb_energy(otop, (x / 10.0) * 10.0, oracle.gb_params(name, salt=salt))
    assert rel(g.total, e) < 1e-10
    np.testing.assert_allclose(g.born_radii(), R, rtol=1e-12)


def test_gb_cutoff_and_single_ion(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = dcd_coords(fr[1])
    g = rst.compute_gb_energy(top, x / 10.0, rst.GbParams(cutoff=8.0))
    e, _ = oracle.gb_energy(otop, (x / 10.0) * 10.0, oracle.gb_params(cutoff=8.0))
    assert rel(g.total, e) < 1e-10
    # gb_energy.rs:451-494 single ion on the GPU
    ion = rst.AmberTopology.from_arrays([18.2223], [1.5], screen=[0.8])
    g = rst.compute_gb_energy(ion, np.zeros((1, 3)), rst.GbParams(salt_concentration=0.0))
    assert abs(g.born_radii()[0] - 1.41) < 1e-10
    assert abs(g.total - (-0.5 * (1 - 1 / 78.3) * 18.2223 ** 2 / 1.41)) < 0.01


def test_mm_plain_matches_restatement(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = dcd_coords(fr[0])
    m = rst.compute_mm_energy(top, x / 10.0)
    ref = oracle.mm_energy(otop, (x / 10.0) * 10.0)
    for k, v in zip(("bond", "angle", "dihedral", "vdw", "elec", "vdw_14", "elec_14"), ref):
        assert rel(getattr(m, k), v) < 1e-10, k
    assert abs(m.total() - sum([m.bond, m.angle, m.dihedral, m.vdw, m.elec, m.vdw_14, m.elec_14])) < 1e-6


def test_sasa_plain_bit_identical(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = dcd_coords(fr[2])
    for npts in (480, 960):
        e = rst.compute_sa_energy(top, x / 10.0, rst.SaParams(n_sphere_points=npts))
        oe, ot, per = oracle.sa_energy(otop, (x / 10.0) * 10.0, oracle.sa_params(n_points=npts))
        np.testing.assert_array_equal(e.per_atom_sasa(), per)
        assert rel(e.total_sasa, ot) < 1e-12
        assert np.all(e.per_atom_sasa() >= 0) and abs(e.total_sasa - e.per_atom_sasa().sum()) < 1e-6


def test_bonded_known_answers_on_gpu(rst):
    # mm_energy.rs:316-365 through the GPU path
    t = rst.AmberTopology.from_arrays([0.0, 0.0], [1.5, 1.5], bonds=[(0, 1, 0)], bond_k=[300.0], bond_req=[1.5],
                                      num_excluded=[1, 0], excluded_list=[1], atom_type_indices=[0, 0])
    assert abs(rst.compute_mm_energy(t, np.array([[0, 0, 0], [0.2, 0, 0]])).bond - 75.0) < 1e-10
    t = rst.AmberTopology.from_arrays([0.0] * 3, [1.5] * 3, angles=[(0, 1, 2, 0)], angle_k=[50.0],
                                      angle_teq=[math.pi], num_excluded=[2, 1, 0], excluded_list=[1, 2, 2],
                                      atom_type_indices=[0] * 3)
    e = rst.compute_mm_energy(t, np.array([[0.1, 0, 0], [0, 0, 0], [0, 0.1, 0]]))
    assert abs(e.angle - 50.0 * (math.pi / 2) ** 2) < 1e-10


def test_binding_frame_plain_matches_restatement(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    gb = rst.GbParams(model=rst.GbModel.ObcII, solvent_dielectric=78.5)
    sa = rst.SaParams(n_sphere_points=960)
    x = dcd_coords(fr[0])
    f = rst.compute_binding_energy_single_frame(top, x / 10.0, s.receptor_residues, s.ligand_residues,
                                                gb_params=gb, sa_params=sa)
    ref = oracle.binding_frame(otop, (x / 10.0) * 10.0, s.receptor_residues, s.ligand_residues,
                               gb=oracle.gb_params("obc2", solvent_dielectric=78.5), sa=oracle.sa_params(n_points=960))
    for k in FRAME[:9]:
        assert rel(getattr(f, k), ref[k]) < 1e-10, k
    # binding.rs:401-404 identities
    assert abs(f.delta_gb - (f.complex_gb - f.receptor_gb - f.ligand_gb)) < 1e-4
    assert abs(f.delta_total - (f.delta_mm + f.delta_polar + f.delta_sa)) < 1e-4


def test_decompose_plain_matches_restatement(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    x = dcd_coords(fr[3])
    d = rst.decompose_binding_energy(top, x / 10.0, s.receptor_residues, s.ligand_residues,
                                     rst.GbParams(model=rst.GbModel.ObcII), rst.SaParams(n_sphere_points=960))
    ro, lo = oracle.decompose(otop, (x / 10.0) * 10.0, s.receptor_residues, s.ligand_residues,
                              oracle.gb_params("obc2"), oracle.sa_params(n_points=960))
    got = np.array([[r.vdw, r.elec, r.polar, r.sa] for r in d.receptor_residues + d.ligand_residues])
    ref = np.concatenate([ro, lo])
    np.testing.assert_allclose(got, ref, rtol=1e-9, atol=1e-9)
    r0 = d.receptor_residues[0]
    assert r0.residue_label == "RES" and abs(r0.total() - (r0.vdw + r0.elec + r0.gb + r0.sa)) < 1e-12


def fused_vs_accurate(rst, oracle, prm, s, fr, gb_name="obc2", eps=78.5, npts=960, salt=0.15, decompose=True,
                      **sys_kw):
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    gb = rst.GbParams(model={"hct": 0, "obc1": 1, "obc2": 2}[gb_name], solvent_dielectric=eps,
                      salt_concentration=salt)
    sa = rst.SaParams(n_sphere_points=npts)
    sysf = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb, sa_params=sa, **sys_kw)
    out, dec = sysf.run(fr, decompose=True)
    og = oracle.gb_params(gb_name, solvent_dielectric=eps, salt=salt)
    osa = oracle.sa_params(n_points=npts)
    for f in range(len(fr)):
        x = dcd_coords(fr[f])
        acc = oracle.binding_frame(otop, x, s.receptor_residues, s.ligand_residues, gb=og, sa=osa, accurate=True)
        for k in (9, 10, 11, 12):
            assert abs(out[f, k] - acc[FRAME[k]]) < 1e-3, (f, FRAME[k], out[f, k], acc[FRAME[k]])
        assert abs(out[f, 11] - acc["delta_sa"]) < 1e-9
        for k in range(9):
            assert rel(out[f, k], acc[FRAME[k]]) < 1e-6, (f, FRAME[k], out[f, k], acc[FRAME[k]])
        if decompose:
            ro, lo = oracle.decompose(otop, x, s.receptor_residues, s.ligand_residues, og, osa, accurate=True)
            np.testing.assert_allclose(dec[f], np.concatenate([ro, lo]), rtol=0, atol=1e-4)
    return out, sysf


def test_fused_matches_accurate_restatement(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    out, sysf = fused_vs_accurate(rst, oracle, prm, s, fr)
    st = sysf.last_stats()
    assert st["neighbour_overflow"] == 0 and st["launches"] > 0


@pytest.mark.parametrize("gb_name,salt", [("hct", 0.0), ("obc1", 0.15)])
def test_fused_other_models(rst, oracle, sysdata, gb_name, salt):
    s, fr, prm, _ = sysdata
    fused_vs_accurate(rst, oracle, prm, s, fr[:2], gb_name=gb_name, eps=78.3, npts=480, salt=salt,
                      decompose=False)


def test_fused_batches_and_graphs_agree(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top = rst.read_prmtop(prm)
    gb = rst.GbParams(model=rst.GbModel.ObcII)
    a = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb, batch_frames=3).run(fr)
    b = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb, batch_frames=1,
                          use_graphs=False).run(fr)
    c = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb).run(fr)
    np.testing.assert_array_equal(a, b)
    np.testing.assert_array_equal(a, c)


def test_plain_system_matches_single_frame(rst, oracle, sysdata):
    s, fr, prm, _ = sysdata
    top = rst.read_prmtop(prm)
    p = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, mode="plain").run(fr[:2])
    for f in range(2):
        e = rst.compute_binding_energy_single_frame(top, dcd_coords(fr[f]) / 10.0, s.receptor_residues,
                                                    s.ligand_residues)
        np.testing.assert_allclose(p[f], e.as_array(), rtol=1e-13, atol=1e-9)


def test_trajectory_api_dcd(rst, oracle, sysdata):
    s, fr, prm, dcd = sysdata
    top = rst.read_prmtop(prm)
    res = rst.compute_binding_energy(top, dcd, s.receptor_residues, s.ligand_residues, trajectory_format="dcd",
                                     stride=2, start_frame=1)
    assert len(res.frames) == 2  # frames 1 and 3
    direct = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues).run(fr[[1, 3]])
    got = np.array([f.as_array() for f in res.frames])
    np.testing.assert_array_equal(got, direct)
    d = got[:, 12]
    assert abs(res.mean_delta_total - d.mean()) < 1e-9
    assert abs(res.std_delta_total - d.std(ddof=1)) < 1e-9
    assert abs(res.sem_delta_total - d.std(ddof=1) / math.sqrt(2)) < 1e-9
    np.testing.assert_allclose(res.last_frame_coords(), dcd_coords(fr[3]))
    with pytest.raises(ValueError, match="No frames"):
        rst.compute_binding_energy(top, dcd, s.receptor_residues, s.ligand_residues, trajectory_format="dcd",
                                   start_frame=10)
    with pytest.raises(ValueError, match="out of range"):
        rst.compute_binding_energy(top, dcd, [0, 10 ** 6], s.ligand_residues, trajectory_format="dcd")


def test_bonded_exclusions_and_14_in_fused(rst, oracle):
    """A hand-built complex with bonds, angles, dihedrals (one spanning the
    receptor/ligand cut), exclusions and 1-4 pairs: fused vs accurate
    restatement and plain vs faithful restatement."""
    rng = np.random.default_rng(5)
    n = 40
    x = rng.uniform(-6, 6, size=(n, 3))
    x[30:] += np.array([9.0, 0, 0])
    q = rng.uniform(-0.5, 0.5, n) * 18.2223
    radii = rng.choice([1.2, 1.5, 1.7], n)
    screen = rng.choice([0.72, 0.85], n)
    types = rng.integers(0, 3, n)
    sig = np.array([1.8, 2.5, 3.2])
    eps = np.array([0.05, 0.1, 0.15])
    A, B, nbi = [], [], np.zeros(9, np.int64)
    for i in range(3):
        for j in range(i, 3):
            s_ = 0.5 * (sig[i] + sig[j])
            e_ = math.sqrt(eps[i] * eps[j])
            A.append(4 * e_ * s_ ** 12)
            B.append(4 * e_ * s_ ** 6)
            nbi[3 * i + j] = nbi[3 * j + i] = len(A)
    bonds = [(k, k + 1, 0) for k in range(0, 38)]
    angles = [(k, k + 1, k + 2, 0) for k in range(0, 36, 3)]
    # (27..30) and (28,29,31,32) put 1-4 pairs across the cut; (26,30,31,27)
    # makes (26,27) a 1-4 pair of the complex that the receptor alone excludes
    dih = [(k, k + 1, k + 2, k + 3, 0, 0) for k in range(0, 36, 4)] + [(27, 28, 29, 30, 0, 0), (28, 29, 31, 32, 0, 0),
                                                                        (26, 30, 31, 27, 0, 0)]
    excl_pairs = sorted({(min(a, b), max(a, b)) for a, b, _ in bonds} | {(a, c) for a, _, c, _ in angles} |
                        {(d[0], d[3]) for d in dih})
    num = np.zeros(n, np.int64)
    lst = []
    for i in range(n):
        js = [j for a, j in excl_pairs if a == i]
        if not js:
            js = [-1]
        num[i] = len(js)
        lst.extend(js)
    kw = dict(screen=screen, n_types=3, lj_acoef=A, lj_bcoef=B, nb_parm_index=nbi,
              residue_pointers=[0, 10, 20, 30], bonds=bonds, bond_k=[300.0], bond_req=[1.5], angles=angles,
              angle_k=[50.0], angle_teq=[1.9], dihedrals=dih, num_excluded=num, excluded_list=lst)
    top = rst.AmberTopology.from_arrays(q, radii, atom_type_indices=types, dihedral_pk=[1.2], dihedral_pn=[3.0],
                                        dihedral_phase=[0.0], **kw)
    otop = oracle.Topology.from_arrays(q, radii, type_idx=types, lj_a=A, lj_b=B, nb_index=nbi, dih_pk=[1.2],
                                       dih_pn=[3.0], dih_phase=[0.0],
                                       **{k: v for k, v in kw.items()
                                          if k not in ("n_types", "lj_acoef", "lj_bcoef", "nb_parm_index")},
                                       n_types=3)
    rec, lig = [0, 1, 2], [3]
    gb, og = rst.GbParams(model=rst.GbModel.ObcII), oracle.gb_params("obc2")
    sa, osa = rst.SaParams(n_sphere_points=480), oracle.sa_params(n_points=480)
    f = rst.compute_binding_energy_single_frame(top, x / 10.0, rec, lig, gb_params=gb, sa_params=sa)
    ref = oracle.binding_frame(otop, (x / 10.0) * 10.0, rec, lig, gb=og, sa=osa)
    for k in FRAME[:9]:
        assert rel(getattr(f, k), ref[k]) < 1e-10, k
    frames = np.stack([x, x + rng.normal(0, 0.05, x.shape)]).astype(np.float32)
    out = rst.BindingSystem(top, rec, lig, gb_params=gb, sa_params=sa).run(frames)
    for fi in range(2):
        acc = oracle.binding_frame(otop, dcd_coords(frames[fi]), rec, lig, gb=og, sa=osa, accurate=True)
        for k in range(9, 13):
            assert abs(out[fi, k] - acc[FRAME[k]]) < 1e-3, (fi, FRAME[k], out[fi, k], acc[FRAME[k]])
        for k in range(9):
            assert rel(out[fi, k], acc[FRAME[k]]) < 1e-6, (fi, FRAME[k])


def test_server_results_same_alone_and_in_mix(rst, sysdata):
    from rust_simulation_tools import synthetic as S

    s, fr, prm, _ = sysdata
    top = rst.read_prmtop(prm)
    s2 = S.make_system(150, 20, seed=31)
    fr2 = S.make_frames(s2, 5, seed=32)
    import tempfile, os
    d = tempfile.mkdtemp()
    S.write_prmtop(s2, os.path.join(d, "b.prmtop"))
    top2 = rst.read_prmtop(os.path.join(d, "b.prmtop"))
    A = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues)
    B = rst.BindingSystem(top2, s2.receptor_residues, s2.ligand_residues)
    alone_a, alone_b = A.run(fr), B.run(fr2)
    srv = rst.Server(max_inflight=3)
    ids = [srv.submit(A, fr), srv.submit(B, fr2), srv.submit(B, fr2[:2]), srv.submit(A, fr[1:3])]
    res = [srv.wait(i, 60000) for i in ids]
    np.testing.assert_array_equal(res[0], alone_a)
    np.testing.assert_array_equal(res[1], alone_b)
    np.testing.assert_array_equal(res[2], alone_b[:2])
    np.testing.assert_array_equal(res[3], alone_a[1:3])
    st = srv.stats()
    assert st["completed"] == 4 and st["p99_ms"] >= st["p50_ms"] > 0
    srv.close()


def test_server_evicts_idle_systems_under_budget(rst, sysdata):
    # a budget smaller than any request: requests run one at a time and each
    # admission evicts the idle system's resident buffers (and its captured
    # graph); re-admitted systems rebuild them and give the same bits
    from rust_simulation_tools import synthetic as S
    import tempfile, os

    s, fr, prm, _ = sysdata
    top = rst.read_prmtop(prm)
    s2 = S.make_system(150, 20, seed=33)
    fr2 = S.make_frames(s2, 4, seed=34)
    d = tempfile.mkdtemp()
    S.write_prmtop(s2, os.path.join(d, "c.prmtop"))
    top2 = rst.read_prmtop(os.path.join(d, "c.prmtop"))
    A = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues)
    B = rst.BindingSystem(top2, s2.receptor_residues, s2.ligand_residues)
    alone_a, alone_b = A.run(fr), B.run(fr2)
    srv = rst.Server(memory_budget_bytes=1, max_inflight=2)
    ids = [srv.submit(A, fr), srv.submit(B, fr2), srv.submit(A, fr), srv.submit(B, fr2[1:])]
    res = [srv.wait(i, 60000) for i in ids]
    st = srv.stats()
    srv.close()
    np.testing.assert_array_equal(res[0], alone_a)
    np.testing.assert_array_equal(res[1], alone_b)
    np.testing.assert_array_equal(res[2], alone_a)
    np.testing.assert_array_equal(res[3], alone_b[1:])
    assert st["completed"] == 4


def test_gb_cache_reuses_radii(rst, oracle, sysdata):
    # gb_energy.rs:66-120,372-387: first call computes and caches the radii;
    # a frame within the RMSD threshold reuses them (energy from the cached
    # radii at the new coordinates); a frame beyond it recomputes.
    s, fr, prm, _ = sysdata
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    gp = rst.GbParams(model=2)
    og = oracle.gb_params("obc2")
    x0 = dcd_coords(fr[0])
    cache = rst.GbCache(0.5)
    a = rst.compute_gb_energy_cached(top, x0 / 10.0, gp, cache)
    assert not cache.last_reused
    b = rst.compute_gb_energy(top, x0 / 10.0, gp)
    assert a.total == b.total
    np.testing.assert_array_equal(a.born_radii(), b.born_radii())
    x1 = x0 + 0.05  # RMSD 0.087 A
    c = rst.compute_gb_energy_cached(top, x1 / 10.0, gp, cache)
    assert cache.last_reused
    np.testing.assert_array_equal(c.born_radii(), a.born_radii())
    ref = oracle.gb_energy_from_radii(otop, (x1 / 10.0) * 10.0, og, a.born_radii())
    assert rel(c.total, ref) < 1e-10
    x2 = dcd_coords(fr[1])  # sigma 0.5 A noise per coordinate: RMSD ~1.2 A
    d = rst.compute_gb_energy_cached(top, x2 / 10.0, gp, cache)
    assert not cache.last_reused
    assert d.total == rst.compute_gb_energy(top, x2 / 10.0, gp).total


def test_sharded_frames_equal_single_process(rst, sysdata):
    """Frames split over three emulated ranks (each evaluated on this GPU) and
    merged on the host equal one pass over all frames."""
    from rust_simulation_tools import sharding as SH

    s, fr, prm, _ = sysdata
    top = rst.read_prmtop(prm)
    sysf = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues)
    world = 3
    blocks = []
    for r in range(world):
        a, b = SH.frame_range(fr.shape[0], r, world)
        blocks.append(sysf.run(fr[a:b]) if b > a else np.zeros((0, 13)))
    rows = SH.gather_rows(blocks[1], fr.shape[0], 1, world, lambda obj: blocks)
    np.testing.assert_array_equal(rows, sysf.run(fr))
    st = SH.statistics(rows)
    d = rows[:, 12]
    assert abs(st["mean_delta_total"] - d.mean()) < 1e-9 and abs(st["std_delta_total"] - d.std(ddof=1)) < 1e-9


@pytest.fixture(scope="module")
def w2(tmp_path_factory):
    from rust_simulation_tools import synthetic as S

    d = tmp_path_factory.mktemp("w2")
    s, fr = S.workload(2, n_frames=3)
    S.write_prmtop(s, str(d / "w2.prmtop"))
    return s, fr, str(d / "w2.prmtop")


def test_fused_binding_terms_at_workload_size(rst, oracle, w2):
    # 5,050 atoms (12.7 M pairs per frame): the binding GB difference is
    # formed from per-pair differences, so it stays far inside 1e-3 kcal/mol
    # of the FP64 form (guard 1e-4); delta_mm against the accurate restatement
    s, fr, prm = w2
    top, otop = rst.read_prmtop(prm), oracle.Topology.load(prm)
    kw = dict(gb_params=rst.GbParams(model=2, solvent_dielectric=78.5), sa_params=rst.SaParams(n_sphere_points=960))
    fused = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, **kw).run(fr)
    plain = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, mode="plain", **kw).run(fr)
    assert np.abs(fused[:, 10] - plain[:, 10]).max() < 1e-4
    assert np.abs(fused[:, 11] - plain[:, 11]).max() < 1e-9
    acc = oracle.binding_frame(otop, dcd_coords(fr[0]), s.receptor_residues, s.ligand_residues,
                               gb=oracle.gb_params("obc2", solvent_dielectric=78.5),
                               sa=oracle.sa_params(n_points=960), accurate=True)
    assert abs(fused[0, 9] - acc["delta_mm"]) < 1e-3
    assert abs(fused[0, 10] - acc["delta_polar"]) < 1e-3
