"""Periodic reimaging of a boxed trajectory (reimage_complex,
binding.rs:234-308): a DCD whose frames carry a unit cell and whose complex
is wrapped into the primary cell -- molecules split across the cell faces --
gives, after the reference's bond-graph unwrap and minimum-image shift of
every component towards the first, the same complex as the intact frames up
to one lattice translation, and the same energies to rounding.  Bonds of
zero force constant chain each receptor residue and the ligand (they add no
energy and no exclusion: they only connect the molecules)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

L = 64.0  # cubic cell edge, A


@pytest.fixture(scope="module")
def rst():
    import rust_simulation_tools as r

    if r.device_count() < 1:
        pytest.skip("no CUDA device")
    return r


def test_wrapped_boxed_trajectory_reimages_to_intact(rst, tmp_path):
    from rust_simulation_tools import synthetic as S

    s = S.make_system(300, 24, seed=61)
    ptr = list(s.residue_pointers) + [s.n_atoms]
    bonds = [(a, a + 1) for r in range(len(ptr) - 1) for a in range(ptr[r], ptr[r + 1] - 1)]
    prm = str(tmp_path / "box.prmtop")
    S.write_prmtop(s, prm, bonds=bonds)
    # coordinates on a 1/256 A lattice, so float32 wrapping by L is exact
    fr = np.round(S.make_frames(s, 3, seed=62).astype(np.float64) * 256.0) / 256.0
    fr += np.array([-21.0, 7.5, 30.25])  # straddle the cell faces at 0
    wrapped = fr - L * np.floor(fr / L)
    assert (wrapped.max(axis=1) - wrapped.min(axis=1)).max() > L / 2  # split across the cell
    S.write_dcd(fr.astype(np.float32), str(tmp_path / "intact.dcd"))
    S.write_dcd(wrapped.astype(np.float32), str(tmp_path / "wrapped.dcd"), cell=(L, L, L, 90.0, 90.0, 90.0))
    S.write_dcd(wrapped.astype(np.float32), str(tmp_path / "torn.dcd"))  # same frames, no cell
    top = rst.read_prmtop(prm)
    gb = rst.GbParams(model=rst.GbModel.ObcII, solvent_dielectric=78.5)
    sa = rst.SaParams(n_sphere_points=480)
    kw = dict(gb_params=gb, sa_params=sa, trajectory_format="dcd")
    for mode in ("plain", "fused"):
        a = rst.compute_binding_energy(top, str(tmp_path / "intact.dcd"), s.receptor_residues, s.ligand_residues,
                                       mode=mode, **kw)
        b = rst.compute_binding_energy(top, str(tmp_path / "wrapped.dcd"), s.receptor_residues,
                                       s.ligand_residues, mode=mode, **kw)
        ea = np.array([f.as_array() for f in a.frames])
        eb = np.array([f.as_array() for f in b.frames])
        scale = np.maximum(np.abs(ea[:, :9]).max(axis=1, keepdims=True), 1.0)
        np.testing.assert_allclose(eb[:, :9], ea[:, :9], rtol=1e-9, atol=0)
        assert np.all(np.abs(eb[:, 9:] - ea[:, 9:]) <= 1e-9 * scale), (eb[:, 9:] - ea[:, 9:])
        # the last frame's reimaged complex is the intact one moved by one lattice vector
        shift = b.last_frame_coords() - a.last_frame_coords()
        k = np.round(shift[0] / L)
        np.testing.assert_allclose(shift, np.broadcast_to(k * L, shift.shape), rtol=0, atol=1e-9)
    # without the cell nothing is reimaged: the torn complex has other energies
    c = rst.compute_binding_energy(top, str(tmp_path / "torn.dcd"), s.receptor_residues, s.ligand_residues,
                                   mode="plain", **kw)
    ec = np.array([f.as_array() for f in c.frames])
    assert np.abs(ec[:, 10] - ea[:, 10]).max() > 1e-3


def test_device_reimage_matches_host_and_oracle(rst, tmp_path):
    """The device form (one block per frame, the walk's levels in order) and
    the host form of reimage_complex give the bits of the restatement
    (oracle.reimage_complex) on wrapped frames with per-frame cells: a
    150-atom bonded chain (walk depth 149), several components, the
    ligand a component of its own."""
    import oracle as O
    from rust_simulation_tools import synthetic as S

    s = S.make_system(300, 24, seed=71)
    ptr = list(s.residue_pointers) + [s.n_atoms]
    bonds = [(a, a + 1) for r in range(len(ptr) - 1) for a in range(ptr[r], ptr[r + 1] - 1)]
    nres_rec = len(s.receptor_residues)
    bonds += [(ptr[r + 1] - 1, ptr[r + 1]) for r in range(nres_rec // 2)]  # chain the first half of the receptor
    prm = str(tmp_path / "chain.prmtop")
    S.write_prmtop(s, prm, bonds=bonds)
    top = rst.read_prmtop(prm)
    bs = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues,
                           gb_params=rst.GbParams(model=rst.GbModel.ObcII), sa_params=rst.SaParams(n_sphere_points=120))
    rng = np.random.default_rng(72)
    fr = S.make_frames(s, 5, seed=73).astype(np.float64) + rng.uniform(-30, 30, size=(5, 1, 3))
    boxes = rng.uniform(38.0, 70.0, size=(5, 3))
    wrapped = fr - boxes[:, None, :] * np.floor(fr / boxes[:, None, :])
    dev = bs.reimage(wrapped, boxes, on_device=True)
    host = bs.reimage(wrapped, boxes, on_device=False)
    assert np.array_equal(dev, host)
    for f in range(5):
        want = O.reimage_complex(wrapped[f], bonds, boxes[f])
        assert np.array_equal(host[f], want), f
    assert not np.array_equal(dev, wrapped)  # the frames were torn and have been mended
    twice = bs.reimage(dev, boxes, on_device=True)  # a mended frame stays as it is
    assert np.array_equal(twice, dev)
