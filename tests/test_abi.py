"""CPU-side checks of the C-ABI library: it loads, exports every symbol that
include/rstg.h declares, and its host-only functions (prmtop parsing,
sub-topology extraction, trajectory readers, selections) agree with the CPU
restatement.  No compute call runs here."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "rstg.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(rstg_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import rust_simulation_tools._native as N

    names = declared_symbols()
    assert len(names) > 40
    missing = [n for n in names if not hasattr(N.lib, n)]
    assert not missing, missing


def test_library_is_sm100a_build():
    import rust_simulation_tools._native as N

    assert b"sm_100a" in N.lib.rstg_version()


def test_prmtop_parse_matches_oracle(oracle, small_system):
    import rust_simulation_tools as rst

    s, fr, prm, dcd = small_system
    top = rst.read_prmtop(prm)
    ref = oracle.Topology.load(prm).arrays()
    assert top.n_atoms == s.n_atoms and top.n_residues == len(s.residue_labels)
    np.testing.assert_array_equal(top.charges(), ref["charges"])
    np.testing.assert_array_equal(top.radii(), ref["radii"])
    np.testing.assert_array_equal(top.residue_pointers(), ref["residue_pointers"])
    assert top.residue_labels[-1] == "LIG"


def test_dcd_reader_matches_oracle(oracle, small_system):
    import rust_simulation_tools as rst

    s, fr, prm, dcd = small_system
    r = rst.DcdReader(dcd)
    assert (r.n_frames, r.n_atoms) == fr.shape[:2]
    a, _ = r.read_all()
    np.testing.assert_array_equal(a, oracle.read_dcd_nm(dcd))
    np.testing.assert_array_equal(r.read_all_f32_angstrom(), fr)
    f0, box = r.read_frame()
    assert box is None and f0.shape == (s.n_atoms, 3)


def test_mdcrd_reader(tmp_path):
    import rust_simulation_tools as rst

    x = np.round(np.random.default_rng(0).uniform(-50, 50, size=(2, 5, 3)), 3)
    p = tmp_path / "t.mdcrd"
    with open(p, "w") as f:
        f.write("title\n")
        for fr in x:
            vals = fr.reshape(-1)
            for s in range(0, len(vals), 10):
                f.write("".join("%8.3f" % v for v in vals[s:s + 10]) + "\n")
    r = rst.MdcrdReader(str(p), 5, False)
    np.testing.assert_allclose(r.read_frame(), x[0])
    np.testing.assert_allclose(r.read_frame(), x[1])
    assert r.read_frame() is None


def test_errors_map_to_reference_exceptions(small_system):
    import rust_simulation_tools as rst

    with pytest.raises(IOError):
        rst.read_prmtop("/nonexistent/file.prmtop")
    s, fr, prm, dcd = small_system
    top = rst.read_prmtop(prm)
    with pytest.raises(ValueError, match="out of range"):
        top.get_atom_indices([10 ** 6])
    with pytest.raises(IOError):
        rst.DcdReader(prm)


def test_extract_subtopology_and_selection(small_system):
    import rust_simulation_tools as rst

    s, fr, prm, dcd = small_system
    top = rst.read_prmtop(prm)
    sel = top.build_selection([0, 2])
    assert list(sel["residue_offsets"]) == [0, 15, 30]
    sub = rst.extract_subtopology(top, sel["atom_indices"])
    assert sub.n_atoms == 30 and sub.n_residues == 2
    np.testing.assert_array_equal(sub.charges(), top.charges()[sel["atom_indices"]])


def test_params_defaults():
    import rust_simulation_tools as rst

    g = rst.GbParams()
    assert g.model == rst.GbModel.ObcI and g.solvent_dielectric == 78.3 and g.salt_concentration == 0.15
    assert rst.SaParams().n_sphere_points == 480
    p = rst.PbParams()
    assert p.grid_spacing == 0.5 and p.solvent_dielectric == 80.0


def test_interaction_entropy_host():
    import rust_simulation_tools as rst

    class F:
        def __init__(self, v):
            self.delta_mm = v

    assert rst.interaction_entropy([F(1.0)]) is None
    e = rst.interaction_entropy([F(-10.0), F(-12.0), F(-11.0)], 298.15)
    kt = 0.00198688 * 298.15
    x = np.array([1.0, -1.0, 0.0]) / kt
    assert abs(e.minus_tds - kt * np.log(np.exp(x).mean())) < 1e-12


def test_compute_without_gpu_raises(small_system):
    import rust_simulation_tools as rst

    if rst.device_count() > 0:
        pytest.skip("a GPU is present")
    s, fr, prm, dcd = small_system
    top = rst.read_prmtop(prm)
    with pytest.raises(Exception):
        rst.compute_gb_energy(top, fr[0] / 10.0)


def test_rust_binding_declares_every_entry_point():
    """The Rust binding a crate maintainer drops in declares every function
    of include/rstg.h, and each #[repr(C)] struct has the header's fields in
    the header's order."""
    import re

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    h = open(os.path.join(root, "include", "rstg.h")).read()
    r = open(os.path.join(root, "rust-simulation-tools_b200", "bindings", "rstg_sys.rs")).read()
    names = set(re.findall(r"\b(rstg_[a-z0-9_]+)\s*\(", h))
    assert names and all(("fn " + n + "(") in r for n in names), sorted(n for n in names if ("fn " + n + "(") not in r)
    for st in ("rstg_gb_params", "rstg_pb_params", "rstg_frame_energy", "rstg_topology_desc", "rstg_system_opts",
               "rstg_server_opts", "rstg_pb_diag"):
        body = re.search(r"typedef struct " + st + r" \{(.*?)\} " + st + ";", h, re.S).group(1)
        body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
        fields = []
        for decl in body.split(";"):
            decl = decl.strip()
            if not decl:
                continue
            for part in decl.split(","):
                nm = re.findall(r"([A-Za-z_][A-Za-z0-9_]*)\s*(?:\[[^\]]*\])?\s*$", part.strip())
                if nm:
                    fields.append(nm[0])
        rs = re.search(r"pub struct " + st + r" \{(.*?)\n\}", r, re.S).group(1)
        assert re.findall(r"pub ([a-z_0-9]+):", rs) == fields, st
