"""Writes the golden fixtures of the benchmark configurations (CPU only).

The fixtures pin the GPU engines at the sizes they are measured on: each
holds the CPU restatement's results (oracle/, a C++ FP64 restatement of the
reference path) for frames of the seeded synthetic workloads, plus SHA-256
digests of the generated inputs so that a change of the generator is caught
before any energy is compared.

  cfg1  2,000 + 30 atoms, OBC-II GB + SASA (960 points), all 10 frames:
        faithful rows (the reference's arithmetic and FP64 binding
        differences of totals) and accurate rows (exact binding differences)
  cfg2  5,000 + 50 atoms, first 4 frames: faithful and accurate rows and the
        accurate per-residue decomposition (335 residues x vdw, elec, polar, sa)
  cfg3  3,000 + 40 atoms, linearised PB on 0.5 A grids (buffer 12 A, DH
        boundary, 150 mM), first 2 frames: faithful rows (the reference's
        iteration schedule: absolute-RMS stop, 200-cycle cap, SOR fallback)
        and converged rows (every grid solved to a 1e-10 relative FP64
        residual; MM and SA binding terms exact)
  cfg5  25,000 + 80 atoms, first frame: GB + SASA faithful and accurate rows;
        PB (0.5 A, buffer 11.2 A) faithful and converged rows

Run from the repository root:  python tests/golden/make_golden.py [cfg ...]
Rows are the 13 FrameEnergy terms in the order complex mm/polar/sa,
receptor mm/polar/sa, ligand mm/polar/sa, delta mm/polar/sa/total.
"""
import hashlib
import json
import os
import sys
import tempfile
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "rust-simulation-tools_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

GB = dict(model="obc2", solvent_dielectric=78.5)  # 0.15 M, 300 K, offset 0.09, rgbmax 25, no cutoff
NPTS = 960
PB3 = dict(grid_spacing=0.5, grid_buffer=12.0, fillratio=0.0)
PB5 = dict(grid_spacing=0.5, grid_buffer=11.2, fillratio=0.0)
CONVERGED = dict(converged_rel_tol=1e-10, converged_method=1)
CONFIGS = {1: 10, 2: 4, 3: 2, 5: 1}


def inputs(k, n_frames):
    """(system, float32 frames, prmtop path, digests) of workload k."""
    from rust_simulation_tools import synthetic as S

    s, fr = S.workload(k, n_frames=n_frames)
    d = tempfile.mkdtemp()
    prm = os.path.join(d, f"w{k}.prmtop")
    S.write_prmtop(s, prm)
    dig = {"frames_sha256": hashlib.sha256(np.ascontiguousarray(fr, dtype=np.float32).tobytes()).hexdigest(),
           "prmtop_sha256": hashlib.sha256(open(prm, "rb").read()).hexdigest()}
    return s, fr, prm, dig


def coords(fr):
    # the reference's DCD path: float32 A -> f64 nm -> A (dcd.rs:429-437, binding.rs:630-633)
    return (fr.astype(np.float64) * 0.1) * 10.0


def rows(a):
    return [[float(v) for v in r] for r in np.asarray(a)]


def make(k):
    import oracle as O

    O.build()
    nf = CONFIGS[k]
    s, fr, prm, dig = inputs(k, nf)
    top = O.Topology.load(prm)
    x = coords(fr)
    rr, lr = s.receptor_residues, s.ligand_residues
    gb, sa = O.gb_params(**GB), O.sa_params(n_points=NPTS)
    out = {"workload": k, "frames": nf, "n_receptor_atoms": int(s.n_rec), "n_ligand_atoms": int(s.n_lig),
           "inputs": dig, "generator": "rust_simulation_tools.synthetic.workload(%d, n_frames=%d)" % (k, nf),
           "gb": "OBC-II, eps 1 / 78.5, 0.15 M, 300 K, offset 0.09, rgbmax 25, no cutoff",
           "sa": "probe 1.4 A, 960 points, gamma 0.0072, offset 0"}
    t0 = time.time()
    if k in (1, 2, 5):
        out["gb_faithful"] = rows(O.binding_frames(top, x, rr, lr, gb=gb, sa=sa))
        out["gb_accurate"] = rows(O.binding_frames(top, x, rr, lr, gb=gb, sa=sa, accurate=True))
    if k == 2:
        dec = []
        for f in range(nf):
            ro, lo = O.decompose(top, x[f], rr, lr, gb, sa, accurate=True)
            dec.append(rows(np.concatenate([ro, lo])))
        out["decomposition_accurate"] = dec
    if k in (3, 5):
        pb = PB3 if k == 3 else PB5
        out["pb"] = "linearised PB, spacing %.1f A, buffer %.1f A, eps 1 / 80, 0.15 M, DH boundary" % (
            pb["grid_spacing"], pb["grid_buffer"])
        out["pb_faithful"] = rows(O.binding_frames(top, x, rr, lr, pb=O.pb_params(**pb), sa=sa))
        out["pb_converged"] = rows(O.binding_frames(top, x, rr, lr, pb=O.pb_params(**pb, **CONVERGED), sa=sa,
                                                    accurate=True))
        out["pb_converged_rule"] = "every grid to a relative FP64 residual of 1e-10 (flexible CG, V-cycle)"
    out["seconds"] = round(time.time() - t0, 1)
    out["oracle_threads"] = O.threads()
    path = os.path.join(HERE, f"cfg{k}.json")
    with open(path, "w") as f:
        json.dump(out, f, indent=0)
    print(f"cfg{k}: {out['seconds']} s -> {path}", flush=True)


if __name__ == "__main__":
    for k in [int(a) for a in sys.argv[1:]] or sorted(CONFIGS):
        make(k)
