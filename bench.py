#!/usr/bin/env python
"""MM-GBSA throughput on B200: frames/s of the batched, binding-fused engine.

Workload (default): synthetic receptor of 5,000 atoms + 50-atom ligand
(receptor residues of 15 atoms), 1,000 frames (sigma 0.5 A), OBC-II GB with
eps 1/78.5, 0.15 M salt, no cutoff, SASA with 960 points per atom, and
per-residue decomposition of every frame.  One step = one pass of the engine
over the 1,000 frames.

Reported (one JSON line on rank 0):
  value      frames/s, frames resident in HBM, device time of K steps
             (CUDA events on the library's stream), max over ranks
  e2e        frames/s through BindingSystem.run with pinned host frames:
             host->device copy of the frames and device->host copy of the
             per-frame energies and per-residue terms inside the timed region
  plain_gpu  frames/s of the plain FP64 form (one subsystem per launch
             sequence, per frame) on a sample of frames
  roofline   dominant kernel: algorithmic FLOPs / its CUDA-event duration vs
             the measured FP32 FMA peak of this GPU
  cpu_baseline  the CPU restatement of the reference (all host threads) on a
             bounded sample of the same frames
  serving    p50 / p99 request latency and frames/s of a bounded mixed
             request stream through the serving loop
  pbsa       MM-PBSA on the 3,000 + 40-atom workload (linearised PB, 0.5 A
             grid of 145 x 123 x 125 points, Debye-Hueckel boundary, 150 mM):
             frames/s of the batched mixed-precision engine (FP32 V-cycles
             under FP64 defect correction) and of the plain FP64 form, the
             largest polar-term difference between them, per-kernel HBM
             rooflines of the level-0 multigrid kernels, and the same with the
             reference's default two-level focusing
With --gpus N each rank runs its own 1,000 frames (weak scaling, replicas:
the path has no exchange step).
"""
import argparse
import faulthandler
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "rust-simulation-tools_b200"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import numpy as np  # noqa: E402

METRIC = "MM-GBSA frames/s (batched, binding-fused, mixed precision)"
GB = dict(model=2, solvent_dielectric=78.5, salt_concentration=0.15)
NPTS = 960


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def _synthetic():
    """The seeded input generator, loaded from its file without importing the
    package (whose __init__ maps librstg.so): the reference arm must run on
    the host cores with no GPU library in the process."""
    name = "_rstg_synthetic"
    if name not in sys.modules:
        import importlib.util

        spec = importlib.util.spec_from_file_location(
            name, os.path.join(ROOT, "rust-simulation-tools_b200", "rust_simulation_tools", "synthetic.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def host_facts():
    """CPU model and logical core count of this host (reported beside every
    CPU number)."""
    model = "unknown"
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


def workload(n_frames, rank):
    S = _synthetic()
    s = S.make_system(5000, 50, seed=1002)
    fr = S.make_frames(s, n_frames, seed=2002 + 7919 * rank)
    return s, fr


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, device):
        self.device, self.rows, self.proc = device, [], None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows if len(r) > 8 for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_baseline(s, fr, n_sample, gpu_rows=None, gpu_dec=None, n_check=2):
    """The CPU restatement of the reference (faithful mode, all host threads)
    timed on the first n_sample frames.  With the GPU's rows and per-residue
    terms for those frames, the largest differences against the accurate
    restatement (binding terms, per-residue terms) and against the faithful
    one (polar and SA binding terms) on the first n_check frames ride along,
    untimed, so the line carries its own parity."""
    import oracle as O

    O.build()
    d = tempfile.mkdtemp()
    S = _synthetic()

    S.write_prmtop(s, os.path.join(d, "w.prmtop"))
    top = O.Topology.load(os.path.join(d, "w.prmtop"))
    x = (fr[:n_sample].astype(np.float64) * 0.1) * 10.0
    gb = O.gb_params("obc2", solvent_dielectric=78.5)
    sa = O.sa_params(n_points=NPTS)
    t = time.perf_counter()
    faithful = O.binding_frames(top, x, s.receptor_residues, s.ligand_residues, gb=gb, sa=sa)
    for f in range(n_sample):  # decomposition of every frame, as the GPU step does
        O.decompose(top, x[f], s.receptor_residues, s.ligand_residues, gb, sa)
    dt = time.perf_counter() - t
    hf = host_facts()
    out = {"value": n_sample / dt, "unit": "frames/s", "cores": O.threads(), "kind": "port",
           "threads": O.threads(), "nproc": hf["nproc"], "cpu_model": hf["cpu_model"],
           "sample": f"{n_sample} frames of the 5,050-atom workload, binding frame + decomposition, "
                     f"C++ restatement of the reference, {O.threads()} OpenMP threads on a "
                     f"{hf['nproc']}-thread host"}
    if gpu_rows is not None:
        nc = min(n_check, n_sample)
        keys = ("delta_mm", "delta_polar", "delta_sa", "delta_total")
        acc = O.binding_frames(top, x[:nc], s.receptor_residues, s.ligand_residues, gb=gb, sa=sa, accurate=True)
        par = {"frames": nc, "tolerance_kcal": {"frame": 1e-3, "residue": 1e-4},
               "max_abs_vs_accurate_oracle": {k: float(np.abs(gpu_rows[:nc, 9 + i] - acc[:, 9 + i]).max())
                                              for i, k in enumerate(keys)},
               "max_abs_vs_faithful_oracle": {k: float(np.abs(gpu_rows[:nc, 9 + i] - faithful[:nc, 9 + i]).max())
                                              for i, k in enumerate(keys) if k in ("delta_polar", "delta_sa")}}
        if gpu_dec is not None:
            worst = 0.0
            for f in range(nc):
                ro, lo = O.decompose(top, x[f], s.receptor_residues, s.ligand_residues, gb, sa, accurate=True)
                worst = max(worst, float(np.abs(gpu_dec[f] - np.concatenate([ro, lo])).max()))
            par["max_abs_residue_vs_accurate_oracle"] = worst
        out["parity"] = par
    return out


PB = dict(grid_spacing=0.5, grid_buffer=12.0, fillratio=0.0)  # linearised PB, DH boundary, no focusing


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of this pool's B200s when
    MEASURED_PEAKS.json is present, else the earlier measurement on this pool."""
    try:
        return float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _golden(k):
    """Committed CPU-restatement results of workload k (tests/golden), or None."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", f"cfg{k}.json")) as f:
            return json.load(f)
    except OSError:
        return None


POLAR = (("complex_polar", 1), ("receptor_polar", 4), ("ligand_polar", 7), ("delta_polar", 10))


def _polar_err(a, b):
    n = min(len(a), len(b))
    return {k: float(np.abs(np.asarray(a)[:n, c] - np.asarray(b)[:n, c]).max()) for k, c in POLAR}


def pbsa_leg(rst, ctx, n_frames, n_plain, peak_gbs, rel_tols=(1e-6, 1e-9)):
    """MM-PBSA on the 3,040-atom workload: frames/s of the batched engine on
    the reference's stopping rule and on the relative-residual rule (FP32
    V-cycles of a consistent multigrid under FP64 defect correction), beside
    the plain FP64 form (reference schedule) on the first n_plain frames;
    polar-term differences against the plain form and against the oracle's
    golden rows (the reference's own iterate, and the converged solution)."""
    import torch
    S = _synthetic()

    s, fr = S.workload(3, n_frames=n_frames)
    d = tempfile.mkdtemp()
    S.write_prmtop(s, os.path.join(d, "w3.prmtop"))
    top = rst.read_prmtop(os.path.join(d, "w3.prmtop"))
    gold = _golden(3)
    out = {}
    for name, kw in (("linear_dh", PB), ("focusing_default", dict(fillratio=4.0))):
        nf = n_frames if name == "linear_dh" else min(n_frames, 32)
        p = rst.PbParams(**kw)
        fused = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p, ctx=ctx)
        fused.run(fr[:nf])  # warm-up at the timed size: the engine's pools are sized by the batch
        torch.cuda.synchronize()
        st0 = fused.pb_stats()
        t = time.perf_counter()
        ef = fused.run(fr[:nf])
        tf = time.perf_counter() - t
        st = {k: v - st0[k] for k, v in fused.pb_stats().items()}  # the timed run alone
        plain = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, pb_params=p, mode="plain", ctx=ctx)
        plain.run(fr[:1])
        t = time.perf_counter()
        ep = plain.run(fr[:n_plain])
        tp = time.perf_counter() - t
        pv = n_plain / tp
        r = {"reference_rule": {"fused_frames_per_s": nf / tf, "speedup_vs_plain_gpu": (nf / tf) / pv,
                                "max_abs_diff_vs_plain_fp64_kcal": _polar_err(ef, ep),
                                "grids": st["grids"], "lockstep_cycles": st["cycles"],
                                "sor_grids": st["fp64_fallbacks"],
                                "host_ms_setup_cycles_finish": [st["ms_setup"], st["ms_cycles"], st["ms_finish"]]},
             "plain_frames_per_s": pv, "plain_frames": n_plain, "frames": nf, "tolerance_kcal": 1e-3}
        if name == "linear_dh" and gold is not None:
            r["reference_rule"]["max_abs_diff_vs_oracle_reference_iterate_kcal"] = _polar_err(ef, gold["pb_faithful"])
            r["reference_rule"]["max_abs_diff_vs_oracle_converged_kcal"] = _polar_err(ef, gold["pb_converged"])
            r["plain_max_abs_diff_vs_oracle_converged_kcal"] = _polar_err(ep, gold["pb_converged"])
            r["oracle_frames"] = len(gold["pb_converged"])
        for tol in rel_tols:
            fused.set_pb_convergence(tol)
            st0 = fused.pb_stats()
            t = time.perf_counter()
            er = fused.run(fr[:nf])
            tr = time.perf_counter() - t
            st = {k: v - st0[k] for k, v in fused.pb_stats().items()}
            plain.set_pb_convergence(tol)  # the plain FP64 form on the same rule
            t = time.perf_counter()
            epr = plain.run(fr[:n_plain])
            tpr = time.perf_counter() - t
            plain.set_pb_convergence(0.0)
            q = {"fused_frames_per_s": nf / tr, "speedup_vs_plain_gpu_reference_rule": (nf / tr) / pv,
                 "plain_frames_per_s_same_rule": n_plain / tpr,
                 "speedup_vs_plain_gpu_same_rule": (nf / tr) / (n_plain / tpr),
                 "lockstep_cycles": st["cycles"], "sor_grids": st["fp64_fallbacks"],
                 "max_abs_diff_vs_plain_fp64_same_rule_kcal": _polar_err(er, epr)}
            if name == "linear_dh" and gold is not None:
                q["max_abs_diff_vs_oracle_converged_kcal"] = _polar_err(er, gold["pb_converged"])
                q["plain_max_abs_diff_vs_oracle_converged_kcal"] = _polar_err(epr, gold["pb_converged"])
            r[f"relative_residual_{tol:g}"] = q
        fused.set_pb_convergence(0.0)
        if name == "linear_dh":  # HBM roofline of the level-0 kernels (event-timed, no graph capture)
            fused.set_pb_profile(True)
            fused.run(fr[:8])
            prof = fused.pb_profile()
            r["roofline_level0"] = {k: {"achieved_gbs": v["bytes"] / (v["ms"] / 1e3) / 1e9,
                                        "frac_of_hbm": v["bytes"] / (v["ms"] / 1e3) / 1e9 / peak_gbs[0],
                                        "hbm_peak": peak_gbs[1],
                                        "ms": v["ms"], "launches": v["launches"]}
                                    for k, v in prof.items() if v["ms"] > 0}
            r["grid"] = "145 x 123 x 125 (complex), 0.5 A, buffer 12 A"
        out[name] = r
    return out


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return
    s, fr = workload(max(args.ref_frames, 1), 0)
    samples = []
    for k in range(args.warmup + args.steps):
        r = cpu_baseline(s, fr, args.ref_frames)
        if k >= args.warmup:
            samples.append(r["value"])
    v = float(np.median(samples))
    line = {"metric": METRIC, "value": v, "unit": "frames/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * args.ref_frames / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "MM-GBSA + per-residue decomposition, 5,000 + 50 atoms, 1,000 frames",
                       "sample_frames_per_step": args.ref_frames},
            "cpu_baseline": {"value": v, "unit": "frames/s", "cores": r["cores"], "kind": "port",
                             "threads": r["threads"], "nproc": r["nproc"], "cpu_model": r["cpu_model"],
                             "sample": r["sample"]},
            "e2e": {"value": v, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _fifo_latencies(arrivals, service):
    """Latencies of requests served one at a time in arrival order."""
    t, lat = 0.0, []
    for a, sv in zip(arrivals, service):
        t = max(t, a) + sv
        lat.append(t - a)
    return np.array(lat)


def serving_stream(rst, ctx, n_req, n_systems=32, seed=4, load=0.7):
    """Mixed MM-GBSA request stream: a pool of n_systems systems with
    receptors log-uniform over 1k-20k atoms and ligands of 20-80 atoms; each
    request takes a system of the pool and 1-200 frames (uniform); Poisson
    arrivals at `load` of the one-at-a-time capacity.  Beside the continuous
    batching loop: the same requests served one at a time in arrival order
    through the fused engine (each request's service time measured alone)
    and through the plain FP64 form (per-frame time of each system measured
    on 2 frames), FIFO queues on the same arrival times."""
    S = _synthetic()

    rng = np.random.default_rng(seed)
    d = tempfile.mkdtemp()
    systems = []
    for k in range(n_systems):
        nr = int(round(np.exp(rng.uniform(np.log(1000), np.log(20000)))))
        nl = int(rng.integers(20, 81))
        s = S.make_system(nr, nl, seed=3000 + k)
        p = os.path.join(d, f"s{k}.prmtop")
        S.write_prmtop(s, p)
        top = rst.read_prmtop(p)
        kw = dict(gb_params=rst.GbParams(**GB), sa_params=rst.SaParams(n_sphere_points=NPTS), ctx=ctx)
        bs = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, **kw)
        bp = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, mode="plain", **kw)
        pool = S.make_frames(s, 200, seed=5000 + k)  # requests take slices of this pool
        systems.append((s, bs, bp, nr + nl, pool))
    reqs = []
    for _ in range(n_req):
        k = int(rng.integers(0, n_systems))
        nf = int(rng.integers(1, 201))
        a = int(rng.integers(0, 201 - nf))
        reqs.append((k, a, nf))
    frames_of = lambda k, a, nf: systems[k][4][a:a + nf]
    for s, bs, bp, _, pool in systems:  # first-use preparation (layout, tuning) outside the stream
        bs.run(pool[:1])
    svc = []
    for k, a, nf in reqs:  # one request at a time through the fused engine
        t = time.perf_counter()
        systems[k][1].run(frames_of(k, a, nf))
        svc.append(time.perf_counter() - t)
    mean_gap = sum(svc) / n_req / load
    arrivals = np.cumsum(rng.exponential(mean_gap, size=n_req))
    srv = rst.Server(max_inflight=4, ctx=ctx)
    t0 = time.perf_counter()
    ids = []
    for (k, a, nf), at in zip(reqs, arrivals):
        dt = at - (time.perf_counter() - t0)
        if dt > 0:
            time.sleep(dt)
        ids.append(srv.submit(systems[k][1], frames_of(k, a, nf)))
    for i in ids:
        srv.wait(i, 1200000)
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    frames = sum(nf for _, _, nf in reqs)
    lat = _fifo_latencies(arrivals, svc)
    per_frame = []
    for s, bs, bp, _, pool in systems:
        bp.run(pool[:1])
        t = time.perf_counter()
        bp.run(pool[1:3])
        per_frame.append((time.perf_counter() - t) / 2)
    psvc = [per_frame[k] * nf for k, _, nf in reqs]
    plat = _fifo_latencies(arrivals, psvc)
    atoms = sorted(int(x[3]) for x in systems)
    return {"requests": n_req, "frames": frames, "systems": n_systems,
            "complex_atoms_min_median_max": [atoms[0], atoms[len(atoms) // 2], atoms[-1]],
            "continuous_batching": {"p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
                                    "delivered_frames_per_s": frames / wall,
                                    "note": "delivered rate follows the offered load"},
            "one_at_a_time_fused": {"p50_ms": 1e3 * float(np.percentile(lat, 50)),
                                    "p99_ms": 1e3 * float(np.percentile(lat, 99)),
                                    "mean_ms": 1e3 * float(lat.mean()),
                                    "capacity_frames_per_s": frames / sum(svc)},
            "one_at_a_time_plain_fp64": {"p50_ms": 1e3 * float(np.percentile(plat, 50)),
                                         "p99_ms": 1e3 * float(np.percentile(plat, 99)),
                                         "capacity_frames_per_s": frames / sum(psvc),
                                         "how": "per-frame time of each system measured on 2 frames; FIFO queue "
                                                "on the same arrival times"},
            "arrival_mean_ms": 1e3 * mean_gap, "load": load}


def large_mixed(rst, ctx, n_frames=500, per_request=50, pb_rel_tol=1e-9, seed=5):
    """25,000 + 80 atoms: MM-GBSA (SASA 960 points) and MM-PBSA (0.5 A grids of
    ~193^3, DH boundary, relative-residual stop) requests of per_request
    frames each, n_frames of each kind, interleaved in one serving loop with
    Poisson gaps; throughput, latency percentiles, and the errors of frame 0
    against the oracle's golden rows (accurate GB rows, converged PB rows)."""
    S = _synthetic()

    s, fr = S.workload(5, n_frames=n_frames)
    d = tempfile.mkdtemp()
    S.write_prmtop(s, os.path.join(d, "w5.prmtop"))
    top = rst.read_prmtop(os.path.join(d, "w5.prmtop"))
    gbkw = dict(gb_params=rst.GbParams(**GB), sa_params=rst.SaParams(n_sphere_points=NPTS), ctx=ctx)
    pbp = rst.PbParams(grid_spacing=0.5, grid_buffer=11.2, fillratio=0.0)
    pbkw = dict(pb_params=pbp, sa_params=rst.SaParams(n_sphere_points=NPTS), ctx=ctx)
    gsys = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, **gbkw)
    psys = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, **pbkw)
    psys.set_pb_convergence(pb_rel_tol)
    gsys.run(fr[:1])
    psys.run(fr[:1])
    rng = np.random.default_rng(seed)
    starts = list(range(0, n_frames, per_request))
    jobs = [("gb", a) for a in starts] + [("pb", a) for a in starts]
    rng.shuffle(jobs)
    srv = rst.Server(max_inflight=4, ctx=ctx)
    t0 = time.perf_counter()
    ids = []
    for kind, a in jobs:
        time.sleep(float(rng.exponential(0.05)))
        ids.append((kind, a, srv.submit(gsys if kind == "gb" else psys, fr[a:a + per_request])))
    outs = {(kind, a): srv.wait(i, 1800000) for kind, a, i in ids}
    wall = time.perf_counter() - t0
    st = srv.stats()
    srv.close()
    gb0, pb0 = outs[("gb", 0)][:1], outs[("pb", 0)][:1]
    gold = _golden(5)
    err = {}
    if gold is not None:
        cols = (("complex_polar", 1), ("receptor_polar", 4), ("ligand_polar", 7), ("delta_mm", 9),
                ("delta_polar", 10), ("delta_sa", 11), ("delta_total", 12))
        err["gb_vs_oracle_accurate"] = {k: float(abs(gb0[0, c] - gold["gb_accurate"][0][c])) for k, c in cols}
        err["pb_vs_oracle_converged"] = {k: float(abs(pb0[0, c] - gold["pb_converged"][0][c])) for k, c in cols}
        err["pb_oracle_reference_iterate_vs_converged"] = {
            k: float(abs(gold["pb_faithful"][0][c] - gold["pb_converged"][0][c])) for k, c in cols}
    return {"atoms": int(s.n_atoms), "gb_frames": n_frames, "pb_frames": n_frames, "frames_per_request": per_request,
            "requests": len(jobs), "frames_per_s": 2 * n_frames / wall, "wall_s": wall,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "pb_rule": f"relative residual {pb_rel_tol:g}",
            "pb_stats": psys.pb_stats(), "errors_frame0_kcal": err}


def main():
    faulthandler.enable()  # a crash in native code prints the Python stack
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--frames", type=int, default=1000)
    ap.add_argument("--ref-frames", type=int, default=8)
    ap.add_argument("--plain-frames", type=int, default=16)
    ap.add_argument("--serve-requests", type=int, default=200)
    ap.add_argument("--serve-systems", type=int, default=32)
    ap.add_argument("--pb-frames", type=int, default=100, help="MM-PBSA leg frames (0: skip)")
    ap.add_argument("--pb-plain-frames", type=int, default=24, help="frames of the plain FP64 PB form")
    ap.add_argument("--no-large", action="store_true", help="skip the 25,080-atom mixed GB/PB serving leg")
    ap.add_argument("--pb-only", action="store_true", help="run only the MM-PBSA leg (--pb-frames frames) and print it")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving leg (--serve-requests over --serve-systems) and print it")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e/plain/cpu/serving legs")
    ap.add_argument("--no-autotune", action="store_true",
                    help="fixed launch shapes (the tuner's usual picks on B200) instead of timing candidates on "
                         "the first run: for profiling, where the profiler distorts the candidates' timings")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.serve_only:
        import torch

        import rust_simulation_tools as rst
        from rust_simulation_tools import _native as N

        torch.cuda.set_device(0)
        ctx = N.make_ctx(0, torch.cuda.current_stream().cuda_stream)
        print(json.dumps(serving_stream(rst, ctx, args.serve_requests, args.serve_systems)), flush=True)
        return
    if args.pb_only:
        import torch

        import rust_simulation_tools as rst
        from rust_simulation_tools import _native as N

        torch.cuda.set_device(0)
        ctx = N.make_ctx(0, torch.cuda.current_stream().cuda_stream)
        print(json.dumps(pbsa_leg(rst, ctx, args.pb_frames, args.pb_plain_frames, hbm_peak())), flush=True)
        return

    import torch

    rank, world, local = dist_env()
    pg = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=datetime.timedelta(seconds=600))
        pg = dist
    torch.cuda.set_device(local)
    import rust_simulation_tools as rst
    from rust_simulation_tools import _native as N

    stream = torch.cuda.current_stream()
    ctx = N.make_ctx(local, stream.cuda_stream)
    s, fr = workload(args.frames, rank)
    d = tempfile.mkdtemp()
    S = _synthetic()

    S.write_prmtop(s, os.path.join(d, "w.prmtop"))
    top = rst.read_prmtop(os.path.join(d, "w.prmtop"))
    gb, sa = rst.GbParams(**GB), rst.SaParams(n_sphere_points=NPTS)
    sysf = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb, sa_params=sa, ctx=ctx,
                             autotune=not args.no_autotune)
    F, nres = fr.shape[0], sysf.n_residues
    d_fr = torch.from_numpy(fr).cuda()
    d_out = torch.empty((F, 13), dtype=torch.float64, device="cuda")
    d_dec = torch.empty((F, nres, 4), dtype=torch.float64, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def step():
        sysf.run_device(d_fr.data_ptr(), F, d_out.data_ptr(), d_dec.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = int(N.lib.rstg_ctx_kernel_launches(ctx))
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for a, b in evs:
            flush.zero_()  # L2 flush between timed steps (outside the events)
            a.record(stream)
            step()
            b.record(stream)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    launches = int(N.lib.rstg_ctx_kernel_launches(ctx)) - launches0
    ms = sum(a.elapsed_time(b) for a, b in evs)
    if pg:
        t = torch.tensor([ms], device="cuda")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())
    value = world * F * args.steps / (ms / 1000.0)
    stats = sysf.last_stats()
    out_np = d_out.cpu().numpy()

    extras = {}
    if not args.no_extras:
        # end to end through the public API with pinned host buffers
        h_fr = torch.from_numpy(fr).pin_memory().numpy()
        sysf.run(h_fr, decompose=True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if pg:
            pg.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        res, dec = sysf.run(h_fr, decompose=True)
        e1.record(stream)
        torch.cuda.synchronize()
        e2e_ms = e0.elapsed_time(e1)
        if pg:
            t = torch.tensor([e2e_ms], device="cuda")
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            e2e_ms = float(t.item())
        extras["e2e"] = {"value": world * F / (e2e_ms / 1000.0), "unit": "frames/s",
                         "h2d_bytes_per_step": int(fr.nbytes), "d2h_bytes_per_step": int(res.nbytes + dec.nbytes)}
        assert np.array_equal(res, out_np), "host and device paths disagree"
        # per-kernel roofline
        import ctypes as C

        n = C.c_int32()
        names = C.create_string_buffer(8 * 32)
        kms, kfl, kby = np.zeros(8), np.zeros(8), np.zeros(8)
        N.check(N.lib.rstg_system_profile(sysf._h, N.vp(d_fr.data_ptr()), F, C.byref(n), names,
                                          kms.ctypes.data_as(C.POINTER(C.c_double)),
                                          kfl.ctypes.data_as(C.POINTER(C.c_double)),
                                          kby.ctypes.data_as(C.POINTER(C.c_double))))
        kn = [names.raw[32 * k:32 * k + 32].split(b"\0")[0].decode() for k in range(n.value)]
        cal = np.zeros(4)
        N.check(N.lib.rstg_calibrate(local, cal.ctypes.data_as(C.POINTER(C.c_double))))
        tot = kms[:n.value].sum()
        share = {kn[k]: round(float(kms[k] / tot), 4) for k in range(n.value)}
        top_k = int(np.argmax(kms[:n.value]))
        fl_k = max(int(np.argmax(np.where(kfl[:n.value] > 0, kms[:n.value], -1))), 0)
        ach = kfl[fl_k] / (kms[fl_k] / 1000.0) / 1e12
        # DRAM traffic of one k_pairs launch: ncu dram read + write of a 64-frame
        # launch of this workload (19.6 MB, the committed ncu summary of k_pairs),
        # scaled by frames to this run's launches (the engine batches at most 256
        # frames); the traffic is coordinates, radii and per-block sums, in
        # proportion to frames
        per_launch = F / -(-F // 256)
        traffic = 19.6e6 / 64 * per_launch if kn[fl_k] == "pairs" else None
        extras["roofline"] = {"bound": "fp32", "kernel": kn[fl_k], "achieved": ach, "peak": float(cal[0]),
                              "unit": "TFLOP/s", "frac": ach / cal[0], "traffic": traffic,
                              "traffic_source": "ncu capture of a 64-frame launch scaled by frames per launch",
                              "peak_source": "measured FP32 FMA loop (rstg_calibrate) on this GPU",
                              "dominant_kernel": kn[top_k], "kernel_share": share,
                              "kernel_ms_per_1000_frames": {kn[k]: round(float(kms[k]) * 1000.0 / F, 3)
                                                            for k in range(n.value)},
                              "fp64_fma_tflops": float(cal[1]), "mufu_ex2_gops": float(cal[2]),
                              "sm_max_mhz_attr": float(cal[3])}
        # plain FP64 GPU form on a sample
        if args.plain_frames > 0:
            sysp = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb, sa_params=sa,
                                     mode="plain", ctx=ctx)
            sysp.run(fr[:1], decompose=True)
            t = time.perf_counter()
            sysp.run(fr[:args.plain_frames], decompose=True)
            pv = args.plain_frames / (time.perf_counter() - t)
            extras["plain_gpu"] = {"value": pv, "unit": "frames/s", "sample_frames": args.plain_frames,
                                   "form": "FP64, one subsystem per launch sequence, per frame, decomposition"}
            extras["speedup_vs_plain_gpu"] = value / world / pv
            # the middle form: the same FP32-pair / FP64-reduction kernels with
            # one frame per launch sequence, so the gain of batching stands
            # apart from that of the precision split
            sysm = rst.BindingSystem(top, s.receptor_residues, s.ligand_residues, gb_params=gb, sa_params=sa,
                                     batch_frames=1, ctx=ctx)
            nm = 4 * args.plain_frames
            sysm.run(fr[:1], decompose=True)
            t = time.perf_counter()
            sysm.run(fr[:nm], decompose=True)
            mv = nm / (time.perf_counter() - t)
            extras["mixed_unbatched"] = {"value": mv, "unit": "frames/s", "sample_frames": nm,
                                         "form": "FP32 pairs with FP64 reductions, binding-fused kernels, "
                                                 "one frame per launch sequence (batch of 1)",
                                         "speedup_vs_plain_gpu": mv / pv,
                                         "batched_speedup_over_it": value / world / mv}
        if rank == 0 and world == 1 and args.ref_frames > 0:
            extras["cpu_baseline"] = cpu_baseline(s, fr, args.ref_frames, out_np, d_dec.cpu().numpy())
        if rank == 0 and world == 1 and args.serve_requests > 0:
            extras["serving"] = serving_stream(rst, ctx, args.serve_requests, args.serve_systems)
        if rank == 0 and world == 1 and args.pb_frames > 0:
            # plain on the same frames
            extras["pbsa"] = pbsa_leg(rst, ctx, args.pb_frames, args.pb_plain_frames, hbm_peak())
        if rank == 0 and world == 1 and not args.no_large:
            extras["large_mixed"] = large_mixed(rst, ctx)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "frames/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32 pairs, f64 reductions",
                "data": "synthetic (seeded generator, 0.12 atoms/A^3, sigma 0.5 A frames)",
                "config": {"workload": "MM-GBSA + per-residue decomposition, receptor 5,000 + ligand 50 atoms, "
                                       "335 residues, 1,000 frames per GPU",
                           "gb": "OBC-II eps 1/78.5 0.15 M no cutoff", "sasa_points": NPTS,
                           "frames_per_gpu": F, "l2": "256 MB flush between timed steps",
                           "parallelism": f"replicas x{world} (frames sharded, no exchange)"},
                "gpu_launches": launches, "clocks": clk.summary(),
                "precision_stats": stats, "tuning": sysf.tuning()}
        line.update(extras)
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
