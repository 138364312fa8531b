"""Quasi-harmonic entropy (crates/mmpbsa/src/entropy.rs:97-225).

Post-processing off the per-frame path: the mass-weighted covariance of the
coordinates is diagonalised and each mode contributes the quantum
harmonic-oscillator entropy.  The reference diagonalises with cyclic Jacobi
rotations to 1e-10; a symmetric eigen-solver yields the same spectrum.
"""
from __future__ import annotations

import math

import numpy as np


def quasi_harmonic(traj: np.ndarray, masses: np.ndarray, temperature: float):
    if traj.ndim != 3 or traj.shape[2] != 3:
        raise ValueError("trajectory must be (n_frames, n_atoms, 3)")
    n_frames, n_atoms = traj.shape[0], masses.shape[0]
    if n_frames < 2 or n_atoms == 0:
        return None
    if traj.shape[1] != n_atoms:
        raise ValueError("masses and trajectory disagree on the atom count")
    w = np.repeat(np.sqrt(masses), 3)
    x = traj.reshape(n_frames, -1) * w
    d = x - x.mean(axis=0)
    cov = d.T @ d / n_frames
    lam = np.linalg.eigvalsh(cov)
    kbt = 1.380649e-23 * temperature
    conv = 1e-20 * 1.66054e-27
    s = 0.0
    for v in lam:
        if v < 1e-10:
            continue
        a = 1.054571817e-34 / math.sqrt(kbt * v * conv)
        if a > 500.0:
            continue
        s += a / (math.exp(a) - 1.0) - math.log(1.0 - math.exp(-a))
    return -temperature * 0.00198688 * s
