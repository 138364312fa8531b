"""Quasi-harmonic entropy (crates/mmpbsa/src/entropy.rs:97-225).

Post-processing off the per-frame path.  The mass-weighted coordinate
covariance (O((3N)^2 F), the expensive part) is formed on the GPU by
``rstg_qh_covariance`` with the reference's frame-ordered FP64 sums; its
eigenvalues come from a symmetric eigen-solver on the host (the reference
uses cyclic Jacobi rotations to 1e-10: the same spectrum to rounding), and
each mode contributes the quantum harmonic-oscillator entropy.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _native as N

KB_SI = 1.380649e-23      # J/K
HBAR = 1.054571817e-34    # J s
A2AMU_TO_SI = 1e-20 * 1.66054e-27  # A^2 amu -> m^2 kg
R_KCAL = 0.00198688       # kcal/(mol K)


def covariance(traj: np.ndarray, masses: np.ndarray) -> np.ndarray:
    """(3N, 3N) mass-weighted covariance of (F, N, 3) Angstrom coordinates."""
    traj = np.ascontiguousarray(traj, dtype=np.float64)
    masses = np.ascontiguousarray(masses, dtype=np.float64)
    F, n = traj.shape[0], masses.shape[0]
    cov = np.zeros((3 * n, 3 * n))
    dp = C.POINTER(C.c_double)
    N.check(N.lib.rstg_qh_covariance(N.ctx(), traj.ctypes.data_as(dp), F, n, masses.ctypes.data_as(dp),
                                     cov.ctypes.data_as(dp)))
    return cov


def entropy_from_eigenvalues(lam, temperature: float) -> float:
    """-T S in kcal/mol from covariance eigenvalues in A^2 amu (entropy.rs:180-222)."""
    kbt = KB_SI * temperature
    s = 0.0
    for v in lam:
        if v < 1e-10:
            continue  # translation / rotation and numerically zero modes
        a = HBAR / math.sqrt(kbt * (v * A2AMU_TO_SI))
        if a > 500.0:
            continue
        s += a / (math.exp(a) - 1.0) - math.log(1.0 - math.exp(-a))
    return -temperature * R_KCAL * s


def quasi_harmonic(traj: np.ndarray, masses: np.ndarray, temperature: float):
    if traj.ndim != 3 or traj.shape[2] != 3:
        raise ValueError("trajectory must be (n_frames, n_atoms, 3)")
    n_frames, n_atoms = traj.shape[0], masses.shape[0]
    if n_frames < 2 or n_atoms == 0:
        return None
    if traj.shape[1] != n_atoms:
        raise ValueError("masses and trajectory disagree on the atom count")
    lam = np.linalg.eigvalsh(covariance(traj, masses))
    return entropy_from_eigenvalues(lam, temperature)
