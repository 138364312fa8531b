"""Entropy estimates (crates/mmpbsa/src/entropy.rs): the interaction entropy
and the quasi-harmonic entropy against hand-computed answers.

CPU: the per-mode quantum harmonic-oscillator sum on a given spectrum, and
the interaction entropy's log-mean-exp, each against an independent
evaluation of the published formulas.  GPU: the mass-weighted covariance
(rstg_qh_covariance) against numpy on random frames, and the whole estimate
on a designed trajectory whose covariance -- and so its spectrum -- is known
exactly."""
import math

import numpy as np
import pytest

HBAR, KB, CONV, R = 1.054571817e-34, 1.380649e-23, 1e-20 * 1.66054e-27, 0.00198688


def qho_minus_ts(lams, T):
    """-T S of independent quantum oscillators, S/k = a/(e^a - 1) - ln(1 - e^-a),
    a = hbar / sqrt(k T lambda) (lambda in A^2 amu), modes below 1e-10 skipped."""
    lams = np.asarray([v for v in lams if v >= 1e-10], dtype=np.float64)
    a = HBAR / np.sqrt(KB * T * lams * CONV)
    a = a[a <= 500.0]
    return float(-T * R * np.sum(a / np.expm1(a) - np.log(-np.expm1(-a))))


def test_quasi_harmonic_sum_of_a_known_spectrum():
    from rust_simulation_tools._entropy import entropy_from_eigenvalues

    lams = [2.5, 0.7, 0.04, 3e-3, 5e-9, 0.0, -1e-12]
    for T in (298.15, 310.0):
        assert abs(entropy_from_eigenvalues(lams, T) - qho_minus_ts(lams, T)) < 1e-12 * abs(qho_minus_ts(lams, T))
    # one classical mode (a << 1): S/k -> 1 - ln(a)
    a = 1e-4
    lam = (HBAR / a) ** 2 / (KB * 300.0 * CONV)
    assert abs(entropy_from_eigenvalues([lam], 300.0) - (-300.0 * R * (1.0 - math.log(a)))) < 1e-6


def test_interaction_entropy_formula():
    import rust_simulation_tools as rst

    class F:
        def __init__(self, d):
            self.delta_mm = d

    de = [1.0, -0.5, 2.0, 0.25]
    kt = R * 298.15
    mean = sum(de) / len(de)
    want = kt * math.log(sum(math.exp((d - mean) / kt) for d in de) / len(de))
    got = rst.interaction_entropy([F(d) for d in de])
    assert abs(got.minus_tds - want) < 1e-12 and got.method == "interaction_entropy"
    assert rst.interaction_entropy([F(1.0)]) is None


@pytest.mark.gpu
def test_covariance_matches_numpy():
    import rust_simulation_tools as rst
    from rust_simulation_tools._entropy import covariance

    if rst.device_count() < 1:
        pytest.skip("no CUDA device")
    rng = np.random.default_rng(5)
    for F, n in ((7, 3), (40, 37)):  # 9 and 111 coordinates: partial 64-wide tiles
        traj = rng.normal(size=(F, n, 3)) * 2.0 + 10.0
        m = rng.uniform(1.0, 32.0, size=n)
        x = traj.reshape(F, -1) * np.repeat(np.sqrt(m), 3)
        d = x - x.mean(axis=0)
        want = d.T @ d / F
        got = covariance(traj, m)
        np.testing.assert_allclose(got, want, rtol=1e-10, atol=1e-12)
        np.testing.assert_array_equal(got, got.T)


@pytest.mark.gpu
def test_quasi_harmonic_on_a_designed_trajectory():
    """Two atoms, eight frames: the six coordinates follow the columns of an
    8 x 8 Hadamard matrix (orthogonal, zero-mean) scaled by s_k, so the
    mass-weighted covariance is exactly diag(m_k s_k^2) and its spectrum is
    known."""
    import rust_simulation_tools as rst

    if rst.device_count() < 1:
        pytest.skip("no CUDA device")
    h2 = np.array([[1, 1], [1, -1]])
    H = np.kron(np.kron(h2, h2), h2).astype(np.float64)  # 8 x 8, columns orthogonal
    s = np.array([0.3, 0.1, 0.05, 0.2, 0.02, 0.4])
    m = np.array([12.01, 1.008])
    traj = (H[:, 1:7] * s).reshape(8, 2, 3) + np.array([[1.0, 2.0, 3.0], [4.0, 5.0, 6.0]])
    lam = np.repeat(m, 3) * s ** 2
    got = rst.quasi_harmonic_entropy(traj, m, temperature=300.0)
    want = qho_minus_ts(lam, 300.0)
    assert got.method == "quasi_harmonic"
    assert abs(got.minus_tds - want) < 1e-9 * abs(want), (got.minus_tds, want)
    assert rst.quasi_harmonic_entropy(traj[:1], m) is None
