"""The solver's f64 host algebra through its host-only C-ABI hooks (no device is touched), against the reference's own
known answers: the Rayleigh-Ritz step on the 23 x 23 problem dumped from a failing reference run
(tests/golden/rr_i1_{a,b}.txt; crates/qm-gpu/src/eigen.rs:1188-1201 rayleigh_ritz_pairs_survive_a_bad_symmetric_eigen),
and the Fermi-Dirac occupation rule (crates/qm/src/occupations.rs:474-612), which must also agree with the oracle's
restatement. CPU only."""
import math
import os

import numpy as np
import pytest

import fd_known_answers

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rr_problem():
    return (np.loadtxt(os.path.join(GOLDEN, "rr_i1_a.txt")), np.loadtxt(os.path.join(GOLDEN, "rr_i1_b.txt")))


def test_rayleigh_ritz_survives_the_bad_symmetric_eigen(ks):
    """The reference's assertions: every returned coefficient vector's Rayleigh quotient equals its Ritz value to
    1e-9 and theta_0 = -0.8686699 to 1e-6 (the mispaired decomposition gave +0.7195). Also: theta ascending, the
    columns B-orthonormal to 1e-9, and the Ritz values those of the full generalised problem (scipy) to 1e-9."""
    from scipy.linalg import eigh
    a, b = _rr_problem()
    assert a.shape == b.shape and a.shape[0] == a.shape[1]
    theta, c, alpha = ks.rayleigh_ritz(a, b, 8)
    for k in range(8):
        ck = c[:, k]
        ray = (ck @ a @ ck) / (ck @ b @ ck)
        assert abs(ray - theta[k]) < 1e-9, (k, ray, theta[k])
    assert abs(theta[0] + 0.8686699) < 1e-6, theta
    assert np.all(np.diff(theta) >= 0)
    assert np.max(np.abs(c.T @ b @ c - np.eye(8))) < 1e-9
    assert np.max(np.abs(theta - eigh(a, b, eigvals_only=True)[:8])) < 1e-9
    assert alpha >= 1.0 - 1e-12


def test_rayleigh_ritz_refusals(ks):
    """A non-positive norm on B's diagonal and a subspace that lost rank are numerical errors (eigen.rs:522-531);
    bad sizes are argument errors."""
    a, b = _rr_problem()
    bad = b.copy()
    bad[3, 3] = 0.0
    with pytest.raises(ks.Numerical):
        ks.rayleigh_ritz(a, bad, 8)
    m = 6
    s = np.random.default_rng(1).standard_normal((m, 3))
    with pytest.raises(ks.Numerical):  # rank 3 < nk = 4
        ks.rayleigh_ritz(np.eye(m), s @ s.T + 1e-30 * np.eye(m), 4)
    with pytest.raises(ValueError):
        ks.rayleigh_ritz(a, b, a.shape[0] + 1)


def test_fermi_dirac_known_answers_of_the_solver(ks):
    fd_known_answers.check(ks.fermi_dirac)


def test_fermi_dirac_matches_the_oracle(ks, oracle):
    """The solver's rule and the oracle's restatement on 300 random spectra (spreads from 1e-6 to 20 Ha, kT from 1e-4
    to 0.05 Ha): f and S to 1e-14, mu to 1e-12 absolute."""
    rng = np.random.default_rng(0xFD)
    for _ in range(300):
        k = 2 + int(rng.integers(30))
        n = 1 + int(rng.integers(k - 1))
        kt = 1e-4 * 500 ** rng.uniform()
        evals = -(1e-6 * 2e7 ** rng.uniform()) * rng.uniform(size=k)
        f1, mu1, s1 = ks.fermi_dirac(evals, n, kt)
        f2, mu2, s2 = oracle.fermi_dirac(evals, n, kt)
        assert np.max(np.abs(f1 - f2)) <= 1e-14 and abs(s1 - s2) <= 1e-14 and abs(mu1 - mu2) <= 1e-12, (k, n, kt)


def test_witness_known_answers(ks):
    """The reference's witness tests on levels with zero residuals (crates/qm/src/occupations.rs:615-631
    witness_both_arms; :686-707 witness_keep_trims_the_overshoot, its zero-residual cases), on the solver's rule."""
    lvl = lambda top: [-0.3, top, -0.5]  # eps_(2) = -0.3, in any order
    assert not ks.fd_witness(lvl(-0.3 + 0.099), 2, -0.4, 5e-3)[0]   # the gap arm fails
    assert not ks.fd_witness(lvl(-0.1), 2, -0.1 - 0.105, 3e-3)[0]   # the tail arm fails: 0.105 < 36 kT = 0.108
    assert ks.fd_witness(lvl(-0.1), 2, -0.1 - 0.2, 3e-3)[0]         # both met
    assert not ks.fd_witness([-0.5, -0.3], 2, -0.9, 3e-3)[0]        # no level above the n-th
    assert ks.fd_witness([], 0, 0.0, 3e-3)[0]                       # an empty channel needs none
    kt, mu = 5e-3, -0.4
    evals = [-0.5, -0.3, -0.25, -0.1, -0.05, 0.0, 0.3]
    reached, keep = ks.fd_witness(evals, 1, mu, kt)
    assert reached and keep == 5      # the witness -0.1 at rank 3 and the passing spare -0.05
    assert ks.fd_witness(evals[:keep], 1, mu, kt)[0]  # what is kept passes on its own
    assert ks.fd_witness(evals, 0, mu, kt)[1] == 7    # an empty channel keeps its block
    assert ks.fd_witness([0.3, -0.5, -0.05, -0.1, 0.0, -0.25, -0.3], 1, mu, kt)[1] == 5  # order does not matter


def test_witness_reads_the_lower_bound(ks):
    """The reference's tests of the witness on theta - r (crates/qm/src/occupations.rs:666-683
    witness_reads_the_lower_bound; :686-704 witness_keep_trims_the_overshoot, its residual cases), on the rule the
    solver reads after each eigensolve."""
    kt, mu = 5e-3, -0.4
    top = mu + 36.0 * kt + 0.001  # the Ritz value clears the tail arm by 1 mHa (the gap arm by far)
    evals = [-0.5, top, -0.3]
    assert ks.fd_witness(evals, 1, mu, kt)[0]
    assert ks.fd_witness(evals, 1, mu, kt, residuals=[0.0, 0.0009, 0.0])[0]      # theta - r still clears it
    assert not ks.fd_witness(evals, 1, mu, kt, residuals=[0.0, 0.002, 0.0])[0]  # theta - r = top - 2 mHa does not
    near = [-0.5, -0.399]  # the gap arm on the lower bound: top - r must be >= -0.4
    assert ks.fd_witness(near, 1, -0.9, kt)[0]
    assert not ks.fd_witness(near, 1, -0.9, kt, residuals=[0.0, 0.002])[0]
    assert not ks.fd_witness(evals, 1, mu, kt, residuals=[0.0, float("nan"), 0.0])[0]  # a NaN residual never passes
    assert ks.fd_witness([], 0, 0.0, kt, residuals=[])[0]
    assert not ks.fd_witness([-0.5], 1, -0.9, kt, residuals=[0.0])[0]
    block = [-0.5, -0.3, -0.25, -0.1, -0.05, 0.0, 0.3]
    zero = [0.0] * 7
    assert ks.fd_witness(block, 1, mu, kt, residuals=zero)[1] == 5
    spare_fails = [0.0, 0.0, 0.0, 0.0, 0.2, 0.0, 0.0]
    assert ks.fd_witness(block, 1, mu, kt, residuals=spare_fails)[1] == 4                      # the witness alone on top
    assert ks.fd_witness(block, 1, mu, kt, residuals=[0.0, 0.0, 0.0, 0.15, 0.0, 0.0, 0.0])[1] == 6  # pushed up a rank
    for res in (zero, spare_fails):  # whatever is kept passes the witness on its own
        k = ks.fd_witness(block, 1, mu, kt, residuals=res)[1]
        assert ks.fd_witness(block[:k], 1, mu, kt, residuals=res[:k])[0]
    assert ks.fd_witness(block, 0, mu, kt, residuals=zero)[1] == 7  # an empty channel keeps its block
    with pytest.raises(ValueError):
        ks.fd_witness(block, 1, mu, kt, residuals=zero[:3])


def test_scf_settings_for_grid_has_the_reference_defaults(ks):
    """ScfSettings::for_grid (crates/qm/src/scf.rs:381-395): sigma = h, tol 1e-6, 200 iterations, mixing 0.3, eig_tol
    1e-6, DIIS history 6, Fermi-Dirac at ELECTRON_KT = 5e-3, the stall window 50; the plain constructor keeps Aufbau."""
    s = ks.ScfSettings.for_grid(0.25)
    assert (s.sigma, s.tol, s.max_iter, s.mixing, s.eig_tol, s.diis_history, s.stall_window) == (0.25, 1e-6, 200, 0.3, 1e-6, 6, 50)
    assert s.occupations == "fermi_dirac" and s.kt == 5e-3
    assert ks.ScfSettings().occupations == "aufbau"


def test_witness_keep_within_reads_the_lowest_converged_witness(ks):
    """The reference's test of the lowest converged witness (crates/qm/src/occupations.rs:706-745
    witness_keep_within_reads_the_lowest_converged_witness), on the rule the solver applies on a tight step whose top
    level passes only above 1.5e-3 Ha."""
    kt, mu, r_max = 5e-3, -0.4, 1.5e-3  # the arms: lower bound >= mu + 0.18 = -0.22 and >= eps_(1) + 0.1 = -0.4
    evals = [-0.5, -0.3, -0.25, -0.1, -0.05, 0.0, 0.3]
    zero = [0.0] * 7
    kw = ks.fd_witness_keep_within
    assert kw(evals, zero, 1, mu, kt, r_max) == ks.fd_witness(evals, 1, mu, kt, residuals=zero)[1] == 5
    top_loose = [0.0, 0.0, 0.0, 1e-4, 0.0, 0.0, 3e-3]
    assert kw(evals, top_loose, 1, mu, kt, r_max) == 5
    first_loose = [0.0, 0.0, 0.0, 2e-3, 1e-3, 3e-3, 3e-3]
    assert kw(evals, first_loose, 1, mu, kt, r_max) == 6
    only_top = [0.0, 0.0, 0.0, 2e-3, 2e-3, 2e-3, 1e-3]
    assert kw(evals, only_top, 1, mu, kt, r_max) == 7
    assert kw(evals, [0.0, 0.0, 0.0, 2e-3, 2e-3, 2e-3, 2e-3], 1, mu, kt, r_max) is None
    assert kw(evals[:3], zero[:3], 1, mu, kt, r_max) is None               # rank 2, -0.25 < -0.22: no witness
    assert kw(evals[:3], zero[:3], 1, mu, kt, r_max, tail_kt=6.0) == 3     # a 6 kT tail lets rank 1 decide
    for res in (zero, top_loose, first_loose, only_top):
        k = kw(evals, res, 1, mu, kt, r_max)
        assert ks.fd_witness(evals[:k], 1, mu, kt, residuals=res[:k])[0]
        assert res[k - 1] <= r_max or res[k - 2] <= r_max
    assert kw(evals, zero, 0, mu, kt, r_max) == 7
    assert kw(evals[:1], zero[:1], 1, mu, kt, r_max) is None
    e2, r2 = [0.0, -0.5, 0.3, -0.1, -0.3, -0.05, -0.25], [0.0, 0.0, 3e-3, 2e-3, 0.0, 1e-3, 0.0]
    assert kw(e2, r2, 1, mu, kt, r_max) == 6                                # order-independent
    assert kw(evals, [0.0, 0.0, 0.0, float("nan"), 0.0, 0.0, 0.0], 1, mu, kt, r_max) == 6  # a NaN residual never qualifies


def test_step_tail_follows_the_step_accuracy(ks):
    """The reference's test of the loosened step's witness tail (crates/qm/src/occupations.rs:773-786
    step_tail_follows_the_step_accuracy): ln(n_w / (1e-3 drho)) kT clamped to [6, 36]."""
    assert abs(ks.fd_step_tail_kt(10, 1e-2) - math.log(1e6)) < 1e-12
    assert abs(ks.fd_step_tail_kt(10, 10.0) - math.log(1e3)) < 1e-12
    assert ks.fd_step_tail_kt(10, 100.0) == 6.0
    assert ks.fd_step_tail_kt(10, 1e-15) == 36.0
    for d in (float("inf"), float("nan"), 0.0, -1.0):
        assert ks.fd_step_tail_kt(7, d) == 36.0
    xs = [ks.fd_step_tail_kt(8, 10 ** (2.0 - e / 4.0)) for e in range(60)]
    assert all(b >= a for a, b in zip(xs, xs[1:])) and xs[0] == 6.0 and xs[-1] == 36.0


def test_tight_columns_follow_f_and_the_stop(ks):
    """The reference's test of the Fermi-Dirac tight count (crates/qm/src/occupations.rs:630-664
    tight_columns_follow_f_and_the_stop): one electron, a 0.2 Ha gap, mu at mid-gap, the level above at f = e^-20."""
    kt = 5e-3
    evals = [-0.5, -0.3, 0.0, 0.1]
    zero = [0.0] * 4
    mu = ks.fermi_dirac(evals, 1, kt)[1]
    f1 = 1.0 / (1.0 + math.exp((-0.3 - mu) / kt))
    assert 1e-9 <= f1 < 1e-8
    assert ks.fd_tight_columns(evals, zero, mu, kt, 1e-6) == 1           # limit 1e-8 > f1 + tail: loose
    assert ks.fd_tight_columns(evals, zero, mu, kt, 1e-7) == 2           # limit 1e-9 < f1: tight (the stop decides)
    assert ks.fd_tight_columns(evals, [0.0, 0.03, 0.0, 0.0], mu, kt, 1e-6) == 2  # r raises f(theta - r)
    assert ks.fd_tight_columns([-0.3, -0.5, 0.1, 0.0], zero, mu, kt, 1e-6) == 2  # positions, not ranks
    p = [-0.5, -0.49, 0.3]
    mp = ks.fermi_dirac(p, 1, kt)[1]
    assert ks.fd_tight_columns(p, [0.0] * 3, mp, kt, 1e-6) == 2          # a partly occupied level stays tight
    many = [-0.5] + [mu + kt * math.log(1e9)] * 20 + [0.3]               # twenty levels at f ~ 1e-9 each
    t = ks.fd_tight_columns(many, [0.0] * len(many), mu, kt, 1e-6)
    assert 2 <= t <= len(many) - 9, t                                     # the tail is a sum
    assert ks.fd_tight_columns([0.1, 0.2], [0.0, 0.0], None, kt, 1e-6) == 0  # an empty channel
    assert ks.fd_tight_columns(evals, [0.0, 0.0, 0.0, float("nan")], mu, kt, 1e-6) == 4  # a NaN residual is never loose


def test_tight_start_reads_the_stored_occupations(ks):
    """tight_start (crates/qm/src/occupations.rs:355-366): the stored ascending f's loose tail at 1e-2 tol, at least n;
    n without a state."""
    assert ks.fd_tight_start(None, 3, 1e-6) == 3
    assert ks.fd_tight_start([1.0, 1.0, 5e-9, 1e-12], 2, 1e-6) == 2      # the tail 5e-9 + 1e-12 < 1e-8
    assert ks.fd_tight_start([1.0, 1.0, 5e-9, 1e-12], 2, 1e-7) == 3      # 5e-9 >= 1e-9: tight
    assert ks.fd_tight_start([1.0, 0.6, 0.4, 1e-12], 1, 1e-6) == 3       # partial levels stay tight
    assert ks.fd_tight_start([1.0, 1e-12], 3, 1e-6) == 3                 # never below n
