"""The reference's own known answers for the Fermi-Dirac occupation rule (crates/qm/src/occupations.rs:474-612:
fd_degenerate_pair_half_filled, fd_gap_symmetric_mu, fd_order_follows_evals, fd_gapped_plateau_midpoint,
fd_empty_channel, fd_non_finite_is_numerical, fd_bad_count_or_kt_is_numerical, fd_sums_to_n), as one check that runs
on any implementation of the rule: fermi_dirac(evals, n, kt) -> (f, mu, S), raising ValueError on a refusal."""
import math

import numpy as np
import pytest


def check(fermi_dirac):
    kt = 5e-3
    f, mu, S = fermi_dirac([-0.3, -0.3], 1, 1e-3)  # fd_degenerate_pair_half_filled
    assert list(f) == [0.5, 0.5] and abs(mu + 0.3) <= 1e-15 and abs(S - 2 * math.log(2)) <= 1e-14
    f, mu, S = fermi_dirac([-0.3, -0.3 + 5 * kt], 1, kt)  # fd_gap_symmetric_mu
    assert abs(f[0] - 1 / (1 + math.exp(-2.5))) <= 1e-14 and abs(f[1] - 1 / (1 + math.exp(2.5))) <= 1e-14
    assert abs(mu - (-0.3 + 2.5 * kt)) <= 1e-12
    a = fermi_dirac([-0.4, -0.31, -0.3, 0.2], 2, kt)  # fd_order_follows_evals
    b = fermi_dirac([0.2, -0.3, -0.4, -0.31], 2, kt)
    assert list(b[0]) == [a[0][3], a[0][2], a[0][0], a[0][1]] and a[1] == b[1]
    f, mu, S = fermi_dirac([-0.5, -0.5, 0.1], 2, kt)  # fd_gapped_plateau_midpoint
    assert f[0] == 1.0 and f[1] == 1.0 and 0.0 < f[2] <= math.exp(-36) and S <= 1e-14
    assert -0.5 + 30 * kt <= mu <= 0.1 - 30 * kt and abs(mu - (-0.2 + 0.5 * kt)) <= 2 * kt
    f, mu, S = fermi_dirac([-0.3, 0.1], 0, kt)  # fd_empty_channel
    assert list(f) == [0.0, 0.0] and math.isnan(mu) and S == 0.0
    for evals, n, t in (([-0.3, float("nan")], 1, kt), ([-0.3, 0.1], 2, kt), ([-0.3], 1, kt), ([-0.3, 0.1], 1, 0.0)):
        with pytest.raises(ValueError):  # fd_non_finite_is_numerical, fd_bad_count_or_kt_is_numerical
            fermi_dirac(evals, n, t)
    rng = np.random.default_rng(0x5EEDF00D)  # fd_sums_to_n: 200 spectra, spread log-uniform in [1e-6, 20] Ha
    for t in range(200):
        k = 2 + int(rng.integers(19))
        n = 1 + int(rng.integers(k - 1))
        spread = 1e-6 if t == 0 else (20.0 if t == 1 else 1e-6 * 2e7 ** rng.uniform())
        evals = -spread * rng.uniform(size=k)
        f, _, _ = fermi_dirac(evals, n, kt)
        assert abs(f.sum() - n) <= 1e-12 and ((f >= 0) & (f <= 1)).all()
