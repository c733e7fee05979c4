"""The oracle's results do not depend on its thread count: its parallel loops write only their own elements, every
reduction is one serial Neumaier sum (run as one task), and the modified Gram-Schmidt's wavefront keeps each vector's
projections in order. LOBPCG, the Jacobi-CG Poisson solve and a small SCF with forces, bit for bit on 1 and 4
threads. CPU only."""
import os

import numpy as np

NUC = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]


def _run(oracle, threads):
    n, h = 25, 0.35
    oracle.set_threads(threads)
    try:
        v = oracle.nuclear_potential(n, h, NUC, 0.5)
        ev, x, it, mr = oracle.lobpcg(n, h, v, oracle.initial_orbitals(n, h, NUC, 5, 1), tol=1e-6, max_iter=40,
                                      precond_lambda=-1.0)
        pv, pit, pres = oracle.poisson_solve(n, h, oracle.deposit_charge(n, h, NUC, 1.0), tol=1e-9, max_iter=400)
        st, stats = oracle.scf(n, h, NUC, 5, 5, sigma=0.5, tol=1e-4)
        f = oracle.forces(st, NUC, 0.5)
    finally:
        oracle.set_threads(min(8, os.cpu_count() or 1))  # the session fixture's setting
    return [ev, x, np.array([it, mr]), pv, np.array([pit, pres]), st.evals()[0], f], stats


def test_results_are_bitwise_independent_of_threads(oracle):
    a, sa = _run(oracle, 1)
    b, sb = _run(oracle, 4)
    for x, y in zip(a, b):
        assert np.array_equal(np.asarray(x), np.asarray(y))
    assert repr(sorted(sa.items())) == repr(sorted(sb.items()))
