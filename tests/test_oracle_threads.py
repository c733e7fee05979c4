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


def test_pseudo_path_is_bitwise_independent_of_threads(oracle):
    """The pseudised-ion path (V_loc, the partial core, the Kleinman-Bylander operator, its SCF and the five force
    terms) on 1 and 4 threads, bit for bit."""
    import synthetic_species as ss
    n, h, sigma = 25, 0.35, 0.5
    sp = [ss.oxygen_like(h)]
    out = []
    for threads in (1, 4):
        oracle.set_threads(threads)
        try:
            x = np.random.default_rng(3).uniform(-0.5, 0.5, (2, n ** 3))
            nl, c = oracle.nonlocal_apply(n, h, NUC, sp, x)
            v_loc = oracle.ionic_local_potential(n, h, NUC, sigma, sp)
            st, stats = oracle.scf_ionic(n, h, NUC, 4, 4, sp, sigma=sigma, tol=1e-4)
            f = oracle.forces_ionic(st, NUC, sigma, sp)
            out.append(([nl, c, v_loc, st.evals()[0], st.evals()[1], f], repr(sorted(stats.items()))))
        finally:
            oracle.set_threads(min(8, os.cpu_count() or 1))
    for a, b in zip(out[0][0], out[1][0]):
        assert np.array_equal(np.asarray(a), np.asarray(b))
    assert out[0][1] == out[1][1]
