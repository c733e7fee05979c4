"""The oracle's pseudised-ion restatement (crates/qm/src/nuclear.rs:297-378, nonlocal.rs, forces.rs) against the
reference's own known answers and identities. CPU only.

The reference's table generator (its radial atom solver) cannot run here, so the tables are the analytic ones of
tests/synthetic_species.py; every property checked holds for any table."""
import numpy as np
import pytest

import synthetic_species as ss


def test_solid_harmonic_gradients_match_finite_differences(oracle):
    """solid_harmonic_gradients_match_finite_differences (crates/qm/src/nonlocal.rs:251-268): grad R_lm for l <= 2
    against central differences of the solid harmonics at r = (0.37, -0.52, 0.81), step 1e-6, to 1e-8."""
    r = np.array([0.37, -0.52, 0.81])
    g = oracle.solid_harmonic_gradients(r)
    e = 1e-6
    for lm in range(9):
        for a in range(3):
            p, m = r.copy(), r.copy()
            p[a] += e
            m[a] -= e
            fd = (oracle.solid_harmonics(p)[lm] - oracle.solid_harmonics(m)[lm]) / (2 * e)
            assert abs(g[lm, a] - fd) < 1e-8, (lm, a, g[lm, a], fd)


def test_uniform_table_reads(oracle):
    """The 4-point Lagrange read of filter.rs:302-317: exact for a cubic in d away from d = 0 (value and
    derivative), exact at the nodes, the mirrored index -1 for an even function near 0, and 0 beyond the radius or
    the table."""
    du = 0.3 / 256
    k = np.arange(400)
    cubic = lambda d: 1.0 + 2.0 * d - 3.0 * d ** 2 + 0.5 * d ** 3
    dcubic = lambda d: 2.0 - 6.0 * d + 1.5 * d ** 2
    f = cubic(k * du)
    rng = np.random.default_rng(3)
    for d in rng.uniform(du, 390 * du, 50):
        v, dv = oracle.table_read(f, du, 1.0, d)
        assert abs(v - cubic(d)) < 1e-12 and abs(dv - dcubic(d)) < 1e-9, (d, v, cubic(d), dv, dcubic(d))
    for i in (1, 7, 100, 300):
        assert oracle.table_read(f, du, 1.0, i * du)[0] == pytest.approx(f[i], abs=1e-15)
    even = lambda d: np.exp(-d * d)
    fe = even(k * du)
    for d in (0.0, 0.3 * du, 0.9 * du):
        v, dv = oracle.table_read(fe, du, 1.0, d)
        assert abs(v - even(d)) < 1e-12 and abs(dv + 2 * d * even(d)) < 1e-6
    assert oracle.table_read(f, du, 0.2, 0.2 + 1e-9) == (0.0, 0.0)
    assert oracle.table_read(f, du, 10.0, 398 * du) == (0.0, 0.0)  # the 4-point stencil leaves the table


def test_bare_hydrogen_local_potential_is_the_nuclear_potential(oracle):
    """A pseudised species with Z_v = Z, the all-electron width and no tables is exactly the smeared nucleus
    (nuclear.rs:297-315: V_LR is the same erf), bit for bit."""
    n, h, sigma = 25, 0.3, 0.5
    nuc = [(0.7, 0.0, 0.1, 1), (-0.7, 0.05, 0.0, 1)]
    v_ae = oracle.nuclear_potential(n, h, nuc, sigma)
    v_ps = oracle.ionic_local_potential(n, h, nuc, sigma, [ss.bare_hydrogen(h, sigma)])
    assert np.array_equal(v_ae, v_ps)


def test_nonlocal_is_symmetric_with_a_clipped_sphere(oracle):
    """projector_sphere_clipped_by_the_box_stays_symmetric (crates/qm/src/nonlocal.rs:314-336): an ion 0.4 Bohr
    inside a face, its balls clipped by the box, <a | V_NL b> = <V_NL a | b> to 1e-12."""
    n, h = 33, 0.2
    edge = -(n - 1) * h / 2 + 0.4
    sp = [ss.oxygen_like(h)]
    rng = np.random.default_rng(0x5EED)
    a, b = rng.uniform(-0.5, 0.5, (2, n ** 3))
    (na, nb), c = oracle.nonlocal_apply(n, h, [(edge, 0.1, -0.2, 8)], sp, np.stack([a, b]))
    (wa,), cw = oracle.nonlocal_apply(n, h, [(0.0, 0.1, -0.2, 8)], sp, a[None])
    assert np.count_nonzero(na) < 0.75 * np.count_nonzero(wa), "the balls are clipped"
    x, y = np.dot(a, nb), np.dot(na, b)
    assert abs(x - y) <= 1e-12 * max(abs(x), abs(y))
    assert c.shape == (2, 4)  # s (1 row) + p (3 rows)


@pytest.fixture(scope="module")
def pseudo_water_small(oracle):
    n, h, sigma = 25, 0.35, 0.5
    sp = [ss.oxygen_like(h)]
    nuc = [(0.05, -0.03, 0.02, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
    st, stats = oracle.scf_ionic(n, h, nuc, 4, 4, sp, sigma=sigma, tol=1e-6)
    assert stats["status"] == 0, stats
    return st, nuc, sp, sigma


def test_forces_are_the_frozen_energy_derivative(oracle, pseudo_water_small):
    """The five force terms are minus the R-derivative of the energy at frozen orbitals and densities (forces.rs,
    pseudised ions: each term is the derivative of one frozen energy): central differences, step 1e-4 Bohr, on every
    coordinate of the O-like ion (long range, short range, partial core, nonlocal) and of one H (long range, ion-ion)."""
    st, nuc, sp, sigma = pseudo_water_small
    f = oracle.forces_ionic(st, nuc, sigma, sp)
    e = 1e-4
    for a in (0, 1):
        for ax in range(3):
            def moved(s):
                out = [list(x) for x in nuc]
                out[a][ax] += s
                return [tuple(x) for x in out]
            fd = -(oracle.frozen_energy(st, moved(e), sigma, sp) - oracle.frozen_energy(st, moved(-e), sigma, sp)) / (2 * e)
            assert abs(f[a, ax] - fd) <= 2e-6 + 1e-5 * abs(fd), (a, ax, f[a, ax], fd)


def test_pseudo_scf_energy_bookkeeping(oracle, pseudo_water_small):
    """The valence count, the valence-charge repulsion and a bound state: electrons = 8, E_nuclear = sum q q / R with
    q_O = 6, and the lowest level of each spin below zero."""
    st, nuc, sp, sigma = pseudo_water_small
    up, dn = st.evals()
    assert up[0] < 0 and dn[0] < 0
    r = np.array([x[:3] for x in nuc])
    q = [6.0, 1.0, 1.0]
    e_ii = sum(q[i] * q[j] / np.linalg.norm(r[i] - r[j]) for i in range(3) for j in range(i + 1, 3))
    st2, stats = oracle.scf_ionic(25, 0.35, nuc, 4, 4, sp, sigma=sigma, tol=1e-3)
    assert abs(stats["nuclear"] - e_ii) < 1e-12
    assert abs(sum(stats["electrons"]) - 8.0) < 1e-6
