"""The oracle against the reference's own known answers (tests/golden/reference_pins.json, made by
tests/golden/make_pins.py from the reference's test sources). CPU only."""
import json
import math
import os

import numpy as np
import pytest

import fd_known_answers

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))


@pytest.mark.parametrize("name", ["H2", "LiH"])
def test_33_aufbau_pins(oracle, name):
    """none_policy_is_bitwise_today (crates/qm/src/scf.rs:1276-1331): the restatement reproduces the
    reference's pinned energy and force to ~1e-10 (bitwise is out of reach: nalgebra's eigen
    rounding and the platform libm differ)."""
    g = GOLDEN["pins_33"]
    s = g[name]
    nuc = [tuple(x) for x in s["nuclei"]]
    st, stats = oracle.scf(33, 0.25, nuc, s["n_up"], s["n_dn"], sigma=0.25, tol=1e-6)
    assert stats["status"] == 0, stats
    f = oracle.forces(st, nuc, 0.25)
    assert abs(stats["total"] - s["energy"]) < 1e-9, (stats["total"], s["energy"])
    assert abs(f[0, 0] - s["force_x0"]) < 1e-8, (f[0, 0], s["force_x0"])
    assert stats["iterations"] == s["steps"]


@pytest.mark.parametrize("name", ["H", "He", "H2"])
def test_49_cpu_energies(oracle, name):
    """The published 49^3 CPU energies (crates/validate/references.md:156-158), 9 decimals."""
    g = GOLDEN["cpu_49"]
    s = g["systems"][name]
    nuc = [tuple(x) for x in s["nuclei"]]
    st, stats = oracle.scf(49, 0.25, nuc, s["n_up"], s["n_dn"], sigma=0.25, tol=1e-6)
    assert stats["status"] == 0
    assert abs(stats["total"] - g["energy"][name]) < 2e-9, (stats["total"], g["energy"][name])
    if name == "H2":
        f = oracle.forces(st, nuc, 0.25)
        assert abs(f[0, 0] - g["forces"]["H2_R1.4_F0x"]) < 1e-8


def test_pw92_known_values(oracle):
    """crates/qm/src/xc.rs:236-245: unpolarised eps_c at r_s = 2 and 10."""
    p = GOLDEN["pw92"]
    for rs, want in ((2.0, p["eps_c_rs2"]), (10.0, p["eps_c_rs10"])):
        n = 3.0 / (4.0 * math.pi * rs ** 3)
        e, _, _ = oracle.exc_point(n / 2, n / 2)
        ex = -(3.0 / 4.0) * (3.0 / math.pi) ** (1.0 / 3.0) * n ** (4.0 / 3.0)
        assert abs((e - ex) / n - want) < p["tol"]


def test_xc_potential_is_the_energy_derivative(oracle):
    """potentials_match_finite_difference (crates/qm/src/xc.rs:281-293)."""
    for nu, nd in ((0.3, 0.3), (0.05, 0.2), (0.001, 0.0004), (0.1, 0.0)):
        _, vu, vd = oracle.exc_point(nu, nd)
        d = 1e-6 * (nu + nd)
        fd_u = (oracle.exc_point(nu + d, nd)[0] - oracle.exc_point(nu - d, nd)[0]) / (2 * d)
        assert abs(vu - fd_u) <= 1e-7 + 1e-6 * abs(fd_u)
        if nd > 0:
            fd_d = (oracle.exc_point(nu, nd + d)[0] - oracle.exc_point(nu, nd - d)[0]) / (2 * d)
            assert abs(vd - fd_d) <= 1e-7 + 1e-6 * abs(fd_d)
    assert oracle.exc_point(0.0, 0.0) == (0.0, 0.0, 0.0)


def test_coulomb_far_field_and_on_site(oracle):
    """potential_is_coulombic_far_away (crates/qm/src/nuclear.rs:500-509): erf pinned to 1e-12."""
    a = GOLDEN["analytic"]["coulomb_far_49"]
    v = oracle.nuclear_potential(49, 0.25, [(0.0, 0.0, 0.0, a["z"])], a["sigma"])
    i, j, k = a["far_index"]
    assert abs(v[i + 49 * (j + 49 * k)] - a["far_value"]) < a["tol"]
    on = v[24 + 49 * (24 + 49 * 24)]
    assert abs(on - (-a["z"] * math.sqrt(2 / math.pi) / a["sigma"])) < 1e-12


def test_stencil_converges_at_eighth_order(oracle):
    """converges_at_eighth_order (crates/qm/src/stencil.rs:85-92)."""
    def err(n, h):
        x, y, z = oracle.grid_points(n, h)
        r2 = x * x + y * y + z * z
        f = np.exp(-r2 / 2)
        exact = (r2 - 3) * np.exp(-r2 / 2)
        lap = oracle.laplacian(n, h, f).reshape(n, n, n)
        e = np.abs(lap - exact.reshape(n, n, n))[4:-4, 4:-4, 4:-4]
        return e.max()
    coarse, fine = err(25, 0.5), err(49, 0.25)
    assert fine < 1e-4 and coarse / fine > 64


def test_solid_harmonics_closed_forms_and_addition_theorem(oracle):
    """crates/qm/src/poisson.rs:320-362."""
    x, y, z = 0.7, -0.4, 1.1
    r2 = x * x + y * y + z * z
    h = oracle.solid_harmonics([x, y, z])
    s3 = math.sqrt(3)
    lm = lambda l, m: l * l + l + m
    for (l, m, v) in ((0, 0, 1), (1, 0, z), (1, 1, x), (1, -1, y), (2, 0, (3 * z * z - r2) / 2), (2, 1, s3 * x * z),
                      (2, -1, s3 * y * z), (2, 2, s3 * (x * x - y * y) / 2), (2, -2, s3 * x * y)):
        assert abs(h[lm(l, m)] - v) < 1e-14
    a, b = np.array([0.3, -0.2, 0.5]), np.array([2.0, 1.5, -1.0])
    ha, hb = oracle.solid_harmonics(a), oracle.solid_harmonics(b)
    na, nb = np.linalg.norm(a), np.linalg.norm(b)
    exact = 1 / np.linalg.norm(a - b)
    partial, prev = 0.0, np.inf
    for l in range(7):
        for m in range(-l, l + 1):
            partial += ha[lm(l, m)] * hb[lm(l, m)] / nb ** (2 * l + 1)
        e = abs(partial - exact)
        assert e <= (na / nb) ** (l + 1) / (nb - na) and e < prev
        prev = e


def test_gaussian_charge_potential_and_hartree_energy(oracle):
    """gaussian_potential_off_centre_uses_dipole_boundary + hartree_energy_of_gaussian
    (crates/qm/src/poisson.rs:291-315): max error < 1e-4 and E_H = q^2/(2 sigma sqrt(pi)) to 1e-4."""
    n, h, sigma = 49, 0.25, 0.5
    x, y, z = oracle.grid_points(n, h)
    c = (1.3, -0.7, 0.4)
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    rho = (2 * math.pi * sigma ** 2) ** -1.5 * np.exp(-r ** 2 / (2 * sigma ** 2))
    from scipy.special import erf
    exact = np.where(r < 1e-12, math.sqrt(2 / math.pi) / sigma, erf(r / (sigma * math.sqrt(2))) / np.maximum(r, 1e-300))
    v, it, res = oracle.poisson_solve(n, h, rho, tol=1e-10)
    assert res < 1e-10
    assert np.abs(v - exact).max() < 1e-4
    eh = 0.5 * np.dot(rho, v) * h ** 3
    q = GOLDEN["analytic"]["gaussian_poisson_49"]
    rc = (2 * math.pi * sigma ** 2) ** -1.5 * np.exp(-(x * x + y * y + z * z) / (2 * sigma ** 2))
    vc, _, _ = oracle.poisson_solve(n, h, rc, tol=1e-10)
    assert abs(0.5 * np.dot(rc, vc) * h ** 3 - q["hartree"]) < q["hartree_tol"]
    assert eh > 0


def test_oscillator_spectrum(oracle):
    """oscillator_spectrum (crates/qm/src/eigen.rs:394-404): 1.5 and 2.5 (x3) to 1e-4 at 49^3."""
    n, h = 49, 0.25
    x, y, z = oracle.grid_points(n, h)
    v = 0.5 * (x * x + y * y + z * z)
    seed = 12345
    guess = np.empty((4, n ** 3))
    r2 = (x * x + y * y + z * z) / 8.0
    for k in range(4):
        for p in range(n ** 3):
            seed = (seed * 6364136223846793005 + 1442695040888963407) % (1 << 64)
            guess[k, p] = (seed >> 11) / float(1 << 53) - 0.5
        guess[k] *= np.exp(-r2)
    ev, _, it, mr = oracle.lobpcg(n, h, v, guess, tol=1e-6, max_iter=500)
    assert mr < 1e-6
    assert abs(ev[0] - 1.5) < 1e-4 and all(abs(e - 2.5) < 1e-4 for e in ev[1:])


def test_diis_and_sym_eigen(oracle):
    """Host algebra of the oracle: the Jacobi eigen-decomposition (crates/qm/src/eigen.rs:175-211)
    and the bordered Pulay system (crates/qm/src/scf.rs:681-697)."""
    rng = np.random.default_rng(7)
    q, _ = np.linalg.qr(rng.standard_normal((12, 12)))
    lam = np.concatenate([[-0.8686, -0.8686 + 1e-12, -0.8686 + 2e-12], np.linspace(1, 70, 9)])
    a = (q * lam) @ q.T
    a = 0.5 * (a + a.T)
    ev, vec = oracle.sym_eigen(a)
    assert np.abs(np.sort(ev) - np.sort(lam)).max() < 1e-10
    assert np.abs(a @ vec - vec * ev).max() < 1e-10
    r = rng.standard_normal((4, 50))
    c = oracle.diis_coefficients(r @ r.T)
    assert abs(c.sum() - 1) < 1e-12
    # the minimiser of |sum c_i r_i| under sum c = 1
    g = r @ r.T
    ones = np.ones(4)
    w = np.linalg.solve(g / g.diagonal().max() + 1e-12 * np.eye(4), ones)
    assert np.allclose(c, w / w.sum(), atol=1e-9)


# ---- Fermi-Dirac occupations: the reference's own known answers (crates/qm/src/occupations.rs:474-612)
def test_fermi_dirac_known_answers(oracle):
    fd_known_answers.check(oracle.fermi_dirac)


def _xorshift_uniforms(seed):
    """A deterministic xorshift64* stream of uniforms in [0, 1) (the generator of the reference's sampling tests)."""
    s = seed

    def u():
        nonlocal s
        s ^= s >> 12
        s ^= (s << 25) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 27
        return (((s * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF) >> 11) / float(1 << 53)
    return u


def test_trilinear_known_answers(oracle):
    """trilinear_reproduces_a_linear_field_exactly_and_is_zero_outside (crates/qm/src/grid.rs:143-165): on the
    9^3 grid of spacing 0.5 ([-2, 2]^3) a linear field is reproduced to 1e-13 at random points; grid points,
    the 8 corners and a face centre return the stored value bitwise; points outside by a little or a lot, and
    NaN, give 0."""
    n, h = 9, 0.5
    xs = -2.0 + h * np.arange(n)
    z, y, x = np.meshgrid(xs, xs, xs, indexing="ij")
    lin = lambda p: 1.0 + 2.0 * p[..., 0] - p[..., 1] + 3.0 * p[..., 2]
    f = lin(np.stack([x, y, z], axis=-1)).reshape(-1)
    u = _xorshift_uniforms(0x5EED0001)
    pts = np.array([[-2.0 + 4.0 * u(), -2.0 + 4.0 * u(), -2.0 + 4.0 * u()] for _ in range(50)])
    got = oracle.trilinear(n, h, f, pts)
    assert np.max(np.abs(got - lin(pts))) <= 1e-13

    def idx(i, j, k):
        return i + n * (j + n * k)
    nodes = [(0, 0, 0), (3, 5, 7), (8, 0, 0), (0, 8, 0), (0, 0, 8), (8, 8, 0), (8, 0, 8), (0, 8, 8), (8, 8, 8), (8, 4, 4), (4, 4, 4)]
    pn = np.array([[xs[i], xs[j], xs[k]] for i, j, k in nodes])
    gn = oracle.trilinear(n, h, f, pn)
    for (i, j, k), v in zip(nodes, gn):
        assert v == f[idx(i, j, k)]
    outside = np.array([[2.0 + 1e-12, 0, 0], [-2.0 - 1e-12, 0, 0], [0, 2.5, 0], [0, -7.0, 0], [0, 0, 2.000001], [0, 0, -2.1],
                        [3.0, 3.0, 3.0], [np.nan, 0, 0]])
    assert np.all(oracle.trilinear(n, h, f, outside) == 0.0)
