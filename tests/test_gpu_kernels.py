"""Kernel parity: every hot-path kernel of the CUDA library, called through the C ABI, against the
f64 oracle on the same seeded inputs. Bounds follow the reference's own GPU tests: end to end
(f64 input) and kernel-only (the oracle applied to the f32-rounded input the GPU sees)."""
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def f32(a):
    return np.asarray(a, dtype=np.float32).astype(np.float64)


def smooth_field(oracle, n, h, seed, centre=(0.3, -0.2, 0.1)):
    x, y, z = oracle.grid_points(n, h)
    rng = np.random.default_rng(seed)
    c = rng.standard_normal(4)
    r2 = (x - centre[0]) ** 2 + (y - centre[1]) ** 2 + (z - centre[2]) ** 2
    return (c[0] + c[1] * x + c[2] * y * z + c[3] * x * y) * np.exp(-r2 / 2)


def test_laplacian_matches_oracle_33(ks, oracle):
    """laplacian_matches_cpu_stencil (crates/qm-gpu/src/stencil.rs:150-171): 1e-5 end to end,
    1e-6 kernel-only, Gaussian on 33^3 at h = 0.25."""
    n, h = 33, 0.25
    x, y, z = oracle.grid_points(n, h)
    f = np.exp(-(x * x + y * y + z * z))
    gpu = ks.apply_laplacian(n, h, f)
    err = np.abs(gpu - oracle.laplacian(n, h, f)).max()
    err_kernel = np.abs(gpu - oracle.laplacian(n, h, f32(f))).max()
    assert err < 1e-5, err
    assert err_kernel < 1e-6, err_kernel


@pytest.mark.parametrize("n", [5, 6, 9, 17, 32, 33, 48, 50, 127, 128, 129, 200])
def test_hamiltonian_block_matches_oracle(ks, oracle, n):
    """H psi = -1/2 lap psi + V psi for a block of 3 vectors, every tile / chunk edge case of the
    TMA tiling (n below, at and above multiples of the 32 x 16 tile and of the pitch), down to the
    reference's smallest grid, n = 5 (crates/qm-gpu/src/grid.rs:200-211: the whole box inside one
    tile's halo, the pitch 8 > n), and up to the large grids of the configurations (127..129 around a
    multiple of every tile edge, 200 with several z-chunks per tile column)."""
    h = 0.3
    nuc = [(0.4, 0.0, -0.3, 3), (-1.1, 0.5, 0.2, 1)]
    v = f32(oracle.nuclear_potential(n, h, nuc, 0.5))
    psi = np.stack([f32(smooth_field(oracle, n, h, s)) for s in range(3)])
    gpu = ks.apply_hamiltonian(n, h, psi, v)
    for i in range(3):
        want = oracle.hamiltonian(n, h, psi[i], v)
        scale = np.abs(want).max() + np.abs(v * psi[i]).max()
        err = np.abs(gpu[i] - want).max()
        assert err < 1e-6 * scale, (i, err, scale)


def test_dirichlet_boundary_is_exact_zero_outside(ks, oracle):
    """A delta next to each face: the stencil reads zeros beyond the box (TMA out-of-bounds fill)
    and the result equals the oracle's bounds-checked stencil exactly up to f32 rounding."""
    n, h = 17, 0.25
    f = np.zeros(n ** 3)
    for (i, j, k) in ((0, 5, 7), (n - 1, 3, 2), (4, 0, 9), (6, n - 1, 1), (2, 8, 0), (11, 12, n - 1)):
        f[i + n * (j + n * k)] = 1.0
    gpu = ks.apply_laplacian(n, h, f)
    want = oracle.laplacian(n, h, f)
    assert np.abs(gpu - want).max() < 1e-6 * np.abs(want).max()


@pytest.mark.parametrize("n", [5, 25, 96, 129])
def test_precond_matches_oracle(ks, oracle, n):
    """precond_init + 3 jacobi_step sweeps (shaders/eigen.wgsl:25-34, stencil.wgsl:94-106), at the reference's
    smallest grid, a middle one and the large grids of the configurations (96, and 129 past a tile edge)."""
    h, lam = 0.25, -0.6
    v = f32(oracle.nuclear_potential(n, h, [(0.0, 0.0, 0.0, 2)], 0.5))
    r = f32(smooth_field(oracle, n, h, 4))
    gpu = ks.apply_precond(n, h, v, lam, r)
    want = oracle.jacobi_precond(n, h, v, lam, r)
    assert np.abs(gpu - want).max() < 2e-6 * np.abs(want).max()


def test_xc_matches_oracle(ks, oracle):
    """xc_lsda (crates/qm-gpu/src/physics.rs:243-260 bounds): relative 3e-6 or absolute 1e-8,
    vacuum points exactly zero."""
    rng = np.random.default_rng(3)
    up = f32(10 ** rng.uniform(-12, 1, 4000))
    dn = f32(10 ** rng.uniform(-12, 1, 4000))
    dn[:500] = 0.0
    up[500:600] = 0.0
    up[600:650] = 0.0
    dn[600:650] = 0.0
    e, vu, vd = ks.xc_lsda(up, dn)
    we, wvu, wvd = oracle.lsda(up, dn)
    for got, want in ((e, we), (vu, wvu), (vd, wvd)):
        abs_err = np.abs(got - want)
        ok = (abs_err <= 3e-6 * np.abs(want)) | (abs_err <= 1e-8)
        assert ok.all(), abs_err[~ok][:5]
    assert (e[600:650] == 0).all() and (vu[600:650] == 0).all() and (vd[600:650] == 0).all()


def test_nuclear_potential_matches_oracle(ks, oracle):
    """nuclear_potential (crates/qm-gpu/src/physics.rs:150-205): |dV| < 3e-7 max|V|, on-site limit."""
    n, h, sigma = 33, 0.25, 0.4
    nuc = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
    gpu = ks.nuclear_potential(n, h, nuc, sigma)
    want = oracle.nuclear_potential(n, h, nuc, sigma)
    assert np.abs(gpu - want).max() < 3e-7 * np.abs(want).max()


def test_poisson_matches_analytic_and_oracle(ks, oracle):
    """GpuPoisson on an off-centre Gaussian (crates/qm-gpu/src/poisson.rs:406-520): V within 1e-4 of
    q erf(r/(sigma sqrt2))/r, within the f32 floor of the oracle's f64 solve, true residual reported."""
    from scipy.special import erf
    n, h, sigma = 49, 0.25, 0.5
    x, y, z = oracle.grid_points(n, h)
    c = (1.3, -0.7, 0.4)
    r = np.sqrt((x - c[0]) ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2)
    rho = (2 * math.pi * sigma ** 2) ** -1.5 * np.exp(-r ** 2 / (2 * sigma ** 2))
    exact = erf(r / (sigma * math.sqrt(2))) / r
    v, it, res = ks.poisson_solve(n, h, rho, tol=1e-8)
    assert res < 3e-5, res
    assert 3 <= it < 60, it
    assert np.abs(v - exact).max() < 1e-4
    vo, _, _ = oracle.poisson_solve(n, h, rho, tol=1e-10)
    assert np.abs(v - vo).max() < 2e-5
    # warm start from the converged V takes fewer iterations (warm_start_reduces_iterations)
    _, it2, res2 = ks.poisson_solve(n, h, rho, v0=v, tol=1e-8)
    assert it2 < it and res2 < 3e-5


def test_multipole_moments_match_oracle(ks, oracle):
    n, h = 33, 0.25
    rho = np.abs(f32(smooth_field(oracle, n, h, 9, centre=(0.8, -0.5, 0.3))))
    q = ks.multipole_moments(n, h, rho)
    want = oracle.multipole_moments(n, h, rho)
    x, y, z = oracle.grid_points(n, h)
    rr = np.sqrt(x * x + y * y + z * z)
    for l in range(7):
        scale = np.sum(rho * rr ** l) * h ** 3
        for m in range(-l, l + 1):
            i = l * l + l + m
            assert abs(q[i] - want[i]) <= 1e-9 * scale + 1e-12, (l, m, q[i], want[i])


def test_gram_matches_numpy(ks, oracle):
    """The Gram block S^T [S | T] (crates/qm-gpu/src/reduce.rs:340-420): ~1e-6 relative of the f64
    products of the f32 inputs."""
    n = 29
    rng = np.random.default_rng(1)
    s = f32(rng.standard_normal((10, n ** 3)))
    t = f32(rng.standard_normal((7, n ** 3)))
    g = ks.gram(n, s, t)
    want = s @ np.concatenate([s, t]).T
    scale = np.sqrt(np.outer((s * s).sum(1), np.concatenate([(s * s).sum(1), (t * t).sum(1)])))
    assert np.abs(g - want).max() / scale.max() < 2e-6


def test_lobpcg_oscillator_matches_oracle(ks, oracle):
    """LOBPCG on the harmonic oscillator (crates/qm-gpu/src/eigen.rs:1009-1100): the GPU eigenvalues
    equal the oracle's f64 ones to 1e-5 on the same grid."""
    n, h = 33, 0.25
    x, y, z = oracle.grid_points(n, h)
    v = f32(0.5 * (x * x + y * y + z * z))
    rng = np.random.default_rng(5)
    guess = (rng.uniform(-0.5, 0.5, (4, n ** 3)) * np.exp(-(x * x + y * y + z * z) / 8.0))
    ev, xs, it, mr = ks.lobpcg(n, h, v, guess, tol=2e-5, max_iter=400)
    evo, _, _, _ = oracle.lobpcg(n, h, v, guess, tol=1e-8, max_iter=500, precond_lambda=1.5)
    assert np.abs(np.sort(ev) - np.sort(evo)).max() < 1e-5, (ev, evo)
    gm = xs @ xs.T * h ** 3
    assert np.abs(gm / np.sqrt(np.outer(gm.diagonal(), gm.diagonal())) - np.eye(4)).max() < 1e-5


@pytest.mark.parametrize("m,mt", [(8, 8), (24, 24), (10, 15), (60, 60)])
def test_tensor_core_gram_matches_numpy(ks, m, mt):
    """The 3xTF32 tcgen05 Gram (the "mixed" form): the same pairs as the CUDA-core Gram to ~1e-6
    relative, including blocks whose row counts are not multiples of 8 and the largest block (60)."""
    n = 33 if m < 60 else 21
    rng = np.random.default_rng(m + mt)
    s = f32(rng.standard_normal((m, n ** 3)))
    t = f32(rng.standard_normal((mt, n ** 3)))
    g = ks.gram(n, s, t, gram_mode=1)
    want = s @ np.concatenate([s, t]).T
    scale = np.sqrt(np.outer((s * s).sum(1), np.concatenate([(s * s).sum(1), (t * t).sum(1)])))
    err = np.abs(g - want).max() / scale.max()
    assert err < 2e-6, err


def test_lobpcg_tensor_core_gram_matches_oracle(ks, oracle):
    n, h = 33, 0.25
    x, y, z = oracle.grid_points(n, h)
    v = f32(0.5 * (x * x + y * y + z * z))
    rng = np.random.default_rng(5)
    guess = (rng.uniform(-0.5, 0.5, (4, n ** 3)) * np.exp(-(x * x + y * y + z * z) / 8.0))
    ev, xs, it, mr = ks.lobpcg(n, h, v, guess, tol=2e-5, max_iter=400, gram_mode=1)
    evo, _, _, _ = oracle.lobpcg(n, h, v, guess, tol=1e-8, max_iter=500, precond_lambda=1.5)
    assert np.abs(np.sort(ev) - np.sort(evo)).max() < 1e-5, (ev, evo)


def _check_rel(name, got, want, mag, rel=1e-6):
    """The reference's pointwise bound (crates/qm-gpu/src/pointwise.rs check: |gpu - cpu| <= 1e-6 * max(mag, 1e-6))."""
    bad = np.abs(got - want) > rel * np.maximum(mag, 1e-6)
    assert not bad.any(), (name, np.abs(got - want)[bad].max(), int(bad.sum()))


@pytest.mark.parametrize("n", [5, 17, 33])
def test_density_residual_matches_f64(ks, oracle, n):
    """The SCF's density step: rho_out = sum_i f_i psi_i^2 over three orbitals, r = rho_out - rho_in, and the step's
    reductions (h^3 sum |r|, h^3 sum rho_out), against the f64 formula on the f32-rounded inputs the kernel sees, to
    the reference's pointwise bound (axpy_scale_lincomb_mul_density_match_cpu, crates/qm-gpu/src/pointwise.rs:329-438,
    its mul_add_sq case): once with Fermi-Dirac weights (f32 on the device) and once with f = 1."""
    h = 0.3
    psi = np.stack([smooth_field(oracle, n, h, 40 + i, centre=(0.1 * i, -0.2, 0.3)) for i in range(3)])
    x, y, z = oracle.grid_points(n, h)
    rho_in = 0.2 * np.exp(-(x * x + y * y + z * z) / 3)
    p32, rin32 = f32(psi), f32(rho_in)
    for f in ([1.0, 0.6, 0.05], None):
        w = np.ones(3) if f is None else f32(f)
        out, r, sums = ks.density_residual(n, h, psi, rho_in, f=f)
        want = (w[:, None] * p32 * p32).sum(0)
        mag = (np.abs(w)[:, None] * p32 * p32).sum(0)
        _check_rel("rho_out", out, want, mag)
        _check_rel("r", r, want - rin32, mag + np.abs(rin32))
        # the reductions read the device's own rho_out and r (f32), summed in f64
        assert abs(sums[0] - h ** 3 * np.abs(f32(r)).sum()) <= 1e-12 * max(1.0, sums[0]), (sums[0], h ** 3 * np.abs(r).sum())
        assert abs(sums[1] - h ** 3 * f32(out).sum()) <= 1e-12 * max(1.0, sums[1]), (sums[1], h ** 3 * out.sum())
    out, r, sums = ks.density_residual(n, h, np.zeros((0, n ** 3)), rho_in)  # an empty channel: rho_out = 0
    assert np.all(out == 0.0) and np.allclose(r, -rin32, rtol=0, atol=0)


@pytest.mark.parametrize("m", [1, 3, 6])
def test_diis_mix_matches_oracle_step(ks, oracle, m):
    """The SCF's Pulay mix with the oracle's coefficients (oracle.diis_coefficients on the residuals' Gram) against the
    oracle's own mix step, max(sum_e c_e (rho_e + alpha r_e), 0) (oracle/ks_oracle.cpp diis_mix, crates/qm/src/scf.rs),
    to the reference's pointwise bound (crates/qm-gpu/src/pointwise.rs diis_mix case: 1e-6 of the terms' magnitude);
    with one and three entries the mixed density goes negative somewhere, so the clamp at 0 is exercised (six entries
    cancel the residuals too well for that)."""
    n, h, alpha = 17, 0.3, 0.3
    x, y, z = oracle.grid_points(n, h)
    rng = np.random.default_rng(0xD115 + m)
    base = np.exp(-(x * x + y * y + z * z) / 2)
    rho = np.stack([base * (1.0 + 0.05 * rng.standard_normal()) + 0.01 * smooth_field(oracle, n, h, 60 + e) for e in range(m)])
    r = np.stack([0.5 * smooth_field(oracle, n, h, 80 + e) for e in range(m)])
    c = oracle.diis_coefficients(np.array([[h ** 3 * (r[i] * r[j]).sum() for j in range(m)] for i in range(m)]))
    assert c is not None and abs(c.sum() - 1.0) < 1e-12
    out = ks.diis_mix(n, rho, r, c[:-1], alpha * c)
    rho32, r32 = f32(rho), f32(r)
    want = np.maximum((c[:, None] * (rho32 + alpha * r32)).sum(0), 0.0)
    b = rho32[-1]
    mag = np.abs(b) + (np.abs(c[:-1, None]) * np.abs(rho32[:-1] - b)).sum(0) + (alpha * np.abs(c[:, None] * r32)).sum(0)
    _check_rel("diis_mix", out, want, mag)
    if m < 6:
        assert (want == 0.0).any() and (out == 0.0).any(), "the clamp must be exercised"
    assert np.all(out >= 0.0)
