"""Readouts of a converged state on the GPU against the oracle: trilinear sampling
(crates/qm-gpu/src/sample.rs tests gpu_sampling_matches_the_cpu_trilinear_to_f32 and sampling_reads_back_once),
the headless density volume, its maximum and the spin integral (crates/qm-gpu/src/scf.rs:1776-1842)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, H = 25, 0.25                 # [-3, 3]^3
NUC = [(0.13, -0.21, 0.05, 1)]  # one H atom, spin up


def _uniforms(seed):
    s = seed

    def u():
        nonlocal s
        s ^= s >> 12
        s ^= (s << 25) & 0xFFFFFFFFFFFFFFFF
        s ^= s >> 27
        return (((s * 0x2545F4914F6CDD1D) & 0xFFFFFFFFFFFFFFFF) >> 11) / float(1 << 53)
    return u


@pytest.fixture(scope="module")
def h_atom(ks):
    so = ks.GpuSolver(N, H, gram_mode=1, n_extra=3)
    so.solve(ks.System(NUC, 1, 0), ks.ScfSettings(sigma=H, tol=1e-5))
    yield so
    so.close()


def _check(points, gpu, cpu):
    bound = 1e-6 * np.maximum(1.0, np.abs(cpu))
    d = np.abs(gpu.astype(np.float64) - cpu)
    assert np.all(d <= bound), (points[np.argmax(d / bound)], float(np.max(d / bound)))
    return float(np.max(d / bound))


def test_sampling_matches_the_oracle_trilinear(ks, oracle, h_atom):
    """300 points: 270 random in the box (90 of them within 0.6 Bohr of the nucleus), 20 outside (6 by 1e-9
    Bohr), 10 grid points (corners and faces among them). |gpu - cpu| <= 1e-6 max(1, rho) against the oracle's
    f64 trilinear of the same f32 values; outside exactly 0; a grid point returns the stored f32 exactly."""
    so = h_atom
    rho32 = so.density_f32()
    rho = rho32.astype(np.float64)
    u = _uniforms(0x5A31E5)
    half = 3.0
    pts = np.array([[half * (2 * u() - 1), half * (2 * u() - 1), half * (2 * u() - 1)] for _ in range(270)])
    for p in pts[:90]:
        for c in range(3):
            p[c] = NUC[0][c] + 0.6 * (2 * u() - 1)
    outside = []
    for i in range(20):
        p = [half * (2 * u() - 1), half * (2 * u() - 1), half * (2 * u() - 1)]
        axis, sign = i % 3, (1.0 if i % 2 == 0 else -1.0)
        p[axis] = sign * (half + (1e-9 if i < 6 else 0.5 + 4.0 * u()))
        outside.append(p)
    nodes = [(12, 12, 12), (0, 0, 0), (24, 24, 24), (24, 0, 12), (13, 11, 12), (0, 24, 3), (5, 6, 7), (12, 12, 24), (24, 12, 12),
             (1, 23, 17)]
    grid = -3.0 + H * np.arange(N)
    node_pts = [[grid[i], grid[j], grid[k]] for i, j, k in nodes]
    allp = np.vstack([pts, np.array(outside), np.array(node_pts)])
    r0, _ = so.sampling_counters()
    gpu = so.sample_density(allp)
    assert so.sampling_counters()[0] == r0 + 1, "one readback per call"
    _check(allp[:270], gpu[:270], oracle.trilinear(N, H, rho, allp[:270]))
    assert np.all(gpu[270:290] == 0.0)
    for (i, j, k), v in zip(nodes, gpu[290:]):
        assert v == rho32[i + N * (j + N * k)]
    assert gpu.max() > 0.1, "an H atom's density was sampled"


def test_sampling_every_node_is_exact_and_buffers_are_reused(ks, h_atom):
    """All n^3 grid points return the stored field exactly; a smaller call reuses the buffers, a larger one grows
    them once; no points, no GPU work; the same points give the same values."""
    so = h_atom
    rho32 = so.density_f32()
    g = -3.0 + H * np.arange(N)
    z, y, x = np.meshgrid(g, g, g, indexing="ij")
    nodes = np.stack([x.reshape(-1), y.reshape(-1), z.reshape(-1)], axis=1)
    r0, a0 = so.sampling_counters()
    assert len(so.sample_density(np.empty((0, 3)))) == 0
    assert so.sampling_counters() == (r0, a0), "no points, no GPU work"
    allv = so.sample_density(nodes)
    assert np.array_equal(allv, rho32)
    r1, a1 = so.sampling_counters()
    again = so.sample_density(nodes[:1000])
    assert np.array_equal(again, allv[:1000])
    assert so.sampling_counters() == (r1 + 1, a1), "a smaller call reuses the buffers"
    more = so.sample_density(np.vstack([nodes, nodes]))
    assert np.array_equal(more[len(nodes):], allv)
    assert so.sampling_counters() == (r1 + 2, a1 + 1), "a larger call grows them once"


def test_volume_max_and_spin_integral(ks, h_atom):
    """The headless volume is the stored density exactly (written on a foreign stream, ordered after the solver);
    density_max is its maximum; the spin integral is the f64 sum of |rho_up - rho_dn| h^3 (one electron, fully
    polarised: equal to the total charge)."""
    import torch
    so = h_atom
    rho32 = so.density_f32()
    vol = torch.full((N ** 3,), float("nan"), dtype=torch.float32, device="cuda:0")
    side = torch.cuda.Stream(device="cuda:0")
    so.copy_density_to_volume(vol.data_ptr(), side.cuda_stream)
    side.synchronize()
    assert np.array_equal(vol.cpu().numpy(), rho32)
    assert so.density_max() == float(rho32.max())
    up, dn = so.density()
    want = float(np.sum(np.abs(up - dn))) * H ** 3
    got = so.spin_abs_integral()
    assert abs(got - want) <= 1e-12 * max(1.0, abs(want)), (got, want)
    assert abs(got - 1.0) < 1e-3
