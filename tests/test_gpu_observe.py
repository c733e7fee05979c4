"""GpuSolver::solve_observed / solve_polled on the GPU (crates/qm-gpu/src/scf.rs:1213-1235): the per-step observer
(qm::ScfProgress, its Harris-Foulkes energy) changes no number of the solve, and the inner cancellation point
abandons a solve inside an eigensolve with the iterate parked as the next warm start."""
import pytest

pytestmark = pytest.mark.gpu

WATER = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]


def test_observer_sees_every_step_and_changes_nothing(ks):
    settings = ks.ScfSettings(sigma=0.5)
    with ks.GpuSolver(48, 0.3, gram_mode=1, n_extra=3, init_mode=1) as so:
        plain = so.solve(ks.System(WATER, 5, 5), settings)
    seen = []
    with ks.GpuSolver(48, 0.3, gram_mode=1, n_extra=3, init_mode=1) as so:
        observed = so.solve(ks.System(WATER, 5, 5), settings, observe=seen.append)
    assert observed["energy"] == plain["energy"] and observed["iterations"] == plain["iterations"]
    assert [p["iteration"] for p in seen] == list(range(1, plain["iterations"] + 1))
    assert seen[-1]["delta_rho"] == plain["delta_rho"] and seen[-1]["tol"] == settings.tol
    assert all(p["max_iter"] == settings.max_iter and p["window"] == settings.stall_window for p in seen)
    best = [p["best_delta_rho"] for p in seen]
    assert all(b1 <= b0 for b0, b1 in zip(best, best[1:])) and best[-1] == min(p["delta_rho"] for p in seen)
    assert abs(seen[-1]["stall_level"] - 1e-3 * 10) < 1e-15
    # the Harris-Foulkes energy of the input density is stationary: at convergence it meets the total energy
    assert abs(seen[-1]["energy"] - plain["energy"]["total"]) < 1e-4, (seen[-1]["energy"], plain["energy"]["total"])


def test_inner_abort_lands_inside_an_eigensolve_and_parks_the_iterate(ks):
    settings = ks.ScfSettings(sigma=0.5)
    polls = []

    def inner():
        polls.append(1)
        return len(polls) >= 40
    steps = []
    with ks.GpuSolver(48, 0.3, gram_mode=1, n_extra=3, init_mode=1) as so:
        with pytest.raises(ks.Aborted, match="inside SCF step"):
            so.solve(ks.System(WATER, 5, 5), settings, inner_abort=inner, observe=steps.append)
        assert len(polls) == 40 and len(steps) < 20
        warm = so.solve(ks.System(WATER, 5, 5), settings, warm=True)
    with ks.GpuSolver(48, 0.3, gram_mode=1, n_extra=3, init_mode=1) as so:
        cold = so.solve(ks.System(WATER, 5, 5), settings)
    assert abs(warm["energy"]["total"] - cold["energy"]["total"]) < 1e-5


def test_density_extrapolation_in_md(ks):
    """GpuSolver::set_density_extrapolation (crates/qm-gpu/src/scf.rs:1146-1163) in velocity-Verlet MD: from the third
    solve on, the warm start extrapolates the last two converged densities; the trajectory is the one without it
    (every step converged to the same tolerance) and takes no more SCF steps."""
    import ks_drivers as drv
    nuc = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
    vel = [(0.0, 0.0, 0.0), (2e-4, 1e-4, 0.0), (-2e-4, 1e-4, 0.0)]
    settings = ks.ScfSettings(sigma=0.5, tol=1e-6)
    runs = {}
    for ex in (False, True):
        with ks.GpuSolver(48, 0.3, gram_mode=1, n_extra=3, init_mode=1) as so:
            runs[ex] = drv.velocity_verlet(so, nuc, 5, 5, settings, 20.0, 6, velocities=vel, extrapolate=ex)
    assert [r["extrapolated"] for r in runs[True]] == [False, False] + [True] * 5
    assert not any(r["extrapolated"] for r in runs[False])
    for a, b in zip(runs[False], runs[True]):
        assert abs(a["potential"] - b["potential"]) < 2e-5
    assert sum(r["iterations"] for r in runs[True]) <= sum(r["iterations"] for r in runs[False])


def test_effective_eig_tol_and_witness_cap(ks):
    with ks.GpuSolver(33, 0.25, n_extra=1) as so:
        assert so.effective_eig_tol(1e-3) == 1e-3
        floor = so.effective_eig_tol(1e-15)
        assert 1e-9 < floor < 1e-4
        so.set_witness_cap(1)
        # four up levels cannot hold the B atom's witness above its 2p triple, and the cap forbids growth
        with pytest.raises(ks.QmError) as err:
            so.solve(ks.System([(0.0, 0.0, 0.0, 5)], 3, 2), ks.ScfSettings(sigma=0.25, occupations="fermi_dirac", kt=5e-3))
        if isinstance(err.value, ks.Numerical):
            assert "witness cap of 1" in str(err.value)
