"""The MD driver's host logic (ks_drivers.velocity_verlet: kick-drift-kick velocity Verlet of crates/sim/src/integrator.rs,
one warm-started solve per step, the provider's cold retry of crates/providers/src/ks.rs:585-601) on a fake solver whose
potential is a harmonic H2 bond with exact forces. CPU only: the fake stands where GpuSolver stands."""
import numpy as np
import pytest


def _drivers():
    import ks_b200 as ks
    import ks_drivers as kd
    return ks, kd


class HarmonicBond:
    """E = k/2 (|r0 - r1| - d0)^2 with its exact forces, behind GpuSolver's methods. Records every solve's warm flag and
    raises `fail` (ScfStalled or ScfNotConverged) on the warm solve numbered in `fail_warm_calls` (1-based over all
    solve calls)."""

    def __init__(self, ks, k=0.37, d0=1.4, fail=None, fail_warm_calls=()):
        self.ks, self.k, self.d0 = ks, k, d0
        self.fail, self.fail_warm_calls = fail, set(fail_warm_calls)
        self.warm_flags, self.extrapolation = [], None

    def set_density_extrapolation(self, on):
        self.extrapolation = on

    def solve(self, system, settings, warm=False):
        self.warm_flags.append(warm)
        if warm and len(self.warm_flags) in self.fail_warm_calls:
            e = self.fail("warm solve failed")
            e.iterations, e.delta_rho = 50, 3e-4
            raise e
        r = np.array([a[:3] for a in system.nuclei], dtype=float)
        d = np.linalg.norm(r[0] - r[1])
        return {"energy": {"total": 0.5 * self.k * (d - self.d0) ** 2}, "iterations": 4 if warm else 9}

    def forces(self, nuclei, sigma):
        r = np.array([a[:3] for a in nuclei], dtype=float)
        u = r[0] - r[1]
        d = np.linalg.norm(u)
        f0 = -self.k * (d - self.d0) * u / d
        return np.array([f0, -f0])

    def profile(self):
        return {"extrapolated": 0}


def _run(kd, ks, solver, steps, dt, nuclei=None, velocities=None, **kw):
    nuclei = nuclei or [(0.8, 0.0, 0.0, 1), (-0.8, 0.0, 0.0, 1)]
    return kd.velocity_verlet(solver, nuclei, 1, 1, ks.ScfSettings(sigma=0.5), dt, steps, velocities=velocities, **kw)


def test_energy_is_conserved_to_second_order_in_dt():
    """A stretched bond oscillates (omega = sqrt(k / mu) = 0.020 au, period 313 au); over 8000 au the total energy's
    spread shrinks about 4x when dt halves from 5 to 2.5 au (velocity Verlet's O(dt^2) energy error), and it stays
    below 1 % of the oscillation's energy."""
    ks, kd = _drivers()
    spreads = []
    for dt in (5.0, 2.5):
        traj = _run(kd, ks, HarmonicBond(ks), int(8000 / dt), dt)
        e = np.array([t["total"] for t in traj])
        assert traj[0]["kinetic"] == 0.0 and traj[0]["potential"] > 0.0
        spreads.append(e.max() - e.min())
        assert spreads[-1] < 1e-2 * traj[0]["potential"]
    assert 3.0 < spreads[0] / spreads[1] < 5.0, spreads


def test_trajectory_is_time_reversible():
    """Run 200 steps, reverse the velocities, run 200 more: the nuclei return to the start (velocity Verlet is
    time-reversible) to rounding."""
    ks, kd = _drivers()
    fwd = _run(kd, ks, HarmonicBond(ks), 200, 15.0, velocities=[(0.0, 3e-4, 0.0), (0.0, -3e-4, 0.0)])
    end = fwd[-1]
    back = _run(kd, ks, HarmonicBond(ks), 200, 15.0, nuclei=[tuple(p) + (1,) for p in end["positions"]],
                velocities=-end["velocities"])
    assert np.max(np.abs(back[-1]["positions"] - fwd[0]["positions"])) < 1e-9
    assert np.max(np.abs(back[-1]["velocities"] + fwd[0]["velocities"])) < 1e-12


def test_warm_starts_and_the_cold_retry():
    """The first solve is cold and every later one warm; a warm solve that stalls (or does not converge) is retried
    cold once, that step is flagged, and the trajectory equals the one without the failure (the fake's energy does
    not depend on the start). Without the retry the failure propagates. The extrapolation switch is passed on."""
    ks, kd = _drivers()
    ref = _run(kd, ks, HarmonicBond(ks), 6, 20.0)
    for fail in (ks.ScfStalled, ks.ScfNotConverged):
        so = HarmonicBond(ks, fail=fail, fail_warm_calls=(3,))
        traj = _run(kd, ks, so, 6, 20.0, extrapolate=True)
        assert so.extrapolation is True
        assert so.warm_flags == [False, True, True, False, True, True, True, True]
        assert [t["cold_retry"] for t in traj] == [False, False, True, False, False, False, False]
        assert [t["iterations"] for t in traj] == [9, 4, 9, 4, 4, 4, 4]
        for a, b in zip(traj, ref):
            assert np.array_equal(a["positions"], b["positions"]) and a["total"] == b["total"]
    so = HarmonicBond(ks, fail=ks.ScfStalled, fail_warm_calls=(2,))
    with pytest.raises(ks.ScfStalled):
        _run(kd, ks, so, 3, 20.0, retry_cold=False)
