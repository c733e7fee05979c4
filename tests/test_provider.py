"""The provider's evaluation semantics on the host (crates/providers/src/ks.rs): the cold retry of a failed warm solve
(retry_cold_on_stall, ks.rs:585-601) with fake solves, the solver footprint (ks_footprint_bytes; no GPU needed) and the
GPU-memory refusal before any solver is built (GpuKs::check_vram, ks.rs:1303-1324). CPU only."""
import pytest


def _drivers():
    import ks_b200 as ks
    import ks_drivers as kd
    return ks, kd


def _raiser(ks, kind, iterations, delta_rho):
    e = kind("failed")
    e.iterations, e.delta_rho = iterations, delta_rho
    return e


def test_retry_cold_on_stall_policy():
    ks, kd = _drivers()
    calls = []

    def script(outcomes):
        it = iter(outcomes)

        def solve(w):
            calls.append(w)
            o = next(it)
            if isinstance(o, Exception):
                raise o
            return o
        return solve

    # success: untouched, no stall
    calls.clear()
    assert kd.retry_cold_on_stall(True, script(["ok"])) == ("ok", None) and calls == [True]
    # a warm non-convergence: exactly one cold retry, its outcome returned with the stall record
    calls.clear()
    r, stall = kd.retry_cold_on_stall(True, script([_raiser(ks, ks.ScfNotConverged, 200, 3e-4), "cold"]))
    assert r == "cold" and calls == [True, False]
    assert stall == kd.Stall(200, 3e-4, False) and "did not converge" in stall.note() and "retried cold" in stall.note()
    # a warm stall: the same, marked stalled
    calls.clear()
    r, stall = kd.retry_cold_on_stall(True, script([_raiser(ks, ks.ScfStalled, 60, 1e-4), "cold"]))
    assert r == "cold" and stall.stalled and "stalled" in stall.note()
    # a cold failure is the first attempt's, untouched
    calls.clear()
    with pytest.raises(ks.ScfNotConverged):
        kd.retry_cold_on_stall(False, script([_raiser(ks, ks.ScfNotConverged, 200, 1e-3)]))
    assert calls == [False]
    # another error kind is not retried
    calls.clear()
    with pytest.raises(ks.Numerical):
        kd.retry_cold_on_stall(True, script([ks.Numerical("nan")]))
    assert calls == [True]
    # the retry's own failure propagates
    calls.clear()
    with pytest.raises(ks.ScfStalled):
        kd.retry_cold_on_stall(True, script([_raiser(ks, ks.ScfNotConverged, 200, 1e-3), _raiser(ks, ks.ScfStalled, 50, 2e-3)]))
    assert calls == [True, False]


def test_footprint_is_monotone_and_checked():
    ks, _ = _drivers()
    a = ks.footprint_bytes(95, 5, 5, n_extra=3)
    assert 600 * 2 ** 20 < a < 1000 * 2 ** 20  # ~805 MiB measured on B200 for H2O 95^3
    assert ks.footprint_bytes(128, 5, 5, n_extra=3) > a
    assert ks.footprint_bytes(95, 9, 9, n_extra=3) > a
    assert ks.footprint_bytes(95, 5, 5, n_extra=3, with_core=True) > a
    assert ks.footprint_bytes(95, 5, 0, n_extra=3) < a
    for bad in ((4, 1, 1), (95, -1, 1)):
        with pytest.raises(ValueError):
            ks.footprint_bytes(*bad)


def test_vram_budget_refuses_before_building_a_solver():
    ks, kd = _drivers()
    p = kd.GpuKs(n_extra=3).with_vram_budget(200 * 2 ** 20, "test share")
    with pytest.raises(ValueError, match=r"over the 0\.2 GB budget \(test share\)"):
        p.evaluate([(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)], 95, 0.25, 5, 5, ks.ScfSettings(sigma=0.5))
    assert p.solver is None
    p.check_vram(33, 5, 5, ks.ScfSettings(sigma=0.5))  # ~65 MiB fits
