"""Failure paths and the saved-state warm start, through the C ABI on the B200, as the reference tests them:

- a NaN in the parked warm density is a Numerical error, not a crash, and the solver recovers
  (nan_density_returns_numerical_error_not_panic, crates/qm-gpu/src/scf.rs:2400-2420);
- a readback that never delivers is a Device error wherever in the solve it strikes, the failed solve leaves no
  state, and the next solve is bit for bit a fresh solver's (a_failed_readback_is_a_device_error_wherever_it_strikes,
  scf.rs:2422-2460, with the reference's per-readback fault hook crates/gpu/src/readback.rs:36-58);
- a state exported from one solver and imported into another resumes warm (the parked GpuState, scf.rs:1286-1323).

The failures are injected on the host (a NaN written into a field, a readback reported as lost): no GPU fault."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N, H = 33, 0.25


def _hydrogen(ks):
    return ks.System([(0.0, 0.0, 0.0, 1)], 1, 0)


def _h2(ks):
    return ks.System([(0.7, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)], 1, 1)


def test_nan_density_returns_numerical_error_not_panic(ks):
    """A NaN written into the parked warm density reaches the first Poisson solve of the next warm solve: the solve
    ends in Numerical inside its first SCF step, exposes no state and parks nothing, so the next warm request runs
    cold and is bit-identical to a fresh solver's cold solve."""
    st = ks.ScfSettings(sigma=H, tol=1e-6)
    sys_ = _hydrogen(ks)
    with ks.GpuSolver(N, H) as so:
        so.solve(sys_, st)
        so.poison_parked_density()
        with pytest.raises(ks.Numerical):
            so.solve(sys_, st, warm=True)
        assert so.profile()["steps"] == 1, so.profile()
        with pytest.raises(ks.NoState):
            so.counts()
        after = so.solve(sys_, st, warm=True)
        assert so.profile()["start_s"] > 0.0, "the warm request after a failure must run cold"
    with ks.GpuSolver(N, H) as fresh:
        ref = fresh.solve(sys_, st)
    assert after["energy"]["total"] == ref["energy"]["total"], (after["energy"]["total"], ref["energy"]["total"])


def test_a_failed_readback_is_a_device_error_wherever_it_strikes(ks):
    """The first, second, ..., last readback of a solve fails in turn: each solve ends in Device (never a success on
    the zeros a lost readback would give), leaves no state, and the solve after the failures is bit-identical to the
    undisturbed one. forces reports a lost readback too, and works again once the hook is cleared."""
    st = ks.ScfSettings(sigma=H, tol=1e-6)
    sys_ = _hydrogen(ks)
    with ks.GpuSolver(N, H) as so:
        ref = so.solve(sys_, st)
        total = so.profile()["readbacks"]
        assert total > 10, total
        for skip in sorted({0, 1, 2, 3, total // 4, total // 2, total - 3, total - 1}):
            so.fail_readbacks(skip, 1)
            with pytest.raises(ks.Device, match="did not deliver"):
                so.solve(sys_, st)
            so.fail_readbacks(0, 0)
            with pytest.raises(ks.NoState):
                so.counts()
        after = so.solve(sys_, st, warm=True)
        assert after["energy"]["total"] == ref["energy"]["total"], "the solve after the failures must be a cold one"
        so.fail_readbacks(0, 1)
        with pytest.raises(ks.Device):
            so.forces(sys_.nuclei, st.sigma)
        so.fail_readbacks(0, 0)
        f = so.forces(sys_.nuclei, st.sigma)
        assert np.all(np.isfinite(f))


def test_imported_state_resumes_warm(ks):
    """H2 on 33^3: the state of a converged solve (orbitals, levels, densities, V_H) exported through the getters and
    imported into a fresh solver makes its next warm solve converge in a few steps to the same energy (within the
    f32 noise of a warm re-solve, 1e-7 Ha) -- and an import fully defines the warm start: importing the same state
    into the first solver gives a bit-identical warm solve."""
    st = ks.ScfSettings(sigma=H, tol=1e-6)
    sys_ = _h2(ks)
    with ks.GpuSolver(N, H, n_extra=3) as a:
        cold = a.solve(sys_, st)
        up, dn = a.evals()
        saved = dict(orbitals=(a.orbitals(0), a.orbitals(1)), evals=(up, dn), density=a.density(), v_h=a.potentials()[1])
        with ks.GpuSolver(N, H, n_extra=3) as b:
            b.import_state(1, 1, **saved)
            with pytest.raises(ks.NoState):
                b.counts()  # an imported warm start is not a converged state
            warm_b = b.solve(sys_, st, warm=True)
            assert b.profile()["start_s"] == 0.0, "the imported state must be used as a warm start"
        a.import_state(1, 1, **saved)
        warm_a = a.solve(sys_, st, warm=True)
    assert warm_b["iterations"] <= 4, warm_b["iterations"]
    assert abs(warm_b["energy"]["total"] - cold["energy"]["total"]) < 1e-6
    assert warm_a["energy"]["total"] == warm_b["energy"]["total"]
    assert warm_a["iterations"] == warm_b["iterations"]


def test_state_import_refuses_inconsistent_sizes(ks):
    """Fewer orbitals than occupied levels, or more than the block holds, are argument errors."""
    n3 = N ** 3
    z = np.zeros(n3)
    with ks.GpuSolver(N, H, n_extra=1) as so:
        with pytest.raises(ValueError):
            so.import_state(2, 1, (np.zeros((1, n3)), np.zeros((1, n3))), (np.zeros(1), np.zeros(1)), (z, z), z)
        with pytest.raises(ValueError):
            so.import_state(1, 1, (np.zeros((3, n3)), np.zeros((1, n3))), (np.zeros(3), np.zeros(1)), (z, z), z)
