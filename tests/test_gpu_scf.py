"""SCF parity through the C ABI: the CUDA solver against the reference's pinned answers and the
oracle, plus the solver's contract (determinism, warm start, abort, errors)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_pins.json")))


def _system(ks, spec):
    return ks.System([tuple(x) for x in spec["nuclei"]], spec["n_up"], spec["n_dn"])


@pytest.mark.parametrize("name", ["H2", "LiH"])
def test_scf_matches_reference_pins_33(ks, oracle, name):
    """The 33^3 Aufbau pins (crates/qm/src/scf.rs:1276-1279): |dE| < 1e-5 Ha, |dF| < 1e-4 Ha/Bohr,
    occupied eigenvalues within 1e-5 Ha of the oracle's."""
    spec = GOLDEN["pins_33"][name]
    sys_ = _system(ks, spec)
    with ks.GpuSolver(33, 0.25) as so:
        st = so.solve(sys_, ks.ScfSettings(sigma=0.25, tol=1e-6))
        f = so.forces(sys_.nuclei, 0.25)
        ev_up, ev_dn = so.evals()
    assert abs(st["energy"]["total"] - spec["energy"]) < 1e-5, st
    assert abs(f[0, 0] - spec["force_x0"]) < 1e-4, f
    ost, ostats = oracle.scf(33, 0.25, sys_.nuclei, sys_.n_up, sys_.n_dn, sigma=0.25, tol=1e-6)
    o_up, o_dn = ost.evals()
    assert np.abs(np.sort(ev_up) - np.sort(o_up)).max() < 1e-5
    assert np.abs(np.sort(ev_dn) - np.sort(o_dn)).max() < 1e-5
    of = oracle.forces(ost, sys_.nuclei, 0.25)
    assert np.abs(f - of).max() < 1e-4
    assert abs(st["electrons"][0] - sys_.n_up) < 1e-5 and abs(st["electrons"][1] - sys_.n_dn) < 1e-5


def test_scf_is_deterministic(ks):
    spec = GOLDEN["pins_33"]["H2"]
    sys_ = _system(ks, spec)
    with ks.GpuSolver(33, 0.25) as a:
        e1 = a.solve(sys_, ks.ScfSettings(sigma=0.25))["energy"]["total"]
        e2 = a.solve(sys_, ks.ScfSettings(sigma=0.25))["energy"]["total"]
    with ks.GpuSolver(33, 0.25) as b:
        e3 = b.solve(sys_, ks.ScfSettings(sigma=0.25))["energy"]["total"]
    assert e1 == e2 == e3


def test_warm_start_takes_fewer_steps(ks):
    """warm_start_converges_in_few_iterations (crates/qm/src/scf.rs:1217-1235)."""
    nuc0 = [(0.0, 0.0, 0.0, 1)]
    nuc1 = [(0.02, 0.0, 0.0, 1)]
    with ks.GpuSolver(33, 0.25) as so:
        so.solve(ks.System(nuc0, 1, 0), ks.ScfSettings())
        warm = so.solve(ks.System(nuc1, 1, 0), ks.ScfSettings(), warm=True)
    with ks.GpuSolver(33, 0.25) as so2:
        cold = so2.solve(ks.System(nuc1, 1, 0), ks.ScfSettings())
    assert warm["iterations"] < cold["iterations"]
    assert abs(warm["energy"]["total"] - cold["energy"]["total"]) < 1e-5


def test_abort_parks_the_iterate_and_resumes(ks):
    calls = {"n": 0}

    def stop_after_three():
        calls["n"] += 1
        return calls["n"] > 3

    sys_ = _system(ks, GOLDEN["pins_33"]["H2"])
    with ks.GpuSolver(33, 0.25) as so:
        with pytest.raises(ks.Aborted):
            so.solve(sys_, ks.ScfSettings(sigma=0.25), should_abort=stop_after_three)
        with pytest.raises(ks.NoState):
            so.forces(sys_.nuclei)
        st = so.solve(sys_, ks.ScfSettings(sigma=0.25), warm=True)
    assert abs(st["energy"]["total"] - GOLDEN["pins_33"]["H2"]["energy"]) < 1e-5


def test_coincident_nuclei_is_an_error(ks):
    with ks.GpuSolver(17, 0.3) as so:
        with pytest.raises(ks.CoincidentNuclei):
            so.solve(ks.System([(0.1, 0, 0, 1), (0.1, 0, 0, 1)], 1, 1), ks.ScfSettings())


def test_not_converged_within_the_cap(ks):
    sys_ = _system(ks, GOLDEN["pins_33"]["H2"])
    with ks.GpuSolver(33, 0.25) as so:
        with pytest.raises(ks.ScfNotConverged):
            so.solve(sys_, ks.ScfSettings(max_iter=2))


@pytest.mark.parametrize("name", ["H2", "LiH"])
def test_scf_mixed_precision_matches_reference_pins_33(ks, name):
    """The mixed form (tensor-core 3xTF32 Gram) meets the same bars as plain FP32."""
    spec = GOLDEN["pins_33"][name]
    sys_ = _system(ks, spec)
    with ks.GpuSolver(33, 0.25, gram_mode=1) as so:
        st = so.solve(sys_, ks.ScfSettings(sigma=0.25, tol=1e-6))
        f = so.forces(sys_.nuclei, 0.25)
    assert abs(st["energy"]["total"] - spec["energy"]) < 1e-5, st
    assert abs(f[0, 0] - spec["force_x0"]) < 1e-4, f


H2O95 = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_h2o95.json")))


@pytest.mark.parametrize("gram_mode", [0, 1])
def test_h2o_95_matches_oracle_record(ks, gram_mode):
    """The timed workload (H2O, 95^3, h = 0.25, sigma = 0.5, tol 1e-6) against a full oracle SCF of
    it (tests/golden/oracle_h2o95.json): |dE| < 1e-5 Ha, occupied eigenvalues within 1e-5 Ha and
    forces within 1e-4 Ha/Bohr, for the all-CUDA-core form and the tensor-core Gram form."""
    nuc = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
    with ks.GpuSolver(95, 0.25, gram_mode=gram_mode, n_extra=3, init_mode=1) as so:
        st = so.solve(ks.System(nuc, 5, 5), ks.ScfSettings(sigma=0.5, tol=1e-6))
        f = so.forces(nuc, 0.5)
        ev_up, ev_dn = so.evals()
    assert abs(st["energy"]["total"] - H2O95["stats"]["total"]) < 1e-5, st["energy"]
    assert np.abs(np.sort(ev_up)[:5] - np.array(H2O95["evals_up"])).max() < 1e-5
    assert np.abs(np.sort(ev_dn)[:5] - np.array(H2O95["evals_dn"])).max() < 1e-5
    assert np.abs(f - np.array(H2O95["forces"])).max() < 1e-4


def test_density_into_caller_buffers(ks):
    """GpuSolver.density(out=...) fills the caller's float64 arrays (here page-locked, as the bench's end-to-end
    readback uses them) with the same bits as a fresh readback, and refuses arrays of the wrong size or type."""
    import torch
    n = 33
    with ks.GpuSolver(n, 0.25) as so:
        so.solve(ks.System([(0.7, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)], 1, 1), ks.ScfSettings(sigma=0.25, tol=1e-6))
        up, dn = so.density()
        out = tuple(torch.empty(n ** 3, dtype=torch.float64, pin_memory=True).numpy() for _ in range(2))
        got = so.density(out=out)
        assert got[0] is out[0] and got[1] is out[1]
        assert np.array_equal(out[0], up) and np.array_equal(out[1], dn)
        with pytest.raises(ValueError):
            so.density(out=(np.empty(n ** 3), np.empty(n ** 3 - 1)))
        with pytest.raises(ValueError):
            so.density(out=(np.empty(n ** 3, dtype=np.float32), np.empty(n ** 3)))
