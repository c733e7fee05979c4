"""The provider's semantics on the GPU (crates/providers/src/ks.rs GpuKs): the footprint estimate against the device
memory a solve really takes, warm evaluations on one grid, the rebuild on a grid change and a pseudised scene."""
import pytest

import synthetic_species as ss

pytestmark = pytest.mark.gpu

WATER = [(0.0, 0.0, 0.0, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]


def test_footprint_matches_the_device_memory_of_a_solve(ks):
    """ks_footprint_bytes against cudaMemGetInfo around a solver's construction, solve and forces (after one solve has
    loaded the library's kernels): within -5 % / +25 % at 48^3 and 95^3."""
    import torch
    torch.zeros(1, device="cuda:0")
    settings = ks.ScfSettings(sigma=0.5, tol=1e-4)
    with ks.GpuSolver(33, 0.3, gram_mode=1, n_extra=3, init_mode=1) as so:
        so.solve(ks.System(WATER, 5, 5), settings)
        so.forces(WATER, 0.5)
    for n, h in ((48, 0.3), (95, 0.25)):
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info()
        with ks.GpuSolver(n, h, gram_mode=1, n_extra=3, init_mode=1) as so:
            so.solve(ks.System(WATER, 5, 5), settings)
            so.forces(WATER, 0.5)
            torch.cuda.synchronize()
            used = free0 - torch.cuda.mem_get_info()[0]
        est = ks.footprint_bytes(n, 5, 5, n_extra=3)
        assert 0.95 * used <= est <= 1.25 * used, (n, used, est)


def test_gpuks_warm_evaluations_and_grid_rebuild(ks):
    import ks_drivers as kd
    p = kd.GpuKs(n_extra=3)
    try:
        settings = ks.ScfSettings(sigma=0.5)
        a = p.evaluate(WATER, 33, 0.3, 5, 5, settings)
        first_solver = p.solver
        moved = [(0.0, 0.01, 0.0, 8)] + WATER[1:]
        b = p.evaluate(moved, 33, 0.3, 5, 5, settings)
        assert p.solver is first_solver and b["stats"]["iterations"] < a["stats"]["iterations"], "warm start on one grid"
        assert a["notes"] == [] and b["notes"] == []
        c = p.evaluate(WATER, 41, 0.3, 5, 5, settings)
        assert p.solver is not first_solver, "a grid change rebuilds the solver"
        # the 41^3 box (+-6 Bohr) confines the molecule less than the 33^3 one (+-4.8 Bohr): 0.03 Ha apart
        assert abs(c["energy"] - a["energy"]) < 5e-2 and c["forces"].shape == (3, 3)
        sp = [ss.oxygen_like(0.3)]
        d = p.evaluate(WATER, 33, 0.3, 4, 4, settings, species=sp)
        assert abs(d["stats"]["electrons"][0] - 4) < 1e-4
        e = p.evaluate(WATER, 33, 0.3, 4, 4, settings, species=sp)
        assert e["stats"]["iterations"] <= 3 and abs(e["energy"] - d["energy"]) < 1e-5
    finally:
        p.close()
