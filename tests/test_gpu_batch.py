"""ks_solve_batch: independent cold solves of many geometries in the library's own thread pool, each job's result
bit for bit that of a lone GpuSolver solve + forces, and a failing job reported in its own status while the others
run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_native_batch_equals_lone_solves(ks):
    import ks_drivers as drv
    jobs = drv.batch_workload(count=6, seed=11, n_min=40, n_max=56)
    for j in jobs:
        sys_ = ks.neutral_system(j["nuclei"])
        j["n_up"], j["n_dn"] = sys_.n_up, sys_.n_dn
        j["settings"] = ks.ScfSettings(sigma=0.5)
    bad = dict(jobs[0], nuclei=[(0.0, 0.0, 0.0, 1), (0.0, 0.0, 0.0, 1)], n_up=1, n_dn=1)
    tiny = dict(jobs[0], n=3)
    out = ks.solve_batch(jobs + [bad, tiny], workers=3)
    assert out[-2]["status"] == ks.KS_COINCIDENT_NUCLEI and "coincide" in out[-2]["error"]
    assert out[-1]["status"] == ks.KS_INVALID
    for j, r in zip(jobs, out):
        assert r["status"] == 0, r["error"]
        with ks.GpuSolver(j["n"], j["h"], gram_mode=1, n_extra=3, init_mode=1) as so:
            st = so.solve(ks.System(j["nuclei"], j["n_up"], j["n_dn"]), j["settings"])
            f = so.forces(j["nuclei"], 0.5)
        assert r["stats"]["energy"] == st["energy"] and r["stats"]["iterations"] == st["iterations"]
        assert np.array_equal(r["forces"], f)
