"""The all-electron H3+ with its 0-2 pair stretched to 1.6 r0, 49^3 x 0.25, Fermi-Dirac at the reference's defaults
(ScfSettings::for_grid), cold: the case of the reference's gpu_fd_stretched_h3plus_converges_cold
(crates/qm-gpu/src/scf.rs:2014-2043). Its diffuse witness column is what the split stop test, the locked head, the
buffer column and the frozen-step DIIS rules exist for: with one block-wide residual the steps alternated between
0 and ~25 LOBPCG iterations, reset DIIS every other step and cycled to the 200-step cap. The reference's bars: at most
20 steps, at most one DIIS reset, a second cold solve bitwise the same. Here the energy and forces are also checked
against a full f64 oracle SCF of the same case (tests/golden/oracle_h3plus_49.json)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REC = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_h3plus_49.json")))


@pytest.mark.parametrize("gram_mode", [0, 1])  # the plain and the mixed (tensor-core Gram) form
def test_stretched_h3plus_converges_cold(ks, gram_mode):
    nuc = [tuple(a) for a in REC["nuclei"]]
    settings = ks.ScfSettings.for_grid(REC["h"])
    system = ks.System(nuc, REC["n_up"], REC["n_dn"])
    with ks.GpuSolver(REC["grid"], REC["h"], gram_mode=gram_mode, n_extra=1) as so:  # the reference's cold block: N_sigma + 1
        a = so.solve(system, settings)
        p = so.profile()
        f = so.forces(nuc, REC["sigma"])
        b = so.solve(system, settings)
    assert a["iterations"] <= 20, (a["iterations"], p)
    assert p["diis_resets"] <= 1, p
    assert (a["energy"]["total"], a["delta_rho"], a["iterations"]) == (b["energy"]["total"], b["delta_rho"], b["iterations"]), \
        "cold solves are bitwise reproducible"
    ref = REC["stats"]
    assert abs(a["energy"]["total"] - ref["total"]) < 1e-5, (a["energy"]["total"], ref["total"])
    assert abs(a["energy"]["ts"] - ref["ts"]) < 1e-6, (a["energy"]["ts"], ref["ts"])
    assert np.abs(f - np.array(REC["forces"])).max() < 1e-4
