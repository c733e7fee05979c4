"""A sampling pass's warm path in a large box: all-electron H2 at 81^3 x 0.25 (20 Bohr), Fermi-Dirac at the reference's
defaults, cold at R = 1.4, then three displaced geometries each warm from the one before -- the reference's
warm_displaced_steps_take_the_lowest_converged_witness (crates/qm-gpu/src/scf.rs:2057-2085). On these warm steps the
top tested column leaves LOBPCG above 1.5 x the guard tolerance while a lower level has converged; the lowest converged
witness decides instead of growing the block one fresh box state at a time. The reference's bars: at least one lower
witness (the case is reached), at most one one-vector growth, a peak block of at most 8, and the last geometry's chain
energy within 1e-6 Ha of its own cold solve. That cold solve is also checked against a full f64 oracle SCF of the same
geometry (tests/golden/oracle_h2_81.json)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(__file__)
REC = json.load(open(os.path.join(HERE, "golden", "oracle_h2_81.json")))


def geometry(r, d):
    """Atom 0 at (R/2 + d0, d1, d2), atom 1 at (-R/2, -d1, 0.3 d2) (the reference test's geo)."""
    return [(0.5 * r + d[0], d[1], d[2], 1), (-0.5 * r, -d[1], 0.3 * d[2], 1)]


def test_warm_displaced_steps_take_the_lowest_converged_witness(ks):
    settings = ks.ScfSettings.for_grid(REC["h"])
    residual_growths = lower = peak = 0
    with ks.GpuSolver(REC["grid"], REC["h"], n_extra=1) as so:  # the reference's cold block: N_sigma + 1
        for i, (r, d) in enumerate(REC["path"]):
            st = so.solve(ks.System(geometry(r, d), 1, 1), settings, warm=i > 0)
            p = so.profile()
            residual_growths += p["witness_residual_growths"]
            lower += p["lower_witnesses"]
            peak = max(peak, p["peak_block"])
        last = st["energy"]["total"]
    nuc = geometry(*REC["path"][3])
    with ks.GpuSolver(REC["grid"], REC["h"], n_extra=1) as so:
        cold = so.solve(ks.System(nuc, 1, 1), settings)
        f = so.forces(nuc, REC["sigma"])
    assert lower >= 1, "the warm path no longer reaches a top above 1.5 g with a converged level below it"
    assert residual_growths <= 1, residual_growths
    assert peak <= 8, peak
    assert abs(last - cold["energy"]["total"]) < 1e-6, (last, cold["energy"]["total"])
    assert abs(cold["energy"]["total"] - REC["stats"]["total"]) < 1e-5, (cold["energy"]["total"], REC["stats"]["total"])
    assert np.abs(f - np.array(REC["forces"])).max() < 1e-4
