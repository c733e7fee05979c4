"""Fermi-Dirac occupations (crates/qm/src/occupations.rs, the first of the SCF's next rows) through the
C ABI against full oracle SCFs (tests/golden/oracle_fd.json): the B atom, whose 2p triple holds 2 and
1 electrons fractionally (f = 2/3 and 1/3), and LiH (gapped), both at kT = 5e-3 Ha on 33^3 with
4 extra levels per channel."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
REC = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_fd.json")))


@pytest.mark.parametrize("name", ["B", "LiH"])
def test_fermi_dirac_scf_matches_oracle(ks, name):
    case = REC["cases"][name]
    nuc = [tuple(a) for a in case["nuclei"]]
    settings = ks.ScfSettings(sigma=REC["sigma"], tol=REC["tol"], occupations="fermi_dirac", kt=REC["kt"])
    with ks.GpuSolver(REC["grid"], REC["h"], n_extra=REC["n_extra"]) as so:
        st = so.solve(ks.System(nuc, case["n_up"], case["n_dn"]), settings)
        fu, fd = so.occupations()
        eu, ed = so.evals()
        f = so.forces(nuc, REC["sigma"])
        g, _ = so.vjp(nuc, REC["sigma"])
    ref = case["stats"]
    assert abs(st["energy"]["total"] - ref["total"]) < 1e-5, (st["energy"], ref["total"])
    assert abs(st["energy"]["ts"] - ref["ts"]) < 1e-6, (st["energy"]["ts"], ref["ts"])
    assert abs(st["entropy"] - ref["entropy"]) < 1e-3
    # at least N_sigma + n_extra levels: a buffer column whose own bound passes above the guard tolerance grows the block
    # by one (crates/qm-gpu/src/scf.rs:993-1012); the levels past the five that carry weight hold no charge
    assert len(fu) >= case["n_up"] + REC["n_extra"] and len(fd) >= case["n_dn"] + REC["n_extra"]
    assert fu[5:].max() < 1e-6 and fd[5:].max() < 1e-6
    assert abs(fu.sum() - case["n_up"]) < 1e-9 and abs(fd.sum() - case["n_dn"]) < 1e-9
    k = 5  # the levels that carry weight
    assert np.abs(eu[:k] - np.array(case["evals_up"][:k])).max() < 1e-5
    assert np.abs(ed[:k] - np.array(case["evals_dn"][:k])).max() < 1e-5
    assert np.abs(fu[:k] - np.array(case["occ_up"][:k])).max() < 1e-4
    assert np.abs(fd[:k] - np.array(case["occ_dn"][:k])).max() < 1e-4
    assert np.abs(f - np.array(case["forces"])).max() < 1e-4
    assert np.abs(g + f).max() < 1e-6  # the adjoint of F uses the same occupation-weighted density
    assert st["partial"] == (name == "B")


def test_fermi_dirac_needs_extra_levels(ks):
    with ks.GpuSolver(33, 0.25) as so:
        with pytest.raises(ValueError, match="n_extra"):
            so.solve(ks.System([(0.0, 0.0, 0.0, 5)], 3, 2), ks.ScfSettings(occupations="fermi_dirac"))


def test_witness_growth_reaches_the_fixed_block_answer(ks):
    """With one extra level the B atom's up block (2s and the 2p triple) has no gap witness: the block grows by
    doubling its extra levels (crates/qm/src/scf.rs:810-877) until its top level lies 0.1 Ha above level N and 36 kT
    above mu, then keeps the overshoot trimmed. F, kT S and the forces equal the fixed-block oracle answer."""
    case = REC["cases"]["B"]
    nuc = [tuple(a) for a in case["nuclei"]]
    settings = ks.ScfSettings(sigma=REC["sigma"], tol=REC["tol"], occupations="fermi_dirac", kt=REC["kt"])
    with ks.GpuSolver(REC["grid"], REC["h"], n_extra=1) as so:
        st = so.solve(ks.System(nuc, case["n_up"], case["n_dn"]), settings)
        grown = so.profile()["witness_growths"]
        fu, fd = so.occupations()
        f = so.forces(nuc, REC["sigma"])
        warm = so.solve(ks.System(nuc, case["n_up"], case["n_dn"]), settings, warm=True)
    assert grown >= 1
    assert len(fu) > case["n_up"] + 1
    ref = case["stats"]
    assert abs(st["energy"]["total"] - ref["total"]) < 1e-5, (st["energy"]["total"], ref["total"])
    assert abs(st["energy"]["ts"] - ref["ts"]) < 1e-6
    assert abs(fu.sum() - case["n_up"]) < 1e-9 and abs(fd.sum() - case["n_dn"]) < 1e-9
    assert np.abs(f - np.array(case["forces"])).max() < 1e-4
    assert warm["iterations"] <= 3 and abs(warm["energy"]["total"] - st["energy"]["total"]) < 1e-6, "the grown block is the warm start"
