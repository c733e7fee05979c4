"""The pseudopotential path on the GPU (ks_set_ionic) against the oracle: the SCF of water with a pseudised O
(tests/golden/oracle_pseudo.json, made by tests/golden/make_oracle_pseudo.py), V_loc, rho_pc and the
Kleinman-Bylander operator on their own, the forces against energy differences, and the setup's guards
(crates/qm/src/scf.rs:114-140, crates/qm-gpu/src/ionic.rs, crates/qm/src/nonlocal.rs, forces.rs).

Bounds: |dE| < 1e-5 Ha, occupied levels 1e-5 Ha, forces 1e-4 Ha/Bohr against the f64 oracle; the operators, stored
in f32, to 1e-6 of their scale."""
import json
import os

import numpy as np
import pytest

import synthetic_species as ss

pytestmark = pytest.mark.gpu

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "oracle_pseudo.json")))
N, H, SIGMA = GOLD["grid"], GOLD["h"], GOLD["sigma"]
NUC = [tuple(x) for x in GOLD["nuclei"]]


def _solve(ks, species, settings=None, nuclei=NUC, so=None):
    own = so is None
    so = so or ks.GpuSolver(N, H, gram_mode=1, n_extra=3, init_mode=1)
    so.set_ionic(species)
    st = so.solve(ks.System(nuclei, 4, 4), settings or ks.ScfSettings(sigma=SIGMA, tol=1e-6))
    return so, st, own


@pytest.mark.parametrize("case", ["full", "local"])
def test_pseudo_water_matches_the_oracle(ks, case):
    ref = GOLD["cases"][case]
    so, st, _ = _solve(ks, [ss.oxygen_like(H, **ref["species"])])
    try:
        f = so.forces(NUC, SIGMA)
        eu, ed = so.evals()
    finally:
        so.close()
    e, r = st["energy"], ref["stats"]
    assert abs(e["total"] - r["total"]) < 1e-5, (e["total"], r["total"])
    for k in ("kinetic", "external", "hartree", "xc"):
        assert abs(e[k] - r[k]) < 2e-5, (k, e[k], r[k])
    assert abs(e["nuclear"] - r["nuclear"]) < 1e-12, "valence-charge repulsion"
    assert np.max(np.abs(eu[:4] - np.array(ref["evals_up"]))) < 1e-5
    assert np.max(np.abs(ed[:4] - np.array(ref["evals_dn"]))) < 1e-5
    assert np.max(np.abs(f - np.array(ref["forces"]))) < 1e-4, (f, ref["forces"])
    assert abs(st["electrons"][0] - 4) < 1e-4 and abs(st["electrons"][1] - 4) < 1e-4


def test_bare_hydrogen_setup_is_the_all_electron_solver(ks):
    """A species with Z_v = Z, the all-electron width and no tables is the smeared nucleus: the SCF takes the same
    steps to the same energy bit for bit (IonicPolicy::None is today's solver, crates/qm/src/scf.rs:1296-1330),
    and the ionic force path gives the all-electron forces."""
    nuc = [(0.7, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)]
    settings = ks.ScfSettings(sigma=SIGMA, tol=1e-6)
    with ks.GpuSolver(N, H, gram_mode=1, n_extra=3, init_mode=1) as a, ks.GpuSolver(N, H, gram_mode=1, n_extra=3, init_mode=1) as b:
        s0 = a.solve(ks.System(nuc, 1, 1), settings)
        f0 = a.forces(nuc, SIGMA)
        b.set_ionic([ss.bare_hydrogen(H, SIGMA)])
        s1 = b.solve(ks.System(nuc, 1, 1), settings)
        f1 = b.forces(nuc, SIGMA)
    assert s1["iterations"] == s0["iterations"]
    assert s1["energy"] == s0["energy"]
    assert np.max(np.abs(f1 - f0)) < 1e-9


def test_local_potential_and_partial_core_match_the_oracle(ks, oracle):
    """V_loc (the solve's v_nuc) and rho + rho_pc (the volume with core) against the oracle's f64 fields, to the f32
    storage; without a core the volume is the plain density."""
    sp = [ss.oxygen_like(H)]
    so, _, _ = _solve(ks, sp, ks.ScfSettings(sigma=SIGMA, tol=1e-3))
    try:
        import torch
        v_loc, _ = so.potentials()
        want = oracle.ionic_local_potential(N, H, NUC, SIGMA, sp)
        assert np.max(np.abs(v_loc - want) / np.maximum(1.0, np.abs(want))) < 1e-6
        rho = so.density_f32().astype(np.float64)
        vol = torch.empty(N ** 3, dtype=torch.float32, device="cuda:0")
        m = so.copy_density_with_core_to_volume(vol.data_ptr())
        v = vol.cpu().numpy()
        assert m == float(v.max())
        pc = oracle.partial_core(N, H, NUC, sp)
        assert pc.max() > 0.5
        assert np.max(np.abs((v.astype(np.float64) - rho) - pc)) < 1e-6 * max(1.0, pc.max())
    finally:
        so.close()
    so, _, _ = _solve(ks, [ss.oxygen_like(H, with_core=False)], ks.ScfSettings(sigma=SIGMA, tol=1e-3))
    try:
        import torch
        vol = torch.empty(N ** 3, dtype=torch.float32, device="cuda:0")
        so.copy_density_with_core_to_volume(vol.data_ptr())
        assert np.array_equal(vol.cpu().numpy(), so.density_f32())
    finally:
        so.close()


def test_nonlocal_operator_matches_the_oracle(ks, oracle):
    """V_NL x and the projections c = h^3 <beta, x> for random x, with one ion centred and one 0.4 Bohr inside a face
    (its balls clipped by the box): to 1e-6 of max |V_NL x| and of max |c|; <a | V_NL b> = <V_NL a | b> to 1e-6."""
    edge = -(N - 1) * H / 2 + 0.4
    nuc = [(0.05, -0.02, 0.01, 8), (edge, 0.1, -0.2, 8)]
    sp = [ss.oxygen_like(H)]
    rng = np.random.default_rng(7)
    x = rng.uniform(-0.5, 0.5, (2, N ** 3))
    want, c_want = oracle.nonlocal_apply(N, H, nuc, sp, x)
    with ks.GpuSolver(N, H) as so:
        so.set_ionic(sp)
        got, c_got = so.apply_nonlocal(nuc, x)
    assert c_got.shape == c_want.shape == (2, 8)
    assert np.max(np.abs(got - want)) < 1e-6 * np.max(np.abs(want))
    assert np.max(np.abs(c_got - c_want)) < 1e-6 * np.max(np.abs(c_want))
    ab, ba = np.dot(x[0], got[1]), np.dot(got[0], x[1])
    assert abs(ab - ba) < 1e-6 * max(abs(ab), abs(ba))


def test_forces_match_energy_differences(ks):
    """The pseudised O's force (long and short range, partial core, nonlocal) and an H's against central differences of
    the converged total energy, step 0.01 Bohr, SCF tightened to tol 5e-7 / eig_tol 1e-8: within 2e-4 Ha/Bohr (the
    reference's finite-difference bound for forces)."""
    sp = [ss.oxygen_like(H)]
    settings = ks.ScfSettings(sigma=SIGMA, tol=5e-7, eig_tol=1e-8)
    base = [(0.05, -0.03, 0.02, 8), (1.43, 1.11, 0.0, 1), (-1.43, 1.11, 0.0, 1)]
    with ks.GpuSolver(N, H, gram_mode=1, n_extra=3, init_mode=1) as so:
        so.set_ionic(sp)
        so.solve(ks.System(base, 4, 4), settings)
        f = so.forces(base, SIGMA)
        d = 0.01
        for a, ax in ((0, 0), (0, 1), (1, 0)):
            e = []
            for s in (d, -d):
                nuc = [list(x) for x in base]
                nuc[a][ax] += s
                e.append(so.solve(ks.System([tuple(x) for x in nuc], 4, 4), settings)["energy"]["total"])
            fd = -(e[0] - e[1]) / (2 * d)
            assert abs(f[a, ax] - fd) < 2e-4, (a, ax, f[a, ax], fd)


def test_setup_guards(ks):
    """Bad tables are refused with a message (nothing changes); a state converged under another setup is not a warm
    start (the warm pseudo solve equals a cold one bit for bit); the adjoint refuses a pseudo state."""
    good = ss.oxygen_like(H)
    bad_l = ss.oxygen_like(H)
    bad_l.projectors = [ss.Projector(3, 1.0, 1.6, good.projectors[0].t)]
    bad_du = ss.oxygen_like(H)
    bad_du.du = 0.0
    short = ss.oxygen_like(H)
    short.v_sr = short.v_sr[:2]
    with ks.GpuSolver(N, H, gram_mode=1, n_extra=3, init_mode=1) as so:
        for bad in ([bad_l], [bad_du], [short], [good, good]):
            with pytest.raises(ValueError):
                so.set_ionic(bad)
        so.solve(ks.System(NUC, 4, 4), ks.ScfSettings(sigma=SIGMA, tol=1e-6))  # all-electron water 2+, the same counts
        so.set_ionic([good])
        warm = so.solve(ks.System(NUC, 4, 4), ks.ScfSettings(sigma=SIGMA, tol=1e-6), warm=True)
        with pytest.raises(ValueError):
            so.vjp(NUC, SIGMA)
    with ks.GpuSolver(N, H, gram_mode=1, n_extra=3, init_mode=1) as so:
        so.set_ionic([good])
        cold = so.solve(ks.System(NUC, 4, 4), ks.ScfSettings(sigma=SIGMA, tol=1e-6))
    assert warm["energy"] == cold["energy"] and warm["iterations"] == cold["iterations"]
