"""The workloads beyond the timed H2O one, through the C ABI on the B200:
the adjoint (ks_vjp) against forces and central finite differences, NH3 96^3 forces / adjoint /
20-step Born-Oppenheimer MD, n-butane 128^3 in both Gram forms, H2 48^3 against a full oracle
SCF, and a concurrent batch of geometries against the same geometries solved one by one."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def drv(ks):
    import ks_drivers
    return ks_drivers


def _h2(x0):
    return [(x0, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)]


def test_vjp_position_part_is_minus_forces_and_scales_with_e_bar(ks):
    with ks.GpuSolver(49, 0.25) as so:
        so.solve(ks.System(_h2(0.7), 1, 1), ks.ScfSettings(sigma=0.25, tol=1e-7, eig_tol=1e-8))
        f = so.forces(_h2(0.7), 0.25)
        g, gs = so.vjp(_h2(0.7), 0.25)
        g2, gs2 = so.vjp(_h2(0.7), 0.25, e_bar=-3.0)
    assert np.abs(g + f).max() < 1e-7, (g, f)
    assert np.abs(g2 + 3.0 * g).max() < 1e-12 and abs(gs2 + 3.0 * gs) < 1e-12
    assert gs > 0  # a wider smearing weakens the nuclear attraction


def test_vjp_matches_central_differences_of_the_energy(ks):
    """dE/dx0 and dE/dsigma of H2 49^3 (sigma = h, tol 1e-7, eig_tol 1e-8) against central differences,
    the bounds of the reference's force_matches_finite_difference_of_gpu_energy
    (crates/qm-gpu/src/forces.rs:616-670): |HF - FD(0.01)| < 2e-4 and the Richardson extrapolation
    (4 FD(d) - FD(2d)) / 3 within 2e-5."""
    sig = 0.25
    with ks.GpuSolver(49, 0.25) as so:
        def energy(x0, s=sig):
            st = so.solve(ks.System(_h2(x0), 1, 1), ks.ScfSettings(sigma=s, tol=1e-7, eig_tol=1e-8))
            return st["energy"]["total"]
        energy(0.7)
        g, gs = so.vjp(_h2(0.7), sig)
        fd = {d: (energy(0.7 + d) - energy(0.7 - d)) / (2 * d) for d in (0.01, 0.02)}
        fs = {d: (energy(0.7, sig + d) - energy(0.7, sig - d)) / (2 * d) for d in (0.005, 0.01)}
    assert abs(g[0, 0] - fd[0.01]) < 2e-4, (g[0, 0], fd)
    assert abs(g[0, 0] - (4 * fd[0.01] - fd[0.02]) / 3) < 2e-5, (g[0, 0], fd)
    assert abs(gs - fs[0.005]) < 2e-4, (gs, fs)
    assert abs(gs - (4 * fs[0.005] - fs[0.01]) / 3) < 2e-5, (gs, fs)


def test_vjp_error_from_a_loose_solve(ks):
    """The adjoint is the explicit derivative, exact at self-consistency; its error away from it grows with the
    solve's own residual. H2 49^3 (sigma = h): the dE/dx0 after solves at tol 1e-3, 1e-4 and 1e-5 (density
    residual 3.5e-5 .. 1.3e-6) against the one after a tight solve (tol 1e-7, eig_tol 1e-8). Measured on the B200:
    2e-7 Ha/Bohr at tol 1e-3, below the reference's 2e-4 force bound (crates/qm-gpu/src/forces.rs:667) by three
    orders; the bound here is 2e-6."""
    sig = 0.25
    with ks.GpuSolver(49, 0.25) as so:
        so.solve(ks.System(_h2(0.7), 1, 1), ks.ScfSettings(sigma=sig, tol=1e-7, eig_tol=1e-8))
        g_tight, _ = so.vjp(_h2(0.7), sig)
        for tol in (1e-3, 1e-4, 1e-5):
            st = so.solve(ks.System(_h2(0.7), 1, 1), ks.ScfSettings(sigma=sig, tol=tol, eig_tol=min(1e-6, tol)))
            g, _ = so.vjp(_h2(0.7), sig)
            assert st["delta_rho"] < tol
            assert np.abs(g - g_tight).max() < 2e-6, (tol, st["delta_rho"], g[0, 0], g_tight[0, 0])


def test_nh3_96_forces_adjoint_and_md(ks, drv):
    """NH3 on 96^3 at h = 0.22 (N at the origin, H at 1.91 Bohr, 106.7 deg, seeded 0.05 Bohr jitter,
    the reference's default smearing sigma = h), mixed form: the adjoint equals -forces and matches
    central differences -- the 1e-3 Bohr step of the configuration, with the SCF tightened (tol 5e-7,
    eig_tol 1e-8) so that the energy noise (~1e-7 Ha) stays below the difference's resolution, and the
    reference's 0.01 Bohr step and 2e-4 bound (crates/qm-gpu/src/forces.rs:667). 20 velocity-Verlet
    steps of 0.5 fs keep the total energy within a bounded O(dt^2) oscillation (about 1e-3 Ha here: the
    jittered molecule starts 0.16 Ha/Bohr from equilibrium and the hydrogens reach ~0.08 Ha of kinetic
    energy) with every step converging warm."""
    nuc = drv.nh3(jitter=0.05, seed=0x5EED + 3)
    sig = 0.22
    st_ = ks.ScfSettings(sigma=sig)
    tight = ks.ScfSettings(sigma=sig, tol=5e-7, eig_tol=1e-8)
    with ks.GpuSolver(96, 0.22, gram_mode=1, n_extra=3) as so:
        so.solve(ks.System(nuc, 5, 5), tight)
        f = so.forces(nuc, sig)
        g, gs = so.vjp(nuc, sig)
        assert np.abs(g + f).max() < 1e-6
        for atom, axis in ((0, 0), (1, 2), (2, 1)):
            def e_at(d):
                moved = [list(a) for a in nuc]
                moved[atom][axis] += d
                return so.solve(ks.System([tuple(a) for a in moved], 5, 5), tight, warm=True)["energy"]["total"]
            fd3 = (e_at(1e-3) - e_at(-1e-3)) / 2e-3
            fd2 = (e_at(1e-2) - e_at(-1e-2)) / 2e-2
            assert abs(fd3 - g[atom, axis]) < 5e-4, (atom, axis, fd3, g[atom, axis])
            assert abs(fd2 - g[atom, axis]) < 2e-4, (atom, axis, fd2, g[atom, axis])
        dt = 0.5 / drv.FS_PER_AU
        traj = drv.velocity_verlet(so, nuc, 5, 5, st_, dt, 20)
    e = np.array([t["total"] for t in traj])
    assert len(traj) == 21
    assert not any(t["cold_retry"] for t in traj)
    assert np.abs(e - e[0]).max() < 3e-3, e - e[0]
    moved = np.abs(traj[-1]["positions"] - traj[0]["positions"]).max()
    assert moved > 1e-3  # the jittered molecule vibrates


def test_nh3_96_matches_oracle_record(ks, drv):
    """NH3 96^3 (h = 0.22, sigma = h, seeded 0.05 Bohr jitter) in the mixed form against a full f64 oracle SCF of the
    same geometry (tests/golden/oracle_nh3_96.json, tests/golden/make_oracle_configs.py): |dE| < 1e-5 Ha, occupied
    levels within 1e-5 Ha and forces within 1e-4 Ha/Bohr -- the bars of the reference's GPU-against-CPU checks
    (crates/validate/tests/gpu_vs_cpu.rs:152-160)."""
    rec = json.load(open(os.path.join(GOLDEN, "oracle_nh3_96.json")))
    nuc = drv.nh3(jitter=0.05, seed=0x5EED + 3)
    assert np.allclose(np.array(nuc), np.array(rec["nuclei"]), atol=0, rtol=0)
    with ks.GpuSolver(96, 0.22, gram_mode=1, n_extra=3, init_mode=1) as so:
        st = so.solve(ks.System(nuc, 5, 5), ks.ScfSettings(sigma=0.22, tol=1e-6))
        f = so.forces(nuc, 0.22)
        up, dn = so.evals()
    assert abs(st["energy"]["total"] - rec["stats"]["total"]) < 1e-5, (st["energy"]["total"], rec["stats"]["total"])
    assert np.abs(up[:5] - np.array(rec["evals_up"])).max() < 1e-5 and np.abs(dn[:5] - np.array(rec["evals_dn"])).max() < 1e-5
    assert np.abs(f - np.array(rec["forces"])).max() < 1e-4, np.abs(f - np.array(rec["forces"])).max()


def test_butane_128_mixed_matches_plain_and_oracle_record(ks, drv):
    """n-butane (anti, seeded 0.02 Bohr jitter) on 128^3 at h = 0.2: LOBPCG blocks of 20 bands per spin
    (17 occupied in the all-electron model + 3 extra), the tensor-core Gram (m = 60) against the
    CUDA-core form, and the mixed form against a full f64 oracle SCF of the same geometry
    (tests/golden/oracle_butane_128.json, tests/golden/make_oracle_configs.py butane, 4 hours on 4 host threads):
    |dE| < 1e-5 Ha, occupied eigenvalues within 1e-5 Ha and forces within 1e-4 Ha/Bohr (the bars of
    crates/validate/tests/gpu_vs_cpu.rs:152-160), 34 electrons. The density tolerance is 2e-6: the f32 storage floor of
    the mixed density is ~3e-8 N = 1.0e-6 for N = 34 (crates/qm-gpu/src/scf.rs module doc, "The mixing step"), so tol
    1e-6 sits on it (the oracle, in f64, stops at 1e-6)."""
    rec = json.load(open(os.path.join(GOLDEN, "oracle_butane_128.json")))
    nuc = drv.butane_anti(jitter=0.02, seed=0x5EED + 2)
    assert np.allclose(np.array(nuc), np.array(rec["nuclei"]), atol=0, rtol=0)
    out = {}
    for gm in (0, 1):
        with ks.GpuSolver(128, 0.2, gram_mode=gm, n_extra=3, init_mode=1) as so:
            st = so.solve(ks.System(nuc, 17, 17), ks.ScfSettings(sigma=0.5, tol=2e-6))
            out[gm] = (st, so.evals(), so.forces(nuc, 0.5))
    (s0, (u0, d0), _), (s1, (u1, d1), f1) = out[0], out[1]
    assert abs(s0["energy"]["total"] - s1["energy"]["total"]) < 1e-5, (s0["energy"], s1["energy"])
    assert np.abs(u0 - u1).max() < 1e-5 and np.abs(d0 - d1).max() < 1e-5
    assert abs(sum(s1["electrons"]) - 34) < 1e-4
    assert abs(s1["energy"]["total"] - rec["stats"]["total"]) < 1e-5, (s1["energy"]["total"], rec["stats"]["total"])
    eu, ed = np.array(rec["evals_up"]), np.array(rec["evals_dn"])
    assert np.abs(u1[:17] - eu[:17]).max() < 1e-5 and np.abs(d1[:17] - ed[:17]).max() < 1e-5, (u1[:17] - eu[:17], d1[:17] - ed[:17])
    assert np.abs(f1 - np.array(rec["forces"])).max() < 1e-4, np.abs(f1 - np.array(rec["forces"])).max()


def test_h2_48_matches_oracle_record(ks):
    """The H2 48^3 configuration (h = 0.25, sigma = 0.5, 1 + 3 bands per spin, uniform(-1, 1) start)
    against a full oracle SCF (tests/golden/oracle_h2_48.json)."""
    path = os.path.join(GOLDEN, "oracle_h2_48.json")
    rec = json.load(open(path))
    nuc = [(0.7, 0.0, 0.0, 1), (-0.7, 0.0, 0.0, 1)]
    with ks.GpuSolver(48, 0.25, n_extra=3, init_mode=1) as so:
        st = so.solve(ks.System(nuc, 1, 1), ks.ScfSettings(sigma=0.5, tol=1e-6))
        f = so.forces(nuc, 0.5)
        up, dn = so.evals()
    assert abs(st["energy"]["total"] - rec["stats"]["total"]) < 1e-5
    assert abs(up[0] - rec["evals_up"][0]) < 1e-5 and abs(dn[0] - rec["evals_dn"][0]) < 1e-5
    assert np.abs(f - np.array(rec["forces"])).max() < 1e-4


def test_batch_concurrent_equals_one_by_one(ks, drv):
    """Eight seeded batch molecules (48^3..64^3, the small boxes where the SCF is hardest) solved by three
    concurrent workers give bit-for-bit the energies of the same molecules solved one at a time."""
    jobs = drv.batch_workload(count=8, n_min=48, n_max=64)
    conc, wall = drv.solve_batch(jobs, workers=3)
    serial, _ = drv.solve_batch(jobs, workers=1)
    for a, b, j in zip(conc, serial, jobs):
        assert a["energy"] == b["energy"], (j["name"], a["energy"], b["energy"])
        assert np.array_equal(a["forces"], b["forces"])
    assert wall > 0


def test_batch_subset_matches_oracle_records(ks, drv):
    """The same eight seeded batch molecules (H2, NH3, H2O, CH4 on 49^3..59^3 grids) solved concurrently in the mixed
    form against full f64 oracle SCFs of each (tests/golden/oracle_batch8.json, tests/golden/make_oracle_configs.py):
    |dE| < 1e-5 Ha and forces within 1e-4 Ha/Bohr per molecule (crates/validate/tests/gpu_vs_cpu.rs:152-160)."""
    rec = json.load(open(os.path.join(GOLDEN, "oracle_batch8.json")))["molecules"]
    jobs = drv.batch_workload(count=8, n_min=48, n_max=64)
    assert [j["n"] for j in jobs] == [r["n"] for r in rec]
    out, _ = drv.solve_batch(jobs, workers=3)
    for j, o, r in zip(jobs, out, rec):
        assert np.array_equal(np.array(j["nuclei"]), np.array(r["nuclei"]))
        assert abs(o["energy"] - r["stats"]["total"]) < 1e-5, (j["name"], j["n"], o["energy"], r["stats"]["total"])
        assert np.abs(o["forces"] - np.array(r["forces"])).max() < 1e-4, (j["name"], j["n"])
