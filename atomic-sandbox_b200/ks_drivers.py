"""Callers either side of the SCF path, on the B200 solver: the provider's evaluation semantics (GpuKs: one solver per
grid, warm starts, the cold retry of a failed warm solve, the GPU-memory guard), Born-Oppenheimer molecular dynamics
(velocity Verlet with warm-started solves), concurrent solves of a batch of geometries, and the synthetic workload
geometries (H2, H2O, NH3, n-butane and the batch templates).

Reference anchors: the integrator is crates/sim/src/integrator.rs (kick-drift-kick, atomic units,
dt converted once from fs); masses are isotope masses in amu times AMU_IN_ME
(crates/units/src/lib.rs:13, :26). The batch mirrors the reference's independent per-geometry
solves (one GpuSolver per grid, crates/providers/src/ks.rs) run concurrently on one GPU.
"""
import concurrent.futures
import dataclasses
import math
import time

import numpy as np

import ks_b200 as ks

AMU_IN_ME = 1822.888486209      # electron masses per atomic mass unit (crates/units/src/lib.rs:13)
FS_PER_AU = 0.024188843         # femtoseconds per atomic unit of time (hbar / E_h)
# most abundant isotope, amu
ISOTOPE_MASS_AMU = {1: 1.00782503223, 3: 7.0160034366, 6: 12.0, 7: 14.00307400443, 8: 15.99491461957, 9: 18.99840316273}


def mass_au(z):
    return ISOTOPE_MASS_AMU[int(z)] * AMU_IN_ME


# ------------------------------------------------------------------ workload geometries (Bohr)
def h2(separation=1.4):
    return [(separation / 2, 0.0, 0.0, 1), (-separation / 2, 0.0, 0.0, 1)]


def h2o(r_oh=1.81, angle_deg=104.5):
    a = math.radians(angle_deg) / 2
    return [(0.0, 0.0, 0.0, 8), (r_oh * math.sin(a), r_oh * math.cos(a), 0.0, 1), (-r_oh * math.sin(a), r_oh * math.cos(a), 0.0, 1)]


def _pyramid(center_z, r, angle_deg, n_h=3):
    """n_h hydrogens at distance r from a central atom at the origin with H-X-H angle angle_deg (C3v)."""
    c = math.cos(math.radians(angle_deg))
    theta = math.acos(math.sqrt((1 + 2 * c) / 3))  # angle of each X-H bond from the -z axis
    out = [(0.0, 0.0, 0.0, center_z)]
    for k in range(n_h):
        phi = 2 * math.pi * k / n_h
        out.append((r * math.sin(theta) * math.cos(phi), r * math.sin(theta) * math.sin(phi), r * math.cos(theta), 1))
    return out


def nh3(r_nh=1.91, angle_deg=106.7, jitter=0.0, seed=0):
    return jittered(_pyramid(7, r_nh, angle_deg), jitter, seed)


def ch4(r_ch=2.06):
    s = r_ch / math.sqrt(3)
    return [(0.0, 0.0, 0.0, 6), (s, s, s, 1), (s, -s, -s, 1), (-s, s, -s, 1), (-s, -s, s, 1)]


def lih(r=3.015):
    return [(r / 2, 0.0, 0.0, 3), (-r / 2, 0.0, 0.0, 1)]


def hf(r=1.733):
    return [(r / 2, 0.0, 0.0, 9), (-r / 2, 0.0, 0.0, 1)]


def butane_anti(r_cc=2.91, r_ch=2.06, jitter=0.0, seed=0):
    """n-butane, anti conformer: a planar zigzag C4 backbone (C-C-C 109.47 deg) in the xy plane, CH2
    hydrogens above and below the plane, staggered CH3 groups with one H anti in the plane."""
    tet = math.acos(-1.0 / 3.0)
    half = (math.pi - tet) / 2  # backbone bonds alternate +-half from the x axis
    c = [np.zeros(3)]
    for i in range(3):
        ang = half if i % 2 == 0 else -half
        c.append(c[-1] + r_cc * np.array([math.cos(ang), math.sin(ang), 0.0]))
    c = [p - sum(c) / 4 for p in c]
    atoms = [tuple(p) + (6,) for p in c]

    def unit(v):
        return v / np.linalg.norm(v)

    # CH2 (inner carbons): two H along the bisector opposite the neighbours, +-z out of plane
    for i in (1, 2):
        u1, u2 = unit(c[i - 1] - c[i]), unit(c[i + 1] - c[i])
        b = -unit(u1 + u2)
        nrm = unit(np.cross(u1, u2))
        for sgn in (1, -1):
            d = b * math.cos(tet / 2) + sgn * nrm * math.sin(tet / 2)
            atoms.append(tuple(c[i] + r_ch * d) + (1,))
    # CH3 (terminal carbons): three H at 109.47 deg from the C-C bond, one anti in the backbone plane
    for i, j, k in ((0, 1, 2), (3, 2, 1)):
        u = unit(c[j] - c[i])
        e1 = unit((c[k] - c[j]) - np.dot(c[k] - c[j], u) * u)  # in plane, perpendicular to the bond
        e2 = np.cross(u, e1)
        for phi in (math.pi, math.pi / 3, -math.pi / 3):  # phi = pi: anti to the next C-C bond
            d = -u / 3 + math.sqrt(8 / 9) * (math.cos(phi) * e1 + math.sin(phi) * e2)
            atoms.append(tuple(c[i] + r_ch * d) + (1,))
    return jittered(atoms, jitter, seed)


def jittered(nuclei, sigma, seed):
    if sigma <= 0:
        return [tuple(float(v) for v in a[:3]) + (int(a[3]),) for a in nuclei]
    rng = np.random.default_rng(seed)
    return [tuple(float(v) for v in np.asarray(a[:3]) + rng.normal(0.0, sigma, 3)) + (int(a[3]),) for a in nuclei]


BATCH_TEMPLATES = {"H2": h2, "LiH": lih, "H2O": h2o, "NH3": lambda: _pyramid(7, 1.91, 106.7), "CH4": ch4, "HF": hf}


def batch_workload(count=64, seed=0x5EED, n_min=48, n_max=96, h=0.25, jitter=0.05):
    """Seeded molecules from the templates with Gaussian displacements and per-molecule cubic grids
    n ~ U{n_min..n_max}: a list of dicts (name, nuclei, n, h)."""
    rng = np.random.default_rng(seed)
    names = sorted(BATCH_TEMPLATES)
    out = []
    for i in range(count):
        name = names[int(rng.integers(len(names)))]
        nuc = jittered(BATCH_TEMPLATES[name](), jitter, int(rng.integers(1 << 31)))
        out.append({"name": name, "nuclei": nuc, "n": int(rng.integers(n_min, n_max + 1)), "h": h})
    return out


# ------------------------------------------------------------------ the provider's evaluation (crates/providers/src/ks.rs)
@dataclasses.dataclass(frozen=True)
class Stall:
    """A warm solve that failed before the cold retry (crates/providers/src/ks.rs:566-584): its SCF iterations and
    dRho, and whether the stall stop ended it."""
    iterations: int
    delta_rho: float
    stalled: bool

    def note(self):
        if self.stalled:
            return (f"warm SCF stalled (dRho {self.delta_rho:.2e}, not improved 2x in the stall window; stopped after "
                    f"{self.iterations} iterations); retried cold")
        return f"warm SCF did not converge (dRho {self.delta_rho:.2e} after {self.iterations} steps); retried cold"


def retry_cold_on_stall(warm, solve):
    """crates/providers/src/ks.rs:585-601: `solve(w)` runs one SCF, warm iff w. A warm attempt that ends in
    ScfNotConverged or ScfStalled is retried cold exactly once and that outcome returned, with the Stall; every other
    outcome (success, a cold failure, another error) is the first attempt's. Returns (result, Stall or None)."""
    try:
        return solve(warm), None
    except ks.ScfNotConverged as e:
        if not warm:
            raise
        stall = Stall(getattr(e, "iterations", 0), getattr(e, "delta_rho", float("nan")), False)
    except ks.ScfStalled as e:
        if not warm:
            raise
        stall = Stall(getattr(e, "iterations", 0), getattr(e, "delta_rho", float("nan")), True)
    return solve(False), stall


VRAM_SLACK = 1.1


class GpuKs:
    """The Kohn-Sham force provider's semantics on the B200 solver (crates/providers/src/ks.rs:1014-1700, GpuKs):

    - one GpuSolver per grid; a grid change (n or h) rebuilds it and drops the warm state (ks.rs:12-14);
    - every evaluation starts warm from the previous converged state on the same grid and setup, with the cold retry
      of retry_cold_on_stall; its note is returned with the result;
    - with a memory budget, a scene whose solver footprint (ks_footprint_bytes) exceeds it is refused with a
      ValueError before any solver is built (GpuKs::check_vram, ks.rs:1303-1324);
    - a device failure drops the solver and its state (the next evaluation rebuilds it), and is raised;
    - should_abort is polled before every SCF step (ks.Aborted).
    """

    def __init__(self, gram_mode=1, n_extra=3, vram_budget=None, vram_note=None, init_mode=1):
        self.gram_mode, self.n_extra, self.init_mode = gram_mode, n_extra, init_mode
        self.vram_budget, self.vram_note = vram_budget, vram_note
        self.solver = None
        self._grid = None
        self._species = None
        self._warm = False

    def with_vram_budget(self, nbytes, note=None):
        self.vram_budget, self.vram_note = int(nbytes), note
        return self

    def _budget_words(self):
        b = f"the {self.vram_budget / 1e9:.1f} GB budget"
        return f"{b} ({self.vram_note})" if self.vram_note else b

    def check_vram(self, n, n_up, n_dn, settings, species=None):
        if self.vram_budget is None:
            return
        core = any(getattr(sp, "pc_radius", 0.0) > 0.0 for sp in (species or []))
        # the solver's buffers (measured within a few percent on B200) plus 10 % for the allocator's granularity
        need = int(VRAM_SLACK * ks.footprint_bytes(n, n_up, n_dn, self.n_extra, settings.diis_history, core))
        if need > self.vram_budget:
            kind = "valence " if species else ""
            raise ValueError(f"this scene needs ~{need / 1e9:.2f} GB of GPU memory at {n}^3 ({n_up + n_dn} {kind}electrons), "
                             f"over {self._budget_words()}: choose a coarser grid or fewer atoms")

    def close(self):
        if self.solver is not None:
            self.solver.close()
        self.solver, self._grid, self._warm = None, None, False

    def evaluate(self, nuclei, n, h, n_up, n_dn, settings=None, species=None, should_abort=None):
        """One evaluation: {energy, forces (n, 3), stats, notes}. Raises the solver's QmError subclasses."""
        settings = settings or ks.ScfSettings(sigma=h)
        self.check_vram(n, n_up, n_dn, settings, species)
        if self._grid != (n, h):
            self.close()
            self.solver = ks.GpuSolver(n, h, gram_mode=self.gram_mode, n_extra=self.n_extra, init_mode=self.init_mode)
            self._grid, self._species = (n, h), None
        sp_key = None if not species else [id(x) for x in species]
        if sp_key != self._species:
            self.solver.set_ionic(list(species or []))
            self._species = sp_key
        system = ks.System(nuclei, n_up, n_dn)
        try:
            stats, stall = retry_cold_on_stall(self._warm, lambda w: self.solver.solve(system, settings, warm=w,
                                                                                       should_abort=should_abort))
            forces = self.solver.forces(nuclei, settings.sigma if settings.sigma is not None else h)
        except ks.Device:
            self.close()
            raise
        except ks.QmError:
            self._warm = False
            raise
        self._warm = True
        return {"energy": stats["energy"]["total"], "forces": forces, "stats": stats, "notes": [stall.note()] if stall else []}


# ------------------------------------------------------------------ molecular dynamics
def velocity_verlet(solver, nuclei, n_up, n_dn, settings, dt_au, steps, velocities=None, sigma=None, retry_cold=True,
                    extrapolate=False):
    """Born-Oppenheimer MD, kick-drift-kick velocity Verlet (crates/sim/src/integrator.rs): one SCF
    solve per step, warm-started from the previous geometry; a warm solve that fails is retried
    cold, as the reference's provider does (crates/providers/src/ks.rs:590-601). Returns a list of
    per-step records: positions (Bohr), velocities, potential (the total KS energy), kinetic and
    total energy (Ha), SCF iterations and whether the step needed the cold retry. extrapolate starts every
    warm solve from the linear extrapolation in time of the last two converged densities
    (GpuSolver::set_density_extrapolation, crates/qm-gpu/src/scf.rs:1146-1163)."""
    solver.set_density_extrapolation(bool(extrapolate))
    sigma = settings.sigma if sigma is None else sigma
    z = [int(a[3]) for a in nuclei]
    m = np.array([mass_au(q) for q in z])[:, None]
    r = np.array([a[:3] for a in nuclei], dtype=float)
    v = np.zeros_like(r) if velocities is None else np.array(velocities, dtype=float)

    def solve(pos, warm):
        nuc = [tuple(p) + (q,) for p, q in zip(pos, z)]
        system = ks.System(nuc, n_up, n_dn)
        if retry_cold:
            st, stall = retry_cold_on_stall(warm, lambda w: solver.solve(system, settings, warm=w))
        else:
            st, stall = solver.solve(system, settings, warm=warm), None
        return st, solver.forces(nuc, sigma), stall is not None

    st, f, retried = solve(r, False)
    traj = []

    def record():
        ke = 0.5 * float((m * v * v).sum())
        e_pot = st["energy"]["total"]
        traj.append({"positions": r.copy(), "velocities": v.copy(), "potential": e_pot, "kinetic": ke, "total": e_pot + ke,
                     "iterations": st["iterations"], "cold_retry": retried, "extrapolated": bool(solver.profile()["extrapolated"])})

    record()
    for _ in range(steps):
        v = v + 0.5 * dt_au * f / m
        r = r + dt_au * v
        st, f, retried = solve(r, True)
        v = v + 0.5 * dt_au * f / m
        record()
    return traj


# ------------------------------------------------------------------ batches
def solve_batch(jobs, settings_for=None, workers=4, gram_mode=1, n_extra=3, native=False):
    """Solves independent geometries concurrently on the current GPU: `workers` host threads, each
    job on its own GpuSolver (own streams; the C ABI releases the GIL while it runs), or with native=True
    the library's own thread pool (ks_solve_batch). jobs: dicts with nuclei, n, h (and optional n_up /
    n_dn, default neutral lowest multiplicity). Returns (results in job order, wall seconds); each result
    holds energy, iterations and forces."""
    settings_for = settings_for or (lambda job: ks.ScfSettings(sigma=0.5))
    if native:
        full = []
        for job in jobs:
            sys_ = ks.neutral_system(job["nuclei"]) if "n_up" not in job else ks.System(job["nuclei"], job["n_up"], job["n_dn"])
            full.append(dict(job, n_up=sys_.n_up, n_dn=sys_.n_dn, settings=settings_for(job)))
        t0 = time.perf_counter()
        out = ks.solve_batch(full, workers=workers, gram_mode=gram_mode, n_extra=n_extra, init_mode=1)
        wall = time.perf_counter() - t0
        for r in out:
            if r["status"] != 0:
                raise ks.QmError(r["error"])
        return [{"energy": r["stats"]["energy"]["total"], "iterations": r["stats"]["iterations"], "forces": r["forces"]} for r in out], wall

    def run(job):
        sys_ = ks.neutral_system(job["nuclei"]) if "n_up" not in job else ks.System(job["nuclei"], job["n_up"], job["n_dn"])
        st_ = settings_for(job)
        with ks.GpuSolver(job["n"], job["h"], gram_mode=gram_mode, n_extra=n_extra, init_mode=1) as so:
            stats = so.solve(sys_, st_)
            f = so.forces(sys_.nuclei, st_.sigma)
        return {"energy": stats["energy"]["total"], "iterations": stats["iterations"], "forces": f}

    t0 = time.perf_counter()
    with concurrent.futures.ThreadPoolExecutor(max_workers=workers) as ex:
        results = list(ex.map(run, jobs))
    return results, time.perf_counter() - t0
