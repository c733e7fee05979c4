"""ctypes binding of the CPU f64 oracle (``oracle/libksoracle.so``).

TEST INFRASTRUCTURE ONLY: the oracle checks the CUDA solver. It is loaded by ``tests/``,
``__graft_entry__.smoke()`` and the CPU legs of ``bench.py`` and by nothing in the product.
Array layout is the reference's ``qm::Grid``: a flat n^3 array, idx = i + n*(j + n*k)
(crates/qm/src/grid.rs:1-16).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libksoracle.so")


class Nucleus(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_double * 3), ("z", ctypes.c_int)]


class Settings(ctypes.Structure):
    _fields_ = [("sigma", ctypes.c_double), ("tol", ctypes.c_double), ("mixing", ctypes.c_double),
                ("eig_tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("diis_history", ctypes.c_int),
                ("stall_window", ctypes.c_int), ("occupations", ctypes.c_int), ("n_extra", ctypes.c_int), ("kt", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("delta_rho", ctypes.c_double),
                ("kinetic", ctypes.c_double), ("external", ctypes.c_double), ("hartree", ctypes.c_double),
                ("xc", ctypes.c_double), ("nuclear", ctypes.c_double), ("total", ctypes.c_double),
                ("boundary_density", ctypes.c_double), ("max_eigen_residual", ctypes.c_double),
                ("poisson_residual", ctypes.c_double), ("poisson_iterations", ctypes.c_int),
                ("electrons", ctypes.c_double * 2), ("status", ctypes.c_int),
                ("eigen_iterations_total", ctypes.c_int), ("poisson_iterations_total", ctypes.c_int),
                ("ts", ctypes.c_double), ("entropy", ctypes.c_double), ("mu", ctypes.c_double * 2)]


def build():
    """Compiles the oracle in place (make)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(os.path.join(HERE, "ks_oracle.cpp")):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        L.ora_neumaier.restype = ctypes.c_double
        L.ora_jacobi_omega.restype = ctypes.c_double
        L.ora_scf.restype = ctypes.c_void_p
        L.ora_scf.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                              ctypes.POINTER(Settings), ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.ora_state_free.argtypes = [ctypes.c_void_p]
        L.ora_state_counts.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.ora_state_evals.argtypes = [ctypes.c_void_p, dp, dp]
        L.ora_state_density.argtypes = [ctypes.c_void_p, dp, dp]
        L.ora_state_potentials.argtypes = [ctypes.c_void_p, dp, dp]
        L.ora_state_orbitals.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.ora_forces.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double, dp]
        L.ora_state_occupations.argtypes = [ctypes.c_void_p, dp, dp]
        L.ora_trilinear.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp, ctypes.c_int, dp]
        L.ora_fermi_dirac.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp]
        sp = ctypes.POINTER(SpeciesStruct)
        L.ora_scf_ionic.restype = ctypes.c_void_p
        L.ora_scf_ionic.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.POINTER(Settings), sp, ctypes.c_int, ctypes.c_void_p, ctypes.POINTER(Stats)]
        L.ora_ionic_local_potential.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double,
                                                sp, ctypes.c_int, dp]
        L.ora_partial_core.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(Nucleus), ctypes.c_int, sp, ctypes.c_int, dp]
        L.ora_nonlocal_apply.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(Nucleus), ctypes.c_int, sp, ctypes.c_int, dp,
                                         ctypes.c_int, dp, dp]
        L.ora_frozen_energy.restype = ctypes.c_double
        L.ora_frozen_energy.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double, sp, ctypes.c_int]
        L.ora_table_read.argtypes = [dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, dp, dp]
        L.ora_solid_harmonic_gradients.argtypes = [dp, dp]
        L.ora_forces_ionic.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double, sp, ctypes.c_int, dp]
        _lib = L
    return _lib


def set_threads(n):
    lib().ora_set_threads(int(n))


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a, size=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if size is not None:
        assert a.size == size, (a.size, size)
    return a


def nuclei_array(nuclei):
    """[(x, y, z, Z), ...] -> ctypes array of Nucleus."""
    arr = (Nucleus * max(len(nuclei), 1))()
    for i, (x, y, z, Z) in enumerate(nuclei):
        arr[i].pos[0], arr[i].pos[1], arr[i].pos[2] = x, y, z
        arr[i].z = int(Z)
    return arr


def grid_points(n, h):
    """(x, y, z) coordinate arrays of the cubic grid, flat in the reference's order."""
    half = (n - 1) * h / 2.0
    c = -half + np.arange(n) * h
    z, y, x = np.meshgrid(c, c, c, indexing="ij")
    return x.ravel(), y.ravel(), z.ravel()


def neumaier(v):
    v = _f64(v)
    return lib().ora_neumaier(_p(v), ctypes.c_size_t(v.size))


def laplacian(n, h, f):
    f = _f64(f, n ** 3)
    out = np.empty_like(f)
    lib().ora_laplacian(n, ctypes.c_double(h), _p(f), _p(out))
    return out


def hamiltonian(n, h, f, v):
    f, v = _f64(f, n ** 3), _f64(v, n ** 3)
    out = np.empty_like(f)
    lib().ora_hamiltonian(n, ctypes.c_double(h), _p(f), _p(v), _p(out))
    return out


def lsda(nu, nd):
    nu, nd = _f64(nu), _f64(nd)
    e, vu, vd = np.empty_like(nu), np.empty_like(nu), np.empty_like(nu)
    lib().ora_lsda(ctypes.c_size_t(nu.size), _p(nu), _p(nd), _p(e), _p(vu), _p(vd))
    return e, vu, vd


def exc_point(nu, nd):
    e, vu, vd = ctypes.c_double(), ctypes.c_double(), ctypes.c_double()
    lib().ora_exc_point(ctypes.c_double(nu), ctypes.c_double(nd), ctypes.byref(e), ctypes.byref(vu), ctypes.byref(vd))
    return e.value, vu.value, vd.value


def nuclear_potential(n, h, nuclei, sigma):
    out = np.empty(n ** 3)
    lib().ora_nuclear_potential(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), ctypes.c_double(sigma), _p(out))
    return out


def deposit_charge(n, h, nuclei, sigma):
    out = np.empty(n ** 3)
    lib().ora_deposit_charge(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), ctypes.c_double(sigma), _p(out))
    return out


def nuclear_repulsion(nuclei):
    e = ctypes.c_double()
    rc = lib().ora_nuclear_repulsion(nuclei_array(nuclei), len(nuclei), ctypes.byref(e))
    if rc != 0:
        raise ValueError("coincident nuclei")
    return e.value


def initial_orbitals(n, h, nuclei, k, seed):
    out = np.empty(max(k, 1) * n ** 3)
    lib().ora_initial_orbitals(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), k, ctypes.c_ulonglong(seed), _p(out))
    return out[: k * n ** 3].reshape(k, n ** 3)


def solid_harmonics(r):
    rr = _f64(r, 3)
    out = np.empty(49)
    lib().ora_solid_harmonics(_p(rr), _p(out))
    return out


def jacobi_omega():
    return lib().ora_jacobi_omega()


def jacobi_precond(n, h, v, lam, r):
    v, r = _f64(v, n ** 3), _f64(r, n ** 3)
    w = np.empty_like(r)
    lib().ora_jacobi_precond(n, ctypes.c_double(h), _p(v), ctypes.c_double(lam), _p(r), _p(w))
    return w


def poisson_solve(n, h, rho, v0=None, tol=1e-10, max_iter=5000):
    rho = _f64(rho, n ** 3)
    v = np.zeros(n ** 3) if v0 is None else _f64(v0, n ** 3).copy()
    res = ctypes.c_double()
    it = lib().ora_poisson_solve(n, ctypes.c_double(h), _p(rho), _p(v), ctypes.c_double(tol), max_iter, ctypes.byref(res))
    return v, it, res.value


def multipole_moments(n, h, rho):
    rho = _f64(rho, n ** 3)
    q = np.empty(49)
    lib().ora_multipole_moments(n, ctypes.c_double(h), _p(rho), _p(q))
    return q


def lobpcg(n, h, v, x0, tol=1e-6, max_iter=500, precond_lambda=None):
    x = _f64(x0).copy()
    k = x.shape[0]
    ev = np.empty(k)
    mr = ctypes.c_double()
    it = lib().ora_lobpcg(n, ctypes.c_double(h), _p(_f64(v, n ** 3)), k, _p(x), _p(ev), int(precond_lambda is not None),
                          ctypes.c_double(precond_lambda or 0.0), ctypes.c_double(tol), max_iter, ctypes.byref(mr))
    if it < 0:
        raise RuntimeError("oracle lobpcg lost rank")
    return ev, x, it, mr.value


def sym_eigen(a):
    a = _f64(a)
    m = a.shape[0]
    ev, vec = np.empty(m), np.empty(m * m)
    lib().ora_sym_eigen(m, _p(a), _p(ev), _p(vec))
    return ev, vec.reshape(m, m).T  # columns are eigenvectors


def diis_coefficients(gram):
    g = _f64(gram)
    m = g.shape[0]
    c = np.empty(m)
    ok = lib().ora_diis_coefficients(m, _p(g), _p(c))
    return c if ok else None


class State:
    """A converged oracle state (orbitals, eigenvalues, densities, potentials)."""

    def __init__(self, ptr, n):
        self.ptr, self.n = ptr, n

    def __del__(self):
        if getattr(self, "ptr", None):
            lib().ora_state_free(self.ptr)
            self.ptr = None

    def counts(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        lib().ora_state_counts(self.ptr, ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def evals(self):
        nu, nd = self.counts()
        up, dn = np.empty(max(nu, 1)), np.empty(max(nd, 1))
        lib().ora_state_evals(self.ptr, _p(up), _p(dn))
        return up[:nu], dn[:nd]

    def occupations(self):
        nu, nd = self.counts()
        up, dn = np.empty(max(nu, 1)), np.empty(max(nd, 1))
        lib().ora_state_occupations(self.ptr, _p(up), _p(dn))
        return up[:nu], dn[:nd]

    def density(self):
        up, dn = np.empty(self.n ** 3), np.empty(self.n ** 3)
        lib().ora_state_density(self.ptr, _p(up), _p(dn))
        return up, dn

    def potentials(self):
        a, b = np.empty(self.n ** 3), np.empty(self.n ** 3)
        lib().ora_state_potentials(self.ptr, _p(a), _p(b))
        return a, b

    def orbitals(self, spin):
        nu, nd = self.counts()
        k = nd if spin else nu
        out = np.empty(max(k, 1) * self.n ** 3)
        lib().ora_state_orbitals(self.ptr, spin, _p(out))
        return out[: k * self.n ** 3].reshape(k, self.n ** 3)


def scf(n, h, nuclei, n_up, n_dn, sigma=None, tol=1e-6, mixing=0.3, eig_tol=1e-6, max_iter=200, diis_history=6,
        stall_window=50, warm=None, kt=None, n_extra=1):
    """SCF (crates/qm/src/scf.rs:909): Aufbau, or Fermi-Dirac occupations at temperature kt (Ha) over
    N_sigma + n_extra levels per occupied channel. Returns (State or None, stats dict)."""
    s = Settings(h if sigma is None else sigma, tol, mixing, eig_tol, max_iter, diis_history, stall_window,
                 0 if kt is None else 1, int(n_extra), 0.0 if kt is None else float(kt))
    st = Stats()
    ptr = lib().ora_scf(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), n_up, n_dn, ctypes.byref(s),
                        warm.ptr if warm is not None else None, ctypes.byref(st))
    stats = {f[0]: getattr(st, f[0]) for f in Stats._fields_}
    stats["electrons"] = list(st.electrons)
    stats["mu"] = list(st.mu)
    return (State(ptr, n) if ptr else None), stats


# ---- pseudised ions (crates/qm/src/scf.rs:114-140, ionic.rs, nonlocal.rs, forces.rs)
class SpeciesStruct(ctypes.Structure):
    """ora_species (ks_oracle.h): one pseudised species' uniform tables."""
    _fields_ = [("z", ctypes.c_int), ("z_v", ctypes.c_double), ("sigma_lr", ctypes.c_double), ("du", ctypes.c_double),
                ("v_sr", ctypes.POINTER(ctypes.c_double)), ("n_v_sr", ctypes.c_int), ("r_sr", ctypes.c_double),
                ("rho_pc", ctypes.POINTER(ctypes.c_double)), ("n_rho_pc", ctypes.c_int), ("pc_radius", ctypes.c_double),
                ("n_proj", ctypes.c_int), ("proj_l", ctypes.POINTER(ctypes.c_int)), ("proj_e_kb", ctypes.POINTER(ctypes.c_double)),
                ("proj_radius", ctypes.POINTER(ctypes.c_double)), ("proj_t", ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
                ("proj_n", ctypes.POINTER(ctypes.c_int))]


def species_array(species):
    """(ctypes array, keep-alive list) from objects with the fields z, z_v, sigma_lr, du, v_sr, r_sr, rho_pc,
    pc_radius and projectors (each with l, e_kb, radius, t)."""
    keep = []

    def dptr(a):
        a = np.ascontiguousarray(a if a is not None else np.zeros(0), dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size

    arr = (SpeciesStruct * max(len(species), 1))()
    for i, sp in enumerate(species):
        st = arr[i]
        st.z, st.z_v, st.sigma_lr, st.du = int(sp.z), float(sp.z_v), float(sp.sigma_lr), float(sp.du)
        st.v_sr, st.n_v_sr = dptr(sp.v_sr)
        st.r_sr = float(sp.r_sr)
        st.rho_pc, st.n_rho_pc = dptr(sp.rho_pc)
        st.pc_radius = float(sp.pc_radius)
        k = len(sp.projectors)
        st.n_proj = k
        ls = (ctypes.c_int * max(k, 1))(*[p.l for p in sp.projectors])
        ek = (ctypes.c_double * max(k, 1))(*[p.e_kb for p in sp.projectors])
        rr = (ctypes.c_double * max(k, 1))(*[p.radius for p in sp.projectors])
        tp = (ctypes.POINTER(ctypes.c_double) * max(k, 1))()
        tn = (ctypes.c_int * max(k, 1))()
        for j, p in enumerate(sp.projectors):
            tp[j], tn[j] = dptr(p.t)
        keep += [ls, ek, rr, tp, tn]
        st.proj_l, st.proj_e_kb, st.proj_radius, st.proj_t, st.proj_n = ls, ek, rr, tp, tn
    return arr, keep


def scf_ionic(n, h, nuclei, n_up, n_dn, species, sigma=None, tol=1e-6, mixing=0.3, eig_tol=1e-6, max_iter=200, diis_history=6,
              stall_window=50, kt=None, n_extra=1):
    """SCF under an ionic setup (the species listed are pseudised). Returns (State or None, stats dict)."""
    s = Settings(h if sigma is None else sigma, tol, mixing, eig_tol, max_iter, diis_history, stall_window,
                 0 if kt is None else 1, int(n_extra), 0.0 if kt is None else float(kt))
    st = Stats()
    arr, keep = species_array(species)
    ptr = lib().ora_scf_ionic(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), n_up, n_dn, ctypes.byref(s), arr, len(species),
                              None, ctypes.byref(st))
    stats = {f[0]: getattr(st, f[0]) for f in Stats._fields_}
    stats["electrons"] = list(st.electrons)
    stats["mu"] = list(st.mu)
    return (State(ptr, n) if ptr else None), stats


def ionic_local_potential(n, h, nuclei, sigma_ae, species):
    arr, keep = species_array(species)
    out = np.empty(n ** 3)
    lib().ora_ionic_local_potential(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), ctypes.c_double(sigma_ae), arr,
                                    len(species), _p(out))
    return out


def partial_core(n, h, nuclei, species):
    arr, keep = species_array(species)
    out = np.empty(n ** 3)
    lib().ora_partial_core(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), arr, len(species), _p(out))
    return out


def nonlocal_apply(n, h, nuclei, species, x):
    """(V_NL x for each row of x (count, n^3), c (count, rows) = h^3 <beta_row, x>)."""
    arr, keep = species_array(species)
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, n ** 3))
    out = np.empty_like(x)
    c = np.empty(len(x) * 4096)
    rows = lib().ora_nonlocal_apply(n, ctypes.c_double(h), nuclei_array(nuclei), len(nuclei), arr, len(species), _p(x), len(x),
                                    _p(out), _p(c))
    return out, c[:len(x) * rows].reshape(len(x), rows)


def frozen_energy(state, nuclei, sigma, species):
    """integral rho V_loc + E_NL + E_xc[rho + rho_pc/2 per spin] + E_ii at the state's frozen orbitals and densities."""
    arr, keep = species_array(species)
    return lib().ora_frozen_energy(state.ptr, nuclei_array(nuclei), len(nuclei), ctypes.c_double(sigma), arr, len(species))


def table_read(f, du, radius, d):
    """(value, d/dd) of the 4-point Lagrange read of a uniform table (0 beyond radius)."""
    f = _f64(f)
    v, dv = ctypes.c_double(), ctypes.c_double()
    lib().ora_table_read(_p(f), f.size, ctypes.c_double(du), ctypes.c_double(radius), ctypes.c_double(d), ctypes.byref(v), ctypes.byref(dv))
    return v.value, dv.value


def solid_harmonic_gradients(r):
    """(9, 3): grad R_lm for l <= 2 in lm order."""
    out = np.empty(27)
    lib().ora_solid_harmonic_gradients(_p(_f64(r)), _p(out))
    return out.reshape(9, 3)


def forces_ionic(state, nuclei, sigma, species):
    arr, keep = species_array(species)
    out = np.empty(3 * len(nuclei))
    if lib().ora_forces_ionic(state.ptr, nuclei_array(nuclei), len(nuclei), ctypes.c_double(sigma), arr, len(species), _p(out)) != 0:
        raise ValueError("coincident nuclei")
    return out.reshape(-1, 3)


def trilinear(n, h, f, points):
    """qm::Grid::trilinear (crates/qm/src/grid.rs:54-86) of the n^3 field f at points (m, 3), f64."""
    pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
    out = np.empty(max(len(pts), 1))
    lib().ora_trilinear(int(n), ctypes.c_double(h), _p(_f64(f, n ** 3)), _p(pts), len(pts), _p(out))
    return out[:len(pts)]


def fermi_dirac(evals, n, kt):
    """Fermi-Dirac occupations of one channel (crates/qm/src/occupations.rs fermi_dirac): (f, mu, S)."""
    ev = _f64(evals)
    f = np.empty(max(ev.size, 1))
    mu, S = ctypes.c_double(), ctypes.c_double()
    if lib().ora_fermi_dirac(_p(ev), ev.size, int(n), ctypes.c_double(kt), _p(f), ctypes.byref(mu), ctypes.byref(S)) != 0:
        raise ValueError("Fermi-Dirac occupations refused (fewer than n + 1 levels, a non-finite level or kT)")
    return f[:ev.size], mu.value, S.value


def forces(state, nuclei, sigma):
    out = np.empty(3 * len(nuclei))
    rc = lib().ora_forces(state.ptr, nuclei_array(nuclei), len(nuclei), ctypes.c_double(sigma), _p(out))
    if rc != 0:
        raise ValueError("coincident nuclei")
    return out.reshape(-1, 3)
