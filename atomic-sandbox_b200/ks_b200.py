"""Python mirror of the reference's ``qm_gpu::GpuSolver`` over the C ABI of ``libks_b200.so``.

The reference's host side is Rust (crates/qm-gpu/src/scf.rs:1042-1235); this module is the
binding a Python caller uses, with the reference's names and error behaviour:

- ``GpuSolver(grid_n, h)``            -> ``GpuSolver::new`` (scf.rs:1083)
- ``solver.solve(system, settings, warm)`` -> ``GpuSolver::solve`` (scf.rs:1195); raises the
  ``QmError`` subclasses below on failure, as the reference returns ``Err(QmError)``
- ``solver.forces(nuclei, sigma)``   -> ``GpuSolver::forces`` (forces.rs:239)
- ``solver.evals()``, ``density()``, ``orbitals()``, ``potentials()`` -> ``state()`` / ``ks_state``

The CUDA library is required: importing this module on a machine where ``libks_b200.so`` is
missing or cannot be loaded raises at load time -- there is no CPU fallback.
"""
import ctypes
import dataclasses
import json
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libks_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "ks_cuda.h")


class Nucleus(ctypes.Structure):
    _fields_ = [("pos", ctypes.c_double * 3), ("z", ctypes.c_int)]


class _Settings(ctypes.Structure):
    _fields_ = [("sigma", ctypes.c_double), ("tol", ctypes.c_double), ("mixing", ctypes.c_double),
                ("eig_tol", ctypes.c_double), ("max_iter", ctypes.c_int), ("diis_history", ctypes.c_int),
                ("stall_window", ctypes.c_int), ("occupations", ctypes.c_int), ("kt", ctypes.c_double)]


class _Options(ctypes.Structure):
    _fields_ = [("gram_mode", ctypes.c_int), ("n_extra", ctypes.c_int), ("init_mode", ctypes.c_int),
                ("reserved", ctypes.c_int)]


class _Energy(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in ("kinetic", "external", "hartree", "xc", "nuclear", "internal", "ts", "total")]


class _Stats(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("delta_rho", ctypes.c_double), ("energy", _Energy),
                ("boundary_density", ctypes.c_double), ("max_eigen_residual", ctypes.c_double),
                ("poisson_residual", ctypes.c_double), ("poisson_iterations", ctypes.c_int),
                ("electrons", ctypes.c_double * 2), ("tol_used", ctypes.c_double), ("n_warnings", ctypes.c_int),
                ("entropy", ctypes.c_double), ("mu", ctypes.c_double * 2), ("partial", ctypes.c_int)]


class _Profile(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in ("steps", "readbacks", "eigen_iterations", "poisson_iterations", "eigen_calls",
                                              "diis_resets")] + \
               [(n, ctypes.c_double) for n in ("wall_s", "start_s", "poisson_s", "eigen_s", "host_dense_s", "sync_wait_s")] + \
               [("witness_growths", ctypes.c_int), ("extrapolated", ctypes.c_int)] + \
               [(n, ctypes.c_int) for n in ("locked_calls", "class_raises", "buffer_witnesses", "buffer_growths",
                                            "lower_witnesses", "witness_residual_growths", "witness_trims", "frozen_steps",
                                            "diis_freeze_trims", "peak_block")]


class _EigenStats(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int) for f in ("iterations", "stop", "head_kept", "locked", "restores", "fallbacks", "readbacks")] + \
               [(f, ctypes.c_double) for f in ("max_residual", "head_residual", "tail_residual", "alpha_worst")]


class _KernelTime(ctypes.Structure):
    _fields_ = [("kernel", ctypes.c_int), ("count", ctypes.c_int), ("aux", ctypes.c_int), ("launches", ctypes.c_int),
                ("total_ms", ctypes.c_double), ("bytes", ctypes.c_double)]


KERNEL_NAMES = {0: "hpsi", 1: "jacobi", 2: "residual_precond", 3: "gram", 4: "block_update", 5: "hpsi_residual"}

ABORT_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)


class Progress(ctypes.Structure):
    """ks_progress: qm::ScfProgress (crates/qm/src/scf.rs:488-498)."""
    _fields_ = [("iteration", ctypes.c_int), ("max_iter", ctypes.c_int), ("delta_rho", ctypes.c_double), ("tol", ctypes.c_double),
                ("energy", ctypes.c_double), ("best_delta_rho", ctypes.c_double), ("since_gain", ctypes.c_int), ("window", ctypes.c_int),
                ("stall_level", ctypes.c_double)]


OBSERVE_FN = ctypes.CFUNCTYPE(None, ctypes.POINTER(Progress), ctypes.c_void_p)


class _BatchJob(ctypes.Structure):
    """ks_batch_job (include/ks_cuda.h)."""
    _fields_ = [("n", ctypes.c_int), ("h", ctypes.c_double), ("nuclei", ctypes.POINTER(Nucleus)), ("n_nuclei", ctypes.c_int),
                ("n_up", ctypes.c_int), ("n_dn", ctypes.c_int), ("settings", _Settings), ("forces3n", ctypes.POINTER(ctypes.c_double)),
                ("stats", _Stats), ("status", ctypes.c_int), ("error", ctypes.c_char * 160)]


@dataclasses.dataclass
class Projector:
    """One Kleinman-Bylander projector of a pseudised species: angular momentum l <= 2, E_KB (Ha), the radius of
    its ball (Bohr) and its radial table t_l(k du) (crates/qm/src/radial/filter.rs:323 FilteredProjector)."""
    l: int
    e_kb: float
    radius: float
    t: np.ndarray


@dataclasses.dataclass
class Species:
    """One pseudised species as the grid samples it (crates/qm/src/radial/filter.rs:330-363 FilteredTable): valence
    charge, width of the long-range erf part, the uniform-table spacing du and the V_SR / rho_pc / projector tables
    (even functions at d = k du, read by 4-point Lagrange, 0 beyond their radius). pc_radius <= 0: no partial core."""
    z: int
    z_v: float
    sigma_lr: float
    du: float
    v_sr: np.ndarray
    r_sr: float
    rho_pc: np.ndarray = None
    pc_radius: float = 0.0
    projectors: list = dataclasses.field(default_factory=list)


class SpeciesStruct(ctypes.Structure):
    """ks_species (include/ks_cuda.h); the oracle's ora_species has the same layout."""
    _fields_ = [("z", ctypes.c_int), ("z_v", ctypes.c_double), ("sigma_lr", ctypes.c_double), ("du", ctypes.c_double),
                ("v_sr", ctypes.POINTER(ctypes.c_double)), ("n_v_sr", ctypes.c_int), ("r_sr", ctypes.c_double),
                ("rho_pc", ctypes.POINTER(ctypes.c_double)), ("n_rho_pc", ctypes.c_int), ("pc_radius", ctypes.c_double),
                ("n_proj", ctypes.c_int), ("proj_l", ctypes.POINTER(ctypes.c_int)), ("proj_e_kb", ctypes.POINTER(ctypes.c_double)),
                ("proj_radius", ctypes.POINTER(ctypes.c_double)), ("proj_t", ctypes.POINTER(ctypes.POINTER(ctypes.c_double))),
                ("proj_n", ctypes.POINTER(ctypes.c_int))]


def species_array(species):
    """(ctypes array of SpeciesStruct, keep-alive list) for a list of Species."""
    keep = []

    def dptr(a):
        a = np.ascontiguousarray(a, dtype=np.float64)
        keep.append(a)
        return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), a.size

    arr = (SpeciesStruct * max(len(species), 1))()
    for i, sp in enumerate(species):
        st = arr[i]
        st.z, st.z_v, st.sigma_lr, st.du = int(sp.z), float(sp.z_v), float(sp.sigma_lr), float(sp.du)
        st.v_sr, st.n_v_sr = dptr(sp.v_sr if sp.v_sr is not None else np.zeros(0))
        st.r_sr = float(sp.r_sr)
        st.rho_pc, st.n_rho_pc = dptr(sp.rho_pc if sp.rho_pc is not None else np.zeros(0))
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
        st.proj_l, st.proj_e_kb, st.proj_radius = ls, ek, rr
        st.proj_t, st.proj_n = tp, tn
    return arr, keep

KS_OK, KS_COINCIDENT_NUCLEI, KS_NOT_CONVERGED, KS_STALLED, KS_NUMERICAL, KS_DEVICE, KS_INVALID, KS_ABORTED, KS_NO_STATE = range(9)


class QmError(RuntimeError):
    """qm::QmError (crates/qm/src/error.rs:4-31)."""


class CoincidentNuclei(QmError):
    pass


class ScfNotConverged(QmError):
    pass


class ScfStalled(QmError):
    pass


class Numerical(QmError):
    pass


class Device(QmError):
    pass


class Aborted(QmError):
    pass


class NoState(QmError):
    pass


_ERRORS = {KS_COINCIDENT_NUCLEI: CoincidentNuclei, KS_NOT_CONVERGED: ScfNotConverged, KS_STALLED: ScfStalled,
           KS_NUMERICAL: Numerical, KS_DEVICE: Device, KS_INVALID: ValueError, KS_ABORTED: Aborted, KS_NO_STATE: NoState}

EXPORTED = [
    "ks_solver_create", "ks_solver_destroy", "ks_solve", "ks_forces", "ks_last_error", "ks_state_counts", "ks_state_evals",
    "ks_state_density", "ks_state_potentials", "ks_state_orbitals", "ks_profile_get", "ks_apply_hamiltonian",
    "ks_apply_laplacian", "ks_apply_precond", "ks_xc_lsda", "ks_nuclear_potential", "ks_poisson_solve", "ks_gram", "ks_lobpcg",
    "ks_lobpcg_guarded",
    "ks_multipole_moments", "ks_field_pitch", "ks_hpsi_device", "ks_solver_stream", "ks_launch_count",
    "ks_gram_device_noalloc", "ks_vjp", "ks_state_occupations", "ks_sample_density", "ks_sampling_counters",
    "ks_state_density_f32", "ks_density_to_volume", "ks_density_max", "ks_spin_abs_integral", "ks_set_ionic",
    "ks_apply_nonlocal", "ks_density_with_core_to_volume", "ks_footprint_bytes", "ks_solve_observed", "ks_solve_batch",
    "ks_set_density_extrapolation", "ks_set_witness_cap", "ks_effective_eig_tol", "ks_rayleigh_ritz", "ks_fermi_dirac",
    "ks_fd_witness", "ks_fd_witness_bound", "ks_fd_witness_keep_within", "ks_fd_step_tail_kt", "ks_fd_tight_columns",
    "ks_fd_tight_start", "ks_density_residual", "ks_diis_mix", "ks_autotune_stencil",
    "ks_stencil_tuning_get", "ks_stencil_tuning_set", "ks_stencil_tuning_clear", "ks_device_status", "ks_set_kernel_timing", "ks_kernel_times", "ks_state_import",
    "ks_test_poison_parked_density", "ks_test_fail_readbacks",
]


def build():
    """Compiles libks_b200.so for sm_100a in place (make)."""
    subprocess.run(["make", "-s", "-j8", "-C", HERE], check=True)


_lib = None


def lib():
    """The loaded CUDA library (raises OSError when it is missing: no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"{LIB_PATH} is not built (run make -C {HERE})")
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int)
        L.ks_solver_create.restype = ctypes.c_void_p
        L.ks_solver_create.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(_Options)]
        L.ks_solver_destroy.argtypes = [ctypes.c_void_p]
        L.ks_last_error.restype = ctypes.c_char_p
        L.ks_last_error.argtypes = [ctypes.c_void_p]
        L.ks_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                               ctypes.POINTER(_Settings), ctypes.c_int, ABORT_FN, ctypes.c_void_p, ctypes.POINTER(_Stats)]
        L.ks_forces.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double, dp]
        L.ks_vjp.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double, ctypes.c_double, dp, dp]
        L.ks_state_counts.argtypes = [ctypes.c_void_p, ip, ip]
        L.ks_state_evals.argtypes = [ctypes.c_void_p, dp, dp]
        L.ks_state_occupations.argtypes = [ctypes.c_void_p, dp, dp]
        L.ks_state_density.argtypes = [ctypes.c_void_p, dp, dp]
        L.ks_state_potentials.argtypes = [ctypes.c_void_p, dp, dp]
        L.ks_state_orbitals.argtypes = [ctypes.c_void_p, ctypes.c_int, dp]
        L.ks_profile_get.argtypes = [ctypes.c_void_p, ctypes.POINTER(_Profile)]
        L.ks_set_kernel_timing.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ks_state_import.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp, dp, ctypes.c_int, dp, dp, dp, dp, dp,
                                      ctypes.c_int, dp, dp]
        L.ks_test_poison_parked_density.argtypes = [ctypes.c_void_p]
        L.ks_test_fail_readbacks.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ks_kernel_times.argtypes = [ctypes.c_void_p, ctypes.POINTER(_KernelTime), ctypes.c_int]
        L.ks_apply_hamiltonian.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, dp, dp, dp]
        L.ks_apply_laplacian.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.ks_apply_precond.argtypes = [ctypes.c_int, ctypes.c_double, dp, ctypes.c_double, dp, dp]
        L.ks_xc_lsda.argtypes = [ctypes.c_size_t, dp, dp, dp, dp, dp]
        L.ks_nuclear_potential.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_double, dp]
        L.ks_poisson_solve.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp, ctypes.c_double, ctypes.c_int, dp, ip]
        L.ks_gram.argtypes = [ctypes.c_int, ctypes.c_int, dp, ctypes.c_int, dp, ctypes.c_int, dp]
        L.ks_density_residual.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_int, dp, dp, dp, dp, dp, dp]
        L.ks_diis_mix.argtypes = [ctypes.c_int, ctypes.c_int, dp, dp, dp, dp, dp]
        L.ks_lobpcg.argtypes = [ctypes.c_int, ctypes.c_double, dp, ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_int, ctypes.c_int,
                                dp, ip]
        L.ks_lobpcg_guarded.argtypes = [ctypes.c_int, ctypes.c_double, dp, ctypes.c_int, dp, dp, ctypes.c_double, ctypes.c_double,
                                        ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, dp,
                                        ctypes.POINTER(_EigenStats)]
        L.ks_multipole_moments.argtypes = [ctypes.c_int, ctypes.c_double, dp, dp]
        L.ks_rayleigh_ritz.argtypes = [ctypes.c_int, dp, dp, ctypes.c_int, dp, dp, dp]
        L.ks_fermi_dirac.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, dp, dp, dp]
        L.ks_fd_witness.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ip, ip]
        L.ks_fd_witness_bound.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ip, ip]
        L.ks_fd_step_tail_kt.argtypes = [ctypes.c_int, ctypes.c_double, dp]
        L.ks_fd_tight_columns.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double, ip]
        L.ks_fd_tight_start.argtypes = [dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ip]
        L.ks_fd_witness_keep_within.argtypes = [dp, dp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                ctypes.c_double, ip]
        L.ks_field_pitch.argtypes = [ctypes.c_int]
        L.ks_autotune_stencil.argtypes = [ctypes.c_int, ip, ctypes.c_int, ip]
        L.ks_stencil_tuning_get.restype = ctypes.c_int
        L.ks_stencil_tuning_get.argtypes = [ip, ctypes.c_int]
        L.ks_stencil_tuning_set.argtypes = [ip, ctypes.c_int]
        L.ks_stencil_tuning_clear.argtypes = []
        L.ks_launch_count.restype = ctypes.c_longlong
        L.ks_launch_count.argtypes = []
        L.ks_solver_stream.restype = ctypes.c_void_p
        L.ks_solver_stream.argtypes = [ctypes.c_void_p]
        L.ks_device_status.argtypes = [ctypes.c_void_p]
        L.ks_hpsi_device.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]
        L.ks_gram_device_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_void_p, ctypes.c_void_p]
        fp = ctypes.POINTER(ctypes.c_float)
        L.ks_sample_density.argtypes = [ctypes.c_void_p, dp, ctypes.c_int, fp]
        L.ks_sampling_counters.argtypes = [ctypes.c_void_p, ip, ip]
        L.ks_state_density_f32.argtypes = [ctypes.c_void_p, fp]
        L.ks_density_to_volume.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.ks_density_max.argtypes = [ctypes.c_void_p, dp]
        L.ks_spin_abs_integral.argtypes = [ctypes.c_void_p, dp]
        L.ks_set_ionic.argtypes = [ctypes.c_void_p, ctypes.POINTER(SpeciesStruct), ctypes.c_int]
        L.ks_apply_nonlocal.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_int, dp, dp, dp, ip]
        L.ks_solve_observed.argtypes = [ctypes.c_void_p, ctypes.POINTER(Nucleus), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                        ctypes.POINTER(_Settings), ctypes.c_int, ABORT_FN, ABORT_FN, OBSERVE_FN, ctypes.c_void_p,
                                        ctypes.POINTER(_Stats)]
        L.ks_set_density_extrapolation.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ks_set_witness_cap.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ks_effective_eig_tol.argtypes = [ctypes.c_void_p, ctypes.c_double, dp]
        L.ks_solve_batch.argtypes = [ctypes.POINTER(_BatchJob), ctypes.c_int, ctypes.POINTER(_Options), ctypes.c_int]
        L.ks_footprint_bytes.restype = ctypes.c_longlong
        L.ks_footprint_bytes.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_Options), ctypes.c_int, ctypes.c_int]
        L.ks_density_with_core_to_volume.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, dp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _f64(a, size=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if size is not None and a.size != size:
        raise ValueError(f"expected {size} values, got {a.size}")
    return a


def _check(status, handle=None):
    if status != KS_OK:
        msg = lib().ks_last_error(handle).decode(errors="replace")
        raise _ERRORS.get(status, QmError)(msg)


def nuclei_array(nuclei):
    """[(x, y, z, Z), ...] (Bohr, atomic number) -> ctypes array."""
    arr = (Nucleus * max(len(nuclei), 1))()
    for i, (x, y, z, Z) in enumerate(nuclei):
        arr[i].pos[0], arr[i].pos[1], arr[i].pos[2] = float(x), float(y), float(z)
        arr[i].z = int(Z)
    return arr


@dataclasses.dataclass
class ScfSettings:
    """qm::ScfSettings (crates/qm/src/scf.rs:375) with Aufbau occupations; sigma None = h."""
    sigma: float = None
    tol: float = 1e-6
    max_iter: int = 200
    mixing: float = 0.3
    eig_tol: float = 1e-6
    diis_history: int = 6
    stall_window: int = 50
    occupations: str = "aufbau"  # or "fermi_dirac" (qm::Occupations, crates/qm/src/scf.rs:278)
    kt: float = 5e-3             # Fermi-Dirac temperature (Ha), ELECTRON_KT (crates/qm/src/occupations.rs)

    @classmethod
    def for_grid(cls, h):
        """The reference's defaults (ScfSettings::for_grid, crates/qm/src/scf.rs:381-395): sigma = h and Fermi-Dirac
        occupations at ELECTRON_KT; the solver then needs n_extra >= 1 (room for the gap witness)."""
        return cls(sigma=float(h), occupations="fermi_dirac", kt=5e-3)


@dataclasses.dataclass
class System:
    """qm::System (crates/qm/src/scf.rs:329): nuclei [(x, y, z, Z)] and electrons per spin."""
    nuclei: list
    n_up: int
    n_dn: int


def spin_split(total, multiplicity=None):
    """(n_up, n_dn) for `total` electrons (crates/qm/src/scf.rs:333-345)."""
    if total < 0:
        raise ValueError("negative electron count")
    if multiplicity is None:
        unpaired = total % 2
    else:
        m = int(multiplicity)
        if not (m >= 1 and m - 1 <= total and (total - (m - 1)) % 2 == 0):
            raise ValueError("bad multiplicity")
        unpaired = m - 1
    n_dn = (total - unpaired) // 2
    return n_dn + unpaired, n_dn


def neutral_system(nuclei, charge=0, multiplicity=None):
    """System::new: N = sum Z - charge, the lowest multiplicity unless given."""
    n_up, n_dn = spin_split(sum(int(z) for *_, z in nuclei) - charge, multiplicity)
    return System(list(nuclei), n_up, n_dn)


class GpuSolver:
    """One grid, one CUDA stream, every device buffer of the solve (crates/qm-gpu/src/scf.rs:1042)."""

    GRAM_FP32, GRAM_TENSOR = 0, 1

    def __init__(self, n, h, gram_mode=0, n_extra=0, init_mode=0):
        # the library's own argument checks (ks_solver_create), raised as argument errors before any device work
        if not (5 <= int(n) <= 1024 and float(h) > 0 and math.isfinite(float(h))):
            raise ValueError(f"grid: need 5 <= n <= 1024 and h > 0 (got n = {n}, h = {h})")
        if gram_mode not in (0, 1) or int(n_extra) < 0 or init_mode not in (0, 1):
            raise ValueError(f"invalid options: gram_mode {gram_mode}, n_extra {n_extra}, init_mode {init_mode}")
        opts = _Options(gram_mode, n_extra, init_mode, 0)
        self._h = lib().ks_solver_create(int(n), float(h), ctypes.byref(opts))
        if not self._h:
            raise Device(lib().ks_last_error(None).decode(errors="replace"))
        self.n, self.h = int(n), float(h)
        self._abort_ref = None

    def close(self):
        if getattr(self, "_h", None):
            lib().ks_solver_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the module's globals may already be gone; the process frees the GPU
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def solve(self, system, settings=None, warm=False, should_abort=None, inner_abort=None, observe=None):
        """Runs the SCF; returns the stats dict (ScfStats) or raises a QmError subclass. should_abort is polled before
        every SCF step, inner_abort once per LOBPCG iteration (GpuSolver::solve_polled); observe(progress_dict) gets one
        qm::ScfProgress per step (GpuSolver::solve_observed)."""
        s = settings or ScfSettings()
        if s.occupations not in ("aufbau", "fermi_dirac"):
            raise ValueError("occupations: 'aufbau' or 'fermi_dirac'")
        cs = _Settings(self.h if s.sigma is None else s.sigma, s.tol, s.mixing, s.eig_tol, s.max_iter, s.diis_history,
                       s.stall_window, 1 if s.occupations == "fermi_dirac" else 0, float(s.kt))
        st = _Stats()
        arr = nuclei_array(system.nuclei)
        cb = ABORT_FN(lambda _u: 1 if should_abort() else 0) if should_abort else ABORT_FN()
        self._abort_ref = cb
        if inner_abort is None and observe is None:
            rc = lib().ks_solve(self._h, arr, len(system.nuclei), int(system.n_up), int(system.n_dn), ctypes.byref(cs),
                                1 if warm else 0, cb, None, ctypes.byref(st))
        else:
            icb = ABORT_FN(lambda _u: 1 if inner_abort() else 0) if inner_abort else ABORT_FN()
            ocb = OBSERVE_FN(lambda p, _u: observe({n: getattr(p.contents, n) for n, _ in Progress._fields_})) if observe else OBSERVE_FN()
            self._observe_refs = (icb, ocb)
            rc = lib().ks_solve_observed(self._h, arr, len(system.nuclei), int(system.n_up), int(system.n_dn), ctypes.byref(cs),
                                         1 if warm else 0, cb, icb, ocb, None, ctypes.byref(st))
        if rc in (KS_NOT_CONVERGED, KS_STALLED):
            # QmError::ScfNotConverged(iterations, dRho) / ScfStalled { iterations, .. }: the counts ride on the exception
            err = _ERRORS[rc](lib().ks_last_error(self._h).decode(errors="replace"))
            err.iterations, err.delta_rho = st.iterations, st.delta_rho
            raise err
        _check(rc, self._h)
        e = st.energy
        return {
            "iterations": st.iterations, "delta_rho": st.delta_rho,
            "energy": {n: getattr(e, n) for n, _ in _Energy._fields_},
            "boundary_density": st.boundary_density, "max_eigen_residual": st.max_eigen_residual,
            "poisson_residual": st.poisson_residual, "poisson_iterations": st.poisson_iterations,
            "electrons": list(st.electrons), "tol_used": st.tol_used, "n_warnings": st.n_warnings,
            "entropy": st.entropy, "mu": list(st.mu), "partial": bool(st.partial),
        }

    def forces(self, nuclei, sigma=None):
        out = np.empty(3 * len(nuclei))
        _check(lib().ks_forces(self._h, nuclei_array(nuclei), len(nuclei), float(self.h if sigma is None else sigma), _p(out)), self._h)
        return out.reshape(-1, 3)

    def vjp(self, nuclei, sigma=None, e_bar=1.0):
        """Reverse-mode derivative of the converged total energy: (e_bar * dE/dR as (n, 3), e_bar * dE/dsigma)
        (ks_vjp). dE/dR equals minus forces()."""
        g = np.empty(3 * len(nuclei))
        gs = ctypes.c_double()
        _check(lib().ks_vjp(self._h, nuclei_array(nuclei), len(nuclei), float(self.h if sigma is None else sigma), float(e_bar), _p(g),
                            ctypes.byref(gs)), self._h)
        return g.reshape(-1, 3), gs.value

    def counts(self):
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(lib().ks_state_counts(self._h, ctypes.byref(a), ctypes.byref(b)), self._h)
        return a.value, b.value

    def evals(self):
        nu, nd = self.counts()
        up, dn = np.empty(max(nu, 1)), np.empty(max(nd, 1))
        _check(lib().ks_state_evals(self._h, _p(up), _p(dn)), self._h)
        return up[:nu], dn[:nd]

    def occupations(self):
        """One occupation per stored orbital: 1 under Aufbau, the final Fermi-Dirac f over the block otherwise."""
        nu, nd = self.counts()
        up, dn = np.empty(max(nu, 1)), np.empty(max(nd, 1))
        _check(lib().ks_state_occupations(self._h, _p(up), _p(dn)), self._h)
        return up[:nu], dn[:nd]

    def density(self, out=None):
        """(rho_up, rho_dn), f64 n^3 each. out: two C-contiguous float64 arrays of n^3 to fill instead of new ones (e.g.
        views of page-locked buffers, which the device writes at full copy speed)."""
        if out is None:
            up, dn = np.empty(self.n ** 3), np.empty(self.n ** 3)
        else:
            up, dn = out
            for a in (up, dn):
                if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.size == self.n ** 3 and a.flags.c_contiguous):
                    raise ValueError("density: out must be two C-contiguous float64 arrays of n^3 values")
        _check(lib().ks_state_density(self._h, _p(up), _p(dn)), self._h)
        return up, dn

    def set_density_extrapolation(self, on):
        """Warm starts from max(2 rho_t - rho_{t-1}, 0) of the last two converged outputs (ks_set_density_extrapolation)."""
        _check(lib().ks_set_density_extrapolation(self._h, 1 if on else 0), self._h)

    def set_witness_cap(self, cap):
        """At most `cap` (1..32) extra Fermi-Dirac levels per channel (ks_set_witness_cap)."""
        _check(lib().ks_set_witness_cap(self._h, int(cap)), self._h)

    def effective_eig_tol(self, eig_tol=1e-6):
        """The LOBPCG tolerance of the final SCF step: max(eig_tol, 3 x the f32 residual floor) (ks_effective_eig_tol)."""
        v = ctypes.c_double()
        _check(lib().ks_effective_eig_tol(self._h, float(eig_tol), ctypes.byref(v)), self._h)
        return v.value

    def set_ionic(self, species):
        """The ionic setup of the next solves (ks_set_ionic): a list of Species (pseudised Z), [] = all-electron."""
        arr, keep = species_array(list(species))
        _check(lib().ks_set_ionic(self._h, arr, len(species)), self._h)

    def apply_nonlocal(self, nuclei, x):
        """(V_NL x for each row of x (count, n^3), projections c (count, rows)) under the ionic setup at nuclei."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1, self.n ** 3))
        out = np.empty_like(x)
        c = np.empty(len(x) * 640)
        rows = ctypes.c_int()
        _check(lib().ks_apply_nonlocal(self._h, nuclei_array(nuclei), len(nuclei), len(x), _p(x), _p(out), _p(c), ctypes.byref(rows)),
               self._h)
        return out, c[:len(x) * rows.value].reshape(len(x), rows.value)

    def copy_density_with_core_to_volume(self, dense_dev_ptr, stream=None):
        """The n^3 f32 image of rho + rho_pc (the plain density without a partial core) on a device buffer, ordered after
        the solver's work on `stream`; returns the maximum of the field written."""
        m = ctypes.c_double()
        _check(lib().ks_density_with_core_to_volume(self._h, ctypes.c_void_p(int(dense_dev_ptr)), ctypes.c_void_p(stream or 0),
                                                    ctypes.byref(m)), self._h)
        return m.value

    # ---- readouts (crates/qm-gpu/src/sample.rs, crates/qm-gpu/src/scf.rs:1776-1842)
    def sample_density(self, points):
        """rho_up + rho_dn at points (m, 3) Bohr by trilinear interpolation (f32 values, 0 outside the box);
        one launch and one readback per non-empty call."""
        pts = np.ascontiguousarray(np.asarray(points, dtype=np.float64).reshape(-1, 3))
        out = np.empty(len(pts), dtype=np.float32)
        if len(pts) == 0:
            _check(lib().ks_sample_density(self._h, None, 0, None), self._h)
            return out
        _check(lib().ks_sample_density(self._h, _p(pts), len(pts), out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self._h)
        return out

    def sampling_counters(self):
        """(readbacks, buffer allocations) of sample_density so far."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(lib().ks_sampling_counters(self._h, ctypes.byref(a), ctypes.byref(b)), self._h)
        return a.value, b.value

    def density_f32(self):
        """The stored total density rho_up + rho_dn, f32, n^3 (x fastest)."""
        out = np.empty(self.n ** 3, dtype=np.float32)
        _check(lib().ks_state_density_f32(self._h, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))), self._h)
        return out

    def copy_density_to_volume(self, dense_dev_ptr, stream=None):
        """Writes the n^3 f32 image of the density to a device buffer (e.g. a torch tensor's data_ptr()), enqueued
        on `stream` (a cudaStream_t as an int; None = the solver's stream). Does not wait."""
        _check(lib().ks_density_to_volume(self._h, ctypes.c_void_p(int(dense_dev_ptr)), ctypes.c_void_p(stream or 0)), self._h)

    def density_max(self):
        v = ctypes.c_double()
        _check(lib().ks_density_max(self._h, ctypes.byref(v)), self._h)
        return v.value

    def spin_abs_integral(self):
        """The integral of |rho_up - rho_dn| (electrons)."""
        v = ctypes.c_double()
        _check(lib().ks_spin_abs_integral(self._h, ctypes.byref(v)), self._h)
        return v.value

    def potentials(self):
        a, b = np.empty(self.n ** 3), np.empty(self.n ** 3)
        _check(lib().ks_state_potentials(self._h, _p(a), _p(b)), self._h)
        return a, b

    def orbitals(self, spin):
        nu, nd = self.counts()
        k = nd if spin else nu
        out = np.empty(max(k, 1) * self.n ** 3)
        _check(lib().ks_state_orbitals(self._h, int(spin), _p(out)), self._h)
        return out[: k * self.n ** 3].reshape(k, self.n ** 3)

    def import_state(self, n_up, n_dn, orbitals, evals, density, v_h, occupations=None):
        """The warm start of the next solve(warm=True) from a saved state (ks_state_import): orbitals / evals per spin
        as (k, n^3) and (k,) arrays (N_sigma <= k <= N_sigma + n_extra), density = (rho_up, rho_dn), v_h an n^3
        array, occupations None (Aufbau) or a per-spin pair of f arrays (Fermi-Dirac)."""
        n3 = self.n ** 3
        orb = [np.ascontiguousarray(o, dtype=np.float64).reshape(-1, n3) for o in orbitals]
        ev = [np.ascontiguousarray(e, dtype=np.float64) for e in evals]
        rho = [np.ascontiguousarray(r, dtype=np.float64).reshape(n3) for r in density]
        vh = np.ascontiguousarray(v_h, dtype=np.float64).reshape(n3)
        occ = None if occupations is None else [np.ascontiguousarray(f, dtype=np.float64) for f in occupations]
        empty = np.zeros(1)

        def ptr(a):
            return _p(a if a is not None and a.size else empty)
        _check(lib().ks_state_import(self._h, int(n_up), int(n_dn), orb[0].shape[0], ptr(orb[0]), ptr(ev[0]), orb[1].shape[0],
                                     ptr(orb[1]), ptr(ev[1]), _p(rho[0]), _p(rho[1]), _p(vh), 0 if occ is None else 1,
                                     ptr(occ[0]) if occ else None, ptr(occ[1]) if occ else None), self._h)

    def poison_parked_density(self):
        """Failure-path test hook: a NaN in the parked warm density (ks_test_poison_parked_density)."""
        _check(lib().ks_test_poison_parked_density(self._h), self._h)

    def fail_readbacks(self, skip, count):
        """Failure-path test hook: let `skip` readbacks through, fail the next `count` (ks_test_fail_readbacks)."""
        _check(lib().ks_test_fail_readbacks(self._h, int(skip), int(count)), self._h)

    def stream(self):
        """The cudaStream_t (as an int) every kernel of this solver runs on."""
        return lib().ks_solver_stream(self._h)

    def profile(self):
        p = _Profile()
        _check(lib().ks_profile_get(self._h, ctypes.byref(p)), self._h)
        return {n: getattr(p, n) for n, _ in _Profile._fields_}

    def set_kernel_timing(self, on=True):
        """Per-shape device timing of the LOBPCG chain's launches (ks_set_kernel_timing); switching on clears it."""
        _check(lib().ks_set_kernel_timing(self._h, 1 if on else 0), self._h)

    def kernel_times(self):
        """Launches, device time and algorithmic bytes per launch shape since the timing was switched on
        (ks_kernel_times): a list of dicts with kernel, count, aux, launches, total_ms, bytes, mean_us, gbs."""
        cap = 64
        buf = (_KernelTime * cap)()
        n = lib().ks_kernel_times(self._h, buf, cap)
        if n < 0:
            _check(KS_DEVICE, self._h)
        out = []
        for t in buf[:min(n, cap)]:
            mean_s = t.total_ms / 1000.0 / t.launches if t.launches else 0.0
            out.append({"kernel": KERNEL_NAMES.get(t.kernel, str(t.kernel)), "count": t.count, "aux": t.aux,
                        "launches": t.launches, "total_ms": t.total_ms, "bytes": t.bytes, "mean_us": mean_s * 1e6,
                        "gbs": t.bytes / mean_s / 1e9 if mean_s > 0 else 0.0})
        return out


def _stats_dict(st):
    e = st.energy
    return {
        "iterations": st.iterations, "delta_rho": st.delta_rho,
        "energy": {n: getattr(e, n) for n, _ in _Energy._fields_},
        "boundary_density": st.boundary_density, "max_eigen_residual": st.max_eigen_residual,
        "poisson_residual": st.poisson_residual, "poisson_iterations": st.poisson_iterations,
        "electrons": list(st.electrons), "tol_used": st.tol_used, "n_warnings": st.n_warnings,
        "entropy": st.entropy, "mu": list(st.mu), "partial": bool(st.partial),
    }


def solve_batch(jobs, workers=4, gram_mode=1, n_extra=3, init_mode=1, forces=True):
    """Independent cold solves (and forces) of many geometries on the current GPU in the library's own thread pool
    (ks_solve_batch). jobs: dicts with nuclei, n, h, n_up, n_dn and settings (ScfSettings). Returns one dict per job:
    status (0 = KS_OK), error, stats (as GpuSolver.solve) and forces ((n, 3), or None)."""
    arr = (_BatchJob * max(len(jobs), 1))()
    keep = []
    for i, job in enumerate(jobs):
        s = job.get("settings") or ScfSettings()
        nuc = nuclei_array(job["nuclei"])
        f = np.zeros(3 * len(job["nuclei"]))
        keep += [nuc, f]
        a = arr[i]
        a.n, a.h, a.nuclei, a.n_nuclei = int(job["n"]), float(job["h"]), nuc, len(job["nuclei"])
        a.n_up, a.n_dn = int(job["n_up"]), int(job["n_dn"])
        a.settings = _Settings(float(job["h"]) if s.sigma is None else s.sigma, s.tol, s.mixing, s.eig_tol, s.max_iter,
                               s.diis_history, s.stall_window, 1 if s.occupations == "fermi_dirac" else 0, float(s.kt))
        a.forces3n = _p(f) if forces else None
    opts = _Options(int(gram_mode), int(n_extra), int(init_mode), 0)
    _check(lib().ks_solve_batch(arr, len(jobs), ctypes.byref(opts), int(workers)))
    out = []
    for i, job in enumerate(jobs):
        a = arr[i]
        ok = a.status == KS_OK
        out.append({"status": a.status, "error": a.error.decode(errors="replace"), "stats": _stats_dict(a.stats) if ok else None,
                    "forces": keep[2 * i + 1].reshape(-1, 3).copy() if (ok and forces) else None})
    return out


def footprint_bytes(n, n_up, n_dn, n_extra=0, diis_history=6, with_core=False):
    """Device bytes a GpuSolver of the n^3 grid holds through a solve and its forces (ks_footprint_bytes)."""
    o = _Options(0, int(n_extra), 0, 0)
    b = lib().ks_footprint_bytes(int(n), int(n_up), int(n_dn), ctypes.byref(o), int(diis_history), 1 if with_core else 0)
    if b < 0:
        raise ValueError("footprint: invalid grid, counts or history")
    return int(b)


# ---- grid-kernel entry points (host f64 in/out)
def apply_hamiltonian(n, h, psi, v):
    psi = _f64(psi)
    count = psi.size // n ** 3
    out = np.empty(count * n ** 3)
    _check(lib().ks_apply_hamiltonian(n, h, count, _p(psi), _p(_f64(v, n ** 3)), _p(out)))
    return out.reshape(psi.shape)


def apply_laplacian(n, h, f):
    out = np.empty(n ** 3)
    _check(lib().ks_apply_laplacian(n, h, _p(_f64(f, n ** 3)), _p(out)))
    return out


def apply_precond(n, h, v, lam, r):
    out = np.empty(n ** 3)
    _check(lib().ks_apply_precond(n, h, _p(_f64(v, n ** 3)), float(lam), _p(_f64(r, n ** 3)), _p(out)))
    return out


def xc_lsda(up, dn):
    up, dn = _f64(up), _f64(dn, np.size(up))
    e, vu, vd = np.empty_like(up), np.empty_like(up), np.empty_like(up)
    _check(lib().ks_xc_lsda(ctypes.c_size_t(up.size), _p(up), _p(dn), _p(e), _p(vu), _p(vd)))
    return e, vu, vd


def nuclear_potential(n, h, nuclei, sigma):
    out = np.empty(n ** 3)
    _check(lib().ks_nuclear_potential(n, h, nuclei_array(nuclei), len(nuclei), float(sigma), _p(out)))
    return out


def poisson_solve(n, h, rho, v0=None, tol=1e-8, max_iter=5000):
    v = np.zeros(n ** 3) if v0 is None else _f64(v0, n ** 3).copy()
    res, it = ctypes.c_double(), ctypes.c_int()
    _check(lib().ks_poisson_solve(n, h, _p(_f64(rho, n ** 3)), _p(v), float(tol), int(max_iter), ctypes.byref(res), ctypes.byref(it)))
    return v, it.value, res.value


def multipole_moments(n, h, rho):
    q = np.empty(49)
    _check(lib().ks_multipole_moments(n, h, _p(_f64(rho, n ** 3)), _p(q)))
    return q


def rayleigh_ritz(a, b, nk):
    """The LOBPCG Rayleigh-Ritz step on the host (crates/qm-gpu/src/eigen.rs:515-542): the lowest nk pairs of
    A c = theta B c. Returns (theta ascending, C as an m x nk array of B-orthonormal columns, alpha)."""
    a = np.ascontiguousarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    m = a.shape[0]
    if a.shape != (m, m) or b.shape != (m, m):
        raise ValueError("rayleigh_ritz: A and B must be square and of one size")
    theta, c, alpha = np.empty(nk), np.empty(m * nk), ctypes.c_double()
    _check(lib().ks_rayleigh_ritz(m, _p(a), _p(b), int(nk), _p(theta), _p(c), ctypes.byref(alpha)))
    return theta, c.reshape(nk, m).T.copy(), alpha.value


def fermi_dirac(evals, n, kt):
    """Fermi-Dirac occupations of one channel (crates/qm/src/occupations.rs fermi_dirac), as the solver computes
    them: (f, mu, S). ValueError on the reference's refusals."""
    ev = _f64(evals)
    f = np.empty(max(ev.size, 1))
    mu, s = ctypes.c_double(), ctypes.c_double()
    _check(lib().ks_fermi_dirac(_p(ev), ev.size, int(n), float(kt), _p(f), ctypes.byref(mu), ctypes.byref(s)))
    return f[:ev.size], mu.value, s.value


def fd_witness(evals, n, mu, kt, residuals=None):
    """The solver's gap witness of a Fermi-Dirac block: (reached, keep). Without residuals it is read on the levels
    themselves (crates/qm/src/occupations.rs witness_reached, witness_keep); with them on the lower bounds
    theta - r, as the solver reads it (witness_bound_reached, witness_keep)."""
    ev = _f64(evals)
    reached, keep = ctypes.c_int(), ctypes.c_int()
    if residuals is None:
        _check(lib().ks_fd_witness(_p(ev), ev.size, int(n), float(mu), float(kt), ctypes.byref(reached), ctypes.byref(keep)))
    else:
        r = _f64(residuals)
        if r.size != ev.size:
            raise ValueError("fd_witness: one residual per level")
        _check(lib().ks_fd_witness_bound(_p(ev), _p(r), ev.size, int(n), float(mu), float(kt), ctypes.byref(reached),
                                         ctypes.byref(keep)))
    return bool(reached.value), keep.value


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


STENCIL_MODES = {1: "hpsi", 2: "jacobi"}


def autotune_stencil(n, counts):
    """Times every z-chunking of H psi and of the Jacobi sweep for each vector count on an n^3 grid and keeps the
    fastest for this process's later launches on this device (the outputs do not depend on the chunking).
    Returns {count: {"hpsi": chunks, "jacobi": chunks}}."""
    c = np.ascontiguousarray(counts, dtype=np.int32)
    out = np.zeros(2 * c.size, dtype=np.int32)
    _check(lib().ks_autotune_stencil(int(n), _ip(c), c.size, _ip(out)))
    return {int(k): {"hpsi": int(out[2 * i]), "jacobi": int(out[2 * i + 1])} for i, k in enumerate(c)}


def stencil_tuning():
    """The current device's tuning table: [(n, count, mode, chunks)], mode 1 = H psi, 2 = the Jacobi sweep."""
    total = lib().ks_stencil_tuning_get(None, 0)
    if total < 0:
        raise Device("stencil_tuning: no CUDA device")
    buf = np.zeros(4 * max(total, 1), dtype=np.int32)
    total = lib().ks_stencil_tuning_get(_ip(buf), total)
    return [tuple(int(v) for v in buf[4 * i:4 * i + 4]) for i in range(total)]


def set_stencil_tuning(entries):
    """Installs (n, count, mode, chunks) entries on the current device (e.g. loaded from a file)."""
    e = np.ascontiguousarray(np.asarray(list(entries), dtype=np.int32).reshape(-1, 4))
    _check(lib().ks_stencil_tuning_set(_ip(e), e.shape[0]))


def clear_stencil_tuning():
    _check(lib().ks_stencil_tuning_clear())


def save_stencil_tuning(path):
    """Writes the current device's tuning table as JSON (with the device's name, which a load checks)."""
    import torch
    with open(path, "w") as f:
        json.dump({"device": torch.cuda.get_device_name(), "entries": [list(e) for e in stencil_tuning()]}, f)


def load_stencil_tuning(path):
    """Installs a table written by save_stencil_tuning; a table from another device model is refused (ValueError)."""
    import torch
    with open(path) as f:
        d = json.load(f)
    if d.get("device") != torch.cuda.get_device_name():
        raise ValueError(f"stencil tuning for {d.get('device')!r}, not {torch.cuda.get_device_name()!r}")
    set_stencil_tuning(d["entries"])


def density_residual(n, h, psi, rho_in, f=None):
    """The SCF's density step (the solver's kernel and finish): (rho_out = sum_i f_i psi_i^2, r = rho_out - rho_in,
    (h^3 sum |r|, h^3 sum rho_out)) for psi of shape (k, n^3); f None means every f_i = 1."""
    n3 = n ** 3
    psi = np.ascontiguousarray(np.asarray(psi, dtype=np.float64).reshape(-1, n3))
    k = psi.shape[0]
    rin = _f64(rho_in, n3)
    fa = None if f is None else _f64(f, k)
    out, r, sums = np.empty(n3), np.empty(n3), np.empty(2)
    _check(lib().ks_density_residual(n, float(h), k, _p(psi), None if fa is None else _p(fa), _p(rin), _p(out), _p(r), _p(sums)))
    return out, r, sums


def diis_mix(n, rho, r, c, a):
    """The SCF's Pulay mix: max(base + sum_{i<m-1} c_i (rho_i - base) + sum_i a_i r_i, 0), base = rho_{m-1}, for rho
    and r of shape (m, n^3)."""
    n3 = n ** 3
    rho = np.ascontiguousarray(np.asarray(rho, dtype=np.float64).reshape(-1, n3))
    r = np.ascontiguousarray(np.asarray(r, dtype=np.float64).reshape(-1, n3))
    m = rho.shape[0]
    if r.shape[0] != m:
        raise ValueError("diis_mix: one residual per density")
    ca, aa = _f64([] if c is None else c, m - 1), _f64(a, m)
    out = np.empty(n3)
    _check(lib().ks_diis_mix(n, m, _p(rho), _p(r), _p(ca) if m > 1 else None, _p(aa), _p(out)))
    return out


def fd_step_tail_kt(n_w, delta_rho_prev):
    """The witness tail (in kT) of a loosened SCF step (crates/qm/src/occupations.rs step_tail_kt)."""
    out = ctypes.c_double()
    _check(lib().ks_fd_step_tail_kt(int(n_w), float(delta_rho_prev), ctypes.byref(out)))
    return out.value


def fd_tight_columns(evals, residuals, mu, kt, tol):
    """tight_columns (crates/qm/src/occupations.rs:334-350): the positions the step's tolerance must hold (mu None or
    NaN: an empty channel, 0)."""
    ev = _f64(evals)
    rv = _f64(residuals)
    out = ctypes.c_int()
    _check(lib().ks_fd_tight_columns(_p(ev), _p(rv), len(ev), float("nan") if mu is None else float(mu), float(kt), float(tol),
                                     ctypes.byref(out)))
    return out.value


def fd_tight_start(f, n, tol):
    """tight_start (crates/qm/src/occupations.rs:355-366): a warm state's tight count from its ascending occupations
    (f None: n)."""
    fv = _f64(f) if f is not None else np.empty(0)
    out = ctypes.c_int()
    _check(lib().ks_fd_tight_start(_p(fv) if f is not None else None, len(fv), int(n), float(tol), ctypes.byref(out)))
    return out.value


def fd_witness_keep_within(evals, residuals, n, mu, kt, r_max, tail_kt=36.0):
    """The lowest converged witness (crates/qm/src/occupations.rs witness_keep_within): the count of levels to keep, or
    None when no level above the n-th passes both arms on its lower bound at a residual within r_max."""
    ev, r = _f64(evals), _f64(residuals)
    if r.size != ev.size:
        raise ValueError("fd_witness_keep_within: one residual per level")
    keep = ctypes.c_int()
    _check(lib().ks_fd_witness_keep_within(_p(ev), _p(r), ev.size, int(n), float(mu), float(kt), float(tail_kt), float(r_max),
                                           ctypes.byref(keep)))
    return None if keep.value < 0 else keep.value


def gram(n, s, t, gram_mode=0):
    s = _f64(s).reshape(-1, n ** 3)
    t = _f64(t).reshape(-1, n ** 3)
    m, mt = s.shape[0], t.shape[0]
    out = np.empty(m * (m + mt))
    _check(lib().ks_gram(n, m, _p(s), mt, _p(t), int(gram_mode), _p(out)))
    return out.reshape(m, m + mt)


def lobpcg(n, h, v, x0, tol=1e-5, max_iter=500, gram_mode=0):
    x = _f64(x0).copy()
    k = x.shape[0]
    ev = np.empty(k)
    mr, it = ctypes.c_double(), ctypes.c_int()
    _check(lib().ks_lobpcg(n, h, _p(_f64(v, n ** 3)), k, _p(x), _p(ev), float(tol), int(max_iter), int(gram_mode),
                           ctypes.byref(mr), ctypes.byref(it)))
    return ev, x, it.value, mr.value


def lobpcg_guarded(n, h, v, x0, tol, guess_tol, head, tail_tol, checked, max_iter=500, lock=True, gram_mode=0):
    """lobpcg_guarded (lock) / lobpcg_split (crates/qm-gpu/src/eigen.rs:613-653) through ks_lobpcg_guarded: columns
    [0, head) at tol, [head, checked) at tail_tol, the rest untested. Returns (evals, x, residuals, stats) with stats the
    EigenStats fields as a dict (head_kept a bool)."""
    x = _f64(x0).copy()
    k = x.shape[0]
    ev = np.empty(k)
    res = np.empty(k)
    st = _EigenStats()
    _check(lib().ks_lobpcg_guarded(n, h, _p(_f64(v, n ** 3)), k, _p(x), _p(ev), float(tol), float(guess_tol), int(head),
                                   float(tail_tol), int(checked), int(max_iter), 1 if lock else 0, int(gram_mode), _p(res),
                                   ctypes.byref(st)))
    stats = {f: getattr(st, f) for f, _ in _EigenStats._fields_}
    stats["head_kept"] = bool(stats["head_kept"])
    return ev, x, res, stats


def field_pitch(n):
    return lib().ks_field_pitch(int(n))


def launch_count():
    """Kernels of this library launched so far by the process."""
    return lib().ks_launch_count()


def gram_device_noalloc(stream, n, m, s_ptr, mt, t_ptr, out_ptr):
    """G = S^T [S | T] (CUDA-core form) on device pointers, enqueued on `stream`, allocating no device
    memory: the partial sums live in the library's 4 MiB static scratch, so m * (m + mt) is limited to
    2^19 / (2 * SMs) and calls on one device must not overlap (ks_gram_device_noalloc)."""
    _check(lib().ks_gram_device_noalloc(ctypes.c_void_p(stream), int(n), int(m), ctypes.c_void_p(s_ptr), int(mt),
                                        ctypes.c_void_p(t_ptr), ctypes.c_void_p(out_ptr)))


def hpsi_device(stream, n, h, count, psi_ptr, v_ptr, out_ptr):
    """H psi on device pointers in the pitched layout (ks_hpsi_device)."""
    _check(lib().ks_hpsi_device(ctypes.c_void_p(stream), int(n), float(h), int(count), ctypes.c_void_p(psi_ptr),
                                ctypes.c_void_p(v_ptr), ctypes.c_void_p(out_ptr)))


def device_status(stream):
    """Synchronises `stream` and raises Device when a kernel of the device-pointer entry points gave up a bounded
    wait since the last check (ks_device_status); the flag is cleared."""
    _check(lib().ks_device_status(ctypes.c_void_p(stream)))
