//! qm-b200-sys: raw bindings to `include/ks_cuda.h`, the C ABI of `libks_b200.so` (the sm_100a Kohn-Sham SCF).
//!
//! The crate a maintainer adds as `crates/qm-b200-sys` so that `qm_gpu::GpuSolver` keeps its public signatures
//! (`crates/qm-gpu/src/scf.rs:1083`, `:1195-1235`; `crates/qm-gpu/src/forces.rs:239`) and calls the B200 library
//! instead of wgpu. Every declaration below mirrors one in `include/ks_cuda.h` (same order of parameters, same C
//! types); statuses are the header's `ks_status` values (0 = KS_OK).
#![allow(non_camel_case_types)]
use std::os::raw::{c_char, c_double, c_int, c_void};

#[repr(C)] pub struct ks_nucleus { pub pos: [c_double; 3], pub z: c_int }
#[repr(C)] pub struct ks_settings { pub sigma: c_double, pub tol: c_double, pub mixing: c_double,
    pub eig_tol: c_double, pub max_iter: c_int, pub diis_history: c_int, pub stall_window: c_int,
    pub occupations: c_int /* 0 Aufbau, 1 FermiDirac */, pub kt: c_double }
#[repr(C)] pub struct ks_options { pub gram_mode: c_int, pub n_extra: c_int, pub init_mode: c_int, pub reserved: c_int }
#[repr(C)] #[derive(Default)] pub struct ks_energy { pub kinetic: f64, pub external_: f64, pub hartree: f64,
    pub xc: f64, pub nuclear: f64, pub internal: f64, pub ts: f64, pub total: f64 }
#[repr(C)] #[derive(Default)] pub struct ks_stats { pub iterations: c_int, pub delta_rho: f64, pub energy: ks_energy,
    pub boundary_density: f64, pub max_eigen_residual: f64, pub poisson_residual: f64,
    pub poisson_iterations: c_int, pub electrons: [f64; 2], pub tol_used: f64, pub n_warnings: c_int,
    pub entropy: f64, pub mu: [f64; 2], pub partial: c_int }
pub type ks_abort_fn = Option<unsafe extern "C" fn(user: *mut c_void) -> c_int>;
#[repr(C)] pub struct ks_progress { pub iteration: c_int, pub max_iter: c_int, pub delta_rho: f64, pub tol: f64, pub energy: f64,
    pub best_delta_rho: f64, pub since_gain: c_int, pub window: c_int, pub stall_level: f64 }
pub type ks_observe_fn = Option<unsafe extern "C" fn(p: *const ks_progress, user: *mut c_void)>;
#[repr(C)] #[derive(Default, Clone, Copy)] pub struct ks_eigen_stats { pub iterations: c_int, pub stop: c_int, pub head_kept: c_int,
    pub locked: c_int, pub restores: c_int, pub fallbacks: c_int, pub readbacks: c_int, pub max_residual: c_double,
    pub head_residual: c_double, pub tail_residual: c_double, pub alpha_worst: c_double }
#[repr(C)] pub struct ks_species { pub z: c_int, pub z_v: c_double, pub sigma_lr: c_double, pub du: c_double,
    pub v_sr: *const c_double, pub n_v_sr: c_int, pub r_sr: c_double,
    pub rho_pc: *const c_double, pub n_rho_pc: c_int, pub pc_radius: c_double,
    pub n_proj: c_int, pub proj_l: *const c_int, pub proj_e_kb: *const c_double, pub proj_radius: *const c_double,
    pub proj_t: *const *const c_double, pub proj_n: *const c_int }

#[link(name = "ks_b200")]
extern "C" {
    pub fn ks_solver_create(n: c_int, h: c_double, opts: *const ks_options) -> *mut c_void;
    pub fn ks_solver_destroy(s: *mut c_void);
    pub fn ks_solve(s: *mut c_void, nuc: *const ks_nucleus, n_nuc: c_int, n_up: c_int, n_dn: c_int,
                    settings: *const ks_settings, warm: c_int, abort: ks_abort_fn, user: *mut c_void,
                    out: *mut ks_stats) -> c_int;
    pub fn ks_forces(s: *mut c_void, nuc: *const ks_nucleus, n_nuc: c_int, sigma: c_double, out3n: *mut c_double) -> c_int;
    pub fn ks_last_error(s: *const c_void) -> *const c_char;
    pub fn ks_state_counts(s: *const c_void, n_up: *mut c_int, n_dn: *mut c_int) -> c_int;
    pub fn ks_state_evals(s: *const c_void, up: *mut c_double, dn: *mut c_double) -> c_int;
    pub fn ks_state_density(s: *const c_void, up: *mut c_double, dn: *mut c_double) -> c_int;
    pub fn ks_vjp(s: *mut c_void, nuc: *const ks_nucleus, n_nuc: c_int, sigma: c_double, e_bar: c_double,
                  de_dr3n: *mut c_double, de_dsigma: *mut c_double) -> c_int;
    pub fn ks_solve_observed(s: *mut c_void, nuc: *const ks_nucleus, n_nuc: c_int, n_up: c_int, n_dn: c_int,
                             settings: *const ks_settings, warm: c_int, abort: ks_abort_fn, inner_abort: ks_abort_fn,
                             observe: ks_observe_fn, user: *mut c_void, out: *mut ks_stats) -> c_int;
    pub fn ks_footprint_bytes(n: c_int, n_up: c_int, n_dn: c_int, opts: *const ks_options, diis_history: c_int,
                              with_core: c_int) -> i64;
    pub fn ks_set_ionic(s: *mut c_void, species: *const ks_species, n: c_int) -> c_int;
    pub fn ks_sample_density(s: *mut c_void, pts3: *const c_double, count: c_int, out: *mut f32) -> c_int;
    pub fn ks_state_density_f32(s: *mut c_void, rho: *mut f32) -> c_int;
    pub fn ks_density_max(s: *mut c_void, out: *mut c_double) -> c_int;
    pub fn ks_spin_abs_integral(s: *mut c_void, out: *mut c_double) -> c_int;
    pub fn ks_sampling_counters(s: *const c_void, readbacks: *mut c_int, allocations: *mut c_int) -> c_int;
    pub fn ks_state_occupations(s: *const c_void, up: *mut c_double, dn: *mut c_double) -> c_int;
    pub fn ks_state_potentials(s: *const c_void, v_nuc: *mut c_double, v_h: *mut c_double) -> c_int;
    pub fn ks_state_orbitals(s: *const c_void, spin: c_int, out: *mut c_double) -> c_int;
    pub fn ks_profile_get(s: *const c_void, out: *mut ks_profile) -> c_int;
    pub fn ks_state_import(s: *mut c_void, n_up: c_int, n_dn: c_int, k_up: c_int, orbitals_up: *const c_double,
                           evals_up: *const c_double, k_dn: c_int, orbitals_dn: *const c_double, evals_dn: *const c_double,
                           rho_up: *const c_double, rho_dn: *const c_double, v_h: *const c_double, occupations: c_int,
                           occ_up: *const c_double, occ_dn: *const c_double) -> c_int;
    // failure-injection hooks (the tests of the failure paths)
    pub fn ks_test_poison_parked_density(s: *mut c_void) -> c_int;
    pub fn ks_test_fail_readbacks(s: *mut c_void, skip: c_int, count: c_int) -> c_int;
    pub fn ks_set_kernel_timing(s: *mut c_void, on: c_int) -> c_int;
    pub fn ks_kernel_times(s: *mut c_void, out: *mut ks_kernel_time, cap: c_int) -> c_int;
    pub fn ks_apply_nonlocal(s: *mut c_void, nuc: *const ks_nucleus, n_nuc: c_int, count: c_int, x: *const c_double,
                             out: *mut c_double, c: *mut c_double, rows: *mut c_int) -> c_int;
    // component entry points (one stage of the SCF on host f64 arrays in the qm::Grid layout)
    pub fn ks_apply_hamiltonian(n: c_int, h: c_double, count: c_int, psi: *const c_double, v: *const c_double,
                                out: *mut c_double) -> c_int;
    pub fn ks_apply_laplacian(n: c_int, h: c_double, f: *const c_double, out: *mut c_double) -> c_int;
    pub fn ks_apply_precond(n: c_int, h: c_double, v: *const c_double, lambda: c_double, r: *const c_double,
                            w: *mut c_double) -> c_int;
    pub fn ks_xc_lsda(len: usize, up: *const c_double, dn: *const c_double, e: *mut c_double, vu: *mut c_double,
                      vd: *mut c_double) -> c_int;
    pub fn ks_nuclear_potential(n: c_int, h: c_double, nuc: *const ks_nucleus, n_nuc: c_int, sigma: c_double,
                                out: *mut c_double) -> c_int;
    pub fn ks_poisson_solve(n: c_int, h: c_double, rho: *const c_double, v: *mut c_double, tol: c_double, max_iter: c_int,
                            residual: *mut c_double, iterations: *mut c_int) -> c_int;
    pub fn ks_lobpcg(n: c_int, h: c_double, v: *const c_double, k: c_int, x: *mut c_double, evals: *mut c_double,
                     tol: c_double, max_iter: c_int, gram_mode: c_int, max_residual: *mut c_double,
                     iterations: *mut c_int) -> c_int;
    pub fn ks_lobpcg_guarded(n: c_int, h: c_double, v: *const c_double, k: c_int, x: *mut c_double, evals: *mut c_double,
                             tol: c_double, guess_tol: c_double, head: c_int, tail_tol: c_double, checked: c_int,
                             max_iter: c_int, lock: c_int, gram_mode: c_int, residuals: *mut c_double,
                             stats: *mut ks_eigen_stats) -> c_int;
    pub fn ks_multipole_moments(n: c_int, h: c_double, rho: *const c_double, q49: *mut c_double) -> c_int;
    pub fn ks_launch_count() -> i64;
    // host-only parity hooks (the solver's f64 host algebra)
    pub fn ks_rayleigh_ritz(m: c_int, a: *const c_double, b: *const c_double, nk: c_int, theta: *mut c_double,
                            c: *mut c_double, alpha: *mut c_double) -> c_int;
    pub fn ks_fermi_dirac(evals: *const c_double, k: c_int, n: c_int, kt: c_double, f: *mut c_double, mu: *mut c_double,
                          entropy: *mut c_double) -> c_int;
    pub fn ks_fd_witness(evals: *const c_double, k: c_int, n: c_int, mu: c_double, kt: c_double, reached: *mut c_int,
                         keep: *mut c_int) -> c_int;
    pub fn ks_fd_step_tail_kt(n_w: c_int, delta_rho_prev: c_double, tail_kt: *mut c_double) -> c_int;
    pub fn ks_fd_tight_columns(evals: *const c_double, residuals: *const c_double, k: c_int, mu: c_double, kt: c_double,
                               tol: c_double, tight: *mut c_int) -> c_int;
    pub fn ks_fd_tight_start(f: *const c_double, k: c_int, n: c_int, tol: c_double, tight: *mut c_int) -> c_int;
    pub fn ks_fd_witness_keep_within(evals: *const c_double, residuals: *const c_double, k: c_int, n: c_int, mu: c_double,
                                     kt: c_double, tail_kt: c_double, r_max: c_double, keep: *mut c_int) -> c_int;
    pub fn ks_fd_witness_bound(evals: *const c_double, residuals: *const c_double, k: c_int, n: c_int, mu: c_double,
                               kt: c_double, reached: *mut c_int, keep: *mut c_int) -> c_int;
    pub fn ks_solve_batch(jobs: *mut ks_batch_job, n_jobs: c_int, opts: *const ks_options, workers: c_int) -> c_int;
    pub fn ks_set_density_extrapolation(s: *mut c_void, on: c_int) -> c_int;
    pub fn ks_set_witness_cap(s: *mut c_void, cap: c_int) -> c_int;
    pub fn ks_effective_eig_tol(s: *const c_void, eig_tol: c_double, out: *mut c_double) -> c_int;
    pub fn ks_density_to_volume(s: *mut c_void, dense_dev: *mut f32, stream: *mut c_void) -> c_int;
    pub fn ks_density_with_core_to_volume(s: *mut c_void, dense_dev: *mut f32, stream: *mut c_void,
                                          max_out: *mut c_double) -> c_int;
    pub fn ks_autotune_stencil(n: c_int, counts: *const c_int, ncount: c_int, chunks_out: *mut c_int) -> c_int;
    pub fn ks_stencil_tuning_get(entries4: *mut c_int, cap: c_int) -> c_int;
    pub fn ks_stencil_tuning_set(entries4: *const c_int, count: c_int) -> c_int;
    pub fn ks_stencil_tuning_clear() -> c_int;
    pub fn ks_density_residual(n: c_int, h: c_double, k: c_int, psi: *const c_double, f: *const c_double, rho_in: *const c_double,
                               rho_out: *mut c_double, r: *mut c_double, sums: *mut c_double) -> c_int;
    pub fn ks_diis_mix(n: c_int, m: c_int, rho: *const c_double, r: *const c_double, c: *const c_double, a: *const c_double,
                       out: *mut c_double) -> c_int;
    pub fn ks_gram(n: c_int, m: c_int, s: *const c_double, mt: c_int, t: *const c_double, gram_mode: c_int,
                   out: *mut c_double) -> c_int;
    // device-pointer entry points (pitched f32 fields on the caller's stream; section 4)
    pub fn ks_field_pitch(n: c_int) -> c_int;
    pub fn ks_solver_stream(s: *mut c_void) -> *mut c_void;
    pub fn ks_hpsi_device(stream: *mut c_void, n: c_int, h: c_double, count: c_int, psi: *const f32, v: *const f32,
                          out: *mut f32) -> c_int;
    pub fn ks_gram_device_noalloc(stream: *mut c_void, n: c_int, m: c_int, s: *const f32, mt: c_int, t: *const f32,
                                  out: *mut c_double) -> c_int;
    // wait-timeout status of the device-pointer entry points (synchronises the stream)
    pub fn ks_device_status(stream: *mut c_void) -> c_int;
}
#[repr(C)] pub struct ks_batch_job { pub n: c_int, pub h: c_double, pub nuclei: *const ks_nucleus, pub n_nuclei: c_int,
    pub n_up: c_int, pub n_dn: c_int, pub settings: ks_settings, pub forces3n: *mut c_double, pub stats: ks_stats,
    pub status: c_int, pub error: [c_char; 160] }
#[repr(C)] #[derive(Default)] pub struct ks_profile { pub steps: c_int, pub readbacks: c_int, pub eigen_iterations: c_int,
    pub poisson_iterations: c_int, pub eigen_calls: c_int, pub diis_resets: c_int, pub wall_s: f64, pub start_s: f64,
    pub poisson_s: f64, pub eigen_s: f64, pub host_dense_s: f64, pub sync_wait_s: f64, pub witness_growths: c_int,
    pub extrapolated: c_int, pub locked_calls: c_int, pub class_raises: c_int, pub buffer_witnesses: c_int,
    pub buffer_growths: c_int, pub lower_witnesses: c_int, pub witness_residual_growths: c_int, pub witness_trims: c_int,
    pub frozen_steps: c_int, pub diis_freeze_trims: c_int, pub peak_block: c_int }
#[repr(C)] #[derive(Default, Clone, Copy)] pub struct ks_kernel_time { pub kernel: c_int, pub count: c_int, pub aux: c_int,
    pub launches: c_int, pub total_ms: f64, pub bytes: f64 }
