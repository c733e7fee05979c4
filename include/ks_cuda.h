/*
 * ks_cuda.h -- C ABI of the B200 (sm_100a) real-space Kohn-Sham solver.
 *
 * This is the drop-in boundary for the reference's GPU solver, the Rust type
 * `qm_gpu::GpuSolver` (crates/qm-gpu/src/scf.rs:1042-1235, crates/qm-gpu/src/forces.rs:239).
 * A handle owns one grid, one CUDA stream and every device buffer of the solve; it is
 * thread-affine like the reference (`Send`, not `Sync`: one handle per worker thread). Every
 * call is synchronous with respect to the host and returns a status -- the library never traps.
 *
 * Array conventions at the boundary: grids are cubic n^3 with spacing h (Bohr), origin
 * -(n-1)h/2 on every axis, and a host array of a grid field is the reference's `qm::Grid`
 * layout, f64, idx = i + n*(j + n*k) (crates/qm/src/grid.rs:1-16). Energies in Hartree, forces
 * in Hartree/Bohr. Nothing here takes a torch type.
 */
#ifndef KS_CUDA_H
#define KS_CUDA_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

/* qm::Nucleus (crates/qm/src/nuclear.rs:88-92): position in Bohr and atomic number. */
typedef struct { double pos[3]; int z; } ks_nucleus;

/* qm::QmError (crates/qm/src/error.rs:4-31) plus the C-side conditions. */
typedef enum {
    KS_OK = 0,
    KS_COINCIDENT_NUCLEI = 1, /* QmError::CoincidentNuclei */
    KS_NOT_CONVERGED = 2,     /* QmError::ScfNotConverged */
    KS_STALLED = 3,           /* QmError::ScfStalled */
    KS_NUMERICAL = 4,         /* QmError::Numerical */
    KS_DEVICE = 5,            /* QmError::Device (a CUDA error or a kernel wait that gave up) */
    KS_INVALID = 6,           /* bad argument (the reference panics on these) */
    KS_ABORTED = 7,           /* should_abort returned nonzero: the iterate is parked as the warm start */
    KS_NO_STATE = 8           /* forces / state access without a converged state */
} ks_status;

/* qm::ScfSettings (crates/qm/src/scf.rs:375), Aufbau occupations. */
typedef struct {
    double sigma;      /* nuclear smearing width (Bohr); the reference's default is h */
    double tol;        /* on the density change dRho = integral |rho_out - rho_in| (electrons) */
    double mixing;     /* DIIS step alpha (0.3) */
    double eig_tol;    /* LOBPCG residual tolerance (1e-6) */
    int max_iter;      /* SCF iteration cap (200) */
    int diis_history;  /* Pulay history (6) */
    int stall_window;  /* stall stop W (50; 0 = off) */
    int occupations;   /* qm::Occupations (crates/qm/src/scf.rs:278): 0 Aufbau, 1 Fermi-Dirac at kt over a block of at least
                          N_sigma + n_extra levels per occupied channel (ks_options.n_extra >= 1), solved as the reference's
                          GPU channel solve (crates/qm-gpu/src/scf.rs:875-1029): the top column an untested buffer, the
                          block grown by one vector or by doubling its extra levels (at most 32) until a tested level's
                          lower bound theta - r is a gap witness (crates/qm/src/occupations.rs), the overshoot trimmed */
    double kt;         /* Fermi-Dirac temperature (Ha), e.g. 5e-3 (ELECTRON_KT, occupations.rs) */
} ks_settings;

/* Solver construction options (no reference counterpart: B200 choices). */
typedef struct {
    int gram_mode;     /* LOBPCG Gram: 0 = FP32 CUDA cores ("plain FP32"), 1 = tensor cores (3xTF32, "mixed") */
    int n_extra;       /* extra LOBPCG bands per occupied spin channel (buffer columns, not occupied) */
    int init_mode;     /* cold orbitals: 0 = the reference's initial_orbitals (crates/qm/src/scf.rs:636-644), 1 = uniform(-1,1) */
    int reserved;
} ks_options;

/* qm::Energy (crates/qm/src/scf.rs:533) */
typedef struct { double kinetic, external_, hartree, xc, nuclear, internal, ts, total; } ks_energy;

/* qm::ScfStats (crates/qm/src/scf.rs:558-574), Aufbau subset. */
typedef struct {
    int iterations;
    double delta_rho;
    ks_energy energy;
    double boundary_density;
    double max_eigen_residual;
    double poisson_residual;
    int poisson_iterations;
    double electrons[2];
    double tol_used;
    int n_warnings;
    double entropy;    /* Fermi-Dirac: S summed over the channels (energy.ts = kt * S, energy.total = F = internal - ts) */
    double mu[2];      /* Fermi-Dirac: mu per spin (NaN for an empty channel or under Aufbau) */
    int partial;       /* Fermi-Dirac: the final step had a partly occupied level (stop at max(tol, 1e-5)) */
} ks_stats;

/* qm_gpu::SolveProfile (crates/qm-gpu/src/scf.rs:448-514), subset. */
typedef struct {
    int steps, readbacks, eigen_iterations, poisson_iterations, eigen_calls, diis_resets;
    double wall_s, start_s, poisson_s, eigen_s;
    double host_dense_s;  /* host time in the f64 Rayleigh-Ritz / DIIS algebra */
    double sync_wait_s;   /* host time blocked on device results (readbacks) */
    int witness_growths;  /* Fermi-Dirac blocks grown for their gap witness (SolveProfile's witness growth count) */
    int extrapolated;     /* the warm start's input density was extrapolated (SolveProfile::extrapolated) */
    /* Fermi-Dirac channel solves (SolveProfile, crates/qm-gpu/src/scf.rs:473-503): LOBPCG calls that locked the head while
       only the loose columns iterated; re-solves for a column that needed the step's tol (class raises); solves decided
       by the buffer's own bound; buffers that passed above the guard tolerance and grew the block by one; tight steps
       decided by a lower converged witness; tight steps grown by one for a top witness above 1.5 x the guard tolerance;
       trims above the lowest witness; frozen steps (every call kept its tight columns); frozen steps that stalled and
       dropped the older DIIS entries; the largest block any channel solved with. */
    int locked_calls, class_raises, buffer_witnesses, buffer_growths, lower_witnesses, witness_residual_growths;
    int witness_trims, frozen_steps, diis_freeze_trims, peak_block;
} ks_profile;

/* Device time of one launch shape of a solver's hot kernels (instrumentation, no reference counterpart): kernel
   (KS_K_*), count (vectors of a stencil or residual launch, m of a Gram or block update), aux (mt of a Gram, q of a
   block update, else 0), launches, their summed device time (CUDA events on the stream they ran on) and the
   algorithmic bytes of one launch (what it must read and write once, on the n^3 interior points). */
typedef struct { int kernel, count, aux, launches; double total_ms, bytes; } ks_kernel_time;
enum { KS_K_HPSI = 0, KS_K_JACOBI = 1, KS_K_RESIDUAL = 2, KS_K_GRAM = 3, KS_K_BLOCK_UPDATE = 4, KS_K_HPSI_RESIDUAL = 5 };

/* Polled before every SCF step (GpuSolver::solve_with, crates/qm-gpu/src/scf.rs:1208): nonzero abandons the solve. */
typedef int (*ks_abort_fn)(void* user);

/* GpuSolver::new (crates/qm-gpu/src/scf.rs:1083): a solver for the cubic grid n^3, spacing h, on the
   current CUDA device. opts may be NULL (defaults: plain FP32 Gram, no extra bands, reference guess).
   Returns NULL on failure (ks_last_error(NULL) holds the message). */
void* ks_solver_create(int n, double h, const ks_options* opts);
void ks_solver_destroy(void* solver);

/* The device memory (bytes) a solver of the n^3 grid holds through a solve with n_up / n_dn electrons and its forces:
   its own buffers, not the CUDA context or the loaded kernels; with_core adds the fields of an ionic setup with a
   partial core. The B200 counterpart of the provider's footprint estimate (crates/providers/src/ks.rs:465-470,
   solve_footprint_bytes), which a caller compares with a memory budget before building a solver
   (GpuKs::check_vram, ks.rs:1303-1324). opts may be NULL; negative for invalid arguments. */
long long ks_footprint_bytes(int n, int n_up, int n_dn, const ks_options* opts, int diis_history, int with_core);

/* qm::ScfProgress (crates/qm/src/scf.rs:488-498): one SCF step as an observer sees it, after its dRho readback and
   before the convergence test. energy is the Harris-Foulkes energy of the step's input density (F_HF = sum f eps
   + double counting - kT S of the step's occupations); best_delta_rho, since_gain, window and stall_level are the
   stall watch's. */
typedef struct {
    int iteration, max_iter;
    double delta_rho, tol, energy, best_delta_rho;
    int since_gain, window;
    double stall_level;
} ks_progress;
typedef void (*ks_observe_fn)(const ks_progress* progress, void* user);

/* One pseudised species: what the grid samples of the reference's qm::radial::filter::FilteredTable
   (crates/qm/src/radial/filter.rs:323-363) for one element at this grid's h. Every table is an even function
   tabulated at d = k du, k = 0 .. n-1 (the reference's du = h / 256), read by 4-point Lagrange with index -1
   mirrored onto 1 and 0 beyond its radius (filter.rs:302-317). The caller keeps the arrays; ks_set_ionic copies them.
     V_LR(d)  = -z_v erf(d / (sigma_lr sqrt2)) / d           (analytic; every pseudised centre)
     V_SR(d)  = v_sr table within r_sr                         (n_v_sr = 0: none)
     rho_pc   = rho_pc table within pc_radius                 (pc_radius <= 0: no partial core)
     beta_lm  = t_l(d) sqrt((2l+1)/4pi) R_lm(d - R)           (projector i: l <= 2, E_KB, radius, table t) */
typedef struct {
    int z;                       /* nuclei of this atomic number are pseudised */
    double z_v;                  /* valence charge */
    double sigma_lr;             /* width of the long-range part (the reference uses 2h) */
    double du;                   /* table spacing (Bohr) */
    const double* v_sr; int n_v_sr; double r_sr;
    const double* rho_pc; int n_rho_pc; double pc_radius;
    int n_proj;                  /* at most 4 */
    const int* proj_l; const double* proj_e_kb; const double* proj_radius;
    const double* const* proj_t; const int* proj_n;
} ks_species;

/* The ionic setup of the solver's next solves (qm::ionic::IonicSetup, crates/qm/src/ionic.rs:56-63, its tables given
   as above): nuclei whose Z is listed are pseudised, every other nucleus stays an all-electron smeared charge of width
   settings.sigma. n_species = 0 restores the all-electron solver. Under a setup (crates/qm/src/scf.rs:114-140):
   V_ext is V_loc = sum V_LR + sum V_SR; every H psi adds the Kleinman-Bylander V_NL = sum E_KB |beta><beta| (the
   Jacobi preconditioner stays local); XC runs on (rho_up + rho_pc/2, rho_dn + rho_pc/2); energy.external_ =
   integral rho V_loc + E_NL; energy.nuclear is the repulsion of the valence charges; the cold guess deposits each
   centre's charge. n_up / n_dn passed to ks_solve count the valence electrons. A converged state from another setup
   is never reused as a warm start. At most 8 species, 4 projectors each (l <= 2), 32 nuclei. */
ks_status ks_set_ionic(void* solver, const ks_species* species, int n_species);

/* The Kleinman-Bylander operator of the solver's ionic setup at these nuclei (the GPU's proj_dot / proj_finish /
   proj_axpy, crates/qm-gpu/src/ionic.rs; qm::nonlocal::NonlocalOp::apply_add): out_v = V_NL x_v for count host
   vectors (n^3 each, f64 in and out, f32 on the device), and, when c is not NULL, the projections
   c[v * rows + row] = h^3 <beta_row, x_v> in sphere order (ion, projector, m = -l..l). *rows gets the row count. */
ks_status ks_apply_nonlocal(void* solver, const ks_nucleus* nuclei, int n_nuclei, int count, const double* x, double* out, double* c,
                            int* rows);

/* GpuSolver::solve / solve_with (crates/qm-gpu/src/scf.rs:1195-1235): n_up / n_dn electrons per spin,
   warm != 0 reuses the last converged state when its counts match. abort may be NULL. */
ks_status ks_solve(void* solver, const ks_nucleus* nuclei, int n_nuclei, int n_up, int n_dn, const ks_settings* settings,
                   int warm, ks_abort_fn abort_fn, void* user, ks_stats* out);

/* GpuSolver::solve_observed / solve_polled (crates/qm-gpu/src/scf.rs:1213-1235): ks_solve with a second cancellation
   point and an observer. inner_abort (may be NULL) is also polled once per LOBPCG iteration of the calling thread's
   eigensolve, so an abort lands within one iteration rather than one SCF step; it abandons the solve like abort_fn
   (KS_ABORTED, the iterate parked as the next warm start). observe (may be NULL) gets one ks_progress per SCF step; it
   changes no number of the solve. Both callbacks run on the calling thread and get `user`. */
ks_status ks_solve_observed(void* solver, const ks_nucleus* nuclei, int n_nuclei, int n_up, int n_dn, const ks_settings* settings,
                            int warm, ks_abort_fn abort_fn, ks_abort_fn inner_abort, ks_observe_fn observe, void* user, ks_stats* out);

/* GpuSolver::forces (crates/qm-gpu/src/forces.rs:239): Hellmann-Feynman force on each nucleus
   (out3n[3*i + axis]) from the converged state, plus the point nuclear repulsion. */
ks_status ks_forces(void* solver, const ks_nucleus* nuclei, int n_nuclei, double sigma, double* out3n);

/* Reverse-mode derivative (vector-Jacobian product) of the converged total energy E with respect to the
   nuclear positions and the smearing width: dE_dR3n[3*i + axis] = e_bar * dE/dR_i, *dE_dsigma = e_bar *
   dE/dsigma. At self-consistency E is stationary in the density, so the Hartree, XC and kinetic responses
   vanish and the product is the explicit derivative of the external energy (rho recomputed on the device
   from the occupied orbitals) plus the point-nuclear repulsion. No reference counterpart (new API); its
   position part equals -GpuSolver::forces (crates/qm-gpu/src/forces.rs:239). */
ks_status ks_vjp(void* solver, const ks_nucleus* nuclei, int n_nuclei, double sigma, double e_bar, double* dE_dR3n,
                 double* dE_dsigma);

/* One geometry of a batch: its grid, system and settings in; its statistics, forces and status out. */
typedef struct {
    int n;                     /* grid points per axis */
    double h;                  /* spacing (Bohr) */
    const ks_nucleus* nuclei;
    int n_nuclei;
    int n_up, n_dn;
    ks_settings settings;
    double* forces3n;          /* out (3 * n_nuclei doubles), or NULL for no forces */
    ks_stats stats;            /* out */
    int status;                /* out: the job's ks_status */
    char error[160];           /* out: the job's message when status != KS_OK */
} ks_batch_job;

/* Independent cold solves (and forces) of many geometries on the current device: the batched sample generation of the
   providers (one GpuSolver per grid, crates/providers/src/ks.rs) run by `workers` host threads, each with its own solver
   and streams, so one geometry's kernels fill the GPU while another waits on a readback. A thread keeps its solver for
   the next job on the same grid. Each job's result is that of a lone cold ks_solve + ks_forces (bit for bit, whatever
   the scheduling). Returns KS_OK once every job has run (see each job's status), KS_INVALID for bad arguments.
   No reference counterpart: the reference solves a batch one geometry at a time. */
ks_status ks_solve_batch(ks_batch_job* jobs, int n_jobs, const ks_options* opts, int workers);

/* GpuSolver::set_density_extrapolation (crates/qm-gpu/src/scf.rs:1146-1163): with on != 0 a warm solve starts from
   rho_in = max(2 rho_t - rho_{t-1}, 0), the linear extrapolation in time of the last two converged output densities,
   instead of rho_t (the caller's contract: equal time steps). rho_{t-1} is dropped by a cold solve, a solve that does not
   converge (error or abandoned), a change of orbital counts and by turning extrapolation off; an MD caller resets the
   chain after a discontinuous move by turning it off and on. Orbitals and V_H are warm-started as without it. */
ks_status ks_set_density_extrapolation(void* solver, int on);
/* GpuSolver::set_witness_cap (scf.rs:1122-1132): at most cap extra Fermi-Dirac levels per channel, clamped to 1..32. */
ks_status ks_set_witness_cap(void* solver, int cap);
/* GpuSolver::effective_eig_tol (scf.rs:1713-1715): the LOBPCG tolerance the SCF's final step converges to,
   max(eig_tol, 3 x the f32 residual floor of this grid). */
ks_status ks_effective_eig_tol(const void* solver, double eig_tol, double* out);

/* The message of the last failure on this handle (or of ks_solver_create when solver is NULL). */
const char* ks_last_error(const void* solver);

/* State access (GpuSolver::state / ks_state, crates/qm-gpu/src/scf.rs:1172, :1713-1775). */
ks_status ks_state_counts(const void* solver, int* n_up, int* n_dn);
ks_status ks_state_evals(const void* solver, double* up, double* dn);
/* One occupation per stored orbital (qm::KsState occ_up / occ_dn): all 1 under Aufbau, the final step's Fermi-Dirac f
   otherwise, where the stored block is N_sigma + n_extra levels (ks_state_counts reports the block sizes). */
ks_status ks_state_occupations(const void* solver, double* up, double* dn);
ks_status ks_state_density(const void* solver, double* rho_up, double* rho_dn);   /* n^3 each */
ks_status ks_state_potentials(const void* solver, double* v_nuc, double* v_h);     /* n^3 each */
ks_status ks_state_orbitals(const void* solver, int spin, double* out);            /* count * n^3 */
/* The warm start of the next ks_solve(warm = 1) from a saved state, the inverse of the getters above: the reference
   parks the whole GpuState (orbitals, levels, rho_up / rho_dn, V_H, occupations) between solves and resumes from it
   (crates/qm-gpu/src/scf.rs:1286-1323, GpuState :410-418); here the state can come from host memory, e.g. one
   exported by another solver of the same grid. Per spin k_up / k_dn orbitals (f64, k * n^3 in the qm::Grid layout)
   with their levels, N_sigma <= k <= N_sigma + n_extra; columns of the block beyond k start from the uniform(-1, 1)
   guess. rho_up, rho_dn, v_h: n^3 each. occupations: 0 Aufbau, 1 Fermi-Dirac (occ_up / occ_dn then hold one f per
   orbital; NULL under Aufbau). The next solve must name the same n_up / n_dn and occupation scheme to be warm.
   The imported state is not a converged state: the getters and ks_forces report KS_NO_STATE until a solve converges. */
ks_status ks_state_import(void* solver, int n_up, int n_dn, int k_up, const double* orbitals_up, const double* evals_up,
                          int k_dn, const double* orbitals_dn, const double* evals_dn, const double* rho_up,
                          const double* rho_dn, const double* v_h, int occupations, const double* occ_up, const double* occ_dn);
/* Failure-injection hooks for the failure-path tests, the counterparts of the reference's fault-injection feature
   (crates/gpu/src/readback.rs:36-58, crates/qm-gpu/src/scf.rs:2400-2460); nothing calls them in normal use.
   ks_test_poison_parked_density writes a NaN into the parked warm density (the next warm solve must end in
   KS_NUMERICAL). ks_test_fail_readbacks lets `skip` of this solver's readbacks through and fails the next `count`
   as a readback that never delivers (KS_DEVICE); (0, 0) clears it. Neither touches the GPU's state. */
ks_status ks_test_poison_parked_density(void* solver);
ks_status ks_test_fail_readbacks(void* solver, int skip, int count);
ks_status ks_profile_get(const void* solver, ks_profile* out);                     /* GpuSolver::profile */
/* Kernel timing of the LOBPCG chain (H psi, the Jacobi sweeps, the residual, the Gram, the block update), off by
   default: while on, each launch is bracketed by two CUDA events on its stream and the two spin channels run one
   after the other, so that each launch is timed alone (the results are unchanged; the solve is slower). Switching
   it on clears the totals. ks_kernel_times waits for the recorded
   launches, fills at most cap shapes into out and returns the number of shapes (negative on an invalid handle). */
ks_status ks_set_kernel_timing(void* solver, int on);
int ks_kernel_times(void* solver, ks_kernel_time* out, int cap);

/* ---- readouts of the converged state (display and diagnostics; nothing is fed back into a solve) ---- */
/* GpuSolver::sample_density (crates/qm-gpu/src/sample.rs:84-121): rho_up + rho_dn at count points (pts3[3*q + axis],
   Bohr) by trilinear interpolation with the cell and fractions of qm::Grid::trilinear_cell (crates/qm/src/grid.rs:54-67,
   resolved in f64) and the blend a(1 - t) + b t along x, then y, then z in f32; 0 outside [origin, origin + (n-1)h]^3
   (NaN coordinates included); a grid point returns the stored f32 exactly. One launch and one readback per call with
   count > 0; count = 0 does no GPU work. The point buffers grow to the largest request and are reused. */
ks_status ks_sample_density(void* solver, const double* pts3, int count, float* out);
/* Calls of ks_sample_density that reached the GPU, and the buffer sets it has allocated (the reuse witness:
   sample.rs sampling_readbacks / sampling_buffer_allocations). */
ks_status ks_sampling_counters(const void* solver, int* readbacks, int* allocations);
/* GpuSolver::density_f32 (crates/qm-gpu/src/scf.rs:1776-1779): the interior of rho_up + rho_dn as stored (f32, n^3,
   x fastest). */
ks_status ks_state_density_f32(void* solver, float* rho);
/* GpuSolver::copy_density_to_volume (crates/qm-gpu/src/scf.rs:1780-1797) with a headless device buffer in place of
   the 3-D texture: writes the n^3 f32 image (x fastest, no padding) of rho_up + rho_dn to dense_dev on the solver's
   device, enqueued on `stream` (a cudaStream_t; NULL = the solver's stream) after the solver's own work. Does not
   wait. */
ks_status ks_density_to_volume(void* solver, float* dense_dev, void* stream);
/* GpuSolver::copy_density_with_core_to_volume (crates/qm-gpu/src/scf.rs:1798-1829): as ks_density_to_volume for
   rho_up + rho_dn + rho_pc, the model partial core of a state solved under an ionic setup (the plain density when
   there is none); *max_out gets the maximum of the field written (one readback). */
ks_status ks_density_with_core_to_volume(void* solver, float* dense_dev, void* stream, double* max_out);
/* GpuSolver::density_max (scf.rs:1831-1834): max of rho_up + rho_dn over the interior (one readback). */
ks_status ks_density_max(void* solver, double* out);
/* GpuSolver::spin_abs_integral (scf.rs:1836-1842): the integral of |rho_up - rho_dn| in electrons (one readback). */
ks_status ks_spin_abs_integral(void* solver, double* out);

/* ---- grid-kernel entry points (host f64 in / out; the kernels run on the solver's device in f32) ----
   One parity hook per hot-path kernel; each mirrors the reference kernel named beside it. */
/* hamiltonian (crates/qm-gpu/src/shaders/stencil.wgsl:77-90): out_v = -1/2 lap psi_v + V psi_v for count vectors */
ks_status ks_apply_hamiltonian(int n, double h, int count, const double* psi, const double* v, double* out);
/* laplacian (stencil.wgsl:67-75) */
ks_status ks_apply_laplacian(int n, double h, const double* f, double* out);
/* precond_init + jacobi_step x3 (shaders/eigen.wgsl:25-34, stencil.wgsl:94-106): w = T r at shift lambda */
ks_status ks_apply_precond(int n, double h, const double* v, double lambda, const double* r, double* w);
/* xc_lsda (shaders/xc.wgsl:137-152): e = n eps_xc, v_up, v_dn for len points */
ks_status ks_xc_lsda(size_t len, const double* up, const double* dn, double* e, double* vu, double* vd);
/* nuclear_potential (shaders/nuclear.wgsl:124-139) */
ks_status ks_nuclear_potential(int n, double h, const ks_nucleus* nuclei, int n_nuclei, double sigma, double* out);
/* GpuPoisson::solve (crates/qm-gpu/src/poisson.rs:284-342): MG-PCG with l<=6 multipole ghosts.
   v is the initial guess and the output; returns the true relative residual and the iteration count. */
ks_status ks_poisson_solve(int n, double h, const double* rho, double* v, double tol, int max_iter, double* residual,
                           int* iterations);
/* The SCF's density step on host arrays, the kernel and finish the solve runs (crates/qm-gpu/src/scf.rs: the output
   density as pointwise mul_add_sq over the orbitals, its residual against the input and the step's |r| and charge
   reductions): rho_out = sum_i f_i psi_i^2 over k orbitals of n^3 points (f NULL: every f_i = 1; f is applied in f32),
   r = rho_out - rho_in, sums = (h^3 sum |r|, h^3 sum rho_out) summed in f64. 0 <= k <= 64. */
ks_status ks_density_residual(int n, double h, int k, const double* psi, const double* f, const double* rho_in, double* rho_out,
                              double* r, double* sums);
/* The SCF's Pulay mix on host arrays (crates/qm-gpu/src/scf.rs:628-645, pointwise diis_mix re-centred on the latest
   input): out = max(base + sum_{i<m-1} c_i (rho_i - base) + sum_{i<m} a_i r_i, 0) with base = rho_{m-1}; rho and r
   hold m fields of n^3 points each, c m - 1 and a m coefficients (applied in f32), 1 <= m <= 16; c may be NULL for
   m = 1. */
ks_status ks_diis_mix(int n, int m, const double* rho, const double* r, const double* c, const double* a, double* out);
/* The stencil's launch-shape autotuner. For an n^3 grid and each of the ncount vector counts (1..64), times every
   distinct z-chunking of H psi and of the Jacobi sweep on zeroed scratch fields of the current device (CUDA events, the
   best of three timings of four launches) and records the fastest in a process-wide table that later launches of that
   shape on this device use. Only these two modes are tuned: their outputs do not depend on the chunking, so a tuned
   solve gives the same bits as an untuned one. chunks_out (2 * ncount ints, may be NULL) receives the choices, H psi
   then the sweep for each count. Synchronises the device's work on its own stream; takes well under a second at 95^3. */
ks_status ks_autotune_stencil(int n, const int* counts, int ncount, int* chunks_out);
/* The tuning table of the current device as (n, count, mode, chunks) quadruples (mode 1 H psi, 2 the sweep): copies up
   to cap entries and returns their total number (-1 without a device). _set installs entries (e.g. saved by an earlier
   process), _clear drops this device's. */
int ks_stencil_tuning_get(int* entries4, int cap);
ks_status ks_stencil_tuning_set(const int* entries4, int count);
ks_status ks_stencil_tuning_clear(void);
/* Reducer::gram / block_dots (crates/qm-gpu/src/reduce.rs:340-420): G = S^T [S | T], m and mt fields, gram_mode as
   in ks_options; out row-major m x (m + mt). */
ks_status ks_gram(int n, int m, const double* s, int mt, const double* t, int gram_mode, double* out);
/* lobpcg (crates/qm-gpu/src/eigen.rs:685-1000) on H = -1/2 lap + V: k vectors x (guess and result), evals out. */
ks_status ks_lobpcg(int n, double h, const double* v, int k, double* x, double* evals, double tol, int max_iter,
                    int gram_mode, double* max_residual, int* iterations);
/* EigenStats (crates/qm-gpu/src/eigen.rs:286-305): stop 0 converged, 1 the f32 floor, 2 max_iter; head_kept: the head
   columns came back bitwise (a 0-iteration accept or a locked head); locked: the locked head's columns; head_residual /
   tail_residual: the true max residuals of the columns [0, head) and [head, checked). */
typedef struct {
    int iterations, stop, head_kept, locked, restores, fallbacks, readbacks;
    double max_residual, head_residual, tail_residual, alpha_worst;
} ks_eigen_stats;
/* lobpcg_split (lock 0) and lobpcg_guarded (lock 1) (crates/qm-gpu/src/eigen.rs:613-653): columns [0, head) held to tol,
   [head, checked) to tail_tol >= tol, columns from `checked` on untested buffers; the guess accepted at guess_tol on the
   same scale. With lock, a head under guess_tol at the guess whose tail is not is locked: returned bitwise while the
   other columns iterate in its B-orthogonal complement. residuals (k, may be NULL): every column's exit residual.
   KS_INVALID unless 0 <= head <= checked <= k, checked >= 1, tol <= tail_tol. */
ks_status ks_lobpcg_guarded(int n, double h, const double* v, int k, double* x, double* evals, double tol, double guess_tol,
                            int head, double tail_tol, int checked, int max_iter, int lock, int gram_mode, double* residuals,
                            ks_eigen_stats* stats);
/* multipole moments Q_lm = sum rho R_lm dV (crates/qm-gpu/src/poisson.rs:237-244) */
ks_status ks_multipole_moments(int n, double h, const double* rho, double* q49);

/* ---- host-only parity hooks: the solver's f64 host algebra (no device is touched) ---- */
/* rayleigh_ritz (crates/qm-gpu/src/eigen.rs:515-542; its test rayleigh_ritz_pairs_survive_a_bad_symmetric_eigen,
   :1188-1201): the lowest nk pairs of A c = theta B c for symmetric m x m A and B (row-major, B with a positive
   diagonal); theta ascending, c column-major m x nk (B-orthonormal coefficient vectors), alpha (may be NULL) the
   coefficient amplification max_i |T y_i|. KS_NUMERICAL on a non-positive diagonal of B or on rank loss (fewer than
   nk directions above the drop tolerance). */
ks_status ks_rayleigh_ritz(int m, const double* a, const double* b, int nk, double* theta, double* c, double* alpha);
/* fermi_dirac (crates/qm/src/occupations.rs): occupations f (in evals' order) of k levels holding n electrons at kt
   (Ha), the chemical potential mu (NaN for n = 0) and the entropy S. KS_INVALID on the reference's refusals (fewer
   than n + 1 levels, a non-finite level or kT). */
ks_status ks_fermi_dirac(const double* evals, int k, int n, double kt, double* f, double* mu, double* entropy);
/* The gap witness of a Fermi-Dirac block, read on its k levels (any order) for n electrons at mu and kt:
   reached = witness_reached (crates/qm/src/occupations.rs:283-292: the top level 0.1 Ha above the n-th lowest and
   36 kT above mu; always for n = 0), keep = witness_keep on the levels themselves (occupations.rs:372-394: t + 1 for
   the lowest rank t >= n that passes both arms, t + 2 when rank t + 1 passes too, k when none does or n = 0). */
ks_status ks_fd_witness(const double* evals, int k, int n, double mu, double kt, int* reached, int* keep);
/* The same witness read on the lower bounds theta_j - r_j, r the levels' residual norms |H x - theta x| (the
   Krylov-Weinstein bound, as the solver reads it): reached = witness_bound_reached (crates/qm/src/occupations.rs:299-317),
   keep = witness_keep (:372-394). residuals may be NULL (all zero: ks_fd_witness); a NaN residual never passes. */
ks_status ks_fd_witness_bound(const double* evals, const double* residuals, int k, int n, double mu, double kt, int* reached,
                              int* keep);
/* The witness tail of a loosened SCF step (crates/qm/src/occupations.rs:319-326 step_tail_kt), in kT:
   ln(n_w / (1e-3 delta_rho_prev)) clamped to [6, 36], n_w the block's levels; 36 for a non-finite or non-positive
   delta_rho_prev. The solver reads the witness with this tail on a step whose eigen tolerance is loosened. */
ks_status ks_fd_step_tail_kt(int n_w, double delta_rho_prev, double* tail_kt);
/* tight_columns (crates/qm/src/occupations.rs:334-350): the positions the step's tolerance must hold among k levels (any
   order) with residuals r, the ranks from the top whose running sum of f((eps - r - mu) / kT) stays below 1e-2 tol being
   loose; a NaN mu (an empty channel) gives 0, a NaN residual is never loose. tight_start (:355-366): the same tail rule
   on a warm state's ascending occupations f, at least n (f NULL: n). */
ks_status ks_fd_tight_columns(const double* evals, const double* residuals, int k, double mu, double kt, double tol, int* tight);
ks_status ks_fd_tight_start(const double* f, int k, int n, double tol, int* tight);
/* The lowest converged witness (crates/qm/src/occupations.rs:396-419 witness_keep_within): the lowest level above the
   n-th whose lower bound theta - r passes both arms (the tail arm at tail_kt kT) with r <= r_max decides, and keep gets
   the levels to keep (its rank + 1, + 2 with a passing spare above it); keep = -1 when no level qualifies (the block must
   grow), k for n = 0. The solver applies it on a tight step whose top level passes only at r > 1.5e-3 Ha. */
ks_status ks_fd_witness_keep_within(const double* evals, const double* residuals, int k, int n, double mu, double kt, double tail_kt,
                                    double r_max, int* keep);

/* ---- device-pointer entry points for callers that keep fields on the GPU (bench, integrations) ----
   Fields are in the pitched layout: element (i, j, k) at (k*n + j)*P + i, P = ks_field_pitch(n),
   F = n*n*P floats per field, blocks of fields contiguous with stride F; pad columns hold 0. */
int ks_field_pitch(int n);
/* The cudaStream_t every kernel of this solver runs on (for callers that time or order work on it). */
void* ks_solver_stream(void* solver);
/* How many of this library's kernels the process has launched so far (instrumentation). */
long long ks_launch_count(void);
/* out_v = -1/2 lap psi_v + V psi_v, v = 0..count-1, enqueued on `stream` (a cudaStream_t, NULL = legacy).
   Like every device-pointer entry point it returns before its kernel runs, so its status covers the arguments and
   the launch only; a bounded wait of the kernel that gave up is reported by ks_device_status. */
ks_status ks_hpsi_device(void* stream, int n, double h, int count, const float* psi, const float* v, float* out);
/* Wait-timeout status of the device-pointer entry points (ks_hpsi_device, ks_gram_device_noalloc). Their kernels
   wait on TMA and bulk copies with bounded spins; a wait that gives up raises the current device's shared timeout
   flag and leaves that launch's output undefined. This call synchronises `stream` (a cudaStream_t, NULL = legacy),
   reads the flag, clears it, and returns KS_DEVICE (message in ks_last_error(NULL)) when it was raised, else KS_OK.
   Solvers keep their own flags and report a timeout from the call that hit it. No counterpart in the reference,
   whose wgpu path has no device-side waits. */
ks_status ks_device_status(void* stream);

/* G = S^T [S | T] with the CUDA-core Gram (the gram_mode 0 form of ks_gram, bit-for-bit the same result) for
   callers that must not allocate device memory: a host framework whose caching allocator owns the GPU's memory
   (a stray cudaMalloc can fail for lack of memory or fragment its pool), and latency-critical stream pipelines
   (cudaFree synchronises the whole device). No counterpart in the reference: its Gram always runs inside a
   solver that owns its buffers.
   s: m fields, t: mt fields (NULL when mt = 0), pitched layout on the current device; out: m x (m + mt) doubles on
   the device, row-major. Enqueued on `stream` (a cudaStream_t, NULL = legacy); nothing is read back.
   Allocates nothing: the per-CTA partial sums live in a 4 MiB static device array (2^19 doubles) that every
   launch overwrites in full, so nothing needs to start at zero. Limit: 2 * SMs * m * (m + mt) <= 2^19, i.e.
   m * (m + mt) <= 1771 on a 148-SM B200; larger blocks return KS_INVALID with a message and launch nothing.
   The first call on each device looks the array up (cudaGetSymbolAddress, with that device current); make that
   first call before any stream capture begins. Calls on one device share the array: calls that overlap in time
   (other streams, other host threads) race, so order them on one stream. */
ks_status ks_gram_device_noalloc(void* stream, int n, int m, const float* s, int mt, const float* t, double* out);

#ifdef __cplusplus
}
#endif
#endif
