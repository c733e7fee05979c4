/*
 * ks_oracle.h -- C interface of the CPU f64 oracle.
 *
 * TEST INFRASTRUCTURE ONLY. The oracle is a single-threaded (optionally OpenMP)
 * f64 restatement of the reference's CPU Kohn-Sham solver, crate `qm`
 * (crates/qm/src/{grid,stencil,xc,nuclear,poisson,eigen,scf,forces}.rs). The CUDA
 * solver is tested against it: only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may load it. The product never calls it.
 *
 * Grid layout of every array here: the reference's `qm::Grid`, idx = i + n*(j + n*k),
 * cubic n^3, origin = -(n-1)h/2 on every axis (crates/qm/src/grid.rs:1-16).
 */
#ifndef KS_ORACLE_H
#define KS_ORACLE_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

typedef struct { double pos[3]; int z; } ora_nucleus;

/* One pseudised species: the uniform tables (spacing du, index 0 at d = 0) the reference's grid samples of a
   qm::radial::filter::FilteredTable (crates/qm/src/radial/filter.rs:323-363); the same layout as ks_species. */
typedef struct {
    int z;
    double z_v, sigma_lr, du;
    const double* v_sr; int n_v_sr; double r_sr;
    const double* rho_pc; int n_rho_pc; double pc_radius;
    int n_proj;
    const int* proj_l; const double* proj_e_kb; const double* proj_radius;
    const double* const* proj_t; const int* proj_n;
} ora_species;

/* Settings of one SCF (crates/qm/src/scf.rs:375 ScfSettings). occupations: 0 Aufbau, 1 Fermi-Dirac at kt
   (crates/qm/src/occupations.rs) over a block of n_sigma + n_extra levels per occupied channel. */
typedef struct {
    double sigma, tol, mixing, eig_tol;
    int max_iter, diis_history, stall_window;
    int occupations, n_extra;
    double kt;
} ora_settings;

typedef struct {
    int iterations;
    double delta_rho;
    double kinetic, external_, hartree, xc, nuclear, total;
    double boundary_density, max_eigen_residual, poisson_residual;
    int poisson_iterations;
    double electrons[2];
    int status;          /* 0 ok, 1 not converged, 2 stalled, 3 coincident nuclei, 5 no Fermi-Dirac gap witness */
    int eigen_iterations_total, poisson_iterations_total;  /* work counters over the whole solve */
    double ts, entropy, mu[2];  /* Fermi-Dirac: kT*S (total = internal - ts), S, mu per spin (NaN when empty) */
} ora_stats;

/* Fermi-Dirac occupations of one channel (crates/qm/src/occupations.rs fermi_dirac): f in evals' order, mu the
   plateau midpoint of two tie-directed bisections, S Neumaier. Returns 0, or -1 on refused inputs. */
int ora_fermi_dirac(const double* evals, int k, int n, double kt, double* f, double* mu, double* entropy);

/* qm::Grid::trilinear (crates/qm/src/grid.rs:54-86) of an n^3 field f at count points (pts3, Bohr): the cell and
   fractions of trilinear_cell, neighbours beyond an upper face read 0, blended a(1 - t) + b t along x, then y,
   then z in f64; 0 outside [origin, origin + (n-1)h]^3 (NaN included). */
void ora_trilinear(int n, double h, const double* f, const double* pts3, int count, double* out);

/* thread count for the parallel loops (stencils, pointwise); sums stay sequential */
void ora_set_threads(int n);

/* ---- grid and pointwise pieces ---- */
double ora_neumaier(const double* v, size_t n);
void ora_laplacian(int n, double h, const double* f, double* out);
void ora_hamiltonian(int n, double h, const double* f, const double* v, double* out);
void ora_exc_point(double nu, double nd, double* e, double* vu, double* vd);
void ora_lsda(size_t len, const double* nu, const double* nd, double* e, double* vu, double* vd);
void ora_nuclear_potential(int n, double h, const ora_nucleus* nuc, int nn, double sigma, double* out);
void ora_deposit_charge(int n, double h, const ora_nucleus* nuc, int nn, double sigma, double* out);
int  ora_nuclear_repulsion(const ora_nucleus* nuc, int nn, double* e);
void ora_initial_orbitals(int n, double h, const ora_nucleus* nuc, int nn, int k, unsigned long long seed, double* out);
void ora_solid_harmonics(const double r[3], double out[49]);
double ora_jacobi_omega(void);
void ora_jacobi_precond(int n, double h, const double* v, double lambda, const double* r, double* w);

/* ---- sub-solvers ---- */
/* Jacobi-CG Poisson with l<=6 multipole ghosts; v is guess and output. Returns iterations. */
int ora_poisson_solve(int n, double h, const double* rho, double* v, double tol, int max_iter, double* residual);
void ora_multipole_moments(int n, double h, const double* rho, double q[49]);
/* LOBPCG (MGS-orthonormalised [X,W,P], Jacobi preconditioner at lambda when precond != 0). */
int ora_lobpcg(int n, double h, const double* v, int k, double* x, double* evals, int precond, double lambda,
               double tol, int max_iter, double* max_residual);
/* Cyclic Jacobi symmetric eigen-decomposition (column-major evecs), unsorted like the reference's. */
void ora_sym_eigen(int m, const double* a, double* evals, double* evecs);
/* bordered Pulay system on a Gram matrix (m x m row-major). Returns 1 and c on success. */
int ora_diis_coefficients(int m, const double* gram, double* c);

/* ---- SCF, state and forces ---- */
typedef struct ora_state ora_state;
/* Runs the Aufbau SCF. warm may be NULL. Returns a new state (owned by the caller) or NULL on
   coincident nuclei; stats->status carries convergence. */
ora_state* ora_scf(int n, double h, const ora_nucleus* nuc, int nn, int n_up, int n_dn,
                   const ora_settings* s, const ora_state* warm, ora_stats* stats);
void ora_state_free(ora_state* st);
int  ora_state_counts(const ora_state* st, int* n_up, int* n_dn);
void ora_state_evals(const ora_state* st, double* up, double* dn);
void ora_state_occupations(const ora_state* st, double* up, double* dn);
void ora_state_density(const ora_state* st, double* rho_up, double* rho_dn);
void ora_state_potentials(const ora_state* st, double* v_nuc, double* v_h);
void ora_state_orbitals(const ora_state* st, int spin, double* out);
int  ora_forces(const ora_state* st, const ora_nucleus* nuc, int nn, double sigma, double* out3n);

/* ---- pseudised ions (crates/qm/src/scf.rs:114-140, ionic.rs, nonlocal.rs, forces.rs) ---- */
/* ora_scf under an ionic setup: nuclei whose Z is listed are pseudised, the others all-electron at s->sigma.
   n_species = 0 is ora_scf. A warm state is reused only between all-electron solves. */
ora_state* ora_scf_ionic(int n, double h, const ora_nucleus* nuc, int nn, int n_up, int n_dn, const ora_settings* s,
                         const ora_species* species, int n_species, const ora_state* warm, ora_stats* stats);
/* V_loc (nuclear.rs:338-346) and rho_pc (:350-359) of the geometry */
void ora_ionic_local_potential(int n, double h, const ora_nucleus* nuc, int nn, double sigma_ae, const ora_species* species,
                               int n_species, double* out);
void ora_partial_core(int n, double h, const ora_nucleus* nuc, int nn, const ora_species* species, int n_species, double* out);
/* out_v = V_NL x_v for count vectors (n^3 each), and c[v * rows + row] = h^3 <beta_row, x_v> when c is not NULL;
   returns the number of projector rows */
int ora_nonlocal_apply(int n, double h, const ora_nucleus* nuc, int nn, const ora_species* species, int n_species, const double* x,
                       int count, double* out, double* c);
/* The R-dependent energy at the state's frozen orbitals and densities: integral rho V_loc + E_NL +
   E_xc[rho_up + rho_pc/2, rho_dn + rho_pc/2] + E_ii (valence charges). Its R-derivative is minus ora_forces_ionic. */
double ora_frozen_energy(const ora_state* st, const ora_nucleus* nuc, int nn, double sigma, const ora_species* species,
                         int n_species);
/* filter.rs:302-317 uniform_lagrange behind the radius test of FilteredTable::read: value and derivative */
void ora_table_read(const double* f, int len, double du, double radius, double d, double* v, double* dv);
/* nonlocal.rs:87-98 grad R_lm for l <= 2, out[3 * lm + axis], lm = l^2 + l + m */
void ora_solid_harmonic_gradients(const double r[3], double out[27]);
/* forces of a state solved by ora_scf_ionic with the same setup: local long/short range, partial core, nonlocal,
   ion-ion (crates/qm/src/forces.rs, pseudised ions). Returns 0, or -1 on coincident nuclei. */
int ora_forces_ionic(const ora_state* st, const ora_nucleus* nuc, int nn, double sigma, const ora_species* species, int n_species,
                     double* out3n);

#ifdef __cplusplus
}
#endif
#endif
