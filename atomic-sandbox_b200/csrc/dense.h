// dense.h -- small dense f64 linear algebra on the host: the Rayleigh-Ritz and DIIS solves of the
// SCF (matrices of a few dozen rows). Row-major storage unless stated.
#pragma once
#include <algorithm>
#include <vector>

namespace ks {
namespace dense {

using Mat = std::vector<double>;  // row-major n x n

// Symmetric eigen-decomposition, checked like the reference's `qm::eigen::sym_eigen`
// (crates/qm/src/eigen.rs:150-173): Householder tridiagonalisation + implicit QL, then every
// pair's residual |A v - lambda v| against 1e-11 (1 + max|lambda|); a failing decomposition is
// refined by cyclic Jacobi (crates/qm/src/eigen.rs:175-211). evals unsorted; evecs column-major
// (evecs[i + n*k] = component i of eigenvector k).
void sym_eigen(int n, const Mat& a, std::vector<double>& evals, std::vector<double>& evecs);
// The cyclic Jacobi method alone (the reference's fallback).
void jacobi_eigen(int n, Mat a, std::vector<double>& evals, std::vector<double>& evecs);
// Householder + implicit QL alone (no check).
void tridiag_ql_eigen(int n, const Mat& a, std::vector<double>& evals, std::vector<double>& evecs);

// Cholesky A = L L^T of an SPD matrix (lower factor in place). False if a pivot is not positive.
bool cholesky(int n, Mat& a);
// Solves L L^T X = B for q right-hand sides (B row-major n x q, overwritten by X).
void cholesky_solve(int n, const Mat& l, int q, std::vector<double>& b);
// Gaussian elimination with partial pivoting; false on a zero pivot (nalgebra's `lu().solve`).
bool lu_solve(int n, Mat a, std::vector<double>& b);

// Bordered Pulay system on a residual Gram matrix (m x m row-major), scaled by its largest
// diagonal with a 1e-12 relative diagonal shift (crates/qm/src/scf.rs:681-697). False when the
// solve fails or gives non-finite coefficients.
bool diis_coefficients(int m, const Mat& gram, std::vector<double>& c);

// Fermi-Dirac occupations of one channel with n electrons over k levels at temperature kt (Ha)
// (crates/qm/src/occupations.rs fermi_dirac): f in evals' order, mu the midpoint of the plateau
// found by two tie-directed bisections over [min - 50 kT, max + 50 kT], S = sum s(x) compensated.
// n = 0 gives every f = 0 and mu = NaN. Returns false on refused inputs (k < n + 1, a non-finite
// level or kT).
bool fermi_dirac(const double* evals, int k, int n, double kt, double* f, double& mu, double& entropy);
// The gap witness on the lower bounds theta_j - r_j of k levels (any order) with residual norms r (NULL: all zero):
// the highest level's bound at least 0.1 Ha above the n-th lowest level and 36 kT above mu (occupations.rs:299-317
// witness_bound_reached; with r = 0 it is witness_reached, :283-292). A NaN residual never passes.
bool fd_witness(const double* evals, const double* res, int k, int n, double mu, double kt, double tail_kt = 36.0);
// After a passed witness, how many of the lowest levels to keep (occupations.rs:372-394 witness_keep, on the same lower
// bounds): t + 1 for the lowest rank t >= n whose bound passes both arms, t + 2 when the rank above passes too; k when
// none does or n = 0.
int fd_witness_keep(const double* evals, const double* res, int k, int n, double mu, double kt, double tail_kt = 36.0);
// The witness tail of a loosened SCF step (occupations.rs:319-326 step_tail_kt): ln(n_w / (1e-3 delta_rho_prev)) kT
// clamped to [6, 36], n_w the block's levels; 36 for a non-finite or non-positive delta_rho_prev.
double fd_step_tail_kt(int n_w, double delta_rho_prev);
// The lowest converged witness (occupations.rs:396-419 witness_keep_within, the tail arm at tail_kt kT): the lowest rank
// t >= n whose lower bound passes both arms with its residual at most r_max decides, keeping t + 1 levels (t + 2 when
// rank t + 1 passes on its lower bound too); -1 when no such level exists (the block must grow); k for n = 0. A NaN
// residual never qualifies.
int fd_witness_keep_within(const double* evals, const double* res, int k, int n, double mu, double kt, double tail_kt, double r_max);

// The positions the step's tolerance must hold (occupations.rs:334-350 tight_columns): from the top rank down, the
// ranks whose running sum of f((theta - r - mu) / kT) stays below 1e-2 tol are loose; the result is one past the highest
// position of a tight rank (0 without mu, NaN mu).
int fd_tight_columns(const double* evals, const double* res, int k, double mu, double kt, double tol);
// The tight count a solve starts from (occupations.rs:355-366 tight_start): the positions of a warm state's ascending
// occupations f that the same tail rule needs at tol, at least n; n without f.
int fd_tight_start(const double* f, int k, int n, double tol);
// The extra block after a failed witness (occupations.rs:423 grown_extras): 2 extras, at least one more, at most cap.
inline int fd_grown_extras(int extras, int cap) { return std::min(std::max(2 * extras, extras + 1), cap); }

}  // namespace dense
}  // namespace ks
