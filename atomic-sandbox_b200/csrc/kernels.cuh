// kernels.cuh -- host-side launchers of the B200 kernels (sm_100a). Every launcher takes the
// stream it enqueues on and returns immediately; none synchronises.
#pragma once
#include <array>
#include <vector>
#include <cuda.h>
#include "common.cuh"

namespace ks {

// A nucleus on the device: position (Bohr) and charge Z in w.
struct Nuc { double x, y, z, Z; };

// ---------------------------------------------------------------- generators (k_pointwise.cu)
// V_nuc = -sum Z erf(d/(sigma sqrt2))/d, d -> 0 limit -Z sqrt(2/pi)/sigma (crates/qm/src/nuclear.rs:258-272);
// f64 arithmetic, stored f32, pads 0.
void launch_nuclear_potential(const Layout& L, const Nuc* nuc, int nn, double sigma, float* out, cudaStream_t s);
// rho = scale * sum Z (2 pi sigma^2)^-3/2 exp(-d^2/(2 sigma^2)) (nuclear.rs:98-107).
void launch_deposit_charge(const Layout& L, const Nuc* nuc, int nn, double sigma, double scale, float* out, cudaStream_t s);
// k orbitals from one LCG stream (crates/qm/src/scf.rs:636-644): mode 0 = (u + 0.5) * sum exp(-d^2/4),
// mode 1 = 2u - 1 (uniform(-1, 1)). Stream position of (vector v, point p) = v*n^3 + p + 1.
void launch_initial_orbitals(const Layout& L, const Nuc* nuc, int nn, int k, unsigned long long seed, int mode, float* out,
                             cudaStream_t s);
// dense f64 n^3 (reference layout) <-> pitched f32 field
void launch_pack(const Layout& L, int count, const double* dense, float* field, cudaStream_t s);
void launch_unpack(const Layout& L, int count, const float* field, double* dense, cudaStream_t s);
void launch_fill(float* out, float value, long long count, cudaStream_t s);

// ---------------------------------------------------------------- pointwise (k_pointwise.cu)
struct Terms {
    static constexpr int MAX = 8;
    int count = 0;
    const float* x[MAX];
    float c[MAX];
};
// y = sum_t c_t x_t over `count` fields of F floats each (blocks with stride F)
void launch_lincomb(long long F, int count, float* y, const Terms& t, cudaStream_t s);
// out_j' = sum_i C[i + m*j] * S_i for j < q, j' = j (j < split) or j + gap (j >= split);
// S: m fields (stride F), C: device f64 m x q column-major.
void launch_block_lincomb(long long F, int m, const float* S, int q, const double* C, float* out, int split, int gap, cudaStream_t s);
// LOBPCG residual, first Jacobi sweep and |r|^2 partials in one pass (crates/qm-gpu/src/eigen.rs:743-759):
//   R_i = HX_i - th_hi_i X_i - th_lo_i X_i,  W0_i = R_i / max(diag_t + V - lambda_i, 0.1)
// theta/lambda device f64 [k]; partials: [blocks][k] f64 of sum R_i^2 (dv not applied).
// With dinv set, each vector's sweep factor omega / max(diag_t + V - lambda, 0.1) is written there too (dinv may be HX
// itself: each element is read before it is overwritten).
void launch_residual_precond(const Layout& L, int k, const float* HX, const float* X, const double* theta, const float* V,
                             const double* lambda, double diag_t, float* R, float* W0, double* partials, int blocks, cudaStream_t s,
                             float omega = 0.f, float* dinv = nullptr);
// XC (LSDA: Slater exchange + PW92, crates/qm/src/xc.rs:88-207) on (up, dn), f64 arithmetic, and the
// effective potentials v_sigma = vnuc + vh + vxc_sigma. exc gets n*eps_xc. With a partial core pc, XC runs on
// (up + pc/2, dn + pc/2).
void launch_xc_veff(long long F, const float* up, const float* dn, const float* vnuc, const float* vh, float* exc, float* vup,
                    float* vdn, float* vxc_up, float* vxc_dn, cudaStream_t s, const float* pc = nullptr);
// rho_out = sum_i f_i psi_i^2 over k orbitals (f: device f64 or null = 1), r = rho_out - rho_in, and
// partials [blocks][2] = (sum |rho_out - rho_in|, sum rho_out).
void launch_density_residual(long long F, int k, const float* psi, const double* f, const float* rho_in, float* rho_out, float* r,
                             double* partials, int blocks, cudaStream_t s);
// Pulay mix about the latest input (crates/qm-gpu/src/scf.rs:628-645):
//   out = base + sum_{i<m-1} c_i (rho_i - base) + sum_i a_i r_i, clamped at 0.
void launch_diis_mix(long long F, int m, const float* const* rho, const float* const* r, const float* c, const float* a,
                     float* out, cudaStream_t s);
void launch_scale(long long F, float* x, float a, cudaStream_t s);
// out = max(2 cur - prev, 0): the linear extrapolation in time of a density
void launch_extrapolate(long long F, const float* cur, const float* prev, float* out, cudaStream_t s);
// x *= target / *sum_dev when both are positive (the SCF's charge renormalisation, no host round trip)
void launch_scale_ratio(long long F, float* x, const double* sum_dev, double target, cudaStream_t s);

// ---------------------------------------------------------------- stencil (k_stencil.cu)
// ST_HAM_RESIDUAL: H x followed, in the same pass, by the LOBPCG residual r = Hx - theta x, the first Jacobi sweep
// w0 = r / max(diag_t + V - lambda, 0.1) and the |r|^2 partials -- what launch_residual_precond computes from a stored
// Hx, bit for bit (out = R, out2 = W0; dot_partials = [CTAs per vector][count] f64 sums of r^2, dv not applied).
enum StencilMode { ST_LAPLACIAN = 0, ST_HAMILTONIAN = 1, ST_JACOBI = 2, ST_HAM_RESIDUAL = 3 };
struct StencilArgs {
    int mode = ST_LAPLACIAN;
    float scale = 0;        // multiplies sum_m c_m (second differences): 1/h^2 or -1/(2 h^2)
    const float* V = nullptr;   // potential (HAMILTONIAN, JACOBI)
    const float* R = nullptr;   // JACOBI right-hand sides (block, stride F)
    const double* lambda = nullptr; // JACOBI shift per vector (device)
    float omega = 0, diag_t = 0;
    double* dot_partials = nullptr; // optional: sum_points x*out per CTA (Poisson's p.Ap), [CTAs] f64
    int vec0 = 0;               // first vector of the tensor map's block to read (outputs, R, lambda are indexed from 0)
    const double* theta = nullptr;  // HAM_RESIDUAL: Ritz value per vector (device f64)
    float* out2 = nullptr;          // HAM_RESIDUAL: the first sweep W0 (block, stride F)
    // the sweep's per-point factor omega / max(diag_t + V - lambda, 0.1) of each vector (block, stride F): written by
    // HAM_RESIDUAL when set, read by JACOBI when set (else JACOBI computes it, to the same bits)
    float* dinv = nullptr;
    // z-chunks per tile column; 0: the tuned choice for this shape (ST_HAMILTONIAN without dots, ST_JACOBI) when the
    // autotuner recorded one on this device, else the cost model's
    int chunks = 0;
};
// The launch-shape autotuner's table (per device, process-wide): the z-chunk count for H psi (ST_HAMILTONIAN without
// dots) and the Jacobi sweep (ST_JACOBI) of `count` vectors on an n^3 grid. Those two modes are the ones whose outputs
// do not depend on the chunking (no per-CTA partial sums), so a tuned launch gives the same bits.
void stencil_set_tuned_chunks(int n, int count, int mode, int chunks);
int stencil_tuned_chunks(int n, int count, int mode);  // 0: none
int stencil_max_chunks(const Layout& L);                // the candidates are 1 .. this
int stencil_model_chunks(const Layout& L, int count);   // the cost model's choice
// the current device's entries as (n, count, mode, chunks) quadruples
std::vector<std::array<int, 4>> stencil_tuning_entries();
void stencil_tuning_clear();
// CTAs per vector of a stencil launch of `count` vectors (the leading dimension of ST_HAM_RESIDUAL's partials)
int stencil_ctas_per_vector(const Layout& L, int count);
// out_v = op(x_v) for the `count` vectors of the block x (stride F). `tmap` must describe x
// (make_field_tmap). Returns the number of CTAs launched (for dot partials).
int launch_stencil(const Layout& L, const CUtensorMap& tmap, int count, const StencilArgs& a, float* out, cudaStream_t s);
// A 4-D tensor map (n, n, n, count) over a block of pitched fields with the stencil's halo box.
void make_field_tmap(CUtensorMap* map, const Layout& L, const float* base, int count);
int stencil_ctas(const Layout& L, int count);

// ---------------------------------------------------------------- reductions (k_reduce.cu)
// Deterministic two-stage reductions: a kernel writes one f64 partial per CTA and value, then
// launch_finish sums the CTA partials in a fixed order (Neumaier) into out[nvals].
void launch_finish(const double* partials, int blocks, int nvals, double scale, double* out, cudaStream_t s);
// the same for a rows x cols matrix of values, written transposed (out[c*rows + r])
void launch_finish_transposed(const double* partials, int blocks, int rows, int cols, double scale, double* out, cudaStream_t s);
// Two finishes in one launch, each value summed exactly as launch_finish / launch_finish_transposed would (bitwise):
// trows > 0 writes value r*tcols + c to out[c*trows + r].
struct FinishDesc {
    const double* partials = nullptr;
    int blocks = 0, nvals = 0;
    double scale = 1.0;
    double* out = nullptr;
    int trows = 0, tcols = 0;
};
void launch_finish_pair(const FinishDesc& a, const FinishDesc& b, cudaStream_t s);
// G = S^T [S | T] on the tensor cores (k_gram_tc.cu): partials [gram_tc_blocks(m, mt)][(m + mt) x m] of the
// transpose D = [S | T]^T S; m <= 64, round8(m) + mt <= 128.
int gram_tc_blocks(int m, int mt);
void launch_gram_tc(long long F, int m, const float* S, int mt, const float* T, double* partials, cudaStream_t s);
int reduce_blocks(long long F);
// out-of-place dot products: partials [blocks][npairs] of sum a_p*b_p over F floats.
struct Pairs {
    static constexpr int MAX = 16;
    int count = 0;
    const float* a[MAX];
    const float* b[MAX];
};
void launch_dots(long long F, const Pairs& p, double* partials, int blocks, cudaStream_t s);
// G = S^T [S | T] on CUDA cores: S m fields, T mt fields (both blocks stride F); partials [gram_blocks(m, mt)][m*(m+mt)]
// row-major (row i = S_i, column j < m = S_j, j >= m = T_{j-m}). Returns the number of partial blocks written.
int gram_blocks(int m, int mt);
int launch_gram(long long F, int m, const float* S, int mt, const float* T, double* partials, cudaStream_t s);
// multipole moments Q_lm = sum rho R_lm(r) (l <= 6, Racah real solid harmonics, crates/qm/src/poisson.rs:89-120)
void launch_moments(const Layout& L, const float* rho, double* partials, int blocks, cudaStream_t s);
// max |f| over the six outer planes of the box -> partials [blocks] (max, finished by launch_finish_max)
void launch_face_max(const Layout& L, const float* f, double* partials, int blocks, cudaStream_t s);
void launch_finish_max(const double* partials, int blocks, double* out, cudaStream_t s);
// Hellmann-Feynman electronic force partials: [blocks][3*nn] of sum rho * (-Z g'(d)/d) * (r - R)
// (crates/qm/src/forces.rs:205-218)
// dE/dR_I and dE/dsigma of the converged state (adjoint of the stationary KS energy; rho recomputed
// from the orbitals, weighted by wu / wd when given): partials [blocks][3 nn + 1] (dE/dR of nucleus a at
// 3a..3a+2, dE/dsigma last).
void launch_vjp(const Layout& L, const float* up, int nup, const double* wu, const float* dn, int ndn, const double* wd, const Nuc* nuc,
                int nn, double sigma, double* partials, int blocks, cudaStream_t s);
// ---------------------------------------------------------------- readouts (k_readout.cu)
// out[q] = trilinear blend of f at pts[3q..3q+3) (Bohr), 0 outside [origin, origin + (n-1)h]^3
// (crates/qm-gpu/src/sample.rs:84-121, crates/qm/src/grid.rs:54-86).
void launch_sample(const Layout& L, const float* f, const double* pts, int count, float* out, cudaStream_t s);
// dense n^3 f32 (x fastest) = f (+ g) without the pads, and per-block maxima in partials[blocks].
void launch_volume(const Layout& L, const float* f, const float* g, float* dense, double* partials, int blocks, cudaStream_t s);
// partials[blocks] of sum |a - b| over F floats (f64)
void launch_abs_diff(long long F, const float* a, const float* b, double* partials, int blocks, cudaStream_t s);
void launch_forces(const Layout& L, const float* rho, const Nuc* nuc, int nn, double sigma, double* partials, int blocks,
                   cudaStream_t s);

// ---------------------------------------------------------------- Poisson (k_poisson.cu)
// b = 4 pi rho + L_bc with the ghost values V_bc(r) = sum_lm Q_lm R_lm(r)/|r|^(2l+1) of the
// multipole moments q[49] (device f64) (crates/qm/src/poisson.rs:161-203).
// ghost: scratch of 24 n^2 doubles (the V_bc table of the 4-deep shell beyond the six faces).
void launch_poisson_rhs(const Layout& L, const float* rho, const double* q, double* ghost, float* b, cudaStream_t s);
// multigrid level descriptor: Dirichlet boundary d_low/d_high spacings beyond the first/last point
struct MgLevel { int n, P; long long F; double h; float g_low, g_high; };
void launch_mg_jacobi(const MgLevel& lv, const float* x, const float* b, float* out, float omega, cudaStream_t s);
void launch_mg_residual(const MgLevel& lv, const float* x, const float* b, float* out, cudaStream_t s);
void launch_mg_restrict(const MgLevel& coarse, const MgLevel& fine, const float* rf, float* bc, cudaStream_t s);
void launch_mg_prolong_add(const MgLevel& coarse, const MgLevel& fine, const float* xc, float* xf, cudaStream_t s);
// all levels from `first` to the coarsest in one single-CTA launch (levels small enough for one SM)
struct MgCoarse {
    static constexpr int MAXL = 8;
    int nlev = 0;
    MgLevel lv[MAXL];
    float* x[MAXL];
    float* b[MAXL];
    float* res[MAXL];
    float* tmp[MAXL];
};
void launch_mg_coarse(const MgCoarse& c, float omega, int pre, int post, int coarsest_sweeps, cudaStream_t s);
// CG updates with the scalars read on the device (scal: f64 solver scalars; scal[0] = p.Ap,
// scal[rz_slot] = r.z): v += alpha p, r += alpha (L p) with alpha = r.z / p.Ap (A = -L); and
// p = z + beta p with beta = scal[rz_new] / scal[rz_old]. A non-positive p.Ap or r.z gives alpha = 0.
void launch_cg_update(long long F, float* v, float* r, const float* p, const float* ap, const double* scal, int rz_slot, cudaStream_t s);
void launch_cg_direction(long long F, float* p, const float* z, const double* scal, int rz_old, int rz_new, cudaStream_t s);

}  // namespace ks
