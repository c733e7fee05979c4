// ionic.cuh -- device data and launchers of the pseudopotential terms (k_ionic.cu), and the host-side
// owner of one solver's ionic setup (ionic.cu): the species tables on the device, the centres and the
// projector spheres of the current geometry, and the nonlocal operator's scratch.
#pragma once
#include <vector>
#include "kernels.cuh"
#include "../../include/ks_cuda.h"

namespace ks {

constexpr int MAX_CENTRES = 32;      // nuclei per solve (as the all-electron path)
constexpr int MAX_CHUNKS = 64;       // projection chunks per sphere
constexpr int MAX_SPECIES = 8;
constexpr int MAX_PROJECTORS = 4;    // per species, l <= 2

// One nucleus as the electrons see it: charge q and width sigma of its long-range erf part (Z and
// sigma_AE for an all-electron species, Z_v and sigma_LR for a pseudised one), species index or -1.
struct IonicCentre {
    double x, y, z, q, sigma;
    int species, pad;
};

// A pseudised species' uniform tables on the device (spacing du, index 0 at d = 0).
struct IonicSpeciesDev {
    double du, r_sr, pc_radius;
    const double* v_sr;
    const double* rho_pc;
    int n_v_sr, n_pc;
};

// One projector ball of one ion, as a box of grid points clipped to the grid; beta_lm of its 2l + 1
// rows live at beta0 + row * (ni nj nk) in the beta buffer; its projection runs in `chunks` chunks.
struct Sphere {
    double cx, cy, cz, radius, e_kb, du;
    const double* t;
    int n_t, l, rows, row0;
    int i0, j0, k0, ni, nj, nk;
    long long beta0;
    int chunks, chunk0;
};

void launch_ionic_local(const Layout& L, const IonicCentre* c, int nc, const IonicSpeciesDev* sp, float* out, cudaStream_t s);
void launch_partial_core(const Layout& L, const IonicCentre* c, int nc, const IonicSpeciesDev* sp, float* out, cudaStream_t s);
void launch_beta(const Layout& L, const Sphere* sph, int ns, int max_pts, float* beta, cudaStream_t s);
// coef[v * rows_total + row] = h^3 sum beta_row x_v (partials: count * rows_total * MAX_CHUNKS doubles)
void launch_nl_project(const Layout& L, const Sphere* sph, int ns, const int* chunk_sphere, int total_chunks, const float* beta,
                       const float* x, int count, int rows_total, double* partials, double* coef, cudaStream_t s);
// out_v += sum_row E_KB coef[v, row] beta_row over the union box ubox = {i0, j0, k0, ni, nj, nk}
void launch_nl_scatter(const Layout& L, const Sphere* sph, int ns, const float* beta, const double* coef, int rows_total, const int ubox[6],
                       int count, float* out, cudaStream_t s);
void launch_local_forces(const Layout& L, const IonicCentre* c, int nc, const IonicSpeciesDev* sp, const float* rho, const float* xu,
                         const float* xd, double* partials, int blocks, cudaStream_t s);
// partials: count * rows_total * MAX_CHUNKS * 4 doubles
void launch_nl_forces(const Layout& L, const Sphere* sph, const int* chunk_sphere, int total_chunks, const float* psi, int count,
                      int rows_total, double* partials, cudaStream_t s);

}  // namespace ks
