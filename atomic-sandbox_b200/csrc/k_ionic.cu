// k_ionic.cu -- the pseudopotential terms of the Kohn-Sham Hamiltonian on sm_100a: the local ionic
// potential V_loc, the model partial core rho_pc, the Kleinman-Bylander nonlocal operator V_NL and
// the ionic force terms.
//
// Reference: crates/qm/src/nuclear.rs:297-359 (smeared_potential with per-centre charge and width,
// ionic_local_potential, partial_core_field), crates/qm/src/nonlocal.rs (the operator on the grid),
// crates/qm/src/radial/filter.rs:296-363 (the uniform tables and their 4-point Lagrange reads),
// crates/qm-gpu/src/ionic.rs (the GPU form: the same quantities, projector rows over the ball of
// each ion, the Jacobi preconditioner left local) and crates/qm/src/forces.rs (the five force terms).
//
// All geometry and table reads are f64; fields are stored f32 (V_loc, rho_pc) and the projector
// values beta_lm are computed once per geometry on the device in f64 and stored f32, as the reference
// uploads them. The projections c = h^3 sum beta psi are summed in f64 per chunk and finished in a
// fixed order (deterministic). V_NL psi is gathered per grid point over the balls that contain it, so
// overlapping balls never race and the result does not depend on scheduling.
#include "ionic.cuh"
#include "harmonics.cuh"
#include "reduce_util.cuh"

namespace ks {

namespace {

constexpr int TPB_I = 256;
constexpr double PI_D = 3.14159265358979323846;

__device__ __forceinline__ void coords(long long e, int n, int P, int& i, int& j, int& k) {
    const long long row = e / P;
    i = (int)(e - row * P);
    j = (int)(row % n);
    k = (int)(row / n);
}

// filter.rs:302-317 uniform_lagrange: (value, d/dd) of the 4-point Lagrange interpolant of an even
// function tabulated at d = k du (index -1 mirrors index 1); zero beyond the table.
__device__ __forceinline__ void lagrange(const double* f, int len, double du, double d, double& v, double& dv) {
    const double s = d / du;
    const long long i0 = (long long)floor(s) - 1;
    if (i0 + 3 >= len) { v = 0.0; dv = 0.0; return; }
    auto at = [&](long long i) { return f[i < 0 ? -i : i]; };
    const double t = s - (double)i0;
    const double a = at(i0), b = at(i0 + 1), c = at(i0 + 2), e = at(i0 + 3);
    const double l0 = -(t - 1.0) * (t - 2.0) * (t - 3.0) / 6.0, l1 = t * (t - 2.0) * (t - 3.0) / 2.0;
    const double l2 = -t * (t - 1.0) * (t - 3.0) / 2.0, l3 = t * (t - 1.0) * (t - 2.0) / 6.0;
    const double d0 = -((t - 2.0) * (t - 3.0) + (t - 1.0) * (t - 3.0) + (t - 1.0) * (t - 2.0)) / 6.0;
    const double d1 = ((t - 2.0) * (t - 3.0) + t * (t - 3.0) + t * (t - 2.0)) / 2.0;
    const double d2 = -((t - 1.0) * (t - 3.0) + t * (t - 3.0) + t * (t - 1.0)) / 2.0;
    const double d3 = ((t - 1.0) * (t - 2.0) + t * (t - 2.0) + t * (t - 1.0)) / 6.0;
    v = a * l0 + b * l1 + c * l2 + e * l3;
    dv = (a * d0 + b * d1 + c * d2 + e * d3) / du;
}

// filter.rs:355 read: zero beyond the radius, else the interpolant
__device__ __forceinline__ void table_read(const double* f, int len, double du, double radius, double d, double& v, double& dv) {
    if (d > radius) { v = 0.0; dv = 0.0; return; }
    lagrange(f, len, du, d, v, dv);
}

// V_loc = sum over centres of -q erf(d / (sigma sqrt2)) / d (-q sqrt(2/pi) / sigma below 1e-10), then
// + V_SR(d) of every pseudised centre within its r_sr, in centre order (nuclear.rs:297-302, :338-346).
__global__ void __launch_bounds__(TPB_I) local_kernel(int n, int P, long long F, double h, double origin,
                                                      const IonicCentre* __restrict__ c, int nc,
                                                      const IonicSpeciesDev* __restrict__ sp, float* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        coords(e, n, P, i, j, k);
        if (i >= n) { out[e] = 0.0f; continue; }
        const double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        double acc = -0.0;
        for (int a = 0; a < nc; ++a) {
            const double dx = x - c[a].x, dy = y - c[a].y, dz = z - c[a].z;
            const double d = sqrt(dx * dx + dy * dy + dz * dz);
            const double on_site = sqrt(2.0 / PI_D) / c[a].sigma;
            acc += (d < 1e-10) ? -c[a].q * on_site : -c[a].q * erf(d / (c[a].sigma * sqrt(2.0))) / d;
        }
        for (int a = 0; a < nc; ++a) {
            if (c[a].species < 0) continue;
            const IonicSpeciesDev& s = sp[c[a].species];
            if (s.n_v_sr == 0) continue;
            const double dx = x - c[a].x, dy = y - c[a].y, dz = z - c[a].z;
            const double d = sqrt(dx * dx + dy * dy + dz * dz);
            if (d > s.r_sr) continue;
            double v, dv;
            lagrange(s.v_sr, s.n_v_sr, s.du, d, v, dv);
            acc += v;
        }
        out[e] = (float)acc;
    }
}

// rho_pc = sum over pseudised centres with a core of rho_pc(d) within pc_radius (nuclear.rs:350-359)
__global__ void __launch_bounds__(TPB_I) partial_core_kernel(int n, int P, long long F, double h, double origin,
                                                             const IonicCentre* __restrict__ c, int nc,
                                                             const IonicSpeciesDev* __restrict__ sp, float* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        coords(e, n, P, i, j, k);
        if (i >= n) { out[e] = 0.0f; continue; }
        const double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        double acc = 0.0;
        for (int a = 0; a < nc; ++a) {
            if (c[a].species < 0) continue;
            const IonicSpeciesDev& s = sp[c[a].species];
            if (!(s.pc_radius > 0.0)) continue;
            const double dx = x - c[a].x, dy = y - c[a].y, dz = z - c[a].z;
            const double d = sqrt(dx * dx + dy * dy + dz * dz);
            if (d > s.pc_radius) continue;
            double v, dv;
            lagrange(s.rho_pc, s.n_pc, s.du, d, v, dv);
            acc += v;
        }
        out[e] = (float)acc;
    }
}

// beta_lm on every point of each sphere's box: t(d) N_l R_lm(d) within the radius, 0 outside the ball
// (nonlocal.rs build_inner); stored [row][box point] as f32.
__global__ void __launch_bounds__(TPB_I) beta_kernel(const Sphere* __restrict__ sph, double h, double origin, float* __restrict__ beta) {
    const Sphere& s = sph[blockIdx.y];
    const int npts = s.ni * s.nj * s.nk;
    const double norm = sqrt((2.0 * s.l + 1.0) / (4.0 * PI_D));
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < npts; q += gridDim.x * blockDim.x) {
        const int ii = q % s.ni, jj = (q / s.ni) % s.nj, kk = q / (s.ni * s.nj);
        const double dx = origin + (s.i0 + ii) * h - s.cx, dy = origin + (s.j0 + jj) * h - s.cy, dz = origin + (s.k0 + kk) * h - s.cz;
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        double t = 0.0, dt = 0.0;
        if (d <= s.radius) lagrange(s.t, s.n_t, s.du, d, t, dt);
        double sh[49];
        solid_harmonics_dev(dx, dy, dz, sh);
        for (int m = -s.l; m <= s.l; ++m) {
            const double b = (d <= s.radius) ? t * norm * sh[s.l * s.l + s.l + m] : 0.0;
            beta[s.beta0 + (long long)(m + s.l) * npts + q] = (float)b;
        }
    }
}

__device__ __forceinline__ long long field_index(const Sphere& s, int q, int n, int P) {
    const int ii = q % s.ni, jj = (q / s.ni) % s.nj, kk = q / (s.ni * s.nj);
    return ((long long)(s.k0 + kk) * n + (s.j0 + jj)) * P + (s.i0 + ii);
}

// partials[(v * rows_total + row) * MAX_CHUNKS + c] = sum over chunk c of the sphere's box of beta_row x_v
__global__ void __launch_bounds__(TPB_I) project_kernel(const Sphere* __restrict__ sph, const int* __restrict__ chunk_sphere,
                                                        const float* __restrict__ beta, int n, int P, long long F,
                                                        const float* __restrict__ x, int rows_total, double* __restrict__ partials) {
    const int gc = blockIdx.x, v = blockIdx.y;
    const Sphere& s = sph[chunk_sphere[gc]];
    const int c = gc - s.chunk0;
    const int npts = s.ni * s.nj * s.nk;
    const int per = (npts + s.chunks - 1) / s.chunks;
    const int q0 = c * per, q1 = min(npts, q0 + per);
    const float* xv = x + (long long)v * F;
    double acc[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        const double xq = (double)xv[field_index(s, q, n, P)];
#pragma unroll
        for (int r = 0; r < 5; ++r)
            if (r < s.rows) acc[r] += (double)beta[s.beta0 + (long long)r * npts + q] * xq;
    }
    for (int r = 0; r < s.rows; ++r) {
        const double t = block_sum(acc[r]);
        if (threadIdx.x == 0) partials[((long long)v * rows_total + s.row0 + r) * MAX_CHUNKS + c] = t;
    }
}

// coef[v * rows_total + row] = h^3 * (Neumaier sum of the row's chunk partials, in chunk order)
__global__ void project_finish_kernel(const Sphere* __restrict__ sph, int ns, const double* __restrict__ partials, int rows_total,
                                      int count, double dv, double* __restrict__ coef) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= rows_total * count) return;
    const int v = t / rows_total, row = t % rows_total;
    int si = 0;
    while (si + 1 < ns && sph[si + 1].row0 <= row) ++si;
    const int chunks = sph[si].chunks;
    double sum = 0.0, comp = 0.0;
    for (int c = 0; c < chunks; ++c) {
        const double x = partials[((long long)v * rows_total + row) * MAX_CHUNKS + c];
        const double tt = sum + x;
        if (fabs(sum) >= fabs(x)) comp += (sum - tt) + x; else comp += (x - tt) + sum;
        sum = tt;
    }
    coef[t] = (sum + comp) * dv;
}

// out_v += sum over the spheres whose box holds the point of E_KB c_{v,row} beta_row, for every point of
// the union box [i0, i0 + ni) x ... ; f64 accumulation, one f32 rounding.
__global__ void __launch_bounds__(TPB_I) scatter_kernel(const Sphere* __restrict__ sph, int ns, const float* __restrict__ beta,
                                                        const double* __restrict__ coef, int rows_total, int n, int P, long long F,
                                                        int ui0, int uj0, int uk0, int uni, int unj, int unk, float* __restrict__ out) {
    const int v = blockIdx.y;
    const long long upts = (long long)uni * unj * unk;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < upts; q += (long long)gridDim.x * blockDim.x) {
        const int i = ui0 + (int)(q % uni), j = uj0 + (int)((q / uni) % unj), k = uk0 + (int)(q / ((long long)uni * unj));
        double acc = 0.0;
        bool any = false;
        for (int si = 0; si < ns; ++si) {
            const Sphere& s = sph[si];
            const int ii = i - s.i0, jj = j - s.j0, kk = k - s.k0;
            if (ii < 0 || jj < 0 || kk < 0 || ii >= s.ni || jj >= s.nj || kk >= s.nk) continue;
            any = true;
            const int npts = s.ni * s.nj * s.nk;
            const int lq = (kk * s.nj + jj) * s.ni + ii;
            for (int r = 0; r < s.rows; ++r)
                acc += s.e_kb * coef[(long long)v * rows_total + s.row0 + r] * (double)beta[s.beta0 + (long long)r * npts + lq];
        }
        if (any) {
            float* o = out + (long long)v * F + ((long long)k * n + j) * P + i;
            *o = (float)((double)*o + acc);
        }
    }
}

// Per-centre force partials [blocks][3 nc] of the local terms (forces.rs, the pseudised-ion terms):
//   long range (every centre, its own q and sigma):  rho V_LR'(d) (r - R)/d
//   short range (pseudised, d <= r_sr):              rho V_SR'(d) (r - R)/d
//   partial core (pseudised with a core):            vbar rho_pc'(d) (r - R)/d,  vbar = (vxc_up + vxc_dn)/2
// summed over the grid (times dv in the finish). Points with d < 1e-8 contribute nothing.
__global__ void __launch_bounds__(TPB_I) local_forces_kernel(int n, int P, long long F, double h, double origin,
                                                             const IonicCentre* __restrict__ c, int nc,
                                                             const IonicSpeciesDev* __restrict__ sp, const float* __restrict__ rho,
                                                             const float* __restrict__ xu, const float* __restrict__ xd,
                                                             double* __restrict__ partials) {
    double acc[3 * MAX_CENTRES];
    for (int q = 0; q < 3 * MAX_CENTRES; ++q) acc[q] = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        coords(e, n, P, i, j, k);
        if (i >= n) continue;
        const double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        const double r = (double)rho[e];
        const double vbar = xu ? 0.5 * ((double)xu[e] + (double)xd[e]) : 0.0;
        for (int a = 0; a < nc; ++a) {
            const double dx = x - c[a].x, dy = y - c[a].y, dz = z - c[a].z;
            const double d = sqrt(dx * dx + dy * dy + dz * dz);
            if (d < 1e-8) continue;
            const double s2 = c[a].sigma * sqrt(2.0);
            const double u = d / s2;
            // V_LR'(d) = -q [(2/sqrt(pi)) u e^{-u^2} - erf(u)] / d^2 (filter.rs:344-348)
            double g = -c[a].q * ((2.0 / sqrt(PI_D)) * u * exp(-u * u) - erf(u)) / (d * d) * r;
            if (c[a].species >= 0) {
                const IonicSpeciesDev& s = sp[c[a].species];
                double v, dv;
                if (s.n_v_sr > 0) {
                    table_read(s.v_sr, s.n_v_sr, s.du, s.r_sr, d, v, dv);
                    g += r * dv;
                }
                if (s.pc_radius > 0.0 && xu) {
                    table_read(s.rho_pc, s.n_pc, s.du, s.pc_radius, d, v, dv);
                    g += vbar * dv;
                }
            }
            const double w = g / d;
            acc[3 * a] += w * dx;
            acc[3 * a + 1] += w * dy;
            acc[3 * a + 2] += w * dz;
        }
    }
    for (int q = 0; q < 3 * nc; ++q) {
        const double t = block_sum(acc[q]);
        if (threadIdx.x == 0) partials[(long long)blockIdx.x * 3 * nc + q] = t;
    }
}

// grad R_lm for l <= 2 in lm order (nonlocal.rs:87-98)
__device__ __forceinline__ void grad_rlm(int l, int m, double x, double y, double z, double g[3]) {
    const double s3 = 1.7320508075688772;
    g[0] = g[1] = g[2] = 0.0;
    if (l == 1) {
        if (m == -1) g[1] = 1.0;
        else if (m == 0) g[2] = 1.0;
        else g[0] = 1.0;
    } else if (l == 2) {
        switch (m) {
            case -2: g[0] = s3 * y; g[1] = s3 * x; break;
            case -1: g[1] = s3 * z; g[2] = s3 * y; break;
            case 0: g[0] = -x; g[1] = -y; g[2] = 2.0 * z; break;
            case 1: g[0] = s3 * z; g[2] = s3 * x; break;
            default: g[0] = s3 * x; g[1] = -s3 * y; break;
        }
    }
}

// Nonlocal force partials: for orbital v and every projector row of every sphere, over the sphere's
// box points (chunked like the projection) the four sums  sum grad(beta_row) psi_v (3) and sum beta_row psi_v,
// with grad beta = t'(d) N R_lm d/|d| + t(d) N grad R_lm (nonlocal.rs build_with_gradients, 0 beyond the
// radius; the first term 0 at d = 0), all in f64 from the tables.
// partials[((v * rows_total + row) * MAX_CHUNKS + c) * 4 + {x, y, z, beta}]
__global__ void __launch_bounds__(TPB_I) nl_force_kernel(const Sphere* __restrict__ sph, const int* __restrict__ chunk_sphere, int n,
                                                         int P, long long F, double h, double origin, const float* __restrict__ psi,
                                                         int rows_total, double* __restrict__ partials) {
    const int gc = blockIdx.x, v = blockIdx.y;
    const Sphere& s = sph[chunk_sphere[gc]];
    const int c = gc - s.chunk0;
    const int npts = s.ni * s.nj * s.nk;
    const int per = (npts + s.chunks - 1) / s.chunks;
    const int q0 = c * per, q1 = min(npts, q0 + per);
    const double norm = sqrt((2.0 * s.l + 1.0) / (4.0 * PI_D));
    const float* pv = psi + (long long)v * F;
    double acc[5][4];
    for (int r = 0; r < 5; ++r)
        for (int a = 0; a < 4; ++a) acc[r][a] = 0.0;
    for (int q = q0 + threadIdx.x; q < q1; q += blockDim.x) {
        const int ii = q % s.ni, jj = (q / s.ni) % s.nj, kk = q / (s.ni * s.nj);
        const double dx = origin + (s.i0 + ii) * h - s.cx, dy = origin + (s.j0 + jj) * h - s.cy, dz = origin + (s.k0 + kk) * h - s.cz;
        const double d = sqrt(dx * dx + dy * dy + dz * dz);
        if (d > s.radius) continue;
        double t, dt;
        lagrange(s.t, s.n_t, s.du, d, t, dt);
        double sh[49];
        solid_harmonics_dev(dx, dy, dz, sh);
        const double p = (double)pv[((long long)(s.k0 + kk) * n + (s.j0 + jj)) * P + (s.i0 + ii)];
        for (int r = 0; r < s.rows; ++r) {
            const int m = r - s.l;
            const double rlm = sh[s.l * s.l + s.l + m];
            double g[3];
            grad_rlm(s.l, m, dx, dy, dz, g);
            const double radial = d > 1e-12 ? dt * norm * rlm / d : 0.0;
            const double tn = t * norm;
            acc[r][0] += (radial * dx + tn * g[0]) * p;
            acc[r][1] += (radial * dy + tn * g[1]) * p;
            acc[r][2] += (radial * dz + tn * g[2]) * p;
            acc[r][3] += tn * rlm * p;
        }
    }
    for (int r = 0; r < s.rows; ++r)
        for (int a = 0; a < 4; ++a) {
            const double t = block_sum(acc[r][a]);
            if (threadIdx.x == 0) partials[(((long long)v * rows_total + s.row0 + r) * MAX_CHUNKS + c) * 4 + a] = t;
        }
}

}  // namespace

void launch_ionic_local(const Layout& L, const IonicCentre* c, int nc, const IonicSpeciesDev* sp, float* out, cudaStream_t s) {
    local_kernel<<<std::min(ceil_div(L.F, TPB_I), 8 * sm_count()), TPB_I, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, c, nc, sp, out);
    KS_LAUNCH_CHECK();
}

void launch_partial_core(const Layout& L, const IonicCentre* c, int nc, const IonicSpeciesDev* sp, float* out, cudaStream_t s) {
    partial_core_kernel<<<std::min(ceil_div(L.F, TPB_I), 8 * sm_count()), TPB_I, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, c, nc, sp, out);
    KS_LAUNCH_CHECK();
}

void launch_beta(const Layout& L, const Sphere* sph, int ns, int max_pts, float* beta, cudaStream_t s) {
    if (ns <= 0) return;
    dim3 grid(std::max(1, std::min(ceil_div(max_pts, TPB_I), 64)), ns);
    beta_kernel<<<grid, TPB_I, 0, s>>>(sph, L.h, L.origin, beta);
    KS_LAUNCH_CHECK();
}

void launch_nl_project(const Layout& L, const Sphere* sph, int ns, const int* chunk_sphere, int total_chunks, const float* beta,
                       const float* x, int count, int rows_total, double* partials, double* coef, cudaStream_t s) {
    if (ns <= 0 || count <= 0) return;
    project_kernel<<<dim3(total_chunks, count), TPB_I, 0, s>>>(sph, chunk_sphere, beta, L.n, L.P, L.F, x, rows_total, partials);
    KS_LAUNCH_CHECK();
    project_finish_kernel<<<ceil_div((long long)rows_total * count, 128), 128, 0, s>>>(sph, ns, partials, rows_total, count,
                                                                                       L.h * L.h * L.h, coef);
    KS_LAUNCH_CHECK();
}

void launch_nl_scatter(const Layout& L, const Sphere* sph, int ns, const float* beta, const double* coef, int rows_total, const int ubox[6],
                       int count, float* out, cudaStream_t s) {
    if (ns <= 0 || count <= 0) return;
    const long long upts = (long long)ubox[3] * ubox[4] * ubox[5];
    dim3 grid(std::max(1, std::min(ceil_div(upts, TPB_I), 4 * sm_count())), count);
    scatter_kernel<<<grid, TPB_I, 0, s>>>(sph, ns, beta, coef, rows_total, L.n, L.P, L.F, ubox[0], ubox[1], ubox[2], ubox[3], ubox[4],
                                          ubox[5], out);
    KS_LAUNCH_CHECK();
}

void launch_local_forces(const Layout& L, const IonicCentre* c, int nc, const IonicSpeciesDev* sp, const float* rho, const float* xu,
                         const float* xd, double* partials, int blocks, cudaStream_t s) {
    if (nc > MAX_CENTRES) throw std::invalid_argument("ionic forces: at most 32 centres");
    local_forces_kernel<<<blocks, TPB_I, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, c, nc, sp, rho, xu, xd, partials);
    KS_LAUNCH_CHECK();
}

void launch_nl_forces(const Layout& L, const Sphere* sph, const int* chunk_sphere, int total_chunks, const float* psi, int count,
                      int rows_total, double* partials, cudaStream_t s) {
    if (total_chunks <= 0 || count <= 0) return;
    nl_force_kernel<<<dim3(total_chunks, count), TPB_I, 0, s>>>(sph, chunk_sphere, L.n, L.P, L.F, L.h, L.origin, psi, rows_total, partials);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
