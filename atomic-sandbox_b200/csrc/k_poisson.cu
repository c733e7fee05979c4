// k_poisson.cu -- Hartree solve pieces on sm_100a: the multipole boundary right-hand side, the
// geometric-multigrid V-cycle kernels and the device-side CG scalar updates.
//
// Equation and boundary split: crates/qm/src/poisson.rs:1-70 (A V = b, A = -L_int,
// b = 4 pi rho + L_bc, ghost values from the l <= 6 solid-harmonic expansion). Multigrid:
// crates/qm-gpu/src/multigrid.rs:1-60 and shaders/multigrid.wgsl -- 2nd-order 7-point operator per
// level, coarse points at odd fine indices, Dirichlet boundary d spacings beyond the end points
// (linear extrapolation of the missing neighbour, x_ghost = (1 - 1/d) x_0), damped Jacobi with
// omega = 6/7, full weighting and trilinear prolongation. No ghost cells are stored: a missing
// neighbour is an explicit bounds test, and the levels at or below 24^3 run as one single-CTA
// kernel (one launch for the whole bottom of the V-cycle instead of ~30 tiny launches).
#include <cmath>
#include "kernels.cuh"
#include "reduce_util.cuh"
#include "harmonics.cuh"

namespace ks {

namespace {

constexpr int TPB = 256;
constexpr double PI = 3.14159265358979323846;

inline int blocks_for(long long work) {
    long long b = (work + TPB - 1) / TPB;
    long long cap = 8LL * sm_count();
    return (int)std::max(1LL, std::min(b, cap));
}

// V_bc(r) = sum_l (sum_m Q_lm R_lm(r)) / |r|^(2l+1)  (crates/qm/src/poisson.rs:185-199)
__device__ double bc_value(const double* q, double x, double y, double z) {
    double d2 = x * x + y * y + z * z;
    double hv[49];
    solid_harmonics_dev(x, y, z, hv);
    double acc = 0.0, inv_pow = 1.0 / sqrt(d2);
    for (int l = 0; l <= 6; ++l) {
        double s = 0.0;
        for (int m = -l; m <= l; ++m) s += q[l * l + l + m] * hv[l * l + l + m];
        acc += s * inv_pow;
        inv_pow /= d2;
    }
    return acc;
}

// ghost table: face = 2*axis + (high side), depth 1..4 beyond the face, (u, v) = the other two
// axes in increasing order
__global__ void ghost_kernel(int n, double h, double origin, const double* __restrict__ q, double* __restrict__ ghost) {
    const long long per = (long long)n * n;
    const long long total = 6LL * 4 * per;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        int face = (int)(t / (4 * per));
        long long rem = t % (4 * per);
        int depth = (int)(rem / per) + 1;
        long long uv = rem % per;
        int u = (int)(uv % n), v = (int)(uv / n);
        int axis = face >> 1;
        bool high = face & 1;
        int c[3];
        int ua = axis == 0 ? 1 : 0, va = axis == 2 ? 1 : 2;
        c[ua] = u;
        c[va] = v;
        c[axis] = high ? n - 1 + depth : -depth;
        ghost[t] = bc_value(q, origin + c[0] * h, origin + c[1] * h, origin + c[2] * h);
    }
}

__global__ void rhs_kernel(int n, int P, long long F, double h, const float* __restrict__ rho, const double* __restrict__ ghost,
                           float* __restrict__ b) {
    const double COEFF[5] = {-205.0 / 72.0, 8.0 / 5.0, -1.0 / 5.0, 8.0 / 315.0, -1.0 / 560.0};
    const double inv_h2 = 1.0 / (h * h);
    const long long per = (long long)n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        int i = (int)(e % P);
        long long row = e / P;
        int j = (int)(row % n), k = (int)(row / n);
        if (i >= n) { b[e] = 0.0f; continue; }
        double val = 4.0 * PI * (double)rho[e];
        int pos[3] = {i, j, k};
        bool near = false;
        for (int a = 0; a < 3; ++a) near = near || pos[a] < 4 || pos[a] >= n - 4;
        if (near) {
            double acc = 0.0;
            for (int axis = 0; axis < 3; ++axis) {
                int ua = axis == 0 ? 1 : 0, va = axis == 2 ? 1 : 2;
                long long uv = pos[ua] + (long long)n * pos[va];
                for (int m = 1; m <= 4; ++m) {
                    // sign -1 then +1 (crates/qm/src/poisson.rs:166-176)
                    if (pos[axis] - m < 0) {
                        int depth = m - pos[axis];
                        acc += COEFF[m] * ghost[((long long)(2 * axis) * 4 + (depth - 1)) * per + uv];
                    }
                    if (pos[axis] + m >= n) {
                        int depth = pos[axis] + m - (n - 1);
                        acc += COEFF[m] * ghost[((long long)(2 * axis + 1) * 4 + (depth - 1)) * per + uv];
                    }
                }
            }
            val += acc * inv_h2;
        }
        b[e] = (float)val;
    }
}

// ---- multigrid (7-point A_2 per level with boundary-distance ghost factors)
__device__ __forceinline__ void mg_stencil(const MgLevel& L, const float* __restrict__ x, int i, int j, int k, float& nb, float& diag) {
    const int n = L.n, P = L.P;
    const long long q = ((long long)k * n + j) * P + i;
    const long long sy = P, sz = (long long)n * P;
    float s = 0.f;
    float xm = i > 0 ? x[q - 1] : 0.f, xp = i < n - 1 ? x[q + 1] : 0.f;
    float ym = j > 0 ? x[q - sy] : 0.f, yp = j < n - 1 ? x[q + sy] : 0.f;
    float zm = k > 0 ? x[q - sz] : 0.f, zp = k < n - 1 ? x[q + sz] : 0.f;
    s = ((xp + xm) + (yp + ym)) + (zp + zm);
    float g = 0.f;
    if (i == 0) g += L.g_low;
    if (j == 0) g += L.g_low;
    if (k == 0) g += L.g_low;
    if (i == n - 1) g += L.g_high;
    if (j == n - 1) g += L.g_high;
    if (k == n - 1) g += L.g_high;
    nb = s;
    diag = 6.0f - g;
}

__device__ __forceinline__ void mg_jacobi_point(const MgLevel& L, const float* x, const float* b, float* out, float omega, long long e) {
    int i = (int)(e % L.P);
    long long row = e / L.P;
    int j = (int)(row % L.n), k = (int)(row / L.n);
    if (i >= L.n) return;
    float nb, diag;
    mg_stencil(L, x, i, j, k, nb, diag);
    float xq = x[e];
    out[e] = xq + (omega / diag) * ((float)(L.h * L.h) * b[e] + nb - diag * xq);
}

__device__ __forceinline__ void mg_residual_point(const MgLevel& L, const float* x, const float* b, float* out, long long e) {
    int i = (int)(e % L.P);
    long long row = e / L.P;
    int j = (int)(row % L.n), k = (int)(row / L.n);
    if (i >= L.n) return;
    float nb, diag;
    mg_stencil(L, x, i, j, k, nb, diag);
    out[e] = b[e] + (nb - diag * x[e]) / (float)(L.h * L.h);
}

__device__ __forceinline__ void mg_restrict_point(const MgLevel& C, const MgLevel& Fi, const float* rf, float* bc, long long e) {
    int i = (int)(e % C.P);
    long long row = e / C.P;
    int j = (int)(row % C.n), k = (int)(row / C.n);
    if (i >= C.n) return;
    const int fi = 2 * i + 1, fj = 2 * j + 1, fk = 2 * k + 1;
    float s = 0.f;
    for (int dz = -1; dz <= 1; ++dz) {
        int z = fk + dz;
        if (z >= Fi.n) continue;
        float wz = dz == 0 ? 0.5f : 0.25f;
        for (int dy = -1; dy <= 1; ++dy) {
            int y = fj + dy;
            if (y >= Fi.n) continue;
            float wy = dy == 0 ? 0.5f : 0.25f;
            for (int dx = -1; dx <= 1; ++dx) {
                int x = fi + dx;
                if (x >= Fi.n) continue;
                float wx = dx == 0 ? 0.5f : 0.25f;
                s += wx * wy * wz * rf[((long long)z * Fi.n + y) * Fi.P + x];
            }
        }
    }
    bc[e] = s;
}

__device__ __forceinline__ void mg_prolong_point(const MgLevel& C, const MgLevel& Fi, const float* xc, float* xf, long long e) {
    int i = (int)(e % Fi.P);
    long long row = e / Fi.P;
    int j = (int)(row % Fi.n), k = (int)(row / Fi.n);
    if (i >= Fi.n) return;
    // odd fine index 2c+1 -> coarse c (weight 1); even 2c -> coarse c-1 and c (weight 1/2 each)
    int ci[2], cj[2], ck[2];
    float wi[2], wj[2], wk[2];
    int ni = (i & 1) ? 1 : 2, nj = (j & 1) ? 1 : 2, nk = (k & 1) ? 1 : 2;
    if (i & 1) { ci[0] = i >> 1; wi[0] = 1.f; } else { ci[0] = (i >> 1) - 1; ci[1] = i >> 1; wi[0] = wi[1] = 0.5f; }
    if (j & 1) { cj[0] = j >> 1; wj[0] = 1.f; } else { cj[0] = (j >> 1) - 1; cj[1] = j >> 1; wj[0] = wj[1] = 0.5f; }
    if (k & 1) { ck[0] = k >> 1; wk[0] = 1.f; } else { ck[0] = (k >> 1) - 1; ck[1] = k >> 1; wk[0] = wk[1] = 0.5f; }
    float s = 0.f;
    for (int c3 = 0; c3 < nk; ++c3) {
        if (ck[c3] < 0 || ck[c3] >= C.n) continue;
        for (int c2 = 0; c2 < nj; ++c2) {
            if (cj[c2] < 0 || cj[c2] >= C.n) continue;
            for (int c1 = 0; c1 < ni; ++c1) {
                if (ci[c1] < 0 || ci[c1] >= C.n) continue;
                s += wi[c1] * wj[c2] * wk[c3] * xc[((long long)ck[c3] * C.n + cj[c2]) * C.P + ci[c1]];
            }
        }
    }
    xf[e] += s;
}

__global__ void mg_jacobi_kernel(MgLevel L, const float* __restrict__ x, const float* __restrict__ b, float* __restrict__ out, float omega) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < L.F; e += (long long)gridDim.x * blockDim.x)
        mg_jacobi_point(L, x, b, out, omega, e);
}
__global__ void mg_residual_kernel(MgLevel L, const float* __restrict__ x, const float* __restrict__ b, float* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < L.F; e += (long long)gridDim.x * blockDim.x)
        mg_residual_point(L, x, b, out, e);
}
__global__ void mg_restrict_kernel(MgLevel C, MgLevel Fi, const float* __restrict__ rf, float* __restrict__ bc) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < C.F; e += (long long)gridDim.x * blockDim.x)
        mg_restrict_point(C, Fi, rf, bc, e);
}
__global__ void mg_prolong_kernel(MgLevel C, MgLevel Fi, const float* __restrict__ xc, float* __restrict__ xf) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < Fi.F; e += (long long)gridDim.x * blockDim.x)
        mg_prolong_point(C, Fi, xc, xf, e);
}

// The bottom of the V-cycle in one CTA: level lv[0] receives its right-hand side in b[0]; the
// result lands in x[0]. Same sequence as the per-level launches (x <- 0, pre sweeps, residual,
// restrict, recurse, prolong-add, post sweeps; the coarsest level does `coarsest` sweeps).
__global__ void __launch_bounds__(1024) mg_coarse_kernel(MgCoarse c, float omega, int pre, int post, int coarsest) {
    const int nl = c.nlev;
    auto zero = [&](int l) {
        for (long long e = threadIdx.x; e < c.lv[l].F; e += blockDim.x) c.x[l][e] = 0.f;
    };
    auto smooth = [&](int l, int sweeps) {
        for (int s = 0; s < sweeps; ++s) {
            const float* src = (s & 1) ? c.tmp[l] : c.x[l];
            float* dst = (s & 1) ? c.x[l] : c.tmp[l];
            for (long long e = threadIdx.x; e < c.lv[l].F; e += blockDim.x) mg_jacobi_point(c.lv[l], src, c.b[l], dst, omega, e);
            __syncthreads();
        }
    };
    // descend
    for (int l = 0; l < nl; ++l) {
        zero(l);
        __syncthreads();
        if (l == nl - 1) {
            smooth(l, coarsest);
            break;
        }
        smooth(l, pre);
        for (long long e = threadIdx.x; e < c.lv[l].F; e += blockDim.x) mg_residual_point(c.lv[l], c.x[l], c.b[l], c.res[l], e);
        __syncthreads();
        for (long long e = threadIdx.x; e < c.lv[l + 1].F; e += blockDim.x) mg_restrict_point(c.lv[l + 1], c.lv[l], c.res[l], c.b[l + 1], e);
        __syncthreads();
    }
    // ascend
    for (int l = nl - 2; l >= 0; --l) {
        for (long long e = threadIdx.x; e < c.lv[l].F; e += blockDim.x) mg_prolong_point(c.lv[l + 1], c.lv[l], c.x[l + 1], c.x[l], e);
        __syncthreads();
        smooth(l, post);
    }
}

// ---- CG scalars. scal layout: [0] pap, [1],[2] rz (alternating), [3] rr, [4] error flag
__global__ void cg_update_kernel(long long F4, float4* __restrict__ v, float4* __restrict__ r, const float4* __restrict__ p,
                                 const float4* __restrict__ ap, const double* __restrict__ scal, int rz_slot) {
    const double pap = scal[0], rz = scal[rz_slot];
    const bool ok = pap > 0.0 && rz > 0.0;
    const float alpha = ok ? (float)(rz / pap) : 0.0f;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F4; e += (long long)gridDim.x * blockDim.x) {
        float4 pv = p[e], a = ap[e], vv = v[e], rv = r[e];
        // v += alpha p; r -= alpha A p = r + alpha L p  (ap holds L p)
        vv.x = fmaf(alpha, pv.x, vv.x); vv.y = fmaf(alpha, pv.y, vv.y); vv.z = fmaf(alpha, pv.z, vv.z); vv.w = fmaf(alpha, pv.w, vv.w);
        rv.x = fmaf(alpha, a.x, rv.x); rv.y = fmaf(alpha, a.y, rv.y); rv.z = fmaf(alpha, a.z, rv.z); rv.w = fmaf(alpha, a.w, rv.w);
        v[e] = vv;
        r[e] = rv;
    }
}

__global__ void cg_direction_kernel(long long F4, float4* __restrict__ p, const float4* __restrict__ z, const double* __restrict__ scal,
                                    int rz_old, int rz_new) {
    const float beta = (float)(scal[rz_new] / scal[rz_old]);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F4; e += (long long)gridDim.x * blockDim.x) {
        float4 zz = z[e], pp = p[e];
        pp.x = fmaf(beta, pp.x, zz.x); pp.y = fmaf(beta, pp.y, zz.y); pp.z = fmaf(beta, pp.z, zz.z); pp.w = fmaf(beta, pp.w, zz.w);
        p[e] = pp;
    }
}

}  // namespace

void launch_poisson_rhs(const Layout& L, const float* rho, const double* q, double* ghost, float* b, cudaStream_t s) {
    const long long need = 24LL * L.n * L.n;
    ghost_kernel<<<blocks_for(need), TPB, 0, s>>>(L.n, L.h, L.origin, q, ghost);
    KS_LAUNCH_CHECK();
    rhs_kernel<<<blocks_for(L.F), TPB, 0, s>>>(L.n, L.P, L.F, L.h, rho, ghost, b);
    KS_LAUNCH_CHECK();
}

void launch_mg_jacobi(const MgLevel& lv, const float* x, const float* b, float* out, float omega, cudaStream_t s) {
    mg_jacobi_kernel<<<blocks_for(lv.F), TPB, 0, s>>>(lv, x, b, out, omega);
    KS_LAUNCH_CHECK();
}
void launch_mg_residual(const MgLevel& lv, const float* x, const float* b, float* out, cudaStream_t s) {
    mg_residual_kernel<<<blocks_for(lv.F), TPB, 0, s>>>(lv, x, b, out);
    KS_LAUNCH_CHECK();
}
void launch_mg_restrict(const MgLevel& coarse, const MgLevel& fine, const float* rf, float* bc, cudaStream_t s) {
    mg_restrict_kernel<<<blocks_for(coarse.F), TPB, 0, s>>>(coarse, fine, rf, bc);
    KS_LAUNCH_CHECK();
}
void launch_mg_prolong_add(const MgLevel& coarse, const MgLevel& fine, const float* xc, float* xf, cudaStream_t s) {
    mg_prolong_kernel<<<blocks_for(fine.F), TPB, 0, s>>>(coarse, fine, xc, xf);
    KS_LAUNCH_CHECK();
}
void launch_mg_coarse(const MgCoarse& c, float omega, int pre, int post, int coarsest_sweeps, cudaStream_t s) {
    if (c.nlev <= 0) return;
    mg_coarse_kernel<<<1, 1024, 0, s>>>(c, omega, pre, post, coarsest_sweeps);
    KS_LAUNCH_CHECK();
}

void launch_cg_update(long long F, float* v, float* r, const float* p, const float* ap, const double* scal, int rz_slot, cudaStream_t s) {
    cg_update_kernel<<<blocks_for(F / 4), TPB, 0, s>>>(F / 4, reinterpret_cast<float4*>(v), reinterpret_cast<float4*>(r),
                                                      reinterpret_cast<const float4*>(p), reinterpret_cast<const float4*>(ap), scal, rz_slot);
    KS_LAUNCH_CHECK();
}
void launch_cg_direction(long long F, float* p, const float* z, const double* scal, int rz_old, int rz_new, cudaStream_t s) {
    cg_direction_kernel<<<blocks_for(F / 4), TPB, 0, s>>>(F / 4, reinterpret_cast<float4*>(p), reinterpret_cast<const float4*>(z), scal,
                                                         rz_old, rz_new);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
