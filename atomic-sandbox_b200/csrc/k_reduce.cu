// k_reduce.cu -- deterministic reductions over pitched fields (sm_100a).
//
// The reference finishes every reduction in f64 on the host from f32 workgroup partials
// (crates/qm-gpu/src/reduce.rs:1-3, :225-234). Here the whole reduction stays on the device: a
// kernel writes one f64 partial per CTA and value (fixed grid size, fixed per-thread order, fixed
// shuffle tree), and `finish` sums the partials of all CTAs in index order with Neumaier
// compensation. The same inputs therefore give the same bits on every run, and no host round
// trip is needed until a scalar is actually wanted on the host.
#include <cmath>
#include "kernels.cuh"
#include "reduce_util.cuh"
#include "harmonics.cuh"

namespace ks {

namespace {

constexpr int TPB = 256;

// One warp per value: lane l sums the partials of CTAs l, l+32, ... (Neumaier), then the lanes are
// combined by a fixed shuffle tree -- the same order on every run. With trows > 0 the value v =
// r*tcols + c is written transposed, to out[c*trows + r].
__global__ void finish_kernel(const double* __restrict__ partials, int blocks, int nvals, double scale, double* __restrict__ out,
                              int trows, int tcols) {
    const int v = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (v >= nvals) return;
    double sum = 0.0, comp = 0.0;
    for (int b = lane; b < blocks; b += 32) {
        double x = partials[(size_t)b * nvals + v];
        double t = sum + x;
        if (fabs(sum) >= fabs(x)) comp += (sum - t) + x; else comp += (x - t) + sum;
        sum = t;
    }
    double total = warp_sum(sum + comp);
    if (lane == 0) {
        int o = v;
        if (trows > 0) o = (v % tcols) * trows + v / tcols;
        out[o] = total * scale;
    }
}

// finish_kernel over two descriptors: warps [0, a.nvals) finish a, the next b.nvals warps finish b
__global__ void finish_pair_kernel(FinishDesc a, FinishDesc b) {
    int v = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    const FinishDesc& d = v < a.nvals ? a : b;
    if (v >= a.nvals) v -= a.nvals;
    if (v >= d.nvals) return;
    double sum = 0.0, comp = 0.0;
    for (int blk = lane; blk < d.blocks; blk += 32) {
        double x = d.partials[(size_t)blk * d.nvals + v];
        double t = sum + x;
        if (fabs(sum) >= fabs(x)) comp += (sum - t) + x; else comp += (x - t) + sum;
        sum = t;
    }
    double total = warp_sum(sum + comp);
    if (lane == 0) {
        int o = v;
        if (d.trows > 0) o = (v % d.tcols) * d.trows + v / d.tcols;
        d.out[o] = total * d.scale;
    }
}

__global__ void finish_max_kernel(const double* __restrict__ partials, int blocks, double* __restrict__ out) {
    double m = 0.0;
    for (int b = threadIdx.x; b < blocks; b += blockDim.x) m = fmax(m, partials[b]);
    m = block_max(m);
    if (threadIdx.x == 0) out[0] = m;
}

__global__ void dots_kernel(long long F4, Pairs p, double* __restrict__ partials) {
    double acc[Pairs::MAX];
#pragma unroll
    for (int q = 0; q < Pairs::MAX; ++q) acc[q] = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F4; e += (long long)gridDim.x * blockDim.x) {
#pragma unroll
        for (int q = 0; q < Pairs::MAX; ++q) {
            if (q < p.count) {
                float4 a = reinterpret_cast<const float4*>(p.a[q])[e];
                float4 b = reinterpret_cast<const float4*>(p.b[q])[e];
                acc[q] += (double)a.x * b.x + (double)a.y * b.y + (double)a.z * b.z + (double)a.w * b.w;
            }
        }
    }
    for (int q = 0; q < p.count; ++q) {
        double s = block_sum(acc[q]);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * p.count + q] = s;
    }
}

// ---- the Gram block G = S^T [S | T] on CUDA cores.
// Thread-per-point, register-blocked warp tiles: lane l of a warp owns one grid point of the
// CTA's current 32-point chunk and an 8 x 8 tile of G (64 f32 accumulators); the warps of the CTA
// cover up to GW tiles of G and walk the same chunks, so each field value is fetched from HBM
// once and served to the other warps from L1. Lanes accumulate in f32 over their points (a few
// dozen per lane), the lanes of a warp are combined in f64.
constexpr int GT = 8;    // warp tile edge
constexpr int GW = 16;   // warps per CTA (tiles per CTA row of blockIdx.y)

__global__ void __launch_bounds__(GW * 32) gram_kernel(long long F, int m, const float* __restrict__ S, int mt,
                                                       const float* __restrict__ T, int tiles_c, int ntiles,
                                                       double* __restrict__ partials) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.y * GW + warp;
    const int mc = m + mt;
    const long long chunks = (F + 31) / 32;
    float acc[GT][GT];
#pragma unroll
    for (int a = 0; a < GT; ++a)
#pragma unroll
        for (int b = 0; b < GT; ++b) acc[a][b] = 0.f;
    int r0 = 0, c0 = 0;
    const float* rowp[GT];
    const float* colp[GT];
    if (tile < ntiles) {
        r0 = (tile / tiles_c) * GT;
        c0 = (tile % tiles_c) * GT;
#pragma unroll
        for (int a = 0; a < GT; ++a) {
            int r = min(r0 + a, m - 1);
            rowp[a] = S + (long long)r * F;
            int c = min(c0 + a, mc - 1);
            colp[a] = c < m ? S + (long long)c * F : T + (long long)(c - m) * F;
        }
        for (long long ch = blockIdx.x; ch < chunks; ch += gridDim.x) {
            long long e = ch * 32 + lane;
            if (e < F) {
                float rv[GT], cv[GT];
#pragma unroll
                for (int a = 0; a < GT; ++a) rv[a] = __ldg(rowp[a] + e);
#pragma unroll
                for (int b = 0; b < GT; ++b) cv[b] = __ldg(colp[b] + e);
#pragma unroll
                for (int a = 0; a < GT; ++a)
#pragma unroll
                    for (int b = 0; b < GT; ++b) acc[a][b] = fmaf(rv[a], cv[b], acc[a][b]);
            }
        }
    }
    if (tile >= ntiles) return;  // whole warp: no CTA-wide sync below
    const size_t base = (size_t)(blockIdx.x) * ((size_t)m * mc);
#pragma unroll
    for (int a = 0; a < GT; ++a)
#pragma unroll
        for (int b = 0; b < GT; ++b) {
            double v = warp_sum((double)acc[a][b]);
            if (lane == 0 && r0 + a < m && c0 + b < mc) partials[base + (size_t)(r0 + a) * mc + (c0 + b)] = v;
        }
}

// ---- multipole moments with on-the-fly real solid harmonics (harmonics.cuh)
__global__ void __launch_bounds__(TPB) moments_kernel(int n, int P, long long F, double h, double origin, const float* __restrict__ rho,
                                                      double* __restrict__ partials) {
    double acc[49];
#pragma unroll
    for (int q = 0; q < 49; ++q) acc[q] = 0.0;
    const long long N = (long long)n * n * n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n);
        long long rest = p / n;
        int j = (int)(rest % n), k = (int)(rest / n);
        double r = (double)rho[((long long)k * n + j) * P + i];
        if (r == 0.0) continue;
        double hv[49];
        solid_harmonics_dev(origin + i * h, origin + j * h, origin + k * h, hv);
#pragma unroll
        for (int q = 0; q < 49; ++q) acc[q] += r * hv[q];
    }
    for (int q = 0; q < 49; ++q) {
        double s = block_sum(acc[q]);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * 49 + q] = s;
    }
}

__global__ void face_max_kernel(int n, int P, const float* __restrict__ f, double* __restrict__ partials) {
    double m = 0.0;
    const long long per_face = (long long)n * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 6 * per_face; t += (long long)gridDim.x * blockDim.x) {
        int face = (int)(t / per_face);
        long long uv = t % per_face;
        int u = (int)(uv % n), v = (int)(uv / n);
        int c = (face & 1) ? n - 1 : 0;
        int i, j, k;
        switch (face >> 1) {
            case 0: i = c; j = u; k = v; break;
            case 1: i = u; j = c; k = v; break;
            default: i = u; j = v; k = c; break;
        }
        m = fmax(m, fabs((double)f[((long long)k * n + j) * P + i]));
    }
    m = block_max(m);
    if (threadIdx.x == 0) partials[blockIdx.x] = m;
}

// forces.rs:167-172 g'(d) for g(d) = erf(d/(sigma sqrt2))/d; 0 below 1e-8
__device__ __forceinline__ double g_prime(double d, double sigma) {
    if (d < 1e-8) return 0.0;
    double u = d / (sigma * 1.4142135623730951);
    return ((2.0 / 1.7724538509055159) * u * exp(-u * u) - erf(u)) / (d * d);
}

constexpr int MAX_NUC = 32;
__global__ void __launch_bounds__(TPB) forces_kernel(int n, int P, double h, double origin, const float* __restrict__ rho,
                                                     const Nuc* __restrict__ nuc, int nn, double sigma, double* __restrict__ partials) {
    double acc[3 * MAX_NUC];
    for (int q = 0; q < 3 * nn; ++q) acc[q] = 0.0;
    const long long N = (long long)n * n * n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n);
        long long rest = p / n;
        int j = (int)(rest % n), k = (int)(rest / n);
        double r = (double)rho[((long long)k * n + j) * P + i];
        if (r == 0.0) continue;
        double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        for (int a = 0; a < nn; ++a) {
            double dx = x - nuc[a].x, dy = y - nuc[a].y, dz = z - nuc[a].z;
            double d = sqrt(dx * dx + dy * dy + dz * dz);
            if (d < 1e-8) continue;
            double gp = -nuc[a].Z * g_prime(d, sigma) / d;
            double w = r * gp;
            acc[3 * a] += w * dx;
            acc[3 * a + 1] += w * dy;
            acc[3 * a + 2] += w * dz;
        }
    }
    for (int q = 0; q < 3 * nn; ++q) {
        double s = block_sum(acc[q]);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * 3 * nn + q] = s;
    }
}

// The adjoint of the Kohn-Sham energy with respect to the nuclear positions and the smearing width.
// At self-consistency E is stationary in the density, so the response of the Hartree and XC terms
// (and of the kinetic energy) to a change of V_ext vanishes and the VJP reduces to
//     dE/dR_I     = integral rho(r) dV_I/dR_I = integral rho Z_I g'(d)/d (r - R_I),   g(d) = erf(d / (sigma sqrt 2)) / d
//     dE/dsigma   = integral rho(r) sum_I dV_I/dsigma = integral rho sum_I Z_I sqrt(2/pi) exp(-d^2 / (2 sigma^2)) / sigma^2
// (V_I = -Z_I g(d); crates/qm/src/nuclear.rs:258-272 and crates/qm/src/forces.rs:177-227 for the
// position term). rho is recomputed here from the occupied orbitals of both spins in f64, not read
// from a stored density. partials: [blocks][3 nn + 1], dV not applied.
__global__ void __launch_bounds__(TPB) vjp_kernel(int n, int P, long long F, double h, double origin, const float* __restrict__ up, int nup,
                                                  const double* __restrict__ wu, const float* __restrict__ dn, int ndn,
                                                  const double* __restrict__ wd, const Nuc* __restrict__ nuc, int nn, double sigma,
                                                  double* __restrict__ partials) {
    double acc[3 * MAX_NUC + 1];
    for (int q = 0; q < 3 * nn + 1; ++q) acc[q] = 0.0;
    const long long N = (long long)n * n * n;
    const double inv2s2 = 1.0 / (2.0 * sigma * sigma);
    const double csig = 0.79788456080286536 / (sigma * sigma);  // sqrt(2/pi) / sigma^2
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n);
        long long rest = p / n;
        int j = (int)(rest % n), k = (int)(rest / n);
        const long long e = ((long long)k * n + j) * P + i;
        double r = 0.0;
        for (int v = 0; v < nup; ++v) {
            const double x = (double)up[(long long)v * F + e];
            r += (wu ? wu[v] : 1.0) * x * x;
        }
        for (int v = 0; v < ndn; ++v) {
            const double x = (double)dn[(long long)v * F + e];
            r += (wd ? wd[v] : 1.0) * x * x;
        }
        if (r == 0.0) continue;
        double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        for (int a = 0; a < nn; ++a) {
            double dx = x - nuc[a].x, dy = y - nuc[a].y, dz = z - nuc[a].z;
            double d2 = dx * dx + dy * dy + dz * dz;
            acc[3 * nn] += r * nuc[a].Z * csig * exp(-d2 * inv2s2);
            double d = sqrt(d2);
            if (d < 1e-8) continue;
            double w = r * nuc[a].Z * g_prime(d, sigma) / d;
            acc[3 * a] += w * dx;
            acc[3 * a + 1] += w * dy;
            acc[3 * a + 2] += w * dz;
        }
    }
    for (int q = 0; q < 3 * nn + 1; ++q) {
        double s = block_sum(acc[q]);
        if (threadIdx.x == 0) partials[(size_t)blockIdx.x * (3 * nn + 1) + q] = s;
    }
}

}  // namespace

int reduce_blocks(long long F) {
    long long want = (F / 4 + TPB - 1) / TPB;
    long long cap = 2LL * sm_count();
    return (int)std::max(1LL, std::min(want, cap));
}

void launch_finish(const double* partials, int blocks, int nvals, double scale, double* out, cudaStream_t s) {
    finish_kernel<<<ceil_div((long long)nvals * 32, 256), 256, 0, s>>>(partials, blocks, nvals, scale, out, 0, 0);
    KS_LAUNCH_CHECK();
}

void launch_finish_pair(const FinishDesc& a, const FinishDesc& b, cudaStream_t s) {
    finish_pair_kernel<<<ceil_div((long long)(a.nvals + b.nvals) * 32, 256), 256, 0, s>>>(a, b);
    KS_LAUNCH_CHECK();
}

void launch_finish_transposed(const double* partials, int blocks, int rows, int cols, double scale, double* out, cudaStream_t s) {
    finish_kernel<<<ceil_div((long long)rows * cols * 32, 256), 256, 0, s>>>(partials, blocks, rows * cols, scale, out, rows, cols);
    KS_LAUNCH_CHECK();
}

void launch_finish_max(const double* partials, int blocks, double* out, cudaStream_t s) {
    finish_max_kernel<<<1, TPB, 0, s>>>(partials, blocks, out);
    KS_LAUNCH_CHECK();
}

void launch_dots(long long F, const Pairs& p, double* partials, int blocks, cudaStream_t s) {
    if (p.count < 1 || p.count > Pairs::MAX) throw std::invalid_argument("dots: 1..16 pairs");
    dots_kernel<<<blocks, TPB, 0, s>>>(F / 4, p, partials);
    KS_LAUNCH_CHECK();
}

void launch_gram(long long F, int m, const float* S, int mt, const float* T, double* partials, int blocks, cudaStream_t s) {
    const int tiles_r = ceil_div(m, GT), tiles_c = ceil_div(m + mt, GT);
    const int ntiles = tiles_r * tiles_c;
    dim3 grid(blocks, ceil_div(ntiles, GW));
    // partials are indexed by blockIdx.x only: every tile of a CTA column writes its own entries
    gram_kernel<<<grid, GW * 32, 0, s>>>(F, m, S, mt, T, tiles_c, ntiles, partials);
    KS_LAUNCH_CHECK();
}

void launch_moments(const Layout& L, const float* rho, double* partials, int blocks, cudaStream_t s) {
    moments_kernel<<<blocks, TPB, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, rho, partials);
    KS_LAUNCH_CHECK();
}

void launch_face_max(const Layout& L, const float* f, double* partials, int blocks, cudaStream_t s) {
    face_max_kernel<<<blocks, TPB, 0, s>>>(L.n, L.P, f, partials);
    KS_LAUNCH_CHECK();
}

void launch_vjp(const Layout& L, const float* up, int nup, const double* wu, const float* dn, int ndn, const double* wd, const Nuc* nuc,
                int nn, double sigma, double* partials, int blocks, cudaStream_t s) {
    if (nn > MAX_NUC) throw std::invalid_argument("vjp: at most 32 nuclei");
    vjp_kernel<<<blocks, TPB, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, up, nup, wu, dn, ndn, wd, nuc, nn, sigma, partials);
    KS_LAUNCH_CHECK();
}

void launch_forces(const Layout& L, const float* rho, const Nuc* nuc, int nn, double sigma, double* partials, int blocks,
                   cudaStream_t s) {
    if (nn > MAX_NUC) throw std::invalid_argument("forces: at most 32 nuclei");
    forces_kernel<<<blocks, TPB, 0, s>>>(L.n, L.P, L.h, L.origin, rho, nuc, nn, sigma, partials);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
