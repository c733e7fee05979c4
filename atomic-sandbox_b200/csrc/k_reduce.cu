// k_reduce.cu -- deterministic reductions over pitched fields (sm_100a).
//
// The reference finishes every reduction in f64 on the host from f32 workgroup partials
// (crates/qm-gpu/src/reduce.rs:1-3, :225-234). Here the whole reduction stays on the device: a
// kernel writes one f64 partial per CTA and value (fixed grid size, fixed per-thread order, fixed
// shuffle tree), and `finish` sums the partials of all CTAs in index order with Neumaier
// compensation. The same inputs therefore give the same bits on every run, and no host round
// trip is needed until a scalar is actually wanted on the host.
#include <cmath>
#include <cudaTypedefs.h>
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

// ---- the Gram block on CUDA cores with the chunk staged in shared memory (blocks whose tiles fit one CTA).
// The CTA's warps cover every 8 x 8 tile of G, so each field value is read from HBM once for all of them: per chunk of
// 32 points, two TMA boxes (the 32-point slab of the m rows of S, and of the mt rows of T) land in a shared-memory
// slice, with the next G2_RING - 1 chunks in flight. Lane l owns point l of each chunk; the arithmetic is the form
// above (f32 per lane over its points, f64 across the lanes). S^T S is symmetric bit for bit (the same products in the
// same order), so only its upper tiles are computed and each off-diagonal one is also written transposed: at
// m = mt = 24 that is 6 + 9 = 15 tiles, one warp each.
constexpr int G2_MAX_TILES = 16;  // warps per CTA (512 threads: up to 128 registers each)
constexpr int G2_RING = 8;        // shared-memory slices: the next G2_RING - 1 chunks in flight
constexpr long long G2_WAIT_LIMIT = 1LL << 22;
// a 32-point box's inner extent is 128 bytes and its x coordinate a multiple of 32 floats: both multiples of 16 bytes,
// as TMA requires (a violation faults the GPU instead of returning an error)
static_assert((32 * 4) % 16 == 0, "TMA box inner extent and x coordinates must be multiples of 16 bytes");
__device__ __forceinline__ unsigned g2_su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
__device__ __forceinline__ bool g2_wait(uint64_t* bar, unsigned parity, long long limit) {
    for (long long n = 0;; ++n) {
        unsigned ok;
        asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(ok)
                     : "r"(g2_su32(bar)), "r"(parity)
                     : "memory");
        if (ok) return true;
        if (n > limit) return false;
    }
}
__device__ __forceinline__ void g2_tma(void* dst, const CUtensorMap* map, int x, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(g2_su32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(0), "r"(g2_su32(bar))
        : "memory");
}

__global__ void __launch_bounds__(G2_MAX_TILES * 32, 1) gram2_kernel(const __grid_constant__ CUtensorMap tm_s,
                                                                     const __grid_constant__ CUtensorMap tm_t, long long F, int m,
                                                                     int mt, int ntiles, double* __restrict__ partials, int* err) {
    // G2_RING slices of rows x 32 points: S at rows [0, m), T at rows [r8m, r8m + mt), r8m = round8(m); rows that no box
    // writes only feed tile entries that are discarded, so every tile reads 8 whole rows without clamping
    extern __shared__ __align__(128) float g2buf[];
    __shared__ __align__(8) uint64_t bar[G2_RING];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int mc = m + mt;
    const int r8m = (m + 7) & ~7;
    const int rows = r8m + ((mt + 7) & ~7);
    const long long chunks = (F + 31) / 32;
    const int nmine = (int)((chunks - blockIdx.x + gridDim.x - 1) / gridDim.x);  // chunks blockIdx.x + j * gridDim.x
    if (threadIdx.x == 0) {
        for (int i = 0; i < G2_RING; ++i) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(g2_su32(&bar[i])) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    const unsigned box_bytes = (unsigned)(mc * 32 * 4);  // whole boxes land, the zero fill past F included
    auto issue = [&](int j) {  // thread 0: this CTA's j-th chunk into slice j % G2_RING
        const int sl = j % G2_RING;
        const int x = (int)(((long long)blockIdx.x + (long long)j * gridDim.x) * 32);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(g2_su32(&bar[sl])), "r"(box_bytes) : "memory");
        float* dst = g2buf + (size_t)sl * rows * 32;
        g2_tma(dst, &tm_s, x, &bar[sl]);
        if (mt > 0) g2_tma(dst + (size_t)r8m * 32, &tm_t, x, &bar[sl]);
    };
    // tiles: the upper triangle of S^T S (tile rows ti <= tj), then S^T T (tiles_r x tiles_t); c0 is the shared-memory
    // row of the tile's first column, col0 its column in G
    const int tiles_r = (m + GT - 1) / GT, tiles_t = (mt + GT - 1) / GT;
    const int nsym = tiles_r * (tiles_r + 1) / 2;
    const bool active = warp < ntiles;
    int r0 = 0, c0 = 0, col0 = 0;
    bool mirror = false;
    if (active) {
        if (warp < nsym) {
            int ti = 0, rem = warp;
            while (rem >= tiles_r - ti) { rem -= tiles_r - ti; ++ti; }
            const int tj = ti + rem;
            r0 = ti * GT;
            c0 = col0 = tj * GT;
            mirror = tj != ti;
        } else {
            const int t = warp - nsym;
            r0 = (t / tiles_t) * GT;
            c0 = r8m + (t % tiles_t) * GT;
            col0 = m + (t % tiles_t) * GT;
        }
    }
    float acc[GT][GT];
#pragma unroll
    for (int a = 0; a < GT; ++a)
#pragma unroll
        for (int c = 0; c < GT; ++c) acc[a][c] = 0.f;
    int issued = min(G2_RING - 1, nmine);
    if (threadIdx.x == 0)
        for (int j = 0; j < issued; ++j) issue(j);
    bool alive = true;
    for (int j = 0; j < nmine; ++j) {
        const int sl = j % G2_RING;
        // the slice of chunk j - 1 was released by the barrier that ended it: keep G2_RING - 1 chunks in flight
        if (alive && issued < nmine) {
            if (threadIdx.x == 0) issue(issued);
            ++issued;
        }
        if (!g2_wait(&bar[sl], (unsigned)((j / G2_RING) & 1), alive ? G2_WAIT_LIMIT : 1)) {
            if (alive && err) atomicExch(err, 1);
            alive = false;  // the partials are undefined; the host's next readback reports the error
        }
        if (active) {  // points past F are the boxes' zero fill: they add nothing
            const float* slp = g2buf + (size_t)sl * rows * 32 + lane;
            float cv[GT];
#pragma unroll
            for (int c = 0; c < GT; ++c) cv[c] = slp[(c0 + c) * 32];
#pragma unroll
            for (int a = 0; a < GT; ++a) {
                const float r = slp[(r0 + a) * 32];
#pragma unroll
                for (int c = 0; c < GT; ++c) acc[a][c] = fmaf(r, cv[c], acc[a][c]);
            }
        }
        __syncthreads();  // slice sl is free for chunk j + G2_RING
    }
    if (!alive && threadIdx.x == 0)  // copies still in flight land before the CTA's shared memory is released
        for (int j = max(0, issued - G2_RING); j < issued; ++j) g2_wait(&bar[j % G2_RING], (unsigned)((j / G2_RING) & 1), 1LL << 16);
    if (!active) return;
    const size_t base = (size_t)blockIdx.x * ((size_t)m * mc);
    const int cend = col0 < m ? m : mc;  // a tile's columns stay inside its block (S or T)
#pragma unroll
    for (int a = 0; a < GT; ++a)
#pragma unroll
        for (int c = 0; c < GT; ++c) {
            const double v = warp_sum((double)acc[a][c]);
            if (lane == 0 && r0 + a < m && col0 + c < cend) {
                partials[base + (size_t)(r0 + a) * mc + (col0 + c)] = v;
                if (mirror) partials[base + (size_t)(col0 + c) * mc + (r0 + a)] = v;
            }
        }
}

PFN_cuTensorMapEncodeTiled_v12000 g2_encode() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        cudaDriverEntryPointQueryResult q;
        void* ptr = nullptr;
        KS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !ptr) throw DeviceError("cuTensorMapEncodeTiled is not available");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }();
    return fn;
}

// rows fields of F floats (stride F) as a 2-D tensor map with 32-point x rows boxes, no swizzle
void g2_rows_map(CUtensorMap* map, const float* base, long long F, int rows) {
    cuuint64_t dims[2] = {(cuuint64_t)F, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)F * 4};
    cuuint32_t box[2] = {32, (cuuint32_t)rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = g2_encode()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw DeviceError("cuTensorMapEncodeTiled (CUDA-core Gram) failed, code " + std::to_string((int)r));
}

// ---- multipole moments with on-the-fly real solid harmonics: the recurrence of harmonics.cuh with its (l, m) constants
// read from a table (f_l = sqrt((2l - 1) / (2l)), b_lm = sqrt(max((l - 1)^2 - m^2, 0)) and 1 / sqrt(l^2 - m^2), computed once
// on the host), the two previous rows kept in registers and each R_lm added to its moment as it is formed: no square
// root or division per point, no per-point array in local memory. The only difference from solid_harmonics_dev is the
// product by 1 / d instead of the division by d (within an ulp per step).
__constant__ double c_hf[7];
__constant__ double c_hb[7][7];
__constant__ double c_hinvd[7][7];

__global__ void __launch_bounds__(TPB) moments_kernel(int n, int P, long long F, double h, double origin, const float* __restrict__ rho,
                                                      double* __restrict__ partials) {
    double acc[49];
#pragma unroll
    for (int q = 0; q < 49; ++q) acc[q] = 0.0;
    const double s2 = 1.4142135623730951;
    const long long N = (long long)n * n * n;
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < N; p += (long long)gridDim.x * blockDim.x) {
        int i = (int)(p % n);
        long long rest = p / n;
        int j = (int)(rest % n), k = (int)(rest / n);
        const double r = (double)rho[((long long)k * n + j) * P + i];
        if (r == 0.0) continue;
        const double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        const double r2 = x * x + y * y + z * z;
        double pr[7], pi[7], qr[7], qi[7];  // rows l - 1 and l - 2 of the recurrence
        pr[0] = 1.0;
        pi[0] = 0.0;
        acc[0] += r * 1.0;
#pragma unroll
        for (int l = 1; l <= 6; ++l) {
            double cr[7], ci[7];
            cr[l] = c_hf[l] * (x * pr[l - 1] - y * pi[l - 1]);
            ci[l] = c_hf[l] * (x * pi[l - 1] + y * pr[l - 1]);
            const double a = (2.0 * l - 1.0) * z;
#pragma unroll
            for (int m = 0; m < l; ++m) {
                const double r0 = (l >= 2 && m <= l - 2) ? qr[m] : 0.0, i0 = (l >= 2 && m <= l - 2) ? qi[m] : 0.0;
                const double b = c_hb[l][m] * r2;
                cr[m] = (a * pr[m] - b * r0) * c_hinvd[l][m];
                ci[m] = (a * pi[m] - b * i0) * c_hinvd[l][m];
            }
            acc[l * l + l] += r * cr[0];
#pragma unroll
            for (int m = 1; m <= l; ++m) {
                acc[l * l + l + m] += r * (s2 * cr[m]);
                acc[l * l + l - m] += r * (s2 * ci[m]);
            }
#pragma unroll
            for (int m = 0; m <= l; ++m) {
                qr[m] = pr[m];
                qi[m] = pi[m];
                pr[m] = cr[m];
                pi[m] = ci[m];
            }
        }
    }
    // unrolled, so that acc stays in registers (a runtime index would put it in local memory for the whole kernel)
#pragma unroll
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

// warps of the staged form: the upper tiles of S^T S and the tiles of S^T T
static int gram2_tiles(int m, int mt) {
    const int tr = ceil_div(m, GT), tt = ceil_div(mt, GT);
    return tr * (tr + 1) / 2 + tr * tt;
}

int gram_blocks(int m, int mt) { return gram2_tiles(m, mt) <= G2_MAX_TILES ? sm_count() : 2 * sm_count(); }

int launch_gram(long long F, int m, const float* S, int mt, const float* T, double* partials, cudaStream_t s) {
    const int tiles_r = ceil_div(m, GT), tiles_c = ceil_div(m + mt, GT);
    const int ntiles = tiles_r * tiles_c;
    const int blocks = gram_blocks(m, mt);
    const int tiles2 = gram2_tiles(m, mt);
    if (tiles2 <= G2_MAX_TILES) {
        if (F % 4 != 0 || reinterpret_cast<uintptr_t>(S) % 16 != 0 || (mt > 0 && reinterpret_cast<uintptr_t>(T) % 16 != 0))
            throw std::invalid_argument("gram: fields must be 16-byte aligned with F a multiple of 4 floats");
        const size_t smem = (size_t)G2_RING * (((m + 7) & ~7) + ((mt + 7) & ~7)) * 32 * sizeof(float);
        static std::atomic<unsigned long long> attr_set{0};
        once_per_device(attr_set, [] {
            KS_CUDA(cudaFuncSetAttribute(gram2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, G2_RING * 136 * 32 * (int)sizeof(float)));
        });
        CUtensorMap ms, mtm;
        g2_rows_map(&ms, S, F, m);
        g2_rows_map(&mtm, mt > 0 ? T : S, F, mt > 0 ? mt : 1);
        gram2_kernel<<<blocks, tiles2 * 32, smem, s>>>(ms, mtm, F, m, mt, tiles2, partials, device_error_flag());
        KS_LAUNCH_CHECK();
        return blocks;
    }
    dim3 grid(blocks, ceil_div(ntiles, GW));
    // partials are indexed by blockIdx.x only: every tile of a CTA column writes its own entries
    gram_kernel<<<grid, GW * 32, 0, s>>>(F, m, S, mt, T, tiles_c, ntiles, partials);
    KS_LAUNCH_CHECK();
    return blocks;
}

void launch_moments(const Layout& L, const float* rho, double* partials, int blocks, cudaStream_t s) {
    static std::atomic<unsigned long long> consts_set{0};
    once_per_device(consts_set, [] {
        double f[7] = {0}, b[7][7] = {{0}}, invd[7][7] = {{0}};
        for (int l = 1; l <= 6; ++l) {
            f[l] = std::sqrt((2.0 * l - 1.0) / (2.0 * l));
            for (int m = 0; m < l; ++m) {
                b[l][m] = std::sqrt(std::fmax((l - 1.0) * (l - 1.0) - (double)m * m, 0.0));
                invd[l][m] = 1.0 / std::sqrt((double)l * l - (double)m * m);
            }
        }
        KS_CUDA(cudaMemcpyToSymbol(c_hf, f, sizeof(f)));
        KS_CUDA(cudaMemcpyToSymbol(c_hb, b, sizeof(b)));
        KS_CUDA(cudaMemcpyToSymbol(c_hinvd, invd, sizeof(invd)));
    });
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
