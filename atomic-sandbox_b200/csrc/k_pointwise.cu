// k_pointwise.cu -- field generators and pointwise kernels of the Kohn-Sham hot path (sm_100a).
//
// All of these are HBM-streaming kernels: float4 loads/stores over whole blocks of pitched fields,
// grid-stride loops sized to a multiple of the SM count. Physics that needs precision (erf, the
// PW92 fit, the LCG guess) is evaluated in f64 and rounded to f32 once on the store.
#include <cmath>
#include "kernels.cuh"
#include "reduce_util.cuh"

namespace ks {

namespace {

constexpr int TPB = 256;

inline int stream_blocks(long long work_items) {
    long long b = (work_items + TPB - 1) / TPB;
    long long cap = 8LL * sm_count();
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

__device__ __forceinline__ void field_coords(long long e, int n, int P, int& i, int& j, int& k) {
    i = (int)(e % P);
    long long row = e / P;
    j = (int)(row % n);
    k = (int)(row / n);
}

// ------------------------------------------------------------------ generators
__global__ void nuclear_potential_kernel(int n, int P, long long F, double h, double origin, const Nuc* __restrict__ nuc, int nn,
                                         double sigma, float* __restrict__ out) {
    const double s2 = sigma * sqrt(2.0);
    const double on_site = sqrt(2.0 / 3.14159265358979323846) / sigma;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        field_coords(e, n, P, i, j, k);
        if (i >= n) { out[e] = 0.0f; continue; }
        double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        double acc = -0.0;
        for (int a = 0; a < nn; ++a) {
            double dx = x - nuc[a].x, dy = y - nuc[a].y, dz = z - nuc[a].z;
            double d = sqrt(dx * dx + dy * dy + dz * dz);
            acc += (d < 1e-10) ? -nuc[a].Z * on_site : -nuc[a].Z * erf(d / s2) / d;
        }
        out[e] = (float)acc;
    }
}

__global__ void deposit_charge_kernel(int n, int P, long long F, double h, double origin, const Nuc* __restrict__ nuc, int nn,
                                      double sigma, double scale, float* __restrict__ out) {
    const double norm = 1.0 / pow(2.0 * 3.14159265358979323846 * sigma * sigma, 1.5);
    const double inv_2s2 = 1.0 / (2.0 * sigma * sigma);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        int i, j, k;
        field_coords(e, n, P, i, j, k);
        if (i >= n) { out[e] = 0.0f; continue; }
        double x = origin + i * h, y = origin + j * h, z = origin + k * h;
        double acc = -0.0;
        for (int a = 0; a < nn; ++a) {
            double dx = x - nuc[a].x, dy = y - nuc[a].y, dz = z - nuc[a].z;
            acc += nuc[a].Z * norm * exp(-(dx * dx + dy * dy + dz * dz) * inv_2s2);
        }
        out[e] = (float)(acc * scale);
    }
}

// The LCG of crates/qm/src/scf.rs:640, advanced t steps from s0 in O(log t) (affine-map powers).
__device__ __forceinline__ unsigned long long lcg_skip(unsigned long long s0, unsigned long long t) {
    const unsigned long long A = 6364136223846793005ULL, C = 1442695040888963407ULL;
    unsigned long long am = 1, ap = 0, cm = A, cp = C;
    while (t) {
        if (t & 1ULL) { am *= cm; ap = ap * cm + cp; }
        cp = (cm + 1) * cp;
        cm *= cm;
        t >>= 1;
    }
    return am * s0 + ap;
}

__global__ void initial_orbitals_kernel(int n, int P, long long F, double h, double origin, const Nuc* __restrict__ nuc, int nn,
                                        int k, unsigned long long seed, int mode, float* __restrict__ out) {
    const long long total = F * k;
    const long long N = (long long)n * n * n;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        long long v = e / F, f = e % F;
        int i, j, kk;
        field_coords(f, n, P, i, j, kk);
        if (i >= n) { out[e] = 0.0f; continue; }
        long long p = i + (long long)n * (j + (long long)n * kk);
        unsigned long long s = lcg_skip(seed, (unsigned long long)(v * N + p + 1));
        double u = (double)(s >> 11) / 9007199254740992.0;  // 2^53
        double val;
        if (mode == 0) {
            double x = origin + i * h, y = origin + j * h, z = origin + kk * h;
            double env = -0.0;
            for (int a = 0; a < nn; ++a) {
                double dx = x - nuc[a].x, dy = y - nuc[a].y, dz = z - nuc[a].z;
                env += exp(-(dx * dx + dy * dy + dz * dz) / 4.0);
            }
            val = (u + 0.5) * env;
        } else {
            val = 2.0 * u - 1.0;
        }
        out[e] = (float)val;
    }
}

__global__ void pack_kernel(int n, int P, long long F, int count, const double* __restrict__ dense, float* __restrict__ field) {
    const long long N = (long long)n * n * n;
    const long long total = F * count;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        long long v = e / F, f = e % F;
        int i, j, k;
        field_coords(f, n, P, i, j, k);
        field[e] = (i < n) ? (float)dense[v * N + i + (long long)n * (j + (long long)n * k)] : 0.0f;
    }
}

__global__ void unpack_kernel(int n, int P, long long F, int count, const float* __restrict__ field, double* __restrict__ dense) {
    const long long N = (long long)n * n * n;
    const long long total = N * count;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
        long long v = e / N, p = e % N;
        int i = (int)(p % n), j = (int)((p / n) % n), k = (int)(p / ((long long)n * n));
        dense[e] = (double)field[v * F + ((long long)k * n + j) * P + i];
    }
}

__global__ void fill_kernel(float* out, float value, long long count) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count; e += (long long)gridDim.x * blockDim.x)
        out[e] = value;
}

// ------------------------------------------------------------------ pointwise arithmetic
__global__ void lincomb_kernel(long long n4, float4* __restrict__ y, Terms t) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n4; e += (long long)gridDim.x * blockDim.x) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int q = 0; q < t.count; ++q) {
            float4 v = reinterpret_cast<const float4*>(t.x[q])[e];
            float c = t.c[q];
            acc.x = fmaf(c, v.x, acc.x);
            acc.y = fmaf(c, v.y, acc.y);
            acc.z = fmaf(c, v.z, acc.z);
            acc.w = fmaf(c, v.w, acc.w);
        }
        y[e] = acc;
    }
}

// out_j = sum_i C_ij S_i for up to QG outputs per CTA row (blockIdx.y picks the output group). The CTA
// stages its slice of the m inputs (LCB float4 of each field, m x 2 KB: at most 128 KB for m = 64) in
// shared memory with one cp.async.bulk per field, all completing on one mbarrier, so the whole slice is
// in flight at once without holding registers; each thread then combines its float4 with packed f32x2
// FMAs, in input order: the same roundings as one fmaf chain per output element.
// m = 24, q = 16 at 95^3: the whole H2O solve 1.7 % faster than loading the inputs four at a time
// through registers (bitwise-identical results). The FMA pairs are two OUTPUTS of one component,
// (c_ij, c_ij+1) x (v_k, v_k), so one 16-byte shared load brings four coefficients: 5 shared loads per
// input instead of 17 (coefficient pairs (c, c) per output), 37.6 instead of 47.3 us per launch.
constexpr int QG = 16;
constexpr int LCB = 128;  // float4 per field per CTA = threads per CTA
constexpr long long LC_WAIT_LIMIT = 1LL << 22;
__device__ __forceinline__ unsigned long long lc_fma2(unsigned long long a, unsigned long long b, unsigned long long c) {
    unsigned long long d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ unsigned lc_su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__global__ void __launch_bounds__(LCB) block_lincomb_kernel(long long F4, int m, const ulonglong2* __restrict__ S, int q,
                                                            const double* __restrict__ C, ulonglong2* __restrict__ out, int split,
                                                            int gap, int* err) {
    extern __shared__ __align__(128) ulonglong2 sv[];  // m x LCB
    __shared__ __align__(16) float cs[64 * QG];        // c_ij at [i][jj], zero past the group's last output
    __shared__ __align__(8) uint64_t bar;
    const long long e0 = (long long)blockIdx.x * LCB;
    const int cnt = (int)min((long long)LCB, F4 - e0);  // >= 1: the grid is ceil(F4 / LCB)
    const unsigned bytes = (unsigned)cnt * 16u;          // a multiple of 16, from 16-byte aligned field rows
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lc_su32(&bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        if (threadIdx.x == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(lc_su32(&bar)), "r"(bytes * (unsigned)m)
                         : "memory");
        __syncwarp();
        for (int i = threadIdx.x; i < m; i += 32)
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                             lc_su32(sv + (size_t)i * LCB)),
                         "l"(S + (long long)i * F4 + e0), "r"(bytes), "r"(lc_su32(&bar))
                         : "memory");
    }
    // the coefficients while the copies are in flight
    const int j0 = blockIdx.y * QG;
    const int qn = min(QG, q - j0);
    for (int t = threadIdx.x; t < m * QG; t += blockDim.x) {
        const int i = t / QG, jj = t % QG;
        cs[t] = jj < qn ? (float)C[i + (size_t)m * (j0 + jj)] : 0.0f;
    }
    __syncthreads();
    // bounded wait on the copies: on timeout the error flag is raised (the host's next readback reports it) and the
    // outputs are undefined; a second bounded wait then gives the copies in flight time to land before the CTA exits
    // and its shared memory is reused
    auto wait_copies = [&](long long limit) {
        for (long long n = 0;; ++n) {
            unsigned ok;
            asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                         : "=r"(ok)
                         : "r"(lc_su32(&bar))
                         : "memory");
            if (ok) return true;
            if (n > limit) return false;
        }
    };
    if (!wait_copies(LC_WAIT_LIMIT)) {
        if (err) atomicExch(err, 1);
        wait_copies(1LL << 16);
    }
    const int tid = threadIdx.x;
    if (tid >= cnt) return;
    // acc[p][k]: component k of outputs (2p, 2p + 1)
    unsigned long long acc[QG / 2][4];
#pragma unroll
    for (int p = 0; p < QG / 2; ++p) acc[p][0] = acc[p][1] = acc[p][2] = acc[p][3] = 0ull;
    const float4* sv4 = reinterpret_cast<const float4*>(sv);
    const ulonglong2* cs4 = reinterpret_cast<const ulonglong2*>(cs);
#pragma unroll 4
    for (int i = 0; i < m; ++i) {
        const float4 v = sv4[(size_t)i * LCB + tid];
        unsigned long long vv[4];  // (v.k, v.k)
        asm("mov.b64 %0, {%1, %1};" : "=l"(vv[0]) : "f"(v.x));
        asm("mov.b64 %0, {%1, %1};" : "=l"(vv[1]) : "f"(v.y));
        asm("mov.b64 %0, {%1, %1};" : "=l"(vv[2]) : "f"(v.z));
        asm("mov.b64 %0, {%1, %1};" : "=l"(vv[3]) : "f"(v.w));
#pragma unroll
        for (int p4 = 0; p4 < QG / 4; ++p4) {
            if (4 * p4 < qn) {
                const ulonglong2 c4 = cs4[i * (QG / 4) + p4];  // (c_4p4, c_4p4+1), (c_4p4+2, c_4p4+3)
#pragma unroll
                for (int k = 0; k < 4; ++k) acc[2 * p4][k] = lc_fma2(c4.x, vv[k], acc[2 * p4][k]);
                if (4 * p4 + 2 < qn) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) acc[2 * p4 + 1][k] = lc_fma2(c4.y, vv[k], acc[2 * p4 + 1][k]);
                }
            }
        }
    }
    const long long e = e0 + tid;
#pragma unroll
    for (int p = 0; p < QG / 2; ++p) {
        unsigned lo[4], hi[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) asm("mov.b64 {%0, %1}, %2;" : "=r"(lo[k]), "=r"(hi[k]) : "l"(acc[p][k]));
        const int ja = j0 + 2 * p, jb = ja + 1;
        if (2 * p < qn)
            out[(long long)(ja < split ? ja : ja + gap) * F4 + e] =
                make_ulonglong2(lo[0] | ((unsigned long long)lo[1] << 32), lo[2] | ((unsigned long long)lo[3] << 32));
        if (2 * p + 1 < qn)
            out[(long long)(jb < split ? jb : jb + gap) * F4 + e] =
                make_ulonglong2(hi[0] | ((unsigned long long)hi[1] << 32), hi[2] | ((unsigned long long)hi[3] << 32));
    }
}

__global__ void residual_precond_kernel(long long F4, const float4* HX, const float4* __restrict__ X,
                                        const double* __restrict__ theta, const float4* __restrict__ V,
                                        const double* __restrict__ lambda, float diag_t, float4* __restrict__ R,
                                        float4* __restrict__ W0, double* __restrict__ partials, float omega, float4* Dinv) {
    const int v = blockIdx.y;
    const double th = theta[v];
    const float hi = (float)th;
    const float lo = (float)(th - (double)hi);
    const float lam = (float)lambda[v];
    const long long off = (long long)v * F4;
    double acc = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F4; e += (long long)gridDim.x * blockDim.x) {
        float4 hx = HX[off + e], x = X[off + e], vv = V[e];
        float4 r;
        r.x = fmaf(-lo, x.x, fmaf(-hi, x.x, hx.x));
        r.y = fmaf(-lo, x.y, fmaf(-hi, x.y, hx.y));
        r.z = fmaf(-lo, x.z, fmaf(-hi, x.z, hx.z));
        r.w = fmaf(-lo, x.w, fmaf(-hi, x.w, hx.w));
        R[off + e] = r;
        float4 w;
        w.x = r.x / fmaxf(diag_t + vv.x - lam, 0.1f);
        w.y = r.y / fmaxf(diag_t + vv.y - lam, 0.1f);
        w.z = r.z / fmaxf(diag_t + vv.z - lam, 0.1f);
        w.w = r.w / fmaxf(diag_t + vv.w - lam, 0.1f);
        W0[off + e] = w;
        if (Dinv) {  // the later sweeps' factor, as they compute it (HX[off + e] was read above: Dinv may be HX)
            float4 d;
            d.x = omega * (1.0f / fmaxf(diag_t + vv.x - lam, 0.1f));
            d.y = omega * (1.0f / fmaxf(diag_t + vv.y - lam, 0.1f));
            d.z = omega * (1.0f / fmaxf(diag_t + vv.z - lam, 0.1f));
            d.w = omega * (1.0f / fmaxf(diag_t + vv.w - lam, 0.1f));
            Dinv[off + e] = d;
        }
        acc += (double)r.x * r.x + (double)r.y * r.y + (double)r.z * r.z + (double)r.w * r.w;
    }
    double s = block_sum(acc);
    if (threadIdx.x == 0) partials[(size_t)blockIdx.x * gridDim.y + v] = s;
}

// ---- LSDA in f64 (crates/qm/src/xc.rs:88-207): cube roots by cbrt, n^(4/3) = n cbrt(n)
struct Pw92 { double a, a1, b1, b2, b3, b4; };
__device__ __forceinline__ void pw92_g(double rs, double srs, const Pw92 p, double& G, double& dG) {
    double q0 = -2.0 * p.a * (1.0 + p.a1 * rs);
    double q1 = 2.0 * p.a * (p.b1 * srs + p.b2 * rs + p.b3 * rs * srs + p.b4 * rs * rs);
    double q1p = p.a * (p.b1 / srs + 2.0 * p.b2 + 3.0 * p.b3 * srs + 4.0 * p.b4 * rs);
    double ln = log1p(1.0 / q1);
    G = q0 * ln;
    dG = -2.0 * p.a * p.a1 * ln - q0 * q1p / (q1 * q1 + q1);
}

__device__ __forceinline__ void lsda_point(double nu, double nd, double& e, double& vu, double& vd) {
    const double PI = 3.14159265358979323846;
    nu = fmax(nu, 0.0);
    nd = fmax(nd, 0.0);
    double n = nu + nd;
    if (n < 1e-20) { e = vu = vd = 0.0; return; }
    // exchange
    const double cx = 0.75 * cbrt(3.0 / PI) * cbrt(2.0);
    double cu = cbrt(nu), cd = cbrt(nd);
    double ex = -cx * (nu * cu + nd * cd);
    const double c6 = cbrt(6.0 / PI);
    double vxu = -c6 * cu, vxd = -c6 * cd;
    // correlation
    const Pw92 PARA = {0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294};
    const Pw92 FERRO = {0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517};
    const Pw92 MALPHA = {0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671};
    const double FPP0 = 1.709921;
    double rs = cbrt(3.0 / (4.0 * PI * n));
    double srs = sqrt(rs);
    double z = fmin(fmax((nu - nd) / n, -1.0), 1.0);
    double ec0, dec0, ec1, dec1, mac, dmac;
    pw92_g(rs, srs, PARA, ec0, dec0);
    pw92_g(rs, srs, FERRO, ec1, dec1);
    pw92_g(rs, srs, MALPHA, mac, dmac);
    double ac = -mac, dac = -dmac;
    const double denom = 2.0 * cbrt(2.0) - 2.0;
    double cp = cbrt(1.0 + z), cm = cbrt(1.0 - z);
    double f = ((1.0 + z) * cp + (1.0 - z) * cm - 2.0) / denom;
    double fp = (4.0 / 3.0) * (cp - cm) / denom;
    double z3 = z * z * z, z4 = z3 * z;
    double ec = ec0 + ac * f / FPP0 * (1.0 - z4) + (ec1 - ec0) * f * z4;
    double dec_drs = dec0 + dac * f / FPP0 * (1.0 - z4) + (dec1 - dec0) * f * z4;
    double dec_dz = ac / FPP0 * (fp * (1.0 - z4) - 4.0 * z3 * f) + (ec1 - ec0) * (fp * z4 + 4.0 * z3 * f);
    double common = ec - rs / 3.0 * dec_drs;
    e = ex + n * ec;
    vu = vxu + (common - (z - 1.0) * dec_dz);
    vd = vxd + (common - (z + 1.0) * dec_dz);
}

__global__ void xc_veff_kernel(long long F, const float* __restrict__ up, const float* __restrict__ dn,
                               const float* __restrict__ vnuc, const float* __restrict__ vh, float* __restrict__ exc,
                               float* __restrict__ vup, float* __restrict__ vdn, float* __restrict__ xcu, float* __restrict__ xcd,
                               const float* __restrict__ pc) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        double en, vu, vd;
        double nu = (double)up[e], nd = (double)dn[e];
        if (pc) {  // the unpolarised partial core, half per spin (crates/qm/src/scf.rs:759-768)
            const double c = 0.5 * (double)pc[e];
            nu += c;
            nd += c;
        }
        lsda_point(nu, nd, en, vu, vd);
        exc[e] = (float)en;
        if (vup) {
            double base = (double)vnuc[e] + (double)vh[e];
            vup[e] = (float)(base + vu);
            vdn[e] = (float)(base + vd);
        }
        if (xcu) { xcu[e] = (float)vu; xcd[e] = (float)vd; }
    }
}

__global__ void density_residual_kernel(long long F4, int k, const float4* __restrict__ psi, const double* __restrict__ f,
                                        const float4* __restrict__ rin, float4* __restrict__ rout, float4* __restrict__ r,
                                        double* __restrict__ partials) {
    double sabs = 0.0, ssum = 0.0;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F4; e += (long long)gridDim.x * blockDim.x) {
        float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);
        for (int i = 0; i < k; ++i) {
            float4 p = psi[(long long)i * F4 + e];
            float w = f ? (float)f[i] : 1.0f;
            acc.x = fmaf(w * p.x, p.x, acc.x);
            acc.y = fmaf(w * p.y, p.y, acc.y);
            acc.z = fmaf(w * p.z, p.z, acc.z);
            acc.w = fmaf(w * p.w, p.w, acc.w);
        }
        float4 in = rin[e];
        rout[e] = acc;
        float4 d = make_float4(acc.x - in.x, acc.y - in.y, acc.z - in.z, acc.w - in.w);
        r[e] = d;
        sabs += (double)fabsf(d.x) + (double)fabsf(d.y) + (double)fabsf(d.z) + (double)fabsf(d.w);
        ssum += (double)acc.x + (double)acc.y + (double)acc.z + (double)acc.w;
    }
    double a = block_sum(sabs);
    double b = block_sum(ssum);
    if (threadIdx.x == 0) { partials[2 * blockIdx.x] = a; partials[2 * blockIdx.x + 1] = b; }
}

struct DiisPtrs {
    static constexpr int MAX = 16;
    const float* rho[MAX];
    const float* r[MAX];
    float c[MAX];
    float a[MAX];
};

__global__ void diis_mix_kernel(long long F, int m, DiisPtrs d, float* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x) {
        float base = d.rho[m - 1][e];
        double small = 0.0;
        for (int i = 0; i < m - 1; ++i) small += (double)d.c[i] * (double)(d.rho[i][e] - base);
        for (int i = 0; i < m; ++i) small += (double)d.a[i] * (double)d.r[i][e];
        float v = (float)((double)base + small);
        out[e] = fmaxf(v, 0.0f);
    }
}

__global__ void scale_kernel(long long n4, float4* x, float a) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n4; e += (long long)gridDim.x * blockDim.x) {
        float4 v = x[e];
        v.x *= a; v.y *= a; v.z *= a; v.w *= a;
        x[e] = v;
    }
}

__global__ void scale_ratio_kernel(long long n4, float4* x, const double* sum, double target) {
    const double s = *sum;
    if (!(s > 0.0 && target > 0.0)) return;
    const float a = (float)(target / s);
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n4; e += (long long)gridDim.x * blockDim.x) {
        float4 v = x[e];
        v.x *= a; v.y *= a; v.z *= a; v.w *= a;
        x[e] = v;
    }
}

}  // namespace

void launch_scale_ratio(long long F, float* x, const double* sum_dev, double target, cudaStream_t s) {
    scale_ratio_kernel<<<stream_blocks(F / 4), TPB, 0, s>>>(F / 4, reinterpret_cast<float4*>(x), sum_dev, target);
    KS_LAUNCH_CHECK();
}

void launch_nuclear_potential(const Layout& L, const Nuc* nuc, int nn, double sigma, float* out, cudaStream_t s) {
    nuclear_potential_kernel<<<stream_blocks(L.F), TPB, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, nuc, nn, sigma, out);
    KS_LAUNCH_CHECK();
}

void launch_deposit_charge(const Layout& L, const Nuc* nuc, int nn, double sigma, double scale, float* out, cudaStream_t s) {
    deposit_charge_kernel<<<stream_blocks(L.F), TPB, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, nuc, nn, sigma, scale, out);
    KS_LAUNCH_CHECK();
}

void launch_initial_orbitals(const Layout& L, const Nuc* nuc, int nn, int k, unsigned long long seed, int mode, float* out,
                             cudaStream_t s) {
    if (k <= 0) return;
    initial_orbitals_kernel<<<stream_blocks(L.F * k), TPB, 0, s>>>(L.n, L.P, L.F, L.h, L.origin, nuc, nn, k, seed, mode, out);
    KS_LAUNCH_CHECK();
}

void launch_pack(const Layout& L, int count, const double* dense, float* field, cudaStream_t s) {
    if (count <= 0) return;
    pack_kernel<<<stream_blocks(L.F * count), TPB, 0, s>>>(L.n, L.P, L.F, count, dense, field);
    KS_LAUNCH_CHECK();
}

void launch_unpack(const Layout& L, int count, const float* field, double* dense, cudaStream_t s) {
    if (count <= 0) return;
    unpack_kernel<<<stream_blocks(L.interior() * count), TPB, 0, s>>>(L.n, L.P, L.F, count, field, dense);
    KS_LAUNCH_CHECK();
}

void launch_fill(float* out, float value, long long count, cudaStream_t s) {
    if (count <= 0) return;
    fill_kernel<<<stream_blocks(count), TPB, 0, s>>>(out, value, count);
    KS_LAUNCH_CHECK();
}

void launch_lincomb(long long F, int count, float* y, const Terms& t, cudaStream_t s) {
    long long n4 = F * count / 4;
    if (n4 <= 0) return;
    // every term advances with the output block: term pointers are block bases with the same stride
    lincomb_kernel<<<stream_blocks(n4), TPB, 0, s>>>(n4, reinterpret_cast<float4*>(y), t);
    KS_LAUNCH_CHECK();
}

void launch_block_lincomb(long long F, int m, const float* S, int q, const double* C, float* out, int split, int gap, cudaStream_t s) {
    if (q <= 0) return;
    if (m > 64) throw std::invalid_argument("block_lincomb: at most 64 input fields");
    // the bulk copies need 16-byte aligned sources and sizes: whole float4 rows of 16-byte aligned fields
    if (F % 4 != 0 || reinterpret_cast<uintptr_t>(S) % 16 != 0 || reinterpret_cast<uintptr_t>(out) % 16 != 0)
        throw std::invalid_argument("block_lincomb: fields must be 16-byte aligned with F a multiple of 4 floats");
    long long F4 = F / 4;
    static std::atomic<unsigned long long> attr_set{0};
    once_per_device(attr_set, [] {  // 64 fields x LCB float4 of dynamic shared memory at most
        KS_CUDA(cudaFuncSetAttribute(block_lincomb_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 64 * LCB * 16));
    });
    dim3 grid((unsigned)((F4 + LCB - 1) / LCB), ceil_div(q, QG));
    block_lincomb_kernel<<<grid, LCB, (size_t)m * LCB * 16, s>>>(F4, m, reinterpret_cast<const ulonglong2*>(S), q, C,
                                                                 reinterpret_cast<ulonglong2*>(out), split, gap, device_error_flag());
    KS_LAUNCH_CHECK();
}

void launch_residual_precond(const Layout& L, int k, const float* HX, const float* X, const double* theta, const float* V,
                             const double* lambda, double diag_t, float* R, float* W0, double* partials, int blocks, cudaStream_t s,
                             float omega, float* dinv) {
    dim3 grid(blocks, k);
    residual_precond_kernel<<<grid, TPB, 0, s>>>(L.F / 4, reinterpret_cast<const float4*>(HX), reinterpret_cast<const float4*>(X),
                                                 theta, reinterpret_cast<const float4*>(V), lambda, (float)diag_t,
                                                 reinterpret_cast<float4*>(R), reinterpret_cast<float4*>(W0), partials, omega,
                                                 reinterpret_cast<float4*>(dinv));
    KS_LAUNCH_CHECK();
}

void launch_xc_veff(long long F, const float* up, const float* dn, const float* vnuc, const float* vh, float* exc, float* vup,
                    float* vdn, float* vxc_up, float* vxc_dn, cudaStream_t s, const float* pc) {
    xc_veff_kernel<<<stream_blocks(F), TPB, 0, s>>>(F, up, dn, vnuc, vh, exc, vup, vdn, vxc_up, vxc_dn, pc);
    KS_LAUNCH_CHECK();
}

void launch_density_residual(long long F, int k, const float* psi, const double* f, const float* rho_in, float* rho_out, float* r,
                             double* partials, int blocks, cudaStream_t s) {
    density_residual_kernel<<<blocks, TPB, 0, s>>>(F / 4, k, reinterpret_cast<const float4*>(psi), f,
                                                   reinterpret_cast<const float4*>(rho_in), reinterpret_cast<float4*>(rho_out),
                                                   reinterpret_cast<float4*>(r), partials);
    KS_LAUNCH_CHECK();
}

void launch_diis_mix(long long F, int m, const float* const* rho, const float* const* r, const float* c, const float* a,
                     float* out, cudaStream_t s) {
    if (m < 1 || m > DiisPtrs::MAX) throw std::invalid_argument("diis_mix: 1..16 entries");
    DiisPtrs d;
    for (int i = 0; i < m; ++i) { d.rho[i] = rho[i]; d.r[i] = r[i]; d.c[i] = c[i]; d.a[i] = a[i]; }
    diis_mix_kernel<<<stream_blocks(F), TPB, 0, s>>>(F, m, d, out);
    KS_LAUNCH_CHECK();
}

// out = max(2 cur - prev, 0) (crates/qm-gpu/src/scf.rs:1146-1163, the density extrapolation in time)
__global__ void extrapolate_kernel(long long F, const float* __restrict__ cur, const float* __restrict__ prev, float* __restrict__ out) {
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < F; e += (long long)gridDim.x * blockDim.x)
        out[e] = fmaxf(2.0f * cur[e] - prev[e], 0.0f);
}

void launch_extrapolate(long long F, const float* cur, const float* prev, float* out, cudaStream_t s) {
    extrapolate_kernel<<<stream_blocks(F), TPB, 0, s>>>(F, cur, prev, out);
    KS_LAUNCH_CHECK();
}

void launch_scale(long long F, float* x, float a, cudaStream_t s) {
    scale_kernel<<<stream_blocks(F / 4), TPB, 0, s>>>(F / 4, reinterpret_cast<float4*>(x), a);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
