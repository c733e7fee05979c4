// k_stencil.cu -- the 8th-order finite-difference stencil family on sm_100a: Laplacian, H psi
// (-1/2 lap + V psi) and the fused damped-Jacobi sweep of the LOBPCG preconditioner.
//
// Reference operators: crates/qm/src/stencil.rs:21-51 (coefficients c = [-205/72, 8/5, -1/5,
// 8/315, -1/560], Dirichlet zero outside the box), crates/qm-gpu/src/shaders/stencil.wgsl:58-106
// (hamiltonian, jacobi_step). The centre is folded into second differences,
//     lap f = s sum_{m=1..4} c_m sum_axes [(f_{+m} - f_0) + (f_{-m} - f_0)],
// exact in real arithmetic because c_0 = -2 sum c_m, and exact per difference in f32 for smooth f (the
// differences carry no rounding, which keeps the f32 residual floor of the reference's stop rules). s is the
// operator's scale (1/h^2, or -1/(2 h^2) for H); smallest coefficients first.
//
// B200 design ("2.5-D" tiling): a CTA owns a 32 x 16 (x, y) tile of one field and marches a z-chunk. Each z-plane
// of the tile plus its 4-point xy halo (40 x 24 floats) is staged in shared memory by one TMA load
// (cp.async.bulk.tensor.4d); the tensor map's extent is n on every axis, so the halo beyond the box arrives as the
// hardware's zero fill -- the Dirichlet boundary costs no branches and no ghost storage. An 8-deep ring of planes
// keeps four planes of prefetch in flight. Each of the 128 threads owns four consecutive x-outputs of one row: it
// reads its centre, x- and y-neighbours as 16-byte quads (11 shared loads per 4 outputs), keeps the nine z-values of
// its quad in a register queue that moves up one plane per step, and computes the two packed pairs of the quad with
// Blackwell's f32x2 arithmetic. A neighbour pair that straddles two quads (odd x offsets) is differenced with two
// scalar subtractions instead of being repacked. The V / R reads (cp.async copies one plane ahead into a small shared
// ring) and the stores are coalesced 16-byte accesses;
// the quad's pad columns are stored as 0. Measured against the 2 x 2-outputs-per-thread form it replaces: the same
// outputs bit for bit at h = 0.25, and H psi on 95^3 at 8 / 16 / 64 vectors 13 / 13 / 21 % faster.
#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <cudaTypedefs.h>
#include "kernels.cuh"
#include "reduce_util.cuh"

namespace ks {

namespace {

typedef unsigned long long u64;

constexpr int BX = 32, BY = 16;
constexpr int HXW = BX + 8, HYW = BY + 8;          // staged plane with halo: 40 x 24
constexpr int NS = 8;                               // ring depth (planes)
constexpr int PLANE_FLOATS = HXW * HYW;             // 960
constexpr unsigned PLANE_BYTES = PLANE_FLOATS * 4;  // 3840 = 30 * 128
constexpr int THREADS = 128;                        // 8 x-quads * 16 rows
// The TMA rules the plane loads rely on, checked here because a violation faults the GPU instead of returning an
// error: the box's inner extent is a multiple of 16 bytes; a load's x coordinate, x0 - 4 with x0 a multiple of BX,
// times 4 bytes is a multiple of 16 (negative x is allowed for loads and reads the zero fill); each ring plane starts
// on a 128-byte boundary. The quads the threads read start on 16-byte boundaries: rows of HXW floats, quads at
// 4 * tx + 4 (and +-4 for the x-neighbours). The z-queue issues plane s + 12 into the buffer plane s + 4 left, which
// needs NS = 8.
static_assert((HXW * 4) % 16 == 0, "TMA box inner extent must be a multiple of 16 bytes");
static_assert((BX * 4) % 16 == 0 && (4 * 4) % 16 == 0, "TMA x coordinate x0 - 4 must be a multiple of 16 bytes");
static_assert(PLANE_BYTES % 128 == 0, "ring planes must start on 128-byte boundaries");
static_assert(NS == 8, "plane s + 12 reuses the buffer of plane s + 4 only with an 8-deep ring");
static_assert(THREADS == (BX / 4) * BY, "one thread per x-quad of a row");
// resident CTAs per SM: registers capped at 96 per thread (no spills) for 20 warps per SM; 4 and 6 CTAs per SM
// measured slower (H psi on 95^3: 4 CTAs 182 us at 64 vectors, 6 CTAs 144 us, against 137 us at 5)
constexpr int CTAS_PER_SM = 5;
// The per-plane global reads of a step (V; r and the stored factor in the Jacobi mode) are staged one plane ahead by
// per-thread cp.async copies into a 2-deep shared "side" ring (12 KB per CTA in the Jacobi mode, 4 KB for H and the
// residual form), so their latency runs behind the previous plane's arithmetic without holding registers. Against
// register loads at the step that uses them: the H2O 95^3 solve 176.5 -> 172.3 ms, Jacobi sweep 34.0 -> 33.0 us,
// bitwise-identical results. Three planes ahead, or V left to the L2 in the Jacobi mode, measured slower.
constexpr int SD = 2;
template <int MODE>
constexpr int n_side() { return MODE == ST_JACOBI ? 3 : (MODE == ST_LAPLACIAN ? 0 : 1); }
__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }
constexpr long long WAIT_LIMIT = 1LL << 22;         // bounded mbarrier waits (~seconds)
constexpr long long DRAIN_LIMIT = 1LL << 16;        // waits for copies in flight after a wait gave up

constexpr float C1 = 1.6f, C2 = -0.2f, C3 = 0.025396825396825397f, C4 = -0.0017857142857142857f;
#ifndef KS_FOLD_SCALE
#define KS_FOLD_SCALE 0
#endif
constexpr bool FOLD_SCALE = KS_FOLD_SCALE != 0;

struct Params {
    int n, P;
    long long F;
    int tiles_x, tiles_y, zc;
    float scale, omega, diag_t;
    const float* V;
    const float* R;
    const double* lambda;
    double* dot_partials;
    int* err;
    int vec0;
    const double* theta;
    float* out2;
    float* dinv;
};

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: false (and the error flag raised) when the copy did not complete within `limit` polls.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int* err, long long limit = WAIT_LIMIT) {
    long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > limit) {
            if (err) atomicExch(err, 1);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void tma_load_plane(float* dst, const CUtensorMap* map, int x, int y, int z, int v, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(v), "r"(smem_u32(bar))
        : "memory");
}

// ---- packed f32x2 arithmetic (sm_100): one instruction for two x-neighbours
__device__ __forceinline__ u64 add2(u64 a, u64 b) { u64 d; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ u64 sub2(u64 a, u64 b) { u64 d; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ u64 mul2(u64 a, u64 b) { u64 d; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
    u64 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ u64 pk(float lo, float hi) {
    u64 d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ float lo_of(u64 v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float hi_of(u64 v) { return __uint_as_float((unsigned)(v >> 32)); }
__device__ __forceinline__ float4 lds4(const float* p) { return *reinterpret_cast<const float4*>(p); }
// (a0 - f0.lo, a1 - f0.hi)
__device__ __forceinline__ u64 dif(float a0, float a1, u64 f0) { return sub2(pk(a0, a1), f0); }

// sum_m (c_m s) d_m of the thread's quad, as two packed pairs (x0, x0+1) and (x0+2, x0+3). cpl: the quad's address
// in the centre plane (x-neighbour quads at -4 / +4, y-neighbours at +-m*HXW); q: the z-queue, q[4] the centre.
// The y-neighbour quads are loaded inside the m loop, largest m first, so that only two are live at a time.
__device__ __forceinline__ void lap_quad(const float* cpl, const float4 (&q)[9], const u64 (&k)[5], u64& o0, u64& o1) {
    const float4 c = q[4];
    const float4 l = lds4(cpl - 4), r = lds4(cpl + 4);
    const float xs[12] = {l.x, l.y, l.z, l.w, c.x, c.y, c.z, c.w, r.x, r.y, r.z, r.w};
    const u64 f0[2] = {pk(c.x, c.y), pk(c.z, c.w)};
    u64 acc[2];
#pragma unroll
    for (int m = 4; m >= 1; --m) {
        const float4 yu = lds4(cpl + m * HXW), yd = lds4(cpl - m * HXW);
        const float4& zu = q[4 + m];
        const float4& zd = q[4 - m];
#pragma unroll
        for (int p = 0; p < 2; ++p) {
            const int b = 4 + 2 * p;  // the pair's first element in xs
            u64 dx;
            if (m & 1) {
                // odd offsets straddle two quads: two scalar differences instead of a repacked pair
                const float a0 = xs[b + m] - lo_of(f0[p]), a1 = xs[b + 1 + m] - hi_of(f0[p]);
                const float b0 = xs[b - m] - lo_of(f0[p]), b1 = xs[b + 1 - m] - hi_of(f0[p]);
                dx = add2(pk(a0, a1), pk(b0, b1));
            } else {
                dx = add2(dif(xs[b + m], xs[b + 1 + m], f0[p]), dif(xs[b - m], xs[b + 1 - m], f0[p]));
            }
            u64 dy, dz;
            if (p == 0) {
                dy = add2(dif(yu.x, yu.y, f0[0]), dif(yd.x, yd.y, f0[0]));
                dz = add2(dif(zu.x, zu.y, f0[0]), dif(zd.x, zd.y, f0[0]));
            } else {
                dy = add2(dif(yu.z, yu.w, f0[1]), dif(yd.z, yd.w, f0[1]));
                dz = add2(dif(zu.z, zu.w, f0[1]), dif(zd.z, zd.w, f0[1]));
            }
            const u64 d = add2(add2(dx, dy), dz);
            acc[p] = (m == 4) ? mul2(k[4], d) : fma2(k[m], d, acc[p]);
        }
    }
    o0 = acc[0];
    o1 = acc[1];
}

// f64 sum of f0 * o over the valid elements of a quad (the Poisson p.Ap and the kinetic <psi, lap psi>)
__device__ __forceinline__ double quad_dot(const float4& f, u64 o0, u64 o1, bool e1, bool e2, bool e3) {
    double d = (double)f.x * (double)lo_of(o0);
    if (e1) d += (double)f.y * (double)hi_of(o0);
    if (e2) d += (double)f.z * (double)lo_of(o1);
    if (e3) d += (double)f.w * (double)hi_of(o1);
    return d;
}

template <int MODE, bool DOT>
__global__ void __launch_bounds__(THREADS, CTAS_PER_SM) stencil_kernel(const __grid_constant__ CUtensorMap tmap, Params p, float* __restrict__ out) {
    extern __shared__ __align__(1024) float ring[];  // NS planes of 40 x 24
    __shared__ __align__(8) uint64_t bar[NS];

    const int vec = blockIdx.y;
    int b = blockIdx.x;
    const int tile_x = b % p.tiles_x;
    b /= p.tiles_x;
    const int tile_y = b % p.tiles_y;
    const int chunk = b / p.tiles_y;
    const int x0 = tile_x * BX, y0 = tile_y * BY;
    const int z0 = chunk * p.zc;
    const int nz = min(z0 + p.zc, p.n) - z0;
    const int nplanes = nz + 8;  // relative plane q <-> z = z0 - 4 + q
    const int tx = threadIdx.x & 7, ty = threadIdx.x >> 3;
    const int gx = x0 + 4 * tx, gy = y0 + ty;
    // the quad's elements inside the box (gx is a multiple of 4 below n <= P, so the whole quad lies inside the
    // row's P floats; elements at or past n are pad columns and are stored as 0)
    const bool ok = gx < p.n && gy < p.n;
    const bool e1 = gx + 1 < p.n, e2 = gx + 2 < p.n, e3 = gx + 3 < p.n;
    const int ci = (ty + 4) * HXW + 4 * tx + 4;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) mbar_init(&bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int q) {
        const int bb = q % NS;
        mbar_expect_tx(&bar[bb], PLANE_BYTES);
        tma_load_plane(ring + bb * PLANE_FLOATS, &tmap, x0 - 4, y0 - 4, z0 - 4 + q, p.vec0 + vec, &bar[bb]);
    };
    // A wait that gives up raises the error flag and marks the thread dead: a dead thread waits no longer than a poll
    // for later planes, thread 0 issues no further loads once dead, and before exiting thread 0 waits a bounded time
    // for its copies still in flight. The CTA's outputs are then undefined (the host reports the error).
    int issued = 0;  // planes issued so far (thread 0's count)
    if (threadIdx.x == 0)
        for (; issued < min(NS, nplanes); ++issued) issue(issued);

    float4 q[9];
    bool alive = true;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        alive = mbar_wait(&bar[i], 0, p.err, alive ? WAIT_LIMIT : 1) && alive;
        q[i] = lds4(ring + i * PLANE_FLOATS + ci);
    }
    __syncthreads();  // planes 0..3 are consumed: their buffers take planes 8..11
    if (alive && threadIdx.x == 0)
        for (; issued < min(NS + 4, nplanes); ++issued) issue(issued);

    // the coefficients; with FOLD_SCALE the operator's scale is folded into them, else it multiplies the sum (the
    // same bits when the scale is a power of two)
    u64 kc[5];
    const float ks = FOLD_SCALE ? p.scale : 1.0f;
    kc[0] = 0;
    kc[1] = pk(C1 * ks, C1 * ks);
    kc[2] = pk(C2 * ks, C2 * ks);
    kc[3] = pk(C3 * ks, C3 * ks);
    kc[4] = pk(C4 * ks, C4 * ks);
    const u64 scale2 = pk(p.scale, p.scale);
    const float lam = (MODE == ST_JACOBI || MODE == ST_HAM_RESIDUAL) ? (float)p.lambda[vec] : 0.0f;
    // theta split into f32 hi + lo, as the residual kernel does: r = fma(-lo, x, fma(-hi, x, Hx))
    const double th = (MODE == ST_HAM_RESIDUAL) ? p.theta[vec] : 0.0;
    const float th_hi = (float)th, th_lo = (float)(th - (double)th_hi);
    const long long plane = (long long)p.n * p.P;
    const long long row0 = ((long long)z0 * p.n + gy) * p.P + gx;
    const long long vbase = (long long)vec * p.F;
    const float* vrow = p.V ? p.V + row0 : nullptr;
    const float* rrow = p.R ? p.R + vbase + row0 : nullptr;
    float* orow = out + vbase + row0;
    float* orow2 = (MODE == ST_HAM_RESIDUAL) ? p.out2 + vbase + row0 : nullptr;
    float* drow = p.dinv ? p.dinv + vbase + row0 : nullptr;
    // the side ring, [SD][NSIDE][THREADS] float4 after the plane ring: slot t % SD holds this thread's V (r, factor)
    // quads of output plane t. Each thread reads only its own copies, after its own wait_group, and refills a slot
    // only after the step that read it has consumed the values.
    constexpr int NSIDE = n_side<MODE>();
    float4* side = reinterpret_cast<float4*>(ring + NS * PLANE_FLOATS);
    auto side_issue = [&](int t) {
        if (NSIDE > 0) {
            if (ok && t < nz) {
                float4* dst = side + (t % SD) * NSIDE * THREADS + threadIdx.x;
                cp_async16(dst, vrow + t * plane);
                if (MODE == ST_JACOBI) {
                    cp_async16(dst + THREADS, rrow + t * plane);
                    if (drow) cp_async16(dst + 2 * THREADS, drow + t * plane);
                }
            }
            cp_async_commit();  // one group per plane, empty or not, so that wait_group counts planes
        }
    };
#pragma unroll
    for (int t = 0; t < SD - 1; ++t) side_issue(t);
    double dot = 0.0;
    // the compact loop body (not unrolled): unrolled bodies measured slower (the instruction cache)
#pragma unroll 1
    for (int s = 0; s < nz; ++s) {
        const int qn = s + 8;
        alive = mbar_wait(&bar[qn % NS], (unsigned)((qn / NS) & 1), p.err, alive ? WAIT_LIMIT : 1) && alive;
        q[8] = lds4(ring + (qn % NS) * PLANE_FLOATS + ci);
        const float* cpl = ring + ((s + 4) % NS) * PLANE_FLOATS + ci;
        // the next plane's side copies go out before this plane's are read
        const float4 zero4 = make_float4(0.f, 0.f, 0.f, 0.f);
        float4 v = zero4, r = zero4, dq = zero4;
        if (NSIDE > 0) {
            side_issue(s + SD - 1);
            cp_async_wait<SD - 1>();
            const float4* sl = side + (s % SD) * NSIDE * THREADS + threadIdx.x;
            if (ok) v = sl[0];
            if (MODE == ST_JACOBI && ok) r = sl[THREADS];
            if (MODE == ST_JACOBI && ok && drow) dq = sl[2 * THREADS];
        }
        u64 o0, o1;
        lap_quad(cpl, q, kc, o0, o1);
        if (!FOLD_SCALE) {
            o0 = mul2(o0, scale2);
            o1 = mul2(o1, scale2);
        }
        const float4 f = q[4];
        if (MODE != ST_LAPLACIAN) {
            const u64 h0 = fma2(pk(v.x, v.y), pk(f.x, f.y), o0), h1 = fma2(pk(v.z, v.w), pk(f.z, f.w), o1);
            if (MODE == ST_HAMILTONIAN) {
                o0 = h0;
                o1 = h1;
            } else if (MODE == ST_HAM_RESIDUAL) {
                // r = Hx - theta x (hi and lo parts of theta), w0 = r / max(diag_t + V - lambda, 0.1)
                o0 = fma2(pk(-th_lo, -th_lo), pk(f.x, f.y), fma2(pk(-th_hi, -th_hi), pk(f.x, f.y), h0));
                o1 = fma2(pk(-th_lo, -th_lo), pk(f.z, f.w), fma2(pk(-th_hi, -th_hi), pk(f.z, f.w), h1));
                if (ok) {
                    const float w0 = lo_of(o0) / fmaxf(p.diag_t + v.x - lam, 0.1f);
                    const float w1 = hi_of(o0) / fmaxf(p.diag_t + v.y - lam, 0.1f);
                    const float w2 = lo_of(o1) / fmaxf(p.diag_t + v.z - lam, 0.1f);
                    const float w3 = hi_of(o1) / fmaxf(p.diag_t + v.w - lam, 0.1f);
                    *reinterpret_cast<float4*>(orow2 + s * plane) = make_float4(w0, e1 ? w1 : 0.f, e2 ? w2 : 0.f, e3 ? w3 : 0.f);
                    if (drow) {  // the sweeps' factor, as the JACOBI mode computes it
                        const float d0 = p.omega * (1.0f / fmaxf(p.diag_t + v.x - lam, 0.1f));
                        const float d1 = p.omega * (1.0f / fmaxf(p.diag_t + v.y - lam, 0.1f));
                        const float d2 = p.omega * (1.0f / fmaxf(p.diag_t + v.z - lam, 0.1f));
                        const float d3 = p.omega * (1.0f / fmaxf(p.diag_t + v.w - lam, 0.1f));
                        *reinterpret_cast<float4*>(drow + s * plane) = make_float4(d0, e1 ? d1 : 0.f, e2 ? d2 : 0.f, e3 ? d3 : 0.f);
                    }
                }
            } else {
                const u64 nl = pk(-lam, -lam);
                // w + (omega / max(diag_t + V - lambda, 0.1)) (r - (H w - lambda w)), as the scalar sweep (an
                // approximate division measured 2 % faster per solve but moved the NH3 96^3 finite-difference check of
                // the adjoint past its bound: the sweep keeps the IEEE division)
                const u64 u0 = sub2(pk(r.x, r.y), fma2(nl, pk(f.x, f.y), h0));
                const u64 u1 = sub2(pk(r.z, r.w), fma2(nl, pk(f.z, f.w), h1));
                float i0, i1, i2, i3;
                if (drow) {  // the factor stored by the residual pass of this iteration
                    i0 = dq.x;
                    i1 = dq.y;
                    i2 = dq.z;
                    i3 = dq.w;
                } else {
                    i0 = p.omega * (1.0f / fmaxf(p.diag_t + v.x - lam, 0.1f));
                    i1 = p.omega * (1.0f / fmaxf(p.diag_t + v.y - lam, 0.1f));
                    i2 = p.omega * (1.0f / fmaxf(p.diag_t + v.z - lam, 0.1f));
                    i3 = p.omega * (1.0f / fmaxf(p.diag_t + v.w - lam, 0.1f));
                }
                o0 = fma2(pk(i0, i1), u0, pk(f.x, f.y));
                o1 = fma2(pk(i2, i3), u1, pk(f.z, f.w));
            }
        }
        if (ok) {
            *reinterpret_cast<float4*>(orow + s * plane) =
                make_float4(lo_of(o0), e1 ? hi_of(o0) : 0.f, e2 ? lo_of(o1) : 0.f, e3 ? hi_of(o1) : 0.f);
            if (DOT) {
                if (MODE == ST_HAM_RESIDUAL) {
                    const double r0 = lo_of(o0), r1 = hi_of(o0), r2 = lo_of(o1), r3 = hi_of(o1);
                    dot += r0 * r0;
                    if (e1) dot += r1 * r1;
                    if (e2) dot += r2 * r2;
                    if (e3) dot += r3 * r3;
                } else {
                    dot += quad_dot(f, o0, o1, e1, e2, e3);
                }
            }
        }
        __syncthreads();  // the centre plane's buffer is free
        if (alive && threadIdx.x == 0 && s + 12 < nplanes) {
            issue(s + 12);
            issued = s + 13;
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) q[i] = q[i + 1];  // the z-queue moves up one plane
    }
    // after a wait gave up: the latest copy issued into each slot may still be in flight (a parity wait on a slot's
    // latest copy is unambiguous, and returns at once for one that arrived)
    if (threadIdx.x == 0 && !alive)
        for (int qq = max(0, issued - NS); qq < issued; ++qq) mbar_wait(&bar[qq % NS], (unsigned)((qq / NS) & 1), nullptr, DRAIN_LIMIT);
    if (DOT) {
        const double sum = block_sum(dot);
        // [vector][CTA] for the Laplacian / H dots; [CTA][vector] for the residual norms (the residual kernel's layout)
        if (threadIdx.x == 0) {
            if (MODE == ST_HAM_RESIDUAL) p.dot_partials[(size_t)blockIdx.x * gridDim.y + blockIdx.y] = sum;
            else p.dot_partials[blockIdx.x + (size_t)gridDim.x * blockIdx.y] = sum;
        }
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    // resolved once (thread-safe static initialisation)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        cudaDriverEntryPointQueryResult q;
        void* ptr = nullptr;
        KS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !ptr) throw DeviceError("cuTensorMapEncodeTiled is not available");
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }();
    return fn;
}

struct Shape { int tiles_x, tiles_y, chunks, zc; };

// The grid: (x, y) tiles x vectors x z-chunks. A CTA's time is about (its planes + prologue) steps
// whatever else runs (the kernel is latency-bound at CTAS_PER_SM CTAs per SM), and the launch takes
// ceil(CTAs / resident slots) such rounds, so the chunk count minimises waves x (zc + c) with c the
// fixed cost of a chunk in plane steps (its 8 halo planes, partly hidden behind the other resident
// CTAs; c = 8 measured best against 12 and 4). At 95^3 with 5 CTAs per SM this gives 5 chunks of 19
// planes for 8 and 16 vectors (720 and 1440 CTAs) and 3 chunks of 32 planes for 48 and 64 vectors.
Shape shape_for(const Layout& L, int count) {
    Shape sh;
    sh.tiles_x = ceil_div(L.n, BX);
    sh.tiles_y = ceil_div(L.n, BY);
    const long long per_chunk = (long long)sh.tiles_x * sh.tiles_y * count;
    const long long slots = (long long)CTAS_PER_SM * sm_count();
    long long best = -1;
    for (int c = 1; c <= std::max(1, L.n / 8); ++c) {
        const int zc = ceil_div(L.n, c);
        const int cc = ceil_div(L.n, zc);
        const long long waves = (cc * per_chunk + slots - 1) / slots;
        const long long cost = waves * (zc + 8);
        if (best < 0 || cost < best) {
            best = cost;
            sh.zc = zc;
            sh.chunks = cc;
        }
    }
    return sh;
}

// the shape of a launch with c z-chunks per tile column
Shape shape_with_chunks(const Layout& L, int c) {
    Shape sh;
    sh.tiles_x = ceil_div(L.n, BX);
    sh.tiles_y = ceil_div(L.n, BY);
    sh.zc = ceil_div(L.n, std::max(1, std::min(c, L.n)));
    sh.chunks = ceil_div(L.n, sh.zc);
    return sh;
}

// the autotuner's table: (device, n, count, mode) -> z-chunks
std::mutex tune_mu;
std::atomic<int> tune_entries{0};  // table size, read without the lock by every tunable launch
std::map<std::tuple<int, int, int, int>, int>& tune_table() {
    static std::map<std::tuple<int, int, int, int>, int> t;
    return t;
}
int current_device() {
    int d = 0;
    KS_CUDA(cudaGetDevice(&d));
    return d;
}

template <int MODE, bool DOT>
void launch_mode(const Shape& sh, int count, const CUtensorMap& tmap, const Params& p, float* out, cudaStream_t s) {
    const int smem = NS * PLANE_BYTES + SD * n_side<MODE>() * THREADS * 16;
    static std::atomic<unsigned long long> attr_set{0};
    once_per_device(attr_set, [smem] {
        KS_CUDA(cudaFuncSetAttribute(stencil_kernel<MODE, DOT>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        // CTAS_PER_SM rings of 30 KB need the large shared-memory carveout
        KS_CUDA(cudaFuncSetAttribute(stencil_kernel<MODE, DOT>, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
    });
    dim3 grid(sh.tiles_x * sh.tiles_y * sh.chunks, count);
    stencil_kernel<MODE, DOT><<<grid, THREADS, smem, s>>>(tmap, p, out);
    KS_LAUNCH_CHECK();
}

}  // namespace

void make_field_tmap(CUtensorMap* map, const Layout& L, const float* base, int count) {
    cuuint64_t dims[4] = {(cuuint64_t)L.n, (cuuint64_t)L.n, (cuuint64_t)L.n, (cuuint64_t)count};
    cuuint64_t strides[3] = {(cuuint64_t)L.P * 4, (cuuint64_t)L.n * L.P * 4, (cuuint64_t)L.F * 4};
    cuuint32_t box[4] = {HXW, HYW, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float*>(base), dims, strides, box, estr,
                             CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw DeviceError("cuTensorMapEncodeTiled failed (code " + std::to_string((int)r) + ")");
}

void stencil_set_tuned_chunks(int n, int count, int mode, int chunks) {
    if (mode != ST_HAMILTONIAN && mode != ST_JACOBI) throw std::invalid_argument("stencil tuning: only H psi and the Jacobi sweep are tuned");
    if (n < 1 || count < 1 || chunks < 1 || chunks > n) throw std::invalid_argument("stencil tuning: need n, count >= 1 and 1 <= chunks <= n");
    std::lock_guard<std::mutex> g(tune_mu);
    tune_table()[std::make_tuple(current_device(), n, count, mode)] = chunks;
    tune_entries.store((int)tune_table().size());
}

int stencil_tuned_chunks(int n, int count, int mode) {
    if (tune_entries.load() == 0) return 0;
    const int dev = current_device();
    std::lock_guard<std::mutex> g(tune_mu);
    auto it = tune_table().find(std::make_tuple(dev, n, count, mode));
    return it == tune_table().end() ? 0 : it->second;
}

int stencil_max_chunks(const Layout& L) { return std::max(1, L.n / 8); }

int stencil_model_chunks(const Layout& L, int count) { return shape_for(L, count).chunks; }

std::vector<std::array<int, 4>> stencil_tuning_entries() {
    const int dev = current_device();
    std::lock_guard<std::mutex> g(tune_mu);
    std::vector<std::array<int, 4>> out;
    for (const auto& e : tune_table())
        if (std::get<0>(e.first) == dev) out.push_back({std::get<1>(e.first), std::get<2>(e.first), std::get<3>(e.first), e.second});
    return out;
}

void stencil_tuning_clear() {
    const int dev = current_device();
    std::lock_guard<std::mutex> g(tune_mu);
    for (auto it = tune_table().begin(); it != tune_table().end();)
        it = std::get<0>(it->first) == dev ? tune_table().erase(it) : std::next(it);
    tune_entries.store((int)tune_table().size());
}

int stencil_ctas(const Layout& L, int count) {
    Shape sh = shape_for(L, count);
    return sh.tiles_x * sh.tiles_y * sh.chunks * count;
}

int stencil_ctas_per_vector(const Layout& L, int count) {
    Shape sh = shape_for(L, count);
    return sh.tiles_x * sh.tiles_y * sh.chunks;
}

int launch_stencil(const Layout& L, const CUtensorMap& tmap, int count, const StencilArgs& a, float* out, cudaStream_t s) {
    if (count <= 0) return 0;
    // the quads' 16-byte loads and stores need 16-byte aligned fields (P is a multiple of 4 floats)
    if ((reinterpret_cast<uintptr_t>(out) & 15) || (a.V && (reinterpret_cast<uintptr_t>(a.V) & 15)) ||
        (a.R && (reinterpret_cast<uintptr_t>(a.R) & 15)) || (a.out2 && (reinterpret_cast<uintptr_t>(a.out2) & 15)) ||
        (a.dinv && (reinterpret_cast<uintptr_t>(a.dinv) & 15)))
        throw std::invalid_argument("stencil: fields must be 16-byte aligned");
    const bool dot = a.dot_partials != nullptr;
    // the chunking: the caller's, else the autotuner's for the modes whose outputs do not depend on it, else the model's
    int chunks = a.chunks;
    if (chunks <= 0 && !dot && (a.mode == ST_HAMILTONIAN || a.mode == ST_JACOBI)) chunks = stencil_tuned_chunks(L.n, count, a.mode);
    if (chunks > 0 && dot) throw std::invalid_argument("stencil: a forced chunking is for the launches without dot partials");
    Shape sh = chunks > 0 ? shape_with_chunks(L, chunks) : shape_for(L, count);
    Params p;
    p.n = L.n;
    p.P = L.P;
    p.F = L.F;
    p.tiles_x = sh.tiles_x;
    p.tiles_y = sh.tiles_y;
    p.zc = sh.zc;
    p.scale = a.scale;
    p.omega = a.omega;
    p.diag_t = a.diag_t;
    p.V = a.V;
    p.R = a.R;
    p.lambda = a.lambda;
    p.dot_partials = a.dot_partials;
    p.err = device_error_flag();
    p.vec0 = a.vec0;
    p.theta = a.theta;
    p.out2 = a.out2;
    p.dinv = a.dinv;
    switch (a.mode) {
        case ST_LAPLACIAN:
            if (dot) launch_mode<ST_LAPLACIAN, true>(sh, count, tmap, p, out, s);
            else launch_mode<ST_LAPLACIAN, false>(sh, count, tmap, p, out, s);
            break;
        case ST_HAMILTONIAN:
            if (dot) launch_mode<ST_HAMILTONIAN, true>(sh, count, tmap, p, out, s);
            else launch_mode<ST_HAMILTONIAN, false>(sh, count, tmap, p, out, s);
            break;
        case ST_HAM_RESIDUAL:
            if (!dot || !a.theta || !a.lambda || !a.out2 || !a.V) throw std::invalid_argument("stencil: the residual form needs theta, lambda, V, W0 and partials");
            launch_mode<ST_HAM_RESIDUAL, true>(sh, count, tmap, p, out, s);
            break;
        default:
            if (dot) throw std::invalid_argument("stencil: dot partials are for the Laplacian, H and the residual form only");
            launch_mode<ST_JACOBI, false>(sh, count, tmap, p, out, s);
            break;
    }
    return sh.tiles_x * sh.tiles_y * sh.chunks * count;
}

}  // namespace ks
