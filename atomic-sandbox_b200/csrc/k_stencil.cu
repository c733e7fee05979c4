// k_stencil.cu -- the 8th-order finite-difference stencil family on sm_100a: Laplacian, H psi
// (-1/2 lap + V psi) and the fused damped-Jacobi sweep of the LOBPCG preconditioner.
//
// Reference operators: crates/qm/src/stencil.rs:21-51 (coefficients c = [-205/72, 8/5, -1/5,
// 8/315, -1/560], Dirichlet zero outside the box), crates/qm-gpu/src/shaders/stencil.wgsl:58-106
// (hamiltonian, jacobi_step). The centre is folded into second differences,
//     lap f = (1/h^2) sum_{m=1..4} c_m sum_axes [(f_{+m} - f_0) + (f_{-m} - f_0)],
// exact in real arithmetic because c_0 = -2 sum c_m, and exact per difference in f32 for smooth f.
//
// B200 design ("2.5-D" tiling): a CTA owns a 32 x 16 (x, y) tile of one field and marches a
// z-chunk. Each z-plane of the tile plus its 4-point xy halo (40 x 24 floats) is staged in shared
// memory by one TMA load (cp.async.bulk.tensor.4d); the tensor map's extent is n on every axis, so
// the halo beyond the box arrives as the hardware's zero fill -- the Dirichlet boundary costs no
// branches and no ghost storage. An 8-deep ring of planes keeps four planes of prefetch in flight.
// Each of the 128 threads computes a 2 x 2 block of outputs (two x-neighbours in two adjacent
// rows) with Blackwell's packed f32x2 arithmetic, keeps the nine z-values of its columns in a
// register queue that moves up one plane per step (a compact loop body: a 9-way unrolled rotation by
// renaming overflowed the instruction cache, 'no instruction' being the top stall), and reads 4.5
// shared-memory words per output. Stores and the V / R reads are coalesced 8-byte accesses.
#include <algorithm>
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
constexpr int THREADS = 128;                        // 16 x-pairs * 8 y-pairs
// The TMA rules the plane loads rely on, checked here because a violation faults the GPU instead of returning an
// error: the box's inner extent is a multiple of 16 bytes; a load's x coordinate, x0 - 4 with x0 a multiple of BX,
// times 4 bytes is a multiple of 16 (negative x is allowed for loads and reads the zero fill); each ring plane starts
// on a 128-byte boundary. The z-queue issues plane s + 12 into the buffer plane s + 4 left, which needs NS = 8.
static_assert((HXW * 4) % 16 == 0, "TMA box inner extent must be a multiple of 16 bytes");
static_assert((BX * 4) % 16 == 0 && (4 * 4) % 16 == 0, "TMA x coordinate x0 - 4 must be a multiple of 16 bytes");
static_assert(PLANE_BYTES % 128 == 0, "ring planes must start on 128-byte boundaries");
static_assert(NS == 8, "plane s + 12 reuses the buffer of plane s + 4 only with an 8-deep ring");
static_assert(THREADS == (BX / 2) * (BY / 2), "one thread per 2 x 2 block of outputs");
// resident CTAs per SM: registers capped at 96 per thread (no spills) for 20 warps per SM; measured on the H2O 95^3
// solve: 4 CTAs (126 registers) 213 ms, 5 CTAs 209 ms, 6 CTAs (80 registers) 216 ms
constexpr int CTAS_PER_SM = 5;
constexpr long long WAIT_LIMIT = 1LL << 22;         // bounded mbarrier waits (~seconds)

constexpr float C1 = 1.6f, C2 = -0.2f, C3 = 0.025396825396825397f, C4 = -0.0017857142857142857f;

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
// Bounded wait: on timeout the error flag is raised and the caller carries on with whatever is
// in shared memory (the result is then garbage, the host reports a device error).
__device__ __forceinline__ void mbar_wait(uint64_t* bar, unsigned parity, int* err) {
    long long spins = 0;
    while (!mbar_try_wait(bar, parity)) {
        if (++spins > WAIT_LIMIT) {
            if (err) atomicExch(err, 1);
            return;
        }
    }
}
__device__ __forceinline__ void tma_load_plane(float* dst, const CUtensorMap* map, int x, int y, int z, int v, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(
            smem_u32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(v), "r"(smem_u32(bar))
        : "memory");
}

// ---- packed f32x2 arithmetic (sm_100): one instruction for both x-neighbours of a thread
__device__ __forceinline__ u64 add2(u64 a, u64 b) { u64 d; asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ u64 sub2(u64 a, u64 b) { u64 d; asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ u64 mul2(u64 a, u64 b) { u64 d; asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b)); return d; }
__device__ __forceinline__ u64 fma2(u64 a, u64 b, u64 c) {
    u64 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}
__device__ __forceinline__ u64 pack(float lo, float hi) {
    u64 d;
    asm("mov.b64 %0, {%1, %2};" : "=l"(d) : "f"(lo), "f"(hi));
    return d;
}
__device__ __forceinline__ float lo_of(u64 v) { return __uint_as_float((unsigned)v); }
__device__ __forceinline__ float hi_of(u64 v) { return __uint_as_float((unsigned)(v >> 32)); }
// (hi of a, lo of b): the pair one float to the right of a
__device__ __forceinline__ u64 straddle(u64 a, u64 b) { return pack(hi_of(a), lo_of(b)); }
__device__ __forceinline__ u64 lds2(const float* p) { return *reinterpret_cast<const u64*>(p); }

// Second differences of one row's two x-outputs at the centre plane c (ci = the thread's even x
// in the staged plane), with the row's z-queue q (plane z+d at q[4 + d]):
// sum_m c_m [dx_m + dy_m + dz_m], smallest coefficients first -- the scalar kernel's order.
__device__ __forceinline__ u64 lap_row(const float* c, int ci, const u64 (&q)[9]) {
    const u64 f0 = q[4];
    const u64 xm4 = lds2(c + ci - 4), xm2 = lds2(c + ci - 2), xp2 = lds2(c + ci + 2), xp4 = lds2(c + ci + 4);
    const u64 xp[5] = {0, straddle(f0, xp2), xp2, straddle(xp2, xp4), xp4};
    const u64 xm[5] = {0, straddle(xm2, f0), xm2, straddle(xm4, xm2), xm4};
    u64 d[5];
#pragma unroll
    for (int m = 1; m <= 4; ++m) {
        const u64 dx = add2(sub2(xp[m], f0), sub2(xm[m], f0));
        const u64 dy = add2(sub2(lds2(c + ci + m * HXW), f0), sub2(lds2(c + ci - m * HXW), f0));
        const u64 dz = add2(sub2(q[4 + m], f0), sub2(q[4 - m], f0));
        d[m] = add2(add2(dx, dy), dz);
    }
    u64 acc = mul2(pack(C4, C4), d[4]);
    acc = fma2(pack(C3, C3), d[3], acc);
    acc = fma2(pack(C2, C2), d[2], acc);
    acc = fma2(pack(C1, C1), d[1], acc);
    return acc;
}

struct Tile {
    int z0, nplanes, vec;
    int gx, gy, ciA;
    long long vbase;
    bool okA, okB, ok2;  // rows A / B in range (and gx < n), gx + 1 < n
};

// One z-step (output plane z0 + s): the new plane z0 + s + 4 enters the queues at q[8].
template <int MODE, bool DOT>
__device__ __forceinline__ void step(const Params& p, const Tile& t, float* ring, uint64_t* bar, u64 (&qa)[9], u64 (&qb)[9], int s,
                                     float lam, float* __restrict__ out, double& dot, const CUtensorMap* tmap, int x0, int y0) {
    const int qn = s + 8;
    mbar_wait(&bar[qn % NS], (unsigned)((qn / NS) & 1), p.err);
    const float* pn = ring + (qn % NS) * PLANE_FLOATS;
    qa[8] = lds2(pn + t.ciA);
    qb[8] = lds2(pn + t.ciA + HXW);
    const float* c = ring + ((s + 4) % NS) * PLANE_FLOATS;
    const u64 sc = pack(p.scale, p.scale);
    const u64 la = mul2(lap_row(c, t.ciA, qa), sc);
    const u64 lb = mul2(lap_row(c, t.ciA + HXW, qb), sc);
    const u64 fa = qa[4], fb = qb[4];
    const long long rowA = ((long long)(t.z0 + s) * p.n + t.gy) * p.P + t.gx;
    const long long rowB = rowA + p.P;
    u64 oa = la, ob = lb;
    if (MODE != ST_LAPLACIAN) {
        const u64 va = t.okA ? *reinterpret_cast<const u64*>(p.V + rowA) : 0ull;
        const u64 vb = t.okB ? *reinterpret_cast<const u64*>(p.V + rowB) : 0ull;
        const u64 ha = fma2(va, fa, la), hb = fma2(vb, fb, lb);
        if (MODE == ST_HAMILTONIAN) {
            oa = ha;
            ob = hb;
        } else {
            const u64 ra = t.okA ? *reinterpret_cast<const u64*>(p.R + t.vbase + rowA) : 0ull;
            const u64 rb = t.okB ? *reinterpret_cast<const u64*>(p.R + t.vbase + rowB) : 0ull;
            const u64 nl = pack(-lam, -lam);
            // w + (omega / max(diag_t + V - lambda, 0.1)) (r - (H w - lambda w)), as the scalar sweep
            const u64 ua = sub2(ra, fma2(nl, fa, ha)), ub = sub2(rb, fma2(nl, fb, hb));
            const float ia0 = p.omega * (1.0f / fmaxf(p.diag_t + lo_of(va) - lam, 0.1f));
            const float ia1 = p.omega * (1.0f / fmaxf(p.diag_t + hi_of(va) - lam, 0.1f));
            const float ib0 = p.omega * (1.0f / fmaxf(p.diag_t + lo_of(vb) - lam, 0.1f));
            const float ib1 = p.omega * (1.0f / fmaxf(p.diag_t + hi_of(vb) - lam, 0.1f));
            oa = fma2(pack(ia0, ia1), ua, fa);
            ob = fma2(pack(ib0, ib1), ub, fb);
        }
    }
    if (t.okA) {
        if (t.ok2) *reinterpret_cast<u64*>(out + t.vbase + rowA) = oa;
        else out[t.vbase + rowA] = lo_of(oa);
    }
    if (t.okB) {
        if (t.ok2) *reinterpret_cast<u64*>(out + t.vbase + rowB) = ob;
        else out[t.vbase + rowB] = lo_of(ob);
    }
    if (DOT) {
        if (t.okA) {
            dot += (double)lo_of(fa) * (double)lo_of(oa);
            if (t.ok2) dot += (double)hi_of(fa) * (double)hi_of(oa);
        }
        if (t.okB) {
            dot += (double)lo_of(fb) * (double)lo_of(ob);
            if (t.ok2) dot += (double)hi_of(fb) * (double)hi_of(ob);
        }
    }
    __syncthreads();  // the centre plane's buffer is free
    if (threadIdx.x == 0 && s + 12 < t.nplanes) {
        const int q = s + 12, b = q % NS;
        mbar_expect_tx(&bar[b], PLANE_BYTES);
        tma_load_plane(ring + b * PLANE_FLOATS, tmap, x0 - 4, y0 - 4, t.z0 - 4 + q, p.vec0 + t.vec, &bar[b]);
    }
}

template <int MODE, bool DOT>
__global__ void __launch_bounds__(THREADS, CTAS_PER_SM) stencil_kernel(const __grid_constant__ CUtensorMap tmap, Params p, float* __restrict__ out) {
    extern __shared__ __align__(1024) float ring[];  // NS planes of 40 x 24
    __shared__ __align__(8) uint64_t bar[NS];

    Tile t;
    t.vec = blockIdx.y;
    int b = blockIdx.x;
    const int tile_x = b % p.tiles_x;
    b /= p.tiles_x;
    const int tile_y = b % p.tiles_y;
    const int chunk = b / p.tiles_y;
    const int x0 = tile_x * BX, y0 = tile_y * BY;
    t.z0 = chunk * p.zc;
    const int nz = min(t.z0 + p.zc, p.n) - t.z0;
    t.nplanes = nz + 8;  // relative plane q <-> z = z0 - 4 + q
    const int lx = (threadIdx.x & 15) * 2;   // even x of the thread's pair
    const int ly = (threadIdx.x >> 4) * 2;   // rows ly and ly + 1
    t.gx = x0 + lx;
    t.gy = y0 + ly;
    const bool okx = t.gx < p.n;
    t.ok2 = t.gx + 1 < p.n;
    t.okA = okx && t.gy < p.n;
    t.okB = okx && t.gy + 1 < p.n;
    t.ciA = (ly + 4) * HXW + (lx + 4);
    t.vbase = (long long)t.vec * p.F;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NS; ++i) mbar_init(&bar[i], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int q) {
        const int bb = q % NS;
        mbar_expect_tx(&bar[bb], PLANE_BYTES);
        tma_load_plane(ring + bb * PLANE_FLOATS, &tmap, x0 - 4, y0 - 4, t.z0 - 4 + q, p.vec0 + t.vec, &bar[bb]);
    };
    if (threadIdx.x == 0)
        for (int q = 0; q < NS; ++q) issue(q);

    u64 qa[9], qb[9];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        mbar_wait(&bar[q], 0, p.err);
        const float* pl = ring + q * PLANE_FLOATS;
        qa[q] = lds2(pl + t.ciA);
        qb[q] = lds2(pl + t.ciA + HXW);
    }
    __syncthreads();  // planes 0..3 are consumed: their buffers take planes 8..11
    if (threadIdx.x == 0)
        for (int q = NS; q < min(NS + 4, t.nplanes); ++q) issue(q);

    const float lam = (MODE == ST_JACOBI) ? (float)p.lambda[t.vec] : 0.0f;
    double dot = 0.0;
    int s = 0;
    for (; s < nz; ++s) {
        step<MODE, DOT>(p, t, ring, bar, qa, qb, s, lam, out, dot, &tmap, x0, y0);
#pragma unroll
        for (int i = 0; i < 8; ++i) {  // the z-queues move up one plane: q[i] <- q[i + 1]
            qa[i] = qa[i + 1];
            qb[i] = qb[i + 1];
        }
    }
    if (DOT) {
        double sum = block_sum(dot);
        if (threadIdx.x == 0) p.dot_partials[blockIdx.x + (size_t)gridDim.x * blockIdx.y] = sum;
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

template <int MODE, bool DOT>
void launch_mode(const Shape& sh, int count, const CUtensorMap& tmap, const Params& p, float* out, cudaStream_t s) {
    const int smem = NS * PLANE_BYTES;
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

int stencil_ctas(const Layout& L, int count) {
    Shape sh = shape_for(L, count);
    return sh.tiles_x * sh.tiles_y * sh.chunks * count;
}

int launch_stencil(const Layout& L, const CUtensorMap& tmap, int count, const StencilArgs& a, float* out, cudaStream_t s) {
    if (count <= 0) return 0;
    Shape sh = shape_for(L, count);
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
    const bool dot = a.dot_partials != nullptr;
    switch (a.mode) {
        case ST_LAPLACIAN:
            if (dot) launch_mode<ST_LAPLACIAN, true>(sh, count, tmap, p, out, s);
            else launch_mode<ST_LAPLACIAN, false>(sh, count, tmap, p, out, s);
            break;
        case ST_HAMILTONIAN:
            if (dot) launch_mode<ST_HAMILTONIAN, true>(sh, count, tmap, p, out, s);
            else launch_mode<ST_HAMILTONIAN, false>(sh, count, tmap, p, out, s);
            break;
        default:
            if (dot) throw std::invalid_argument("stencil: dot partials are for the Laplacian and H only");
            launch_mode<ST_JACOBI, false>(sh, count, tmap, p, out, s);
            break;
    }
    return sh.tiles_x * sh.tiles_y * sh.chunks * count;
}

}  // namespace ks
