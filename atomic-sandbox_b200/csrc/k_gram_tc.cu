// k_gram_tc.cu -- the LOBPCG Gram block on the 5th-generation tensor cores (sm_100a, tcgen05).
//
// Computes D = [S | T]^T S over the grid (the transpose of G = S^T [S | T] the host assembles;
// crates/qm-gpu/src/reduce.rs:340-420 computes the same pairs with CUDA-core f32 partials). The
// reduction dimension K is the grid itself (~10^6 points), split across one persistent CTA per SM.
//
// Precision ("3xTF32"): every f32 input x is split into hi = x with the low 13 mantissa bits
// cleared (exactly a TF32 value) and lo = x - hi rounded to the nearest TF32; each K-step issues
// hi*hi + hi*lo + lo*hi on kind::tf32, so products carry ~22 significant bits (the dropped lo*lo
// term is ~2^-22 relative). kind::tf32 reads only the top 19 bits of each 32-bit operand, so the
// loaded tile itself serves as hi (the test suite checks the result against f64); only lo is
// written, into a second tile. The tensor core rounds toward zero -- its f32 accumulation and its
// reading of an operand's low bits -- so lo is rounded explicitly (truncated, it would bias every
// hi*lo term toward zero: lo has the sign of x) and each stage's hi*hi and cross-term sums get
// their own TMEM slots, drained right after the stage into f32 sums (round-to-nearest) that move
// into f64 every FLUSH stages. Measured relative bias of a Gram diagonal on random data: -3.5e-7
// with truncated lo and a whole-range cross-term slot, -1.3e-7 (one MMA's own 8-product sum) at
// best.
//
// Per CTA (15 warps): warp 12 lane 0 is the TMA producer (one 128B-swizzled box of the S rows and
// one of the T rows per 32-point slab); warps 8..11 form lo;
// warp 13 lane 0 issues the hi*hi MMAs and warp 14 lane 0 the cross-term MMAs (the issue latency of
// one thread, not the tensor core, is the limit), each committing to mbarriers; warps 0..7 drain
// finished slots with tcgen05.ld (warp w: TMEM lane quadrant w % 4, column half w / 4), one row per
// thread. The B operand is the A tile itself (its first N rows), so S is loaded once; every TMA
// destination row is a multiple of 8, so 1024-byte aligned.
//
// The ring is what sets the speed: a stage's round trip (TMA, split, MMA, commit) takes a few
// microseconds, so ~16 stages must be in flight per SM to stream at HBM rate. The tiles are
// therefore compact -- a stage holds only the rows with data (round8(N + mt) rows of 128 B, 6 KB
// at m = mt = 24) -- although the M = 128 MMA reads 128 rows: the rows past the data are whatever
// follows in shared memory (the next stages' tiles, or a zeroed tail), and they only produce rows
// of D the epilogue never reads (each row of D depends on its own row of A). Per-stage scalar work
// is kept small (running ring indices, descriptors advanced by addition): one issuing thread and
// the drains, not the tensor core, bound the stage rate. Every wait is bounded.
#include <algorithm>
#include <cudaTypedefs.h>
#include "kernels.cuh"

namespace ks {

namespace {

constexpr int RMAX = 16;                     // ring depth cap
constexpr int KT = 32;                       // points per stage (one 128-byte swizzle row)
constexpr int ROWS = 128;                    // MMA M: rows of [S | T] padded
constexpr int TILE_BYTES = ROWS * KT * 4;    // 16 KB
// Every TMA load's x coordinate is a multiple of KT points, so KT * 4 bytes must be a multiple of 16 (the TMA rule,
// whose violation faults the GPU), and the 128-byte swizzle wants rows of exactly 128 bytes.
static_assert((KT * 4) % 16 == 0 && KT * 4 == 128, "TMA x coordinates and swizzle rows need KT * 4 == 128 bytes");
constexpr int THREADS = 480;                 // 8 epilogue, 4 split, 1 TMA, 2 MMA warps
constexpr int FLUSH = 8;                     // stages summed in f32 before an f64 add
constexpr int NBUF_MAX = 8;                  // hi*hi accumulator buffers in flight (TMEM permitting)
constexpr long long WAIT_LIMIT = 1LL << 24;

__device__ __forceinline__ unsigned su32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, unsigned count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(su32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(su32(b)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(su32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(su32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// bounded wait: false (and the error flag) when it gave up
__device__ __forceinline__ bool mbar_wait(uint64_t* b, unsigned parity, int* err) {
    long long n = 0;
    while (!mbar_try(b, parity)) {
        if (++n > WAIT_LIMIT) {
            if (err) atomicExch(err, 2);
            return false;
        }
    }
    return true;
}
__device__ __forceinline__ void tma_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(su32(dst)),
        "l"((unsigned long long)map), "r"(x), "r"(y), "r"(su32(bar))
        : "memory");
}
// UMMA shared-memory descriptor, K-major, 128-byte swizzle: 8-row atoms of 128 B (SBO = 1024 B),
// descriptor version 1 (tcgen05), LBO unused (1).
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr) {
    return (unsigned long long)((addr >> 4) & 0x3FFF) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
__device__ __forceinline__ void mma_tf32(unsigned d_tmem, unsigned long long a, unsigned long long b, unsigned idesc, unsigned acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void ld8(unsigned* r, unsigned taddr) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(su32(bar)) : "memory");
}

// x rounded to the nearest TF32 value (ties away from zero): the tensor core itself reads only the top 19
// bits, which truncates toward zero. lo = x - hi has the sign of x (hi is x truncated), so a truncated lo
// would bias every hi*lo term toward zero.
__device__ __forceinline__ float tf32_rn(float x) { return __uint_as_float((__float_as_uint(x) + 0x1000u) & 0xFFFFE000u); }

struct Params {
    long long F;  // points per field (multiple of 4)
    int m, mt;
    int P;        // 32-point slabs per stage (2 when m and mt fit 32-row blocks, else 1)
    int SB;       // row stride of the S blocks of a stage's slabs
    int TR0, TB;  // first T row, row stride of the T blocks
    int N;        // MMA N: rows of the tile used as the B operand
    int rows;     // rows the split converts
    int stages_total;
    int R;        // ring depth
    int tbytes;   // bytes per tile (a multiple of 1024)
    int* err;
};

template <int NMAX>
__global__ void __launch_bounds__(THREADS, 1) gram_tc_kernel(const __grid_constant__ CUtensorMap tm_s, const __grid_constant__ CUtensorMap tm_t,
                                                             Params p, double* __restrict__ partials) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-aligned rings: R hi tiles, R lo tiles, then a zero tail so that an M = 128 read from the
    // last lo tile stays inside the allocation
    unsigned char* base = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
    const int R = p.R;
    unsigned char* hi = base;
    unsigned char* lo = base + (size_t)R * p.tbytes;
    __shared__ __align__(8) uint64_t full[RMAX], conv[RMAX], empty[RMAX], acc_full[NBUF_MAX], acc_empty[NBUF_MAX];
    __shared__ unsigned tmem_base;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nbuf = min(NBUF_MAX, 512 / (2 * p.N));  // TMEM: nbuf buffers of two N-column slots (hi*hi, cross)
    // this CTA's contiguous range of stages (P slabs of 32 points each)
    const int per = (p.stages_total + gridDim.x - 1) / gridDim.x;
    const int s0 = blockIdx.x * per;
    const int s1 = min(p.stages_total, s0 + per);
    const int nst = max(0, s1 - s0);

    if (threadIdx.x == 0) {
        for (int i = 0; i < R; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&conv[i], 4);
            mbar_init(&empty[i], 2);  // both MMA issuers release a tile
        }
        for (int i = 0; i < NBUF_MAX; ++i) {
            mbar_init(&acc_full[i], 2);  // both issuers commit to a buffer
            mbar_init(&acc_empty[i], 8);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // zero the rings and the tail once (rows that are never loaded stay zero)
    const int clear16 = (2 * R * p.tbytes + (TILE_BYTES - p.tbytes)) / 16;
    for (int i = threadIdx.x; i < clear16; i += blockDim.x) reinterpret_cast<float4*>(base)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(su32(&tmem_base)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    if (warp == 12) {
        // ---- TMA producer: slab q of a stage puts its S rows at row q*SB, its T rows at TR0 + q*TB
        if (lane == 0) {
            const unsigned bytes = (unsigned)(p.P * (p.m + p.mt) * KT * 4);
            int s = 0;
            unsigned ph = 0;
            for (int i = 0; i < nst; ++i) {
                if (i >= R && !mbar_wait(&empty[s], ph ^ 1u, p.err)) break;
                mbar_expect_tx(&full[s], bytes);
                unsigned char* dst = hi + (size_t)s * p.tbytes;
                for (int q = 0; q < p.P; ++q) {
                    const int x = ((s0 + i) * p.P + q) * KT;
                    tma_2d(dst + q * p.SB * KT * 4, &tm_s, x, 0, &full[s]);
                    tma_2d(dst + (p.TR0 + q * p.TB) * KT * 4, &tm_t, x, 0, &full[s]);
                }
                if (++s == R) { s = 0; ph ^= 1u; }
            }
        }
    } else if (warp >= 8 && warp < 12) {
        // ---- lo = x - hi of rows [0, rows) of each stage into the lo ring (the loaded tile is hi)
        const int t = threadIdx.x - 256;
        const int n4 = p.rows * KT / 4;  // <= 1024: at most 8 float4 per thread
        int s = 0;
        unsigned ph = 0;
        for (int i = 0; i < nst; ++i) {
            if (!mbar_wait(&full[s], ph, p.err)) break;
            const float4* h4 = reinterpret_cast<const float4*>(hi + (size_t)s * p.tbytes);
            float4* l4 = reinterpret_cast<float4*>(lo + (size_t)s * p.tbytes);
            float4 x[8];
#pragma unroll
            for (int u = 0; u < 8; ++u)
                if (t + 128 * u < n4) x[u] = h4[t + 128 * u];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                if (t + 128 * u < n4) {
                    float4 b;
                    b.x = tf32_rn(x[u].x - __uint_as_float(__float_as_uint(x[u].x) & 0xFFFFE000u));
                    b.y = tf32_rn(x[u].y - __uint_as_float(__float_as_uint(x[u].y) & 0xFFFFE000u));
                    b.z = tf32_rn(x[u].z - __uint_as_float(__float_as_uint(x[u].z) & 0xFFFFE000u));
                    b.w = tf32_rn(x[u].w - __uint_as_float(__float_as_uint(x[u].w) & 0xFFFFE000u));
                    l4[t + 128 * u] = b;
                }
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&conv[s]);
            if (++s == R) { s = 0; ph ^= 1u; }
        }
    } else if (warp == 13 || warp == 14) {
        // ---- MMA issuers (one thread each, so their issue latencies overlap). A stage writes buffer
        // b = i % nbuf: warp 13 its hi*hi products (4 K-steps) into slot M, warp 14 its hi*lo + lo*hi
        // cross terms (8 MMAs) into slot X; the epilogue drains both as soon as the stage is done. The
        // tensor core's f32 accumulation rounds toward zero, so no sum runs longer than one stage (a
        // whole-range cross-term slot biased the Gram by ~1e-7 relative). Descriptors advance by the
        // tile size (ring) and 32 B per K-step (the address field counts 16-byte units).
        if (lane == 0) {
            const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(p.N >> 3) << 17) | ((unsigned)(ROWS >> 4) << 24);
            const unsigned long long dh0 = smem_desc(su32(hi)), dl0 = smem_desc(su32(lo));
            const unsigned long long step = (unsigned long long)(p.tbytes >> 4);
            const bool main_issuer = warp == 13;
            int s = 0, b = 0;
            unsigned ph = 0, bph = 0;
            for (int i = 0; i < nst; ++i) {
                if (i >= nbuf && !mbar_wait(&acc_empty[b], bph ^ 1u, p.err)) break;
                if (!mbar_wait(&conv[s], ph, p.err)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned d = tmem + (unsigned)(2 * b * p.N) + (main_issuer ? 0u : (unsigned)p.N);
                const unsigned long long h0 = dh0 + (unsigned long long)s * step, l0 = dl0 + (unsigned long long)s * step;
                if (main_issuer) {
                    mma_tf32(d, h0, h0, idesc, 0u);
#pragma unroll
                    for (int kk = 1; kk < KT / 8; ++kk) mma_tf32(d, h0 + 2 * kk, h0 + 2 * kk, idesc, 1u);
                } else {
                    mma_tf32(d, h0, l0, idesc, 0u);
                    mma_tf32(d, l0, h0, idesc, 1u);
#pragma unroll
                    for (int kk = 1; kk < KT / 8; ++kk) {
                        mma_tf32(d, h0 + 2 * kk, l0 + 2 * kk, idesc, 1u);
                        mma_tf32(d, l0 + 2 * kk, h0 + 2 * kk, idesc, 1u);
                    }
                }
                mma_commit(&empty[s]);     // this issuer is done with the stage's tiles
                mma_commit(&acc_full[b]);  // and its slot of buffer b is ready to drain
                if (++s == R) { s = 0; ph ^= 1u; }
                if (++b == nbuf) { b = 0; bph ^= 1u; }
            }
        }
    } else {
        // ---- epilogue: warps 0..7; warp w reads TMEM lanes 32(w%4)..+31 (row = lane index) and the
        // column half w/4 of its rows' own N-column block. Each stage's two slots (hi*hi and cross
        // terms) are added to f32 sums (round-to-nearest), which go into f64 totals every FLUSH
        // stages. With two slabs per stage, lane quadrants 0..3 hold S of slab 0, S of slab 1,
        // T of slab 0, T of slab 1, and slab q's columns start at 32q.
        constexpr int HALF = NMAX / 2;
        const int quad = warp & 3, c0 = (warp >> 2) * HALF;
        const int mc = (p.m + 7) & ~7;  // columns of D that hold data
        int orow, colbase, slab;
        if (p.P == 2) {
            slab = quad & 1;
            colbase = 32 * slab;
            orow = (quad < 2) ? (lane < p.m ? lane : -1) : (lane < p.mt ? p.m + lane : -1);
        } else {
            const int r = quad * 32 + lane;
            slab = 0;
            colbase = 0;
            orow = r < p.m ? r : (r >= p.TR0 && r < p.TR0 + p.mt ? r - p.TR0 + p.m : -1);
        }
        const int ncols = max(0, min(HALF, mc - c0));  // multiple of 8, the same for the whole warp
        float fs[HALF];
        double acc[HALF];
#pragma unroll
        for (int j = 0; j < HALF; ++j) { fs[j] = 0.f; acc[j] = 0.0; }
        const unsigned lane_base = tmem + ((unsigned)(quad * 32) << 16) + (unsigned)(colbase + c0);
        int done = 0, b = 0, since = 0;
        unsigned bph = 0;
        for (int i = 0; i < nst; ++i) {
            if (!mbar_wait(&acc_full[b], bph, p.err)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned ta = lane_base + (unsigned)(2 * b * p.N);
            // 16 columns of both slots per tcgen05.ld round (registers: the 64-column form has 32 per thread)
#pragma unroll
            for (int g0 = 0; g0 < HALF; g0 += 16) {
                unsigned r[16], rx[16];
#pragma unroll
                for (int g = 0; g < 16; g += 8)
                    if (g0 + g < ncols) {
                        ld8(r + g, ta + g0 + g);
                        ld8(rx + g, ta + p.N + g0 + g);
                    }
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j)
                    if (g0 + j < ncols) fs[g0 + j] += __uint_as_float(r[j]) + __uint_as_float(rx[j]);
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[b]);
            if (++since == FLUSH) {
#pragma unroll
                for (int j = 0; j < HALF; ++j) { acc[j] += (double)fs[j]; fs[j] = 0.f; }
                since = 0;
            }
            if (++b == nbuf) { b = 0; bph ^= 1u; }
            done = i + 1;
        }
#pragma unroll
        for (int j = 0; j < HALF; ++j) acc[j] += (double)fs[j];
        (void)done;
        if (orow >= 0) {
            double* out = partials + ((size_t)blockIdx.x * p.P + slab) * (p.m + p.mt) * p.m + (size_t)orow * p.m;
#pragma unroll
            for (int j = 0; j < HALF; ++j)
                if (c0 + j < p.m) out[c0 + j] = acc[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

PFN_cuTensorMapEncodeTiled_v12000 encode() {
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

void make_rows_map(CUtensorMap* map, const float* base, long long F, int rows) {
    cuuint64_t dims[2] = {(cuuint64_t)F, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)F * 4};
    cuuint32_t box[2] = {(cuuint32_t)KT, (cuuint32_t)rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = encode()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw DeviceError("cuTensorMapEncodeTiled (gram) failed, code " + std::to_string((int)r));
}

}  // namespace

// Two 32-point slabs per stage when S and T fit 32-row blocks (m, mt <= 32): the 128-row A tile holds
// S(slab 0), S(slab 1), T(slab 0), T(slab 1) at rows 0, 32, 64, 96, and B is its first 64 rows, so one
// MMA serves both slabs (the cross-slab blocks of D are never read) and each slab writes its own
// partials. Otherwise one slab per stage: S at row 0, T at row round8(m).
static int slabs_for(int m, int mt) { return (((m + 7) & ~7) <= 32 && ((mt + 7) & ~7) <= 32) ? 2 : 1; }

int gram_tc_blocks(int m, int mt) { return sm_count() * slabs_for(m, mt); }

// partials: [gram_tc_blocks(m, mt)][(m + mt) x m] of D = [S | T]^T S
void launch_gram_tc(long long F, int m, const float* S, int mt, const float* T, double* partials, cudaStream_t s) {
    if (m < 1 || mt < 1 || ((m + 7) & ~7) + mt > ROWS || m > 64) throw std::invalid_argument("gram_tc: need m <= 64 and round8(m) + mt <= 128");
    if (F % 4 != 0) throw std::invalid_argument("gram_tc: F must be a multiple of 4");
    CUtensorMap ms, mtm;
    make_rows_map(&ms, S, F, m);
    make_rows_map(&mtm, T, F, mt);
    Params p;
    p.F = F;
    p.m = m;
    p.mt = mt;
    p.P = slabs_for(m, mt);
    const int m8 = (m + 7) & ~7, mt8 = (mt + 7) & ~7;
    if (p.P == 2) {
        p.SB = 32; p.TR0 = 64; p.TB = 32; p.N = 64; p.rows = 96 + mt8;
        p.tbytes = TILE_BYTES;
    } else {
        p.SB = 0; p.TR0 = m8; p.TB = 0; p.N = m8; p.rows = m8 + mt8;
        p.tbytes = p.rows * KT * 4;
    }
    const long long slab_pts = (long long)KT * p.P;
    p.stages_total = (int)((F + slab_pts - 1) / slab_pts);
    // dynamic shared memory: two rings, the zero tail, 1 KB of alignment slack; the static barriers
    // take the last KB of the 227 KB a CTA may use
    constexpr int SMEM_BUDGET = 227 * 1024 - 1024;
    const int fixed = (TILE_BYTES - p.tbytes) + 1024;
    p.R = std::min(RMAX, (SMEM_BUDGET - fixed) / (2 * p.tbytes));
    if (p.R < 2) throw std::invalid_argument("gram_tc: tile ring does not fit");
    p.err = device_error_flag();
    const int smem = fixed + 2 * p.R * p.tbytes;
    static std::atomic<unsigned long long> attr_set{0};
    once_per_device(attr_set, [] {
        KS_CUDA(cudaFuncSetAttribute(gram_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BUDGET));
        KS_CUDA(cudaFuncSetAttribute(gram_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BUDGET));
    });
    if (m8 <= 32) gram_tc_kernel<32><<<sm_count(), THREADS, smem, s>>>(ms, mtm, p, partials);
    else gram_tc_kernel<64><<<sm_count(), THREADS, smem, s>>>(ms, mtm, p, partials);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
