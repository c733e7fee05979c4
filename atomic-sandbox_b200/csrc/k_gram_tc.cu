// k_gram_tc.cu -- the LOBPCG Gram block on the 5th-generation tensor cores (sm_100a, tcgen05).
//
// Computes D = [S | T]^T S over the grid (the transpose of G = S^T [S | T] the host assembles;
// crates/qm-gpu/src/reduce.rs:340-420 computes the same pairs with CUDA-core f32 partials). The
// reduction dimension K is the grid itself (~10^6 points), split across one persistent CTA per SM.
//
// Precision ("3xTF32"): every f32 input x is split in shared memory into hi = x with the low 13
// mantissa bits cleared (exactly a TF32 value) and lo = x - hi (exact in f32); each K-step issues
// hi*hi + hi*lo + lo*hi on kind::tf32, so products carry ~22 significant bits (the dropped lo*lo
// term is ~2^-22 relative). The tensor core's f32 accumulation rounds toward zero, so the hi*hi sums
// are kept in two slots per stage (at most one accumulating add each) and the stage is drained to
// f64 in registers; the small cross terms share a third slot.
//
// Per CTA (10 warps): warp 8 lane 0 is the TMA producer (one 128B-swizzled box of the S rows and
// one of the T rows per 32-point stage, 4-stage ring); warps 4..7 split each stage into hi/lo; warp
// 9 lane 0 issues the tcgen05.mma chain into one of two TMEM buffers (128 lanes x 3 slots of N
// columns, N = m rounded up to 8) and commits to mbarriers; warps 0..3 (TMEM lane quadrants 0..3)
// drain a finished buffer with tcgen05.ld into f64 sums, one row per thread. The B operand is
// the A tile itself (its first N rows), so S is loaded once. The T rows start at row N = m rounded
// up to 8, so every TMA destination is 1024-byte aligned. Every wait is bounded.
#include <cudaTypedefs.h>
#include "kernels.cuh"

namespace ks {

namespace {

constexpr int STAGES = 4;
constexpr int KT = 32;                       // points per stage (one 128-byte swizzle row)
constexpr int ROWS = 128;                    // MMA M: rows of [S | T] padded
constexpr int TILE_BYTES = ROWS * KT * 4;    // 16 KB
constexpr int THREADS = 320;
constexpr int NBUF_MAX = 4;                  // hi*hi accumulator buffers in flight (TMEM permitting)
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

struct Params {
    long long F;  // points per field (multiple of 4)
    int m, mt, N;
    int stages_total;
    int* err;
};

template <int NMAX>
__global__ void __launch_bounds__(THREADS, 1) gram_tc_kernel(const __grid_constant__ CUtensorMap tm_s, const __grid_constant__ CUtensorMap tm_t,
                                                             Params p, double* __restrict__ partials) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-aligned tile ring: hi tiles then lo tiles
    unsigned char* base = smem_raw + ((1024 - (su32(smem_raw) & 1023)) & 1023);
    float* hi = reinterpret_cast<float*>(base);
    float* lo = reinterpret_cast<float*>(base + STAGES * TILE_BYTES);
    __shared__ __align__(8) uint64_t full[STAGES], conv[STAGES], empty[STAGES], acc_full[NBUF_MAX], acc_empty[NBUF_MAX];
    __shared__ unsigned tmem_base;

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int m8 = p.N;                 // T rows start at a 1024-byte-aligned row (m rounded up to 8)
    const int rows = m8 + p.mt;         // rows of the A tile that hold data
    const int nbuf = min(NBUF_MAX, (512 - p.N) / (2 * p.N));  // TMEM: slot C + nbuf x (A, B)
    // this CTA's contiguous range of 32-point stages
    const int per = (p.stages_total + gridDim.x - 1) / gridDim.x;
    const int s0 = blockIdx.x * per;
    const int s1 = min(p.stages_total, s0 + per);
    const int nst = max(0, s1 - s0);

    if (threadIdx.x == 0) {
        for (int i = 0; i < STAGES; ++i) {
            mbar_init(&full[i], 1);
            mbar_init(&conv[i], 4);
            mbar_init(&empty[i], 1);
        }
        for (int i = 0; i < NBUF_MAX; ++i) {
            mbar_init(&acc_full[i], 1);
            mbar_init(&acc_empty[i], 4);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // rows >= mc of every hi/lo tile stay zero (the MMA reads all 128 rows)
    for (int i = threadIdx.x; i < 2 * STAGES * TILE_BYTES / 16; i += blockDim.x)
        reinterpret_cast<float4*>(base)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(su32(&tmem_base)) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const unsigned tmem = tmem_base;

    if (warp == 8) {
        // ---- TMA producer
        if (lane == 0) {
            const unsigned bytes = (unsigned)((p.m + p.mt) * KT * 4);
            for (int i = 0; i < nst; ++i) {
                const int s = i % STAGES;
                if (i >= STAGES && !mbar_wait(&empty[s], ((i / STAGES) - 1) & 1, p.err)) break;
                mbar_expect_tx(&full[s], bytes);
                const int x = (s0 + i) * KT;
                tma_2d(hi + s * (TILE_BYTES / 4), &tm_s, x, 0, &full[s]);
                tma_2d(hi + s * (TILE_BYTES / 4) + m8 * KT, &tm_t, x, 0, &full[s]);
            }
        }
    } else if (warp >= 4 && warp < 8) {
        // ---- hi/lo split of rows [0, rows) of each stage
        const int t = threadIdx.x - 128;
        const int n4 = rows * KT / 4;
        for (int i = 0; i < nst; ++i) {
            const int s = i % STAGES;
            if (!mbar_wait(&full[s], (i / STAGES) & 1, p.err)) break;
            float4* h4 = reinterpret_cast<float4*>(hi + s * (TILE_BYTES / 4));
            float4* l4 = reinterpret_cast<float4*>(lo + s * (TILE_BYTES / 4));
            for (int e = t; e < n4; e += 128) {
                float4 x = h4[e], a, b;
                a.x = __uint_as_float(__float_as_uint(x.x) & 0xFFFFE000u); b.x = x.x - a.x;
                a.y = __uint_as_float(__float_as_uint(x.y) & 0xFFFFE000u); b.y = x.y - a.y;
                a.z = __uint_as_float(__float_as_uint(x.z) & 0xFFFFE000u); b.z = x.z - a.z;
                a.w = __uint_as_float(__float_as_uint(x.w) & 0xFFFFE000u); b.w = x.w - a.w;
                h4[e] = a;
                l4[e] = b;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&conv[s]);
        }
    } else if (warp == 9) {
        // ---- MMA issuer. TMEM columns [0, N) hold slot C, the hi*lo + lo*hi cross terms of the whole
        // range (2^-11 of the main terms, so its own truncation is negligible); stage i writes the
        // hi*hi products into buffer b = i % nbuf, two slots of N columns (A: k-steps 0-1, B: 2-3):
        // the tensor core's f32 accumulation rounds toward zero, so no large slot takes more than one
        // accumulating add, and the epilogue drains each buffer as soon as its stage is done.
        if (lane == 0) {
            const unsigned idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((unsigned)(p.N >> 3) << 17) | ((unsigned)(ROWS >> 4) << 24);
            const unsigned dC = tmem;
            for (int i = 0; i < nst; ++i) {
                const int b = i % nbuf, s = i % STAGES;
                if (i >= nbuf && !mbar_wait(&acc_empty[b], ((i / nbuf) - 1) & 1, p.err)) break;
                if (!mbar_wait(&conv[s], (i / STAGES) & 1, p.err)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const unsigned dA = tmem + (unsigned)(p.N + b * 2 * p.N), dB = dA + (unsigned)p.N;
                const unsigned ah = su32(hi + s * (TILE_BYTES / 4)), al = su32(lo + s * (TILE_BYTES / 4));
#pragma unroll
                for (int kk = 0; kk < KT / 8; ++kk) {
                    const unsigned long long dh = smem_desc(ah + kk * 32), dl = smem_desc(al + kk * 32);
                    mma_tf32(kk < 2 ? dA : dB, dh, dh, idesc, (kk & 1) ? 1u : 0u);
                    mma_tf32(dC, dh, dl, idesc, (i > 0 || kk > 0) ? 1u : 0u);
                    mma_tf32(dC, dl, dh, idesc, 1u);
                }
                mma_commit(&empty[s]);     // the stage's tiles are free once these MMAs have read them
                mma_commit(&acc_full[b]);  // and its two slots are ready to drain
            }
        }
    } else {
        // ---- epilogue: warps 0..3 own TMEM lanes 32w..32w+31 (row = lane index); per stage the two
        // hi*hi slots are summed in f32 (round-to-nearest) and added to f64 totals; slot C once at the end
        const int row = warp * 32 + lane;
        double acc[NMAX];
#pragma unroll
        for (int j = 0; j < NMAX; ++j) acc[j] = 0.0;
        const unsigned lane_base = tmem + ((unsigned)(warp * 32) << 16);
        int done = 0;
        for (int i = 0; i < nst; ++i) {
            const int b = i % nbuf;
            if (!mbar_wait(&acc_full[b], (i / nbuf) & 1, p.err)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const unsigned ta = lane_base + (unsigned)(p.N + b * 2 * p.N), tb = ta + (unsigned)p.N;
#pragma unroll
            for (int g = 0; g < NMAX; g += 16) {
                if (g < p.N) {
                    unsigned ra[16], rb[16];
                    ld8(ra, ta + g);
                    ld8(rb, tb + g);
                    if (g + 8 < p.N) {
                        ld8(ra + 8, ta + g + 8);
                        ld8(rb + 8, tb + g + 8);
                    }
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (g + q < p.N) acc[g + q] += (double)(__uint_as_float(ra[q]) + __uint_as_float(rb[q]));
                }
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acc_empty[b]);
            done = i + 1;
        }
        if (done == nst && nst > 0) {
#pragma unroll
            for (int g = 0; g < NMAX; g += 8) {
                if (g < p.N) {
                    unsigned rc[8];
                    ld8(rc, lane_base + g);
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
                    for (int q = 0; q < 8; ++q) acc[g + q] += (double)__uint_as_float(rc[q]);
                }
            }
        }
        // output row: S rows [0, m) and T rows [m8, m8 + mt) -> [0, m + mt)
        const int orow = row < p.m ? row : (row >= m8 && row < rows ? row - m8 + p.m : -1);
        if (orow >= 0) {
            double* out = partials + (size_t)blockIdx.x * (p.m + p.mt) * p.m + (size_t)orow * p.m;
#pragma unroll
            for (int j = 0; j < NMAX; ++j)
                if (j < p.m) out[j] = acc[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

PFN_cuTensorMapEncodeTiled_v12000 encode() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void* ptr = nullptr;
        KS_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !ptr) throw DeviceError("cuTensorMapEncodeTiled is not available");
        fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
    }
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

int gram_tc_blocks() { return sm_count(); }

// partials: [gram_tc_blocks()][(m + mt) x m] of D = [S | T]^T S
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
    p.N = (m + 7) & ~7;
    p.stages_total = (int)((F + KT - 1) / KT);
    p.err = device_error_flag();
    const int smem = 2 * STAGES * TILE_BYTES + 1024;
    static bool attr = false;
    if (!attr) {
        KS_CUDA(cudaFuncSetAttribute(gram_tc_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        KS_CUDA(cudaFuncSetAttribute(gram_tc_kernel<64>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr = true;
    }
    if (p.N <= 32) gram_tc_kernel<32><<<gram_tc_blocks(), THREADS, smem, s>>>(ms, mtm, p, partials);
    else gram_tc_kernel<64><<<gram_tc_blocks(), THREADS, smem, s>>>(ms, mtm, p, partials);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
