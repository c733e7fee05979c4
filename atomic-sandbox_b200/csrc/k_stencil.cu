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
// z-chunk. Each z-plane of the tile plus its 4-point xy halo (40 x 24 floats) is staged in
// shared memory by one TMA load (cp.async.bulk.tensor.4d); the tensor map's extent is n on
// every axis, so the halo beyond the box arrives as the hardware's zero fill -- the Dirichlet
// boundary costs no branches and no ghost storage. An 8-deep ring of planes keeps four planes
// of prefetch in flight. Each thread computes two adjacent y-rows at one x and keeps the nine
// z-values of its two columns in registers (a rolling queue), so per output it reads 8 x- and
// 5 y-neighbours from shared memory and nothing else. Stores and the V / R reads are plain
// coalesced 128-byte warp accesses.
#include <cudaTypedefs.h>
#include "kernels.cuh"
#include "reduce_util.cuh"

namespace ks {

namespace {

constexpr int BX = 32, BY = 16;
constexpr int HXW = BX + 8, HYW = BY + 8;       // staged plane with halo: 40 x 24
constexpr int NS = 8;                            // ring depth (planes)
constexpr int PLANE_FLOATS = HXW * HYW;          // 960
constexpr unsigned PLANE_BYTES = PLANE_FLOATS * 4;  // 3840 = 30 * 128
constexpr int THREADS = 256;                     // 32 (x) * 8 (pairs of y rows)
constexpr long long WAIT_LIMIT = 1LL << 22;      // bounded mbarrier waits (~seconds)

constexpr float C1 = 1.6f, C2 = -0.2f, C3 = 0.025396825396825397f, C4 = -0.0017857142857142857f;

struct Params {
    int n, P;
    long long F;
    int tiles_x, tiles_y, zc;
    int mode;
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

// sum_m c_m * (m-th second differences over the three axes), smallest coefficients first
__device__ __forceinline__ float lap_unscaled(const float* c, int ci, const float* q, float f0) {
    float d[5];
#pragma unroll
    for (int m = 1; m <= 4; ++m) {
        float dx = (c[ci + m] - f0) + (c[ci - m] - f0);
        float dy = (c[ci + m * HXW] - f0) + (c[ci - m * HXW] - f0);
        float dz = (q[4 + m] - f0) + (q[4 - m] - f0);
        d[m] = (dx + dy) + dz;
    }
    float acc = C4 * d[4];
    acc = fmaf(C3, d[3], acc);
    acc = fmaf(C2, d[2], acc);
    acc = fmaf(C1, d[1], acc);
    return acc;
}

__global__ void __launch_bounds__(THREADS) stencil_kernel(const __grid_constant__ CUtensorMap tmap, Params p, float* __restrict__ out) {
    extern __shared__ __align__(1024) float ring[];  // NS planes of 40 x 24
    __shared__ __align__(8) uint64_t bar[NS];

    const int vec = blockIdx.y;
    int t = blockIdx.x;
    const int tile_x = t % p.tiles_x;
    t /= p.tiles_x;
    const int tile_y = t % p.tiles_y;
    const int chunk = t / p.tiles_y;
    const int x0 = tile_x * BX, y0 = tile_y * BY;
    const int z0 = chunk * p.zc;
    const int z1 = min(z0 + p.zc, p.n);
    const int nz = z1 - z0;
    const int nplanes = nz + 8;  // relative plane q <-> z = z0 - 4 + q

    const int lx = threadIdx.x & 31;
    const int ly = (threadIdx.x >> 5) * 2;  // rows ly and ly + 1 of the tile
    const int gx = x0 + lx;
    const int gy = y0 + ly;
    const bool okx = gx < p.n;
    const bool okA = okx && gy < p.n;
    const bool okB = okx && gy + 1 < p.n;
    const int ciA = (ly + 4) * HXW + (lx + 4);
    const int ciB = ciA + HXW;

    if (threadIdx.x == 0) {
        for (int b = 0; b < NS; ++b) mbar_init(&bar[b], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    auto issue = [&](int q) {
        const int b = q % NS;
        mbar_expect_tx(&bar[b], PLANE_BYTES);
        tma_load_plane(ring + b * PLANE_FLOATS, &tmap, x0 - 4, y0 - 4, z0 - 4 + q, p.vec0 + vec, &bar[b]);
    };
    if (threadIdx.x == 0)
        for (int q = 0; q < NS; ++q) issue(q);

    float qa[9], qb[9];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
        mbar_wait(&bar[q], 0, p.err);
        const float* pl = ring + q * PLANE_FLOATS;
        qa[q] = pl[ciA];
        qb[q] = pl[ciB];
    }
    __syncthreads();  // planes 0..3 are consumed: their buffers take planes 8..11
    if (threadIdx.x == 0)
        for (int q = NS; q < min(NS + 4, nplanes); ++q) issue(q);

    const long long vbase = (long long)vec * p.F;
    const float lam = (p.mode == ST_JACOBI) ? (float)p.lambda[vec] : 0.0f;
    double dot = 0.0;
    for (int s = 0; s < nz; ++s) {
        const int qn = s + 8;
        mbar_wait(&bar[qn % NS], (unsigned)((qn / NS) & 1), p.err);
        const float* pn = ring + (qn % NS) * PLANE_FLOATS;
        qa[8] = pn[ciA];
        qb[8] = pn[ciB];
        const float* c = ring + ((s + 4) % NS) * PLANE_FLOATS;
        const int z = z0 + s;
        const long long rowA = ((long long)z * p.n + gy) * p.P + gx;
        const long long rowB = rowA + p.P;
        float la = lap_unscaled(c, ciA, qa, qa[4]) * p.scale;
        float lb = lap_unscaled(c, ciB, qb, qb[4]) * p.scale;
        float oa = la, ob = lb;
        if (p.mode != ST_LAPLACIAN) {
            const float va = okA ? p.V[rowA] : 0.0f;
            const float vb = okB ? p.V[rowB] : 0.0f;
            const float ha = fmaf(va, qa[4], la);
            const float hb = fmaf(vb, qb[4], lb);
            if (p.mode == ST_HAMILTONIAN) {
                oa = ha;
                ob = hb;
            } else {
                const float ra = okA ? p.R[vbase + rowA] : 0.0f;
                const float rb = okB ? p.R[vbase + rowB] : 0.0f;
                const float ia = 1.0f / fmaxf(p.diag_t + va - lam, 0.1f);
                const float ib = 1.0f / fmaxf(p.diag_t + vb - lam, 0.1f);
                oa = qa[4] + p.omega * ia * (ra - (ha - lam * qa[4]));
                ob = qb[4] + p.omega * ib * (rb - (hb - lam * qb[4]));
            }
        }
        if (okA) out[vbase + rowA] = oa;
        if (okB) out[vbase + rowB] = ob;
        if (p.dot_partials) {
            if (okA) dot += (double)qa[4] * (double)oa;
            if (okB) dot += (double)qb[4] * (double)ob;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) { qa[q] = qa[q + 1]; qb[q] = qb[q + 1]; }
        __syncthreads();  // the centre plane's buffer is free
        if (threadIdx.x == 0 && s + 12 < nplanes) issue(s + 12);
    }
    if (p.dot_partials) {
        double sum = block_sum(dot);
        if (threadIdx.x == 0) p.dot_partials[blockIdx.x + (size_t)gridDim.x * blockIdx.y] = sum;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

struct Shape { int tiles_x, tiles_y, chunks, zc; };

Shape shape_for(const Layout& L, int count) {
    Shape sh;
    sh.tiles_x = ceil_div(L.n, BX);
    sh.tiles_y = ceil_div(L.n, BY);
    const long long per_chunk = (long long)sh.tiles_x * sh.tiles_y * count;
    const long long target = 2LL * sm_count();
    int chunks = (int)((target + per_chunk - 1) / per_chunk);
    chunks = std::max(1, std::min(chunks, ceil_div(L.n, 8)));
    sh.zc = ceil_div(L.n, chunks);
    sh.chunks = ceil_div(L.n, sh.zc);
    return sh;
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
    static bool attr_set = false;
    const int smem = NS * PLANE_BYTES;
    if (!attr_set) {
        KS_CUDA(cudaFuncSetAttribute(stencil_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
        attr_set = true;
    }
    Shape sh = shape_for(L, count);
    Params p;
    p.n = L.n;
    p.P = L.P;
    p.F = L.F;
    p.tiles_x = sh.tiles_x;
    p.tiles_y = sh.tiles_y;
    p.zc = sh.zc;
    p.mode = a.mode;
    p.scale = a.scale;
    p.omega = a.omega;
    p.diag_t = a.diag_t;
    p.V = a.V;
    p.R = a.R;
    p.lambda = a.lambda;
    p.dot_partials = a.dot_partials;
    p.err = device_error_flag();
    p.vec0 = a.vec0;
    dim3 grid(sh.tiles_x * sh.tiles_y * sh.chunks, count);
    stencil_kernel<<<grid, THREADS, smem, s>>>(tmap, p, out);
    KS_LAUNCH_CHECK();
    return (int)(grid.x * grid.y);
}

}  // namespace ks
