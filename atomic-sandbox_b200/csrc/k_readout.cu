// k_readout.cu -- display and diagnostic readouts of a converged density on sm_100a: trilinear
// sampling at arbitrary points, the headless "volume" copy (the dense n^3 f32 image a renderer
// would upload as a 3-D texture), its maximum and the spin-polarisation integral.
//
// Reference operators:
//   sample_density          crates/qm-gpu/src/sample.rs:84-121, shaders/sample.wgsl (the blend);
//                           the cell and fractions of crates/qm/src/grid.rs:54-67 (trilinear_cell);
//   copy_density_to_volume  crates/qm-gpu/src/scf.rs:1780-1797 (unpad into rows, then a texture copy);
//   density_max             crates/qm-gpu/src/scf.rs:1831-1834 (Reduction::Max);
//   spin_abs_integral       crates/qm-gpu/src/scf.rs:1836-1842 (Reduction::AbsDiffSum, times dv).
//
// The reference resolves each point's cell on the CPU in f64 and uploads (f32 fractions, corner
// index). Here the same f64 operations run on the device, (p - origin) / h, floor, x - floor(x),
// all IEEE-exact or correctly rounded, so the cell and the f32-rounded fractions are the
// reference's bit for bit, and the host uploads only the points. The blend is a(1 - t) + b t along
// x, then y, then z, in f32 with explicit round-to-nearest operations (no contraction), so a node
// (t = 0 on every axis) returns the stored value exactly. A neighbour beyond an upper face reads 0
// with weight 0, the reference's zero ghost.
#include "kernels.cuh"
#include "reduce_util.cuh"

namespace ks {

namespace {

constexpr int TPB_R = 256;

__device__ __forceinline__ float lerp_rn(float a, float b, float t) {
    return __fadd_rn(__fmul_rn(a, __fsub_rn(1.0f, t)), __fmul_rn(b, t));
}

__global__ void __launch_bounds__(TPB_R) sample_kernel(int n, int P, double h, double origin, const float* __restrict__ f,
                                                       const double* __restrict__ pts, int count, float* __restrict__ out) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < count; q += gridDim.x * blockDim.x) {
        int c[3];
        float t[3];
        bool inside = true;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double x = (pts[3 * (long long)q + a] - origin) / h;
            if (!(x >= 0.0 && x <= (double)(n - 1))) inside = false;  // NaN lands here too
            const double i0 = inside ? floor(x) : 0.0;
            c[a] = (int)i0;
            t[a] = (float)(x - i0);
        }
        if (!inside) {
            out[q] = 0.0f;
            continue;
        }
        const int i = c[0], j = c[1], k = c[2];
        const bool xi = i + 1 < n, yj = j + 1 < n, zk = k + 1 < n;
        auto at = [&](int di, int dj, int dk) -> float {
            if ((di && !xi) || (dj && !yj) || (dk && !zk)) return 0.0f;
            return f[((long long)(k + dk) * n + (j + dj)) * P + (i + di)];
        };
        const float x00 = lerp_rn(at(0, 0, 0), at(1, 0, 0), t[0]);
        const float x10 = lerp_rn(at(0, 1, 0), at(1, 1, 0), t[0]);
        const float x01 = lerp_rn(at(0, 0, 1), at(1, 0, 1), t[0]);
        const float x11 = lerp_rn(at(0, 1, 1), at(1, 1, 1), t[0]);
        out[q] = lerp_rn(lerp_rn(x00, x10, t[1]), lerp_rn(x01, x11, t[1]), t[2]);
    }
}

// dense[(k*n + j)*n + i] = f[(k*n + j)*P + i] (+ g at the same point when g is non-null, f32 add),
// one block per (j, k) row group, and the per-block maximum of the written values.
__global__ void __launch_bounds__(TPB_R) volume_kernel(int n, int P, const float* __restrict__ f, const float* __restrict__ g,
                                                       float* __restrict__ dense, double* __restrict__ partials) {
    const long long N = (long long)n * n * n;
    float m = -INFINITY;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < N; q += (long long)gridDim.x * blockDim.x) {
        const long long row = q / n;
        const int i = (int)(q - row * n);
        const long long src = row * P + i;
        float v = f[src];
        if (g) v = __fadd_rn(v, g[src]);
        dense[q] = v;
        m = fmaxf(m, v);
    }
    double bm = block_max_signed((double)m);
    if (threadIdx.x == 0) partials[blockIdx.x] = bm;
}

// partials[b] = sum over this block's points of |a - b| in f64 (pads are 0 in both fields).
__global__ void __launch_bounds__(TPB_R) abs_diff_kernel(long long F, const float* __restrict__ a, const float* __restrict__ b,
                                                         double* __restrict__ partials) {
    double s = 0.0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < F; q += (long long)gridDim.x * blockDim.x)
        s += fabs((double)a[q] - (double)b[q]);
    s = block_sum(s);
    if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

}  // namespace

void launch_sample(const Layout& L, const float* f, const double* pts, int count, float* out, cudaStream_t s) {
    if (count <= 0) return;
    const int blocks = std::min(ceil_div(count, TPB_R), 16 * sm_count());
    sample_kernel<<<blocks, TPB_R, 0, s>>>(L.n, L.P, L.h, L.origin, f, pts, count, out);
    KS_LAUNCH_CHECK();
}

void launch_volume(const Layout& L, const float* f, const float* g, float* dense, double* partials, int blocks, cudaStream_t s) {
    volume_kernel<<<blocks, TPB_R, 0, s>>>(L.n, L.P, f, g, dense, partials);
    KS_LAUNCH_CHECK();
}

void launch_abs_diff(long long F, const float* a, const float* b, double* partials, int blocks, cudaStream_t s) {
    abs_diff_kernel<<<blocks, TPB_R, 0, s>>>(F, a, b, partials);
    KS_LAUNCH_CHECK();
}

}  // namespace ks
