// solver.cu -- host orchestration of the B200 Kohn-Sham SCF: the device reducer, the MG-PCG
// Hartree solve, LOBPCG with host f64 Rayleigh-Ritz, the Aufbau SCF driver and the forces.
//
// Algorithm sources (the reference's GPU solver, whose decisions this follows):
//   SCF driver      crates/qm-gpu/src/scf.rs:1237-1708 (eig tol tied to dRho, guess band, DIIS restart
//                   on a re-solved frozen set, charge renormalisation to the output charge)
//   LOBPCG          crates/qm-gpu/src/eigen.rs:685-1000 (raw [X, W, P], generalised Rayleigh-Ritz with
//                   the conditioning guard, X columns of A through the residuals, P orthogonalised to X,
//                   formation check, f32 floor stop)
//   Poisson         crates/qm-gpu/src/poisson.rs:284-342 (MG-PCG, true-residual floor detection)
//   DIIS            crates/qm-gpu/src/scf.rs:558-646
//   Forces          crates/qm-gpu/src/forces.rs:187-300
// What changes on the B200: every reduction is finished on the device, the CG scalars never
// leave it, the preconditioner/H-products/Ritz updates run as block kernels over all vectors of a
// channel at once, and the SCF's charge renormalisation is a device-side scale.
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <mutex>
#include <thread>
#include "solver.h"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include "dense.h"

namespace ks {

// ------------------------------------------------------------------ process-wide device facts
// Both caches are shared by the host threads of concurrent spin channels, hence the lock.
static std::mutex g_device_facts;

int sm_count() {
    static int counts[64] = {0};
    int dev = 0;
    KS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw DeviceError("device index out of range");
    std::lock_guard<std::mutex> lock(g_device_facts);
    if (!counts[dev]) KS_CUDA(cudaDeviceGetAttribute(&counts[dev], cudaDevAttrMultiProcessorCount, dev));
    return counts[dev];
}

static std::atomic<long long> g_launches{0};
static thread_local bool t_capturing = false;
void count_launch() {
    if (!t_capturing) g_launches.fetch_add(1, std::memory_order_relaxed);
}
void count_launches(long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void set_capturing(bool on) { t_capturing = on; }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

// Zeroes fresh device memory before any stream uses it. cudaMemset runs on the legacy default stream,
// which does not order against the solver's non-blocking stream: without the wait, a kernel enqueued
// on that stream right afterwards (ones_ = 1, a first iterate) can run first and be wiped.
void zero_device(void* p, size_t bytes) {
    KS_CUDA(cudaMemset(p, 0, bytes));
    KS_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
}

static int* shared_error_flag() {
    static int* flags[64] = {nullptr};
    int dev = 0;
    KS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw DeviceError("device index out of range");
    std::lock_guard<std::mutex> lock(g_device_facts);
    if (!flags[dev]) {
        KS_CUDA(cudaMalloc(&flags[dev], sizeof(int)));
        zero_device(flags[dev], sizeof(int));
    }
    return flags[dev];
}

static thread_local int* t_error_flag = nullptr;

int* device_error_flag() { return t_error_flag ? t_error_flag : shared_error_flag(); }

ErrorFlagScope::ErrorFlagScope(int* flag) : prev_(t_error_flag) { t_error_flag = flag; }
ErrorFlagScope::~ErrorFlagScope() { t_error_flag = prev_; }

void check_device_flag(cudaStream_t s) {
    int* flag = device_error_flag();
    int host = 0;
    KS_CUDA(cudaMemcpyAsync(&host, flag, sizeof(int), cudaMemcpyDeviceToHost, s));
    KS_CUDA(cudaStreamSynchronize(s));
    if (host) {
        KS_CUDA(cudaMemsetAsync(flag, 0, sizeof(int), s));
        KS_CUDA(cudaStreamSynchronize(s));
        throw DeviceError("a kernel's bounded wait gave up (a bulk or TMA copy did not complete)");
    }
}

namespace {

const double COEFF0 = -205.0 / 72.0;
const double COEFF[5] = {-205.0 / 72.0, 8.0 / 5.0, -1.0 / 5.0, 8.0 / 315.0, -1.0 / 560.0};

// LOBPCG constants (crates/qm-gpu/src/eigen.rs:276-317)
constexpr int STALL_WINDOW = 12;
constexpr double FLOOR_BAND = 10.0;
constexpr double RR_DROP = 1e-6;
constexpr double RITZ_FORM_SLACK = 1e-6;
constexpr double RITZ_FORM_RES = 1e-4;
constexpr int MAX_FORM_RESTORES = 3;
constexpr double ALPHA_MAX = 2.0;
constexpr double ALPHA_RESIDUAL_FRACTION = 0.1;
constexpr double GUESS_DEP = 1e-4;
constexpr int MAX_RESEED_ROUNDS = 3;
// SCF constants (crates/qm-gpu/src/scf.rs:359-399)
constexpr double POISSON_TOL = 1e-8;
constexpr int POISSON_MAX_ITER = 5000;
constexpr int EIGEN_MAX_ITER = 200;
constexpr double EIG_TOL_FLOOR_FACTOR = 3.0;
constexpr double EIG_GUESS_FACTOR = 1.5;
// Fermi-Dirac (crates/qm/src/occupations.rs): a level with min(f, 1 - f) at or above PARTIAL_OCCUPATION_MIN is partly
// occupied, and a step with one is tested against max(tol, GPU_PARTIAL_TOL); the columns of the block whose occupation
// tail (on their lower bounds theta - r) stays below 1e-2 tol (dense::fd_tight_columns) are held to the guard tolerance
// WITNESS_GUARD_TOL = WITNESS_GAP / 100 (or the step's eigen tolerance when that is looser; occupations.rs:91-92,
// :184-186), so that their lower bounds, on which the gap witness is read, are within 1e-3 Ha of their levels.
constexpr double PARTIAL_OCCUPATION_MIN = 1e-6;
constexpr double WITNESS_GUARD_TOL = 1e-3;
constexpr double GPU_PARTIAL_TOL = 1e-5;
constexpr double EIG_TOL_FRACTION = 0.0015;
constexpr double EIG_TOL_MAX = 1e-3;
constexpr double LAST_STEP_RESIDUAL_FACTOR = 3.0;
constexpr double BOUNDARY_DENSITY_WARN = 1e-5;
constexpr double STALL_LEVEL_PER_ELECTRON = 1e-3;
// multigrid (crates/qm-gpu/src/multigrid.rs:62-72)
constexpr int PRE_SWEEPS = 2, POST_SWEEPS = 2, COARSEST_SWEEPS = 12;
constexpr double MG_OMEGA = 6.0 / 7.0;
constexpr int FUSED_MAX_N = 12;
constexpr int CHECK_EVERY = 5;

double jacobi_omega() {
    double symbol_pi = COEFF[0] + 2.0 * (-COEFF[1] + COEFF[2] - COEFF[3] + COEFF[4]);
    return 4.0 / (3.0 * (symbol_pi / COEFF[0]));
}

using clk = std::chrono::steady_clock;
double secs(clk::time_point a) { return std::chrono::duration<double>(clk::now() - a).count(); }

// pinned host staging for coefficient uploads (one per process; every upload is followed by a
// synchronising readback before the buffer is rewritten)
// Columns of a Gram matrix within rel^(1/2) of the span of the earlier ones
// (crates/qm-gpu/src/eigen.rs:491-509).
std::vector<int> dependent_columns(int m, const std::vector<double>& b, double rel) {
    std::vector<double> l((size_t)m * m, 0.0);
    std::vector<int> kept, dep;
    for (int i = 0; i < m; ++i) {
        double d = b[(size_t)i * m + i];
        for (int j : kept) {
            double s = b[(size_t)i * m + j];
            for (int q : kept) {
                if (q >= j) break;
                s -= l[(size_t)i * m + q] * l[(size_t)j * m + q];
            }
            l[(size_t)i * m + j] = s / l[(size_t)j * m + j];
            d -= l[(size_t)i * m + j] * l[(size_t)i * m + j];
        }
        bool independent = d > rel * b[(size_t)i * m + i] && b[(size_t)i * m + i] > 0.0;
        if (independent) {
            l[(size_t)i * m + i] = std::sqrt(d);
            kept.push_back(i);
        } else {
            dep.push_back(i);
        }
    }
    return dep;
}

}  // namespace

double residual_floor_estimate(double h) {
    double s = 1.0 / (2.0 * h * h);
    double mean = 3.0 * std::fabs(COEFF[0]) * s;
    double c2 = 0.0;
    for (int m = 1; m <= 4; ++m) c2 += COEFF[m] * COEFF[m];
    double var = 3.0 * 2.0 * c2 * s * s;
    return 2.4e-8 * std::sqrt(mean * mean + var);
}

double rayleigh_ritz(int m, const std::vector<double>& A, const std::vector<double>& B, int nk, std::vector<double>& theta,
                     std::vector<double>& C) {
    for (int i = 0; i < m; ++i)
        if (!(B[(size_t)i * m + i] > 0.0))
            throw NumericalError("lobpcg: column " + std::to_string(i) + " of S has non-positive norm");
    std::vector<double> d(m);
    for (int i = 0; i < m; ++i) d[i] = 1.0 / std::sqrt(B[(size_t)i * m + i]);
    dense::Mat an((size_t)m * m), bn((size_t)m * m);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) {
            an[(size_t)i * m + j] = A[(size_t)i * m + j] * d[i] * d[j];
            bn[(size_t)i * m + j] = B[(size_t)i * m + j] * d[i] * d[j];
        }
    std::vector<double> sb, ub;
    dense::sym_eigen(m, bn, sb, ub);
    double smax = 0.0;
    for (double x : sb) smax = std::max(smax, x);
    std::vector<int> keep;
    for (int i = 0; i < m; ++i)
        if (sb[i] > RR_DROP * smax) keep.push_back(i);
    const int nkp = (int)keep.size();
    if (nkp < nk)
        throw NumericalError("lobpcg: the subspace lost rank (" + std::to_string(nkp) + " of " + std::to_string(m) + " kept)");
    std::vector<double> T((size_t)m * nkp);  // m x nkp row-major
    for (int i = 0; i < m; ++i)
        for (int c = 0; c < nkp; ++c) T[(size_t)i * nkp + c] = ub[i + (size_t)m * keep[c]] / std::sqrt(sb[keep[c]]);
    std::vector<double> at((size_t)m * nkp, 0.0);  // an * T
    for (int i = 0; i < m; ++i)
        for (int c = 0; c < nkp; ++c) {
            double s = 0.0;
            for (int j = 0; j < m; ++j) s += an[(size_t)i * m + j] * T[(size_t)j * nkp + c];
            at[(size_t)i * nkp + c] = s;
        }
    dense::Mat ah((size_t)nkp * nkp);
    for (int a = 0; a < nkp; ++a)
        for (int b = 0; b < nkp; ++b) {
            double s = 0.0;
            for (int i = 0; i < m; ++i) s += T[(size_t)i * nkp + a] * at[(size_t)i * nkp + b];
            ah[(size_t)a * nkp + b] = s;
        }
    for (int a = 0; a < nkp; ++a)
        for (int b = a + 1; b < nkp; ++b) {
            double s = 0.5 * (ah[(size_t)a * nkp + b] + ah[(size_t)b * nkp + a]);
            ah[(size_t)a * nkp + b] = ah[(size_t)b * nkp + a] = s;
        }
    std::vector<double> ea, va;
    dense::sym_eigen(nkp, ah, ea, va);
    std::vector<int> order(nkp);
    for (int i = 0; i < nkp; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return ea[x] < ea[y]; });
    theta.resize(nk);
    for (int c = 0; c < nk; ++c) theta[c] = ea[order[c]];
    double alpha = 0.0;
    for (int c = 0; c < nk; ++c) {
        double s = 0.0;
        for (int q = 0; q < nkp; ++q) {
            double y = va[q + (size_t)nkp * order[c]];
            s += y * y / sb[keep[q]];
        }
        alpha = std::max(alpha, std::sqrt(s));
    }
    C.assign((size_t)m * nk, 0.0);  // column-major m x nk
    for (int c = 0; c < nk; ++c)
        for (int i = 0; i < m; ++i) {
            double s = 0.0;
            for (int q = 0; q < nkp; ++q) s += T[(size_t)i * nkp + q] * va[q + (size_t)nkp * order[c]];
            C[i + (size_t)m * c] = d[i] * s;
        }
    return alpha;
}

double rayleigh_ritz_locked(int m, const std::vector<double>& A, const std::vector<double>& B, int locked, int na,
                            std::vector<double>& theta, std::vector<double>& C) {
    if (locked == 0) return rayleigh_ritz(m, A, B, na, theta, C);
    const int L = locked, mz = m - L;
    dense::Mat byy((size_t)L * L);
    for (int i = 0; i < L; ++i)
        for (int j = 0; j < L; ++j) byy[(size_t)i * L + j] = B[(size_t)i * m + j];
    if (!dense::cholesky(L, byy)) throw NumericalError("lobpcg: Cholesky of the locked columns' Gram failed");
    std::vector<double> kk((size_t)L * mz);  // B_YY^-1 B_YZ, L x mz row-major
    for (int i = 0; i < L; ++i)
        for (int j = 0; j < mz; ++j) kk[(size_t)i * mz + j] = B[(size_t)i * m + L + j];
    dense::cholesky_solve(L, byy, mz, kk);
    // Q = [-B_YY^-1 B_YZ; I], m x mz: Q^T M Q = M_ZZ - K^T M_YZ - M_ZY K + K^T M_YY K
    auto congruence = [&](const std::vector<double>& M) {
        std::vector<double> MQ((size_t)m * mz);  // M Q, m x mz row-major
        for (int i = 0; i < m; ++i)
            for (int c = 0; c < mz; ++c) {
                double s = M[(size_t)i * m + L + c];
                for (int j = 0; j < L; ++j) s -= M[(size_t)i * m + j] * kk[(size_t)j * mz + c];
                MQ[(size_t)i * mz + c] = s;
            }
        std::vector<double> R((size_t)mz * mz);
        for (int a = 0; a < mz; ++a)
            for (int b = 0; b < mz; ++b) {
                double s = MQ[(size_t)(L + a) * mz + b];
                for (int i = 0; i < L; ++i) s -= kk[(size_t)i * mz + a] * MQ[(size_t)i * mz + b];
                R[(size_t)a * mz + b] = s;
            }
        for (int a = 0; a < mz; ++a)
            for (int b = a + 1; b < mz; ++b) R[(size_t)a * mz + b] = R[(size_t)b * mz + a] = 0.5 * (R[(size_t)a * mz + b] + R[(size_t)b * mz + a]);
        return R;
    };
    std::vector<double> Cp;
    const double alpha = rayleigh_ritz(mz, congruence(A), congruence(B), na, theta, Cp);
    C.assign((size_t)m * na, 0.0);  // Q C', column-major m x na
    for (int c = 0; c < na; ++c) {
        for (int i = 0; i < L; ++i) {
            double s = 0.0;
            for (int j = 0; j < mz; ++j) s -= kk[(size_t)i * mz + j] * Cp[j + (size_t)mz * c];
            C[i + (size_t)m * c] = s;
        }
        for (int j = 0; j < mz; ++j) C[L + j + (size_t)m * c] = Cp[j + (size_t)mz * c];
    }
    return alpha;
}

// ------------------------------------------------------------------ kernel timing
KernelTimer::~KernelTimer() {
    for (auto& r : pending_) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (cudaEvent_t e : pool_) cudaEventDestroy(e);
}

cudaEvent_t KernelTimer::take() {
    {
        std::lock_guard<std::mutex> lock(mu_);
        if (!pool_.empty()) {
            cudaEvent_t e = pool_.back();
            pool_.pop_back();
            return e;
        }
    }
    cudaEvent_t e = nullptr;
    KS_CUDA(cudaEventCreate(&e));
    return e;
}

void KernelTimer::enable(bool on) {
    totals();  // settle what is recorded, then start from zero
    std::lock_guard<std::mutex> lock(mu_);
    agg_.clear();
    on_.store(on, std::memory_order_relaxed);
}

std::vector<ks_kernel_time> KernelTimer::totals() {
    std::lock_guard<std::mutex> lock(mu_);
    for (auto& r : pending_) {
        KS_CUDA(cudaEventSynchronize(r.b));
        float ms = 0.f;
        KS_CUDA(cudaEventElapsedTime(&ms, r.a, r.b));
        auto it = std::find_if(agg_.begin(), agg_.end(), [&](const ks_kernel_time& t) {
            return t.kernel == r.kernel && t.count == r.count && t.aux == r.aux;
        });
        if (it == agg_.end()) {
            agg_.push_back(ks_kernel_time{r.kernel, r.count, r.aux, 0, 0.0, r.bytes});
            it = agg_.end() - 1;
        }
        ++it->launches;
        it->total_ms += ms;
        pool_.push_back(r.a);
        pool_.push_back(r.b);
    }
    pending_.clear();
    return agg_;
}

// ------------------------------------------------------------------ buffers
void DevBuf::alloc(size_t n) {
    release();
    if (n == 0) return;
    KS_CUDA(cudaMalloc(&p, n));
    bytes = n;
}
void DevBuf::release() {
    if (p) cudaFree(p);
    p = nullptr;
    bytes = 0;
}

void Block::create(const Layout& L, int c) {
    count = c;
    F = L.F;
    buf.alloc((size_t)std::max(c, 1) * L.F * sizeof(float));
    zero_device(buf.p, buf.bytes);
    make_field_tmap(&tmap, L, buf.f(), std::max(c, 1));
}

// ------------------------------------------------------------------ reducer
void Reducer::init(const Layout& L, cudaStream_t s, size_t partial_doubles) {
    L_ = L;
    s_ = s;
    blocks_ = reduce_blocks(L.F);
    gram_blocks_ = 2 * sm_count();
    partials_.alloc(std::max(partial_doubles, (size_t)1 << 16) * sizeof(double));
    res_.alloc(RES_CAP * sizeof(double));
    KS_CUDA(cudaMallocHost(&host_, RES_CAP * sizeof(double)));
    KS_CUDA(cudaMallocHost(&host_flag_, sizeof(int)));
}

void Lane::init(const Layout& L) {
    KS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    KS_CUDA(cudaEventCreateWithFlags(&ev_join, cudaEventDisableTiming));
    red.init(L, s, 1 << 20);
    norm_part.alloc((size_t)red.blocks() * 64 * sizeof(double));
}

double* Lane::upload_buffer(size_t doubles) {
    if (doubles > up_cap) {
        if (up) cudaFreeHost(up);
        up = nullptr;
        KS_CUDA(cudaMallocHost(&up, doubles * sizeof(double)));
        up_cap = doubles;
    }
    return up;
}

Lane::~Lane() {
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    if (up) cudaFreeHost(up);
    if (ev_join) cudaEventDestroy(ev_join);
}

Reducer::~Reducer() {
    if (host_) cudaFreeHost(host_);
    if (host_flag_) cudaFreeHost(host_flag_);
}

void Reducer::dots(const std::vector<std::pair<const float*, const float*>>& pairs, int off, double scale) {
    for (size_t c0 = 0; c0 < pairs.size(); c0 += Pairs::MAX) {
        Pairs p;
        p.count = (int)std::min(pairs.size() - c0, (size_t)Pairs::MAX);
        for (int q = 0; q < p.count; ++q) { p.a[q] = pairs[c0 + q].first; p.b[q] = pairs[c0 + q].second; }
        launch_dots(L_.F, p, partials_.d(), blocks_, s_);
        launch_finish(partials_.d(), blocks_, p.count, scale, res_.d() + off + c0, s_);
    }
}

void Reducer::gram(int m, const float* S, int mt, const float* T, int off, double scale, const FinishDesc* extra) {
    if (gram_mode == 1) {
        // tensor cores: partials of D = [S | T]^T S, finished transposed into G = S^T [S | T]
        if (m > 64 || ((m + 7) & ~7) + mt > 128) throw std::invalid_argument("tensor-core Gram: block too large (m <= 64, round8(m) + mt <= 128)");
        const int blocks = gram_tc_blocks(m, mt);
        const size_t need = (size_t)blocks * m * (m + mt);
        if (need * sizeof(double) > partials_.bytes) partials_.alloc(need * sizeof(double));
        auto run = [&] { launch_gram_tc(L_.F, m, S, mt, T, partials_.d(), s_); };
        if (timer) timer->time(KS_K_GRAM, m, mt, 4.0 * (m + mt) * L_.interior(), s_, run);
        else run();
        if (extra) {
            FinishDesc g;
            g.partials = partials_.d();
            g.blocks = blocks;
            g.nvals = (m + mt) * m;
            g.scale = scale;
            g.out = res_.d() + off;
            g.trows = m + mt;
            g.tcols = m;
            launch_finish_pair(g, *extra, s_);
        } else {
            launch_finish_transposed(partials_.d(), blocks, m + mt, m, scale, res_.d() + off, s_);
        }
        return;
    }
    const int gblocks = gram_blocks(m, mt);
    const size_t need = (size_t)gblocks * m * (m + mt);
    if (need * sizeof(double) > partials_.bytes) partials_.alloc(need * sizeof(double));
    auto run = [&] { launch_gram(L_.F, m, S, mt, T, partials_.d(), s_); };
    if (timer) timer->time(KS_K_GRAM, m, mt, 4.0 * (m + mt) * L_.interior(), s_, run);
    else run();
    if (extra) {
        FinishDesc g;
        g.partials = partials_.d();
        g.blocks = gblocks;
        g.nvals = m * (m + mt);
        g.scale = scale;
        g.out = res_.d() + off;
        launch_finish_pair(g, *extra, s_);
    } else {
        launch_finish(partials_.d(), gblocks, m * (m + mt), scale, res_.d() + off, s_);
    }
}

const double* Reducer::read(int count) {
    if (count > RES_CAP) throw std::invalid_argument("reducer: result overflow");
    if (faults && faults->count.load() > 0) {
        if (faults->skip.load() > 0) {
            faults->skip.fetch_sub(1);
        } else {
            faults->count.fetch_sub(1);
            ++readbacks;
            throw DeviceError("a readback did not deliver its results (injected failure)");
        }
    }
    if (count > 0) KS_CUDA(cudaMemcpyAsync(host_, res_.d(), (size_t)count * sizeof(double), cudaMemcpyDeviceToHost, s_));
    KS_CUDA(cudaMemcpyAsync(host_flag_, device_error_flag(), sizeof(int), cudaMemcpyDeviceToHost, s_));
    auto t0 = std::chrono::steady_clock::now();
    KS_CUDA(cudaStreamSynchronize(s_));
    wait_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    ++readbacks;
    if (*host_flag_) {
        KS_CUDA(cudaMemsetAsync(device_error_flag(), 0, sizeof(int), s_));
        throw DeviceError("a kernel's bounded wait gave up (TMA copy did not complete)");
    }
    return host_;
}

// ------------------------------------------------------------------ Poisson (MG-PCG)
void Poisson::init(const Layout& L, cudaStream_t s, Reducer* red) {
    L_ = L;
    s_ = s;
    red_ = red;
    r_.create(L, 1); p_.create(L, 1); ap_.create(L, 1); b_.create(L, 1); z_.create(L, 1); res0_.create(L, 1); tmp0_.create(L, 1);
    ghost_.alloc(24 * (size_t)L.n * L.n * sizeof(double));
    scal_.alloc(8 * sizeof(double));
    zero_device(scal_.p, 8 * sizeof(double));
    q_.alloc(49 * sizeof(double));
    // hierarchy (crates/qm-gpu/src/multigrid.rs:105-118): odd-index coarsening down to n <= 2
    MgLevel l0{L.n, L.P, L.F, L.h, 0.f, 0.f};
    lvdesc_.push_back(l0);
    double d_low = 1.0, d_high = 1.0;
    int n = L.n;
    double h = L.h;
    while (n > 2) {
        int nc = n / 2;
        double dl = (d_low + 1.0) / 2.0;
        double dh = (d_high + (double)(n - 2 * nc)) / 2.0;
        Layout C = Layout::make(nc, 2.0 * h);
        MgLevel lv{nc, C.P, C.F, 2.0 * h, (float)(1.0 - 1.0 / dl), (float)(1.0 - 1.0 / dh)};
        lvdesc_.push_back(lv);
        n = nc;
        h = 2.0 * h;
        d_low = dl;
        d_high = dh;
    }
    levels_.resize(lvdesc_.size());
    for (size_t l = 1; l < lvdesc_.size(); ++l) {
        size_t bytes = (size_t)lvdesc_[l].F * sizeof(float);
        levels_[l].lv = lvdesc_[l];
        levels_[l].x.alloc(bytes); levels_[l].b.alloc(bytes); levels_[l].res.alloc(bytes); levels_[l].tmp.alloc(bytes);
        zero_device(levels_[l].x.p, bytes); zero_device(levels_[l].b.p, bytes);
        zero_device(levels_[l].res.p, bytes); zero_device(levels_[l].tmp.p, bytes);
    }
    fused_from_ = (int)lvdesc_.size() - 1;
    for (size_t l = 0; l < lvdesc_.size(); ++l)
        if (lvdesc_[l].n <= FUSED_MAX_N) { fused_from_ = (int)l; break; }
}

void Poisson::cycle(int l, float* x, const float* b) {
    const int nl = (int)lvdesc_.size();
    auto res_of = [&](int i) { return i == 0 ? res0_.at(0) : levels_[i].res.f(); };
    auto tmp_of = [&](int i) { return i == 0 ? tmp0_.at(0) : levels_[i].tmp.f(); };
    if (l >= fused_from_) {
        MgCoarse c;
        c.nlev = nl - l;
        if (c.nlev > MgCoarse::MAXL) throw std::logic_error("multigrid: too many fused levels");
        for (int i = l; i < nl; ++i) {
            int q = i - l;
            c.lv[q] = lvdesc_[i];
            c.x[q] = i == l ? x : levels_[i].x.f();
            c.b[q] = i == l ? const_cast<float*>(b) : levels_[i].b.f();
            c.res[q] = res_of(i);
            c.tmp[q] = tmp_of(i);
        }
        launch_mg_coarse(c, (float)MG_OMEGA, PRE_SWEEPS, POST_SWEEPS, COARSEST_SWEEPS, s_);
        return;
    }
    const MgLevel& lv = lvdesc_[l];
    launch_fill(x, 0.0f, lv.F, s_);
    for (int sw = 0; sw < PRE_SWEEPS; ++sw) {
        if (sw & 1) launch_mg_jacobi(lv, tmp_of(l), b, x, (float)MG_OMEGA, s_);
        else launch_mg_jacobi(lv, x, b, tmp_of(l), (float)MG_OMEGA, s_);
    }
    launch_mg_residual(lv, x, b, res_of(l), s_);
    launch_mg_restrict(lvdesc_[l + 1], lv, res_of(l), levels_[l + 1].b.f(), s_);
    cycle(l + 1, levels_[l + 1].x.f(), levels_[l + 1].b.f());
    launch_mg_prolong_add(lvdesc_[l + 1], lv, levels_[l + 1].x.f(), x, s_);
    for (int sw = 0; sw < POST_SWEEPS; ++sw) {
        if (sw & 1) launch_mg_jacobi(lv, tmp_of(l), b, x, (float)MG_OMEGA, s_);
        else launch_mg_jacobi(lv, x, b, tmp_of(l), (float)MG_OMEGA, s_);
    }
}

void Poisson::vcycle(const float* rhs, float* z) { cycle(0, z, rhs); }

// One PCG iteration between two readbacks (crates/qm-gpu/src/poisson.rs:284-342): ap = L p with p.Ap, the v / r update,
// z = M^-1 r by one V-cycle, r.z and r.r, the new direction. The scalars stay on the device (parity par).
void Poisson::iteration(float* v, int par) {
    double* scal = scal_.d();
    StencilArgs lapd;
    lapd.mode = ST_LAPLACIAN;
    lapd.scale = (float)(1.0 / (L_.h * L_.h));
    lapd.dot_partials = red_->partials();
    const int ctas = launch_stencil(L_, p_.tmap, 1, lapd, ap_.at(0), s_);
    launch_finish(red_->partials(), ctas, 1, -1.0, scal, s_);
    launch_cg_update(L_.F, v, r_.at(0), p_.at(0), ap_.at(0), scal, 1 + 2 * par, s_);
    vcycle(r_.at(0), z_.at(0));
    const int nxt = 1 - par;
    red_->dots({{r_.at(0), z_.at(0)}, {r_.at(0), r_.at(0)}}, 1, 1.0);
    KS_CUDA(cudaMemcpyAsync(scal + 1 + 2 * nxt, red_->res() + 1, 2 * sizeof(double), cudaMemcpyDeviceToDevice, s_));
    launch_cg_direction(L_.F, p_.at(0), z_.at(0), scal, 1 + 2 * par, 1 + 2 * nxt, s_);
    KS_CUDA(cudaMemcpyAsync(red_->res(), scal, sizeof(double), cudaMemcpyDeviceToDevice, s_));
}

// The iteration's ~40 small launches (the V-cycle's coarse levels are a few microseconds each) replayed as one CUDA
// graph per (v, parity): captured on first use, then one cudaGraphLaunch per iteration, so the device runs them
// back to back instead of waiting on the host's launch rate. The graph's kernels count as launches at every replay.
void Poisson::run_iteration(float* v, int par) {
    if (graph_v_ != v) {
        release_graphs();
        graph_v_ = v;
    }
    if (!graph_[par]) {
        cudaGraph_t g = nullptr;
        KS_CUDA(cudaStreamBeginCapture(s_, cudaStreamCaptureModeThreadLocal));
        set_capturing(true);
        try {
            iteration(v, par);
        } catch (...) {
            set_capturing(false);
            cudaStreamEndCapture(s_, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        set_capturing(false);
        KS_CUDA(cudaStreamEndCapture(s_, &g));
        size_t nodes = 0;
        KS_CUDA(cudaGraphGetNodes(g, nullptr, &nodes));
        std::vector<cudaGraphNode_t> list(nodes);
        KS_CUDA(cudaGraphGetNodes(g, list.data(), &nodes));
        int kernels = 0;
        for (auto n : list) {
            cudaGraphNodeType t;
            KS_CUDA(cudaGraphNodeGetType(n, &t));
            if (t == cudaGraphNodeTypeKernel) ++kernels;
        }
        const cudaError_t e = cudaGraphInstantiate(&graph_[par], g, 0);
        cudaGraphDestroy(g);
        KS_CUDA(e);
        graph_kernels_[par] = kernels;
    }
    KS_CUDA(cudaGraphLaunch(graph_[par], s_));
    count_launches(graph_kernels_[par]);
}

void Poisson::release_graphs() {
    for (auto& g : graph_)
        if (g) {
            cudaGraphExecDestroy(g);
            g = nullptr;
        }
}

Poisson::~Poisson() { release_graphs(); }

void Poisson::moments(const float* rho, double* dst) {
    launch_moments(L_, rho, red_->partials(), red_->blocks(), s_);
    launch_finish(red_->partials(), red_->blocks(), 49, L_.h * L_.h * L_.h, dst, s_);
}

void Poisson::true_residual(const CUtensorMap& v_map) {
    StencilArgs a;
    a.mode = ST_LAPLACIAN;
    a.scale = (float)(1.0 / (L_.h * L_.h));
    launch_stencil(L_, v_map, 1, a, ap_.at(0), s_);
    Terms t;
    t.count = 2;
    t.x[0] = b_.at(0); t.c[0] = 1.f;
    t.x[1] = ap_.at(0); t.c[1] = 1.f;
    launch_lincomb(L_.F, 1, ap_.at(0), t, s_);
    red_->dots({{ap_.at(0), ap_.at(0)}}, 0, 1.0);
}

PoissonStats Poisson::solve(const float* rho, float* v, const CUtensorMap& v_map, double tol, int max_iter) {
    NvtxRange range("ks poisson");
    PoissonStats st;
    const int rb0 = red_->readbacks;
    double* scal = scal_.d();
    moments(rho, q_.d());
    launch_poisson_rhs(L_, rho, q_.d(), ghost_.d(), b_.at(0), s_);
    // r = b - A v = b + L v; z = M^-1 r; p = z
    StencilArgs lap;
    lap.mode = ST_LAPLACIAN;
    lap.scale = (float)(1.0 / (L_.h * L_.h));
    launch_stencil(L_, v_map, 1, lap, ap_.at(0), s_);
    Terms t;
    t.count = 2;
    t.x[0] = b_.at(0); t.c[0] = 1.f;
    t.x[1] = ap_.at(0); t.c[1] = 1.f;
    launch_lincomb(L_.F, 1, r_.at(0), t, s_);
    vcycle(r_.at(0), z_.at(0));
    Terms cp;
    cp.count = 1;
    cp.x[0] = z_.at(0); cp.c[0] = 1.f;
    launch_lincomb(L_.F, 1, p_.at(0), cp, s_);
    // scal[1 + 2s] = r.z, scal[2 + 2s] = r.r for parity s
    red_->dots({{r_.at(0), z_.at(0)}, {r_.at(0), r_.at(0)}, {b_.at(0), b_.at(0)}}, 0, 1.0);
    KS_CUDA(cudaMemcpyAsync(scal + 1, red_->res(), 2 * sizeof(double), cudaMemcpyDeviceToDevice, s_));
    const double* h = red_->read(3);
    const double bb = h[2];
    double rz = h[0], rr = h[1];
    if (!(std::isfinite(bb) && std::isfinite(rr) && std::isfinite(rz)))
        throw NumericalError("Poisson: non-finite |b|, |r| or <r, z> (NaN in rho or V)");
    const double b_norm2 = std::max(bb, 1e-300);
    double residual = std::sqrt(rr / b_norm2);
    int it = 0, par = 0;
    double last_true = INFINITY;
    int stop = -1;
    while (residual > tol && it < max_iter) {
        if (!(rz > 0.0))
            throw NumericalError("Poisson: the multigrid preconditioner lost positive-definiteness (r.z = " + std::to_string(rz) + ")");
        const int nxt = 1 - par;
        run_iteration(v, par);
        h = red_->read(3);
        const double pap = h[0];
        rz = h[1];
        rr = h[2];
        if (!(pap > 0.0)) throw NumericalError("Poisson: A lost positive-definiteness (p.Ap = " + std::to_string(pap) + ")");
        par = nxt;
        ++it;
        residual = std::sqrt(rr / b_norm2);
        if (it % CHECK_EVERY == 0 && residual > tol) {
            true_residual(v_map);
            double tr = std::sqrt(red_->read(1)[0] / b_norm2);
            if (!std::isfinite(tr)) throw NumericalError("Poisson: non-finite true residual");
            // crates/qm-gpu/src/poisson.rs:188-190
            if (tr >= 4.0 * residual) { stop = 1; break; }
            if (tr >= 2.0 * residual && tr >= last_true) { stop = 2; break; }
            last_true = tr;
        }
    }
    if (stop < 0) stop = residual <= tol ? 0 : 3;
    true_residual(v_map);
    double tr = std::sqrt(red_->read(1)[0] / b_norm2);
    if (!std::isfinite(tr)) throw NumericalError("Poisson: non-finite true residual");
    st.iterations = it;
    st.residual = tr;
    st.stop = stop;
    st.readbacks = red_->readbacks - rb0;
    return st;
}

// ------------------------------------------------------------------ channels
void Channel::create(const Layout& L, int kk) {
    k = kk;
    A[0].create(L, 3 * k);
    A[1].create(L, 3 * k);
    cur = 0;
    T.create(L, 3 * k);
    HX.create(L, k);
    Q.create(L, k);
    theta_d.alloc((size_t)(2 * k + 6 * k * k) * sizeof(double));  // [theta | lambda | coef 3k x 2k]
    evals.assign(k, -1.0);
    res.assign(k, std::nan(""));
}

// ------------------------------------------------------------------ solver
// The channel's block at newk columns: the lowest min(k, newk) columns of the current iterate are kept (in the first
// arena), new ones are the reference's initial orbital with seed 1000 + 2 * column + spin (crates/qm/src/scf.rs:866).
void Solver::resize_channel(int sp, int newk, const Nuc* dnuc, int nn, cudaStream_t st, const std::vector<int>* cols) {
    if (!st) st = s_;
    Channel& old = ch_[sp];
    const int keep = cols ? (int)cols->size() : std::min(old.k, newk);
    Channel nc;
    nc.create(L_, newk);
    const size_t fb = (size_t)L_.F * sizeof(float);
    if (cols) {  // column j of the new block is column (*cols)[j] of the old one
        for (int j = 0; j < keep; ++j)
            KS_CUDA(cudaMemcpyAsync(nc.A[0].at(j), old.A[old.cur].at((*cols)[j]), fb, cudaMemcpyDeviceToDevice, st));
    } else {
        KS_CUDA(cudaMemcpyAsync(nc.A[0].at(0), old.X(), (size_t)keep * fb, cudaMemcpyDeviceToDevice, st));
    }
    for (int i = keep; i < newk; ++i)
        launch_initial_orbitals(L_, dnuc, nn, 1, 1000ULL + 2ULL * (unsigned long long)i + (unsigned long long)sp, 0, nc.A[0].at(i), st);
    nc.evals.clear();
    for (int j = 0; j < keep; ++j) {
        const int src = cols ? (*cols)[j] : j;
        nc.evals.push_back(src < (int)old.evals.size() ? old.evals[src] : -1.0);
        if (src < (int)old.res.size()) nc.res[j] = old.res[src];
    }
    // a new vector's eigenvalue placeholder: the block's last (crates/qm-gpu/src/scf.rs:843-849)
    while ((int)nc.evals.size() < newk) nc.evals.push_back(nc.evals.empty() ? -1.0 : nc.evals.back());
    nc.cur = 0;
    KS_CUDA(cudaStreamSynchronize(st));  // the old block is freed below
    ch_[sp] = std::move(nc);
}

int Solver::buffer_last(int sp, cudaStream_t st) {
    Channel& ch = ch_[sp];
    const int last = ch.k - 1;
    int top = last;
    for (int i = 0; i < ch.k; ++i)
        if (ch.evals[i] > ch.evals[top]) top = i;
    if (top == last) return -1;
    // swap the two columns of X through the H X scratch (free between LOBPCG calls: each call recomputes it)
    const size_t fb = (size_t)L_.F * sizeof(float);
    float* x = ch.A[ch.cur].at(0);
    float* tmp = ch.HX.at(0);
    KS_CUDA(cudaMemcpyAsync(tmp, x + (size_t)top * L_.F, fb, cudaMemcpyDeviceToDevice, st));
    KS_CUDA(cudaMemcpyAsync(x + (size_t)top * L_.F, x + (size_t)last * L_.F, fb, cudaMemcpyDeviceToDevice, st));
    KS_CUDA(cudaMemcpyAsync(x + (size_t)last * L_.F, tmp, fb, cudaMemcpyDeviceToDevice, st));
    std::swap(ch.evals[top], ch.evals[last]);
    std::swap(ch.res[top], ch.res[last]);
    return top;
}

// Mirrors the allocations of the constructor, Poisson::init, Reducer::init, Channel::create, the DIIS pool and the
// ionic fields; each buffer is counted at cudaMalloc's 2 MiB granularity for large and 512 B for small requests.
size_t Solver::footprint_bytes(int n, int n_up, int n_dn, const SolverOptions& o, int diis_history, bool pseudo_core) {
    const Layout L = Layout::make(n, 1.0);
    auto rounded = [](size_t b) { return b >= ((size_t)1 << 20) ? (b + ((size_t)2 << 20) - 1) & ~(((size_t)2 << 20) - 1) : (b + 511) & ~(size_t)511; };
    const size_t field = (size_t)L.F * sizeof(float);
    size_t total = 0;
    total += 11 * rounded(field);                                        // potentials, densities, XC, ones
    total += 3 * (rounded(((size_t)1 << 20) * sizeof(double)) + rounded(Reducer::RES_CAP * sizeof(double)));  // reducers
    total += 7 * rounded(field) + rounded(24 * (size_t)n * n * sizeof(double));  // Poisson CG fields and ghost table
    for (int m = n; m > 2;) {                                            // multigrid levels, four fields each
        m /= 2;
        total += 4 * rounded((size_t)Layout::make(m, 1.0).F * sizeof(float));
    }
    for (int ne : {n_up, n_dn}) {
        if (ne <= 0) continue;
        const int k = ne + o.n_extra;
        total += 2 * rounded(3 * k * field) + rounded(3 * k * field) + 2 * rounded(k * field);  // [X W P] x2, T, HX, Q
        total += rounded((size_t)(2 * k + 6 * k * k) * sizeof(double));
    }
    total += (size_t)(std::max(diis_history, 1) + 1) * 4 * rounded(field);  // DIIS pool
    if (pseudo_core) total += 3 * rounded(field);                          // partial core and the forces' v_xc
    return total;
}

Solver::Solver(int n, double h, const SolverOptions& o) : L_(Layout::make(n, h)), opt_(o) {
    if (n < 5 || !(h > 0)) throw std::invalid_argument("grid: n >= 5 and h > 0 required");
    KS_CUDA(cudaStreamCreateWithFlags(&s_, cudaStreamNonBlocking));
    KS_CUDA(cudaGetDevice(&dev_));
    KS_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    err_.alloc(256);
    zero_device(err_.p, err_.bytes);
    red_.init(L_, s_, 1 << 20);
    red_.faults = &faults_;
    for (auto& l : lane_) {
        l.reset(new Lane());
        l->init(L_);
        l->red.faults = &faults_;
    }
    poisson_.init(L_, s_, &red_);
    for (Block* b : {&vnuc_, &vh_, &in_up_, &in_dn_, &out_up_, &out_dn_, &rho_tot_, &v_up_, &v_dn_, &exc_, &ones_}) b->create(L_, 1);
    launch_fill(ones_.at(0), 1.0f, L_.F, s_);
    floor_ = residual_floor_estimate(h);
    KS_CUDA(cudaStreamSynchronize(s_));
}

Solver::~Solver() {
    if (s_) {
        cudaStreamSynchronize(s_);
        cudaStreamDestroy(s_);
    }
    if (ev_fork_) cudaEventDestroy(ev_fork_);
}

void Solver::import_state(int n_up, int n_dn, const int k[2], const double* const orb[2], const double* const evals[2],
                          const double* const occ[2], const double* rho_up, const double* rho_dn, const double* v_h, bool fermi_dirac) {
    const int nocc[2] = {n_up, n_dn};
    if (n_up < 0 || n_dn < 0 || !rho_up || !rho_dn || !v_h) throw std::invalid_argument("state_import: invalid arguments");
    if (fermi_dirac && opt_.n_extra < 1) throw std::invalid_argument("state_import: Fermi-Dirac needs n_extra >= 1 (ks_options)");
    int kk[2];
    for (int sp = 0; sp < 2; ++sp) {
        // the block the next warm solve runs: N_sigma + n_extra columns (under Fermi-Dirac a grown block is kept at its size)
        kk[sp] = nocc[sp] > 0 ? std::max(nocc[sp] + opt_.n_extra, fermi_dirac ? k[sp] : 0) : 0;
        if (k[sp] < nocc[sp] || k[sp] > std::max(kk[sp], nocc[sp]) || kk[sp] > 64 || (k[sp] > 0 && (!orb[sp] || !evals[sp])) ||
            (fermi_dirac && k[sp] > 0 && !occ[sp]))
            throw std::invalid_argument("state_import: spin " + std::to_string(sp) + ": need N_sigma <= k <= N_sigma + n_extra orbitals "
                                        "(up to 64), with their levels (and occupations under Fermi-Dirac)");
    }
    converged_ = false;
    have_warm_ = false;
    have_prev_ = false;
    const long long N = L_.interior();
    DevBuf tmp((size_t)N * sizeof(double));
    auto upload = [&](const double* host, float* field) {
        KS_CUDA(cudaMemcpyAsync(tmp.p, host, (size_t)N * sizeof(double), cudaMemcpyHostToDevice, s_));
        launch_pack(L_, 1, tmp.d(), field, s_);
    };
    for (int sp = 0; sp < 2; ++sp) {
        ensure_channel(sp, kk[sp]);
        occ_[sp].assign(kk[sp], 0.0);
        if (kk[sp] == 0) continue;
        Channel& ch = ch_[sp];
        ch.cur = 0;
        for (int i = 0; i < k[sp]; ++i) upload(orb[sp] + (size_t)i * N, ch.A[0].at(i));
        // columns the state does not carry start from the uniform(-1, 1) guess, seeded per column and spin
        for (int i = k[sp]; i < kk[sp]; ++i)
            launch_initial_orbitals(L_, nullptr, 0, 1, 1000ULL + 2ULL * (unsigned long long)i + (unsigned long long)sp, 1, ch.A[0].at(i), s_);
        ch.evals.assign(evals[sp], evals[sp] + k[sp]);
        while ((int)ch.evals.size() < kk[sp]) ch.evals.push_back(ch.evals.empty() ? -1.0 : ch.evals.back());
        ch.res.assign(kk[sp], std::nan(""));
        for (int i = 0; i < kk[sp]; ++i) occ_[sp][i] = fermi_dirac ? (i < k[sp] ? occ[sp][i] : 0.0) : (i < nocc[sp] ? 1.0 : 0.0);
    }
    upload(rho_up, out_up_.at(0));
    upload(rho_dn, out_dn_.at(0));
    upload(v_h, vh_.at(0));
    KS_CUDA(cudaStreamSynchronize(s_));  // tmp is freed on return
    nocc_[0] = n_up;
    nocc_[1] = n_dn;
    fd_state_ = fermi_dirac;
    state_gen_ = ionic_gen();
    have_warm_ = true;
}

void Solver::poison_parked_density() {
    const float nan = std::numeric_limits<float>::quiet_NaN();
    const long long c = ((long long)(L_.n / 2) * L_.n + L_.n / 2) * L_.P + L_.n / 2;  // the box centre
    KS_CUDA(cudaMemcpyAsync(out_up_.at(0) + c, &nan, sizeof(float), cudaMemcpyHostToDevice, s_));
    KS_CUDA(cudaStreamSynchronize(s_));
}

void Solver::ensure_channel(int spin, int k) {
    if (ch_[spin].k != k) {
        ch_[spin] = Channel();
        if (k > 0) ch_[spin].create(L_, k);
    }
}

void Solver::gram_checked(Reducer& red, int m, const float* S, int mt, const float* T, const FinishDesc* extra) {
    red.gram_mode = opt_.gram_mode;
    red.timer = &timer_;
    red.gram(m, S, mt, T, 0, L_.h * L_.h * L_.h, extra);  // the L2 product <a, b> = h^3 sum a b
}

EigenStats Solver::lobpcg(Channel& ch, Lane& lane, const float* V, double tol, double guess_tol, int max_iter, int head,
                          double tail_tol, int checked, bool lock) {
    NvtxRange range("ks lobpcg");
    EigenStats es;
    const int k = ch.k;
    if (checked < 0) checked = std::isfinite(tail_tol) ? k : head;
    checked = std::max(1, std::min(checked, k));
    head = std::max(0, std::min(head, checked));
    const bool split = std::isfinite(tail_tol);  // else the columns past the head are untested (checked == head)
    int locked = 0;  // the locked head (crates/qm-gpu/src/eigen.rs:742); W and P exist for the other columns only
    // LOBPCG_TRACE in the environment, set to any value, prints the reference's per-iteration lines to stderr
    // (crates/qm-gpu/src/eigen.rs:707, :800, :853, :941); the two spin channels' lines carry their spin
    static const bool trace = std::getenv("LOBPCG_TRACE") != nullptr;
    const char* tag = &ch == &ch_[0] ? "[up]" : &ch == &ch_[1] ? "[dn]" : "";
    const int rb0 = lane.red.readbacks;
    const double omega = jacobi_omega();
    const double diag_t = -1.5 * COEFF0 / (L_.h * L_.h);
    const float ham_scale = (float)(-0.5 / (L_.h * L_.h));
    double* theta_d = ch.theta_d.d();
    double* lambda_d = theta_d + k;
    double* coef_d = theta_d + 2 * k;
    const double npts = (double)L_.interior();
    auto apply_h = [&](const Block& in, int vec0, int count, float* out) {
        StencilArgs a;
        a.mode = ST_HAMILTONIAN;
        a.scale = ham_scale;
        a.V = V;
        a.vec0 = vec0;
        timer_.time(KS_K_HPSI, count, 0, (8.0 * count + 4.0) * npts, lane.s, [&] { launch_stencil(L_, in.tmap, count, a, out, lane.s); });
        // + V_NL under a pseudopotential setup (crates/qm-gpu/src/eigen.rs:216-227; the preconditioner stays local)
        if (nl_on_) ionic_.apply_nl(L_, in.at(vec0), count, out, lane.nl, lane.s);
    };
    // --- guess: one readback of X^T X and <x_i, H x_i>; dependent columns are re-seeded
    std::vector<double> theta(k), lambda(k);
    for (int round = 0;; ++round) {
        if (round >= MAX_RESEED_ROUNDS) throw NumericalError("lobpcg: could not generate independent guess vectors");
        apply_h(ch.A[ch.cur], 0, k, ch.HX.at(0));
        gram_checked(lane.red, k, ch.X(), k, ch.HX.at(0));
        const double* g = lane.red.read(k * 2 * k);
        std::vector<double> B((size_t)k * k);
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) B[(size_t)i * k + j] = 0.5 * (g[(size_t)i * 2 * k + j] + g[(size_t)j * 2 * k + i]);
        std::vector<int> dep = dependent_columns(k, B, GUESS_DEP);
        if (dep.empty()) {
            for (int i = 0; i < k; ++i) {
                theta[i] = g[(size_t)i * 2 * k + k + i] / B[(size_t)i * k + i];
                if (!std::isfinite(theta[i])) throw NumericalError("lobpcg: non-finite Rayleigh quotient of a guess vector");
            }
            break;
        }
        // deterministic noise under a Gaussian envelope (crates/qm-gpu/src/eigen.rs:376-389)
        const long long N = L_.interior();
        std::vector<double> noise(N);
        DevBuf tmp((size_t)N * sizeof(double));
        for (int slot : dep) {
            unsigned long long seed = 0x9E3779B97F4A7C15ULL ^ ((unsigned long long)slot << 32) ^ (unsigned long long)(round + 1);
            const int n = L_.n;
            double sigma2 = std::pow((n - 1) * L_.h / 4.0, 2);
            long long q = 0;
            for (int kk = 0; kk < n; ++kk)
                for (int j = 0; j < n; ++j)
                    for (int i = 0; i < n; ++i) {
                        seed = seed * 6364136223846793005ULL + 1442695040888963407ULL;
                        double u = (double)(seed >> 11) / 9007199254740992.0;
                        double x = L_.origin + i * L_.h, y = L_.origin + j * L_.h, z = L_.origin + kk * L_.h;
                        noise[q++] = (u - 0.5) * std::exp(-(x * x + y * y + z * z) / (2.0 * sigma2));
                    }
            KS_CUDA(cudaMemcpyAsync(tmp.p, noise.data(), N * sizeof(double), cudaMemcpyHostToDevice, lane.s));
            launch_pack(L_, 1, tmp.d(), ch.A[ch.cur].at(slot), lane.s);
            KS_CUDA(cudaStreamSynchronize(lane.s));
        }
    }
    lambda = theta;
    auto upload = [&](const std::vector<double>& th, const std::vector<double>& la, const std::vector<double>* coef) {
        size_t nd = 2 * (size_t)k + (coef ? coef->size() : 0);
        double* up = lane.upload_buffer(nd);
        std::copy(th.begin(), th.end(), up);
        std::copy(la.begin(), la.end(), up + k);
        if (coef) std::copy(coef->begin(), coef->end(), up + 2 * k);
        KS_CUDA(cudaMemcpyAsync(theta_d, up, nd * sizeof(double), cudaMemcpyHostToDevice, lane.s));
    };
    upload(theta, lambda, nullptr);
    int np = 0, iterations = 0, best_it = 0;
    double best = INFINITY;
    bool have_prev = false;
    std::vector<double> prev_theta;
    std::vector<double> res(k);
    // the H X launch that ends an iteration also forms the next residual, its first Jacobi sweep and the |r|^2
    // partials (ST_HAM_RESIDUAL, bit for bit the residual kernel's R and W0); a pseudopotential's V_NL is added after
    // the stencil, so under one the residual kernel runs on the stored H X instead
    const int nb = lane.red.blocks();
    const int cpv = stencil_ctas_per_vector(L_, k);
    const size_t norm_cap = (size_t)std::max(nb, cpv) * k;
    if (lane.norm_part.bytes < norm_cap * sizeof(double)) lane.norm_part.alloc(norm_cap * sizeof(double));
    double* norm_partials = lane.norm_part.d();  // finished in the Gram's finish launch
    bool fused_r = false;
    int norm_blocks = nb;
    for (;;) {
        // the inner cancellation point (crates/qm-gpu/src/scf.rs:1224-1235): the calling thread polls, every channel obeys
        if (inner_fn_ && std::this_thread::get_id() == poll_thread_ && inner_fn_(inner_user_)) inner_flag_.store(1);
        if (inner_flag_.load()) throw AbortInside();
        Block& S = ch.A[ch.cur];
        // 1. R = HX - theta X with the first Jacobi sweep fused (into Q), then 3 damped sweeps Q -> W -> Q -> W
        if (!fused_r) {
            timer_.time(KS_K_RESIDUAL, k, 0, (16.0 * k + 4.0) * npts, lane.s, [&] {
                launch_residual_precond(L_, k, ch.HX.at(0), ch.X(), theta_d, V, lambda_d, diag_t, ch.T.at(0), ch.Q.at(0), norm_partials,
                                        nb, lane.s, (float)omega, ch.HX.at(0));
            });
            norm_blocks = nb;
        }
        fused_r = false;
        // the active columns [locked, k): under a lock W and P exist for them only, W_a at [k, k + na) and P_a after it
        const int na = k - locked;
        const int m = k + na + np;
        const int off_norm = m * 2 * m;
        StencilArgs jac;
        jac.mode = ST_JACOBI;
        jac.scale = ham_scale;
        jac.V = V;
        jac.R = ch.T.at(locked);
        jac.lambda = lambda_d + locked;
        jac.omega = (float)omega;
        jac.diag_t = (float)diag_t;
        jac.dinv = ch.HX.at(locked);  // the sweep factors of this iteration (H X itself is not needed past the residual)
        jac.vec0 = locked;
        const double jac_bytes = (16.0 * na + 4.0) * npts;  // w, r and the stored factor in, w' out, V once
        timer_.time(KS_K_JACOBI, na, 0, jac_bytes, lane.s, [&] { launch_stencil(L_, ch.Q.tmap, na, jac, S.at(k), lane.s); });   // Q -> W
        jac.vec0 = k;
        timer_.time(KS_K_JACOBI, na, 0, jac_bytes, lane.s, [&] { launch_stencil(L_, S.tmap, na, jac, ch.Q.at(locked), lane.s); });   // W -> Q
        jac.vec0 = locked;
        timer_.time(KS_K_JACOBI, na, 0, jac_bytes, lane.s, [&] { launch_stencil(L_, ch.Q.tmap, na, jac, S.at(k), lane.s); });   // Q -> W
        // 2. HW and HP in one launch (W and P are contiguous after X)
        apply_h(S, k, na + np, ch.T.at(k));
        // 3. the readback: G = S^T [S | T] and |r_i|^2
        FinishDesc norms;
        norms.partials = norm_partials;
        norms.blocks = norm_blocks;
        norms.nvals = k;
        norms.scale = L_.h * L_.h * L_.h;
        norms.out = lane.red.res() + off_norm;
        gram_checked(lane.red, m, S.at(0), m, ch.T.at(0), &norms);
        const double* g = lane.red.read(off_norm + k);
        const int mc = 2 * m;
        std::vector<double> A((size_t)m * m), B((size_t)m * m);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j <= i; ++j) {
                double bv = g[(size_t)i * mc + j];
                double av = g[(size_t)i * mc + m + j];
                if (j < k) av += theta[j] * bv;  // <s_i, H x_j> = <s_i, r_j> + theta_j <s_i, x_j>
                B[(size_t)i * m + j] = B[(size_t)j * m + i] = bv;
                A[(size_t)i * m + j] = A[(size_t)j * m + i] = av;
            }
        for (double x : A)
            if (!std::isfinite(x)) throw NumericalError("lobpcg: non-finite Gram entry (NaN in a vector or in V)");
        for (double x : B)
            if (!std::isfinite(x)) throw NumericalError("lobpcg: non-finite Gram entry (NaN in a vector or in V)");
        // the split stop test (crates/qm-gpu/src/eigen.rs:768-787): the head at tol, [head, checked) scaled by
        // tol / tail_tol, the rest untested; lock_res the same over the tail alone (a lock holds exactly the head)
        double max_res = 0.0, stop_res = 0.0, lock_res = 0.0, head_res = 0.0, tail_res = 0.0;
        for (int i = 0; i < k; ++i) {
            double xx = B[(size_t)i * m + i];
            lambda[i] = A[(size_t)i * m + i] / xx;
            res[i] = std::sqrt(g[off_norm + i] / xx);
            if (!std::isfinite(res[i]) || !std::isfinite(lambda[i])) throw NumericalError("lobpcg: non-finite residual");
            max_res = std::max(max_res, res[i]);
            if (i < head) head_res = std::max(head_res, res[i]);
            else if (i < checked) tail_res = std::max(tail_res, res[i]);
            if (i < checked) {
                const double scaled = i < head ? res[i] : res[i] * (tol / tail_tol);
                stop_res = std::max(stop_res, scaled);
                if (i >= head) lock_res = std::max(lock_res, scaled);
            }
        }
        ch.evals = lambda;
        ch.res = res;
        // formation check (crates/qm-gpu/src/eigen.rs:800-825): undo a step whose moved columns' stored
        // Rayleigh quotients rose above their Ritz values
        if (have_prev) {
            have_prev = false;
            double rise = 0.0, slack = 0.0;
            for (int i = locked; i < k; ++i) {  // the moved columns
                rise += lambda[i] - theta[i];
                slack += RITZ_FORM_SLACK * (1.0 + std::fabs(theta[i])) + RITZ_FORM_RES * res[i];
            }
            bool bad = !(rise <= slack);
            if (bad && trace)
                std::fprintf(stderr, "lobpcg%s it %d: a Ritz vector does not match its Ritz value (rise %.3e, slack %.3e); the step is redone without P\n",
                             tag, iterations, rise, slack);
            if (bad && es.restores >= MAX_FORM_RESTORES) es.restores_exhausted = true;
            if (bad && es.restores < MAX_FORM_RESTORES) {
                ++es.restores;
                ch.cur ^= 1;
                theta = prev_theta;
                for (int i = locked; i < k; ++i) lambda[i] = theta[i];
                np = 0;
                upload(theta, lambda, nullptr);
                apply_h(ch.A[ch.cur], 0, k, ch.HX.at(0));
                continue;
            }
        }
        // the lock (crates/qm-gpu/src/eigen.rs:814-818): at the guess, a head under guess_tol whose tail is not. Y stays
        // where it is in both X buffers (copied into the other once here); the block update writes the other columns.
        if (lock && iterations == 0 && locked == 0 && head > 0 && head < checked && head_res < guess_tol && !(stop_res < guess_tol) &&
            std::isfinite(stop_res)) {
            locked = head;
            KS_CUDA(cudaMemcpyAsync(ch.A[ch.cur ^ 1].at(0), ch.A[ch.cur].at(0), (size_t)locked * L_.F * sizeof(float),
                                    cudaMemcpyDeviceToDevice, lane.s));
        }
        if (locked > 0) stop_res = lock_res;  // the stop test reads the active columns
        if (stop_res < 0.5 * best) { best = stop_res; best_it = iterations; }
        // stop decision (crates/qm-gpu/src/eigen.rs:322-329)
        int stop = -1;
        if (stop_res < tol || (iterations == 0 && stop_res < guess_tol)) stop = 0;
        else if (stop_res <= FLOOR_BAND * floor_ && iterations - best_it >= STALL_WINDOW) stop = 1;
        else if (iterations >= max_iter) stop = 2;
        if (stop >= 0) {
            es.iterations = iterations;
            es.max_residual = max_res;
            es.stop = stop;
            es.head_res = head_res;
            es.tail_res = split ? tail_res : 0.0;
            es.head_kept = iterations == 0 || locked > 0;
            es.locked = locked;
            if (trace) {
                std::fprintf(stderr, "lobpcg%s exit: iterations %d, max residual %.3e, stop %d, restores %d, fallbacks %d, evals", tag,
                             iterations, max_res, stop, es.restores, es.fallbacks);
                for (int i = 0; i < k; ++i) std::fprintf(stderr, " %.10f", lambda[i]);
                std::fprintf(stderr, "\n");
            }
            break;
        }
        ++iterations;
        auto t_dense = clk::now();
        // 4. Rayleigh-Ritz with the conditioning guard; fallback: drop P and redo on [X, W]
        // (under a lock: the subspace B-orthogonal to Y, the na = k - locked active columns' pairs)
        const int na_rr = k - locked;
        std::vector<double> th, C;
        double alpha = rayleigh_ritz_locked(m, A, B, locked, na_rr, th, C);
        es.alpha_worst = std::max(es.alpha_worst, alpha);
        if (trace) std::fprintf(stderr, "lobpcg%s it %d: max_res %.2e alpha %.2f m %d locked %d\n", tag, iterations, max_res, alpha, m, locked);
        // the noise budget: the tested columns' split residual, or under a lock the active tail's own (unscaled) one
        // (crates/qm-gpu/src/eigen.rs:861-867)
        const double budget_res = locked > 0 ? tail_res : stop_res;
        if (!(alpha <= std::max(ALPHA_MAX, ALPHA_RESIDUAL_FRACTION * budget_res / floor_)) && np > 0) {
            ++es.fallbacks;
            const int m2 = k + na_rr;  // [X, W_a]
            std::vector<double> A2((size_t)m2 * m2), B2((size_t)m2 * m2);
            for (int i = 0; i < m2; ++i)
                for (int j = 0; j < m2; ++j) { A2[(size_t)i * m2 + j] = A[(size_t)i * m + j]; B2[(size_t)i * m2 + j] = B[(size_t)i * m + j]; }
            std::vector<double> C2;
            rayleigh_ritz_locked(m2, A2, B2, locked, na_rr, th, C2);
            C.assign((size_t)m * na_rr, 0.0);
            for (int c = 0; c < na_rr; ++c)
                for (int i = 0; i < m2; ++i) C[i + (size_t)m * c] = C2[i + (size_t)m2 * c];
        }
        // 5. X_new = S C, P_new = X_new - X (X^T X)^-1 X^T X_new = S C_p (X all k columns, Y included)
        std::vector<double> bxx((size_t)k * k), rhs((size_t)k * na_rr, 0.0);
        for (int i = 0; i < k; ++i)
            for (int j = 0; j < k; ++j) bxx[(size_t)i * k + j] = B[(size_t)i * m + j];
        if (!dense::cholesky(k, bxx)) throw NumericalError("lobpcg: Cholesky of X^T X failed (X lost rank)");
        for (int i = 0; i < k; ++i)
            for (int c = 0; c < na_rr; ++c) {
                double s = 0.0;
                for (int j = 0; j < m; ++j) s += B[(size_t)i * m + j] * C[j + (size_t)m * c];
                rhs[(size_t)i * na_rr + c] = s;
            }
        dense::cholesky_solve(k, bxx, na_rr, rhs);
        std::vector<double> coef((size_t)m * 2 * na_rr);
        for (int c = 0; c < na_rr; ++c)
            for (int i = 0; i < m; ++i) {
                coef[i + (size_t)m * c] = C[i + (size_t)m * c];
                coef[i + (size_t)m * (na_rr + c)] = C[i + (size_t)m * c] - (i < k ? rhs[(size_t)i * na_rr + c] : 0.0);
            }
        prev_theta = theta;
        have_prev = true;
        for (int a = 0; a < na_rr; ++a) theta[locked + a] = th[a];
        lane.dense_s += secs(t_dense);
        upload(theta, lambda, &coef);
        const int next = ch.cur ^ 1;
        // X_a to [locked, k) and P_a to [k + na, k + 2 na) of the other buffer: outputs from the base at column
        // `locked`, the P outputs (from na on) shifted by a gap of na
        timer_.time(KS_K_BLOCK_UPDATE, m, 2 * na_rr, 4.0 * (m + 2 * na_rr) * npts, lane.s, [&] {
            launch_block_lincomb(L_.F, m, S.at(0), 2 * na_rr, coef_d, ch.A[next].at(locked), na_rr, na_rr, lane.s);
        });
        ch.cur = next;
        np = na_rr;
        // 6. HX of the new X -- with the next iteration's residual, first sweep and |r|^2 partials formed in the same pass
        if (!nl_on_) {
            StencilArgs a;
            a.mode = ST_HAM_RESIDUAL;
            a.scale = ham_scale;
            a.V = V;
            a.theta = theta_d;
            a.lambda = lambda_d;
            a.diag_t = (float)diag_t;
            a.out2 = ch.Q.at(0);
            a.omega = (float)omega;
            a.dinv = ch.HX.at(0);
            a.dot_partials = norm_partials;
            timer_.time(KS_K_HPSI_RESIDUAL, k, 0, (16.0 * k + 4.0) * npts, lane.s,  // x in; r, w0, factors out; V once
                        [&] { launch_stencil(L_, ch.A[ch.cur].tmap, k, a, ch.T.at(0), lane.s); });
            fused_r = true;
            norm_blocks = cpv;
        } else {
            apply_h(ch.A[ch.cur], 0, k, ch.HX.at(0));
        }
    }
    es.readbacks = lane.red.readbacks - rb0;
    return es;
}

// The Fermi-Dirac channel solve (crates/qm-gpu/src/scf.rs:875-1029, the CPU's qm::scf::solve_fd rule plus the GPU's
// buffer and step-accuracy tail). The block's lowest `tight` columns are held to the step's tol, the others below the top
// to the guard tolerance max(1e-3, step tol) and the top one is an untested buffer while one fits below the cap (a block
// of n + 1 first gets one more vector); the LOBPCG locks a converged head while only the loose columns move. Then:
// - the swap edge: an untested column that buffer_last moved into the tested range is re-solved, at most twice, toward
//   the guard tolerance;
// - the class raise: the tight count is re-read on the lower bounds (tight_columns at the SCF's tol); a solve whose head
//   was too small is repeated with the larger one;
// - the witness on the tested levels' lower bounds theta - r (36 kT, or the loosened step's tail): on a tight step a top
//   tested level that exits above 1.5 x the guard tolerance decides only through the lowest level that passes at or
//   below it (witness_keep_within), else the block grows by one; once witnessed, the overshoot above the lowest witness
//   is trimmed, keeping the next level as the buffer when one fits, never below the configured N_sigma + n_extra;
// - the buffer as the witness: a buffer whose own bound passes decides at r <= the guard tolerance (and one fresh vector
//   becomes the next buffer), else the block grows by one;
// - otherwise the extra block doubles (grown_extras), at most the cap; at the cap the witness check at convergence
//   reports the missing witness.
// New vectors are the reference's initial orbitals with seed 1000 + 2 * index + spin.
Solver::FdOutcome Solver::solve_fd(int sp, const float* V, double step_tol, double guess_tol, bool loosened, double delta_rho_prev,
                                   double kt, double scf_tol, int n, int& kk, int& tight, const Nuc* dnuc, int nn) {
    FdOutcome out;
    Lane& lane = *lane_[sp];
    const int cap = std::min(witness_cap_, 64 - n);
    const int base = n + opt_.n_extra;
    const double guard_tol = std::max(WITNESS_GUARD_TOL, step_tol);
    const double r_witness = EIG_GUESS_FACTOR * WITNESS_GUARD_TOL;
    auto buffered = [&](int len) { return len >= n + 2 && len - n < cap; };
    auto grow_to = [&](int len) {
        resize_channel(sp, len, dnuc, nn, lane.s);
        kk = len;
    };
    if (kk == n + 1 && cap >= 2) grow_to(kk + 1);
    int swap_retries = 0;
    for (;;) {
        const int checked = buffered(kk) ? kk - 1 : kk;
        const int head = std::min(tight, checked);
        out.peak_block = std::max(out.peak_block, kk);
        const double tail_kt = loosened ? dense::fd_step_tail_kt(kk, delta_rho_prev) : 36.0;
        const EigenStats es = lobpcg(ch_[sp], lane, V, step_tol, guess_tol, EIGEN_MAX_ITER, head, guard_tol, checked, true);
        ++out.calls;
        out.iterations += es.iterations;
        if (es.restores_exhausted) throw NumericalError("LOBPCG: a Ritz-vector formation failed again after its restores");
        out.tight_res = es.head_res;
        out.maxiter = es.stop == 2;
        if (checked < kk) {
            const int moved = buffer_last(sp, lane.s);
            if (moved >= 0 && ch_[sp].res[moved] > guard_tol && swap_retries < 2) {
                ++swap_retries;
                continue;
            }
        }
        out.kept = out.kept && es.head_kept;
        if (es.head_kept && es.iterations > 0) ++out.locked_calls;
        const double* ev = ch_[sp].evals.data();
        const double* rv = ch_[sp].res.data();
        std::vector<double> f(checked);
        double mu = NAN, ent = 0.0;
        if (!dense::fermi_dirac(ev, checked, n, kt, f.data(), mu, ent)) throw NumericalError("Fermi-Dirac occupations refused (a non-finite level)");
        const int need = dense::fd_tight_columns(ev, rv, checked, mu, kt, scf_tol);
        tight = need;
        if (need > head) {
            ++out.class_raises;
            continue;  // a column held loose needs the step's tol: re-solve with it tight
        }
        out.tail_kt = std::max(out.tail_kt, tail_kt);
        const bool witness = dense::fd_witness(ev, rv, checked, n, mu, kt, tail_kt);
        int top = 0;
        for (int i = 1; i < checked; ++i)
            if (ev[i] > ev[top]) top = i;
        int keep = -1;
        if (witness && !loosened && rv[top] > r_witness && kk - n < cap) {
            keep = dense::fd_witness_keep_within(ev, rv, checked, n, mu, kt, tail_kt, r_witness);
            if (keep < 0) {
                ++out.residual_growths;
                grow_to(kk + 1);
                continue;
            }
            ++out.lower_witnesses;
        } else if (witness) {
            keep = dense::fd_witness_keep(ev, rv, checked, n, mu, kt, tail_kt);
        }
        if (keep >= 0) {
            const int len = std::max(base, buffered(keep + 1) ? keep + 1 : keep);
            if (len < kk) {
                // the lowest `len` levels by value, in their positions' order
                std::vector<int> order(kk);
                for (int i = 0; i < kk; ++i) order[i] = i;
                std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return ev[a] < ev[b]; });
                std::vector<int> cols(order.begin(), order.begin() + len);
                std::sort(cols.begin(), cols.end());
                resize_channel(sp, len, dnuc, nn, lane.s, &cols);
                kk = len;
                ++out.trims;
                if (buffered(len)) buffer_last(sp, lane.s);
            }
            out.checked = buffered(kk) ? kk - 1 : kk;
            out.witnessed = true;
            return out;
        }
        if (checked < kk && dense::fd_witness(ev, rv, kk, n, mu, kt, tail_kt)) {
            if (rv[kk - 1] <= WITNESS_GUARD_TOL) {
                ++out.buffer_witnesses;
                out.checked = checked;
                out.witnessed = true;
                if (kk - n < cap) grow_to(kk + 1);  // the next step's buffer
                return out;
            }
            if (kk - n < cap) {
                ++out.buffer_growths;
                grow_to(kk + 1);
                continue;
            }
        }
        const int extras = kk - n;
        if (extras >= cap) {
            out.checked = checked;
            return out;
        }
        ++out.growths;
        grow_to(n + dense::fd_grown_extras(extras, cap));
    }
}

double Solver::effective_eig_tol(double eig_tol) const { return std::max(eig_tol, EIG_TOL_FLOOR_FACTOR * floor_); }

ks_status Solver::solve(const ks_nucleus* nuc, int nn, int n_up, int n_dn, const ks_settings& s, bool warm, ks_abort_fn abort_fn,
                        void* user, ks_stats* out, ks_abort_fn inner_abort, ks_observe_fn observe) {
    NvtxRange range("ks solve");
    auto t0 = clk::now();
    inner_fn_ = inner_abort;
    inner_user_ = user;
    poll_thread_ = std::this_thread::get_id();
    inner_flag_.store(0);
    struct ClearInner {
        Solver* so;
        ~ClearInner() { so->inner_fn_ = nullptr; so->inner_user_ = nullptr; }
    } clear_inner{this};
    std::memset(out, 0, sizeof(*out));
    profile = ks_profile{};
    // the solver's own wait-timeout flag: kernels of this solve raise it, its readbacks read it, and a timeout left by an
    // earlier call is not blamed on this one
    ErrorFlagScope flag_scope(err_flag());
    KS_CUDA(cudaMemsetAsync(err_.p, 0, sizeof(int), s_));
    const int rb0 = readbacks_total();
    const double wait0 = wait_total();
    for (auto& l : lane_) l->dense_s = 0.0;
    if (nn < 0 || n_up < 0 || n_dn < 0 || (nn > 0 && !nuc)) { error = "invalid arguments"; return KS_INVALID; }
    const bool fd = s.occupations == 1;
    if (s.occupations < 0 || s.occupations > 1) { error = "occupations must be 0 (Aufbau) or 1 (Fermi-Dirac)"; return KS_INVALID; }
    if (fd && !(std::isfinite(s.kt) && s.kt > 0.0)) { error = "Fermi-Dirac needs a finite kt > 0"; return KS_INVALID; }
    if (fd && opt_.n_extra < 1) { error = "Fermi-Dirac needs n_extra >= 1 levels above N_sigma per channel (ks_options)"; return KS_INVALID; }
    if (fd && std::max(n_up, n_dn) + opt_.n_extra > 64) { error = "Fermi-Dirac: at most 64 levels per channel"; return KS_INVALID; }
    if (nn > 32) { error = "at most 32 nuclei"; return KS_INVALID; }
    const bool ionic = ionic_.active();
    // E_nn (crates/qm/src/nuclear.rs:277-289); under a setup the valence charges (ionic_repulsion, :368-378)
    auto charge = [&](int a) { return ionic ? ionic_.charge_of(nuc[a].z) : (double)nuc[a].z; };
    double e_nn = 0.0;
    for (int i = 0; i < nn; ++i)
        for (int j = i + 1; j < nn; ++j) {
            double dx = nuc[i].pos[0] - nuc[j].pos[0], dy = nuc[i].pos[1] - nuc[j].pos[1], dz = nuc[i].pos[2] - nuc[j].pos[2];
            double d = std::sqrt(dx * dx + dy * dy + dz * dz);
            if (d < 1e-8) {
                error = "nuclei " + std::to_string(i) + " and " + std::to_string(j) + " coincide";
                converged_ = false;
                return KS_COINCIDENT_NUCLEI;
            }
            e_nn += charge(i) * charge(j) / d;
        }
    // under a setup each centre carries its charge q (Z_v or Z): the cold guess deposits q (nuclear.rs:195-206)
    std::vector<Nuc> hn(std::max(nn, 1));
    double z_tot = 0.0;
    for (int i = 0; i < nn; ++i) {
        hn[i] = Nuc{nuc[i].pos[0], nuc[i].pos[1], nuc[i].pos[2], charge(i)};
        z_tot += charge(i);
    }
    try {
        nuc_d_.alloc(hn.size() * sizeof(Nuc));
        KS_CUDA(cudaMemcpyAsync(nuc_d_.p, hn.data(), hn.size() * sizeof(Nuc), cudaMemcpyHostToDevice, s_));
        const Nuc* dnuc = static_cast<const Nuc*>(nuc_d_.p);
        const double dv = L_.h * L_.h * L_.h;
        const double eig_lo = std::max(s.eig_tol, EIG_TOL_FLOOR_FACTOR * floor_);
        const int nocc[2] = {n_up, n_dn};
        int kk[2];
        for (int sp = 0; sp < 2; ++sp) kk[sp] = nocc[sp] > 0 ? nocc[sp] + opt_.n_extra : 0;
        bool reuse = warm && have_warm_ && fd_state_ == fd && nocc_[0] == n_up && nocc_[1] == n_dn && state_gen_ == ionic_gen();
        // under Fermi-Dirac a warm block may have grown for its gap witness: it is reused at its size
        for (int sp = 0; sp < 2 && reuse; ++sp)
            if (fd && kk[sp] > 0 ? ch_[sp].k < kk[sp] : ch_[sp].k != kk[sp]) reuse = false;
        if (reuse && fd)
            for (int sp = 0; sp < 2; ++sp) kk[sp] = ch_[sp].k;
        // columns held to the eigen tolerance: N_sigma; under Fermi-Dirac a warm state's start is the positions its stored
        // occupations need at the SCF's tol (tight_start, crates/qm-gpu/src/scf.rs:1290-1295), and every channel solve
        // re-reads it on its own levels
        int tight[2] = {nocc[0], nocc[1]};
        if (reuse && fd)
            for (int sp = 0; sp < 2; ++sp)
                if (nocc[sp] > 0 && (int)occ_[sp].size() == kk[sp]) tight[sp] = dense::fd_tight_start(occ_[sp].data(), kk[sp], nocc[sp], s.tol);
        double entropy = 0.0, mu[2] = {NAN, NAN};
        bool partial = false;
        occ_d_.alloc(2 * 64 * sizeof(double));
        converged_ = false;
        have_warm_ = false;
        auto t_start = clk::now();
        if (!reuse) {
            for (int sp = 0; sp < 2; ++sp) {
                ensure_channel(sp, kk[sp]);
                if (kk[sp] > 0) {
                    ch_[sp].cur = 0;
                    launch_initial_orbitals(L_, dnuc, nn, kk[sp], (unsigned long long)(sp + 1), opt_.init_mode, ch_[sp].X(), s_);
                    ch_[sp].evals.assign(kk[sp], -1.0);
                    ch_[sp].res.assign(kk[sp], std::nan(""));
                }
            }
            const double total = (double)(n_up + n_dn);
            const double scale = z_tot > 0.0 ? total / z_tot : 0.0;
            const double fu = total > 0.0 ? n_up / total : 0.0, fd = total > 0.0 ? n_dn / total : 0.0;
            // the Aufbau cold density: sigma = 1 Bohr blobs of each nucleus' charge (crates/qm/src/nuclear.rs:212-214)
            launch_deposit_charge(L_, dnuc, nn, 1.0, scale * fu, in_up_.at(0), s_);
            launch_deposit_charge(L_, dnuc, nn, 1.0, scale * fd, in_dn_.at(0), s_);
            launch_fill(vh_.at(0), 0.0f, L_.F, s_);
        } else if (extrapolate_ && have_prev_) {
            // rho_in = max(2 rho_t - rho_{t-1}, 0) from the last two converged outputs (crates/qm-gpu/src/scf.rs:1146-1163)
            launch_extrapolate(L_.F, out_up_.at(0), prev_up_.at(0), in_up_.at(0), s_);
            launch_extrapolate(L_.F, out_dn_.at(0), prev_dn_.at(0), in_dn_.at(0), s_);
            profile.extrapolated = 1;
        } else {
            KS_CUDA(cudaMemcpyAsync(in_up_.at(0), out_up_.at(0), L_.F * sizeof(float), cudaMemcpyDeviceToDevice, s_));
            KS_CUDA(cudaMemcpyAsync(in_dn_.at(0), out_dn_.at(0), L_.F * sizeof(float), cudaMemcpyDeviceToDevice, s_));
        }
        // rho_{t-1} for the next warm start: this solve's starting output, kept only if this solve is warm and converges
        have_prev_ = false;
        if (extrapolate_ && reuse) {
            if (prev_up_.count == 0) { prev_up_.create(L_, 1); prev_dn_.create(L_, 1); }
            KS_CUDA(cudaMemcpyAsync(prev_up_.at(0), out_up_.at(0), L_.F * sizeof(float), cudaMemcpyDeviceToDevice, s_));
            KS_CUDA(cudaMemcpyAsync(prev_dn_.at(0), out_dn_.at(0), L_.F * sizeof(float), cudaMemcpyDeviceToDevice, s_));
        }
        const bool keep_prev = extrapolate_;
        nocc_[0] = n_up;
        nocc_[1] = n_dn;
        const float* pc = nullptr;
        nl_on_ = false;
        if (ionic) {
            // V_loc = sum V_LR + sum V_SR, the partial core, the projector spheres (crates/qm/src/scf.rs:720-745)
            ionic_.update(L_, nuc, nn, s.sigma, s_);
            ionic_.local_potential(L_, vnuc_.at(0), s_);
            if (ionic_.has_core()) {
                if (pc_.count == 0) pc_.create(L_, 1);
                ionic_.partial_core(L_, pc_.at(0), s_);
                pc = pc_.at(0);
            }
            nl_on_ = ionic_.has_nl();
        } else {
            launch_nuclear_potential(L_, dnuc, nn, s.sigma, vnuc_.at(0), s_);
        }
        state_gen_ = ionic_gen();
        if (!reuse) KS_CUDA(cudaStreamSynchronize(s_));
        profile.start_s = reuse ? 0.0 : secs(t_start);

        // DIIS history (crates/qm-gpu/src/scf.rs:558-646) in a pool of field quadruples
        const int cap = std::max(s.diis_history, 1);
        if ((int)diis_pool_.size() < cap + 1) {
            diis_pool_.resize(cap + 1);
            for (auto& e : diis_pool_)
                if (e.r_up.count == 0) { e.rho_up.create(L_, 1); e.rho_dn.create(L_, 1); e.r_up.create(L_, 1); e.r_dn.create(L_, 1); }
        }
        std::vector<int> hist, free_list;
        for (int i = (int)diis_pool_.size() - 1; i >= 0; --i) free_list.push_back(i);
        std::vector<std::vector<double>> gram;
        auto drop_oldest = [&]() {
            free_list.push_back(hist.front());
            hist.erase(hist.begin());
            gram.erase(gram.begin());
            for (auto& r : gram) r.erase(r.begin());
        };

        // SCF_TRACE in the environment, set to any value, prints one line per SCF step to stderr (the reference's switch,
        // crates/qm-gpu/src/scf.rs:1281)
        static const bool trace = std::getenv("SCF_TRACE") != nullptr;
        int iterations = 0;
        double delta_rho = INFINITY, test_tol = s.tol;
        double q_out[2] = {0, 0};
        bool frozen = false, stalled = false;
        // Fermi-Dirac (crates/qm-gpu/src/scf.rs:1370-1374): this step's calls all returned their tight columns bitwise; the
        // DIIS entries measured on the current frozen orbitals' output; the previous step's widest witness tail; the
        // tested levels per channel (the buffer above them holds no charge) and whether a witness decided each channel
        bool step_kept = false;
        int consistent = 0, step_growths = 0;
        double prev_tail = INFINITY, step_tail = 0.0;
        int fd_checked[2] = {0, 0};
        bool fd_witnessed[2] = {false, false};
        double anchor = INFINITY, best = INFINITY;
        int anchor_at = 0;
        const double level = STALL_LEVEL_PER_ELECTRON * (n_up + n_dn);
        double max_eig_res = 0.0, last_step_res = 0.0, pois_res = 0.0;
        int pois_it_max = 0;
        bool last_step_maxiter = false;
        // park the iterate (orbitals, evals, input densities) as the next warm start and report the abort
        auto park = [&](const std::string& why) {
            have_warm_ = true;
            fd_state_ = fd;
            KS_CUDA(cudaMemcpyAsync(out_up_.at(0), in_up_.at(0), L_.F * sizeof(float), cudaMemcpyDeviceToDevice, s_));
            KS_CUDA(cudaMemcpyAsync(out_dn_.at(0), in_dn_.at(0), L_.F * sizeof(float), cudaMemcpyDeviceToDevice, s_));
            KS_CUDA(cudaStreamSynchronize(s_));
            profile.steps = iterations;
            profile.readbacks = readbacks_total() - rb0;
            profile.host_dense_s = lane_[0]->dense_s + lane_[1]->dense_s;
            profile.sync_wait_s = wait_total() - wait0;
            profile.wall_s = secs(t0);
            error = why;
            return KS_ABORTED;
        };
        while (iterations < s.max_iter) {
            if (abort_fn && abort_fn(user)) return park("abandoned before SCF step " + std::to_string(iterations + 1));
            ++iterations;
            profile.steps = iterations;  // also what a failed solve's profile reports
            NvtxRange step_range("ks scf step");
            // a warm guess is accepted within the 1.5x band only in the convergence phase (the previous step's dRho
            // already below tol); before that only within the step's own tol. This is the reference's rule for its
            // Fermi-Dirac channels (crates/qm-gpu/src/scf.rs module doc, "The guess band only in the convergence
            // phase"); its Aufbau path keeps the band on every step, where a head that hovers at the band edge
            // alternates frozen / re-solved, resets DIIS every other step and can stall at dRho ~1e-4 (10 of 64
            // jittered batch molecules); with the rule all 64 converge in fewer steps.
            const double guess_factor = delta_rho < test_tol ? EIG_GUESS_FACTOR : 1.0;
            const double step_tol = delta_rho < test_tol ? eig_lo
                                                         : (std::isfinite(delta_rho) ? std::min(std::max(EIG_TOL_FRACTION * delta_rho, eig_lo),
                                                                                                std::max(EIG_TOL_MAX, eig_lo))
                                                                                       : eig_lo);
            // Hartree potential of rho_in
            Terms tsum;
            tsum.count = 2;
            tsum.x[0] = in_up_.at(0); tsum.c[0] = 1.f;
            tsum.x[1] = in_dn_.at(0); tsum.c[1] = 1.f;
            launch_lincomb(L_.F, 1, rho_tot_.at(0), tsum, s_);
            auto tp = clk::now();
            PoissonStats ps = poisson_.solve(rho_tot_.at(0), vh_.at(0), vh_.tmap, POISSON_TOL, POISSON_MAX_ITER);
            profile.poisson_s += secs(tp);
            profile.poisson_iterations += ps.iterations;
            pois_res = std::max(pois_res, ps.residual);
            pois_it_max = std::max(pois_it_max, ps.iterations);
            if (ps.stop == 3) ++out->n_warnings;
            // XC and the effective potentials
            if (observe && xcu_.count == 0) { xcu_.create(L_, 1); xcd_.create(L_, 1); }
            launch_xc_veff(L_.F, in_up_.at(0), in_dn_.at(0), vnuc_.at(0), vh_.at(0), exc_.at(0), v_up_.at(0), v_dn_.at(0),
                           observe ? xcu_.at(0) : nullptr, observe ? xcd_.at(0) : nullptr, s_, pc);
            // eigensolves
            int eig_its = 0;
            last_step_res = 0.0;
            last_step_maxiter = false;
            auto te = clk::now();
            // the two spin channels are independent: each runs on its own lane (stream, reducer) and,
            // when both are occupied, the down channel on a second host thread, so one channel's
            // kernels fill the GPU while the other waits on a readback or does its host algebra
            EigenStats est[2];
            FdOutcome fdo[2];
            {
                KS_CUDA(cudaEventRecord(ev_fork_, s_));
                for (auto& l : lane_) KS_CUDA(cudaStreamWaitEvent(l->s, ev_fork_, 0));
                auto run = [&](int sp) {
                    const float* vv = sp ? v_dn_.at(0) : v_up_.at(0);
                    if (fd)
                        fdo[sp] = solve_fd(sp, vv, step_tol, guess_factor * step_tol, step_tol > eig_lo, delta_rho, s.kt, s.tol, nocc[sp],
                                           kk[sp], tight[sp], dnuc, nn);
                    else
                        est[sp] = lobpcg(ch_[sp], *lane_[sp], vv, step_tol, guess_factor * step_tol, EIGEN_MAX_ITER, nocc[sp]);
                };
                std::exception_ptr err_dn;
                std::thread worker;
                // under kernel timing the channels run one after the other, so that each launch is timed alone
                const bool both = nocc[0] > 0 && nocc[1] > 0 && !timer_.on();
                if (both)
                    worker = std::thread([&] {
                        ErrorFlagScope worker_flag(err_flag());
                        try {
                            KS_CUDA(cudaSetDevice(dev_));
                            run(1);
                        } catch (...) {
                            err_dn = std::current_exception();
                        }
                    });
                std::exception_ptr err_up;
                try {
                    if (nocc[0] > 0) run(0);
                    if (!both && nocc[1] > 0) run(1);
                } catch (...) {
                    err_up = std::current_exception();
                }
                if (worker.joinable()) {
                    if (err_up) inner_flag_.store(1);  // the other channel leaves at its next iteration
                    worker.join();
                }
                for (auto& l : lane_) {
                    KS_CUDA(cudaEventRecord(l->ev_join, l->s));
                    KS_CUDA(cudaStreamWaitEvent(s_, l->ev_join, 0));
                }
                auto is_abort = [](std::exception_ptr e) {
                    try {
                        std::rethrow_exception(e);
                    } catch (const AbortInside&) {
                        return true;
                    } catch (...) {
                        return false;
                    }
                };
                // a real error wins over the abort it triggered in the other channel
                if (err_up && !is_abort(err_up)) std::rethrow_exception(err_up);
                if (err_dn && !is_abort(err_dn)) std::rethrow_exception(err_dn);
                if (err_up || err_dn) return park("abandoned inside SCF step " + std::to_string(iterations) + " (an eigensolve)");
            }
            step_kept = true;
            step_growths = 0;
            step_tail = 0.0;
            for (int sp = 0; sp < 2; ++sp) {
                if (nocc[sp] == 0) continue;
                if (fd) {
                    // the step's FD bookkeeping (crates/qm-gpu/src/scf.rs:1436-1438, SolveProfile's counters)
                    const FdOutcome& o = fdo[sp];
                    profile.eigen_calls += o.calls;
                    profile.eigen_iterations += o.iterations;
                    eig_its += o.iterations;
                    if (step_tol <= eig_lo) max_eig_res = std::max(max_eig_res, o.tight_res);
                    last_step_res = std::max(last_step_res, o.tight_res);
                    if (o.maxiter) last_step_maxiter = true;
                    step_kept = step_kept && o.kept;
                    step_growths += o.growths;
                    step_tail = std::max(step_tail, o.tail_kt);
                    fd_checked[sp] = o.checked;
                    fd_witnessed[sp] = o.witnessed;
                    profile.witness_growths += o.growths;
                    profile.locked_calls += o.locked_calls;
                    profile.class_raises += o.class_raises;
                    profile.buffer_witnesses += o.buffer_witnesses;
                    profile.buffer_growths += o.buffer_growths;
                    profile.lower_witnesses += o.lower_witnesses;
                    profile.witness_residual_growths += o.residual_growths;
                    profile.witness_trims += o.trims;
                    profile.peak_block = std::max(profile.peak_block, o.peak_block);
                    continue;
                }
                const EigenStats& es = est[sp];
                ++profile.eigen_calls;
                profile.eigen_iterations += es.iterations;
                eig_its += es.iterations;
                if (es.restores_exhausted) throw NumericalError("LOBPCG: a Ritz-vector formation failed again after its restores");
                const double tight_r = es.max_residual;
                if (step_tol <= eig_lo) max_eig_res = std::max(max_eig_res, tight_r);
                last_step_res = std::max(last_step_res, tight_r);
                if (es.stop == 2) last_step_maxiter = true;
            }
            profile.eigen_s += secs(te);
            // occupations of this step's levels (crates/qm/src/scf.rs:996-1013): Aufbau 1 on the N_sigma lowest (the block
            // is sorted by Ritz value), Fermi-Dirac f over the whole block, never mixed between steps
            entropy = 0.0;
            partial = false;
            double occ_host[2 * 64] = {0.0};
            for (int sp = 0; sp < 2; ++sp) {
                occ_[sp].assign(kk[sp], 0.0);
                mu[sp] = NAN;
                if (kk[sp] == 0) continue;
                if (!fd) {
                    for (int i = 0; i < nocc[sp]; ++i) occ_[sp][i] = 1.0;
                    continue;
                }
                // the tested levels (the untested buffer above them, if any, gets f = 0)
                double s_sp = 0.0;
                const int nt = std::max(nocc[sp] + 1, std::min(fd_checked[sp], kk[sp]));
                if (!dense::fermi_dirac(ch_[sp].evals.data(), nt, nocc[sp], s.kt, occ_[sp].data(), mu[sp], s_sp))
                    throw NumericalError("Fermi-Dirac occupations refused (a non-finite level)");
                entropy += s_sp;
                for (int i = 0; i < kk[sp]; ++i) {
                    partial = partial || std::min(occ_[sp][i], 1.0 - occ_[sp][i]) >= PARTIAL_OCCUPATION_MIN;
                    occ_host[64 * sp + i] = occ_[sp][i];
                }
            }
            if (fd) KS_CUDA(cudaMemcpyAsync(occ_d_.p, occ_host, sizeof(occ_host), cudaMemcpyHostToDevice, s_));
            // output densities, residuals, dRho, output charges and the new DIIS Gram row in one readback
            const int fe = free_list.back();
            Entry& E = diis_pool_[fe];
            const int nb = red_.blocks();
            for (int sp = 0; sp < 2; ++sp) {
                const Block& in = sp ? in_dn_ : in_up_;
                Block& outb = sp ? out_dn_ : out_up_;
                Block& r = sp ? E.r_dn : E.r_up;
                if (nocc[sp] > 0)
                    launch_density_residual(L_.F, fd ? kk[sp] : nocc[sp], ch_[sp].X(), fd ? occ_d_.d() + 64 * sp : nullptr, in.at(0),
                                            outb.at(0), r.at(0), red_.partials(), nb, s_);
                else
                    launch_density_residual(L_.F, 0, in.at(0), nullptr, in.at(0), outb.at(0), r.at(0), red_.partials(), nb, s_);
                launch_finish(red_.partials(), nb, 2, dv, red_.res() + 2 * sp, s_);
            }
            std::vector<std::pair<const float*, const float*>> pairs;
            for (int e : hist) {
                pairs.push_back({E.r_up.at(0), diis_pool_[e].r_up.at(0)});
                pairs.push_back({E.r_dn.at(0), diis_pool_[e].r_dn.at(0)});
            }
            pairs.push_back({E.r_up.at(0), E.r_up.at(0)});
            pairs.push_back({E.r_dn.at(0), E.r_dn.at(0)});
            red_.dots(pairs, 4, dv);
            // observed solves only: the Harris-Foulkes double counting of rho_in rides on this readback
            // (int rho_in V_H, int rho_in,sigma v_xc,sigma, E_xc[rho_in]; crates/qm-gpu/src/scf.rs:1500-1505)
            const int hf_off = 4 + (int)pairs.size();
            if (observe)
                red_.dots({{rho_tot_.at(0), vh_.at(0)}, {in_up_.at(0), xcu_.at(0)}, {in_dn_.at(0), xcd_.at(0)}, {exc_.at(0), ones_.at(0)}},
                          hf_off, dv);
            const double* h = red_.read(hf_off + (observe ? 4 : 0));
            delta_rho = h[0] + h[2];
            q_out[0] = h[1];
            q_out[1] = h[3];
            std::vector<double> row;
            for (size_t q = 0; q + 1 < pairs.size(); q += 2) row.push_back(h[4 + q] + h[5 + q]);
            if (trace) {
                // the reference's SCF trace line (crates/qm-gpu/src/scf.rs:1509-1512), plus the occupied eigenvalues
                std::fprintf(stderr, "scf step %d: dRho %.3e (up %.2e dn %.2e), DIIS history %zu, eig tol %.2e, eigen last-step residual %.2e, eigen it this step %d, evals",
                             iterations, delta_rho, h[0], h[2], hist.size(), step_tol, last_step_res, eig_its);
                for (int sp = 0; sp < 2; ++sp) {
                    std::fprintf(stderr, " %s", sp ? "| dn" : "up");
                    for (size_t i = 0; i < ch_[sp].evals.size() && nocc[sp] > 0; ++i)
                        std::fprintf(stderr, "%s%.6f", (int)i == nocc[sp] ? " / " : " ", ch_[sp].evals[i]);
                }
                std::fprintf(stderr, "\n");
            }
            // stall watch (crates/qm/src/scf.rs:440-480)
            if (delta_rho < best) best = delta_rho;
            if (std::isfinite(delta_rho) && (!std::isfinite(anchor) || delta_rho <= 0.5 * anchor)) { anchor = delta_rho; anchor_at = iterations; }
            const int since = iterations - anchor_at;
            if (observe) {
                // qm::ScfProgress (crates/qm/src/scf.rs:488-498): F_HF = sum f eps + double counting - kT S, Neumaier sums
                auto neumaier = [](const std::vector<double>& v) {
                    double sum = 0.0, comp = 0.0;
                    for (double x : v) {
                        const double t = sum + x;
                        if (std::fabs(sum) >= std::fabs(x)) comp += (sum - t) + x; else comp += (x - t) + sum;
                        sum = t;
                    }
                    return sum + comp;
                };
                std::vector<double> band;
                for (int sp = 0; sp < 2; ++sp)
                    for (int i = 0; i < (int)occ_[sp].size() && i < (int)ch_[sp].evals.size(); ++i) band.push_back(occ_[sp][i] * ch_[sp].evals[i]);
                const double dc = neumaier({-0.5 * h[hf_off], -h[hf_off + 1], -h[hf_off + 2], h[hf_off + 3], e_nn});
                ks_progress pg{};
                pg.iteration = iterations;
                pg.max_iter = s.max_iter;
                pg.delta_rho = delta_rho;
                pg.tol = s.tol;
                pg.energy = neumaier(band) + dc - (fd ? s.kt * entropy : 0.0);
                pg.best_delta_rho = best;
                pg.since_gain = since;
                pg.window = s.stall_window;
                pg.stall_level = level;
                observe(&pg, user);
            }
            test_tol = (fd && partial) ? std::max(s.tol, GPU_PARTIAL_TOL) : s.tol;
            if (!std::isfinite(delta_rho) || (delta_rho < test_tol && step_tol <= eig_lo)) break;
            if (!(delta_rho < test_tol) && s.stall_window > 0 && since >= s.stall_window && best >= level) { stalled = true; break; }
            // DIIS restart when the map rho_in -> rho_out changed (crates/qm-gpu/src/scf.rs:1544-1569): a frozen orbital
            // set re-solved (under Fermi-Dirac frozen = every call returned its tight columns bitwise: a witness-only
            // iteration under a locked head moves nothing the density rests on), or a witness window that widened and
            // grew the block. A frozen Fermi-Dirac step that follows a frozen step and does not contract the residual by
            // the mixing's bound (||r_k||^2 > (1 - alpha)^2 ||r_k-1||^2) keeps only the entries measured on the frozen
            // output: the last unfrozen step's and the frozen steps' own.
            const bool step_frozen = fd ? step_kept : eig_its == 0;
            const bool widened = fd && step_tail > prev_tail && step_growths > 0;
            prev_tail = step_tail;
            const bool map_changed = ((frozen && !step_frozen) || widened) && !hist.empty();
            if (map_changed) ++profile.diis_resets;
            consistent = (fd && step_frozen) ? (frozen ? consistent + 1 : 2) : 0;
            const bool stalled_mix = !hist.empty() && row.back() > (1.0 - s.mixing) * (1.0 - s.mixing) * gram.back().back();
            const bool freeze_trim = fd && frozen && step_frozen && !map_changed && stalled_mix && (int)hist.size() + 1 > consistent;
            if (freeze_trim) ++profile.diis_freeze_trims;
            if (fd && step_frozen) ++profile.frozen_steps;
            frozen = step_frozen;
            // push: the entry takes the input densities; their old buffers receive the mix
            free_list.pop_back();
            std::swap(E.rho_up, in_up_);
            std::swap(E.rho_dn, in_dn_);
            if (map_changed) {
                while (!hist.empty()) drop_oldest();
                row.erase(row.begin(), row.end() - 1);
            } else if (freeze_trim) {
                const size_t m0 = hist.size(), keepn = std::min<size_t>((size_t)(consistent - 1), m0);
                while (hist.size() > keepn) drop_oldest();
                row.erase(row.begin(), row.begin() + (m0 - keepn));
            }
            for (size_t i = 0; i < gram.size(); ++i) gram[i].push_back(row[i]);
            gram.push_back(row);
            hist.push_back(fe);
            if ((int)hist.size() > cap) drop_oldest();
            // coefficients: drop the oldest entries while the bordered solve fails
            std::vector<double> c;
            for (;;) {
                const int m = (int)hist.size();
                if (m == 1) { c.assign(1, 1.0); break; }
                dense::Mat gm((size_t)m * m);
                for (int i = 0; i < m; ++i)
                    for (int j = 0; j < m; ++j) gm[(size_t)i * m + j] = gram[i][j];
                if (dense::diis_coefficients(m, gm, c)) break;
                drop_oldest();
            }
            const int m = (int)hist.size();
            std::vector<const float*> rp(m), rr(m);
            std::vector<float> cf(m), af(m);
            for (int i = 0; i < m; ++i) { cf[i] = (float)c[i]; af[i] = (float)(s.mixing * c[i]); }
            for (int sp = 0; sp < 2; ++sp) {
                for (int i = 0; i < m; ++i) {
                    const Entry& e = diis_pool_[hist[i]];
                    rp[i] = sp ? e.rho_dn.at(0) : e.rho_up.at(0);
                    rr[i] = sp ? e.r_dn.at(0) : e.r_up.at(0);
                }
                launch_diis_mix(L_.F, m, rp.data(), rr.data(), cf.data(), af.data(), sp ? in_dn_.at(0) : in_up_.at(0), s_);
            }
            // charge renormalisation to the step's output charge, on the device
            red_.dots({{in_up_.at(0), ones_.at(0)}, {in_dn_.at(0), ones_.at(0)}}, 0, dv);
            if (n_up > 0) launch_scale_ratio(L_.F, in_up_.at(0), red_.res() + 0, q_out[0], s_);
            if (n_dn > 0) launch_scale_ratio(L_.F, in_dn_.at(0), red_.res() + 1, q_out[1], s_);
        }
        profile.steps = iterations;
        out->iterations = iterations;
        out->delta_rho = delta_rho;
        out->poisson_residual = pois_res;
        out->poisson_iterations = pois_it_max;
        out->max_eigen_residual = max_eig_res;
        out->tol_used = test_tol;
        if (stalled) {
            error = "SCF stalled: best dRho " + std::to_string(best) + " not improved 2x in " + std::to_string(s.stall_window) + " iterations";
            profile.readbacks = readbacks_total() - rb0;
            profile.host_dense_s = lane_[0]->dense_s + lane_[1]->dense_s;
            profile.sync_wait_s = wait_total() - wait0;
            profile.wall_s = secs(t0);
            return KS_STALLED;
        }
        if (!(delta_rho < test_tol)) {
            error = "SCF did not converge after " + std::to_string(iterations) + " iterations (dRho = " + std::to_string(delta_rho) + ")";
            profile.readbacks = readbacks_total() - rb0;
            profile.host_dense_s = lane_[0]->dense_s + lane_[1]->dense_s;
            profile.sync_wait_s = wait_total() - wait0;
            profile.wall_s = secs(t0);
            return KS_NOT_CONVERGED;
        }
        if (fd)
            for (int sp = 0; sp < 2; ++sp)
                if (nocc[sp] > 0 && !fd_witnessed[sp]) {  // the last step's channel solve found none below the cap
                    error = "no Fermi-Dirac gap witness in the block of " + std::to_string(kk[sp]) + " levels of spin " + std::to_string(sp) +
                            " (its top level must lie 0.1 Ha above level N and 36 kT above mu) within the witness cap of " +
                            std::to_string(witness_cap_) + " extra levels";
                    profile.wall_s = secs(t0);
                    return KS_NUMERICAL;
                }
        // --- energy from the output density and orbitals
        Terms tsum;
        tsum.count = 2;
        tsum.x[0] = out_up_.at(0); tsum.c[0] = 1.f;
        tsum.x[1] = out_dn_.at(0); tsum.c[1] = 1.f;
        launch_lincomb(L_.F, 1, rho_tot_.at(0), tsum, s_);
        auto tp = clk::now();
        PoissonStats ps = poisson_.solve(rho_tot_.at(0), vh_.at(0), vh_.tmap, POISSON_TOL, POISSON_MAX_ITER);
        profile.poisson_s += secs(tp);
        profile.poisson_iterations += ps.iterations;
        out->poisson_residual = std::max(out->poisson_residual, ps.residual);
        out->poisson_iterations = std::max(out->poisson_iterations, ps.iterations);
        launch_xc_veff(L_.F, out_up_.at(0), out_dn_.at(0), vnuc_.at(0), vh_.at(0), exc_.at(0), nullptr, nullptr, nullptr, nullptr, s_, pc);
        std::vector<std::pair<const float*, const float*>> pairs = {
            {rho_tot_.at(0), vnuc_.at(0)}, {rho_tot_.at(0), vh_.at(0)}, {exc_.at(0), ones_.at(0)}};
        std::vector<double> kin_w;  // the occupation of each orbital pair after the first three entries
        for (int sp = 0; sp < 2; ++sp) {
            if (nocc[sp] == 0) continue;
            const int cols = fd ? kk[sp] : nocc[sp];
            StencilArgs kin;
            kin.mode = ST_LAPLACIAN;
            kin.scale = (float)(-0.5 / (L_.h * L_.h));
            launch_stencil(L_, ch_[sp].A[ch_[sp].cur].tmap, cols, kin, ch_[sp].T.at(0), s_);
            for (int i = 0; i < cols; ++i) {
                pairs.push_back({ch_[sp].A[ch_[sp].cur].at(i), ch_[sp].T.at(i)});
                kin_w.push_back(occ_[sp][i]);
            }
        }
        red_.dots(pairs, 0, dv);
        const int nvals = (int)pairs.size();
        launch_face_max(L_, rho_tot_.at(0), red_.partials(), red_.blocks(), s_);
        launch_finish_max(red_.partials(), red_.blocks(), red_.res() + nvals, s_);
        const double* h = red_.read(nvals + 1);
        double kinetic = 0.0, comp = 0.0;
        for (int q = 3; q < nvals; ++q) {  // Neumaier over the orbitals (crates/qm-gpu/src/scf.rs:1664-1667)
            double x = kin_w[q - 3] * h[q], t = kinetic + x;
            if (std::fabs(kinetic) >= std::fabs(x)) comp += (kinetic - t) + x; else comp += (x - t) + kinetic;
            kinetic = t;
        }
        kinetic += comp;
        const double h_ext = h[0], h_har = h[1], h_xc = h[2], h_bnd = h[nvals];
        // E_NL = sum_sigma sum_i f_i sum_rows E_KB c^2 (crates/qm/src/nonlocal.rs, f64 finish; one readback per spin)
        double e_nl = 0.0, e_nl_c = 0.0;
        if (nl_on_)
            for (int sp = 0; sp < 2; ++sp) {
                if (nocc[sp] == 0) continue;
                const int cols = fd ? kk[sp] : nocc[sp];
                std::vector<double> c;
                ionic_.project(L_, ch_[sp].X(), cols, nl_sc_, s_, c);
                const int R = ionic_.rows();
                for (int i = 0; i < cols; ++i)
                    for (int r = 0; r < R; ++r) {
                        const double x = occ_[sp][i] * ionic_.row_ekb()[r] * c[(size_t)i * R + r] * c[(size_t)i * R + r];
                        const double t = e_nl + x;
                        if (std::fabs(e_nl) >= std::fabs(x)) e_nl_c += (e_nl - t) + x; else e_nl_c += (x - t) + e_nl;
                        e_nl = t;
                    }
            }
        e_nl += e_nl_c;
        ks_energy& en = out->energy;
        en.kinetic = kinetic;
        en.external_ = h_ext + e_nl;
        en.hartree = 0.5 * h_har;
        en.xc = h_xc;
        en.nuclear = e_nn;
        en.internal = en.kinetic + en.external_ + en.hartree + en.xc + en.nuclear;
        en.ts = fd ? s.kt * entropy : 0.0;  // F = E - kT S (crates/qm/src/scf.rs:1015-1018)
        en.total = en.internal - en.ts;
        out->entropy = fd ? entropy : 0.0;
        out->mu[0] = mu[0];
        out->mu[1] = mu[1];
        out->partial = partial ? 1 : 0;
        out->boundary_density = h_bnd;
        out->electrons[0] = q_out[0];
        out->electrons[1] = q_out[1];
        if (out->boundary_density > BOUNDARY_DENSITY_WARN) ++out->n_warnings;
        if (last_step_maxiter || !(last_step_res <= LAST_STEP_RESIDUAL_FACTOR * eig_lo)) ++out->n_warnings;
        converged_ = true;
        have_warm_ = true;
        fd_state_ = fd;
        // prev holds this solve's starting rho_t: the next warm start extrapolates from it (a cold solve keeps none, so
        // the chain restarts: the next warm start uses rho_t itself)
        have_prev_ = keep_prev && reuse;
        profile.readbacks = readbacks_total() - rb0;
        profile.host_dense_s = lane_[0]->dense_s + lane_[1]->dense_s;
        profile.sync_wait_s = wait_total() - wait0;
        profile.wall_s = secs(t0);
        return KS_OK;
    } catch (const NumericalError& e) {
        error = e.what();
        converged_ = false;
        have_warm_ = false;
        return KS_NUMERICAL;
    } catch (const DeviceError& e) {
        error = e.what();
        converged_ = false;
        have_warm_ = false;
        return KS_DEVICE;
    }
}

ks_status Solver::forces(const ks_nucleus* nuc, int nn, double sigma, double* out3n) {
    NvtxRange range("ks forces");
    if (!converged_) { error = "no converged state"; return KS_NO_STATE; }
    if (nn <= 0 || nn > 32 || !nuc || !out3n) { error = "invalid arguments"; return KS_INVALID; }
    if (state_gen_ != 0) return ionic_forces(nuc, nn, sigma, out3n);
    try {
        std::vector<Nuc> hn(nn);
        for (int i = 0; i < nn; ++i) hn[i] = Nuc{nuc[i].pos[0], nuc[i].pos[1], nuc[i].pos[2], (double)nuc[i].z};
        nuc_d_.alloc(hn.size() * sizeof(Nuc));
        KS_CUDA(cudaMemcpyAsync(nuc_d_.p, hn.data(), hn.size() * sizeof(Nuc), cudaMemcpyHostToDevice, s_));
        // rho = rho_up + rho_dn of the converged state
        Terms tsum;
        tsum.count = 2;
        tsum.x[0] = out_up_.at(0); tsum.c[0] = 1.f;
        tsum.x[1] = out_dn_.at(0); tsum.c[1] = 1.f;
        launch_lincomb(L_.F, 1, rho_tot_.at(0), tsum, s_);
        launch_forces(L_, rho_tot_.at(0), static_cast<const Nuc*>(nuc_d_.p), nn, sigma, red_.partials(), red_.blocks(), s_);
        launch_finish(red_.partials(), red_.blocks(), 3 * nn, L_.h * L_.h * L_.h, red_.res(), s_);
        const double* h = red_.read(3 * nn);
        for (int i = 0; i < 3 * nn; ++i) out3n[i] = h[i];
        // nuclear-nuclear part (crates/qm/src/forces.rs:219-226)
        for (int a = 0; a < nn; ++a)
            for (int b = 0; b < nn; ++b) {
                if (a == b) continue;
                double dv[3] = {nuc[a].pos[0] - nuc[b].pos[0], nuc[a].pos[1] - nuc[b].pos[1], nuc[a].pos[2] - nuc[b].pos[2]};
                double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                if (d < 1e-8) {
                    error = "nuclei " + std::to_string(std::min(a, b)) + " and " + std::to_string(std::max(a, b)) + " coincide";
                    return KS_COINCIDENT_NUCLEI;
                }
                double sc = (double)nuc[a].z * (double)nuc[b].z / (d * d * d);
                for (int c = 0; c < 3; ++c) out3n[3 * a + c] += sc * dv[c];
            }
        return KS_OK;
    } catch (const DeviceError& e) {
        error = e.what();
        return KS_DEVICE;
    }
}

// Forces of a state solved under a pseudopotential setup (crates/qm/src/forces.rs, pseudised ions; the GPU form
// crates/qm-gpu/src/ionic.rs "Forces"): F_I = -dE/dR_I at frozen orbitals and occupations, five terms:
//   local long range    integral rho V_LR,I'(d) (r - R_I)/d            (every centre, its own charge and width)
//   local short range   integral rho V_SR,I'(d) (r - R_I)/d            (pseudised, within r_sr)
//   partial core        integral vbar rho_pc,I'(d) (r - R_I)/d          (vbar = (v_xc,up + v_xc,dn)/2 on rho + rho_pc/2)
//   nonlocal            sum_{sigma,i} 2 f_i sum_{rows of I} E_KB c <grad beta | psi_i>
//   ion-ion             sum_J q_I q_J (R_I - R_J)/|R_I - R_J|^3          (valence charges)
ks_status Solver::ionic_forces(const ks_nucleus* nuc, int nn, double sigma, double* out3n) {
    if (state_gen_ != ionic_gen()) { error = "the ionic setup changed after the solve"; return KS_INVALID; }
    try {
        ionic_.update(L_, nuc, nn, sigma, s_);
        total_density();
        const float* xu = nullptr;
        const float* xd = nullptr;
        if (ionic_.has_core()) {
            if (pc_.count == 0) pc_.create(L_, 1);
            if (xcu_.count == 0) { xcu_.create(L_, 1); xcd_.create(L_, 1); }
            ionic_.partial_core(L_, pc_.at(0), s_);
            launch_xc_veff(L_.F, out_up_.at(0), out_dn_.at(0), vnuc_.at(0), vh_.at(0), exc_.at(0), nullptr, nullptr, xcu_.at(0), xcd_.at(0),
                           s_, pc_.at(0));
            xu = xcu_.at(0);
            xd = xcd_.at(0);
        }
        launch_local_forces(L_, ionic_.centres(), ionic_.n_centres(), ionic_.species_dev(), rho_tot_.at(0), xu, xd, red_.partials(),
                            red_.blocks(), s_);
        launch_finish(red_.partials(), red_.blocks(), 3 * nn, L_.h * L_.h * L_.h, red_.res(), s_);
        const double* h = red_.read(3 * nn);
        for (int i = 0; i < 3 * nn; ++i) out3n[i] = h[i];
        if (ionic_.has_nl()) {
            const int R = ionic_.rows();
            for (int sp = 0; sp < 2; ++sp) {
                if (nocc_[sp] == 0) continue;
                const int cols = count(sp);
                std::vector<double> g;
                ionic_.nl_force_sums(L_, ch_[sp].X(), cols, nl_sc_, s_, g);
                for (int i = 0; i < cols; ++i)
                    for (int r = 0; r < R; ++r) {
                        const double* q = &g[((size_t)i * R + r) * 4];
                        const double w = 2.0 * occ_[sp][i] * ionic_.row_ekb()[r] * q[3];
                        const int a = ionic_.row_ion()[r];
                        for (int c = 0; c < 3; ++c) out3n[3 * a + c] += w * q[c];
                    }
            }
        }
        for (int a = 0; a < nn; ++a)
            for (int b = 0; b < nn; ++b) {
                if (a == b) continue;
                double dv[3] = {nuc[a].pos[0] - nuc[b].pos[0], nuc[a].pos[1] - nuc[b].pos[1], nuc[a].pos[2] - nuc[b].pos[2]};
                double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                if (d < 1e-8) {
                    error = "nuclei " + std::to_string(std::min(a, b)) + " and " + std::to_string(std::max(a, b)) + " coincide";
                    return KS_COINCIDENT_NUCLEI;
                }
                const double sc = ionic_.charge_of(nuc[a].z) * ionic_.charge_of(nuc[b].z) / (d * d * d);
                for (int c = 0; c < 3; ++c) out3n[3 * a + c] += sc * dv[c];
            }
        return KS_OK;
    } catch (const DeviceError& e) {
        error = e.what();
        return KS_DEVICE;
    } catch (const std::invalid_argument& e) {
        error = e.what();
        return KS_INVALID;
    }
}

ks_status Solver::vjp(const ks_nucleus* nuc, int nn, double sigma, double e_bar, double* dE_dR3n, double* dE_dsigma) {
    if (state_gen_ != 0) { error = "vjp: all-electron states only (no pseudopotential terms)"; return KS_INVALID; }
    if (!converged_) { error = "no converged state"; return KS_NO_STATE; }
    if (nn <= 0 || nn > 32 || !nuc || !dE_dR3n || !dE_dsigma || !(sigma > 0) || !std::isfinite(e_bar)) {
        error = "invalid arguments";
        return KS_INVALID;
    }
    try {
        std::vector<Nuc> hn(nn);
        for (int i = 0; i < nn; ++i) hn[i] = Nuc{nuc[i].pos[0], nuc[i].pos[1], nuc[i].pos[2], (double)nuc[i].z};
        nuc_d_.alloc(hn.size() * sizeof(Nuc));
        KS_CUDA(cudaMemcpyAsync(nuc_d_.p, hn.data(), hn.size() * sizeof(Nuc), cudaMemcpyHostToDevice, s_));
        const int nv = 3 * nn + 1;
        // the density of the state: the N_sigma orbitals, or the Fermi-Dirac block weighted by its occupations
        const int cu = count(0), cd = count(1);
        const double* wu = fd_state_ ? occ_d_.d() : nullptr;
        const double* wd = fd_state_ ? occ_d_.d() + 64 : nullptr;
        launch_vjp(L_, cu ? ch_[0].X() : nullptr, cu, wu, cd ? ch_[1].X() : nullptr, cd, wd, static_cast<const Nuc*>(nuc_d_.p), nn, sigma,
                   red_.partials(), red_.blocks(), s_);
        launch_finish(red_.partials(), red_.blocks(), nv, L_.h * L_.h * L_.h, red_.res(), s_);
        const double* g = red_.read(nv);
        for (int i = 0; i < 3 * nn; ++i) dE_dR3n[i] = g[i];
        *dE_dsigma = e_bar * g[3 * nn];
        // point-charge repulsion E_nn = sum Z_a Z_b / |R_a - R_b| (independent of sigma)
        for (int a = 0; a < nn; ++a)
            for (int b = 0; b < nn; ++b) {
                if (a == b) continue;
                double dv[3] = {nuc[a].pos[0] - nuc[b].pos[0], nuc[a].pos[1] - nuc[b].pos[1], nuc[a].pos[2] - nuc[b].pos[2]};
                double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
                if (d < 1e-8) {
                    error = "nuclei " + std::to_string(std::min(a, b)) + " and " + std::to_string(std::max(a, b)) + " coincide";
                    return KS_COINCIDENT_NUCLEI;
                }
                double sc = (double)nuc[a].z * (double)nuc[b].z / (d * d * d);
                for (int c = 0; c < 3; ++c) dE_dR3n[3 * a + c] -= sc * dv[c];
            }
        for (int i = 0; i < 3 * nn; ++i) dE_dR3n[i] *= e_bar;
        return KS_OK;
    } catch (const DeviceError& e) {
        error = e.what();
        return KS_DEVICE;
    }
}

// ---------------------------------------------------------------- readouts of the converged state
void Solver::total_density() {
    Terms tsum;
    tsum.count = 2;
    tsum.x[0] = out_up_.at(0); tsum.c[0] = 1.f;
    tsum.x[1] = out_dn_.at(0); tsum.c[1] = 1.f;
    launch_lincomb(L_.F, 1, rho_tot_.at(0), tsum, s_);
}

// crates/qm-gpu/src/sample.rs:84-121: one launch and one readback per non-empty call; the point and
// output buffers grow to the largest request and are reused.
void Solver::sample_density(const double* pts3, int count, float* out) {
    if (count <= 0) return;
    if ((size_t)count > sample_cap_) {
        sample_pts_.alloc((size_t)count * 3 * sizeof(double));
        sample_out_.alloc((size_t)count * sizeof(float));
        sample_cap_ = (size_t)count;
        ++sampling_allocations;
    }
    KS_CUDA(cudaMemcpyAsync(sample_pts_.p, pts3, (size_t)count * 3 * sizeof(double), cudaMemcpyHostToDevice, s_));
    total_density();
    launch_sample(L_, rho_tot_.at(0), sample_pts_.d(), count, sample_out_.f(), s_);
    KS_CUDA(cudaMemcpyAsync(out, sample_out_.p, (size_t)count * sizeof(float), cudaMemcpyDeviceToHost, s_));
    KS_CUDA(cudaStreamSynchronize(s_));
    ++sampling_readbacks;
}

// crates/qm-gpu/src/scf.rs:1776-1779 (density_f32): the interior of rho_up + rho_dn as stored, f32
// the two spin densities of the state as f64 n^3 arrays (ks_state_density): one unpack per spin into a grow-only device
// buffer on the solver's stream and one copy each, without a per-call allocation
void Solver::density_f64(double* up, double* dn) {
    const size_t n3 = (size_t)L_.interior();
    if (dens64_.bytes < 2 * n3 * sizeof(double)) dens64_.alloc(2 * n3 * sizeof(double));
    launch_unpack(L_, 1, out_up_.at(0), dens64_.d(), s_);
    launch_unpack(L_, 1, out_dn_.at(0), dens64_.d() + n3, s_);
    KS_CUDA(cudaMemcpyAsync(up, dens64_.d(), n3 * sizeof(double), cudaMemcpyDeviceToHost, s_));
    KS_CUDA(cudaMemcpyAsync(dn, dens64_.d() + n3, n3 * sizeof(double), cudaMemcpyDeviceToHost, s_));
    KS_CUDA(cudaStreamSynchronize(s_));
}

void Solver::density_f32(float* host_n3) {
    const size_t bytes = (size_t)L_.interior() * sizeof(float);
    if (volume_.bytes < bytes) volume_.alloc(bytes);
    total_density();
    launch_volume(L_, rho_tot_.at(0), nullptr, volume_.f(), red_.partials(), red_.blocks(), s_);
    KS_CUDA(cudaMemcpyAsync(host_n3, volume_.p, bytes, cudaMemcpyDeviceToHost, s_));
    KS_CUDA(cudaStreamSynchronize(s_));
}

// crates/qm-gpu/src/scf.rs:1780-1797: the dense n^3 image of the density on the device, enqueued on
// `s` after the solver's own work; does not wait. (A headless buffer in place of the texture.)
void Solver::density_to_volume(float* dense_dev, cudaStream_t s, bool with_core, double* max_out) {
    total_density();
    // the partial core of the state's setup and geometry (crates/qm-gpu/src/scf.rs:1798-1829); none: the plain density
    const float* core = (with_core && state_gen_ != 0 && state_gen_ == ionic_gen() && ionic_.has_core() && pc_.count > 0) ? pc_.at(0) : nullptr;
    if (s && s != s_) {
        cudaEvent_t ev;
        KS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        KS_CUDA(cudaEventRecord(ev, s_));
        KS_CUDA(cudaStreamWaitEvent(s, ev, 0));
        KS_CUDA(cudaEventDestroy(ev));
    }
    // the per-block maxima land in the reducer's partials; the stream joins keep them ordered
    launch_volume(L_, rho_tot_.at(0), core, dense_dev, red_.partials(), red_.blocks(), s ? s : s_);
    if (s && s != s_) {
        // the solver's stream must not reuse rho_tot_ or the partials before the copy is done
        cudaEvent_t ev;
        KS_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
        KS_CUDA(cudaEventRecord(ev, s));
        KS_CUDA(cudaStreamWaitEvent(s_, ev, 0));
        KS_CUDA(cudaEventDestroy(ev));
    }
    if (max_out) {
        launch_finish_max(red_.partials(), red_.blocks(), red_.res(), s_);
        *max_out = red_.read(1)[0];
    }
}

int Solver::apply_nonlocal(const ks_nucleus* nuc, int nn, int count, const double* x, double* out, double* c) {
    if (!ionic_.active()) throw std::invalid_argument("apply_nonlocal: no ionic setup (ks_set_ionic)");
    if (nn < 1 || nn > MAX_CENTRES || count < 1) throw std::invalid_argument("apply_nonlocal: 1..32 nuclei, count >= 1");
    ionic_.update(L_, nuc, nn, L_.h, s_);
    Block in, res;
    in.create(L_, count);
    res.create(L_, count);
    DevBuf tmp((size_t)L_.interior() * count * sizeof(double));
    KS_CUDA(cudaMemcpyAsync(tmp.p, x, (size_t)L_.interior() * count * sizeof(double), cudaMemcpyHostToDevice, s_));
    launch_pack(L_, count, tmp.d(), in.at(0), s_);
    launch_fill(res.at(0), 0.0f, L_.F * count, s_);
    ionic_.apply_nl(L_, in.at(0), count, res.at(0), nl_sc_, s_);
    if (c) {
        std::vector<double> cc;
        ionic_.project(L_, in.at(0), count, nl_sc_, s_, cc);
        std::copy(cc.begin(), cc.end(), c);
    }
    launch_unpack(L_, count, res.at(0), tmp.d(), s_);
    KS_CUDA(cudaMemcpyAsync(out, tmp.p, (size_t)L_.interior() * count * sizeof(double), cudaMemcpyDeviceToHost, s_));
    KS_CUDA(cudaStreamSynchronize(s_));
    return ionic_.rows();
}

// crates/qm-gpu/src/scf.rs:1831-1834: max rho over the interior (one readback)
double Solver::density_max() {
    total_density();
    const size_t bytes = (size_t)L_.interior() * sizeof(float);
    if (volume_.bytes < bytes) volume_.alloc(bytes);
    launch_volume(L_, rho_tot_.at(0), nullptr, volume_.f(), red_.partials(), red_.blocks(), s_);
    launch_finish_max(red_.partials(), red_.blocks(), red_.res(), s_);
    return red_.read(1)[0];
}

// crates/qm-gpu/src/scf.rs:1836-1842: integral of |rho_up - rho_dn| (electrons)
double Solver::spin_abs_integral() {
    launch_abs_diff(L_.F, out_up_.at(0), out_dn_.at(0), red_.partials(), red_.blocks(), s_);
    launch_finish(red_.partials(), red_.blocks(), 1, L_.h * L_.h * L_.h, red_.res(), s_);
    return red_.read(1)[0];
}

}  // namespace ks
