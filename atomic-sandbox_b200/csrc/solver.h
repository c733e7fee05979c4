// solver.h -- the B200 Kohn-Sham solver behind the C ABI (include/ks_cuda.h).
#pragma once
#include <atomic>
#include <limits>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>
#include "common.cuh"
#include "kernels.cuh"
#include "ionic.cuh"
#include "../../include/ks_cuda.h"

namespace ks {

// Owning device allocation.
struct DevBuf {
    void* p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    explicit DevBuf(size_t n) { alloc(n); }
    ~DevBuf() { release(); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    void alloc(size_t n);
    void release();
    float* f() const { return static_cast<float*>(p); }
    double* d() const { return static_cast<double*>(p); }
};

// A contiguous block of `count` pitched fields with a tensor map over it (stencil input).
struct Block {
    DevBuf buf;
    int count = 0;
    long long F = 0;
    CUtensorMap tmap;
    void create(const Layout& L, int count);
    float* at(int i) const { return buf.f() + (long long)i * F; }
};

// Per-shape device timing of the hot launches (ks_set_kernel_timing): CUDA events around each launch on its own
// stream, collected when read. Shared by the solver's host threads (the two spin channels), hence the lock.
class KernelTimer {
public:
    KernelTimer() = default;
    KernelTimer(const KernelTimer&) = delete;
    KernelTimer& operator=(const KernelTimer&) = delete;
    ~KernelTimer();
    void enable(bool on);
    bool on() const { return on_.load(std::memory_order_relaxed); }
    // runs launch() between two events on s when the timer is on (never while the thread captures a graph)
    template <class Launch>
    void time(int kernel, int count, int aux, double bytes, cudaStream_t s, Launch&& launch) {
        if (!on()) {
            launch();
            return;
        }
        cudaEvent_t a = take(), b = take();
        KS_CUDA(cudaEventRecord(a, s));
        launch();
        KS_CUDA(cudaEventRecord(b, s));
        std::lock_guard<std::mutex> lock(mu_);
        pending_.push_back({kernel, count, aux, bytes, a, b});
    }
    // waits for the recorded launches and returns the totals per shape
    std::vector<ks_kernel_time> totals();

private:
    struct Rec { int kernel, count, aux; double bytes; cudaEvent_t a, b; };
    cudaEvent_t take();
    std::atomic<bool> on_{false};
    std::mutex mu_;
    std::vector<Rec> pending_;
    std::vector<cudaEvent_t> pool_;
    std::vector<ks_kernel_time> agg_;
};

// Device reductions with a fixed grid (deterministic), results kept on the device until read.
class Reducer {
public:
    Reducer() = default;
    Reducer(const Reducer&) = delete;
    Reducer& operator=(const Reducer&) = delete;
    void init(const Layout& L, cudaStream_t s, size_t partial_doubles);
    // sum_p a_p b_p * scale for every pair, written to res()[off + i]
    void dots(const std::vector<std::pair<const float*, const float*>>& pairs, int off, double scale);
    // G = scale * S^T [S | T], written to res()[off...] row-major m x (m + mt)
    void gram(int m, const float* S, int mt, const float* T, int off, double scale = 1.0, const FinishDesc* extra = nullptr);
    double* res() const { return res_.d(); }
    double* partials() const { return partials_.d(); }
    int blocks() const { return blocks_; }
    // copies res[0..count) to the host and synchronises; raises DeviceError on a failed kernel wait
    const double* read(int count);
    // failure injection for the failure-path tests: lets `skip` readbacks through, then fails the next `count` as a
    // readback that never delivers (DeviceError); shared by a solver's reducers
    struct Faults {
        std::atomic<long long> skip{0}, count{0};
    };
    Faults* faults = nullptr;
    int readbacks = 0;
    double wait_s = 0;  // host time blocked in read()
    int gram_mode = 0;  // 0: CUDA-core f32 Gram, 1: tensor-core 3xTF32 Gram
    KernelTimer* timer = nullptr;  // times the Gram launch when set
    double* host() const { return host_; }
    static constexpr int RES_CAP = 1 << 16;

private:
    Layout L_;
    cudaStream_t s_ = nullptr;
    DevBuf partials_, res_;
    double* host_ = nullptr;
    int* host_flag_ = nullptr;
    int blocks_ = 1;
    int gram_blocks_ = 1;

public:
    ~Reducer();
};

// The ionic setup of a solver (crates/qm/src/ionic.rs IonicSetup, its tables from ks_species) and the
// terms of the current geometry: centres, projector spheres and their beta values on the device.
class Ionic {
public:
    struct Scratch {
        DevBuf partials, coef;
        size_t cap = 0;
    };
    void set(const ks_species* sp, int nsp);  // throws std::invalid_argument on a bad table
    bool active() const { return !species_.empty(); }
    int generation() const { return gen_; }
    int species_of(int z) const;              // index, or -1 for an all-electron species
    double charge_of(int z) const;            // z_v when pseudised, else z
    void update(const Layout& L, const ks_nucleus* nuc, int nn, double sigma_ae, cudaStream_t s);
    bool has_core() const { return has_core_; }
    bool has_nl() const { return !sph_h_.empty(); }
    int rows() const { return rows_total_; }
    const std::vector<double>& row_ekb() const { return row_ekb_; }
    const std::vector<int>& row_ion() const { return row_ion_; }
    const IonicCentre* centres() const { return static_cast<const IonicCentre*>(centres_.p); }
    int n_centres() const { return (int)centres_h_.size(); }
    const IonicSpeciesDev* species_dev() const { return static_cast<const IonicSpeciesDev*>(species_dev_.p); }
    void local_potential(const Layout& L, float* out, cudaStream_t s) const;
    void partial_core(const Layout& L, float* out, cudaStream_t s) const;
    // out_v += V_NL x_v, v < count (blocks of stride F)
    void apply_nl(const Layout& L, const float* x, int count, float* out, Scratch& sc, cudaStream_t s) const;
    // c[v * rows + row] = h^3 <beta_row, x_v> (synchronises s)
    void project(const Layout& L, const float* x, int count, Scratch& sc, cudaStream_t s, std::vector<double>& c) const;
    // [(v * rows + row) * 4 + {x, y, z, beta}] = h^3 <(grad beta_row, beta_row), psi_v> (synchronises s)
    void nl_force_sums(const Layout& L, const float* psi, int count, Scratch& sc, cudaStream_t s, std::vector<double>& sums) const;

private:
    void ensure(Scratch& sc, int count) const;
    struct Proj { int l; double e_kb, radius; std::vector<double> t; };
    struct Species {
        int z;
        double z_v, sigma_lr, du, r_sr, pc_radius;
        std::vector<double> v_sr, rho_pc;
        std::vector<Proj> proj;
    };
    std::vector<Species> species_;
    std::vector<size_t> off_v_sr_, off_pc_;
    std::vector<std::vector<size_t>> off_t_;
    DevBuf tables_, species_dev_, centres_, spheres_, chunk_sphere_, beta_;
    std::vector<IonicCentre> centres_h_;
    std::vector<Sphere> sph_h_;
    std::vector<int> chunk_sphere_h_, row_ion_;
    std::vector<double> row_ekb_;
    int rows_total_ = 0, total_chunks_ = 0, max_pts_ = 0;
    int ubox_[6] = {0, 0, 0, 0, 0, 0};
    int gen_ = 0;
    bool has_core_ = false;
};

struct PoissonStats { int iterations = 0; double residual = 0; int stop = 0; int readbacks = 0; };

// Multigrid-preconditioned CG Hartree solve (crates/qm-gpu/src/poisson.rs:111-343).
class Poisson {
public:
    Poisson() = default;
    Poisson(const Poisson&) = delete;
    Poisson& operator=(const Poisson&) = delete;
    ~Poisson();
    void init(const Layout& L, cudaStream_t s, Reducer* red);
    PoissonStats solve(const float* rho, float* v, const CUtensorMap& v_map, double tol, int max_iter);
    void moments(const float* rho, double* dst_dev);  // 49 f64, dV applied

private:
    struct Level { MgLevel lv; DevBuf x, b, res, tmp; };
    void vcycle(const float* rhs, float* z);
    void cycle(int l, float* x, const float* b);
    void true_residual(const CUtensorMap& v_map);  // r = b + L v into ap_, |r|^2 reduced (v is v_map's field)
    void iteration(float* v, int par);
    void run_iteration(float* v, int par);
    void release_graphs();
    cudaGraphExec_t graph_[2] = {nullptr, nullptr};  // one PCG iteration per parity, for the v of graph_v_
    int graph_kernels_[2] = {0, 0};
    const float* graph_v_ = nullptr;
    Layout L_;
    cudaStream_t s_ = nullptr;
    Reducer* red_ = nullptr;
    Block r_, p_, ap_, b_, z_, res0_, tmp0_;
    DevBuf ghost_, scal_, q_;
    std::vector<Level> levels_;   // coarse levels 1..; level 0 is the fine grid (its x/b are z/r)
    int fused_from_ = 0;          // first level handled by the single-CTA kernel
    std::vector<MgLevel> lvdesc_;
};

struct EigenStats {
    int iterations = 0;
    double max_residual = 0;
    int stop = 0;  // 0 converged, 1 floor, 2 max_iter
    int readbacks = 0;
    int restores = 0;
    bool restores_exhausted = false;
    double alpha_worst = 0;
    int fallbacks = 0;
    // the split stop test's two tiers: the true max residual of the head columns and of the tail columns [head, checked)
    double head_res = 0, tail_res = 0;
    // the head columns came back exactly as given: a 0-iteration accept, or a locked head
    bool head_kept = false;
    int locked = 0;  // the locked head's columns (0: no lock)
};

// One spin channel's LOBPCG work space: k vectors, [X | W | P] arenas (ping-pong), [R | HW | HP],
// HX and the preconditioner scratch.
struct Channel {
    int k = 0;
    Block A[2];
    int cur = 0;
    Block T, HX, Q;
    DevBuf theta_d, lambda_d, coef_d;
    std::vector<double> evals;  // Ritz values of the columns (ascending after a solve)
    std::vector<double> res;    // their residual norms |H x - theta x| at the last LOBPCG exit (NaN: not measured)
    void create(const Layout& L, int k);
    float* X() const { return A[cur].at(0); }
};

// A spin channel's execution lane: its own stream, reducer (device partials, pinned readback) and
// pinned upload buffer, so that the two channels' LOBPCG solves can run concurrently.
struct Lane {
    cudaStream_t s = nullptr;
    cudaEvent_t ev_join = nullptr;
    Reducer red;
    double* up = nullptr;
    size_t up_cap = 0;
    double dense_s = 0;  // host time in the Rayleigh-Ritz algebra (profile)
    Ionic::Scratch nl;   // the nonlocal operator's projections on this lane's stream
    DevBuf norm_part;    // per-CTA |r_i|^2 partials of the residual kernel, finished with the Gram
    Lane() = default;
    Lane(const Lane&) = delete;
    Lane& operator=(const Lane&) = delete;
    void init(const Layout& L);
    double* upload_buffer(size_t doubles);
    ~Lane();
};

// Thrown out of an eigensolve when the inner cancellation point fired.
struct AbortInside {};

struct SolverOptions { int gram_mode = 0; int n_extra = 0; int init_mode = 0; };

class Solver {
public:
    // Device bytes a solver of this grid holds through a solve and its forces with n_up / n_dn electrons, the
    // options' extra bands and a DIIS history (its buffers as allocated below; the CUDA context and the loaded
    // kernels are not counted). pseudo_core adds the partial-core fields of an ionic setup.
    static size_t footprint_bytes(int n, int n_up, int n_dn, const SolverOptions& o, int diis_history, bool pseudo_core);
    Solver(int n, double h, const SolverOptions& o);
    ~Solver();
    ks_status solve(const ks_nucleus* nuc, int nn, int n_up, int n_dn, const ks_settings& s, bool warm, ks_abort_fn abort_fn,
                    void* user, ks_stats* out, ks_abort_fn inner_abort = nullptr, ks_observe_fn observe = nullptr);
    ks_status forces(const ks_nucleus* nuc, int nn, double sigma, double* out3n);
    ks_status vjp(const ks_nucleus* nuc, int nn, double sigma, double e_bar, double* dE_dR3n, double* dE_dsigma);
    // rho_in of a warm start extrapolated linearly from the last two converged outputs (crates/qm-gpu/src/scf.rs:1146-1163)
    void set_density_extrapolation(bool on) {
        extrapolate_ = on;
        if (!on) have_prev_ = false;
    }
    // at most `cap` extra Fermi-Dirac levels grown per channel for the gap witness, clamped to 1..32 (scf.rs:1122-1129)
    void set_witness_cap(int cap) { witness_cap_ = std::max(1, std::min(cap, 32)); }
    int witness_cap() const { return witness_cap_; }
    // the LOBPCG tolerance the final SCF step converges to: max(eig_tol, 3 x the f32 residual floor) (scf.rs:1713-1715)
    double effective_eig_tol(double eig_tol) const;
    // the ionic setup of the next solves (n = 0: all-electron); throws std::invalid_argument on bad tables
    void set_ionic(const ks_species* sp, int n) { ionic_.set(sp, n); }
    // lobpcg_split / lobpcg_guarded (crates/qm-gpu/src/eigen.rs:613-653): columns [0, head) are held to tol, columns
    // [head, checked) to tail_tol and columns from `checked` on are untested buffers (the split stop test of
    // eigen.rs:781-787, a column's residual scaled by tol / its own tolerance; the guess accepted at guess_tol on the same
    // scale). checked < 0: every column when tail_tol is finite, else the head alone. lock: at the guess, a head under
    // guess_tol whose tail is not is locked -- returned bitwise while the other columns iterate in its B-orthogonal
    // complement (eigen.rs:174-183, :814-818).
    EigenStats lobpcg(Channel& ch, Lane& lane, const float* V, double tol, double guess_tol, int max_iter, int head,
                      double tail_tol = std::numeric_limits<double>::infinity(), int checked = -1, bool lock = false);
    Lane& lane(int i) { return *lane_[i]; }
    std::string error;
    const Layout& layout() const { return L_; }
    cudaStream_t stream() const { return s_; }
    bool has_state() const { return converged_; }
    // stored orbitals of the converged state: N_sigma under Aufbau, the N_sigma + n_extra block under Fermi-Dirac
    int count(int spin) const { return fd_state_ ? ch_[spin].k : nocc_[spin]; }
    const std::vector<double>& occupations(int spin) const { return occ_[spin]; }
    const Channel& channel(int spin) const { return ch_[spin]; }
    const float* rho(int spin) const { return spin ? out_dn_.at(0) : out_up_.at(0); }
    const float* v_nuc() const { return vnuc_.at(0); }
    const float* v_h() const { return vh_.at(0); }
    // readouts of the converged state (crates/qm-gpu/src/sample.rs, scf.rs:1776-1842)
    void sample_density(const double* pts3, int count, float* out);
    void density_f32(float* host_n3);
    void density_f64(double* up, double* dn);
    void density_to_volume(float* dense_dev, cudaStream_t s, bool with_core = false, double* max_out = nullptr);
    // out_v = V_NL x_v of the ionic setup at nuc (host f64 n^3 each); c = projections; returns the row count
    int apply_nonlocal(const ks_nucleus* nuc, int nn, int count, const double* x, double* out, double* c);
    double density_max();
    double spin_abs_integral();
    int sampling_readbacks = 0, sampling_allocations = 0;
    ks_profile profile{};
    Poisson& poisson() { return poisson_; }
    Reducer& reducer() { return red_; }
    // this solver's wait-timeout flag (device int); its calls install it as the thread's current flag (ErrorFlagScope)
    int* err_flag() const { return static_cast<int*>(err_.p); }
    KernelTimer& timer() { return timer_; }
    // the warm start of the next solve from host arrays (ks_state_import); k_sp orbitals per spin (f64 n^3 each),
    // their levels and occupations, the input densities and V_H. Throws std::invalid_argument on inconsistent sizes.
    void import_state(int n_up, int n_dn, const int k[2], const double* const orb[2], const double* const evals[2],
                      const double* const occ[2], const double* rho_up, const double* rho_dn, const double* v_h, bool fermi_dirac);
    // failure-path test hooks: a NaN in the parked warm density; the next readbacks fail
    void poison_parked_density();
    void fail_readbacks(long long skip, long long count) {
        faults_.skip.store(skip);
        faults_.count.store(count);
    }

private:
    void ensure_channel(int spin, int k);
    // the channel's block resized to newk columns on stream st (0: the solver's): its first columns kept (or, with cols,
    // column j taken from old column cols[j]), new ones seeded with the reference's initial orbital 1000 + 2 j + spin
    void resize_channel(int spin, int newk, const Nuc* dnuc, int nn, cudaStream_t st = nullptr, const std::vector<int>* cols = nullptr);
    // buffer_last (crates/qm-gpu/src/scf.rs:1031-1040): the highest Ritz value moved to the last column; returns the
    // position the former last column moved to, -1 when it was already there
    int buffer_last(int spin, cudaStream_t st);
    // the Fermi-Dirac channel solve of one spin (crates/qm-gpu/src/scf.rs:893-1029 Channel::solve_fd), run on the channel's
    // own lane and thread
    struct FdOutcome {
        bool kept = true;        // every call returned the tight columns bitwise
        bool witnessed = false;  // a gap witness decided the solve (false: the cap was reached without one)
        int calls = 0, iterations = 0, checked = 0;
        double tight_res = 0.0;  // the last call's head (tight) residual
        double tail_kt = 0.0;    // the widest witness tail used
        bool maxiter = false;
        int growths = 0, locked_calls = 0, class_raises = 0, buffer_witnesses = 0, buffer_growths = 0, lower_witnesses = 0,
            residual_growths = 0, trims = 0, peak_block = 0;
    };
    FdOutcome solve_fd(int spin, const float* V, double step_tol, double guess_tol, bool loosened, double delta_rho_prev, double kt,
                       double scf_tol, int n, int& kk, int& tight, const Nuc* dnuc, int nn);
    void gram_checked(Reducer& red, int m, const float* S, int mt, const float* T, const FinishDesc* extra = nullptr);
    int readbacks_total() const { return red_.readbacks + lane_[0]->red.readbacks + lane_[1]->red.readbacks; }
    double wait_total() const { return red_.wait_s + lane_[0]->red.wait_s + lane_[1]->red.wait_s; }
    Layout L_;
    SolverOptions opt_;
    cudaStream_t s_ = nullptr;
    Reducer red_;
    Poisson poisson_;
    Channel ch_[2];
    int nocc_[2] = {0, 0};
    Block vnuc_, vh_, in_up_, in_dn_, out_up_, out_dn_, rho_tot_, v_up_, v_dn_, exc_, ones_, kin_;
    struct Entry { Block rho_up, rho_dn, r_up, r_dn; };
    std::vector<Entry> diis_pool_;
    DevBuf nuc_d_;
    DevBuf sample_pts_, sample_out_, volume_, dens64_;  // grow-only readout buffers
    Ionic ionic_;                              // the pseudopotential setup (inactive: all-electron)
    bool extrapolate_ = false, have_prev_ = false;
    Block prev_up_, prev_dn_;                  // rho_{t-1} of the density extrapolation
    int witness_cap_ = 32;
    Ionic::Scratch nl_sc_;                     // projections on the solver's stream (energy, forces)
    Block pc_, xcu_, xcd_;                     // partial core of the geometry; v_xc scratch of the forces
    bool nl_on_ = false;                       // H psi includes V_NL (inside a solve under a setup)
    // the inner cancellation point: polled by the calling thread once per LOBPCG iteration; a hit sets the flag, which
    // every channel's eigensolve checks at its next iteration and leaves by AbortInside
    ks_abort_fn inner_fn_ = nullptr;
    void* inner_user_ = nullptr;
    std::thread::id poll_thread_;
    std::atomic<int> inner_flag_{0};
    int state_gen_ = 0;                        // ionic generation the state was solved under (0: all-electron)
    int ionic_gen() const { return ionic_.active() ? ionic_.generation() : 0; }
    ks_status ionic_forces(const ks_nucleus* nuc, int nn, double sigma, double* out3n);
    size_t sample_cap_ = 0;
    void total_density();                      // rho_tot_ = rho_up + rho_dn (f32) of the state
    bool converged_ = false;
    bool have_warm_ = false;
    std::unique_ptr<Lane> lane_[2];
    std::vector<double> occ_[2];   // occupation per column of each channel's block (the last step's)
    bool fd_state_ = false;        // the state was converged under Fermi-Dirac
    DevBuf occ_d_;                 // device copy of the occupations (2 x 64 doubles), density weights
    cudaEvent_t ev_fork_ = nullptr;
    DevBuf err_;                   // the solver's own wait-timeout flag
    KernelTimer timer_;            // per-shape kernel timing (off unless asked for)
    Reducer::Faults faults_;       // injected readback failures (tests)
    int dev_ = 0;
    double floor_;
};

long long launch_count();

// Residual floor model of an f32-stored eigenvector (crates/qm-gpu/src/eigen.rs:313-318).
double residual_floor_estimate(double h);
// Generalised Rayleigh-Ritz on a raw subspace (crates/qm-gpu/src/eigen.rs:515-542): lowest nk pairs
// of A c = theta B c; C column-major m x nk. Throws NumericalError on a zero-norm column or rank loss.
double rayleigh_ritz(int m, const std::vector<double>& A, const std::vector<double>& B, int nk, std::vector<double>& theta,
                     std::vector<double>& C);
// rayleigh_ritz_locked (crates/qm-gpu/src/eigen.rs:669-681): the lowest na pairs on the subspace {S c : Y^T B (S c) = 0}
// of the columns after the first `locked` (Y), c = Q c' with Q = [-B_YY^-1 B_YZ; I]; C column-major m x na.
double rayleigh_ritz_locked(int m, const std::vector<double>& A, const std::vector<double>& B, int locked, int na,
                            std::vector<double>& theta, std::vector<double>& C);

}  // namespace ks
