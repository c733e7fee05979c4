// ks_solver.hpp -- the reference's Rust API for the Kohn-Sham hot path, `qm_gpu::GpuSolver`, restated in C++ over the
// C ABI of ks_cuda.h. Header-only; link with -lks_b200.
//
//   GpuSolver::new(ctx, &grid)                   crates/qm-gpu/src/scf.rs:1083   -> GpuSolver(n, h, options)
//   solve(&System, &ScfSettings, warm)           scf.rs:1195                     -> solve(system, settings, warm)
//   solve_with(.., should_abort)                 scf.rs:1208                     -> solve_with(.., should_abort)
//   solve_observed / solve_polled                scf.rs:1213-1235                -> solve_observed(.., inner_abort, observe)
//   forces(&GpuState, &[Nucleus], sigma)         crates/qm-gpu/src/forces.rs:239 -> forces(nuclei, sigma)
//   state() / ks_state / profile()               scf.rs:1172-1175, :1713-1775    -> evals(), occupations(), density(), ...
//   set_density_extrapolation, set_witness_cap,  scf.rs:1122-1163, :1713-1715    -> the same names
//   effective_eig_tol
//
// Errors are the reference's qm::QmError variants (crates/qm/src/error.rs:4-31) as exceptions derived from QmError,
// carrying the C ABI's status and message: CoincidentNuclei, ScfNotConverged (iterations, delta_rho), ScfStalled,
// Numerical, Device. The reference panics on argument errors; here they throw InvalidArgument (a std::invalid_argument).
// An abandoned solve throws Aborted (the iterate is parked as the next warm start), state access without a converged
// state throws NoState. Like the reference's solver, a GpuSolver is movable, not copyable, and used by one thread at a
// time; it owns one grid, one CUDA stream and every device buffer of its solves.
#pragma once

#include <array>
#include <cstddef>
#include <functional>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "ks_cuda.h"

namespace qm_gpu {

// qm::Nucleus (crates/qm/src/nuclear.rs:88-92): position (Bohr) and atomic number.
struct Nucleus {
    std::array<double, 3> pos;
    int z;
};

// qm::System (crates/qm/src/scf.rs:329): nuclei and electrons per spin.
struct System {
    std::vector<Nucleus> nuclei;
    int n_up = 0;
    int n_dn = 0;
};

// qm::Occupations (crates/qm/src/scf.rs:278).
enum class Occupations { Aufbau, FermiDirac };

// qm::ScfSettings (crates/qm/src/scf.rs:375). A default-constructed one has the reference's tolerances, mixing and
// history but Aufbau occupations and no sigma (which the solve refuses): the reference's defaults come from for_grid,
// which needs a grid spacing. ScfSettings::for_grid(h) is that constructor (scf.rs:381-395: sigma = h, Fermi-Dirac at
// ELECTRON_KT); under Fermi-Dirac the solver needs options with n_extra >= 1, a block with room for the gap witness.
struct ScfSettings {
    double sigma = 0.0;
    double tol = 1e-6;
    double mixing = 0.3;
    double eig_tol = 1e-6;
    int max_iter = 200;
    int diis_history = 6;
    int stall_window = 50;
    Occupations occupations = Occupations::Aufbau;
    double kt = 5e-3;  // ELECTRON_KT (crates/qm/src/occupations.rs:166), used under FermiDirac only

    static ScfSettings for_grid(double h) {
        ScfSettings s;
        s.sigma = h;
        s.occupations = Occupations::FermiDirac;
        s.kt = 5e-3;
        return s;
    }
};

using Energy = ks_energy;        // qm::Energy (crates/qm/src/scf.rs:533)
using ScfStats = ks_stats;       // qm::ScfStats (crates/qm/src/scf.rs:558-574)
using ScfProgress = ks_progress; // qm::ScfProgress (crates/qm/src/scf.rs:488-498)
using SolveProfile = ks_profile; // qm_gpu::SolveProfile (crates/qm-gpu/src/scf.rs:448-514), subset
using Vec3 = std::array<double, 3>;

// qm::QmError (crates/qm/src/error.rs:4-31) and the boundary's own conditions.
struct QmError : std::runtime_error {
    ks_status status;
    QmError(ks_status st, const std::string& msg) : std::runtime_error(msg), status(st) {}
};
struct CoincidentNuclei : QmError { using QmError::QmError; };
struct ScfNotConverged : QmError {
    int iterations;
    double delta_rho;
    ScfNotConverged(const std::string& msg, int it, double dr) : QmError(KS_NOT_CONVERGED, msg), iterations(it), delta_rho(dr) {}
};
struct ScfStalled : QmError {
    int iterations;
    double delta_rho;
    ScfStalled(const std::string& msg, int it, double dr) : QmError(KS_STALLED, msg), iterations(it), delta_rho(dr) {}
};
struct Numerical : QmError { using QmError::QmError; };
struct Device : QmError { using QmError::QmError; };
struct Aborted : QmError { using QmError::QmError; };
struct NoState : QmError { using QmError::QmError; };
struct InvalidArgument : std::invalid_argument { using std::invalid_argument::invalid_argument; };

namespace detail {

inline std::string message(const void* handle) {
    const char* m = ks_last_error(handle);
    return m ? std::string(m) : std::string();
}

// Throws the exception of a non-OK status; `stats` (may be null) supplies ScfNotConverged's and ScfStalled's counts.
inline void check(ks_status st, const void* handle, const ks_stats* stats = nullptr) {
    if (st == KS_OK) return;
    const std::string msg = message(handle);
    const int it = stats ? stats->iterations : 0;
    const double dr = stats ? stats->delta_rho : 0.0;
    switch (st) {
        case KS_COINCIDENT_NUCLEI: throw CoincidentNuclei(st, msg);
        case KS_NOT_CONVERGED: throw ScfNotConverged(msg, it, dr);
        case KS_STALLED: throw ScfStalled(msg, it, dr);
        case KS_NUMERICAL: throw Numerical(st, msg);
        case KS_INVALID: throw InvalidArgument(msg.empty() ? std::string("invalid argument") : msg);
        case KS_ABORTED: throw Aborted(st, msg);
        case KS_NO_STATE: throw NoState(st, msg.empty() ? std::string("no converged state") : msg);
        default: throw Device(st, msg);
    }
}

inline std::vector<ks_nucleus> to_c(const std::vector<Nucleus>& nuclei) {
    std::vector<ks_nucleus> out(nuclei.size());
    for (size_t i = 0; i < nuclei.size(); ++i) {
        for (int a = 0; a < 3; ++a) out[i].pos[a] = nuclei[i].pos[a];
        out[i].z = nuclei[i].z;
    }
    return out;
}

inline ks_settings to_c(const ScfSettings& s) {
    ks_settings c{};
    c.sigma = s.sigma;
    c.tol = s.tol;
    c.mixing = s.mixing;
    c.eig_tol = s.eig_tol;
    c.max_iter = s.max_iter;
    c.diis_history = s.diis_history;
    c.stall_window = s.stall_window;
    c.occupations = s.occupations == Occupations::FermiDirac ? 1 : 0;
    c.kt = s.kt;
    return c;
}

inline std::vector<Vec3> to_vec3(const std::vector<double>& flat) {
    std::vector<Vec3> out(flat.size() / 3);
    for (size_t i = 0; i < out.size(); ++i) out[i] = {flat[3 * i], flat[3 * i + 1], flat[3 * i + 2]};
    return out;
}

// The callbacks of one solve: the C ABI passes this struct back as `user`.
struct Callbacks {
    std::function<bool()> should_abort, inner_abort;
    std::function<void(const ScfProgress&)> observe;
    static int abort(void* user) {
        auto* c = static_cast<Callbacks*>(user);
        return c->should_abort && c->should_abort() ? 1 : 0;
    }
    static int inner(void* user) {
        auto* c = static_cast<Callbacks*>(user);
        return c->inner_abort && c->inner_abort() ? 1 : 0;
    }
    static void progress(const ks_progress* p, void* user) {
        auto* c = static_cast<Callbacks*>(user);
        if (c->observe) c->observe(*p);
    }
};

}  // namespace detail

// Construction options of the B200 solver (no reference counterpart): the Gram form (0 plain FP32 CUDA cores, 1 the
// tensor-core 3xTF32 "mixed" form), extra LOBPCG bands per occupied channel, and the cold orbitals (0 the reference's
// initial_orbitals, 1 seeded uniform(-1, 1)).
struct Options {
    int gram_mode = 0;
    int n_extra = 0;
    int init_mode = 0;
};

class GpuSolver {
public:
    // GpuSolver::new (crates/qm-gpu/src/scf.rs:1083) on the current CUDA device: an n^3 grid of spacing h (Bohr).
    GpuSolver(int n, double h, Options opts = {}) : n_(n), h_(h) {
        if (!(n >= 5 && n <= 1024 && h > 0.0 && h < 1e300))
            throw InvalidArgument("grid: need 5 <= n <= 1024 and h > 0");
        if (opts.gram_mode < 0 || opts.gram_mode > 1 || opts.n_extra < 0 || opts.init_mode < 0 || opts.init_mode > 1)
            throw InvalidArgument("invalid options");
        const ks_options c{opts.gram_mode, opts.n_extra, opts.init_mode, 0};
        handle_ = ks_solver_create(n, h, &c);
        if (!handle_) throw Device(KS_DEVICE, detail::message(nullptr));
    }
    ~GpuSolver() { ks_solver_destroy(handle_); }
    GpuSolver(const GpuSolver&) = delete;
    GpuSolver& operator=(const GpuSolver&) = delete;
    GpuSolver(GpuSolver&& o) noexcept : handle_(std::exchange(o.handle_, nullptr)), n_(o.n_), h_(o.h_) {}
    GpuSolver& operator=(GpuSolver&& o) noexcept {
        if (this != &o) {
            ks_solver_destroy(handle_);
            handle_ = std::exchange(o.handle_, nullptr);
            n_ = o.n_;
            h_ = o.h_;
        }
        return *this;
    }

    int n() const { return n_; }
    double h() const { return h_; }
    void* handle() const { return handle_; }
    // The solver's CUDA stream (a cudaStream_t), for ordering or timing the caller's own work against it.
    void* stream() const { return ks_solver_stream(handle_); }

    // solve (scf.rs:1195): one SCF to convergence, warm-started from the last converged state when its counts match.
    ScfStats solve(const System& system, const ScfSettings& settings, bool warm = false) {
        return solve_observed(system, settings, warm, nullptr, nullptr, nullptr);
    }
    // solve_with (scf.rs:1208): should_abort is polled before every SCF step; true abandons the solve (Aborted).
    ScfStats solve_with(const System& system, const ScfSettings& settings, bool warm, std::function<bool()> should_abort) {
        return solve_observed(system, settings, warm, std::move(should_abort), nullptr, nullptr);
    }
    // solve_observed / solve_polled (scf.rs:1213-1235): also inner_abort, polled once per LOBPCG iteration, and an
    // observer of every SCF step.
    ScfStats solve_observed(const System& system, const ScfSettings& settings, bool warm, std::function<bool()> should_abort,
                            std::function<bool()> inner_abort, std::function<void(const ScfProgress&)> observe) {
        const std::vector<ks_nucleus> nuc = detail::to_c(system.nuclei);
        const ks_settings s = detail::to_c(settings);
        detail::Callbacks cb{std::move(should_abort), std::move(inner_abort), std::move(observe)};
        ks_stats out{};
        const ks_status st = ks_solve_observed(handle_, nuc.data(), (int)nuc.size(), system.n_up, system.n_dn, &s, warm ? 1 : 0,
                                               cb.should_abort ? &detail::Callbacks::abort : nullptr,
                                               cb.inner_abort ? &detail::Callbacks::inner : nullptr,
                                               cb.observe ? &detail::Callbacks::progress : nullptr, &cb, &out);
        detail::check(st, handle_, &out);
        return out;
    }

    // forces (crates/qm-gpu/src/forces.rs:239): Hellmann-Feynman forces (Ha/Bohr) of the converged state.
    std::vector<Vec3> forces(const std::vector<Nucleus>& nuclei, double sigma) const {
        const std::vector<ks_nucleus> nuc = detail::to_c(nuclei);
        std::vector<double> f(3 * nuclei.size());
        detail::check(ks_forces(handle_, nuc.data(), (int)nuc.size(), sigma, f.data()), handle_);
        return detail::to_vec3(f);
    }
    // The adjoint (no reference counterpart): e_bar dE/dR per nucleus and e_bar dE/dsigma.
    std::pair<std::vector<Vec3>, double> vjp(const std::vector<Nucleus>& nuclei, double sigma, double e_bar = 1.0) const {
        const std::vector<ks_nucleus> nuc = detail::to_c(nuclei);
        std::vector<double> g(3 * nuclei.size());
        double ds = 0.0;
        detail::check(ks_vjp(handle_, nuc.data(), (int)nuc.size(), sigma, e_bar, g.data(), &ds), handle_);
        return {detail::to_vec3(g), ds};
    }

    // The converged state (state() / ks_state): per-spin levels, occupations, densities, potentials, orbitals.
    std::pair<int, int> counts() const {
        int u = 0, d = 0;
        detail::check(ks_state_counts(handle_, &u, &d), handle_);
        return {u, d};
    }
    std::pair<std::vector<double>, std::vector<double>> evals() const {
        const auto c = counts();
        std::vector<double> up(c.first), dn(c.second);
        detail::check(ks_state_evals(handle_, up.data(), dn.data()), handle_);
        return {up, dn};
    }
    std::pair<std::vector<double>, std::vector<double>> occupations() const {
        const auto c = counts();
        std::vector<double> up(c.first), dn(c.second);
        detail::check(ks_state_occupations(handle_, up.data(), dn.data()), handle_);
        return {up, dn};
    }
    std::pair<std::vector<double>, std::vector<double>> density() const {
        std::vector<double> up(points()), dn(points());
        detail::check(ks_state_density(handle_, up.data(), dn.data()), handle_);
        return {up, dn};
    }
    std::pair<std::vector<double>, std::vector<double>> potentials() const {
        std::vector<double> v_nuc(points()), v_h(points());
        detail::check(ks_state_potentials(handle_, v_nuc.data(), v_h.data()), handle_);
        return {v_nuc, v_h};
    }
    std::vector<double> orbitals(int spin) const {
        const auto c = counts();
        std::vector<double> out(points() * (size_t)(spin ? c.second : c.first));
        detail::check(ks_state_orbitals(handle_, spin, out.data()), handle_);
        return out;
    }
    SolveProfile profile() const {
        SolveProfile p{};
        detail::check(ks_profile_get(handle_, &p), handle_);
        return p;
    }

    // The display readouts (crates/qm-gpu/src/sample.rs:84-121, scf.rs:1776-1842).
    std::vector<float> sample_density(const std::vector<Vec3>& points) {
        std::vector<double> flat(3 * points.size());
        for (size_t i = 0; i < points.size(); ++i)
            for (int a = 0; a < 3; ++a) flat[3 * i + a] = points[i][a];
        std::vector<float> out(points.size());
        detail::check(ks_sample_density(handle_, flat.data(), (int)points.size(), out.data()), handle_);
        return out;
    }
    std::vector<float> density_f32() {
        std::vector<float> out(points());
        detail::check(ks_state_density_f32(handle_, out.data()), handle_);
        return out;
    }
    double density_max() {
        double m = 0.0;
        detail::check(ks_density_max(handle_, &m), handle_);
        return m;
    }
    double spin_abs_integral() {
        double s = 0.0;
        detail::check(ks_spin_abs_integral(handle_, &s), handle_);
        return s;
    }

    // set_density_extrapolation / set_witness_cap / effective_eig_tol (scf.rs:1122-1163, :1713-1715).
    void set_density_extrapolation(bool on) { detail::check(ks_set_density_extrapolation(handle_, on ? 1 : 0), handle_); }
    void set_witness_cap(int cap) { detail::check(ks_set_witness_cap(handle_, cap), handle_); }
    double effective_eig_tol(double eig_tol) const {
        double out = 0.0;
        detail::check(ks_effective_eig_tol(handle_, eig_tol, &out), handle_);
        return out;
    }

private:
    size_t points() const { return (size_t)n_ * n_ * n_; }
    void* handle_ = nullptr;
    int n_ = 0;
    double h_ = 0.0;
};

// The device memory (bytes) a solver of this grid holds through a solve and its forces (the provider's footprint
// estimate, crates/providers/src/ks.rs:465-470). InvalidArgument for impossible sizes.
inline long long footprint_bytes(int n, int n_up, int n_dn, Options opts = {}, int diis_history = 6, bool with_core = false) {
    const ks_options c{opts.gram_mode, opts.n_extra, opts.init_mode, 0};
    const long long b = ks_footprint_bytes(n, n_up, n_dn, &c, diis_history, with_core ? 1 : 0);
    if (b < 0) throw InvalidArgument("footprint_bytes: invalid arguments");
    return b;
}

// The solver's host algebra, callable without a device.
struct RitzPairs {
    std::vector<double> theta;  // ascending
    std::vector<double> c;      // column-major m x nk, B-orthonormal columns
    double alpha = 0.0;         // coefficient amplification
};
// The LOBPCG Rayleigh-Ritz step (crates/qm-gpu/src/eigen.rs:515-542): the lowest nk pairs of A c = theta B c for
// symmetric m x m A and B, row-major. Numerical on a non-positive diagonal of B or on rank loss.
inline RitzPairs rayleigh_ritz(int m, const std::vector<double>& a, const std::vector<double>& b, int nk) {
    if (m < 1 || a.size() != (size_t)m * m || b.size() != (size_t)m * m) throw InvalidArgument("rayleigh_ritz: A and B must be m x m");
    RitzPairs r;
    r.theta.resize(nk > 0 ? nk : 0);
    r.c.resize((size_t)m * (nk > 0 ? nk : 0));
    detail::check(ks_rayleigh_ritz(m, a.data(), b.data(), nk, r.theta.data(), r.c.data(), &r.alpha), nullptr);
    return r;
}

// qm::occupations::FdOccupations: f (in evals' order), mu (NaN for an empty channel) and the entropy S.
struct FdOccupations {
    std::vector<double> f;
    double mu = 0.0;
    double entropy = 0.0;
};
// fermi_dirac (crates/qm/src/occupations.rs): InvalidArgument on the reference's refusals (fewer than n + 1 levels,
// a non-finite level or kT), which the reference reports as QmError::Numerical.
inline FdOccupations fermi_dirac(const std::vector<double>& evals, int n, double kt) {
    FdOccupations o;
    o.f.resize(evals.size());
    detail::check(ks_fermi_dirac(evals.data(), (int)evals.size(), n, kt, o.f.data(), &o.mu, &o.entropy), nullptr);
    return o;
}
// witness_reached and witness_keep (crates/qm/src/occupations.rs:283-292, :372-394) on the levels themselves.
inline std::pair<bool, int> fd_witness(const std::vector<double>& evals, int n, double mu, double kt) {
    int reached = 0, keep = 0;
    detail::check(ks_fd_witness(evals.data(), (int)evals.size(), n, mu, kt, &reached, &keep), nullptr);
    return {reached != 0, keep};
}
// witness_bound_reached and witness_keep (occupations.rs:299-317, :372-394) on the lower bounds theta - r.
inline std::pair<bool, int> fd_witness_bound(const std::vector<double>& evals, const std::vector<double>& residuals, int n, double mu,
                                             double kt) {
    if (residuals.size() != evals.size()) throw InvalidArgument("fd_witness_bound: one residual per level");
    int reached = 0, keep = 0;
    detail::check(ks_fd_witness_bound(evals.data(), residuals.data(), (int)evals.size(), n, mu, kt, &reached, &keep), nullptr);
    return {reached != 0, keep};
}
// witness_keep_within (occupations.rs:396-419): the levels to keep, or -1 when no level above the n-th passes both arms
// on its lower bound at a residual within r_max (the block must grow).
inline int fd_witness_keep_within(const std::vector<double>& evals, const std::vector<double>& residuals, int n, double mu, double kt,
                                  double r_max, double tail_kt = 36.0) {
    if (residuals.size() != evals.size()) throw InvalidArgument("fd_witness_keep_within: one residual per level");
    int keep = 0;
    detail::check(ks_fd_witness_keep_within(evals.data(), residuals.data(), (int)evals.size(), n, mu, kt, tail_kt, r_max, &keep), nullptr);
    return keep;
}
// tight_columns (occupations.rs:334-350): the positions the step's tolerance must hold (mu NaN: an empty channel, 0)
inline int fd_tight_columns(const std::vector<double>& evals, const std::vector<double>& residuals, double mu, double kt, double tol) {
    if (residuals.size() != evals.size()) throw InvalidArgument("fd_tight_columns: one residual per level");
    int t = 0;
    detail::check(ks_fd_tight_columns(evals.data(), residuals.data(), (int)evals.size(), mu, kt, tol, &t), nullptr);
    return t;
}
// tight_start (occupations.rs:355-366): a warm state's tight count from its ascending occupations (empty: n)
inline int fd_tight_start(const std::vector<double>& f, int n, double tol) {
    int t = 0;
    detail::check(ks_fd_tight_start(f.empty() ? nullptr : f.data(), (int)f.size(), n, tol, &t), nullptr);
    return t;
}
// The stencil's launch-shape autotuner (ks_autotune_stencil): for each vector count, the z-chunk counts chosen for H psi
// and for the Jacobi sweep on an n^3 grid of the current device (kept for later launches of those shapes).
inline std::vector<std::pair<int, int>> autotune_stencil(int n, const std::vector<int>& counts) {
    std::vector<int> out(2 * counts.size());
    detail::check(ks_autotune_stencil(n, counts.data(), (int)counts.size(), out.data()), nullptr);
    std::vector<std::pair<int, int>> r;
    for (size_t i = 0; i < counts.size(); ++i) r.push_back({out[2 * i], out[2 * i + 1]});
    return r;
}

}  // namespace qm_gpu
