// host_api_check.cpp -- checks of the C++ mirror (include/ks_solver.hpp). Without a GPU: argument errors as
// InvalidArgument, the solver's host algebra against the reference's own known answers, and, with --no-device on a
// machine without a CUDA device, the loud failure of a valid solver (Device, no CPU fallback). With --scf on a GPU:
// the H2 33^3 SCF and forces through qm_gpu::GpuSolver against the reference's pins, and the solver's contract
// (warm start, abort, coincident nuclei, the cap on SCF steps).
//
//   host_api_check <dir holding rr_i1_a.txt and rr_i1_b.txt> [--no-device | --scf]
//
// Prints one "ok <check>" line per check and exits 0, or prints "FAIL <check>: <why>" and exits 1.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ks_solver.hpp"

namespace {

int g_failures = 0;

void expect(bool ok, const char* what, const std::string& why = "") {
    if (ok) {
        std::printf("ok %s\n", what);
    } else {
        std::printf("FAIL %s: %s\n", what, why.c_str());
        ++g_failures;
    }
}

template <class E, class F>
bool throws(F f) {
    try {
        f();
    } catch (const E&) {
        return true;
    } catch (...) {
        return false;
    }
    return false;
}

std::vector<double> load_square(const std::string& path, int& m) {
    std::ifstream in(path);
    std::vector<double> v;
    std::string line;
    m = 0;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        double x;
        int cols = 0;
        while (ls >> x) {
            v.push_back(x);
            ++cols;
        }
        if (cols) ++m;
    }
    return v;
}

// The reference's test rayleigh_ritz_pairs_survive_a_bad_symmetric_eigen (crates/qm-gpu/src/eigen.rs:1188-1201).
void check_rayleigh_ritz(const std::string& dir) {
    int m = 0, mb = 0;
    const std::vector<double> a = load_square(dir + "/rr_i1_a.txt", m);
    const std::vector<double> b = load_square(dir + "/rr_i1_b.txt", mb);
    if (m == 0 || m != mb || a.size() != (size_t)m * m || b.size() != (size_t)m * m) {
        expect(false, "rr_i1 fixtures", "unreadable or not square");
        return;
    }
    const int nk = 8;
    const qm_gpu::RitzPairs r = qm_gpu::rayleigh_ritz(m, a, b, nk);
    double worst = 0.0;
    for (int k = 0; k < nk; ++k) {
        const double* c = r.c.data() + (size_t)m * k;
        double num = 0.0, den = 0.0;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j < m; ++j) {
                num += c[i] * a[(size_t)i * m + j] * c[j];
                den += c[i] * b[(size_t)i * m + j] * c[j];
            }
        worst = std::fmax(worst, std::fabs(num / den - r.theta[k]));
    }
    expect(worst < 1e-9, "rayleigh_ritz: Rayleigh quotients equal the Ritz values", std::to_string(worst));
    expect(std::fabs(r.theta[0] + 0.8686699) < 1e-6, "rayleigh_ritz: theta_0 = -0.8686699", std::to_string(r.theta[0]));
    std::vector<double> bad = b;
    bad[3 * (size_t)m + 3] = 0.0;
    expect(throws<qm_gpu::Numerical>([&] { qm_gpu::rayleigh_ritz(m, a, bad, nk); }), "rayleigh_ritz: a zero norm is Numerical");
    expect(throws<qm_gpu::InvalidArgument>([&] { qm_gpu::rayleigh_ritz(m, a, b, m + 1); }), "rayleigh_ritz: nk > m is an argument error");
}

// A few of the reference's Fermi-Dirac and witness known answers (crates/qm/src/occupations.rs:474-707).
void check_occupations() {
    const qm_gpu::FdOccupations o = qm_gpu::fermi_dirac({-0.3, -0.3}, 1, 1e-3);
    expect(o.f[0] == 0.5 && o.f[1] == 0.5 && std::fabs(o.mu + 0.3) <= 1e-15 && std::fabs(o.entropy - 2 * std::log(2.0)) <= 1e-14,
           "fermi_dirac: a degenerate pair is half filled");
    const qm_gpu::FdOccupations e = qm_gpu::fermi_dirac({-0.3, 0.1}, 0, 5e-3);
    expect(e.f[0] == 0.0 && e.f[1] == 0.0 && std::isnan(e.mu) && e.entropy == 0.0, "fermi_dirac: an empty channel");
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::fermi_dirac({-0.3}, 1, 5e-3); }), "fermi_dirac: too few levels is refused");
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::fermi_dirac({-0.3, NAN}, 1, 5e-3); }), "fermi_dirac: a NaN level is refused");
    const std::vector<double> evals = {-0.5, -0.3, -0.25, -0.1, -0.05, 0.0, 0.3};
    const auto w = qm_gpu::fd_witness(evals, 1, -0.4, 5e-3);
    expect(w.first && w.second == 5, "fd_witness: the witness and its passing spare are kept");
    expect(!qm_gpu::fd_witness({-0.3, -0.3 + 0.099, -0.5}, 2, -0.4, 5e-3).first, "fd_witness: the gap arm");
    const qm_gpu::ScfSettings fg = qm_gpu::ScfSettings::for_grid(0.25);
    expect(fg.sigma == 0.25 && fg.occupations == qm_gpu::Occupations::FermiDirac && fg.kt == 5e-3 && fg.tol == 1e-6 &&
               fg.eig_tol == 1e-6 && fg.mixing == 0.3 && fg.max_iter == 200 && fg.diis_history == 6 && fg.stall_window == 50,
           "ScfSettings::for_grid: the reference's defaults");
    const auto wb = qm_gpu::fd_witness_bound(evals, {0.0, 0.0, 0.0, 0.15, 0.0, 0.0, 0.0}, 1, -0.4, 5e-3);
    expect(wb.first && wb.second == 6, "fd_witness_bound: the witness's own residual pushes it up a rank");
    expect(throws<qm_gpu::InvalidArgument>([&] { qm_gpu::fd_witness_bound(evals, {0.0}, 1, -0.4, 5e-3); }),
           "fd_witness_bound: one residual per level");
    expect(qm_gpu::fd_witness_keep_within(evals, {0.0, 0.0, 0.0, 2e-3, 1e-3, 3e-3, 3e-3}, 1, -0.4, 5e-3, 1.5e-3) == 6,
           "fd_witness_keep_within: the lowest converged witness and its spare");
    expect(qm_gpu::fd_witness_keep_within(evals, {0.0, 0.0, 0.0, 2e-3, 2e-3, 2e-3, 2e-3}, 1, -0.4, 5e-3, 1.5e-3) == -1,
           "fd_witness_keep_within: none within r_max");
    // occupations.rs:634-664 tight_columns_follow_f_and_the_stop (one electron, a 0.2 Ha gap)
    const std::vector<double> tc = {-0.5, -0.3, 0.0, 0.1};
    const double mu1 = qm_gpu::fermi_dirac(tc, 1, 5e-3).mu;
    expect(qm_gpu::fd_tight_columns(tc, {0.0, 0.0, 0.0, 0.0}, mu1, 5e-3, 1e-6) == 1, "fd_tight_columns: the level above is loose");
    expect(qm_gpu::fd_tight_columns(tc, {0.0, 0.0, 0.0, 0.0}, mu1, 5e-3, 1e-7) == 2, "fd_tight_columns: the stop decides");
    expect(qm_gpu::fd_tight_columns({-0.3, -0.5, 0.1, 0.0}, {0.0, 0.0, 0.0, 0.0}, mu1, 5e-3, 1e-6) == 2,
           "fd_tight_columns: positions, not ranks");
    expect(qm_gpu::fd_tight_start({1.0, 1.0, 5e-9, 1e-12}, 2, 1e-6) == 2 && qm_gpu::fd_tight_start({}, 3, 1e-6) == 3,
           "fd_tight_start: the stored occupations' loose tail, n without a state");
}

void check_arguments() {
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::GpuSolver(4, 0.25); }), "GpuSolver: n < 5 is an argument error");
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::GpuSolver(33, -0.25); }), "GpuSolver: h <= 0 is an argument error");
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::GpuSolver(33, NAN); }), "GpuSolver: a NaN h is an argument error");
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::GpuSolver(33, 0.25, {2, 0, 0}); }), "GpuSolver: gram_mode 2 is an argument error");
    expect(throws<qm_gpu::InvalidArgument>([] { qm_gpu::footprint_bytes(4, 1, 1); }), "footprint_bytes: n < 5 is an argument error");
    const long long f33 = qm_gpu::footprint_bytes(33, 1, 1), f65 = qm_gpu::footprint_bytes(65, 1, 1);
    expect(f33 > 0 && f65 > f33, "footprint_bytes grows with the grid");
}

// The 33^3 Aufbau pins of the reference (crates/qm/src/scf.rs:1276-1279): H2 at (+-0.7, 0, 0), h = sigma = 0.25,
// tol 1e-6: E = -0.952449176828 Ha and F_x0 = +0.128755968665 Ha/Bohr, here to 1e-5 Ha and 1e-4 Ha/Bohr.
void check_scf() {
    using namespace qm_gpu;
    GpuSolver so(33, 0.25);
    const System h2{{{{0.7, 0.0, 0.0}, 1}, {{-0.7, 0.0, 0.0}, 1}}, 1, 1};
    ScfSettings st;
    st.sigma = 0.25;
    const ScfStats cold = so.solve(h2, st);
    expect(std::fabs(cold.energy.total + 0.9524491768275237) < 1e-5, "solve: the H2 33^3 energy pin", std::to_string(cold.energy.total));
    const std::vector<Vec3> f = so.forces(h2.nuclei, st.sigma);
    expect(f.size() == 2 && std::fabs(f[0][0] - 0.12875596866453332) < 1e-4, "forces: the H2 33^3 force pin", std::to_string(f[0][0]));
    const auto ev = so.evals();
    // the two spin channels of H2 converge from different seeded guesses: the same level to the eigen tolerance
    expect(ev.first.size() == 1 && ev.second.size() == 1 && std::fabs(ev.first[0] - ev.second[0]) < 1e-5,
           "evals: one level per spin, equal to the eigen tolerance",
           std::to_string(ev.first.empty() ? 0.0 : ev.first[0]) + " " + std::to_string(ev.second.empty() ? 0.0 : ev.second[0]));
    const ScfStats warm = so.solve(h2, st, true);
    expect(warm.iterations < cold.iterations, "solve: a warm start takes fewer steps");
    expect(throws<Aborted>([&] { so.solve_with(h2, st, false, [] { return true; }); }), "solve_with: should_abort abandons the solve");
    ScfSettings capped = st;
    capped.max_iter = 2;
    GpuSolver fresh(33, 0.25);
    expect(throws<ScfNotConverged>([&] { fresh.solve(h2, capped); }), "solve: two steps is ScfNotConverged");
    const System same{{{{0.1, 0.0, 0.0}, 1}, {{0.1, 0.0, 0.0}, 1}}, 1, 1};
    expect(throws<CoincidentNuclei>([&] { fresh.solve(same, st); }), "solve: coincident nuclei");
    expect(throws<NoState>([&] { fresh.forces(h2.nuclei, st.sigma); }), "forces: no state after a failed solve");
}

void check_no_device() {
    expect(throws<qm_gpu::Device>([] { qm_gpu::GpuSolver(33, 0.25, {1, 3, 1}); }), "GpuSolver: no CUDA device is a Device error");
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 2) {
        std::fprintf(stderr, "usage: %s <golden dir> [--no-device | --scf]\n", argv[0]);
        return 2;
    }
    const std::string dir = argv[1];
    const bool no_device = argc > 2 && std::string(argv[2]) == "--no-device";
    const bool scf = argc > 2 && std::string(argv[2]) == "--scf";
    try {
        check_arguments();
        check_rayleigh_ritz(dir);
        check_occupations();
        if (no_device) check_no_device();
        if (scf) check_scf();
    } catch (const std::exception& e) {
        std::printf("FAIL unexpected exception: %s\n", e.what());
        return 1;
    }
    return g_failures ? 1 : 0;
}
