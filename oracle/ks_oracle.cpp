// ks_oracle.cpp -- CPU f64 oracle of the Kohn-Sham SCF hot path.
//
// TEST INFRASTRUCTURE ONLY (the reference of the tests, never the product). A restatement, in plain C++17,
// of the reference's f64 CPU solver, crate `qm`:
//   grid + Neumaier sums      crates/qm/src/grid.rs:1-99
//   8th-order stencil         crates/qm/src/stencil.rs:21-51
//   LSDA (Slater + PW92)      crates/qm/src/xc.rs:88-207
//   smeared nuclei            crates/qm/src/nuclear.rs:98-132, :255-289 (σ = 1 blobs for the Aufbau cold guess)
//   Poisson (Jacobi-CG, l<=6) crates/qm/src/poisson.rs:70-259
//   LOBPCG + Jacobi smoother  crates/qm/src/eigen.rs:114-369
//   Aufbau SCF, DIIS, stall   crates/qm/src/scf.rs:329-1098
//   Hellmann-Feynman forces   crates/qm/src/forces.rs:162-227
// Third-party arithmetic the reference takes from absent crates, restated here:
//   nalgebra 0.33.3 SymmetricEigen -> the reference's own checked fallback, cyclic Jacobi
//   (crates/qm/src/eigen.rs:175-211), used directly; nalgebra LU (partial pivoting) -> Gaussian
//   elimination with partial pivoting (crates/qm/src/scf.rs:681-697); libm 0.2.16 erf (the
//   fdlibm/musl algorithm) -> the C library's erf, which implements the same fdlibm algorithm.
// Summation orders follow the reference expression by expression so that results agree to
// rounding; the eigensolver's rotations inside degenerate clusters may differ (density-invariant).
#include "ks_oracle.h"
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>
#include <thread>

namespace {

constexpr double PI = 3.14159265358979323846;
// crates/qm/src/stencil.rs:19
const double COEFF[5] = {-205.0 / 72.0, 8.0 / 5.0, -1.0 / 5.0, 8.0 / 315.0, -1.0 / 560.0};
int g_threads = 1;

// Runs body(i) for i in [0, n) on g_threads std::threads (static contiguous chunks). Every
// parallel loop here writes only its own elements, so results do not depend on the thread count.
template <class F>
void par_for(long n, F body) {
    int t = g_threads;
    if (t <= 1 || n < 2 * t) { for (long i = 0; i < n; ++i) body(i); return; }
    std::vector<std::thread> pool;
    long chunk = (n + t - 1) / t;
    for (int w = 0; w < t; ++w) {
        long lo = w * chunk, hi = std::min(n, lo + chunk);
        if (lo >= hi) break;
        pool.emplace_back([=, &body] { for (long i = lo; i < hi; ++i) body(i); });
    }
    for (auto& th : pool) th.join();
}

// Runs body(i) for i in [0, n) on up to g_threads std::threads, task i on thread i % threads: for a few
// large independent tasks (each one a serial reduction, such as a Neumaier dot), so again the results do
// not depend on the thread count.
template <class F>
void par_tasks(long n, F body) {
    const int t = (int)std::min<long>(g_threads, n);
    if (t <= 1) { for (long i = 0; i < n; ++i) body(i); return; }
    std::vector<std::thread> pool;
    for (int w = 0; w < t; ++w) pool.emplace_back([=, &body] { for (long i = w; i < n; i += t) body(i); });
    for (auto& th : pool) th.join();
}

using Vec = std::vector<double>;

// ---------------------------------------------------------------- grid (crates/qm/src/grid.rs)
struct Grid {
    int n;
    double h;
    double origin;
    Grid(int n_, double h_) : n(n_), h(h_) {
        double half = (double)(n - 1) * h / 2.0;   // grid.rs:12
        origin = -half;
    }
    size_t len() const { return (size_t)n * n * n; }
    size_t idx(int i, int j, int k) const { return (size_t)i + (size_t)n * ((size_t)j + (size_t)n * k); }
    void point(size_t id, double r[3]) const {
        int i = (int)(id % n), j = (int)((id / n) % n), k = (int)(id / ((size_t)n * n));
        r[0] = origin + (double)i * h;
        r[1] = origin + (double)j * h;
        r[2] = origin + (double)k * h;
    }
    double dv() const { return h * h * h; }
    bool operator==(const Grid& o) const { return n == o.n && h == o.h; }
};

// grid.rs:91-99
template <class F>
double neumaier_fn(size_t n, F f) {
    double sum = 0.0, comp = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double x = f(i);
        double t = sum + x;
        if (std::fabs(sum) >= std::fabs(x)) comp += (sum - t) + x; else comp += (x - t) + sum;
        sum = t;
    }
    return sum + comp;
}
double integrate(const Grid& g, const Vec& f) { return neumaier_fn(g.len(), [&](size_t i) { return f[i]; }) * g.dv(); }
double gdot(const Grid& g, const Vec& a, const Vec& b) {
    return neumaier_fn(g.len(), [&](size_t i) { return a[i] * b[i]; }) * g.dv();
}

// ---------------------------------------------------------------- stencil (stencil.rs:21-51)
void laplacian(const Grid& g, const double* f, double* out) {
    const int n = g.n;
    const double inv_h2 = 1.0 / (g.h * g.h);
    const size_t strides[3] = {1, (size_t)n, (size_t)n * n};
    par_for(n, [&](long k) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                size_t id = g.idx(i, j, (int)k);
                double acc = 3.0 * COEFF[0] * f[id];
                int pos[3] = {i, j, (int)k};
                for (int axis = 0; axis < 3; ++axis)
                    for (int m = 1; m <= 4; ++m) {
                        double c = COEFF[m];
                        if (pos[axis] + m < n) acc += c * f[id + m * strides[axis]];
                        if (pos[axis] >= m) acc += c * f[id - m * strides[axis]];
                    }
                out[id] = acc * inv_h2;
            }
    });
}
void kinetic(const Grid& g, const double* f, double* out) {
    laplacian(g, f, out);
    const size_t N = g.len();
    par_for((long)N, [&](long i) { out[i] *= -0.5; });
}
// eigen.rs:117-122 LocalHamiltonian::apply: kinetic(x) then y += V x, in one pass with the same roundings per point
// (the Laplacian scaled by 1/h^2, then by -1/2, then V x added)
void hamiltonian(const Grid& g, const double* v, const double* x, double* y) {
    const int n = g.n;
    const double inv_h2 = 1.0 / (g.h * g.h);
    const size_t strides[3] = {1, (size_t)n, (size_t)n * n};
    par_for(n, [&](long k) {
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                size_t id = g.idx(i, j, (int)k);
                double acc = 3.0 * COEFF[0] * x[id];
                int pos[3] = {i, j, (int)k};
                for (int axis = 0; axis < 3; ++axis)
                    for (int m = 1; m <= 4; ++m) {
                        double c = COEFF[m];
                        if (pos[axis] + m < n) acc += c * x[id + m * strides[axis]];
                        if (pos[axis] >= m) acc += c * x[id - m * strides[axis]];
                    }
                double out = acc * inv_h2;
                out *= -0.5;
                out += v[id] * x[id];
                y[id] = out;
            }
    });
}

// ---------------------------------------------------------------- xc (xc.rs:88-207)
struct Pw92 { double a, a1, b1, b2, b3, b4; };
const Pw92 PARA = {0.031091, 0.21370, 7.5957, 3.5876, 1.6382, 0.49294};
const Pw92 FERRO = {0.015545, 0.20548, 14.1189, 6.1977, 3.3662, 0.62517};
const Pw92 MALPHA = {0.016887, 0.11125, 10.357, 3.6231, 0.88026, 0.49671};
const double FPP0 = 1.709921;
const double N_MIN = 1e-20;

void pw92_g(double rs, const Pw92& p, double& G, double& dG) {
    double srs = std::sqrt(rs);
    double q0 = -2.0 * p.a * (1.0 + p.a1 * rs);
    double q1 = 2.0 * p.a * (p.b1 * srs + p.b2 * rs + p.b3 * rs * srs + p.b4 * rs * rs);
    double q1p = p.a * (p.b1 / srs + 2.0 * p.b2 + 3.0 * p.b3 * srs + 4.0 * p.b4 * rs);
    double ln = std::log(1.0 + 1.0 / q1);
    G = q0 * ln;
    dG = -2.0 * p.a * p.a1 * ln - q0 * q1p / (q1 * q1 + q1);
}
void f_zeta(double z, double& f, double& fp) {
    double denom = std::pow(2.0, 4.0 / 3.0) - 2.0;
    f = (std::pow(1.0 + z, 4.0 / 3.0) + std::pow(1.0 - z, 4.0 / 3.0) - 2.0) / denom;
    fp = (4.0 / 3.0) * (std::pow(1.0 + z, 1.0 / 3.0) - std::pow(1.0 - z, 1.0 / 3.0)) / denom;
}
void correlation(double nu, double nd, double& e, double& vu, double& vd) {
    double n = nu + nd;
    if (n < N_MIN) { e = vu = vd = 0.0; return; }
    double rs = std::pow(3.0 / (4.0 * PI * n), 1.0 / 3.0);
    double z = std::min(std::max((nu - nd) / n, -1.0), 1.0);
    double ec0, dec0, ec1, dec1, mac, dmac;
    pw92_g(rs, PARA, ec0, dec0);
    pw92_g(rs, FERRO, ec1, dec1);
    pw92_g(rs, MALPHA, mac, dmac);
    double ac = -mac, dac = -dmac;
    double f, fp;
    f_zeta(z, f, fp);
    double z3 = z * z * z, z4 = z3 * z;
    double ec = ec0 + ac * f / FPP0 * (1.0 - z4) + (ec1 - ec0) * f * z4;
    double dec_drs = dec0 + dac * f / FPP0 * (1.0 - z4) + (dec1 - dec0) * f * z4;
    double dec_dz = ac / FPP0 * (fp * (1.0 - z4) - 4.0 * z3 * f) + (ec1 - ec0) * (fp * z4 + 4.0 * z3 * f);
    double common = ec - rs / 3.0 * dec_drs;
    e = n * ec;
    vu = common - (z - 1.0) * dec_dz;
    vd = common - (z + 1.0) * dec_dz;
}
void exchange(double nu, double nd, double& e, double& vu, double& vd) {
    double c = (3.0 / 4.0) * std::pow(3.0 / PI, 1.0 / 3.0) * std::pow(2.0, 1.0 / 3.0);
    e = -c * (std::pow(nu, 4.0 / 3.0) + std::pow(nd, 4.0 / 3.0));
    vu = -std::pow(6.0 * nu / PI, 1.0 / 3.0);
    vd = -std::pow(6.0 * nd / PI, 1.0 / 3.0);
}
void exc_point(double nu, double nd, double& e, double& vu, double& vd) {
    nu = std::fmax(nu, 0.0);
    nd = std::fmax(nd, 0.0);
    if (nu + nd < N_MIN) { e = vu = vd = 0.0; return; }
    double ex, vxu, vxd, ec, vcu, vcd;
    exchange(nu, nd, ex, vxu, vxd);
    correlation(nu, nd, ec, vcu, vcd);
    e = ex + ec; vu = vxu + vcu; vd = vxd + vcd;
}
void lsda(size_t len, const double* nu, const double* nd, double* e, double* vu, double* vd) {
    par_for((long)len, [&](long i) { exc_point(nu[i], nd[i], e[i], vu[i], vd[i]); });
}

// ---------------------------------------------------------------- nuclei (nuclear.rs)
double dist2(const double a[3], const double b[3]) {
    double dx = a[0] - b[0], dy = a[1] - b[1], dz = a[2] - b[2];
    return dx * dx + dy * dy + dz * dz;
}
// nuclear.rs:258-272
void nuclear_potential(const Grid& g, const ora_nucleus* nuc, int nn, double sigma, double* out) {
    double s2 = sigma * std::sqrt(2.0);
    double on_site = std::sqrt(2.0 / PI) / sigma;
    const size_t N = g.len();
    par_for((long)N, [&](long id) {
        double r[3];
        g.point(id, r);
        double acc = -0.0;
        for (int a = 0; a < nn; ++a) {
            double d = std::sqrt(dist2(r, nuc[a].pos));
            double z = (double)nuc[a].z;
            acc += (d < 1e-10) ? -z * on_site : -z * std::erf(d / s2) / d;
        }
        out[id] = acc;
    });
}
// nuclear.rs:98-107
void deposit_charge(const Grid& g, const ora_nucleus* nuc, int nn, double sigma, double* out) {
    double norm = 1.0 / std::pow(2.0 * PI * sigma * sigma, 1.5);
    double inv_2s2 = 1.0 / (2.0 * sigma * sigma);
    const size_t N = g.len();
    par_for((long)N, [&](long id) {
        double r[3];
        g.point(id, r);
        double acc = -0.0;
        for (int a = 0; a < nn; ++a) acc += (double)nuc[a].z * norm * std::exp(-dist2(r, nuc[a].pos) * inv_2s2);
        out[id] = acc;
    });
}
// nuclear.rs:277-289
int nuclear_repulsion(const ora_nucleus* nuc, int nn, double& e) {
    e = 0.0;
    for (int i = 0; i < nn; ++i)
        for (int j = i + 1; j < nn; ++j) {
            double d = std::sqrt(dist2(nuc[i].pos, nuc[j].pos));
            if (d < 1e-8) return -1;
            e += (double)nuc[i].z * (double)nuc[j].z / d;
        }
    return 0;
}
// scf.rs:636-644 initial_orbitals: one LCG stream across all k vectors
void initial_orbitals(const Grid& g, const ora_nucleus* nuc, int nn, int k, uint64_t seed, double* out) {
    const size_t N = g.len();
    for (int v = 0; v < k; ++v)
        for (size_t id = 0; id < N; ++id) {
            seed = seed * 6364136223846793005ULL + 1442695040888963407ULL;
            double u = (double)(seed >> 11) / (double)(1ULL << 53);
            double r[3];
            g.point(id, r);
            double env = -0.0;
            for (int a = 0; a < nn; ++a) env += std::exp(-dist2(r, nuc[a].pos) / 4.0);
            out[(size_t)v * N + id] = (u + 0.5) * env;
        }
}

// ---------------------------------------------------------------- Poisson (poisson.rs)
constexpr int L_MAX = 6, N_MOM = 49;
inline int lm_index(int l, int m) { return l * l + (m + l); }
// poisson.rs:89-120
void solid_harmonics(const double r[3], double out[N_MOM]) {
    double x = r[0], y = r[1], z = r[2];
    double r2 = x * x + y * y + z * z;
    double cr[L_MAX + 1][L_MAX + 1] = {}, ci[L_MAX + 1][L_MAX + 1] = {};
    cr[0][0] = 1.0;
    for (int l = 1; l <= L_MAX; ++l) {
        double lf = l;
        double f = std::sqrt((2.0 * lf - 1.0) / (2.0 * lf));
        double pr = cr[l - 1][l - 1], pi = ci[l - 1][l - 1];
        cr[l][l] = f * (x * pr - y * pi);
        ci[l][l] = f * (x * pi + y * pr);
        for (int m = 0; m < l; ++m) {
            double mf = m;
            double a = (2.0 * lf - 1.0) * z;
            double r1 = cr[l - 1][m], i1 = ci[l - 1][m];
            double r0 = 0.0, i0 = 0.0;
            if (l >= 2 && m <= l - 2) { r0 = cr[l - 2][m]; i0 = ci[l - 2][m]; }
            double b = std::sqrt(std::fmax((lf - 1.0) * (lf - 1.0) - mf * mf, 0.0)) * r2;
            double d = std::sqrt(lf * lf - mf * mf);
            cr[l][m] = (a * r1 - b * r0) / d;
            ci[l][m] = (a * i1 - b * i0) / d;
        }
    }
    double s2 = std::sqrt(2.0);
    for (int l = 0; l <= L_MAX; ++l) {
        out[lm_index(l, 0)] = cr[l][0];
        for (int m = 1; m <= l; ++m) {
            out[lm_index(l, m)] = s2 * cr[l][m];
            out[lm_index(l, -m)] = s2 * ci[l][m];
        }
    }
}

struct Poisson {
    Grid g;
    Vec r, z, p, ap, b, harm;
    explicit Poisson(const Grid& grid) : g(grid) {
        size_t N = g.len();
        r.assign(N, 0); z.assign(N, 0); p.assign(N, 0); ap.assign(N, 0); b.assign(N, 0);
        harm.assign((size_t)N_MOM * N, 0.0);
        par_for((long)N, [&](long i) {
            double pt[3], hh[N_MOM];
            g.point(i, pt);
            solid_harmonics(pt, hh);
            for (int lm = 0; lm < N_MOM; ++lm) harm[(size_t)lm * N + i] = hh[lm];
        });
    }
    void moments(const Vec& rho, double q[N_MOM]) const {
        size_t N = g.len();
        for (int lm = 0; lm < N_MOM; ++lm) {
            const double* hm = harm.data() + (size_t)lm * N;
            q[lm] = neumaier_fn(N, [&](size_t i) { return rho[i] * hm[i]; }) * g.dv();
        }
    }
    static double bc_value(const double q[N_MOM], const double r[3]) {
        double d2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        double hh[N_MOM];
        solid_harmonics(r, hh);
        double acc = 0.0, inv_pow = 1.0 / std::sqrt(d2);
        for (int l = 0; l <= L_MAX; ++l) {
            double s = 0.0;
            for (int m = -l; m <= l; ++m) { int i = lm_index(l, m); s += q[i] * hh[i]; }
            acc += s * inv_pow;
            inv_pow /= d2;
        }
        return acc;
    }
    void apply_a(const double* x, double* y) const {   // y = -L_int x
        laplacian(g, x, y);
        size_t N = g.len();
        par_for((long)N, [&](long i) { y[i] = -y[i]; });
    }
    // poisson.rs:161-179 add_boundary_term (points farther than 4 from every face add +0.0)
    void add_boundary_term(const double q[N_MOM], double* out) const {
        const int n = g.n;
        const double inv_h2 = 1.0 / (g.h * g.h);
        par_for(n, [&](long kk) {
            int k = (int)kk;
            for (int j = 0; j < n; ++j)
                for (int i = 0; i < n; ++i) {
                    int pos[3] = {i, j, k};
                    bool near = false;
                    for (int a = 0; a < 3; ++a) near = near || pos[a] < 4 || pos[a] >= n - 4;
                    if (!near) continue;
                    double acc = 0.0;
                    for (int axis = 0; axis < 3; ++axis)
                        for (int m = 1; m <= 4; ++m)
                            for (int sign = -1; sign <= 1; sign += 2) {
                                int qa = pos[axis] + sign * m;
                                if (qa < 0 || qa >= n) {
                                    double r[3];
                                    g.point(g.idx(i, j, k), r);
                                    r[axis] += (double)(sign * m) * g.h;
                                    acc += COEFF[m] * bc_value(q, r);
                                }
                            }
                    out[g.idx(i, j, k)] += acc * inv_h2;
                }
        });
    }
    // poisson.rs:200-255
    int solve(const Vec& rho, Vec& v, double tol, int max_iter, double& residual) {
        double q[N_MOM];
        moments(rho, q);
        size_t N = g.len();
        par_for((long)N, [&](long i) { b[i] = 4.0 * PI * rho[i]; });
        add_boundary_term(q, b.data());
        apply_a(v.data(), ap.data());
        const double inv_diag = -(g.h * g.h) / (3.0 * COEFF[0]);
        par_for((long)N, [&](long i) { r[i] = b[i] - ap[i]; z[i] = inv_diag * r[i]; });
        double b_norm = std::fmax(std::sqrt(gdot(g, b, b)), 1e-300);
        p = z;
        double dots[2];  // r.z and r.r: independent serial sums, one task each
        par_tasks(2, [&](long t) { dots[t] = t == 0 ? gdot(g, r, z) : gdot(g, r, r); });
        double rz = dots[0];
        int it = 0;
        residual = std::sqrt(dots[1]) / b_norm;
        while (residual > tol && it < max_iter) {
            apply_a(p.data(), ap.data());
            double pap = gdot(g, p, ap);
            double alpha = rz / pap;
            par_for((long)N, [&](long i) {
                v[i] += alpha * p[i];
                r[i] -= alpha * ap[i];
                z[i] = inv_diag * r[i];
            });
            par_tasks(2, [&](long t) { dots[t] = t == 0 ? gdot(g, r, z) : gdot(g, r, r); });
            double rz_new = dots[0];
            double beta = rz_new / rz;
            rz = rz_new;
            par_for((long)N, [&](long i) { p[i] = z[i] + beta * p[i]; });
            residual = std::sqrt(dots[1]) / b_norm;  // p's update leaves r as it was
            ++it;
        }
        return it;
    }
};

// ---------------------------------------------------------------- dense eigen (eigen.rs:175-211)
// cyclic Jacobi on a row-major m x m matrix; V column-major in evecs (evecs[i + m*k] = v_k[i])
void jacobi_sym_eigen(int n, Vec a, double* evals, double* evecs) {
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    Vec v((size_t)n * n, 0.0);
    auto V = [&](int i, int j) -> double& { return v[(size_t)i * n + j]; };
    for (int i = 0; i < n; ++i) V(i, i) = 1.0;
    double norm = 0.0;
    for (double x : a) norm += x * x;
    norm = std::sqrt(norm);
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                if (j != i) off += A(i, j) * A(i, j);
        off = std::sqrt(off);
        if (!(off > 1e-15 * norm)) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A(p, q);
                if (apq == 0.0) continue;
                double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                double sgn = std::signbit(theta) ? -1.0 : 1.0;
                double t = sgn / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                if (theta == 0.0) t = 1.0;
                double c = 1.0 / std::sqrt(t * t + 1.0);
                double s = t * c;
                for (int k = 0; k < n; ++k) {
                    double akp = A(k, p), akq = A(k, q);
                    A(k, p) = c * akp - s * akq;
                    A(k, q) = s * akp + c * akq;
                }
                for (int k = 0; k < n; ++k) {
                    double apk = A(p, k), aqk = A(q, k);
                    A(p, k) = c * apk - s * aqk;
                    A(q, k) = s * apk + c * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    double vkp = V(k, p), vkq = V(k, q);
                    V(k, p) = c * vkp - s * vkq;
                    V(k, q) = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < n; ++i) evals[i] = A(i, i);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) evecs[i + (size_t)n * k] = V(i, k);
}

// ---------------------------------------------------------------- LOBPCG (eigen.rs:213-369)
double jacobi_omega() {
    double symbol_pi = COEFF[0] + 2.0 * (-COEFF[1] + COEFF[2] - COEFF[3] + COEFF[4]);
    double rho = symbol_pi / COEFF[0];
    return 4.0 / (3.0 * rho);
}

// ---------------------------------------------------------------- pseudised ions (ionic.rs, nonlocal.rs)
// An ionic setup restated from the tables a caller passes (the reference's FilteredTable as the grid
// samples it, crates/qm/src/radial/filter.rs:323-363).
struct OraIonic {
    struct Proj { int l; double e_kb, radius; Vec t; };
    struct Sp { int z; double z_v, sigma_lr, du, r_sr, pc_radius; Vec v_sr, rho_pc; std::vector<Proj> proj; };
    std::vector<Sp> sp;
    int find(int z) const {
        for (size_t i = 0; i < sp.size(); ++i) if (sp[i].z == z) return (int)i;
        return -1;
    }
    double charge(int z) const { int i = find(z); return i < 0 ? (double)z : sp[i].z_v; }
};

OraIonic make_ionic(const ora_species* s, int nsp) {
    OraIonic io;
    for (int i = 0; i < nsp; ++i) {
        OraIonic::Sp t;
        t.z = s[i].z; t.z_v = s[i].z_v; t.sigma_lr = s[i].sigma_lr; t.du = s[i].du;
        t.r_sr = s[i].n_v_sr > 0 ? s[i].r_sr : 0.0;
        t.v_sr.assign(s[i].v_sr, s[i].v_sr + s[i].n_v_sr);
        t.pc_radius = s[i].pc_radius > 0.0 ? s[i].pc_radius : 0.0;
        if (t.pc_radius > 0.0) t.rho_pc.assign(s[i].rho_pc, s[i].rho_pc + s[i].n_rho_pc);
        for (int k = 0; k < s[i].n_proj; ++k)
            t.proj.push_back({s[i].proj_l[k], s[i].proj_e_kb[k], s[i].proj_radius[k], Vec(s[i].proj_t[k], s[i].proj_t[k] + s[i].proj_n[k])});
        io.sp.push_back(std::move(t));
    }
    return io;
}

// filter.rs:302-317 uniform_lagrange, and :355 read (0 beyond the radius): value and d/dd
void table_read(const Vec& f, double du, double radius, double d, double& v, double& dv) {
    v = dv = 0.0;
    if (d > radius) return;
    const double s = d / du;
    const long i0 = (long)std::floor(s) - 1;
    if (i0 + 3 >= (long)f.size()) return;
    auto at = [&](long i) { return f[(size_t)(i < 0 ? -i : i)]; };
    const double t = s - (double)i0;
    const double a = at(i0), b = at(i0 + 1), c = at(i0 + 2), e = at(i0 + 3);
    const double l[4] = {-(t - 1.0) * (t - 2.0) * (t - 3.0) / 6.0, t * (t - 2.0) * (t - 3.0) / 2.0, -t * (t - 1.0) * (t - 3.0) / 2.0,
                         t * (t - 1.0) * (t - 2.0) / 6.0};
    const double dl[4] = {-((t - 2.0) * (t - 3.0) + (t - 1.0) * (t - 3.0) + (t - 1.0) * (t - 2.0)) / 6.0,
                          ((t - 2.0) * (t - 3.0) + t * (t - 3.0) + t * (t - 2.0)) / 2.0,
                          -((t - 1.0) * (t - 3.0) + t * (t - 3.0) + t * (t - 1.0)) / 2.0,
                          ((t - 1.0) * (t - 2.0) + t * (t - 2.0) + t * (t - 1.0)) / 6.0};
    v = a * l[0] + b * l[1] + c * l[2] + e * l[3];
    dv = (a * dl[0] + b * dl[1] + c * dl[2] + e * dl[3]) / du;
}

// nuclear.rs:320-336 points_within: a clipped index box, then |r - c| <= radius, ascending
std::vector<size_t> points_within(const Grid& g, const double c[3], double radius) {
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
        double l = std::fmax(std::floor((c[a] - radius - g.origin) / g.h), 0.0);
        double h = std::fmin(std::ceil((c[a] + radius - g.origin) / g.h), (double)(g.n - 1));
        if (!(h >= l)) return {};
        lo[a] = (int)l;
        hi[a] = (int)h;
    }
    std::vector<size_t> out;
    for (int k = lo[2]; k <= hi[2]; ++k)
        for (int j = lo[1]; j <= hi[1]; ++j)
            for (int i = lo[0]; i <= hi[0]; ++i) {
                size_t p = g.idx(i, j, k);
                double r[3];
                g.point(p, r);
                if (dist2(r, c) <= radius * radius) out.push_back(p);
            }
    return out;
}

// nuclear.rs:297-302 smeared_potential with per-centre (q, sigma) + :338-346 the V_SR tables
void ionic_local_potential(const Grid& g, const ora_nucleus* nuc, int nn, double sigma_ae, const OraIonic& io, double* out) {
    const size_t N = g.len();
    par_for((long)N, [&](long id) {
        double r[3];
        g.point(id, r);
        double acc = -0.0;
        for (int a = 0; a < nn; ++a) {
            const int si = io.find(nuc[a].z);
            const double q = si < 0 ? (double)nuc[a].z : io.sp[si].z_v, sg = si < 0 ? sigma_ae : io.sp[si].sigma_lr;
            const double d = std::sqrt(dist2(r, nuc[a].pos));
            const double on_site = std::sqrt(2.0 / PI) / sg;
            acc += (d < 1e-10) ? -q * on_site : -q * std::erf(d / (sg * std::sqrt(2.0))) / d;
        }
        out[id] = acc;
    });
    for (int a = 0; a < nn; ++a) {
        const int si = io.find(nuc[a].z);
        if (si < 0 || io.sp[si].v_sr.empty()) continue;
        const auto& t = io.sp[si];
        for (size_t p : points_within(g, nuc[a].pos, t.r_sr)) {
            double r[3], v, dv;
            g.point(p, r);
            table_read(t.v_sr, t.du, t.r_sr, std::sqrt(dist2(r, nuc[a].pos)), v, dv);
            out[p] += v;
        }
    }
}

// nuclear.rs:350-359
void partial_core_field(const Grid& g, const ora_nucleus* nuc, int nn, const OraIonic& io, double* out) {
    std::fill(out, out + g.len(), 0.0);
    for (int a = 0; a < nn; ++a) {
        const int si = io.find(nuc[a].z);
        if (si < 0 || !(io.sp[si].pc_radius > 0.0)) continue;
        const auto& t = io.sp[si];
        for (size_t p : points_within(g, nuc[a].pos, t.pc_radius)) {
            double r[3], v, dv;
            g.point(p, r);
            table_read(t.rho_pc, t.du, t.pc_radius, std::sqrt(dist2(r, nuc[a].pos)), v, dv);
            out[p] += v;
        }
    }
}

// nonlocal.rs:87-98 grad R_lm, l <= 2, lm order
void grad_rlm(int l, int m, const double d[3], double g[3]) {
    const double s3 = std::sqrt(3.0), x = d[0], y = d[1], z = d[2];
    g[0] = g[1] = g[2] = 0.0;
    if (l == 1) { if (m == -1) g[1] = 1.0; else if (m == 0) g[2] = 1.0; else g[0] = 1.0; }
    if (l == 2) {
        if (m == -2) { g[0] = s3 * y; g[1] = s3 * x; }
        else if (m == -1) { g[1] = s3 * z; g[2] = s3 * y; }
        else if (m == 0) { g[0] = -x; g[1] = -y; g[2] = 2.0 * z; }
        else if (m == 1) { g[0] = s3 * z; g[2] = s3 * x; }
        else { g[0] = s3 * x; g[1] = -s3 * y; }
    }
}

// One projector sphere (nonlocal.rs Sphere): its ion, l, E_KB, points and beta_lm[m + l][point] (+ gradients)
struct OraSphere {
    int ion, l;
    double e_kb;
    std::vector<size_t> pts;
    std::vector<Vec> beta;
    std::vector<std::vector<double>> grad;  // [m + l][3 * point + axis]
};

// nonlocal.rs build_inner
std::vector<OraSphere> build_nonlocal(const Grid& g, const ora_nucleus* nuc, int nn, const OraIonic& io, bool with_grad) {
    std::vector<OraSphere> out;
    for (int a = 0; a < nn; ++a) {
        const int si = io.find(nuc[a].z);
        if (si < 0) continue;
        const auto& t = io.sp[si];
        for (const auto& p : t.proj) {
            OraSphere s;
            s.ion = a;
            s.l = p.l;
            s.e_kb = p.e_kb;
            s.pts = points_within(g, nuc[a].pos, p.radius);
            const double norm = std::sqrt((2.0 * p.l + 1.0) / (4.0 * PI));
            s.beta.assign(2 * p.l + 1, Vec(s.pts.size()));
            if (with_grad) s.grad.assign(2 * p.l + 1, std::vector<double>(3 * s.pts.size()));
            for (size_t q = 0; q < s.pts.size(); ++q) {
                double r[3];
                g.point(s.pts[q], r);
                double d[3] = {r[0] - nuc[a].pos[0], r[1] - nuc[a].pos[1], r[2] - nuc[a].pos[2]};
                double dd = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                double sh[N_MOM];
                solid_harmonics(d, sh);
                double tv, dt;
                table_read(p.t, t.du, p.radius, dd, tv, dt);
                const double tn = tv * norm;
                for (int m = -p.l; m <= p.l; ++m) {
                    const int lm = lm_index(p.l, m);
                    s.beta[m + p.l][q] = tn * sh[lm];
                    if (with_grad) {
                        double gr[3];
                        grad_rlm(p.l, m, d, gr);
                        const double radial = dd > 1e-12 ? dt * norm * sh[lm] / dd : 0.0;
                        for (int ax = 0; ax < 3; ++ax) s.grad[m + p.l][3 * q + ax] = radial * d[ax] + tn * gr[ax];
                    }
                }
            }
            out.push_back(std::move(s));
        }
    }
    return out;
}

// c_lm[x] = h^3 Neumaier sum over the sphere of beta x (nonlocal.rs "On the grid")
double project(const Grid& g, const OraSphere& s, int row, const double* x) {
    return neumaier_fn(s.pts.size(), [&](size_t q) { return s.beta[row][q] * x[s.pts[q]]; }) * g.dv();
}

// y += V_NL x = sum_spheres sum_m E_KB c_lm[x] beta_lm
void nonlocal_add(const Grid& g, const std::vector<OraSphere>& nl, const double* x, double* y) {
    for (const auto& s : nl)
        for (int r = 0; r < 2 * s.l + 1; ++r) {
            const double w = s.e_kb * project(g, s, r, x);
            for (size_t q = 0; q < s.pts.size(); ++q) y[s.pts[q]] += w * s.beta[r][q];
        }
}

// H = -1/2 lap + V (+ V_NL)
void ham(const Grid& g, const double* v, const std::vector<OraSphere>* nl, const double* x, double* y) {
    hamiltonian(g, v, x, y);
    if (nl && !nl->empty()) nonlocal_add(g, *nl, x, y);
}

struct Precond {
    const Grid& g;
    const double* v;
    double lambda, omega;
    Vec inv_d;
    Precond(const Grid& grid, const double* vv, double lam) : g(grid), v(vv), lambda(lam), omega(jacobi_omega()) {
        double diag_t = -1.5 * COEFF[0] / (g.h * g.h);
        size_t N = g.len();
        inv_d.resize(N);
        par_for((long)N, [&](long i) { inv_d[i] = 1.0 / std::fmax(diag_t + v[i] - lambda, 0.1); });
    }
    void apply(const double* r, double* w) const {
        size_t N = g.len();
        par_for((long)N, [&](long i) { w[i] = r[i] * inv_d[i]; });
        Vec hw(N);
        for (int s = 1; s < 4; ++s) {   // JACOBI_SWEEPS = 4
            hamiltonian(g, v, w, hw.data());
            par_for((long)N, [&](long i) { w[i] += omega * inv_d[i] * (r[i] - (hw[i] - lambda * w[i])); });
        }
    }
};

// modified Gram-Schmidt in Grid::dot; drops norm < 1e-12 (eigen.rs:243-255). Each vector's projections run in order,
// a dot against its current value and then the update, exactly as one loop over the vectors does, so the result is
// bitwise that of one thread. Across vectors they run as a wavefront on g_threads threads: vector s projects out
// vector j as soon as j is final (kept or dropped). Threads take the vectors round-robin in increasing order, so the
// lowest unfinished vector always has every earlier vector final and a thread working on it: no thread waits forever.
void orthonormalise(const Grid& g, std::vector<Vec>& s) {
    const int m = (int)s.size();
    const size_t N = g.len();
    std::vector<std::atomic<int>> state(m);  // 0 in progress, 1 kept, 2 dropped
    for (auto& x : state) x.store(0, std::memory_order_relaxed);
    par_tasks(m, [&](long idx) {
        Vec& v = s[idx];
        for (long j = 0; j < idx; ++j) {
            int st;
            while ((st = state[j].load(std::memory_order_acquire)) == 0) std::this_thread::yield();
            if (st != 1) continue;
            const Vec& q = s[j];
            const double c = gdot(g, q, v);
            for (size_t i = 0; i < N; ++i) v[i] -= c * q[i];
        }
        const double nrm = std::sqrt(gdot(g, v, v));
        const bool keep = nrm > 1e-12;
        if (keep)
            for (size_t i = 0; i < N; ++i) v[i] /= nrm;
        state[idx].store(keep ? 1 : 2, std::memory_order_release);
    });
    std::vector<Vec> kept;
    for (int i = 0; i < m; ++i)
        if (state[i].load(std::memory_order_relaxed) == 1) kept.push_back(std::move(s[i]));
    s = std::move(kept);
}

// eigen.rs:285-369 lobpcg_impl with head = k (no tiers)
int lobpcg(const Grid& g, const double* v, std::vector<Vec>& x, Vec& evals, const Precond* pc, double tol, int max_iter,
           double& max_residual, const std::vector<OraSphere>* nl = nullptr) {
    const int k = (int)x.size();
    const size_t N = g.len();
    std::vector<Vec> xs = x;
    orthonormalise(g, xs);
    if ((int)xs.size() != k) return -1;
    std::vector<Vec> p;
    std::vector<Vec> hx(k, Vec(N));
    int iterations = 0;
    max_residual = std::numeric_limits<double>::infinity();
    for (;;) {
        for (int i = 0; i < k; ++i) ham(g, v, nl, xs[i].data(), hx[i].data());
        par_tasks(k, [&](long i) { evals[i] = gdot(g, xs[i], hx[i]); });
        std::vector<Vec> w;
        double max_res = 0.0;
        Vec r(N);
        for (int i = 0; i < k; ++i) {
            par_for((long)N, [&](long j) { r[j] = hx[i][j] - evals[i] * xs[i][j]; });
            double ri = std::sqrt(gdot(g, r, r));
            max_res = std::fmax(max_res, ri);
            if (std::isnan(ri)) max_res = ri;
            Vec wi(N);
            if (pc) pc->apply(r.data(), wi.data()); else wi = r;
            w.push_back(std::move(wi));
        }
        max_residual = max_res;
        if (max_res < tol || iterations >= max_iter) break;
        ++iterations;
        std::vector<Vec> s;
        for (auto& xi : xs) s.push_back(xi);
        for (auto& wi : w) s.push_back(std::move(wi));
        for (auto& pi : p) s.push_back(pi);
        orthonormalise(g, s);
        const int m = (int)s.size();
        std::vector<Vec> hs(m, Vec(N));
        for (int i = 0; i < m; ++i) ham(g, v, nl, s[i].data(), hs[i].data());
        Vec a((size_t)m * m);
        std::vector<std::pair<int, int>> pairs;
        for (int i = 0; i < m; ++i)
            for (int j = 0; j <= i; ++j) pairs.emplace_back(i, j);
        par_tasks((long)pairs.size(), [&](long t) {  // each entry one serial Neumaier dot
            const int i = pairs[t].first, j = pairs[t].second;
            const double val = gdot(g, s[i], hs[j]);
            a[(size_t)i * m + j] = val;
            a[(size_t)j * m + i] = val;
        });
        Vec ev(m), evec((size_t)m * m);
        jacobi_sym_eigen(m, a, ev.data(), evec.data());
        std::vector<int> order(m);
        for (int i = 0; i < m; ++i) order[i] = i;
        std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return ev[i] < ev[j]; });
        std::vector<Vec> new_x(k, Vec(N, 0.0)), new_p(k, Vec(N, 0.0));
        // per point, each output sums its terms in input order (si ascending) from 0, as a column-by-column pass does
        par_for((long)N, [&](long j) {
            for (int col = 0; col < k; ++col) {
                const double* c = evec.data() + (size_t)m * order[col];
                double sx = new_x[col][j], sp = new_p[col][j];
                for (int si = 0; si < m; ++si) {
                    const double coef = c[si];
                    if (coef == 0.0) continue;
                    sx += coef * s[si][j];
                    if (si >= k) sp += coef * s[si][j];
                }
                new_x[col][j] = sx;
                new_p[col][j] = sp;
            }
        });
        xs = std::move(new_x);
        orthonormalise(g, xs);
        if ((int)xs.size() != k) return -2;
        p = std::move(new_p);
    }
    x = xs;
    return iterations;
}

// ---------------------------------------------------------------- DIIS (scf.rs:674-718)
// LU with partial pivoting (nalgebra's `lu()`), None on a zero pivot
bool lu_solve(int n, Vec a, Vec& b) {
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    for (int col = 0; col < n; ++col) {
        int piv = col;
        double best = std::fabs(A(col, col));
        for (int r = col + 1; r < n; ++r)
            if (std::fabs(A(r, col)) > best) { best = std::fabs(A(r, col)); piv = r; }
        if (A(piv, col) == 0.0) return false;
        if (piv != col) {
            for (int j = 0; j < n; ++j) std::swap(A(col, j), A(piv, j));
            std::swap(b[col], b[piv]);
        }
        for (int r = col + 1; r < n; ++r) {
            double l = A(r, col) / A(col, col);
            A(r, col) = l;
            for (int j = col + 1; j < n; ++j) A(r, j) -= l * A(col, j);
        }
    }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) b[i] -= A(i, j) * b[j];
    for (int i = n - 1; i >= 0; --i) {
        for (int j = i + 1; j < n; ++j) b[i] -= A(i, j) * b[j];
        b[i] /= A(i, i);
    }
    return true;
}
bool diis_coefficients_from_gram(int m, const Vec& gram, Vec& c) {
    Vec b((size_t)(m + 1) * (m + 1), 0.0);
    auto B = [&](int i, int j) -> double& { return b[(size_t)i * (m + 1) + j]; };
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) B(i, j) = gram[(size_t)i * m + j];
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = std::fmax(scale, B(i, i));
    if (!(scale > 0.0)) return false;
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) B(i, j) /= scale;
        B(i, i) += 1e-12;
    }
    for (int i = 0; i < m; ++i) { B(i, m) = 1.0; B(m, i) = 1.0; }
    Vec rhs(m + 1, 0.0);
    rhs[m] = 1.0;
    if (!lu_solve(m + 1, b, rhs)) return false;
    c.assign(rhs.begin(), rhs.begin() + m);
    for (double x : c)
        if (!std::isfinite(x)) return false;
    return true;
}

struct DiisEntry { Vec rho_up, rho_dn, r_up, r_dn; };

void diis_mix(const Grid& g, std::vector<DiisEntry>& hist, double alpha, Vec& up, Vec& dn) {
    Vec c;
    for (;;) {
        if (hist.size() == 1) { c.assign(1, 1.0); break; }
        int m = (int)hist.size();
        Vec gram((size_t)m * m);
        for (int i = 0; i < m; ++i)
            for (int j = 0; j <= i; ++j) {
                double v = gdot(g, hist[i].r_up, hist[j].r_up) + gdot(g, hist[i].r_dn, hist[j].r_dn);
                gram[(size_t)i * m + j] = v;
                gram[(size_t)j * m + i] = v;
            }
        if (diis_coefficients_from_gram(m, gram, c)) break;
        hist.erase(hist.begin());
    }
    size_t N = g.len();
    for (size_t i = 0; i < N; ++i) {
        double u = 0.0, d = 0.0;
        for (size_t e = 0; e < hist.size(); ++e) {
            u += c[e] * (hist[e].rho_up[i] + alpha * hist[e].r_up[i]);
            d += c[e] * (hist[e].rho_dn[i] + alpha * hist[e].r_dn[i]);
        }
        up[i] = std::fmax(u, 0.0);
        dn[i] = std::fmax(d, 0.0);
    }
}

// ---------------------------------------------------------------- forces (forces.rs:162-227)
double g_prime(double d, double sigma) {
    if (d < 1e-8) return 0.0;
    double u = d / (sigma * std::sqrt(2.0));
    return ((2.0 / std::sqrt(PI)) * u * std::exp(-u * u) - std::erf(u)) / (d * d);
}

// ---------------------------------------------------------------- Fermi-Dirac (crates/qm/src/occupations.rs)
// f at x = (e - mu)/kT without forming an e^|x| > 1 (occupations.rs: `occupation`)
double fd_occupation(double x) {
    if (x >= 0.0) {
        double e = std::exp(-x);
        return e / (1.0 + e);
    }
    return 1.0 / (1.0 + std::exp(x));
}
// s(x) = ln(1 + e^-|x|) + |x| / (1 + e^|x|) (occupations.rs: `fd_entropy`)
double fd_entropy(double x) {
    double a = std::fabs(x);
    if (std::isinf(a)) return 0.0;
    return std::log1p(std::exp(-a)) + a / (1.0 + std::exp(a));
}
double fd_total(const double* ev, int k, double mu, double kt) {
    return neumaier_fn((size_t)k, [&](size_t i) { return fd_occupation((ev[i] - mu) / kt); });
}
// one tie-directed bisection: ge -> returns hi (the least mu with sum f >= n), else lo (occupations.rs: `bisect`)
double fd_bisect(const double* ev, int k, double n, double kt, double lo, double hi, bool ge) {
    for (int h = 0; h < 2048; ++h) {
        double mid = 0.5 * lo + 0.5 * hi;
        if (mid <= lo || mid >= hi) break;
        double d = fd_total(ev, k, mid, kt) - n;
        bool to_hi = ge ? d >= 0.0 : d > 0.0;
        if (to_hi) hi = mid; else lo = mid;
    }
    return ge ? hi : lo;
}
// occupations.rs: `fermi_dirac` (n = 0: every f = 0, S = 0)
int fermi_dirac(const double* ev, int k, int n, double kt, double* f, double& mu, double& S) {
    if (n == 0) {
        for (int i = 0; i < k; ++i) f[i] = 0.0;
        mu = NAN;
        S = 0.0;
        return 0;
    }
    if (k < n + 1 || !(std::isfinite(kt) && kt > 0.0)) return -1;
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < k; ++i) {
        if (!std::isfinite(ev[i])) return -1;
        lo = std::fmin(lo, ev[i]);
        hi = std::fmax(hi, ev[i]);
    }
    lo -= 50.0 * kt;
    hi += 50.0 * kt;
    const double nf = (double)n;
    if (!(std::isfinite(lo) && std::isfinite(hi) && fd_total(ev, k, lo, kt) < nf && fd_total(ev, k, hi, kt) > nf)) return -1;
    double mu_minus = fd_bisect(ev, k, nf, kt, lo, hi, true);
    double mu_plus = fd_bisect(ev, k, nf, kt, lo, hi, false);
    mu = 0.5 * mu_minus + 0.5 * mu_plus;
    for (int i = 0; i < k; ++i) f[i] = fd_occupation((ev[i] - mu) / kt);
    S = neumaier_fn((size_t)k, [&](size_t i) { return fd_entropy((ev[i] - mu) / kt); });
    return 0;
}
// occupations.rs: `witness_reached` -- the highest level at least WITNESS_GAP = 0.1 Ha above the n-th lowest and
// 36 kT above mu
bool fd_witness(const Vec& ev, int n, double mu, double kt) {
    if (n == 0) return true;
    if ((int)ev.size() <= n) return false;
    Vec s = ev;
    std::sort(s.begin(), s.end());
    return s.back() >= s[n - 1] + 0.1 && s.back() - mu >= 36.0 * kt;
}

}  // namespace

struct ora_state {
    Grid g{1, 1.0};
    std::vector<Vec> orb_up, orb_dn;
    Vec ev_up, ev_dn, rho_up, rho_dn, v_nuc, v_h;
    Vec occ_up, occ_dn;  // one occupation per stored orbital (all 1 under Aufbau)
    double sigma = 0;
    bool ionic = false;  // solved under an ionic setup
};

extern "C" {

void ora_set_threads(int n) { g_threads = n < 1 ? 1 : n; }

double ora_neumaier(const double* v, size_t n) { return neumaier_fn(n, [&](size_t i) { return v[i]; }); }

void ora_laplacian(int n, double h, const double* f, double* out) { laplacian(Grid(n, h), f, out); }

void ora_hamiltonian(int n, double h, const double* f, const double* v, double* out) { hamiltonian(Grid(n, h), v, f, out); }

void ora_exc_point(double nu, double nd, double* e, double* vu, double* vd) { exc_point(nu, nd, *e, *vu, *vd); }

void ora_lsda(size_t len, const double* nu, const double* nd, double* e, double* vu, double* vd) { lsda(len, nu, nd, e, vu, vd); }

void ora_nuclear_potential(int n, double h, const ora_nucleus* nuc, int nn, double sigma, double* out) {
    nuclear_potential(Grid(n, h), nuc, nn, sigma, out);
}

void ora_deposit_charge(int n, double h, const ora_nucleus* nuc, int nn, double sigma, double* out) {
    deposit_charge(Grid(n, h), nuc, nn, sigma, out);
}

int ora_nuclear_repulsion(const ora_nucleus* nuc, int nn, double* e) { return nuclear_repulsion(nuc, nn, *e); }

void ora_initial_orbitals(int n, double h, const ora_nucleus* nuc, int nn, int k, unsigned long long seed, double* out) {
    initial_orbitals(Grid(n, h), nuc, nn, k, seed, out);
}

void ora_solid_harmonics(const double r[3], double out[49]) { solid_harmonics(r, out); }

double ora_jacobi_omega(void) { return jacobi_omega(); }

void ora_jacobi_precond(int n, double h, const double* v, double lambda, const double* r, double* w) {
    Grid g(n, h);
    Precond pc(g, v, lambda);
    pc.apply(r, w);
}

int ora_poisson_solve(int n, double h, const double* rho, double* v, double tol, int max_iter, double* residual) {
    Grid g(n, h);
    Poisson ps(g);
    Vec r(rho, rho + g.len()), vv(v, v + g.len());
    int it = ps.solve(r, vv, tol, max_iter, *residual);
    std::copy(vv.begin(), vv.end(), v);
    return it;
}

void ora_multipole_moments(int n, double h, const double* rho, double q[49]) {
    Grid g(n, h);
    Poisson ps(g);
    Vec r(rho, rho + g.len());
    ps.moments(r, q);
}

int ora_lobpcg(int n, double h, const double* v, int k, double* x, double* evals, int precond, double lambda, double tol,
               int max_iter, double* max_residual) {
    Grid g(n, h);
    size_t N = g.len();
    std::vector<Vec> xs(k);
    for (int i = 0; i < k; ++i) xs[i].assign(x + (size_t)i * N, x + (size_t)(i + 1) * N);
    Vec ev(k);
    std::unique_ptr<Precond> pc;
    if (precond) pc.reset(new Precond(g, v, lambda));
    int it = lobpcg(g, v, xs, ev, pc.get(), tol, max_iter, *max_residual);
    if (it < 0) return it;
    for (int i = 0; i < k; ++i) std::copy(xs[i].begin(), xs[i].end(), x + (size_t)i * N);
    std::copy(ev.begin(), ev.end(), evals);
    return it;
}

void ora_sym_eigen(int m, const double* a, double* evals, double* evecs) {
    jacobi_sym_eigen(m, Vec(a, a + (size_t)m * m), evals, evecs);
}

int ora_diis_coefficients(int m, const double* gram, double* c) {
    Vec cc;
    if (!diis_coefficients_from_gram(m, Vec(gram, gram + (size_t)m * m), cc)) return 0;
    std::copy(cc.begin(), cc.end(), c);
    return 1;
}

// scf.rs:928-1098 scf_tiered, with the ionic setup of scf.rs:114-140 when io holds species
static ora_state* scf_impl(int n, double h, const ora_nucleus* nuc, int nn, int n_up, int n_dn, const ora_settings* s,
                           const OraIonic* io, const ora_state* warm, ora_stats* st) {
    Grid g(n, h);
    const size_t N = g.len();
    std::memset(st, 0, sizeof(*st));
    const bool ionic = io && !io->sp.empty();
    double e_nn;
    if (nuclear_repulsion(nuc, nn, e_nn) != 0) { st->status = 3; return nullptr; }
    if (ionic) {  // nuclear.rs:368-378 ionic_repulsion: valence charges
        e_nn = 0.0;
        for (int i = 0; i < nn; ++i)
            for (int j = i + 1; j < nn; ++j) e_nn += io->charge(nuc[i].z) * io->charge(nuc[j].z) / std::sqrt(dist2(nuc[i].pos, nuc[j].pos));
    }
    auto state = std::make_unique<ora_state>();
    state->g = g;
    state->sigma = s->sigma;
    state->ionic = ionic;
    Vec v_nuc(N), rho_pc;
    std::vector<OraSphere> nl;
    if (ionic) {
        ionic_local_potential(g, nuc, nn, s->sigma, *io, v_nuc.data());
        bool core = false;
        for (int a = 0; a < nn; ++a) { int si = io->find(nuc[a].z); core = core || (si >= 0 && io->sp[si].pc_radius > 0.0); }
        if (core) { rho_pc.resize(N); partial_core_field(g, nuc, nn, *io, rho_pc.data()); }
        nl = build_nonlocal(g, nuc, nn, *io, false);
    } else {
        nuclear_potential(g, nuc, nn, s->sigma, v_nuc.data());
    }
    // LSDA on (up + pc/2, dn + pc/2) (scf.rs:759-768)
    auto xc = [&](const Vec& up, const Vec& dn, Vec& e, Vec& xu, Vec& xd) {
        if (rho_pc.empty()) { lsda(N, up.data(), dn.data(), e.data(), xu.data(), xd.data()); return; }
        Vec u(N), d(N);
        for (size_t i = 0; i < N; ++i) { u[i] = up[i] + 0.5 * rho_pc[i]; d[i] = dn[i] + 0.5 * rho_pc[i]; }
        lsda(N, u.data(), d.data(), e.data(), xu.data(), xd.data());
    };
    Poisson poisson(g);
    const double ptol = std::fmin(1e-10, 1e-3 * s->tol);   // scf.rs:503 poisson_tol
    const int PMAX = 5000;
    double eig_res = 0.0, pois_res = 0.0;
    int pois_it = 0;

    std::vector<Vec> orb_up, orb_dn;
    Vec ev_up, ev_dn, in_up, in_dn, v_h;
    const bool fd = s->occupations == 1;
    // one block of N_sigma + n_extra levels per occupied channel under Fermi-Dirac (the reference grows a
    // witness block by doubling; a fixed block whose top level passes the witness gives the same f to e^-36)
    const int ku = n_up + ((fd && n_up > 0) ? std::max(1, s->n_extra) : 0);
    const int kd = n_dn + ((fd && n_dn > 0) ? std::max(1, s->n_extra) : 0);
    bool reuse = warm && warm->g == g && (int)warm->orb_up.size() == ku && (int)warm->orb_dn.size() == kd && !ionic && !warm->ionic;
    if (reuse) {
        orb_up = warm->orb_up; orb_dn = warm->orb_dn; ev_up = warm->ev_up; ev_dn = warm->ev_dn;
        in_up = warm->rho_up; in_dn = warm->rho_dn; v_h = warm->v_h;
    } else {
        double total = (double)(n_up + n_dn);
        double z_tot = 0.0;
        for (int a = 0; a < nn; ++a) z_tot += ionic ? io->charge(nuc[a].z) : (double)nuc[a].z;
        Vec guess(N);
        deposit_charge(g, nuc, nn, 1.0, guess.data());   // nuclear.rs:212-214, Aufbau: σ = 1 blobs
        if (ionic) {  // nuclear.rs:204-206 deposit_centres: each centre's charge q in a σ = 1 blob
            const double norm = 1.0 / std::pow(2.0 * PI, 1.5);
            par_for((long)N, [&](long id) {
                double r[3];
                g.point(id, r);
                double acc = -0.0;
                for (int a = 0; a < nn; ++a) acc += io->charge(nuc[a].z) * norm * std::exp(-dist2(r, nuc[a].pos) * 0.5);
                guess[id] = acc;
            });
        }
        double scale = z_tot > 0.0 ? total / z_tot : 0.0;
        double fu = total > 0.0 ? n_up / total : 0.0, fd = total > 0.0 ? n_dn / total : 0.0;
        Vec buf;
        buf.resize((size_t)std::max(ku, 1) * N);
        initial_orbitals(g, nuc, nn, ku, 1, buf.data());
        for (int i = 0; i < ku; ++i) orb_up.emplace_back(buf.begin() + (size_t)i * N, buf.begin() + (size_t)(i + 1) * N);
        buf.assign((size_t)std::max(kd, 1) * N, 0.0);
        initial_orbitals(g, nuc, nn, kd, 2, buf.data());
        for (int i = 0; i < kd; ++i) orb_dn.emplace_back(buf.begin() + (size_t)i * N, buf.begin() + (size_t)(i + 1) * N);
        ev_up.assign(ku, -1.0);
        ev_dn.assign(kd, -1.0);
        in_up.resize(N); in_dn.resize(N);
        for (size_t i = 0; i < N; ++i) { in_up[i] = guess[i] * scale * fu; in_dn[i] = guess[i] * scale * fd; }
        v_h.assign(N, 0.0);
    }

    int iterations = 0;
    double delta_rho = std::numeric_limits<double>::infinity();
    Vec out_up = in_up, out_dn = in_dn;
    Vec occ_up(orb_up.size(), 1.0), occ_dn(orb_dn.size(), 1.0);
    double entropy = 0.0, mu_up = NAN, mu_dn = NAN;
    std::vector<DiisEntry> hist;
    // StallWatch (scf.rs:440-480)
    double anchor = INFINITY, best = INFINITY;
    int anchor_at = 0;
    double level = 1e-3 * (n_up + n_dn);
    bool stalled = false;
    Vec rho_in(N), vu(N), vd(N), exc(N), xu(N), xd(N);
    while (iterations < s->max_iter) {
        ++iterations;
        for (size_t i = 0; i < N; ++i) rho_in[i] = in_up[i] + in_dn[i];
        double pr;
        int pit = poisson.solve(rho_in, v_h, ptol, PMAX, pr);
        pois_res = std::fmax(pois_res, pr);
        pois_it = std::max(pois_it, pit);
        st->poisson_iterations_total += pit;
        xc(in_up, in_dn, exc, xu, xd);
        for (size_t i = 0; i < N; ++i) { vu[i] = v_nuc[i] + v_h[i] + xu[i]; vd[i] = v_nuc[i] + v_h[i] + xd[i]; }
        for (int spin = 0; spin < 2; ++spin) {
            auto& orb = spin ? orb_dn : orb_up;
            auto& ev = spin ? ev_dn : ev_up;
            const Vec& v = spin ? vd : vu;
            if (orb.empty()) continue;
            double lambda = ev.empty() ? -1.0 : ev[0];
            Precond pc(g, v.data(), lambda);
            double mr;
            int it = lobpcg(g, v.data(), orb, ev, &pc, s->eig_tol, 200, mr, &nl);
            if (it < 0) { st->status = 4; return nullptr; }
            eig_res = std::fmax(eig_res, mr);
            st->eigen_iterations_total += it;
        }
        // occupations of this step's levels (Aufbau: the block is exactly N_sigma, all f = 1)
        occ_up.assign(orb_up.size(), 1.0);
        occ_dn.assign(orb_dn.size(), 1.0);
        entropy = 0.0;
        if (fd) {
            double su = 0.0, sd = 0.0;
            if (fermi_dirac(ev_up.data(), (int)ev_up.size(), n_up, s->kt, occ_up.data(), mu_up, su) != 0 ||
                fermi_dirac(ev_dn.data(), (int)ev_dn.size(), n_dn, s->kt, occ_dn.data(), mu_dn, sd) != 0) {
                st->status = 4;
                return nullptr;
            }
            entropy = su + sd;
        }
        out_up.assign(N, 0.0);
        out_dn.assign(N, 0.0);
        for (size_t o = 0; o < orb_up.size(); ++o) for (size_t i = 0; i < N; ++i) out_up[i] += occ_up[o] * orb_up[o][i] * orb_up[o][i];
        for (size_t o = 0; o < orb_dn.size(); ++o) for (size_t i = 0; i < N; ++i) out_dn[i] += occ_dn[o] * orb_dn[o][i] * orb_dn[o][i];
        delta_rho = neumaier_fn(N, [&](size_t i) {
            return std::fabs(out_up[i] - in_up[i]) + std::fabs(out_dn[i] - in_dn[i]);
        }) * g.dv();
        if (delta_rho < best) best = delta_rho;
        if (std::isfinite(delta_rho) && (!std::isfinite(anchor) || delta_rho <= 0.5 * anchor)) { anchor = delta_rho; anchor_at = iterations; }
        int since = iterations - anchor_at;
        bool is_stalled = s->stall_window > 0 && since >= s->stall_window && best >= level;
        if (!std::isfinite(delta_rho)) break;
        if (delta_rho < s->tol) break;
        if (is_stalled) { stalled = true; break; }
        DiisEntry e;
        e.r_up.resize(N); e.r_dn.resize(N);
        for (size_t i = 0; i < N; ++i) { e.r_up[i] = out_up[i] - in_up[i]; e.r_dn[i] = out_dn[i] - in_dn[i]; }
        e.rho_up = std::move(in_up);
        e.rho_dn = std::move(in_dn);
        hist.push_back(std::move(e));
        if ((int)hist.size() > std::max(s->diis_history, 1)) hist.erase(hist.begin());
        in_up.assign(N, 0.0);
        in_dn.assign(N, 0.0);
        diis_mix(g, hist, s->mixing, in_up, in_dn);
    }
    st->iterations = iterations;
    st->delta_rho = delta_rho;
    st->max_eigen_residual = eig_res;
    if (stalled) { st->status = 2; return nullptr; }
    if (!(delta_rho < s->tol)) { st->status = 1; return nullptr; }
    if (fd && !(fd_witness(ev_up, n_up, mu_up, s->kt) && fd_witness(ev_dn, n_dn, mu_dn, s->kt))) { st->status = 5; return nullptr; }

    Vec rho(N);
    for (size_t i = 0; i < N; ++i) rho[i] = out_up[i] + out_dn[i];
    double pr;
    int pit = poisson.solve(rho, v_h, ptol, PMAX, pr);
    pois_res = std::fmax(pois_res, pr);
    pois_it = std::max(pois_it, pit);
    st->poisson_iterations_total += pit;
    Vec t(N);
    double kinetic_e = 0.0;
    for (int spin = 0; spin < 2; ++spin) {
        auto& orb = spin ? orb_dn : orb_up;
        auto& occ = spin ? occ_dn : occ_up;
        for (size_t o = 0; o < orb.size(); ++o) {
            kinetic(g, orb[o].data(), t.data());
            kinetic_e += occ[o] * gdot(g, orb[o], t);
        }
    }
    xc(out_up, out_dn, exc, xu, xd);
    double external_ = gdot(g, rho, v_nuc);
    if (!nl.empty()) {  // E_NL = sum f E_KB c^2, Neumaier over (orbital, sphere, m) (nonlocal.rs)
        Vec terms;
        for (int spin = 0; spin < 2; ++spin) {
            auto& orb = spin ? orb_dn : orb_up;
            auto& occ = spin ? occ_dn : occ_up;
            for (size_t o = 0; o < orb.size(); ++o)
                for (const auto& sp : nl)
                    for (int r = 0; r < 2 * sp.l + 1; ++r) {
                        double c = project(g, sp, r, orb[o].data());
                        terms.push_back(occ[o] * sp.e_kb * c * c);
                    }
        }
        external_ += neumaier_fn(terms.size(), [&](size_t i) { return terms[i]; });
    }
    double hartree = 0.5 * gdot(g, rho, v_h);
    double xc_e = integrate(g, exc);
    double internal = kinetic_e + external_ + hartree + xc_e + e_nn;
    double bmax = 0.0;
    for (int k = 0; k < n; ++k)
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i)
                if (i == 0 || j == 0 || k == 0 || i == n - 1 || j == n - 1 || k == n - 1)
                    bmax = std::fmax(bmax, std::fabs(rho[g.idx(i, j, k)]));
    st->kinetic = kinetic_e; st->external_ = external_; st->hartree = hartree; st->xc = xc_e; st->nuclear = e_nn;
    st->ts = fd ? s->kt * entropy : 0.0;
    st->entropy = entropy;
    st->mu[0] = mu_up;
    st->mu[1] = mu_dn;
    st->total = internal - st->ts;
    st->boundary_density = bmax;
    st->poisson_residual = pois_res;
    st->poisson_iterations = pois_it;
    st->electrons[0] = integrate(g, out_up);
    st->electrons[1] = integrate(g, out_dn);
    st->status = 0;
    state->orb_up = std::move(orb_up); state->orb_dn = std::move(orb_dn);
    state->ev_up = ev_up; state->ev_dn = ev_dn;
    state->occ_up = occ_up; state->occ_dn = occ_dn;
    state->rho_up = std::move(out_up); state->rho_dn = std::move(out_dn);
    state->v_nuc = std::move(v_nuc); state->v_h = std::move(v_h);
    return state.release();
}

ora_state* ora_scf(int n, double h, const ora_nucleus* nuc, int nn, int n_up, int n_dn, const ora_settings* s,
                   const ora_state* warm, ora_stats* st) {
    return scf_impl(n, h, nuc, nn, n_up, n_dn, s, nullptr, warm, st);
}

ora_state* ora_scf_ionic(int n, double h, const ora_nucleus* nuc, int nn, int n_up, int n_dn, const ora_settings* s,
                         const ora_species* species, int n_species, const ora_state* warm, ora_stats* st) {
    OraIonic io = make_ionic(species, n_species);
    return scf_impl(n, h, nuc, nn, n_up, n_dn, s, &io, warm, st);
}

void ora_ionic_local_potential(int n, double h, const ora_nucleus* nuc, int nn, double sigma_ae, const ora_species* species,
                               int n_species, double* out) {
    ionic_local_potential(Grid(n, h), nuc, nn, sigma_ae, make_ionic(species, n_species), out);
}

void ora_partial_core(int n, double h, const ora_nucleus* nuc, int nn, const ora_species* species, int n_species, double* out) {
    partial_core_field(Grid(n, h), nuc, nn, make_ionic(species, n_species), out);
}

int ora_nonlocal_apply(int n, double h, const ora_nucleus* nuc, int nn, const ora_species* species, int n_species, const double* x,
                       int count, double* out, double* c) {
    Grid g(n, h);
    const size_t N = g.len();
    auto nl = build_nonlocal(g, nuc, nn, make_ionic(species, n_species), false);
    int rows = 0;
    for (const auto& sp : nl) rows += 2 * sp.l + 1;
    for (int v = 0; v < count; ++v) {
        std::fill(out + (size_t)v * N, out + (size_t)(v + 1) * N, 0.0);
        nonlocal_add(g, nl, x + (size_t)v * N, out + (size_t)v * N);
        if (c) {
            int row = 0;
            for (const auto& sp : nl)
                for (int r = 0; r < 2 * sp.l + 1; ++r) c[(size_t)v * rows + row++] = project(g, sp, r, x + (size_t)v * N);
        }
    }
    return rows;
}

double ora_frozen_energy(const ora_state* st, const ora_nucleus* nuc, int nn, double sigma, const ora_species* species,
                         int n_species) {
    const Grid& g = st->g;
    const size_t N = g.len();
    OraIonic io = make_ionic(species, n_species);
    Vec rho(N), vloc(N), pc(N, 0.0), e(N), xu(N), xd(N), u(N), d(N);
    for (size_t i = 0; i < N; ++i) rho[i] = st->rho_up[i] + st->rho_dn[i];
    ionic_local_potential(g, nuc, nn, sigma, io, vloc.data());
    partial_core_field(g, nuc, nn, io, pc.data());
    for (size_t i = 0; i < N; ++i) { u[i] = st->rho_up[i] + 0.5 * pc[i]; d[i] = st->rho_dn[i] + 0.5 * pc[i]; }
    lsda(N, u.data(), d.data(), e.data(), xu.data(), xd.data());
    double en = gdot(g, rho, vloc) + integrate(g, e);
    auto nl = build_nonlocal(g, nuc, nn, io, false);
    for (int spin = 0; spin < 2; ++spin) {
        const auto& orb = spin ? st->orb_dn : st->orb_up;
        const auto& occ = spin ? st->occ_dn : st->occ_up;
        for (size_t o = 0; o < orb.size(); ++o)
            for (const auto& sp : nl)
                for (int r = 0; r < 2 * sp.l + 1; ++r) {
                    const double c = project(g, sp, r, orb[o].data());
                    en += occ[o] * sp.e_kb * c * c;
                }
    }
    for (int i = 0; i < nn; ++i)
        for (int j = i + 1; j < nn; ++j) en += io.charge(nuc[i].z) * io.charge(nuc[j].z) / std::sqrt(dist2(nuc[i].pos, nuc[j].pos));
    return en;
}

void ora_table_read(const double* f, int len, double du, double radius, double d, double* v, double* dv) {
    table_read(Vec(f, f + len), du, radius, d, *v, *dv);
}

void ora_solid_harmonic_gradients(const double r[3], double out[27]) {
    for (int l = 0; l <= 2; ++l)
        for (int m = -l; m <= l; ++m) grad_rlm(l, m, r, out + 3 * lm_index(l, m));
}

// forces.rs (pseudised ions): F_I = -dE/dR_I at frozen orbitals and occupations
int ora_forces_ionic(const ora_state* st, const ora_nucleus* nuc, int nn, double sigma, const ora_species* species, int n_species,
                     double* out3n) {
    const Grid& g = st->g;
    const size_t N = g.len();
    OraIonic io = make_ionic(species, n_species);
    Vec rho(N), pc(N, 0.0), vbar(N, 0.0);
    for (size_t i = 0; i < N; ++i) rho[i] = st->rho_up[i] + st->rho_dn[i];
    bool core = false;
    for (int a = 0; a < nn; ++a) { int si = io.find(nuc[a].z); core = core || (si >= 0 && io.sp[si].pc_radius > 0.0); }
    if (core) {
        partial_core_field(g, nuc, nn, io, pc.data());
        par_for((long)N, [&](long i) {
            double e, vu, vd;
            exc_point(st->rho_up[i] + 0.5 * pc[i], st->rho_dn[i] + 0.5 * pc[i], e, vu, vd);
            vbar[i] = 0.5 * (vu + vd);
        });
    }
    Vec comp[3] = {Vec(N), Vec(N), Vec(N)};
    for (int a = 0; a < nn; ++a) {
        const int si = io.find(nuc[a].z);
        const double q = si < 0 ? (double)nuc[a].z : io.sp[si].z_v, sg = si < 0 ? sigma : io.sp[si].sigma_lr;
        for (int c = 0; c < 3; ++c) std::fill(comp[c].begin(), comp[c].end(), 0.0);
        par_for((long)N, [&](long p) {
            double r[3];
            g.point(p, r);
            double dv[3] = {r[0] - nuc[a].pos[0], r[1] - nuc[a].pos[1], r[2] - nuc[a].pos[2]};
            double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            if (d < 1e-8) return;
            const double u = d / (sg * std::sqrt(2.0));
            double gsum = -q * ((2.0 / std::sqrt(PI)) * u * std::exp(-u * u) - std::erf(u)) / (d * d) * rho[p];
            if (si >= 0) {
                const auto& t = io.sp[si];
                double v, dvv;
                if (!t.v_sr.empty()) { table_read(t.v_sr, t.du, t.r_sr, d, v, dvv); gsum += rho[p] * dvv; }
                if (t.pc_radius > 0.0) { table_read(t.rho_pc, t.du, t.pc_radius, d, v, dvv); gsum += vbar[p] * dvv; }
            }
            for (int c = 0; c < 3; ++c) comp[c][p] = gsum / d * dv[c];
        });
        for (int c = 0; c < 3; ++c) out3n[3 * a + c] = integrate(g, comp[c]);
    }
    // nonlocal: sum_{sigma, i} 2 f_i E_KB c <grad beta | psi_i>
    auto nl = build_nonlocal(g, nuc, nn, io, true);
    for (int spin = 0; spin < 2; ++spin) {
        const auto& orb = spin ? st->orb_dn : st->orb_up;
        const auto& occ = spin ? st->occ_dn : st->occ_up;
        for (size_t o = 0; o < orb.size(); ++o)
            for (const auto& sp : nl)
                for (int r = 0; r < 2 * sp.l + 1; ++r) {
                    const double c = project(g, sp, r, orb[o].data());
                    for (int ax = 0; ax < 3; ++ax) {
                        const double gb = neumaier_fn(sp.pts.size(), [&](size_t q) { return sp.grad[r][3 * q + ax] * orb[o][sp.pts[q]]; }) * g.dv();
                        out3n[3 * sp.ion + ax] += 2.0 * occ[o] * sp.e_kb * c * gb;
                    }
                }
    }
    for (int a = 0; a < nn; ++a)
        for (int b = 0; b < nn; ++b) {
            if (b == a) continue;
            double dv[3] = {nuc[a].pos[0] - nuc[b].pos[0], nuc[a].pos[1] - nuc[b].pos[1], nuc[a].pos[2] - nuc[b].pos[2]};
            double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            if (d < 1e-8) return -1;
            double s = io.charge(nuc[a].z) * io.charge(nuc[b].z) / (d * d * d);
            for (int c = 0; c < 3; ++c) out3n[3 * a + c] += s * dv[c];
        }
    return 0;
}

void ora_state_free(ora_state* st) { delete st; }

int ora_state_counts(const ora_state* st, int* n_up, int* n_dn) {
    *n_up = (int)st->orb_up.size();
    *n_dn = (int)st->orb_dn.size();
    return st->g.n;
}

void ora_state_evals(const ora_state* st, double* up, double* dn) {
    std::copy(st->ev_up.begin(), st->ev_up.end(), up);
    std::copy(st->ev_dn.begin(), st->ev_dn.end(), dn);
}

void ora_state_occupations(const ora_state* st, double* up, double* dn) {
    std::copy(st->occ_up.begin(), st->occ_up.end(), up);
    std::copy(st->occ_dn.begin(), st->occ_dn.end(), dn);
}

int ora_fermi_dirac(const double* evals, int k, int n, double kt, double* f, double* mu, double* entropy) {
    double m = NAN, S = 0.0;
    int rc = fermi_dirac(evals, k, n, kt, f, m, S);
    *mu = m;
    *entropy = S;
    return rc;
}

void ora_state_density(const ora_state* st, double* rho_up, double* rho_dn) {
    std::copy(st->rho_up.begin(), st->rho_up.end(), rho_up);
    std::copy(st->rho_dn.begin(), st->rho_dn.end(), rho_dn);
}

void ora_state_potentials(const ora_state* st, double* v_nuc, double* v_h) {
    std::copy(st->v_nuc.begin(), st->v_nuc.end(), v_nuc);
    std::copy(st->v_h.begin(), st->v_h.end(), v_h);
}

void ora_state_orbitals(const ora_state* st, int spin, double* out) {
    const auto& o = spin ? st->orb_dn : st->orb_up;
    size_t N = st->g.len();
    for (size_t i = 0; i < o.size(); ++i) std::copy(o[i].begin(), o[i].end(), out + i * N);
}

// forces.rs:205-227 all_electron_forces
int ora_forces(const ora_state* st, const ora_nucleus* nuc, int nn, double sigma, double* out3n) {
    const Grid& g = st->g;
    size_t N = g.len();
    Vec rho(N);
    for (size_t i = 0; i < N; ++i) rho[i] = st->rho_up[i] + st->rho_dn[i];
    Vec comp[3] = {Vec(N), Vec(N), Vec(N)};
    for (int a = 0; a < nn; ++a) {
        double z = (double)nuc[a].z;
        for (int c = 0; c < 3; ++c) std::fill(comp[c].begin(), comp[c].end(), 0.0);
        par_for((long)N, [&](long p) {
            double r[3];
            g.point(p, r);
            double dv[3] = {r[0] - nuc[a].pos[0], r[1] - nuc[a].pos[1], r[2] - nuc[a].pos[2]};
            double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            if (d < 1e-8) return;
            double gp = -z * g_prime(d, sigma) / d;
            for (int c = 0; c < 3; ++c) comp[c][p] = rho[p] * gp * dv[c];
        });
        for (int c = 0; c < 3; ++c) out3n[3 * a + c] = integrate(g, comp[c]);
        for (int b = 0; b < nn; ++b) {
            if (b == a) continue;
            double dv[3] = {nuc[a].pos[0] - nuc[b].pos[0], nuc[a].pos[1] - nuc[b].pos[1], nuc[a].pos[2] - nuc[b].pos[2]};
            double d = std::sqrt(dv[0] * dv[0] + dv[1] * dv[1] + dv[2] * dv[2]);
            if (d < 1e-8) return -1;
            double s = z * (double)nuc[b].z / (d * d * d);
            for (int c = 0; c < 3; ++c) out3n[3 * a + c] += s * dv[c];
        }
    }
    return 0;
}

// crates/qm/src/grid.rs:54-67 (trilinear_cell) and :74-86 (trilinear)
void ora_trilinear(int n, double h, const double* f, const double* pts3, int count, double* out) {
    const double origin = -((double)(n - 1) * h / 2.0);
    for (int q = 0; q < count; ++q) {
        int c[3];
        double t[3];
        bool inside = true;
        for (int a = 0; a < 3 && inside; ++a) {
            const double x = (pts3[3 * q + a] - origin) / h;
            if (!(x >= 0.0 && x <= (double)(n - 1))) { inside = false; break; }
            const double i0 = std::floor(x);
            c[a] = (int)i0;
            t[a] = x - i0;
        }
        if (!inside) { out[q] = 0.0; continue; }
        auto at = [&](int di, int dj, int dk) {
            const int a = c[0] + di, b = c[1] + dj, cc = c[2] + dk;
            return (a < n && b < n && cc < n) ? f[(size_t)a + (size_t)n * ((size_t)b + (size_t)n * cc)] : 0.0;
        };
        auto lerp = [](double a, double b, double tt) { return a * (1.0 - tt) + b * tt; };
        auto xl = [&](int dj, int dk) { return lerp(at(0, dj, dk), at(1, dj, dk), t[0]); };
        auto yl = [&](int dk) { return lerp(xl(0, dk), xl(1, dk), t[1]); };
        out[q] = lerp(yl(0), yl(1), t[2]);
    }
}

}  // extern "C"
