// dense.cpp -- host f64 dense linear algebra for the Rayleigh-Ritz and DIIS solves.
//
// The symmetric eigensolver is the classic two-phase method (published: Householder reduction to
// tridiagonal form, then the implicit QL iteration with shifts and accumulated rotations, as in
// the public-domain EISPACK tql2 / JAMA formulation), followed by the reference's pair-residual
// check and Jacobi refinement (crates/qm/src/eigen.rs:150-211).
#include "dense.h"
#include <algorithm>
#include <cmath>

namespace ks {
namespace dense {

namespace {
constexpr double SYM_EIGEN_CHECK = 1e-11;  // crates/qm/src/eigen.rs:171
}

void jacobi_eigen(int n, Mat a, std::vector<double>& evals, std::vector<double>& evecs) {
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    std::vector<double> v((size_t)n * n, 0.0);
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
        if (!(std::sqrt(off) > 1e-15 * norm)) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                double apq = A(p, q);
                if (apq == 0.0) continue;
                double theta = (A(q, q) - A(p, p)) / (2.0 * apq);
                double t = (std::signbit(theta) ? -1.0 : 1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                if (theta == 0.0) t = 1.0;
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
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
    evals.resize(n);
    evecs.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) evals[i] = A(i, i);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) evecs[i + (size_t)n * k] = V(i, k);
}

void tridiag_ql_eigen(int n, const Mat& a_in, std::vector<double>& evals, std::vector<double>& evecs) {
    evals.assign(n, 0.0);
    evecs.assign((size_t)n * n, 0.0);
    if (n == 0) return;
    Mat A = a_in;
    auto a = [&](int i, int j) -> double& { return A[(size_t)i * n + j]; };
    Mat Z((size_t)n * n, 0.0);  // row-major accumulator, Z[r][c]
    auto z = [&](int i, int j) -> double& { return Z[(size_t)i * n + j]; };
    for (int i = 0; i < n; ++i) z(i, i) = 1.0;
    std::vector<double> v(n), p(n), w(n);
    // --- Householder: A <- H A H for k = 0..n-3, Z <- Z H
    for (int k = 0; k + 2 < n; ++k) {
        double tail = 0.0;
        for (int i = k + 2; i < n; ++i) tail += a(i, k) * a(i, k);
        if (tail == 0.0) continue;  // column already tridiagonal
        double x0 = a(k + 1, k);
        double xnorm = std::sqrt(tail + x0 * x0);
        double alpha = x0 >= 0.0 ? -xnorm : xnorm;
        std::fill(v.begin(), v.end(), 0.0);
        for (int i = k + 1; i < n; ++i) v[i] = a(i, k);
        v[k + 1] -= alpha;
        double vn2 = 0.0;
        for (int i = k + 1; i < n; ++i) vn2 += v[i] * v[i];
        if (vn2 == 0.0) continue;
        double beta = 2.0 / vn2;
        for (int i = k; i < n; ++i) {
            double s = 0.0;
            for (int j = k + 1; j < n; ++j) s += a(i, j) * v[j];
            p[i] = beta * s;
        }
        double K = 0.0;
        for (int j = k + 1; j < n; ++j) K += v[j] * p[j];
        K *= 0.5 * beta;
        for (int i = k; i < n; ++i) w[i] = p[i] - K * v[i];
        w[k] = p[k];  // v[k] = 0
        for (int i = k; i < n; ++i)
            for (int j = k; j < n; ++j) a(i, j) -= v[i] * w[j] + w[i] * v[j];
        for (int r = 0; r < n; ++r) {
            double qv = 0.0;
            for (int j = k + 1; j < n; ++j) qv += z(r, j) * v[j];
            qv *= beta;
            for (int j = k + 1; j < n; ++j) z(r, j) -= qv * v[j];
        }
    }
    std::vector<double> d(n), e(n, 0.0);
    for (int i = 0; i < n; ++i) d[i] = a(i, i);
    for (int i = 0; i + 1 < n; ++i) e[i] = a(i + 1, i);
    // --- implicit QL with shifts on the tridiagonal (d, e), rotations accumulated into Z
    double f = 0.0, tst1 = 0.0;
    const double eps = std::ldexp(1.0, -52);
    for (int l = 0; l < n; ++l) {
        tst1 = std::max(tst1, std::fabs(d[l]) + std::fabs(e[l]));
        int m = l;
        while (m < n - 1 && std::fabs(e[m]) > eps * tst1) ++m;
        if (m > l) {
            int iter = 0;
            do {
                if (++iter > 200) break;
                double g = d[l];
                double pp = (d[l + 1] - g) / (2.0 * e[l]);
                double r = std::hypot(pp, 1.0);
                if (pp < 0) r = -r;
                d[l] = e[l] / (pp + r);
                d[l + 1] = e[l] * (pp + r);
                double dl1 = d[l + 1];
                double h = g - d[l];
                for (int i = l + 2; i < n; ++i) d[i] -= h;
                f += h;
                pp = d[m];
                double c = 1.0, c2 = 1.0, c3 = 1.0, el1 = e[l + 1], s = 0.0, s2 = 0.0;
                for (int i = m - 1; i >= l; --i) {
                    c3 = c2;
                    c2 = c;
                    s2 = s;
                    g = c * e[i];
                    h = c * pp;
                    r = std::hypot(pp, e[i]);
                    e[i + 1] = s * r;
                    s = e[i] / r;
                    c = pp / r;
                    pp = c * d[i] - s * g;
                    d[i + 1] = h + s * (c * g + s * d[i]);
                    for (int k = 0; k < n; ++k) {
                        double hz = z(k, i + 1);
                        z(k, i + 1) = s * z(k, i) + c * hz;
                        z(k, i) = c * z(k, i) - s * hz;
                    }
                }
                pp = -s * s2 * c3 * el1 * e[l] / dl1;
                e[l] = s * pp;
                d[l] = c * pp;
            } while (std::fabs(e[l]) > eps * tst1);
        }
        d[l] += f;
        e[l] = 0.0;
    }
    for (int k = 0; k < n; ++k) {
        evals[k] = d[k];
        for (int i = 0; i < n; ++i) evecs[i + (size_t)n * k] = z(i, k);
    }
}

void sym_eigen(int n, const Mat& a, std::vector<double>& evals, std::vector<double>& evecs) {
    tridiag_ql_eigen(n, a, evals, evecs);
    double scale = 1.0;
    for (double l : evals) scale = std::max(scale, 1.0 + std::fabs(l));
    bool bad = false;
    for (int k = 0; k < n && !bad; ++k) {
        double r2 = 0.0;
        for (int i = 0; i < n; ++i) {
            double s = -evals[k] * evecs[i + (size_t)n * k];
            for (int j = 0; j < n; ++j) s += a[(size_t)i * n + j] * evecs[j + (size_t)n * k];
            r2 += s * s;
        }
        if (!(std::sqrt(r2) <= SYM_EIGEN_CHECK * scale)) bad = true;
    }
    if (!bad) return;
    // refine: Jacobi on V^T A V when V is orthonormal, else on A itself
    double orth = 0.0;
    for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) {
            double s = (p == q) ? -1.0 : 0.0;
            for (int i = 0; i < n; ++i) s += evecs[i + (size_t)n * p] * evecs[i + (size_t)n * q];
            orth += s * s;
        }
    if (!(std::sqrt(orth) <= 1e-10)) {
        jacobi_eigen(n, a, evals, evecs);
        return;
    }
    Mat av((size_t)n * n, 0.0), m((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
        for (int k = 0; k < n; ++k) {
            double s = 0.0;
            for (int j = 0; j < n; ++j) s += a[(size_t)i * n + j] * evecs[j + (size_t)n * k];
            av[(size_t)i * n + k] = s;
        }
    for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) {
            double s = 0.0;
            for (int i = 0; i < n; ++i) s += evecs[i + (size_t)n * p] * av[(size_t)i * n + q];
            m[(size_t)p * n + q] = s;
        }
    for (int p = 0; p < n; ++p)
        for (int q = p + 1; q < n; ++q) {
            double s = 0.5 * (m[(size_t)p * n + q] + m[(size_t)q * n + p]);
            m[(size_t)p * n + q] = m[(size_t)q * n + p] = s;
        }
    std::vector<double> re, rv;
    jacobi_eigen(n, m, re, rv);
    std::vector<double> out((size_t)n * n, 0.0);
    for (int k = 0; k < n; ++k)
        for (int i = 0; i < n; ++i) {
            double s = 0.0;
            for (int j = 0; j < n; ++j) s += evecs[i + (size_t)n * j] * rv[j + (size_t)n * k];
            out[i + (size_t)n * k] = s;
        }
    evals = re;
    evecs = out;
}

bool cholesky(int n, Mat& a) {
    for (int j = 0; j < n; ++j) {
        double s = a[(size_t)j * n + j];
        for (int k = 0; k < j; ++k) s -= a[(size_t)j * n + k] * a[(size_t)j * n + k];
        if (!(s > 0.0)) return false;
        double ljj = std::sqrt(s);
        a[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; ++i) {
            double t = a[(size_t)i * n + j];
            for (int k = 0; k < j; ++k) t -= a[(size_t)i * n + k] * a[(size_t)j * n + k];
            a[(size_t)i * n + j] = t / ljj;
        }
        for (int i = 0; i < j; ++i) a[(size_t)i * n + j] = 0.0;
    }
    return true;
}

void cholesky_solve(int n, const Mat& l, int q, std::vector<double>& b) {
    for (int c = 0; c < q; ++c) {
        for (int i = 0; i < n; ++i) {
            double s = b[(size_t)i * q + c];
            for (int k = 0; k < i; ++k) s -= l[(size_t)i * n + k] * b[(size_t)k * q + c];
            b[(size_t)i * q + c] = s / l[(size_t)i * n + i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = b[(size_t)i * q + c];
            for (int k = i + 1; k < n; ++k) s -= l[(size_t)k * n + i] * b[(size_t)k * q + c];
            b[(size_t)i * q + c] = s / l[(size_t)i * n + i];
        }
    }
}

bool lu_solve(int n, Mat a, std::vector<double>& b) {
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

bool diis_coefficients(int m, const Mat& gram, std::vector<double>& c) {
    const int n = m + 1;
    Mat b((size_t)n * n, 0.0);
    for (int i = 0; i < m; ++i)
        for (int j = 0; j < m; ++j) b[(size_t)i * n + j] = gram[(size_t)i * m + j];
    double scale = 0.0;
    for (int i = 0; i < m; ++i) scale = std::fmax(scale, b[(size_t)i * n + i]);
    if (!(scale > 0.0)) return false;
    for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) b[(size_t)i * n + j] /= scale;
        b[(size_t)i * n + i] += 1e-12;
    }
    for (int i = 0; i < m; ++i) { b[(size_t)i * n + m] = 1.0; b[(size_t)m * n + i] = 1.0; }
    std::vector<double> rhs(n, 0.0);
    rhs[m] = 1.0;
    if (!lu_solve(n, b, rhs)) return false;
    c.assign(rhs.begin(), rhs.begin() + m);
    for (double x : c)
        if (!std::isfinite(x)) return false;
    return true;
}


namespace {
// f at x = (e - mu)/kT, never forming e^|x| > 1
double fd_occupation(double x) {
    if (x >= 0.0) {
        const double e = std::exp(-x);
        return e / (1.0 + e);
    }
    return 1.0 / (1.0 + std::exp(x));
}
// s(x) = ln(1 + e^-|x|) + |x| / (1 + e^|x|) = -[f ln f + (1 - f) ln(1 - f)], with the 0 ln 0 limits built in
double fd_entropy(double x) {
    const double a = std::fabs(x);
    if (std::isinf(a)) return 0.0;
    return std::log1p(std::exp(-a)) + a / (1.0 + std::exp(a));
}
double compensated(int k, const double* ev, double mu, double kt, bool entropy) {
    double sum = 0.0, c = 0.0;
    for (int i = 0; i < k; ++i) {
        const double x = entropy ? fd_entropy((ev[i] - mu) / kt) : fd_occupation((ev[i] - mu) / kt);
        const double t = sum + x;
        c += std::fabs(sum) >= std::fabs(x) ? (sum - t) + x : (x - t) + sum;
        sum = t;
    }
    return sum + c;
}
double fd_bisect(const double* ev, int k, double n, double kt, double lo, double hi, bool ge) {
    for (int h = 0; h < 2048; ++h) {
        const double mid = 0.5 * lo + 0.5 * hi;
        if (mid <= lo || mid >= hi) break;
        const double d = compensated(k, ev, mid, kt, false) - n;
        if (ge ? d >= 0.0 : d > 0.0) hi = mid;
        else lo = mid;
    }
    return ge ? hi : lo;
}
}  // namespace

bool fermi_dirac(const double* ev, int k, int n, double kt, double* f, double& mu, double& entropy) {
    if (n == 0) {
        for (int i = 0; i < k; ++i) f[i] = 0.0;
        mu = NAN;
        entropy = 0.0;
        return true;
    }
    if (k < n + 1 || !(std::isfinite(kt) && kt > 0.0)) return false;
    double lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < k; ++i) {
        if (!std::isfinite(ev[i])) return false;
        lo = std::fmin(lo, ev[i]);
        hi = std::fmax(hi, ev[i]);
    }
    lo -= 50.0 * kt;
    hi += 50.0 * kt;
    const double nf = (double)n;
    if (!(std::isfinite(lo) && std::isfinite(hi) && compensated(k, ev, lo, kt, false) < nf && compensated(k, ev, hi, kt, false) > nf))
        return false;
    mu = 0.5 * fd_bisect(ev, k, nf, kt, lo, hi, true) + 0.5 * fd_bisect(ev, k, nf, kt, lo, hi, false);
    for (int i = 0; i < k; ++i) f[i] = fd_occupation((ev[i] - mu) / kt);
    entropy = compensated(k, ev, mu, kt, true);
    return true;
}

// ranks of the levels, ascending (ties by index)
static std::vector<int> ascending(const double* ev, int k) {
    std::vector<int> o(k);
    for (int i = 0; i < k; ++i) o[i] = i;
    std::stable_sort(o.begin(), o.end(), [&](int a, int b) { return ev[a] < ev[b]; });
    return o;
}

double fd_step_tail_kt(int n_w, double delta_rho_prev) {
    if (!(std::isfinite(delta_rho_prev) && delta_rho_prev > 0.0)) return 36.0;
    const double x = std::log((double)std::max(n_w, 1) / (1e-3 * delta_rho_prev));
    return std::min(std::max(x, 6.0), 36.0);
}

bool fd_witness(const double* ev, const double* res, int k, int n, double mu, double kt, double tail_kt) {
    if (n == 0) return true;
    if (k <= n) return false;
    const std::vector<int> o = ascending(ev, k);
    const int top = o[k - 1];
    const double lower = ev[top] - (res ? res[top] : 0.0);
    return lower >= ev[o[n - 1]] + 0.1 && lower - mu >= tail_kt * kt;
}

int fd_witness_keep_within(const double* ev, const double* res, int k, int n, double mu, double kt, double tail_kt, double r_max) {
    if (n == 0) return k;
    if (k <= n) return -1;
    const std::vector<int> o = ascending(ev, k);
    const double eps_n = ev[o[n - 1]];
    auto passes = [&](int r) {
        const double lower = ev[o[r]] - (res ? res[o[r]] : 0.0);
        return lower >= eps_n + 0.1 && lower - mu >= tail_kt * kt;
    };
    for (int t = n; t < k; ++t)
        if (passes(t) && (res ? res[o[t]] : 0.0) <= r_max) return (t + 1 < k && passes(t + 1)) ? t + 2 : t + 1;
    return -1;
}

int fd_tight_columns(const double* ev, const double* res, int k, double mu, double kt, double tol) {
    if (!std::isfinite(mu) || k <= 0) return 0;
    const std::vector<int> o = ascending(ev, k);
    const double limit = 1e-2 * tol;  // LOOSE_F_FACTOR x tol
    // from the top rank down: the loose ranks are those whose running tail sum of f(theta - r) stays below the limit
    double tail = 0.0;
    int loose_from = k;
    for (int r = k - 1; r >= 0; --r) {
        tail += fd_occupation((ev[o[r]] - (res ? res[o[r]] : 0.0) - mu) / kt);
        if (!(tail < limit)) break;
        loose_from = r;
    }
    int t = 0;
    for (int r = 0; r < loose_from; ++r) t = std::max(t, o[r] + 1);
    return t;
}

int fd_tight_start(const double* f, int k, int n, double tol) {
    if (!f) return n;
    const double limit = 1e-2 * tol;
    double tail = 0.0;
    int loose_from = k;
    for (int i = k - 1; i >= 0; --i) {
        tail += f[i];
        if (!(tail < limit)) break;
        loose_from = i;
    }
    return std::max(loose_from, n);
}

int fd_witness_keep(const double* ev, const double* res, int k, int n, double mu, double kt, double tail_kt) {
    if (n == 0 || k <= n) return k;
    const std::vector<int> o = ascending(ev, k);
    const double eps_n = ev[o[n - 1]];
    auto passes = [&](int r) {
        const double lower = ev[o[r]] - (res ? res[o[r]] : 0.0);
        return lower >= eps_n + 0.1 && lower - mu >= tail_kt * kt;
    };
    for (int t = n; t < k; ++t)
        if (passes(t)) return (t + 1 < k && passes(t + 1)) ? t + 2 : t + 1;
    return k;
}

}  // namespace dense
}  // namespace ks
