#include "eigh.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>

namespace dftb {

bool eigh(int n, std::vector<double>& a, std::vector<double>& w, std::vector<double>& z) {
    w.assign(n, 0.0);
    z.assign((size_t)n * n, 0.0);
    if (n == 0) return true;
    if (n == 1) {
        w[0] = a[0];
        z[0] = 1.0;
        return true;
    }
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    std::vector<double> d(n), e(n);

    // --- Householder reduction to tridiagonal form (rows from the bottom up) ---------
    for (int i = n - 1; i > 0; --i) {
        const int l = i - 1;
        double h = 0.0;
        if (l > 0) {
            double scale = 0.0;
            for (int k = 0; k <= l; ++k) scale += std::fabs(A(i, k));
            if (scale == 0.0) {
                e[i] = A(i, l);
            } else {
                for (int k = 0; k <= l; ++k) {
                    A(i, k) /= scale;
                    h += A(i, k) * A(i, k);
                }
                double f = A(i, l);
                double g = f >= 0.0 ? -std::sqrt(h) : std::sqrt(h);
                e[i] = scale * g;
                h -= f * g;
                A(i, l) = f - g;
                f = 0.0;
                for (int j = 0; j <= l; ++j) {
                    A(j, i) = A(i, j) / h;
                    g = 0.0;
                    for (int k = 0; k <= j; ++k) g += A(j, k) * A(i, k);
                    for (int k = j + 1; k <= l; ++k) g += A(k, j) * A(i, k);
                    e[j] = g / h;
                    f += e[j] * A(i, j);
                }
                const double hh = f / (h + h);
                for (int j = 0; j <= l; ++j) {
                    f = A(i, j);
                    g = e[j] - hh * f;
                    e[j] = g;
                    for (int k = 0; k <= j; ++k) A(j, k) -= f * e[k] + g * A(i, k);
                }
            }
        } else {
            e[i] = A(i, l);
        }
        d[i] = h;
    }
    d[0] = 0.0;
    e[0] = 0.0;
    // accumulate the transformations
    for (int i = 0; i < n; ++i) {
        const int l = i - 1;
        if (d[i] != 0.0) {
            for (int j = 0; j <= l; ++j) {
                double g = 0.0;
                for (int k = 0; k <= l; ++k) g += A(i, k) * A(k, j);
                for (int k = 0; k <= l; ++k) A(k, j) -= g * A(k, i);
            }
        }
        d[i] = A(i, i);
        A(i, i) = 1.0;
        for (int j = 0; j <= l; ++j) A(j, i) = A(i, j) = 0.0;
    }

    // --- implicit QL on the tridiagonal (d, e), rotations applied to the columns of A --
    for (int i = 1; i < n; ++i) e[i - 1] = e[i];
    e[n - 1] = 0.0;
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        int iter = 0;
        int m;
        do {
            for (m = l; m < n - 1; ++m) {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m != l) {
                if (iter++ == 200) return false;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::hypot(g, 1.0);
                g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
                double s = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; --i) {
                    double f = s * e[i];
                    const double b = c * e[i];
                    r = std::hypot(f, g);
                    e[i + 1] = r;
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    for (int k = 0; k < n; ++k) {
                        f = A(k, i + 1);
                        A(k, i + 1) = s * A(k, i) + c * f;
                        A(k, i) = c * A(k, i) - s * f;
                    }
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }

    // --- sort ascending ------------------------------------------------------------------
    std::vector<int> order(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return d[x] < d[y]; });
    for (int j = 0; j < n; ++j) {
        w[j] = d[order[j]];
        for (int i = 0; i < n; ++i) z[(size_t)i * n + j] = A(i, order[j]);
    }
    return true;
}

}  // namespace dftb

namespace dftb {

namespace {

// eigenvalues of the symmetric tridiagonal (d, e), e[i] couples i and i+1; ascending in d
bool tridiag_eigenvalues(int n, std::vector<double> d, std::vector<double> e, std::vector<double>& out) {
    e.resize(n, 0.0);
    e[n - 1] = 0.0;
    const double eps = std::numeric_limits<double>::epsilon();
    for (int l = 0; l < n; ++l) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; ++m) {
                const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
                if (std::fabs(e[m]) <= eps * dd) break;
            }
            if (m != l) {
                if (iter++ == 200) return false;
                double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
                double r = std::sqrt(g * g + 1.0);
                g = d[m] - d[l] + e[l] / (g + std::copysign(r, g));
                double s = 1.0, c = 1.0, p = 0.0;
                int i;
                for (i = m - 1; i >= l; --i) {
                    const double f = s * e[i], b = c * e[i];
                    r = std::sqrt(f * f + g * g);
                    e[i + 1] = r;
                    if (r == 0.0) {
                        d[i + 1] -= p;
                        e[m] = 0.0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2.0 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                }
                if (r == 0.0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0.0;
            }
        } while (m != l);
    }
    std::sort(d.begin(), d.end());
    out.swap(d);
    return true;
}

// LU factorisation of T - lam I with partial pivoting (tridiagonal: the factor has at most two
// super-diagonals; row i of U holds u0, u1, u2 at columns i, i+1, i+2); pivots smaller than tol
// in magnitude are replaced by tol
struct TriLU {
    std::vector<double> u0, u1, u2, l;
    std::vector<int> piv;
    void factor(int n, const std::vector<double>& d, const std::vector<double>& e, double lam, double tol) {
        u0.resize(n), u1.resize(n), u2.resize(n), l.resize(n), piv.resize(n);
        double a0 = d[0] - lam, a1 = n > 1 ? e[0] : 0.0;
        for (int i = 0; i < n - 1; ++i) {
            const double b0 = e[i], b1 = d[i + 1] - lam, b2 = i + 1 < n - 1 ? e[i + 1] : 0.0;
            if (std::fabs(a0) >= std::fabs(b0)) {
                piv[i] = 0;
                const double m = a0 != 0.0 ? b0 / a0 : 0.0;
                l[i] = m;
                u0[i] = a0, u1[i] = a1, u2[i] = 0.0;
                a0 = b1 - m * a1;
                a1 = b2;
            } else {
                piv[i] = 1;
                const double m = a0 / b0;
                l[i] = m;
                u0[i] = b0, u1[i] = b1, u2[i] = b2;
                a0 = a1 - m * b1;
                a1 = -m * b2;
            }
            if (std::fabs(u0[i]) < tol) u0[i] = std::copysign(tol, u0[i] == 0.0 ? 1.0 : u0[i]);
        }
        u0[n - 1] = std::fabs(a0) < tol ? std::copysign(tol, a0 == 0.0 ? 1.0 : a0) : a0;
    }
    // x <- (T - lam I)^-1 x
    void solve(int n, double* x) const {
        for (int i = 0; i < n - 1; ++i) {
            if (piv[i]) std::swap(x[i], x[i + 1]);
            x[i + 1] -= l[i] * x[i];
        }
        for (int i = n - 1; i >= 0; --i) {
            double v = x[i];
            if (i + 1 < n) v -= u1[i] * x[i + 1];
            if (i + 2 < n) v -= u2[i] * x[i + 2];
            x[i] = v / u0[i];
        }
    }
};

}  // namespace

bool eigh_lowest(int n, std::vector<double>& a, int m, std::vector<double>& w, std::vector<double>& z) {
    m = std::max(1, std::min(m, n));
    if (n <= 48 || 2 * m > n) {
        // small or most vectors wanted: the full solver, truncated
        std::vector<double> wf, zf;
        if (!eigh(n, a, wf, zf)) return false;
        w.assign(wf.begin(), wf.begin() + m);
        z.assign((size_t)n * m, 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < m; ++j) z[(size_t)i * m + j] = zf[(size_t)i * n + j];
        return true;
    }
    const std::vector<double> a0 = a;  // for the fallback
    // only the lower triangle is read and updated below: make it the average of both halves
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < i; ++j) a[(size_t)i * n + j] = 0.5 * (a[(size_t)i * n + j] + a[(size_t)j * n + i]);
    auto A = [&](int i, int j) -> double& { return a[(size_t)i * n + j]; };
    std::vector<double> d(n), e(n, 0.0), tau(n, 0.0), v(n), p(n);
    // ---- Householder: column i below the diagonal -> e[i], reflector I - tau v v^T on i+1..n-1
    for (int i = 0; i < n - 2; ++i) {
        const int r0 = i + 1, s = n - r0;
        double xnorm2 = 0.0;
        for (int r = r0 + 1; r < n; ++r) xnorm2 += A(r, i) * A(r, i);
        const double alpha = A(r0, i);
        if (xnorm2 == 0.0) {
            e[i] = alpha;
            tau[i] = 0.0;
            continue;
        }
        const double beta = -std::copysign(std::sqrt(alpha * alpha + xnorm2), alpha);
        const double t = (beta - alpha) / beta, sc = 1.0 / (alpha - beta);
        e[i] = beta;
        tau[i] = t;
        v[0] = 1.0;
        for (int r = r0 + 1; r < n; ++r) v[r - r0] = A(r, i) * sc;
        // p = t B v over the trailing block B = A[r0:, r0:], reading only its lower triangle:
        // row r contributes sum_{c<r} B[r][c] v[c] to p[r] and B[r][c] v[r] to p[c]
        double* __restrict__ pp = p.data();
        const double* __restrict__ vv = v.data();
        std::fill(p.begin(), p.begin() + s, 0.0);
        for (int r = 0; r < s; ++r) {
            const double* __restrict__ row = &A(r0 + r, r0);
            const double vr = vv[r];
            double acc = 0.0;
            for (int c = 0; c < r; ++c) {
                acc += row[c] * vv[c];
                pp[c] += row[c] * vr;
            }
            pp[r] += acc + row[r] * vr;
        }
        double pv = 0.0;
        for (int r = 0; r < s; ++r) {
            pp[r] *= t;
            pv += pp[r] * vv[r];
        }
        const double K = -0.5 * t * pv;
        for (int r = 0; r < s; ++r) pp[r] += K * vv[r];  // w = p - (t/2)(p.v) v
        // lower triangle of B -= v w^T + w v^T
        for (int r = 0; r < s; ++r) {
            double* __restrict__ row = &A(r0 + r, r0);
            const double vr = vv[r], wr = pp[r];
            for (int c = 0; c <= r; ++c) row[c] -= vr * pp[c] + wr * vv[c];
        }
        for (int r = r0 + 1; r < n; ++r) A(r, i) = v[r - r0];  // keep v (v[0] = 1 implicit)
    }
    for (int i = 0; i < n; ++i) d[i] = A(i, i);
    e[n - 2] = A(n - 1, n - 2);
    e[n - 1] = 0.0;
    // ---- eigenvalues of T, the lowest m
    std::vector<double> lam;
    bool ok = tridiag_eigenvalues(n, d, e, lam);
    double tnorm = 0.0;
    for (int i = 0; i < n; ++i)
        tnorm = std::max(tnorm, std::fabs(d[i]) + (i > 0 ? std::fabs(e[i - 1]) : 0.0) + std::fabs(e[i]));
    if (!(tnorm > 0.0)) tnorm = 1.0;
    const double eps = std::numeric_limits<double>::epsilon();
    const double ortol = 1e-3 * tnorm, pertol = 10.0 * eps * tnorm, pivtol = eps * tnorm;
    // ---- inverse iteration, vectors of close eigenvalues reorthogonalised (MGS)
    std::vector<double> Y((size_t)m * n);  // vector j at Y[j*n ..]
    std::vector<double> x(n);
    TriLU lu;
    int cluster = 0;
    double prev = 0.0;
    for (int j = 0; j < m && ok; ++j) {
        double lj = lam[j];
        if (j > 0 && lam[j] - lam[j - 1] > ortol) cluster = j;
        if (j > 0 && lj - prev < pertol) lj = prev + pertol;  // separate coincident shifts
        prev = lj;
        unsigned long long st = 0x9E3779B97F4A7C15ull * (unsigned long long)(j + 1);
        for (int i = 0; i < n; ++i) {  // deterministic pseudo-random start
            st ^= st << 13, st ^= st >> 7, st ^= st << 17;
            x[i] = (double)(st >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        }
        lu.factor(n, d, e, lj, pivtol);
        for (int itn = 0; itn < 3; ++itn) {
            for (int c = cluster; c < j; ++c) {
                const double* yc = &Y[(size_t)c * n];
                double dot = 0.0;
                for (int i = 0; i < n; ++i) dot += yc[i] * x[i];
                for (int i = 0; i < n; ++i) x[i] -= dot * yc[i];
            }
            double nrm = 0.0;
            for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
            nrm = std::sqrt(nrm);
            if (!(nrm > 0.0) || !std::isfinite(nrm)) {
                ok = false;
                break;
            }
            for (int i = 0; i < n; ++i) x[i] /= nrm;
            lu.solve(n, x.data());
        }
        if (!ok) break;
        for (int c = cluster; c < j; ++c) {
            const double* yc = &Y[(size_t)c * n];
            double dot = 0.0;
            for (int i = 0; i < n; ++i) dot += yc[i] * x[i];
            for (int i = 0; i < n; ++i) x[i] -= dot * yc[i];
        }
        double nrm = 0.0;
        for (int i = 0; i < n; ++i) nrm += x[i] * x[i];
        nrm = std::sqrt(nrm);
        if (!(nrm > 0.0) || !std::isfinite(nrm)) {
            ok = false;
            break;
        }
        double* yj = &Y[(size_t)j * n];
        for (int i = 0; i < n; ++i) yj[i] = x[i] / nrm;
        // residual of the tridiagonal pair (with the unperturbed eigenvalue)
        double res = 0.0;
        for (int i = 0; i < n; ++i) {
            double t = (d[i] - lam[j]) * yj[i];
            if (i > 0) t += e[i - 1] * yj[i - 1];
            if (i + 1 < n) t += e[i] * yj[i + 1];
            res = std::max(res, std::fabs(t));
        }
        if (!(res <= 1e-10 * tnorm)) ok = false;
    }
    // orthogonality within clusters
    for (int j = 1; j < m && ok; ++j)
        for (int c = j - 1; c >= 0 && lam[j] - lam[c] <= ortol; --c) {
            double dot = 0.0;
            for (int i = 0; i < n; ++i) dot += Y[(size_t)c * n + i] * Y[(size_t)j * n + i];
            if (std::fabs(dot) > 1e-10) {
                ok = false;
                break;
            }
        }
    if (!ok) {
        a = a0;
        std::vector<double> wf, zf;
        if (!eigh(n, a, wf, zf)) return false;
        w.assign(wf.begin(), wf.begin() + m);
        z.assign((size_t)n * m, 0.0);
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < m; ++j) z[(size_t)i * m + j] = zf[(size_t)i * n + j];
        return true;
    }
    // ---- back-transform: z = H_0 H_1 ... H_{n-3} y, rows of z contiguous over the m vectors
    z.assign((size_t)n * m, 0.0);
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < m; ++j) z[(size_t)i * m + j] = Y[(size_t)j * n + i];
    std::vector<double> sv(m);
    for (int i = n - 3; i >= 0; --i) {
        if (tau[i] == 0.0) continue;
        const int r0 = i + 1;
        std::fill(sv.begin(), sv.end(), 0.0);
        for (int r = r0; r < n; ++r) {
            const double vr = r == r0 ? 1.0 : A(r, i);
            const double* zr = &z[(size_t)r * m];
            for (int j = 0; j < m; ++j) sv[j] += vr * zr[j];
        }
        for (int j = 0; j < m; ++j) sv[j] *= tau[i];
        for (int r = r0; r < n; ++r) {
            const double vr = r == r0 ? 1.0 : A(r, i);
            double* zr = &z[(size_t)r * m];
            for (int j = 0; j < m; ++j) zr[j] -= vr * sv[j];
        }
    }
    w.assign(lam.begin(), lam.begin() + m);
    return true;
}

}  // namespace dftb
