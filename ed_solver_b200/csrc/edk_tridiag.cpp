// Host eigen-solvers for the small matrices of the Krylov drivers.
//
// The reference calls LAPACK DSTEDC on the Lanczos tridiagonal after every
// iteration (matrices_tridiag.f90:210-259) and DSYEV for tiny sectors
// (ED_ARPACK.f90:590-715).  Only the lowest few eigenpairs are needed, so the
// tridiagonal solver here is Sturm-sequence bisection (lowest m eigenvalues)
// plus inverse iteration for their vectors; the dense solver is cyclic Jacobi.
#include "edk_tridiag.h"

#include <algorithm>
#include <cmath>
#include <limits>

namespace edk {

namespace {

// number of eigenvalues of T strictly below x (LDL^T inertia count)
int sturm_count(int n, const double *d, const double *e, double x, double pivmin)
{
    int cnt = 0;
    double q = d[0] - x;
    if (std::fabs(q) < pivmin) q = -pivmin;
    if (q < 0) ++cnt;
    for (int i = 1; i < n; ++i) {
        q = d[i] - x - (e[i - 1] * e[i - 1]) / q;
        if (std::fabs(q) < pivmin) q = -pivmin;
        if (q < 0) ++cnt;
    }
    return cnt;
}

}  // namespace

void tridiag_lowest(int n, const double *d, const double *e, int m, double *w)
{
    if (n <= 0 || m <= 0) return;
    if (m > n) m = n;
    double lo = d[0], hi = d[0], emax = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? std::fabs(e[i - 1]) : 0.0) + (i < n - 1 ? std::fabs(e[i]) : 0.0);
        lo = std::min(lo, d[i] - r);
        hi = std::max(hi, d[i] + r);
        if (i < n - 1) emax = std::max(emax, std::fabs(e[i]));
    }
    const double scale = std::max(std::fabs(lo), std::fabs(hi));
    const double pivmin = std::max(std::numeric_limits<double>::min(),
                                   std::numeric_limits<double>::min() * emax * emax) * 4.0;
    const double eps = std::numeric_limits<double>::epsilon();
    lo -= 2.0 * eps * scale + pivmin;
    hi += 2.0 * eps * scale + pivmin;
    for (int k = 0; k < m; ++k) {
        // k-th eigenvalue (0-based): smallest x with count(x) > k
        double a = (k > 0) ? w[k - 1] - 2.0 * eps * scale : lo, b = hi;
        if (a < lo) a = lo;
        for (int it = 0; it < 200; ++it) {
            const double mid = 0.5 * (a + b);
            if (b - a <= 2.0 * eps * std::max(std::fabs(a), std::fabs(b)) + pivmin) break;
            if (mid <= a || mid >= b) break;
            if (sturm_count(n, d, e, mid, pivmin) > k) b = mid; else a = mid;
        }
        w[k] = 0.5 * (a + b);
    }
}

void tridiag_vector(int n, const double *d, const double *e, double lambda, const double *prev,
                    int nprev, double *v)
{
    // inverse iteration with a slightly perturbed shift, partial pivoting
    double scale = 0.0;
    for (int i = 0; i < n; ++i) scale = std::max(scale, std::fabs(d[i]) + (i < n - 1 ? std::fabs(e[i]) : 0.0));
    if (scale == 0.0) scale = 1.0;
    const double shift = lambda + 4.0 * std::numeric_limits<double>::epsilon() * scale;
    std::vector<double> a(n), b(n), c(n), u2(n), rhs(n);
    std::vector<int> piv(n);
    for (int i = 0; i < n; ++i) v[i] = 1.0 / std::sqrt((double)n) * (1.0 + 0.01 * ((i * 7919) % 13) / 13.0);
    for (int iter = 0; iter < 4; ++iter) {
        // factor T - shift*I (tridiagonal LU with row interchanges)
        for (int i = 0; i < n; ++i) {
            a[i] = (i > 0) ? e[i - 1] : 0.0;   // sub
            b[i] = d[i] - shift;               // diag
            c[i] = (i < n - 1) ? e[i] : 0.0;   // super
            u2[i] = 0.0;
            rhs[i] = v[i];
        }
        for (int i = 0; i < n - 1; ++i) {
            if (std::fabs(a[i + 1]) > std::fabs(b[i])) {
                // swap rows i and i+1
                std::swap(b[i], a[i + 1]);
                std::swap(c[i], b[i + 1]);
                std::swap(u2[i], c[i + 1]);
                std::swap(rhs[i], rhs[i + 1]);
            }
            if (b[i] == 0.0) b[i] = std::numeric_limits<double>::epsilon() * scale;
            const double f = a[i + 1] / b[i];
            b[i + 1] -= f * c[i];
            c[i + 1] -= f * u2[i];
            rhs[i + 1] -= f * rhs[i];
        }
        if (b[n - 1] == 0.0) b[n - 1] = std::numeric_limits<double>::epsilon() * scale;
        // back substitution
        for (int i = n - 1; i >= 0; --i) {
            double s = rhs[i];
            if (i + 1 < n) s -= c[i] * v[i + 1];
            if (i + 2 < n) s -= u2[i] * v[i + 2];
            v[i] = s / b[i];
        }
        // orthogonalise against earlier vectors of (near) equal eigenvalues
        for (int p = 0; p < nprev; ++p) {
            double dot = 0.0;
            for (int i = 0; i < n; ++i) dot += prev[(size_t)p * n + i] * v[i];
            for (int i = 0; i < n; ++i) v[i] -= dot * prev[(size_t)p * n + i];
        }
        double nrm = 0.0;
        for (int i = 0; i < n; ++i) nrm += v[i] * v[i];
        nrm = std::sqrt(nrm);
        if (nrm == 0.0) { v[0] = 1.0; nrm = 1.0; }
        for (int i = 0; i < n; ++i) v[i] /= nrm;
    }
    // fix the sign: largest component positive (DSTEDC has no fixed sign either)
    int imax = 0;
    for (int i = 1; i < n; ++i) if (std::fabs(v[i]) > std::fabs(v[imax])) imax = i;
    if (v[imax] < 0) for (int i = 0; i < n; ++i) v[i] = -v[i];
}

void dense_eigh(int n, std::vector<double> A, std::vector<double> &w, std::vector<double> &V)
{
    // cyclic Jacobi on a symmetric n x n matrix (row-major); V columns = eigenvectors
    V.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) V[(size_t)i * n + i] = 1.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j) off += A[(size_t)i * n + j] * A[(size_t)i * n + j];
        if (off < 1e-30) break;
        for (int p = 0; p < n; ++p)
            for (int q = p + 1; q < n; ++q) {
                const double apq = A[(size_t)p * n + q];
                if (apq == 0.0) continue;
                const double app = A[(size_t)p * n + p], aqq = A[(size_t)q * n + q];
                const double theta = (aqq - app) / (2.0 * apq);
                const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                const double cth = 1.0 / std::sqrt(t * t + 1.0), sth = t * cth;
                for (int k = 0; k < n; ++k) {
                    const double akp = A[(size_t)k * n + p], akq = A[(size_t)k * n + q];
                    A[(size_t)k * n + p] = cth * akp - sth * akq;
                    A[(size_t)k * n + q] = sth * akp + cth * akq;
                }
                for (int k = 0; k < n; ++k) {
                    const double apk = A[(size_t)p * n + k], aqk = A[(size_t)q * n + k];
                    A[(size_t)p * n + k] = cth * apk - sth * aqk;
                    A[(size_t)q * n + k] = sth * apk + cth * aqk;
                }
                for (int k = 0; k < n; ++k) {
                    const double vkp = V[(size_t)k * n + p], vkq = V[(size_t)k * n + q];
                    V[(size_t)k * n + p] = cth * vkp - sth * vkq;
                    V[(size_t)k * n + q] = sth * vkp + cth * vkq;
                }
            }
    }
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](int a, int b) { return A[(size_t)a * n + a] < A[(size_t)b * n + b]; });
    w.resize(n);
    std::vector<double> V2((size_t)n * n);
    for (int j = 0; j < n; ++j) {
        w[j] = A[(size_t)idx[j] * n + idx[j]];
        for (int k = 0; k < n; ++k) V2[(size_t)k * n + j] = V[(size_t)k * n + idx[j]];
    }
    V.swap(V2);
}

void dense_lowest(int n, std::vector<double> A, int m, std::vector<double> &w, std::vector<double> &V)
{
    // A = Q T Q^T with Q = H_0 H_1 ... H_{n-3}, H_k = 1 - 2 v_k v_k^T acting on indices k+1..n-1
    std::vector<std::vector<double>> refl(n > 2 ? n - 2 : 0);
    std::vector<double> p(n), q(n);
    auto a = [&](int i, int j) -> double & { return A[(size_t)i * n + j]; };
    for (int k = 0; k + 2 < n; ++k) {
        const int len = n - k - 1;
        double nrm = 0.0;
        for (int i = 0; i < len; ++i) nrm += a(k + 1 + i, k) * a(k + 1 + i, k);
        nrm = std::sqrt(nrm);
        std::vector<double> &v = refl[k];
        v.assign(len, 0.0);
        if (nrm == 0.0) continue;
        const double x0 = a(k + 1, k);
        const double alpha = x0 >= 0 ? -nrm : nrm;
        for (int i = 0; i < len; ++i) v[i] = a(k + 1 + i, k);
        v[0] -= alpha;
        double vn = 0.0;
        for (int i = 0; i < len; ++i) vn += v[i] * v[i];
        vn = std::sqrt(vn);
        if (vn == 0.0) { v.assign(len, 0.0); continue; }
        for (int i = 0; i < len; ++i) v[i] /= vn;
        // trailing block: A22 <- A22 - v q^T - q v^T, q = 2 (A22 v) - 2 (v^T A22 v) v
        double c = 0.0;
        for (int i = 0; i < len; ++i) {
            double t = 0.0;
            for (int j = 0; j < len; ++j) t += a(k + 1 + i, k + 1 + j) * v[j];
            p[i] = t;
            c += v[i] * t;
        }
        for (int i = 0; i < len; ++i) q[i] = 2.0 * p[i] - 2.0 * c * v[i];
        for (int i = 0; i < len; ++i)
            for (int j = 0; j < len; ++j) a(k + 1 + i, k + 1 + j) -= v[i] * q[j] + q[i] * v[j];
        a(k + 1, k) = a(k, k + 1) = alpha;
        for (int i = 1; i < len; ++i) a(k + 1 + i, k) = a(k, k + 1 + i) = 0.0;
    }
    std::vector<double> d(n), e(n > 1 ? n - 1 : 1);
    for (int i = 0; i < n; ++i) d[i] = a(i, i);
    for (int i = 0; i + 1 < n; ++i) e[i] = a(i + 1, i);
    m = std::min(m, n);
    w.assign(m, 0.0);
    tridiag_lowest(n, d.data(), e.data(), m, w.data());
    V.assign((size_t)n * m, 0.0);
    std::vector<double> prev((size_t)n * m), y(n);
    for (int j = 0; j < m; ++j) {
        tridiag_vector(n, d.data(), e.data(), w[j], prev.data(), j, y.data());
        std::copy(y.begin(), y.end(), prev.begin() + (size_t)j * n);
        for (int k = n - 3; k >= 0; --k) {
            const std::vector<double> &v = refl[k];
            if (v.empty()) continue;
            double t = 0.0;
            for (size_t i = 0; i < v.size(); ++i) t += v[i] * y[k + 1 + i];
            for (size_t i = 0; i < v.size(); ++i) y[k + 1 + i] -= 2.0 * t * v[i];
        }
        for (int i = 0; i < n; ++i) V[(size_t)i * m + j] = y[i];
    }
}

}  // namespace edk
