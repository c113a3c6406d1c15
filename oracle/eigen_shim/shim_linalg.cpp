// Dense kernels behind the oracle's Eigen-API shim: blocked LU with partial pivoting,
// column-major GEMV and BiCGSTAB.  OpenMP-parallel so the reference's CPU timing is not
// dominated by a naive solver.  Test infrastructure only.
#include "Eigen/Dense"
#include "Eigen/IterativeLinearSolvers"

#include <cmath>
#include <cstring>
#include <vector>

namespace Eigen {
namespace shim_detail {

// y = A x, A column-major rows x cols.  Row blocks in parallel; inside a block the
// columns are accumulated in order, so y_i = sum_j A(i,j) x_j left to right.
void gemv_colmajor(Index rows, Index cols, const double* a, const double* x, double* y) {
    const Index RB = 256;
#pragma omp parallel for schedule(static)
    for (Index r0 = 0; r0 < rows; r0 += RB) {
        Index r1 = std::min(rows, r0 + RB);
        double acc[256];
        for (Index i = r0; i < r1; ++i) acc[i - r0] = 0.0;
        for (Index j = 0; j < cols; ++j) {
            const double xj = x[j];
            const double* col = a + j * rows;
            for (Index i = r0; i < r1; ++i) acc[i - r0] += col[i] * xj;
        }
        for (Index i = r0; i < r1; ++i) y[i] = acc[i - r0];
    }
}

// Right-looking blocked LU, panel width NB, partial pivoting by rows.
// perm[i] = original row index of row i of P*A.
void lu_partial_pivot(Index n, double* a, Index* perm) {
    const Index NB = 64;
    for (Index i = 0; i < n; ++i) perm[i] = i;
    auto A = [&](Index i, Index j) -> double& { return a[i + j * n]; };
    for (Index k0 = 0; k0 < n; k0 += NB) {
        const Index k1 = std::min(n, k0 + NB);
        // unblocked panel factorisation of columns k0..k1-1 (rows k0..n-1),
        // swapping whole rows so that the left factor and right block stay consistent
        for (Index k = k0; k < k1; ++k) {
            Index p = k;
            double best = std::abs(A(k, k));
            for (Index i = k + 1; i < n; ++i) {
                double v = std::abs(A(i, k));
                if (v > best) { best = v; p = i; }
            }
            if (p != k) {
                for (Index j = 0; j < n; ++j) std::swap(A(k, j), A(p, j));
                std::swap(perm[k], perm[p]);
            }
            const double piv = A(k, k);
            if (piv != 0.0)
                for (Index i = k + 1; i < n; ++i) A(i, k) /= piv;
            for (Index j = k + 1; j < k1; ++j) {
                const double ukj = A(k, j);
                for (Index i = k + 1; i < n; ++i) A(i, j) -= A(i, k) * ukj;
            }
        }
        if (k1 >= n) break;
        // U12 = L11^{-1} A12
#pragma omp parallel for schedule(static)
        for (Index j = k1; j < n; ++j)
            for (Index k = k0; k < k1; ++k) {
                const double ukj = A(k, j);
                for (Index i = k + 1; i < k1; ++i) A(i, j) -= A(i, k) * ukj;
            }
        // A22 -= L21 U12
#pragma omp parallel for schedule(dynamic, 8)
        for (Index j = k1; j < n; ++j)
            for (Index k = k0; k < k1; ++k) {
                const double ukj = A(k, j);
                if (ukj == 0.0) continue;
                const double* lk = &A(0, k);
                double* aj = &A(0, j);
                for (Index i = k1; i < n; ++i) aj[i] -= lk[i] * ukj;
            }
    }
}

static double dotv(Index n, const double* u, const double* v) {
    double s = 0.0;
    for (Index i = 0; i < n; ++i) s += u[i] * v[i];
    return s;
}

long long g_bicgstab_solves = 0;
long long g_bicgstab_iters = 0;

void bicgstab_dense(Index n, const double* a, const double* b, double* x, Index max_iters,
                    double tol, Index* iters_out, double* err_out) {
    ++g_bicgstab_solves;
    std::vector<double> r(n), r0(n), p(n, 0.0), v(n, 0.0), y(n), z(n), s(n), t(n), invd(n);
    for (Index i = 0; i < n; ++i) {
        double d = a[i + i * n];
        invd[i] = (d != 0.0) ? 1.0 / d : 1.0;
        x[i] = 0.0;
    }
    const double rhs2 = dotv(n, b, b);
    if (rhs2 == 0.0) {
        *iters_out = 0;
        *err_out = 0.0;
        return;
    }
    // r = b - A*0 = b
    for (Index i = 0; i < n; ++i) r[i] = b[i];
    r0 = r;
    double r0_sq = dotv(n, r0.data(), r0.data());
    double rho = 1.0, alpha = 1.0, w = 1.0;
    const double tol2 = tol * tol * rhs2;
    const double eps = std::numeric_limits<double>::epsilon();
    const double eps2 = eps * eps;
    Index it = 0, restarts = 0;
    while (dotv(n, r.data(), r.data()) > tol2 && it < max_iters) {
        double rho_old = rho;
        rho = dotv(n, r0.data(), r.data());
        if (std::abs(rho) < eps2 * r0_sq) {
            // shadow residual became (numerically) orthogonal: restart from the true residual
            gemv_colmajor(n, n, a, x, t.data());
            for (Index i = 0; i < n; ++i) r[i] = b[i] - t[i];
            r0 = r;
            rho = r0_sq = dotv(n, r.data(), r.data());
            if (restarts++ == 0) it = 0;
        }
        const double beta = (rho / rho_old) * (alpha / w);
        for (Index i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - w * v[i]);
        for (Index i = 0; i < n; ++i) y[i] = invd[i] * p[i];
        gemv_colmajor(n, n, a, y.data(), v.data());
        alpha = rho / dotv(n, r0.data(), v.data());
        for (Index i = 0; i < n; ++i) s[i] = r[i] - alpha * v[i];
        for (Index i = 0; i < n; ++i) z[i] = invd[i] * s[i];
        gemv_colmajor(n, n, a, z.data(), t.data());
        const double tt = dotv(n, t.data(), t.data());
        w = (tt > 0.0) ? dotv(n, t.data(), s.data()) / tt : 0.0;
        for (Index i = 0; i < n; ++i) x[i] += alpha * y[i] + w * z[i];
        for (Index i = 0; i < n; ++i) r[i] = s[i] - w * t[i];
        ++it;
    }
    *iters_out = it;
    g_bicgstab_iters += it;
    *err_out = std::sqrt(dotv(n, r.data(), r.data()) / rhs2);
}

}  // namespace shim_detail
}  // namespace Eigen
