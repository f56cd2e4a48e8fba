// Dense LDL^T for the normal equations (host C++, OpenMP).
//
// Blocked right-looking factorisation of the lower triangle (row-major):
// per block of kNb pivots, an up-looking factorisation of the diagonal
// block applies SparseCholesky's pivot rule (a pivot <= singular_tol becomes
// singular_tol, core/numerical/factorization.cpp:1299-1305), the panel below
// is solved against it, and the trailing lower triangle receives the rank-kNb
// update A_ij -= sum_p (L_ip D_p) L_jp in 4x4 register tiles.
#include <omp.h>

#include <algorithm>
#include <cstring>

#include "hn_lp.hpp"

namespace hn::lp {
namespace {
constexpr std::size_t kNb = 64;

// acc[r][c] = sum_p w[r][p] * lt[p][c]: 4 rows of W (stride nb) against 8
// columns of the transposed panel (stride ld) -- broadcast + 8-wide FMA.
inline void tile4x8(const double* w, std::size_t nb, const double* lt, std::size_t ld, double acc[4][8]) {
    double a0[8] = {0}, a1[8] = {0}, a2[8] = {0}, a3[8] = {0};
    for (std::size_t p = 0; p < nb; ++p) {
        const double x0 = w[p], x1 = w[nb + p], x2 = w[2 * nb + p], x3 = w[3 * nb + p];
        const double* l = lt + p * ld;
#pragma omp simd
        for (int c = 0; c < 8; ++c) {
            a0[c] += x0 * l[c];
            a1[c] += x1 * l[c];
            a2[c] += x2 * l[c];
            a3[c] += x3 * l[c];
        }
    }
    for (int c = 0; c < 8; ++c) {
        acc[0][c] = a0[c];
        acc[1][c] = a1[c];
        acc[2][c] = a2[c];
        acc[3][c] = a3[c];
    }
}

inline double dotn(const double* a, const double* b, std::size_t n) {
    double s = 0.0;
#pragma omp simd reduction(+ : s)
    for (std::size_t p = 0; p < n; ++p) s += a[p] * b[p];
    return s;
}
}  // namespace

bool DenseLDLT::factorize(std::vector<double>& a, std::size_t m, double tol) {
    m_ = m;
    D_.assign(m, 0.0);
    singular_ = false;
    std::vector<double> P, W;  // packed panel L (rows k1..m) and L*D, padded to a multiple of 4 rows
    for (std::size_t k0 = 0; k0 < m; k0 += kNb) {
        const std::size_t k1 = std::min(m, k0 + kNb), nb = k1 - k0;
        // 1. diagonal block, row by row
        for (std::size_t j = k0; j < k1; ++j) {
            double* aj = &a[j * m];
            for (std::size_t p = k0; p < j; ++p) {
                const double* ap = &a[p * m];
                double s = aj[p];
                for (std::size_t q = k0; q < p; ++q) s -= (aj[q] * ap[q]) * D_[q];
                aj[p] = s / D_[p];
            }
            double d = aj[j];
            for (std::size_t q = k0; q < j; ++q) d -= (aj[q] * aj[q]) * D_[q];
            if (d <= tol) {
                d = tol;
                singular_ = true;
            }
            D_[j] = d;
        }
        if (k1 >= m) break;
        // 2. panel below the block; packed as W = L D (rows x nb) and P^T (nb x rows)
        const std::size_t rows = m - k1;
        const std::size_t rows4 = (rows + 3) & ~std::size_t(3), ld = (rows + 7) & ~std::size_t(7);
        W.assign(rows4 * nb, 0.0);
        P.assign(nb * ld, 0.0);
#pragma omp parallel for schedule(static)
        for (std::size_t i = k1; i < m; ++i) {
            double* ai = &a[i * m];
            for (std::size_t p = k0; p < k1; ++p) {
                const double* ap = &a[p * m];
                double s = ai[p];
                for (std::size_t q = k0; q < p; ++q) s -= (ai[q] * ap[q]) * D_[q];
                ai[p] = s / D_[p];
            }
            double* Wi = &W[(i - k1) * nb];
            for (std::size_t p = 0; p < nb; ++p) {
                Wi[p] = ai[k0 + p] * D_[k0 + p];
                P[p * ld + (i - k1)] = ai[k0 + p];
            }
        }
        // 3. trailing lower triangle in 4 x 8 tiles
        const std::size_t tiles = rows4 / 4;
#pragma omp parallel for schedule(dynamic, 1)
        for (std::size_t ti = 0; ti < tiles; ++ti) {
            const std::size_t i0 = ti * 4;
            double acc[4][8];
            for (std::size_t j0 = 0; j0 <= i0 + 3 && j0 < rows; j0 += 8) {
                tile4x8(&W[i0 * nb], nb, &P[j0], ld, acc);
                for (std::size_t r = 0; r < 4; ++r) {
                    const std::size_t i = k1 + i0 + r;
                    if (i >= m) break;
                    double* ai = &a[i * m];
                    const std::size_t cmax = std::min<std::size_t>(8, i - (k1 + j0) + 1);
                    for (std::size_t c = 0; c < cmax; ++c) ai[k1 + j0 + c] -= acc[r][c];
                }
            }
        }
    }
    L_.swap(a);
    return !singular_;
}

void DenseLDLT::solve(std::vector<double>& x) const {
    const std::size_t m = m_;
    for (std::size_t i = 0; i < m; ++i) x[i] -= dotn(&L_[i * m], x.data(), i);  // L y = b
    for (std::size_t i = 0; i < m; ++i) x[i] /= D_[i];
    for (std::size_t i = m; i-- > 0;) {  // L^T x = y (column sweep)
        const double xi = x[i];
        const double* li = &L_[i * m];
        for (std::size_t j = 0; j < i; ++j) x[j] -= li[j] * xi;
    }
}

}  // namespace hn::lp
