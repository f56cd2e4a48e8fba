/* CPU restatement of the HyperNova sparse hot path -- TEST INFRASTRUCTURE ONLY.
 * See hn_oracle.h for the contract of each function and the reference lines
 * it follows. Built with -ffp-contract=off so no FMA changes the rounding the
 * reference's x86-64 build produces. */
#include "hn_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

void hno_csr_multiply(int64_t m, const int64_t* rp, const int64_t* ci, const double* val,
                      const double* x, double* y) {
    /* sparse_matrix.cpp:142-149 */
    for (int64_t i = 0; i < m; ++i) {
        double sum = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) sum += val[k] * x[ci[k]];
        y[i] = sum;
    }
}

void hno_csr_tmultiply(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                       const double* val, const double* x, double* y) {
    /* sparse_matrix.cpp:167-174 */
    for (int64_t j = 0; j < n; ++j) y[j] = 0.0;
    for (int64_t i = 0; i < m; ++i) {
        const double xi = x[i];
        if (xi == 0.0) continue;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) y[ci[k]] += val[k] * xi;
    }
}

void hno_matvec_t(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                  const double* val, const double* x, double* y) {
    /* interior_point.cpp:61-69 */
    for (int64_t j = 0; j < n; ++j) y[j] = 0.0;
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) y[ci[k]] += val[k] * x[i];
}

int64_t hno_csr_transposed(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                           const double* val, int64_t* rpT, int64_t* ciT, double* valT) {
    /* to_triplets enumerates CSR order (sparse_matrix.cpp:264-273); transpose()
     * swaps row/col (:84-90); from_triplets sorts by (row',col') (:19-24) and
     * sum_duplicates merges equal keys and drops zero sums (:240-254). A
     * counting sort by column over CSR order is that sort with ties kept in
     * input order. */
    const int64_t nnz = rp[m];
    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    int64_t* rows = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz ? nnz : 1));
    double* vals = (double*)malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
    for (int64_t k = 0; k < nnz; ++k) cnt[ci[k] + 1]++;
    for (int64_t j = 0; j < n; ++j) cnt[j + 1] += cnt[j];
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
    for (int64_t j = 0; j < n; ++j) cur[j] = cnt[j];
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int64_t p = cur[ci[k]]++;
            rows[p] = i;
            vals[p] = val[k];
        }
    int64_t w = 0;
    rpT[0] = 0;
    for (int64_t j = 0; j < n; ++j) {
        int64_t p = cnt[j];
        while (p < cnt[j + 1]) {
            const int64_t r = rows[p];
            double sum = vals[p];
            ++p;
            while (p < cnt[j + 1] && rows[p] == r) sum += vals[p++];
            if (sum != 0.0) {
                ciT[w] = r;
                valT[w] = sum;
                ++w;
            }
        }
        rpT[j + 1] = w;
    }
    free(cnt);
    free(rows);
    free(vals);
    free(cur);
    return w;
}

void hno_spmm(int64_t m, const int64_t* rp, const int64_t* ci, const double* val,
              const double* B, int64_t k, double* C) {
    /* gpu_backend.cpp:112-121 */
    for (int64_t i = 0; i < m * k; ++i) C[i] = 0.0;
    for (int64_t i = 0; i < m; ++i)
        for (int64_t p = rp[i]; p < rp[i + 1]; ++p) {
            const int64_t j = ci[p];
            const double a = val[p];
            for (int64_t c = 0; c < k; ++c) C[i * k + c] += a * B[j * k + c];
        }
}

double hno_dot(int64_t n, const double* a, const double* b) {
    double s = 0.0; /* gpu_backend.cpp:123-126 */
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

void hno_axpy(int64_t n, double alpha, const double* x, double* y) {
    for (int64_t i = 0; i < n; ++i) y[i] += alpha * x[i]; /* gpu_backend.cpp:127-129 */
}

double hno_norm_inf(int64_t n, const double* v) {
    /* gpu_backend.cpp:130-134: std::max(mx, |v|) keeps mx when |v| is NaN */
    double mx = 0.0;
    for (int64_t i = 0; i < n; ++i) {
        const double a = fabs(v[i]);
        mx = (mx < a) ? a : mx;
    }
    return mx;
}

double hno_nrm2(int64_t n, const double* v) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += v[i] * v[i];
    return sqrt(s);
}

double hno_max_step(int64_t n, const double* v, const double* d) {
    /* interior_point.cpp:134-142: std::min(alpha, r) keeps alpha when r is NaN */
    double alpha = 1.0;
    for (int64_t i = 0; i < n; ++i)
        if (d[i] < 0.0) {
            const double r = -v[i] / d[i];
            alpha = (r < alpha) ? r : alpha;
        }
    const double s = 0.99 * alpha;
    return (s < 1.0) ? s : 1.0;
}

/* ---- build_normal_equations (interior_point.cpp:144-200) ---- */

typedef struct {
    int64_t row, col, seq;
    double value;
} trip_t;

static int i64_cmp_fwd(const void* a, const void* b) {
    const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return x < y ? -1 : (x > y);
}

static int trip_cmp(const void* a, const void* b) {
    const trip_t* x = (const trip_t*)a;
    const trip_t* y = (const trip_t*)b;
    if (x->row != y->row) return x->row < y->row ? -1 : 1;
    if (x->col != y->col) return x->col < y->col ? -1 : 1;
    return (x->seq < y->seq) ? -1 : (x->seq > y->seq);
}

static void csc_of(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                   int64_t* cs, int64_t* crows, double* cvals) {
    /* interior_point.cpp:153-173 */
    for (int64_t j = 0; j <= n; ++j) cs[j] = 0;
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) cs[ci[k] + 1]++;
    for (int64_t j = 0; j < n; ++j) cs[j + 1] += cs[j];
    int64_t* cur = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n ? n : 1));
    for (int64_t j = 0; j < n; ++j) cur[j] = cs[j];
    for (int64_t i = 0; i < m; ++i)
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int64_t j = ci[k];
            crows[cur[j]] = i;
            if (cvals) cvals[cur[j]] = val[k];
            ++cur[j];
        }
    free(cur);
}

int64_t hno_normal_equations_triplets(int64_t m, int64_t n, const int64_t* rp,
                                      const int64_t* ci, const double* D) {
    int64_t* cnt = (int64_t*)calloc((size_t)n + 1, sizeof(int64_t));
    for (int64_t k = 0; k < rp[m]; ++k) cnt[ci[k]]++;
    int64_t t = m;
    for (int64_t j = 0; j < n; ++j)
        if (!(D[j] <= 0.0)) t += cnt[j] * cnt[j];
    free(cnt);
    return t;
}

int64_t hno_normal_equations(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                             const double* val, const double* D, double reg, int64_t* rpN,
                             int64_t* ciN, double* valN, double* dyn_reg_out) {
    const int64_t nnz = rp[m];
    int64_t* cs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t* crows = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz ? nnz : 1));
    double* cvals = (double*)malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
    csc_of(m, n, rp, ci, val, cs, crows, cvals);
    const int64_t nt = hno_normal_equations_triplets(m, n, rp, ci, D);
    trip_t* t = (trip_t*)malloc(sizeof(trip_t) * (size_t)(nt ? nt : 1));
    int64_t w = 0;
    for (int64_t j = 0; j < n; ++j) { /* :176-186 */
        if (D[j] <= 0.0) continue;
        const double d = D[j];
        for (int64_t p = cs[j]; p < cs[j + 1]; ++p)
            for (int64_t q = cs[j]; q < cs[j + 1]; ++q) {
                t[w].row = crows[p];
                t[w].col = crows[q];
                t[w].value = cvals[p] * cvals[q] * d;
                t[w].seq = w;
                ++w;
            }
    }
    double* diag = (double*)calloc((size_t)(m ? m : 1), sizeof(double));
    for (int64_t k = 0; k < w; ++k) /* :188-191 */
        if (t[k].row == t[k].col) diag[t[k].row] += t[k].value;
    double max_diag = 0.0;
    for (int64_t i = 0; i < m; ++i) max_diag = (max_diag < diag[i]) ? diag[i] : max_diag;
    double dyn = 1e-12 * max_diag; /* :193 */
    dyn = (reg < dyn) ? dyn : reg;
    for (int64_t i = 0; i < m; ++i) { /* :194-196 */
        t[w].row = i;
        t[w].col = i;
        t[w].value = dyn;
        t[w].seq = w;
        ++w;
    }
    qsort(t, (size_t)w, sizeof(trip_t), trip_cmp);
    int64_t out = 0;
    int64_t k = 0;
    rpN[0] = 0;
    for (int64_t i = 0; i < m; ++i) {
        while (k < w && t[k].row == i) {
            const int64_t c = t[k].col;
            double s = t[k].value;
            ++k;
            while (k < w && t[k].row == i && t[k].col == c) s += t[k++].value;
            if (s != 0.0) {
                ciN[out] = c;
                valN[out] = s;
                ++out;
            }
        }
        rpN[i + 1] = out;
    }
    if (dyn_reg_out) *dyn_reg_out = dyn;
    free(cs);
    free(crows);
    free(cvals);
    free(t);
    free(diag);
    return out;
}

/* Selected rows of the same N (interior_point.cpp:144-200), for matrices
 * whose full triplet list does not fit: row i of N gathers, for every column
 * j of row i with D_j > 0 (j ascending, the emission order of :176-186), the
 * terms (a_ij * a_kj) * D_j of column j's rows k; each entry sums its terms in
 * that order (as the stable sort of the full restatement does), exact zero
 * sums are dropped, and the diagonal gains dyn_reg = max(reg, 1e-12 * max over
 * ALL rows of sum_j a_ij^2 D_j) last (:188-196). absS (may be NULL) receives
 * the same sums over |terms| (with dyn_reg on the diagonal), the scale of the
 * 1e-12 normwise bar. With ciS == NULL only rpS (nsel + 1 offsets) is filled.
 * Returns the entry count. */
int64_t hno_normal_rows(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                        const double* D, double reg, int64_t nsel, const int64_t* rows, int64_t* rpS,
                        int64_t* ciS, double* valS, double* absS, double* dyn_out) {
    const int64_t nnz = rp[m];
    int64_t* cs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t* crows = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz ? nnz : 1));
    double* cvals = (double*)malloc(sizeof(double) * (size_t)(nnz ? nnz : 1));
    csc_of(m, n, rp, ci, val, cs, crows, cvals);
    double max_diag = 0.0;
    for (int64_t i = 0; i < m; ++i) {
        double dsum = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int64_t j = ci[k];
            if (D[j] <= 0.0) continue;
            dsum += val[k] * val[k] * D[j];
        }
        max_diag = (max_diag < dsum) ? dsum : max_diag;
    }
    double dyn = 1e-12 * max_diag;
    dyn = (reg < dyn) ? dyn : reg;
    double* acc = (double*)calloc((size_t)(m ? m : 1), sizeof(double));
    double* aab = (double*)calloc((size_t)(m ? m : 1), sizeof(double));
    char* seen = (char*)calloc((size_t)(m ? m : 1), 1);
    int64_t* touched = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    int64_t out = 0;
    rpS[0] = 0;
    for (int64_t s = 0; s < nsel; ++s) {
        const int64_t i = rows[s];
        int64_t nt = 0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            const int64_t j = ci[k];
            if (D[j] <= 0.0) continue;
            const double d = D[j], aij = val[k];
            for (int64_t q = cs[j]; q < cs[j + 1]; ++q) {
                const int64_t r = crows[q];
                const double t = aij * cvals[q] * d;
                if (!seen[r]) {
                    seen[r] = 1;
                    touched[nt++] = r;
                }
                acc[r] += t;
                aab[r] += fabs(t);
            }
        }
        if (!seen[i]) {
            seen[i] = 1;
            touched[nt++] = i;
        }
        acc[i] += dyn;
        aab[i] += dyn;
        qsort(touched, (size_t)nt, sizeof(int64_t), i64_cmp_fwd);
        for (int64_t t = 0; t < nt; ++t) {
            const int64_t r = touched[t];
            if (acc[r] != 0.0) {
                if (ciS) {
                    ciS[out] = r;
                    valS[out] = acc[r];
                    if (absS) absS[out] = aab[r];
                }
                ++out;
            }
            acc[r] = 0.0;
            aab[r] = 0.0;
            seen[r] = 0;
        }
        rpS[s + 1] = out;
    }
    if (dyn_out) *dyn_out = dyn;
    free(cs);
    free(crows);
    free(cvals);
    free(acc);
    free(aab);
    free(seen);
    free(touched);
    return out;
}

static int i64_cmp(const void* a, const void* b) {
    const int64_t x = *(const int64_t*)a, y = *(const int64_t*)b;
    return (x > y) - (x < y);
}

int64_t hno_ada_pattern(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci,
                        int64_t* rpN, int32_t* ciN) {
    const int64_t nnz = rp[m];
    int64_t* cs = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
    int64_t* crows = (int64_t*)malloc(sizeof(int64_t) * (size_t)(nnz ? nnz : 1));
    csc_of(m, n, rp, ci, NULL, cs, crows, NULL);
    unsigned char* mark = (unsigned char*)calloc((size_t)(m ? m : 1), 1);
    int64_t* list = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    int64_t total = 0;
    rpN[0] = 0;
    for (int64_t i = 0; i < m; ++i) {
        int64_t cnt = 0;
        mark[i] = 1;
        list[cnt++] = i;
        for (int64_t e = rp[i]; e < rp[i + 1]; ++e) {
            const int64_t j = ci[e];
            for (int64_t p = cs[j]; p < cs[j + 1]; ++p) {
                const int64_t k = crows[p];
                if (!mark[k]) {
                    mark[k] = 1;
                    list[cnt++] = k;
                }
            }
        }
        /* emit in increasing column order */
        if (ciN) {
            qsort(list, (size_t)cnt, sizeof(int64_t), i64_cmp);
            for (int64_t q = 0; q < cnt; ++q) ciN[total + q] = (int32_t)list[q];
        }
        for (int64_t q = 0; q < cnt; ++q) mark[list[q]] = 0;
        total += cnt;
        rpN[i + 1] = total;
    }
    free(cs);
    free(crows);
    free(mark);
    free(list);
    return total;
}

void hno_merge_tiles(int64_t m, int64_t nnz, const int32_t* rp, int64_t items, int64_t ntiles,
                     int32_t* tile_row, int32_t* tile_nz) {
    /* Merge of list A = row ends rp[1..m] with list B = 0..nnz-1: a row end
     * rp[i+1] is taken before nonzero index k when rp[i+1] <= k. */
    const int64_t total = m + nnz;
    for (int64_t t = 0; t <= ntiles; ++t) {
        int64_t diag = t * items;
        if (diag > total) diag = total;
        int64_t lo = diag - nnz > 0 ? diag - nnz : 0;
        int64_t hi = diag < m ? diag : m;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((int64_t)rp[mid + 1] <= diag - mid - 1)
                lo = mid + 1;
            else
                hi = mid;
        }
        tile_row[t] = (int32_t)lo;
        tile_nz[t] = (int32_t)(diag - lo);
    }
}

/* ---------------------------------------------------------------- pricing */

void hno_price_reduced_costs(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                             const double* y, const double* cost, double* rc) {
    /* simplex.cpp:1229-1232 */
    hno_csr_tmultiply(m, n, rp, ci, val, y, rc);
    for (int64_t j = 0; j < n; ++j) rc[j] = cost[j] - rc[j];
}

void hno_price_devex_update(int64_t m, int64_t n, const int64_t* rp, const int64_t* ci, const double* val,
                            const double* u, const int32_t* nonbasis, double* weights, double* alpha) {
    /* simplex.cpp:1249-1270 */
    for (int64_t j = 0; j < n; ++j) alpha[j] = 0.0;
    for (int64_t i = 0; i < m; ++i) {
        if (u[i] == 0.0) continue;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) alpha[ci[k]] += val[k] * u[i];
    }
    double s = 0.0;
    for (int64_t j = 0; j < n; ++j) {
        if (nonbasis[j] < 0) continue;
        const double a = fabs(alpha[j]);
        s = (s < a) ? a : s; /* std::max(s, a) */
    }
    if (s == 0.0) return;
    for (int64_t j = 0; j < n; ++j) {
        if (nonbasis[j] < 0) continue;
        const double t = alpha[j] / s;
        const double w = t * t;
        if (w > weights[j]) weights[j] = w;
    }
}

typedef struct {
    int64_t j;
    double score;
} hno_ranked;

static int hno_ranked_cmp(const void* pa, const void* pb) {
    const hno_ranked* a = (const hno_ranked*)pa;
    const hno_ranked* b = (const hno_ranked*)pb;
    if (a->score != b->score) return a->score > b->score ? -1 : 1;
    return a->j < b->j ? -1 : (a->j > b->j ? 1 : 0);
}

int64_t hno_price_ranked(int64_t n, const double* rc, const double* w, const int32_t* nonbasis,
                         const uint8_t* artificial, int phase1, int maximize, double tol, int64_t cap,
                         int64_t* out) {
    /* simplex.cpp:1283-1308: filter, score |rc|/sqrt(w) with w guarded, sort by
     * (score desc, index asc) -- a total order, so qsort gives stable_sort's result */
    hno_ranked* r = (hno_ranked*)malloc(sizeof(hno_ranked) * (size_t)(n > 0 ? n : 1));
    int64_t cnt = 0;
    for (int64_t j = 0; j < n; ++j) {
        if (nonbasis[j] < 0) continue;
        if (!phase1 && artificial && artificial[j]) continue;
        double c = rc[j];
        if (maximize) c = -c;
        if (c >= -tol) continue;
        double wj = w ? w[j] : 1.0;
        if (!(wj > 0.0) || !isfinite(wj)) wj = 1.0;
        r[cnt].j = j;
        r[cnt].score = fabs(c) / sqrt(wj);
        ++cnt;
    }
    qsort(r, (size_t)cnt, sizeof(hno_ranked), hno_ranked_cmp);
    for (int64_t k = 0; k < cap; ++k) out[k] = k < cnt ? r[k].j : -1;
    free(r);
    return cnt;
}

int64_t hno_price_bland(int64_t n, const double* rc, const int32_t* nonbasis, const uint8_t* artificial,
                        int phase1, int maximize, double tol) {
    /* simplex.cpp:1328-1338 */
    for (int64_t j = 0; j < n; ++j) {
        if (nonbasis[j] < 0) continue;
        if (!phase1 && artificial && artificial[j]) continue;
        double c = rc[j];
        if (maximize) c = -c;
        if (c < -tol) return j;
    }
    return -1;
}

void hno_extract_column(int64_t m, const int64_t* rp, const int64_t* ci, const double* val, int64_t j,
                        double* col) {
    /* simplex.cpp:25-35 */
    for (int64_t i = 0; i < m; ++i) {
        col[i] = 0.0;
        for (int64_t k = rp[i]; k < rp[i + 1]; ++k) {
            if (ci[k] == j) {
                col[i] = val[k];
                break;
            }
        }
    }
}
