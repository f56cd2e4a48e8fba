// Sparse LDL^T of the IPM's normal matrix on the host: the factorisation
// behind HyperNova's SparseCholesky interface (core/numerical/
// factorization.hpp:162-208: analyze / factorize / refactorize / solve),
// with a fill-reducing ordering and supernodal numerics in place of the
// reference's O(m^2)-per-step minimum degree and column-by-column updates.
//
//   ordering   approximate minimum degree (Amestoy, Davis & Duff, SIAM J.
//              Matrix Anal. Appl. 17(4), 1996) on the quotient graph:
//              element absorption, approximate external degrees, aggressive
//              absorption, supervariables found by hashing; rows denser
//              than 10 sqrt(m) are ordered last
//   symbolic   elimination tree (Liu), postorder, column structures by
//              merging children, fundamental supernodes
//   numeric    multifrontal: per supernode a dense front assembled from N
//              and the children's update matrices, its pivot columns
//              factorised (blocked right-looking) with the reference's pivot
//              clamp (d <= tol -> tol, factorization.cpp:1310-1313), the
//              Schur complement passed to the parent
//   solve      forward with unit L, divide by D, backward, in supernodes
#include <omp.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <numeric>
#include <set>
#include <stdexcept>
#include <unordered_map>
#include <utility>
#include <vector>

#include "hn_lp.hpp"

namespace hn::lp {

// ---- ordering ----
std::vector<int> amd_order(int n, const std::vector<int>& rp, const std::vector<int>& ci) {
    enum : char { VAR, ELEM, DEAD, MERGED };
    // symmetric adjacency without the diagonal
    std::vector<std::vector<int>> A(n), E(n);
    for (int i = 0; i < n; ++i)
        for (int k = rp[i]; k < rp[i + 1]; ++k) {
            const int j = ci[k];
            if (j == i) continue;
            A[i].push_back(j);
            A[j].push_back(i);
        }
    for (auto& a : A) {
        std::sort(a.begin(), a.end());
        a.erase(std::unique(a.begin(), a.end()), a.end());
    }
    // dense rows go last, in their original order
    const std::size_t dense = std::max<std::size_t>(16, static_cast<std::size_t>(10.0 * std::sqrt((double)n)));
    std::vector<char> state(n, VAR);
    std::vector<int> tail;
    for (int i = 0; i < n; ++i)
        if (A[i].size() > dense) {
            state[i] = DEAD;
            tail.push_back(i);
        }
    if (!tail.empty())
        for (int i = 0; i < n; ++i) {
            if (state[i] != VAR) continue;
            auto& a = A[i];
            a.erase(std::remove_if(a.begin(), a.end(), [&](int j) { return state[j] != VAR; }), a.end());
        }
    std::vector<int> nv(n, 1), deg(n, 0);
    std::vector<std::vector<int>> members(n);
    std::set<std::pair<int, int>> pq;
    long nleft = 0;
    for (int i = 0; i < n; ++i)
        if (state[i] == VAR) {
            deg[i] = static_cast<int>(A[i].size());
            pq.emplace(deg[i], i);
            ++nleft;
        }
    std::vector<int> order;
    order.reserve(n);
    std::vector<unsigned> mark(n, 0), wtag(n, 0);
    std::vector<long> wval(n, 0);
    unsigned gen = 0;
    std::vector<int> Lp;
    while (!pq.empty()) {
        const int p = pq.begin()->second;
        pq.erase(pq.begin());
        ++gen;
        mark[p] = gen;
        // L_p: the union of p's elements and variables, minus p
        Lp.clear();
        for (int e : E[p]) {
            if (state[e] != ELEM) continue;
            for (int v : A[e])
                if (state[v] == VAR && mark[v] != gen) {
                    mark[v] = gen;
                    Lp.push_back(v);
                }
            state[e] = DEAD;  // absorbed into p
            A[e].clear();
            A[e].shrink_to_fit();
        }
        for (int v : A[p])
            if (state[v] == VAR && mark[v] != gen) {
                mark[v] = gen;
                Lp.push_back(v);
            }
        order.push_back(p);
        order.insert(order.end(), members[p].begin(), members[p].end());
        members[p].clear();
        members[p].shrink_to_fit();
        nleft -= nv[p];
        state[p] = ELEM;
        E[p].clear();
        E[p].shrink_to_fit();
        A[p] = Lp;
        long lpw = 0;
        for (int v : Lp) lpw += nv[v];
        // variables of L_p: p joins their elements; entries covered by p leave
        for (int i : Lp) {
            auto& ei = E[i];
            ei.erase(std::remove_if(ei.begin(), ei.end(), [&](int e) { return state[e] != ELEM; }), ei.end());
            ei.insert(std::lower_bound(ei.begin(), ei.end(), p), p);
            auto& ai = A[i];
            ai.erase(std::remove_if(ai.begin(), ai.end(), [&](int v) { return state[v] != VAR || mark[v] == gen; }),
                     ai.end());
        }
        // |L_e \ L_p| of every other element next to L_p (weighted)
        for (int i : Lp)
            for (int e : E[i]) {
                if (e == p) continue;
                if (wtag[e] != gen) {
                    wtag[e] = gen;
                    auto& le = A[e];
                    le.erase(std::remove_if(le.begin(), le.end(), [&](int v) { return state[v] != VAR; }), le.end());
                    long s = 0;
                    for (int v : le) s += nv[v];
                    wval[e] = s;
                }
                wval[e] -= nv[i];
            }
        // aggressive absorption: an element inside L_p is absorbed by p
        for (int i : Lp)
            for (int e : E[i])
                if (e != p && state[e] == ELEM && wval[e] == 0) {
                    state[e] = DEAD;
                    A[e].clear();
                }
        // approximate external degrees
        for (int i : Lp) {
            auto& ei = E[i];
            ei.erase(std::remove_if(ei.begin(), ei.end(), [&](int e) { return state[e] != ELEM; }), ei.end());
            long ext = 0;
            for (int e : ei)
                if (e != p) ext += wval[e];
            long aw = 0;
            for (int v : A[i]) aw += nv[v];
            const long own = lpw - nv[i];
            long d = std::min<long>(nleft - nv[i], std::min<long>((long)deg[i] + own, aw + own + ext));
            if (d < 0) d = 0;
            pq.erase({deg[i], i});
            deg[i] = static_cast<int>(d);
        }
        // supervariables: equal element and variable sets merge into one
        std::unordered_map<uint64_t, std::vector<int>> buckets;
        for (int i : Lp) {
            uint64_t h = 1469598103934665603ull;
            for (int e : E[i]) h = (h ^ (uint64_t)e) * 1099511628211ull;
            h ^= 0x9e3779b97f4a7c15ull;
            for (int v : A[i]) h = (h ^ (uint64_t)v) * 1099511628211ull;
            buckets[h].push_back(i);
        }
        for (auto& kv : buckets) {
            auto& b = kv.second;
            for (std::size_t x = 0; x < b.size(); ++x) {
                const int i = b[x];
                if (state[i] != VAR) continue;
                for (std::size_t y = x + 1; y < b.size(); ++y) {
                    const int j = b[y];
                    if (state[j] != VAR || E[i] != E[j] || A[i] != A[j]) continue;
                    nv[i] += nv[j];
                    deg[i] = std::max(0, deg[i] - nv[j]);
                    members[i].push_back(j);
                    members[i].insert(members[i].end(), members[j].begin(), members[j].end());
                    members[j].clear();
                    nv[j] = 0;
                    state[j] = MERGED;
                    pq.erase({deg[j], j});
                    E[j].clear();
                    A[j].clear();
                }
            }
        }
        for (int i : Lp)
            if (state[i] == VAR) pq.emplace(deg[i], i);
        // merged variables leave the element lists lazily (state check)
    }
    order.insert(order.end(), tail.begin(), tail.end());
    if (static_cast<int>(order.size()) != n) throw std::logic_error("amd_order: ordering incomplete");
    return order;
}

// ---- symbolic analysis ----
void SparseLDLT::analyze(std::size_t m, const uint64_t* rp, const uint64_t* ci) {
    // the ordering and the symbolic analysis index rows and entries with int
    if (m > static_cast<std::size_t>(INT_MAX) || rp[m] > static_cast<uint64_t>(INT_MAX))
        throw std::invalid_argument("SparseLDLT: " + std::to_string(m) + " rows / " + std::to_string(rp[m]) +
                                    " entries exceed the 2^31 - 1 index range");
    m_ = m;
    const int n = static_cast<int>(m);
    std::vector<int> rp32(m + 1), ci32(rp[m]);
    for (std::size_t i = 0; i <= m; ++i) rp32[i] = static_cast<int>(rp[i]);
    for (uint64_t k = 0; k < rp[m]; ++k) ci32[k] = static_cast<int>(ci[k]);
    std::vector<int> ord = amd_order(n, rp32, ci32);  // new -> old
    std::vector<int> inv(n);
    for (int k = 0; k < n; ++k) inv[ord[k]] = k;
    // elimination tree of the permuted matrix (row-wise lower pattern)
    std::vector<std::vector<int>> rowlow(n);
    for (int i = 0; i < n; ++i)
        for (int k = rp32[i]; k < rp32[i + 1]; ++k) {
            const int a = inv[i], b = inv[ci32[k]];
            if (b < a) rowlow[a].push_back(b);
        }
    std::vector<int> parent(n, -1), anc(n, -1);
    for (int k = 0; k < n; ++k)
        for (int j : rowlow[k]) {
            while (j != -1 && j < k) {
                const int nx = anc[j];
                anc[j] = k;
                if (nx == -1) parent[j] = k;
                j = nx;
            }
        }
    // postorder (children before parents, subtrees contiguous)
    std::vector<std::vector<int>> kids(n);
    std::vector<int> roots;
    for (int j = n - 1; j >= 0; --j) (parent[j] == -1 ? roots : kids[parent[j]]).push_back(j);
    std::vector<int> post;
    post.reserve(n);
    std::vector<std::pair<int, std::size_t>> stack;
    for (auto it = roots.rbegin(); it != roots.rend(); ++it) {
        stack.emplace_back(*it, 0);
        while (!stack.empty()) {
            auto& [v, c] = stack.back();
            if (c < kids[v].size()) {
                const int ch = kids[v][kids[v].size() - 1 - c];
                ++c;
                stack.emplace_back(ch, 0);
            } else {
                post.push_back(v);
                stack.pop_back();
            }
        }
    }
    // final order: AMD then postorder
    perm_.resize(m);
    std::vector<int> relabel(n);
    for (int k = 0; k < n; ++k) {
        perm_[k] = ord[post[k]];
        relabel[post[k]] = k;
    }
    iperm_.assign(m, 0);
    for (int k = 0; k < n; ++k) iperm_[perm_[k]] = k;
    parent_.assign(n, -1);
    for (int j = 0; j < n; ++j)
        if (parent[j] != -1) parent_[relabel[j]] = relabel[parent[j]];
    // lower columns of the permuted matrix: rows > c of column c
    std::vector<std::vector<int>> colrows(n);
    for (int i = 0; i < n; ++i)
        for (int k = rp32[i]; k < rp32[i + 1]; ++k) {
            const int a = iperm_[i], b = iperm_[ci32[k]];
            if (a > b) colrows[b].push_back(a);
        }
    // column structures of L: A's column merged with the children's
    std::vector<std::vector<int>> child(n);
    for (int j = 0; j < n; ++j)
        if (parent_[j] != -1) child[parent_[j]].push_back(j);
    std::vector<std::vector<int>> cstruct(n);
    std::vector<int> marker(n, -1);
    for (int j = 0; j < n; ++j) {
        auto& s = cstruct[j];
        marker[j] = j;
        for (int r : colrows[j])
            if (marker[r] != j) {
                marker[r] = j;
                s.push_back(r);
            }
        for (int c : child[j])
            for (int r : cstruct[c])
                if (r != j && marker[r] != j) {
                    marker[r] = j;
                    s.push_back(r);
                }
        std::sort(s.begin(), s.end());
    }
    // fundamental supernodes: j + 1 = parent(j), j its only child, nested structure
    snode_start_.clear();
    for (int j = 0; j < n; ++j) {
        const bool join = j > 0 && parent_[j - 1] == j && child[j].size() == 1 &&
                          cstruct[j - 1].size() == cstruct[j].size() + 1 && j - snode_start_.back() < 4096;
        if (!join) snode_start_.push_back(j);
    }
    snode_start_.push_back(n);
    const int ns = static_cast<int>(snode_start_.size()) - 1;
    snode_of_.assign(n, 0);
    for (int s = 0; s < ns; ++s)
        for (int j = snode_start_[s]; j < snode_start_[s + 1]; ++j) snode_of_[j] = s;
    // each supernode's rows: its columns then the first column's structure below them
    srows_off_.assign(ns + 1, 0);
    srows_.clear();
    for (int s = 0; s < ns; ++s) {
        const int c0 = snode_start_[s], c1 = snode_start_[s + 1];
        for (int c = c0; c < c1; ++c) srows_.push_back(c);
        for (int r : cstruct[c0])
            if (r >= c1) srows_.push_back(r);
        srows_off_[s + 1] = srows_.size();
    }
    snode_parent_.assign(ns, -1);
    for (int s = 0; s < ns; ++s) {
        const int last = snode_start_[s + 1] - 1;
        if (parent_[last] != -1) snode_parent_[s] = snode_of_[parent_[last]];
    }
    // assembly map: input entry k of the lower permuted triangle -> (supernode, front position)
    std::vector<int> pos(n, -1);
    amap_off_.assign(ns + 1, 0);
    std::vector<std::vector<std::pair<uint64_t, std::size_t>>> per(ns);
    for (int s = 0; s < ns; ++s) {
        const std::size_t r0 = srows_off_[s], nf = srows_off_[s + 1] - r0;
        for (std::size_t t = 0; t < nf; ++t) pos[srows_[r0 + t]] = static_cast<int>(t);
        const int c0 = snode_start_[s], c1 = snode_start_[s + 1];
        for (int c = c0; c < c1; ++c) {
            const int oc = perm_[c];
            for (uint64_t k = rp[oc]; k < rp[oc + 1]; ++k) {
                const int r = iperm_[ci[k]];
                if (r < c) continue;  // the upper copy
                per[s].emplace_back(k, static_cast<std::size_t>(c - c0) * nf + static_cast<std::size_t>(pos[r]));
            }
        }
        for (std::size_t t = 0; t < nf; ++t) pos[srows_[r0 + t]] = -1;
    }
    amap_.clear();
    for (int s = 0; s < ns; ++s) {
        amap_.insert(amap_.end(), per[s].begin(), per[s].end());
        amap_off_[s + 1] = amap_.size();
    }
    // L storage: per supernode a column-major nf x w panel
    panel_off_.assign(ns + 1, 0);
    nnz_L_ = 0;
    for (int s = 0; s < ns; ++s) {
        const std::size_t nf = srows_off_[s + 1] - srows_off_[s];
        const std::size_t w = static_cast<std::size_t>(snode_start_[s + 1] - snode_start_[s]);
        panel_off_[s + 1] = panel_off_[s] + nf * w;
        nnz_L_ += nf * w - w * (w + 1) / 2;
    }
    analyzed_ = true;
}

// ---- numeric factorisation (multifrontal) ----
namespace {
// F(i, j) -= sum_{k in [kb, ke)} L(i, k) (L(j, k) D_k) for ke <= j <= i < nf:
// the trailing triangle's update by one panel, in register tiles of 8 rows
// x 4 columns (per pivot one 8-wide load of L and 4 broadcasts feed 32
// multiply-adds). Tiles on the diagonal also write above it; those entries
// of a front are never read.
void trailing_update(double* F, std::size_t nf, std::size_t kb, std::size_t ke, const double* D) {
    const std::size_t nbk = ke - kb, t = nf - ke, tp = (t + 7) & ~std::size_t(7);
    // LT[k][i] = L(ke+i, kb+k), C[j][k] = L(ke+j, kb+k) D_k, padded to tp rows
    // with zeros; per-thread buffers reused across panels and fronts
    thread_local std::vector<double> LT, C;
    if (LT.size() < nbk * tp) LT.resize(nbk * tp);
    if (C.size() < tp * nbk) C.resize(tp * nbk);
    for (std::size_t k = 0; k < nbk; ++k) {
        const double* lk = F + (kb + k) * nf + ke;
        std::memcpy(LT.data() + k * tp, lk, sizeof(double) * t);
        std::fill(LT.data() + k * tp + t, LT.data() + (k + 1) * tp, 0.0);
        for (std::size_t j = 0; j < t; ++j) C[j * nbk + k] = lk[j] * D[kb + k];
    }
    std::fill(C.data() + t * nbk, C.data() + tp * nbk, 0.0);
    // the parallel loop reads the calling thread's buffers through these
    // (a thread_local name inside the region would be each worker's own)
    const double* const LTp = LT.data();
    const double* const Cp = C.data();
    const std::size_t nj = (t + 3) / 4;
    const bool par = t * t * nbk > (std::size_t(1) << 21);
#pragma omp parallel for schedule(dynamic, 2) if (par)
    for (std::size_t jb = 0; jb < nj; ++jb) {
        const std::size_t j0 = jb * 4, nc = std::min<std::size_t>(4, t - j0);
        const double* c0 = Cp + j0 * nbk;
        for (std::size_t i0 = j0 & ~std::size_t(7); i0 < t; i0 += 8) {
            double acc[4][8] = {};
            for (std::size_t k = 0; k < nbk; ++k) {
                const double* l = LTp + k * tp + i0;
                for (std::size_t jj = 0; jj < 4; ++jj) {
                    const double c = c0[jj * nbk + k];
#pragma omp simd
                    for (std::size_t ii = 0; ii < 8; ++ii) acc[jj][ii] += l[ii] * c;
                }
            }
            const std::size_t nr = std::min<std::size_t>(8, t - i0);
            for (std::size_t jj = 0; jj < nc; ++jj) {
                double* f = F + (ke + j0 + jj) * nf + ke + i0;
                for (std::size_t ii = 0; ii < nr; ++ii) f[ii] -= acc[jj][ii];
            }
        }
    }
}

// front F (nf x nf, column-major, lower used): factor the first w columns
// with the pivot clamp, leave L there, and return the Schur complement
// U = F22 - L21 D L21^T (r x r lower, column-major) in `upd`. Blocked
// right-looking: a panel of up to 32 pivot columns is factorised against
// itself, then the whole trailing lower triangle takes its rank-32 update
// (trailing_update).
void factor_front(double* F, std::size_t nf, std::size_t w, double tol, double* Dout, bool& singular,
                  std::vector<double>& upd) {
    constexpr std::size_t kNb = 32;
    for (std::size_t kb = 0; kb < w; kb += kNb) {
        const std::size_t ke = std::min(w, kb + kNb), nbk = ke - kb;
        for (std::size_t k = kb; k < ke; ++k) {
            double* fk = F + k * nf;
            double d = fk[k];
            if (d <= tol) {
                d = tol;
                singular = true;
            }
            Dout[k] = d;
            fk[k] = 1.0;
            const double inv = 1.0 / d;
            for (std::size_t i = k + 1; i < nf; ++i) fk[i] *= inv;
            for (std::size_t j = k + 1; j < ke; ++j) {
                const double ljd = fk[j] * d;
                if (ljd == 0.0) continue;
                double* fj = F + j * nf;
                for (std::size_t i = j; i < nf; ++i) fj[i] -= fk[i] * ljd;
            }
        }
        if (ke < nf) trailing_update(F, nf, kb, ke, Dout);
    }
    const std::size_t r = nf - w;
    upd.assign(r * r, 0.0);
    for (std::size_t j = 0; j < r; ++j)
        std::memcpy(upd.data() + j * r + j, F + (w + j) * nf + w + j, sizeof(double) * (r - j));
}
}  // namespace

bool SparseLDLT::factorize(const double* val, double tol) {
    if (!analyzed_) throw std::logic_error("SparseLDLT::factorize before analyze");
    const int ns = static_cast<int>(snode_start_.size()) - 1;
    L_.assign(panel_off_[ns], 0.0);
    D_.assign(m_, 0.0);
    singular_ = false;
    // supernodal tree: children, first descendant (subtrees are contiguous
    // id ranges in postorder) and the front work of every subtree
    std::vector<std::vector<int>> kids(ns);
    std::vector<int> first(ns);
    std::vector<double> sub(ns, 0.0);
    double total = 0.0;
    for (int s = 0; s < ns; ++s) {
        const double nf = static_cast<double>(srows_off_[s + 1] - srows_off_[s]);
        const double w = static_cast<double>(snode_start_[s + 1] - snode_start_[s]);
        sub[s] += nf * nf * (w + 1.0);
        const int p = snode_parent_[s];
        if (p != -1) {
            kids[p].push_back(s);
            sub[p] += sub[s];
        } else {
            total += sub[s];
        }
    }
    for (int s = 0; s < ns; ++s) first[s] = s;
    for (int s = 0; s < ns; ++s)
        if (snode_parent_[s] != -1) first[snode_parent_[s]] = std::min(first[snode_parent_[s]], first[s]);
    // independent subtrees below a work cut are factorised in parallel, the
    // top of the tree afterwards in postorder (its big fronts use the
    // parallel front kernel)
    const int threads = std::max(1, omp_get_max_threads());
    const double cut = total / (4.0 * threads);
    std::vector<int> roots;
    std::vector<char> low(ns, 0);
    for (int s = 0; s < ns; ++s) {
        const int p = snode_parent_[s];
        if (sub[s] <= cut && (p == -1 || sub[p] > cut)) roots.push_back(s);
    }
    std::sort(roots.begin(), roots.end(), [&](int x, int y) { return sub[x] > sub[y]; });
    for (int r : roots)
        for (int t = first[r]; t <= r; ++t) low[t] = 1;
    std::vector<std::vector<double>> U(ns);  // update matrices awaiting their parent

    auto process = [&](int s, std::vector<int>& pos, std::vector<double>& F, bool& sing) {
        const std::size_t r0 = srows_off_[s], nf = srows_off_[s + 1] - r0;
        const std::size_t w = static_cast<std::size_t>(snode_start_[s + 1] - snode_start_[s]);
        // only a front's lower triangle is ever read: the buffer is reused and
        // just that part cleared
        if (F.size() < nf * nf) F.resize(nf * nf);
        for (std::size_t j = 0; j < nf; ++j) std::memset(F.data() + j * nf + j, 0, sizeof(double) * (nf - j));
        for (std::size_t a = amap_off_[s]; a < amap_off_[s + 1]; ++a) F[amap_[a].second] += val[amap_[a].first];
        for (std::size_t t = 0; t < nf; ++t) pos[srows_[r0 + t]] = static_cast<int>(t);
        // extend-add the children's update matrices
        for (int c : kids[s]) {
            if (U[c].empty()) continue;
            const std::size_t cr0 = srows_off_[c], cw = snode_start_[c + 1] - snode_start_[c];
            const std::size_t cr = srows_off_[c + 1] - cr0 - cw;
            const int* rows = srows_.data() + cr0 + cw;
            for (std::size_t j = 0; j < cr; ++j) {
                double* fcol = F.data() + static_cast<std::size_t>(pos[rows[j]]) * nf;
                const double* ucol = U[c].data() + j * cr;
                for (std::size_t i = j; i < cr; ++i) fcol[pos[rows[i]]] += ucol[i];
            }
            std::vector<double>().swap(U[c]);
        }
        for (std::size_t t = 0; t < nf; ++t) pos[srows_[r0 + t]] = -1;
        std::vector<double> u;
        factor_front(F.data(), nf, w, tol, D_.data() + snode_start_[s], sing, u);
        double* Lp = L_.data() + panel_off_[s];
        for (std::size_t k = 0; k < w; ++k) std::memcpy(Lp + k * nf, F.data() + k * nf, sizeof(double) * nf);
        if (nf > w && snode_parent_[s] != -1) U[s] = std::move(u);
    };

    bool any_singular = false;
#pragma omp parallel if (roots.size() > 1) reduction(|| : any_singular)
    {
        std::vector<int> pos(m_, -1);
        std::vector<double> F;
        bool sing = false;
#pragma omp for schedule(dynamic, 1)
        for (std::size_t i = 0; i < roots.size(); ++i)
            for (int t = first[roots[i]]; t <= roots[i]; ++t) process(t, pos, F, sing);
        any_singular = any_singular || sing;
    }
    {
        std::vector<int> pos(m_, -1);
        std::vector<double> F;
        bool sing = false;
        for (int s = 0; s < ns; ++s)
            if (!low[s]) process(s, pos, F, sing);
        any_singular = any_singular || sing;
    }
    singular_ = any_singular;
    factored_ = true;
    return !singular_;
}

void SparseLDLT::solve(std::vector<double>& x) const {
    if (!factored_) throw std::logic_error("SparseLDLT::solve before factorize");
    const int ns = static_cast<int>(snode_start_.size()) - 1;
    std::vector<double> y(m_);
    for (std::size_t k = 0; k < m_; ++k) y[k] = x[perm_[k]];
    for (int s = 0; s < ns; ++s) {  // L y = b (unit diagonal)
        const std::size_t r0 = srows_off_[s], nf = srows_off_[s + 1] - r0;
        const std::size_t w = static_cast<std::size_t>(snode_start_[s + 1] - snode_start_[s]);
        const double* Lp = L_.data() + panel_off_[s];
        const int* rows = srows_.data() + r0;
        for (std::size_t k = 0; k < w; ++k) {
            const double yk = y[rows[k]];
            if (yk == 0.0) continue;
            const double* l = Lp + k * nf;
            for (std::size_t i = k + 1; i < nf; ++i) y[rows[i]] -= l[i] * yk;
        }
    }
    for (std::size_t k = 0; k < m_; ++k) y[k] /= D_[k];
    for (int s = ns - 1; s >= 0; --s) {  // L^T x = y
        const std::size_t r0 = srows_off_[s], nf = srows_off_[s + 1] - r0;
        const std::size_t w = static_cast<std::size_t>(snode_start_[s + 1] - snode_start_[s]);
        const double* Lp = L_.data() + panel_off_[s];
        const int* rows = srows_.data() + r0;
        for (std::size_t kk = w; kk-- > 0;) {
            const double* l = Lp + kk * nf;
            double acc = y[rows[kk]];
            for (std::size_t i = kk + 1; i < nf; ++i) acc -= l[i] * y[rows[i]];
            y[rows[kk]] = acc;
        }
    }
    for (std::size_t k = 0; k < m_; ++k) x[perm_[k]] = y[k];
}

}  // namespace hn::lp
