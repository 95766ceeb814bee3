// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's CPU legs use anything
// under oracle/; the shipped library never links it.
//
// Sparse direct solve of the Newton system for NewtonLinearSystem::solve's
// PARDISO backend (NewtonLinearSystem.cpp:41-53, PardisoSolver.cpp:182-248).
// oneMKL PARDISO, the reference's default backend, is a parallel supernodal
// direct solver with a nested-dissection ordering; it cannot be built here.
// This is the same class of algorithm written out: a multifrontal Cholesky
// factorisation under a nested-dissection ordering of the vertex graph, the
// fronts of independent subtrees factorised on separate threads and the large
// fronts near the root split over threads by columns.  Every entry receives
// its updates in pivot order whatever the thread count, so the result does
// not depend on it; like PARDISO's it is exact to round-off.
#include "oracle_core.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <thread>

namespace oracle {
namespace {

constexpr int LEAF = 24;   // a connected subgraph of at most this many vertices is one dense front
constexpr int PANEL = 64;  // pivots per panel of the dense partial factorisation
constexpr int SUB = 16;    // pivots per sub-panel inside a panel

struct Graph {
    std::vector<int> ptr, adj;
    int n() const { return (int)ptr.size() - 1; }
    int degree(int v) const { return ptr[v + 1] - ptr[v]; }
};

// vertex graph (3x3 blocks) of the lower scalar CSR, without self loops
Graph vertexGraph(const LinearSystem& ls, int nv) {
    std::vector<std::vector<int>> a(nv);
    for (int r = 0; r < 3 * nv; ++r)
        for (int k = ls.rowPtr[r]; k < ls.rowPtr[r + 1]; ++k) {
            int u = r / 3, v = ls.col[k] / 3;
            if (u != v) { a[u].push_back(v); a[v].push_back(u); }
        }
    Graph g;
    g.ptr.assign(nv + 1, 0);
    for (int v = 0; v < nv; ++v) {
        std::sort(a[v].begin(), a[v].end());
        a[v].erase(std::unique(a[v].begin(), a[v].end()), a[v].end());
        g.ptr[v + 1] = g.ptr[v] + (int)a[v].size();
    }
    g.adj.reserve(g.ptr[nv]);
    for (const auto& l : a) g.adj.insert(g.adj.end(), l.begin(), l.end());
    return g;
}

// one front of the assembly tree: the vertices it eliminates and the later
// vertices its update reaches
struct Node {
    std::vector<int> verts;  // eliminated here, in elimination order
    std::vector<int> rows;   // later vertices of the front, by elimination position
    std::vector<int> kids;
    double work = 0;         // factorisation flops of the subtree (for load balance)
};

// Recursive bisection.  Two candidate separators per connected subgraph, the
// smaller one kept: breadth-first level sets from a pseudo-peripheral root
// (of one level, the vertices adjacent to the next), and, when vertex
// positions are given, cuts at the median coordinate along each axis (of one
// side, the vertices adjacent to the other).
class Dissection {
public:
    Dissection(const Graph& g, const double* xyz) : g_(g), xyz_(xyz), in_(g.n(), 0), level_(g.n(), -1), side_(g.n(), -1) {}
    std::vector<Node> nodes;

    std::vector<int> dissect(const std::vector<int>& S) {
        if ((int)S.size() <= LEAF) return {leaf(S)};
        const int tag = ++stamp_;
        for (int v : S) { in_[v] = tag; level_[v] = -1; }
        std::vector<std::vector<int>> comps;
        for (int v : S)
            if (level_[v] < 0) {
                comps.emplace_back();
                bfs(v, tag, comps.back());
            }
        if (comps.size() > 1) {
            std::vector<int> roots, bundle;
            for (const auto& c : comps) {
                if ((int)c.size() <= LEAF) {
                    bundle.insert(bundle.end(), c.begin(), c.end());
                    if ((int)bundle.size() >= LEAF) { roots.push_back(leaf(bundle)); bundle.clear(); }
                } else {
                    auto r = dissect(c);
                    roots.insert(roots.end(), r.begin(), r.end());
                }
            }
            if (!bundle.empty()) roots.push_back(leaf(bundle));
            return roots;
        }
        // pseudo-peripheral root: restart from a minimum-degree vertex of the
        // last level while the eccentricity grows
        std::vector<int> order = std::move(comps[0]);
        int ecc = level_[order.back()];
        for (int it = 0; it < 8; ++it) {
            int cand = -1;
            for (int i = (int)order.size() - 1; i >= 0 && level_[order[i]] == ecc; --i)
                if (cand < 0 || g_.degree(order[i]) < g_.degree(cand)) cand = order[i];
            for (int v : S) level_[v] = -1;
            std::vector<int> o2;
            int e2 = bfs(cand, tag, o2);
            order = std::move(o2);
            if (e2 <= ecc) { ecc = e2; break; }
            ecc = e2;
        }
        if (ecc < 1) return {leaf(S)};
        // level L separates {< L} and {> L} by its vertices that touch level
        // L + 1; take the smallest such separator that leaves at least 35 %
        // of the vertices on either side, else the level of the median vertex
        auto touchesNext = [&](int v) {
            for (int k = g_.ptr[v]; k < g_.ptr[v + 1]; ++k) {
                int u = g_.adj[k];
                if (in_[u] == tag && level_[u] == level_[v] + 1) return true;
            }
            return false;
        };
        std::vector<int> cnt(ecc + 1, 0), sepCnt(ecc + 1, 0);
        for (int v : S) {
            cnt[level_[v]]++;
            if (level_[v] < ecc && touchesNext(v)) sepCnt[level_[v]]++;
        }
        const int ns = (int)S.size();
        int L = -1, median = -1;
        for (int l = 0, acc = 0; l < ecc; ++l) {
            acc += cnt[l];
            if (median < 0 && 2 * acc >= ns) median = l;
            const int a = acc - sepCnt[l], b = ns - acc;
            if (20 * std::min(a, b) >= 7 * ns && (L < 0 || sepCnt[l] < sepCnt[L])) L = l;
        }
        if (L < 0) L = median < 0 ? ecc - 1 : std::min(median, ecc - 1);
        std::vector<int> A, B, sep;
        for (int v : S) {
            int l = level_[v];
            if (l < L) A.push_back(v);
            else if (l > L) B.push_back(v);
            else (touchesNext(v) ? sep : A).push_back(v);
        }
        if (xyz_) geometricCut(S, tag, A, B, sep);
        // no split worth having (a near-clique): one dense front
        if (2 * sep.size() > S.size() || A.empty() || B.empty()) return {leaf(S)};
        std::vector<int> kids;
        if (!A.empty()) { auto r = dissect(A); kids.insert(kids.end(), r.begin(), r.end()); }
        if (!B.empty()) { auto r = dissect(B); kids.insert(kids.end(), r.begin(), r.end()); }
        Node n;
        n.verts = std::move(sep);
        n.kids = std::move(kids);
        nodes.push_back(std::move(n));
        return {(int)nodes.size() - 1};
    }

private:
    const Graph& g_;
    const double* xyz_;
    std::vector<int> in_, level_, side_;
    int stamp_ = 0;

    // the coordinate cuts at the median along each axis; the one with the
    // smallest separator replaces (A, B, sep) when that separator is smaller
    void geometricCut(const std::vector<int>& S, int tag, std::vector<int>& A, std::vector<int>& B, std::vector<int>& sep) {
        const size_t half = S.size() / 2;
        if (half == 0) return;
        std::vector<int> T = S, bestA, bestB, bestSep;
        bool found = false;
        auto touchesOther = [&](int v) {
            for (int k = g_.ptr[v]; k < g_.ptr[v + 1]; ++k) {
                int u = g_.adj[k];
                if (in_[u] == tag && side_[u] != side_[v]) return true;
            }
            return false;
        };
        for (int ax = 0; ax < 3; ++ax) {
            std::nth_element(T.begin(), T.begin() + half, T.end(), [&](int a, int b) {
                const double ka = xyz_[3 * a + ax], kb = xyz_[3 * b + ax];
                return ka < kb || (ka == kb && a < b);
            });
            for (size_t i = 0; i < T.size(); ++i) side_[T[i]] = i < half ? 2 * tag : 2 * tag + 1;
            std::vector<int> a0, a1, b0, b1;  // inner and boundary vertices of either side
            for (size_t i = 0; i < T.size(); ++i) {
                const int v = T[i];
                const bool edge = touchesOther(v);
                if (i < half) (edge ? a1 : a0).push_back(v);
                else (edge ? b1 : b0).push_back(v);
            }
            const size_t size = std::min(a1.size(), b1.size());
            if (size >= (found ? bestSep.size() : sep.size())) continue;
            found = true;
            if (a1.size() <= b1.size()) {
                bestA = std::move(a0);
                bestSep = std::move(a1);
                bestB = std::move(b0);
                bestB.insert(bestB.end(), b1.begin(), b1.end());
            } else {
                bestA = std::move(a0);
                bestA.insert(bestA.end(), a1.begin(), a1.end());
                bestSep = std::move(b1);
                bestB = std::move(b0);
            }
        }
        if (found) {
            A = std::move(bestA);
            B = std::move(bestB);
            sep = std::move(bestSep);
        }
    }

    int leaf(const std::vector<int>& verts) {
        Node n;
        n.verts = verts;
        nodes.push_back(std::move(n));
        return (int)nodes.size() - 1;
    }

    // breadth-first search from s inside the set tagged `tag`; appends the
    // visit order and returns the last level
    int bfs(int s, int tag, std::vector<int>& order) {
        size_t head = order.size();
        level_[s] = 0;
        order.push_back(s);
        int last = 0;
        while (head < order.size()) {
            int v = order[head++];
            last = level_[v];
            for (int k = g_.ptr[v]; k < g_.ptr[v + 1]; ++k) {
                int u = g_.adj[k];
                if (in_[u] == tag && level_[u] < 0) { level_[u] = level_[v] + 1; order.push_back(u); }
            }
        }
        return last;
    }
};

// y[i] -= x[i] * a for i < n (no reduction: each y[i] is updated once)
__attribute__((target_clones("avx2", "default")))
void axpyMinus(double* __restrict y, const double* __restrict x, double a, int n) {
    for (int i = 0; i < n; ++i) y[i] -= x[i] * a;
}

typedef double v4 __attribute__((vector_size(32)));
typedef double v4u __attribute__((vector_size(32), aligned(8)));

// Trailing update of columns [jb, je) of the front F (m x m, column-major) by
// the factorised panel columns k0 .. k0+kb-1: F[i][j] -= L[i][k] L[j][k] for
// i >= j, taken one pivot after another (k ascending) for every entry.  Four
// columns by eight rows are held in registers across the panel.  Rows above
// the diagonal inside a group of four columns are updated too; those entries
// of the upper triangle are never read.
__attribute__((target_clones("avx2", "default")))
void panelTrailing(double* F, int m, int k0, int kb, int jb, int je) {
    const size_t M = (size_t)m;
    int j = jb;
    for (; j + 4 <= je; j += 4) {
        double a[PANEL][4];
        for (int t = 0; t < kb; ++t)
            for (int c = 0; c < 4; ++c) a[t][c] = F[(k0 + t) * M + j + c];
        double* C0 = F + j * M;
        int i = j;
        for (; i + 8 <= m; i += 8) {
            v4 r[4][2];
            for (int c = 0; c < 4; ++c) {
                r[c][0] = *(const v4u*)(C0 + c * M + i);
                r[c][1] = *(const v4u*)(C0 + c * M + i + 4);
            }
            for (int t = 0; t < kb; ++t) {
                const double* x = F + (k0 + t) * M + i;
                const v4 x0 = *(const v4u*)x, x1 = *(const v4u*)(x + 4);
                for (int c = 0; c < 4; ++c) {
                    r[c][0] -= x0 * a[t][c];
                    r[c][1] -= x1 * a[t][c];
                }
            }
            for (int c = 0; c < 4; ++c) {
                *(v4u*)(C0 + c * M + i) = r[c][0];
                *(v4u*)(C0 + c * M + i + 4) = r[c][1];
            }
        }
        for (; i < m; ++i)
            for (int c = 0; c < 4; ++c) {
                double s = C0[c * M + i];
                for (int t = 0; t < kb; ++t) s -= F[(k0 + t) * M + i] * a[t][c];
                C0[c * M + i] = s;
            }
    }
    for (; j < je; ++j)
        for (int k = k0; k < k0 + kb; ++k) {
            const double* Fk = F + k * M;
            axpyMinus(F + j * M + j, Fk + j, Fk[j], m - j);
        }
}

// Fixed worker threads: run(f) calls f(q) for every q < size(), q = 0 on the
// calling thread, and returns when all calls have finished.
class Pool {
public:
    explicit Pool(int threads) : n_(std::max(1, threads)) {
        for (int t = 1; t < n_; ++t) th_.emplace_back([this, t] { loop(t); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> l(mu_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& t : th_) t.join();
    }
    int size() const { return n_; }
    void run(const std::function<void(int)>& f) {
        if (n_ == 1) { f(0); return; }
        {
            std::lock_guard<std::mutex> l(mu_);
            job_ = &f;
            left_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        f(0);
        std::unique_lock<std::mutex> l(mu_);
        done_.wait(l, [&] { return left_ == 0; });
    }

private:
    void loop(int t) {
        long seen = 0;
        for (;;) {
            const std::function<void(int)>* job;
            {
                std::unique_lock<std::mutex> l(mu_);
                cv_.wait(l, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                job = job_;
            }
            (*job)(t);
            std::lock_guard<std::mutex> l(mu_);
            if (--left_ == 0) done_.notify_one();
        }
    }
    int n_;
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, done_;
    const std::function<void(int)>* job_ = nullptr;
    int left_ = 0;
    long gen_ = 0;
    bool stop_ = false;
};

// f(jb, je) over [j0, m) split into one range per pool thread; with `lower`
// the ranges hold equal shares of a lower trapezoid (column j has m - j
// entries), else equal numbers of columns.  Inline without a pool or when the
// work is small.
void forColumns(Pool* pool, int j0, int m, long long work, bool lower, const std::function<void(int, int)>& f) {
    const int T = pool ? pool->size() : 1;
    if (T == 1 || work < 100000 || m - j0 < 2 * T) { f(j0, m); return; }
    std::vector<int> cut(T + 1, m);
    cut[0] = j0;
    if (lower) {
        const double total = 0.5 * (double)(m - j0) * (m - j0 + 1);
        double acc = 0;
        int t = 1;
        for (int j = j0; j < m && t < T; ++j) {
            acc += m - j;
            while (t < T && acc >= total * t / T) cut[t++] = j + 1;
        }
    } else {
        for (int t = 1; t < T; ++t) cut[t] = j0 + (int)((long long)(m - j0) * t / T);
    }
    pool->run([&](int q) { if (cut[q] < cut[q + 1]) f(cut[q], cut[q + 1]); });
}

// Partial Cholesky of the first p columns of the m x m front F (column-major,
// lower triangle used): they become L11 and L21 and the trailing block the
// Schur complement.  Pivots go in panels of PANEL (inside a panel, sub-panels
// of SUB); a later column takes a panel's updates one pivot after another, so
// every entry sees the same sequence of roundings as in the column-by-column
// right-looking form, with or without the pool.  The trailing columns of each
// panel are split over the pool.
bool partialCholesky(double* F, int m, int p, Pool* pool) {
    for (int k0 = 0; k0 < p; k0 += PANEL) {
        const int kb = std::min(PANEL, p - k0);
        // the panel itself, by sub-panels
        for (int s0 = k0; s0 < k0 + kb; s0 += SUB) {
            const int sb = std::min(SUB, k0 + kb - s0);
            for (int k = s0; k < s0 + sb; ++k) {
                double* Fk = F + (size_t)k * m;
                double d = Fk[k];
                if (!(d > 0.0)) return false;
                d = std::sqrt(d);
                Fk[k] = d;
                for (int i = k + 1; i < m; ++i) Fk[i] /= d;
                for (int j = k + 1; j < s0 + sb; ++j) axpyMinus(F + (size_t)j * m + j, Fk + j, Fk[j], m - j);
            }
            panelTrailing(F, m, s0, sb, s0 + sb, k0 + kb);
        }
        const int j0 = k0 + kb;
        const long long work = (long long)kb * (m - j0) * (m - j0) / 2;
        forColumns(pool, j0, m, work, true, [&](int jb, int je) { panelTrailing(F, m, k0, kb, jb, je); });
    }
    return true;
}

}  // namespace

// the analysis of the last pattern: its rows and columns, the assembly tree
struct MultifrontalCache {
    std::vector<int> rowPtr, col;
    std::vector<Node> nodes;
    std::vector<int> roots, post;
};

namespace {

struct Factor {
    std::vector<int> idx;   // scalar indices of the front's rows
    std::vector<double> L;  // m x p, column-major (rows from the diagonal down used)
    int m = 0, p = 0;
};

class Multifrontal {
public:
    Multifrontal(const LinearSystem& ls, int nv, int threads, const double* xyz, MultifrontalCache* cache)
        : nv_(nv), threads_(std::max(1, threads)) {
        fullSymmetric(ls);
        if (cache && cache->rowPtr == ls.rowPtr && cache->col == ls.col) {
            nodes_ = cache->nodes;
            roots_ = cache->roots;
            post_ = cache->post;
            return;
        }
        Graph g = vertexGraph(ls, nv);
        Dissection d(g, xyz);
        std::vector<int> all(nv);
        for (int v = 0; v < nv; ++v) all[v] = v;
        roots_ = d.dissect(all);
        nodes_ = std::move(d.nodes);
        postorder();
        symbolic(g);
        if (cache) {
            cache->rowPtr = ls.rowPtr;
            cache->col = ls.col;
            cache->nodes = nodes_;
            cache->roots = roots_;
            cache->post = post_;
        }
    }

    void factor() {
        fac_.assign(nodes_.size(), Factor());
        upd_.assign(nodes_.size(), std::vector<double>());
        Pool pool(threads_);
        // independent subtrees (largest first), one per pool thread at a
        // time; then the nodes above them in post-order, each front split
        // over the pool by columns
        std::vector<char> top(nodes_.size(), 0);
        std::vector<int> sub = cutSubtrees(top);
        std::atomic<int> next(0);
        std::atomic<bool> bad(false);
        pool.run([&](int) {
            std::vector<int> loc(nv_, -1);
            for (int s; (s = next.fetch_add(1)) < (int)sub.size();) {
                std::vector<int> stack{sub[s]}, order;
                while (!stack.empty()) {
                    int n = stack.back();
                    stack.pop_back();
                    order.push_back(n);
                    for (int k : nodes_[n].kids) stack.push_back(k);
                }
                for (int i = (int)order.size() - 1; i >= 0 && !bad; --i)
                    if (!front(order[i], loc, nullptr)) bad = true;
            }
        });
        if (bad) throw std::runtime_error("oracle multifrontal solve: matrix is not positive definite");
        std::vector<int> loc(nv_, -1);
        for (int n : post_)
            if (top[n] && !front(n, loc, &pool)) throw std::runtime_error("oracle multifrontal solve: matrix is not positive definite");
    }

    // forward and backward substitution with the factor, in place on b
    void solve(std::vector<double>& b) const {
        for (int n : post_) {
            const Factor& f = fac_[n];
            for (int k = 0; k < f.p; ++k) {
                const double* Lk = f.L.data() + (size_t)k * f.m;
                double y = b[f.idx[k]] / Lk[k];
                b[f.idx[k]] = y;
                for (int i = k + 1; i < f.m; ++i) b[f.idx[i]] -= Lk[i] * y;
            }
        }
        for (int q = (int)post_.size() - 1; q >= 0; --q) {
            const Factor& f = fac_[post_[q]];
            for (int k = f.p - 1; k >= 0; --k) {
                const double* Lk = f.L.data() + (size_t)k * f.m;
                double s = b[f.idx[k]];
                for (int i = k + 1; i < f.m; ++i) s -= Lk[i] * b[f.idx[i]];
                b[f.idx[k]] = s / Lk[k];
            }
        }
    }

private:
    int nv_, threads_;
    std::vector<int> rp_, ci_;  // full symmetric scalar CSR
    std::vector<double> cv_;
    std::vector<Node> nodes_;
    std::vector<int> roots_, post_;
    std::vector<Factor> fac_;
    std::vector<std::vector<double>> upd_;

    void fullSymmetric(const LinearSystem& ls) {
        int n = 3 * nv_;
        std::vector<int> cnt(n, 0);
        for (int r = 0; r < n; ++r)
            for (int k = ls.rowPtr[r]; k < ls.rowPtr[r + 1]; ++k) { cnt[r]++; if (ls.col[k] != r) cnt[ls.col[k]]++; }
        rp_.assign(n + 1, 0);
        for (int r = 0; r < n; ++r) rp_[r + 1] = rp_[r] + cnt[r];
        ci_.assign(rp_[n], 0);
        cv_.assign(rp_[n], 0.0);
        std::vector<int> pos(rp_.begin(), rp_.end() - 1);
        for (int r = 0; r < n; ++r)
            for (int k = ls.rowPtr[r]; k < ls.rowPtr[r + 1]; ++k) {
                int c = ls.col[k];
                ci_[pos[r]] = c; cv_[pos[r]++] = ls.val[k];
                if (c != r) { ci_[pos[c]] = r; cv_[pos[c]++] = ls.val[k]; }
            }
    }

    void postorder() {
        post_.clear();
        std::vector<std::pair<int, size_t>> st;
        for (int r : roots_) {
            st.push_back({r, 0});
            while (!st.empty()) {
                auto& [n, i] = st.back();
                if (i < nodes_[n].kids.size()) {
                    int k = nodes_[n].kids[i++];
                    st.push_back({k, 0});
                } else {
                    post_.push_back(n);
                    st.pop_back();
                }
            }
        }
    }

    // elimination positions, then each front's row structure bottom-up
    void symbolic(const Graph& g) {
        std::vector<int> pos(nv_, -1);
        int c = 0;
        for (int n : post_)
            for (int v : nodes_[n].verts) pos[v] = c++;
        std::vector<int> tag(nv_, -1);
        for (int n : post_) {
            Node& N = nodes_[n];
            const int last = pos[N.verts.back()];
            auto add = [&](int u) {
                if (pos[u] > last && tag[u] != n) { tag[u] = n; N.rows.push_back(u); }
            };
            for (int v : N.verts)
                for (int k = g.ptr[v]; k < g.ptr[v + 1]; ++k) add(g.adj[k]);
            for (int k : N.kids)
                for (int u : nodes_[k].rows) add(u);
            std::sort(N.rows.begin(), N.rows.end(), [&](int a, int b) { return pos[a] < pos[b]; });
            const double m = 3.0 * (N.verts.size() + N.rows.size()), p = 3.0 * N.verts.size();
            N.work = p * m * m - p * p * m + p * p * p / 3.0;
            for (int k : N.kids) N.work += nodes_[k].work;
        }
    }

    // split the largest subtree until none holds more than an eighth of a
    // thread's share of the flops; the split nodes form the top of the tree
    std::vector<int> cutSubtrees(std::vector<char>& top) {
        std::vector<int> sub = roots_;
        double total = 0;
        for (int r : roots_) total += nodes_[r].work;
        const double limit = threads_ > 1 ? total / (8.0 * threads_) : total;
        while (!sub.empty()) {
            auto it = std::max_element(sub.begin(), sub.end(), [&](int a, int b) { return nodes_[a].work < nodes_[b].work; });
            int n = *it;
            if (nodes_[n].work <= limit || nodes_[n].kids.empty()) break;
            top[n] = 1;
            sub.erase(it);
            sub.insert(sub.end(), nodes_[n].kids.begin(), nodes_[n].kids.end());
        }
        std::stable_sort(sub.begin(), sub.end(), [&](int a, int b) { return nodes_[a].work > nodes_[b].work; });
        return sub;
    }

    // assemble, factorise and pass up one front; with a pool every phase is
    // split by columns (each column is written by one thread only)
    bool front(int n, std::vector<int>& loc, Pool* pool) {
        const Node& N = nodes_[n];
        const int nf = (int)(N.verts.size() + N.rows.size());
        const int m = 3 * nf, p = 3 * (int)N.verts.size();
        const size_t M = (size_t)m;
        Factor& f = fac_[n];
        f.m = m;
        f.p = p;
        f.idx.resize(m);
        for (int i = 0; i < nf; ++i) {
            int w = i < (int)N.verts.size() ? N.verts[i] : N.rows[i - N.verts.size()];
            loc[w] = i;
            for (int a = 0; a < 3; ++a) f.idx[3 * i + a] = 3 * w + a;
        }
        std::unique_ptr<double[]> Fbuf(new double[M * M]);
        double* F = Fbuf.get();
        forColumns(pool, 0, m, (long long)m * m, false, [&](int jb, int je) {
            std::fill(F + jb * M, F + je * M, 0.0);
            // original entries of the columns eliminated here (lower part only)
            for (int lc = jb; lc < std::min(je, p); ++lc) {
                const int c = f.idx[lc];
                double* Fc = F + lc * M;
                for (int k = rp_[c]; k < rp_[c + 1]; ++k) {
                    const int r = ci_[k], lu = loc[r / 3];
                    if (lu < 0) continue;
                    const int lr = 3 * lu + r % 3;
                    if (lr >= lc) Fc[lr] += cv_[k];
                }
            }
        });
        // children's update matrices, in the children's stored order
        std::vector<int> map;
        for (int k : N.kids) {
            const Node& K = nodes_[k];
            const int mk = 3 * (int)K.rows.size();
            map.resize(mk);
            for (int i = 0; i < mk; ++i) map[i] = 3 * loc[K.rows[i / 3]] + i % 3;
            const double* U = upd_[k].data();
            forColumns(pool, 0, mk, (long long)mk * mk / 2, true, [&](int jb, int je) {
                for (int j = jb; j < je; ++j) {
                    double* Fj = F + (size_t)map[j] * M;
                    const double* Uj = U + (size_t)j * mk;
                    for (int i = j; i < mk; ++i) Fj[map[i]] += Uj[i];
                }
            });
            std::vector<double>().swap(upd_[k]);
        }
        for (int i = 0; i < nf; ++i) loc[i < (int)N.verts.size() ? N.verts[i] : N.rows[i - N.verts.size()]] = -1;
        if (!partialCholesky(F, m, p, pool)) return false;
        const int mu = m - p;
        f.L.resize(M * p);
        std::vector<double>& U = upd_[n];
        U.resize((size_t)mu * mu);
        forColumns(pool, 0, m, (long long)m * m, false, [&](int jb, int je) {
            if (jb < p) std::copy(F + jb * M, F + std::min(je, p) * M, f.L.data() + jb * M);
            for (int j = std::max(jb, p); j < je; ++j)
                std::copy(F + j * M + j, F + (j + 1) * M, U.data() + (size_t)(j - p) * mu + (j - p));
        });
        return true;
    }
};

}  // namespace

std::shared_ptr<MultifrontalCache> newMultifrontalCache() { return std::make_shared<MultifrontalCache>(); }

void multifrontalSolve(LinearSystem& ls, int nv, int threads, const double* xyz, MultifrontalCache* cache) {
    if (nv <= 0) { ls.sol.clear(); return; }
    Multifrontal mf(ls, nv, threads, xyz, cache);
    mf.factor();
    ls.sol = ls.rhs;
    mf.solve(ls.sol);
}

}  // namespace oracle
