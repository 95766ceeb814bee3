// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
// anything under oracle/; the shipped library never links it.
//
// Newton linear system, line search, barrier sub-problem and time step
// (CPU IPC/NewtonLinearSystem.cpp, CPU IPC/IPCSolver.cpp).
#include "oracle_core.h"

#include <algorithm>
#include <deque>
#include <limits>
#include <stdexcept>

namespace oracle {

// BHessian::toTriplets + NewtonLinearSystem::assemble
// (ContactMechanics.cpp:12-134, NewtonLinearSystem.cpp:126-154): lower
// triangle, free vertices only, exact zeros dropped, duplicates summed, mass
// diagonal m(1+drag) on every DOF, right-hand side zeroed on non-free vertices.
void assembleSystem(const Mesh& m, const BHessian& BH, const std::vector<V3>& g, LinearSystem& ls) {
    int nv = m.nv(), n = 3 * nv;
    std::vector<std::vector<std::pair<int, double>>> rows(n);
    auto addBlock = [&](const int* vs, int np, const double* H) {
        int N = 3 * np;
        for (int a = 0; a < np; ++a) {
            int rv = vs[a];
            if (rv < 0 || rv >= nv || !isFree(m.btype[rv])) continue;
            for (int b = 0; b < np; ++b) {
                int cv = vs[b];
                if (cv < 0 || cv >= nv || !isFree(m.btype[cv])) continue;
                for (int rd = 0; rd < 3; ++rd)
                    for (int cd = 0; cd < 3; ++cd) {
                        int gr = 3 * rv + rd, gc = 3 * cv + cd;
                        double v = H[(3 * a + rd) * N + 3 * b + cd];
                        if (gr >= gc && v != 0.0) rows[gr].push_back({gc, v});
                    }
            }
        }
    };
    for (size_t i = 0; i < BH.H3.size(); ++i) addBlock(&BH.D1[i], 1, &BH.H3[i].a[0][0]);
    for (size_t i = 0; i < BH.H6.size(); ++i) addBlock(BH.D2[i].data(), 2, &BH.H6[i].a[0][0]);
    for (size_t i = 0; i < BH.H9.size(); ++i) addBlock(BH.D3[i].data(), 3, &BH.H9[i].a[0][0]);
    for (size_t i = 0; i < BH.H12.size(); ++i) addBlock(BH.D4[i].data(), 4, &BH.H12[i].a[0][0]);
    for (int d = 0; d < n; ++d) rows[d].push_back({d, m.mass[d / 3] * (1.0 + m.drag)});
    ls.rowPtr.assign(n + 1, 0);
    ls.col.clear(); ls.val.clear();
    for (int r = 0; r < n; ++r) {
        auto& R = rows[r];
        std::stable_sort(R.begin(), R.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t k = 0; k < R.size();) {
            size_t e = k;
            double s = 0;
            while (e < R.size() && R[e].first == R[k].first) { s += R[e].second; ++e; }
            ls.col.push_back(R[k].first);
            ls.val.push_back(s);
            k = e;
        }
        ls.rowPtr[r + 1] = (int)ls.col.size();
    }
    ls.nnz = (long long)ls.col.size();
    ls.rhs.assign(n, 0.0);
    for (int v = 0; v < nv; ++v)
        if (isFree(m.btype[v])) { ls.rhs[3 * v] = g[v].x; ls.rhs[3 * v + 1] = g[v].y; ls.rhs[3 * v + 2] = g[v].z; }
}

// Full symmetric scalar CSR from the lower CSR.
static void fullCSR(const LinearSystem& ls, std::vector<int>& rp, std::vector<int>& ci, std::vector<double>& cv) {
    int n = (int)ls.rowPtr.size() - 1;
    std::vector<int> cnt(n, 0);
    for (int r = 0; r < n; ++r)
        for (int k = ls.rowPtr[r]; k < ls.rowPtr[r + 1]; ++k) { cnt[r]++; if (ls.col[k] != r) cnt[ls.col[k]]++; }
    rp.assign(n + 1, 0);
    for (int r = 0; r < n; ++r) rp[r + 1] = rp[r] + cnt[r];
    ci.assign(rp[n], 0); cv.assign(rp[n], 0);
    std::vector<int> pos(rp.begin(), rp.end() - 1);
    for (int r = 0; r < n; ++r)
        for (int k = ls.rowPtr[r]; k < ls.rowPtr[r + 1]; ++k) {
            int c = ls.col[k];
            ci[pos[r]] = c; cv[pos[r]++] = ls.val[k];
            if (c != r) { ci[pos[c]] = r; cv[pos[c]++] = ls.val[k]; }
        }
}

// Direct solve: reverse Cuthill-McKee on the vertex graph, then an envelope
// Cholesky factorisation.  Exact to round-off like the reference's PARDISO.
static void directSolve(LinearSystem& ls, int nv) {
    int n = 3 * nv;
    std::vector<std::vector<int>> adj(nv);
    for (int r = 0; r < n; ++r)
        for (int k = ls.rowPtr[r]; k < ls.rowPtr[r + 1]; ++k) {
            int a = r / 3, b = ls.col[k] / 3;
            if (a != b) { adj[a].push_back(b); adj[b].push_back(a); }
        }
    for (auto& A : adj) { std::sort(A.begin(), A.end()); A.erase(std::unique(A.begin(), A.end()), A.end()); }
    std::vector<int> order;
    order.reserve(nv);
    std::vector<char> seen(nv, 0);
    std::vector<int> byDeg(nv);
    for (int i = 0; i < nv; ++i) byDeg[i] = i;
    std::stable_sort(byDeg.begin(), byDeg.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
    for (int s : byDeg) {
        if (seen[s]) continue;
        std::deque<int> q;
        q.push_back(s); seen[s] = 1;
        while (!q.empty()) {
            int u = q.front(); q.pop_front();
            order.push_back(u);
            std::vector<int> nb;
            for (int w : adj[u]) if (!seen[w]) { seen[w] = 1; nb.push_back(w); }
            std::stable_sort(nb.begin(), nb.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
            for (int w : nb) q.push_back(w);
        }
    }
    std::reverse(order.begin(), order.end());
    std::vector<int> perm(nv);
    for (int i = 0; i < nv; ++i) perm[order[i]] = i;
    std::vector<int> rp, ci;
    std::vector<double> cv;
    fullCSR(ls, rp, ci, cv);
    std::vector<int> first(n);
    for (int r = 0; r < n; ++r) {
        int pr = 3 * perm[r / 3] + r % 3;
        first[pr] = pr;
    }
    for (int r = 0; r < n; ++r) {
        int pr = 3 * perm[r / 3] + r % 3;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            int pc = 3 * perm[ci[k] / 3] + ci[k] % 3;
            if (pc < pr) first[pr] = std::min(first[pr], pc);
        }
    }
    std::vector<long long> off(n + 1, 0);
    for (int i = 0; i < n; ++i) off[i + 1] = off[i] + (i - first[i] + 1);
    std::vector<double> L(off[n], 0.0);
    for (int r = 0; r < n; ++r) {
        int pr = 3 * perm[r / 3] + r % 3;
        for (int k = rp[r]; k < rp[r + 1]; ++k) {
            int pc = 3 * perm[ci[k] / 3] + ci[k] % 3;
            if (pc <= pr) L[off[pr] + (pc - first[pr])] += cv[k];
        }
    }
    for (int i = 0; i < n; ++i) {
        double* Li = &L[off[i]];
        int fi = first[i];
        for (int j = fi; j < i; ++j) {
            double* Lj = &L[off[j]];
            int fj = first[j];
            int k0 = std::max(fi, fj);
            double s = Li[j - fi];
            for (int k = k0; k < j; ++k) s -= Li[k - fi] * Lj[k - fj];
            Li[j - fi] = s / Lj[j - fj];
        }
        double s = Li[i - fi];
        for (int k = fi; k < i; ++k) s -= Li[k - fi] * Li[k - fi];
        if (!(s > 0.0)) throw std::runtime_error("oracle direct solve: matrix is not positive definite");
        Li[i - fi] = std::sqrt(s);
    }
    std::vector<double> y(n);
    for (int r = 0; r < n; ++r) y[3 * perm[r / 3] + r % 3] = ls.rhs[r];
    for (int i = 0; i < n; ++i) {
        int fi = first[i];
        double s = y[i];
        for (int k = fi; k < i; ++k) s -= L[off[i] + k - fi] * y[k];
        y[i] = s / L[off[i] + i - fi];
    }
    for (int i = n - 1; i >= 0; --i) {
        int fi = first[i];
        y[i] /= L[off[i] + i - fi];
        double yi = y[i];
        for (int k = fi; k < i; ++k) y[k] -= L[off[i] + k - fi] * yi;
    }
    ls.sol.assign(n, 0.0);
    for (int r = 0; r < n; ++r) ls.sol[r] = y[3 * perm[r / 3] + r % 3];
}

// Block-Jacobi preconditioned CG with the stopping rule of Eigen's
// ConjugateGradient (NewtonLinearSystem.cpp:176-207): ||r||^2 <= tol^2 ||b||^2.
static void pcgSolve(LinearSystem& ls, int nv, double tol, int maxIter) {
    int n = 3 * nv;
    std::vector<int> rp, ci;
    std::vector<double> cv;
    fullCSR(ls, rp, ci, cv);
    std::vector<M3> Dinv(nv);
    for (int v = 0; v < nv; ++v) {
        M3 D;
        for (int a = 0; a < 3; ++a)
            for (int k = rp[3 * v + a]; k < rp[3 * v + a + 1]; ++k) {
                int c = ci[k];
                if (c / 3 == v) D.a[a][c % 3] += cv[k];
            }
        Dinv[v] = inverse3(D);
    }
    auto spmv = [&](const std::vector<double>& x, std::vector<double>& y) {
        for (int r = 0; r < n; ++r) {
            double s = 0;
            for (int k = rp[r]; k < rp[r + 1]; ++k) s += cv[k] * x[ci[k]];
            y[r] = s;
        }
    };
    auto prec = [&](const std::vector<double>& r, std::vector<double>& z) {
        for (int v = 0; v < nv; ++v)
            for (int a = 0; a < 3; ++a)
                z[3 * v + a] = Dinv[v].a[a][0] * r[3 * v] + Dinv[v].a[a][1] * r[3 * v + 1] + Dinv[v].a[a][2] * r[3 * v + 2];
    };
    auto dotv = [&](const std::vector<double>& a, const std::vector<double>& b) {
        double s = 0;
        for (int i = 0; i < n; ++i) s += a[i] * b[i];
        return s;
    };
    std::vector<double> x(n, 0.0), r = ls.rhs, z(n), p(n), t(n);
    double rhs2 = dotv(ls.rhs, ls.rhs);
    ls.pcgIters = 0;
    ls.sol.assign(n, 0.0);
    if (rhs2 == 0.0) { ls.pcgRelResidual = 0; return; }
    double thr = std::max(tol * tol * rhs2, std::numeric_limits<double>::min());
    double res2 = dotv(r, r);
    if (res2 < thr) { ls.pcgRelResidual = std::sqrt(res2 / rhs2); return; }
    prec(r, p);
    double absNew = dotv(r, p);
    int i = 0;
    while (i < maxIter) {
        spmv(p, t);
        double alpha = absNew / dotv(p, t);
        for (int k = 0; k < n; ++k) { x[k] += alpha * p[k]; r[k] -= alpha * t[k]; }
        res2 = dotv(r, r);
        if (res2 < thr) { ++i; break; }
        prec(r, z);
        double absOld = absNew;
        absNew = dotv(r, z);
        double beta = absNew / absOld;
        for (int k = 0; k < n; ++k) p[k] = z[k] + beta * p[k];
        ++i;
    }
    ls.pcgIters = i;
    ls.pcgRelResidual = std::sqrt(res2 / rhs2);
    if (!(res2 < thr)) throw std::runtime_error("oracle PCG did not converge within the iteration limit");
    ls.sol = x;
}

static_assert(sizeof(V3) == 3 * sizeof(double), "positions are passed as packed xyz triples");

void solveSystem(LinearSystem& ls, int nv, const SolverOptions& o, const double* xyz) {
    if (o.linear == 0) directSolve(ls, nv);
    else if (o.linear == 2) {
        if (!o.mfCache) o.mfCache = newMultifrontalCache();
        multifrontalSolve(ls, nv, o.threads, xyz, o.mfCache.get());
    }
    else pcgSolve(ls, nv, o.pcgRelTol, o.pcgMaxIter);
    for (double v : ls.sol)
        if (!std::isfinite(v)) throw std::runtime_error("linear solve produced a non-finite direction");
}

namespace {

double infNorm(const std::vector<V3>& d) {
    double mx = 0;
    for (const V3& v : d) for (int k = 0; k < 3; ++k) mx = std::max(mx, std::fabs(v[k]));
    return mx;
}

// stepForward, IPCSolver.cpp:458-473.
void stepForward(const std::vector<V3>& x0, const std::vector<V3>& dir, Mesh& m, double alpha, bool all = false) {
    for (int v = 0; v < m.nv(); ++v)
        if (isFree(m.btype[v]) || all) m.x[v] = x0[v] - alpha * dir[v];
}

// lineSearch, IPCSolver.cpp:560-749.
bool lineSearch(Mesh& m, BroadPhase& bp, const std::vector<V3>& dir, const std::vector<V3>& grad, double& alpha,
                double kappa, StepStats& st, const SolverOptions& o) {
    double E0 = computeEnergy(m, kappa, o);
    double gTp = 0;
    for (int v = 0; v < m.nv(); ++v) gTp += dot(grad[v], dir[v]);
    if (!std::isfinite(E0) || !std::isfinite(gTp)) throw std::runtime_error("line search received a non-finite energy or direction");
    std::vector<V3> x0 = m.x;
    stepForward(x0, dir, m, alpha);
    int nInter = 0;
    if (m.use_barrier) {
        bp.build(m);
        while (isIntersected(m, bp)) {
            if (nInter >= 64 || alpha <= std::numeric_limits<double>::epsilon())
                throw std::runtime_error("line search could not find a non-intersecting step");
            nInter++;
            alpha /= 2.0;
            stepForward(x0, dir, m, alpha);
            bp.build(m);
        }
    }
    buildCollisionSets(m, bp, false);
    double E = computeEnergy(m, kappa, o);
    int nLS = 0;
    const double LF = alpha;
    auto ok = [&](double e) { return std::isfinite(e) && e < E0; };
    while (!ok(E)) {
        if (nLS >= 64 || alpha <= std::numeric_limits<double>::epsilon() * std::max(1.0, LF)) {
            double thr = m.newtonThr * std::sqrt(m.bboxDiag2) * m.dt;
            if (infNorm(dir) < thr) {
                m.x = x0;
                buildCollisionSets(m, bp);
                st.energyBacktracks += nLS;
                st.intersectionBacktracks += nInter;
                st.backtracks += nInter + nLS;
                st.maxEnergyBacktracksPerNewton = std::max(st.maxEnergyBacktracksPerNewton, nLS);
                if (nLS > 2) ++st.newtonOverTwo;
                return false;
            }
            throw std::runtime_error("line search failed to find a strict energy decrease");
        }
        alpha *= 0.5;
        ++nLS;
        stepForward(x0, dir, m, alpha);
        buildCollisionSets(m, bp);
        E = computeEnergy(m, kappa, o);
    }
    if (alpha < LF) {
        bool recompute = false;
        if (m.use_barrier) {
            int it = 0;
            while (isIntersected(m, bp)) {
                if (it++ >= 64 || alpha <= std::numeric_limits<double>::epsilon())
                    throw std::runtime_error("backtracked step remains intersecting");
                alpha /= 2.0;
                nInter++;
                stepForward(x0, dir, m, alpha);
                bp.build(m);
                recompute = true;
            }
        }
        if (recompute) buildCollisionSets(m, bp, false);
    }
    st.energyBacktracks += nLS;
    st.intersectionBacktracks += nInter;
    st.backtracks += nInter + nLS;
    st.maxEnergyBacktracksPerNewton = std::max(st.maxEnergyBacktracksPerNewton, nLS);
    if (nLS > 2) ++st.newtonOverTwo;
    st.acceptedStepSum += alpha;
    st.minStep = std::min(st.minStep, alpha);
    st.maxStep = std::max(st.maxStep, alpha);
    return true;
}

// solveBarrierSubproblem, IPCSolver.cpp:890-1064.  `kappa` is the by-value copy
// of the reference: postLineSearch doubles it for the energy only, while the
// gradient and Hessian keep reading m.kappa.
int solveBarrierSubproblem(Mesh& m, BroadPhase& bp, double kappa, StepStats& st, const SolverOptions& o) {
    int k = 0;
    std::vector<V3> grad, dir(m.nv());
    BHessian BH;
    LinearSystem ls;
    double beta = 1;
    const int kmin = 6;
    for (; k < 10000; ++k) {
        BH.clear();
        st.collisions += computeGradientAndHessian(m, grad, BH, o);
        assembleSystem(m, BH, grad, ls);
        st.matrixNnz = std::max(st.matrixNnz, ls.nnz);
        solveSystem(ls, m.nv(), o, &m.x[0].x);
        st.pcgIterations += ls.pcgIters;
        ++st.linearSolves;
        for (int v = 0; v < m.nv(); ++v) dir[v] = V3(ls.sol[3 * v], ls.sol[3 * v + 1], ls.sol[3 * v + 2]);
        double thr = m.newtonThr * std::sqrt(m.bboxDiag2) * m.dt;
        if (infNorm(dir) < thr) break;
        double alpha = 1.0;
        limitStepByGround(m, dir, 0.8, alpha);
        if (alpha <= 0) alpha = 1;
        if (m.use_barrier) {
            double partial = alpha;
            selfLargestFeasibleStep(m, dir, 0.8, partial);
            double maxMove = 0.0;
            for (int v : m.surfVerts) maxMove = std::max(maxMove, norm(dir[v]));
            double aCFL = maxMove > 0.0 ? std::sqrt(m.Hhat) / (maxMove * 2.0) : 1.0;
            double full = alpha;
            bp.buildSwept(m, dir, full);
            selfLargestFeasibleStepCCD(m, bp, dir, 0.8, full);
            alpha = std::min(alpha, aCFL);
            if (partial > 2.0 * aCFL) {
                alpha = std::min(partial, full);
                alpha = std::max(alpha, aCFL);
            }
        }
        bool accepted = lineSearch(m, bp, dir, grad, alpha, kappa, st, o);
        if (!accepted) break;
        postLineSearch(m, kappa);
        if (k + 1 >= kmin) beta = (1 - alpha) * beta;
        if (beta <= thr) break;
    }
    st.newton += k;
    return k;
}

}  // namespace

// solveIPCStep, IPCSolver.cpp:1079-1336 (without file output).
int solveIPCStep(Mesh& m, BroadPhase& bp, StepStats& st, int stepIndex, const SolverOptions& o) {
    st = StepStats{};
    st.frame = stepIndex;
    upperBoundKappa(m.kappa, m.Hhat, m.bboxDiag2, m.meanMass);
    if (m.kappa < 1e-16) suggestKappa(m.kappa, m.Hhat, m.bboxDiag2, m.meanMass);
    initKappa(m, m.kappa);
    frictionInitialize(m);
    // soft targets (BoundaryConditions.cpp:112-135)
    if (!m.softIdx.empty() && m.softMotion != MOTION_NONE)
        for (size_t k = 0; k < m.softIdx.size(); ++k) {
            int v = m.softIdx[k];
            m.softTarget[k] = m.x[v] - motionDirection(m.softMotion, m.softRate, m.x[v], m.rest[v], 1.0, m.dt);
        }
    if (!m.dirIdx.empty() && m.dirMotion != MOTION_NONE) {
        auto dirs = [&](double frac, std::vector<V3>& d) {
            d.assign(m.nv(), V3());
            for (int v : m.dirIdx) d[v] = motionDirection(m.dirMotion, m.dirRate, m.x[v], m.rest[v], frac, m.dt);
        };
        std::vector<V3> d;
        double na = 1;
        dirs(na, d);
        bp.buildSwept(m, d, na);
        selfLargestFeasibleStepCCD(m, bp, d, 0.8, na);
        dirs(na, d);
        std::vector<V3> x0 = m.x;
        stepForward(x0, d, m, 1, true);
        bp.build(m);
        int ni = 0;
        while (isIntersected(m, bp)) {
            if (ni++ >= 64 || na <= std::numeric_limits<double>::epsilon())
                throw std::runtime_error("animated boundary update remains intersecting");
            na /= 2.0;
            m.x = x0;
            dirs(na, d);
            stepForward(x0, d, m, 1, true);
            bp.build(m);
        }
        buildCollisionSets(m, bp, false);
    }
    for (; st.kappaIters < 64; ++st.kappaIters) {
        m.closeID.clear(); m.closeMID.clear(); m.closeVal.clear(); m.closeMVal.clear();
        solveBarrierSubproblem(m, bp, m.kappa, st, o);
        std::vector<double> vals;
        for (int v : m.envActive) { double dist = dot(m.groundN, m.x[v]) - m.groundD; vals.push_back(dist * dist); }
        for (const Contact& c : m.selfActive) vals.push_back(selfConstraintVal(m, c));
        if (!vals.empty()) {
            double mn = *std::min_element(vals.begin(), vals.end());
            double mx = *std::max_element(vals.begin(), vals.end());
            st.minDist2 = mn;
            if (mn < m.dTol) break;
            else if (mx < m.Hhat) break;
        } else break;
    }
    if (st.kappaIters == 64) throw std::runtime_error("IPC kappa loop exceeded its iteration limit");
    ++st.kappaIters;
    for (int v = 0; v < m.nv(); ++v) m.vel[v] = m.quasi_static ? V3() : (m.x[v] - m.vprev[v]) / m.dt;
    m.vprev = m.x;
    updateInertialTarget(m);
    st.kappa = m.kappa;
    st.groundContacts = (long long)m.envActive.size();
    st.selfContacts = (long long)m.selfActive.size();
    st.mollifiedContacts = (long long)m.selfEE.size();
    return st.newton;
}

}  // namespace oracle
