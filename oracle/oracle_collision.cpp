// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
// anything under oracle/; the shipped library never links it.
//
// Broad phase (LBVH), contact active sets with the exact AABB filter,
// additive CCD, ground and CFL step bounds and the edge-triangle
// intersection test.
#include "oracle_core.h"

#include <limits>
#include <map>
#include <stdexcept>

namespace oracle {

// ---------------------------------------------------------------------------
// LBVH, CPU IPC/LBVH.cpp:17-282
// ---------------------------------------------------------------------------
static uint32_t expandBits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}
static uint32_t morton(double x, double y, double z) {
    const double res = 1024.0;
    auto q = [&](double v) { v = std::max(0.0, std::min(v * res, res - 1.0)); return (uint32_t)v; };
    return (expandBits(q(x)) << 2) | (expandBits(q(y)) << 1) | expandBits(q(z));
}
static int clz64(uint64_t v) { return v == 0 ? 64 : __builtin_clzll(v); }
static int prefix(const std::vector<uint64_t>& k, int a, int b) {
    if (b < 0 || b >= (int)k.size()) return -1;
    return clz64(k[a] ^ k[b]);
}

void LBVH::build(const std::vector<AABB>& prims) {
    size_t n = prims.size();
    nodes.clear(); boxes.clear();
    if (n == 0) return;
    AABB scene;
    for (const AABB& b : prims) scene.combine(b);
    V3 ext = scene.hi - scene.lo;
    std::vector<std::pair<uint64_t, uint32_t>> ent(n);
    for (size_t p = 0; p < n; ++p) {
        V3 off = prims[p].center() - scene.lo;
        double x = ext.x > 0.0 ? off.x / ext.x : 0.0;
        double y = ext.y > 0.0 ? off.y / ext.y : 0.0;
        double z = ext.z > 0.0 ? off.z / ext.z : 0.0;
        ent[p] = {((uint64_t)morton(x, y, z) << 32) | p, (uint32_t)p};
    }
    std::sort(ent.begin(), ent.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    size_t nn = 2 * n - 1;
    nodes.assign(nn, Node{});
    boxes.assign(nn, AABB{});
    std::vector<uint64_t> keys(n);
    for (size_t s = 0; s < n; ++s) {
        keys[s] = ent[s].first;
        nodes[s + n - 1].prim = ent[s].second;
        boxes[s + n - 1] = prims[ent[s].second];
    }
    if (n == 1) return;
    int leafCount = (int)n;
    for (size_t in = 0; in < n - 1; ++in) {
        uint32_t first, last;
        int cur = (int)in;
        if (cur == 0) { first = 0; last = leafCount - 1; }
        else {
            int lp = prefix(keys, cur, cur - 1), rp = prefix(keys, cur, cur + 1);
            int dir = rp > lp ? 1 : -1;
            int minp = std::min(lp, rp);
            int maxLen = 2;
            while (prefix(keys, cur, cur + dir * maxLen) > minp) maxLen <<= 1;
            int len = 0;
            for (int step = maxLen >> 1; step > 0; step >>= 1)
                if (prefix(keys, cur, cur + dir * (len + step)) > minp) len += step;
            int other = cur + dir * len;
            first = std::min(cur, other); last = std::max(cur, other);
        }
        uint32_t split;
        uint64_t fc = keys[first], lc = keys[last];
        if (fc == lc) split = (first + last) >> 1;
        else {
            int common = clz64(fc ^ lc);
            split = first;
            uint32_t step = last - first;
            do {
                step = (step + 1) >> 1;
                uint32_t cand = split + step;
                if (cand < last && clz64(fc ^ keys[cand]) > common) split = cand;
            } while (step > 1);
        }
        uint32_t l = split, r = split + 1;
        if (split == first) l += leafCount - 1;
        if (split + 1 == last) r += leafCount - 1;
        nodes[in].left = l; nodes[in].right = r;
        nodes[l].parent = (uint32_t)in; nodes[r].parent = (uint32_t)in;
    }
    // post-order box merge
    std::vector<std::pair<uint32_t, bool>> st;
    st.emplace_back(0u, false);
    while (!st.empty()) {
        auto cur = st.back(); st.pop_back();
        const Node& nd = nodes[cur.first];
        if (nd.prim != 0xFFFFFFFFu) continue;
        if (cur.second) { boxes[cur.first] = boxes[nd.left]; boxes[cur.first].combine(boxes[nd.right]); }
        else { st.emplace_back(cur.first, true); st.emplace_back(nd.right, false); st.emplace_back(nd.left, false); }
    }
}

void LBVH::query(const AABB& box, double gap, std::vector<int>& out) const {
    out.clear();
    if (nodes.empty()) return;
    std::vector<uint32_t> st;
    st.push_back(0);
    while (!st.empty()) {
        uint32_t ni = st.back(); st.pop_back();
        if (!box.overlaps(boxes[ni], gap)) continue;
        const Node& nd = nodes[ni];
        if (nd.prim != 0xFFFFFFFFu) { out.push_back((int)nd.prim); continue; }
        if (st.size() + 2 > 128) throw std::runtime_error("CPU LBVH traversal stack overflow");
        st.push_back(nd.right); st.push_back(nd.left);
    }
    std::sort(out.begin(), out.end());
}

static AABB pointBox(const V3& p) { AABB b; b.combine(p); return b; }
static AABB edgeBox(const V3& a, const V3& b) { AABB r; r.combine(a); r.combine(b); return r; }
static AABB triBox(const V3& a, const V3& b, const V3& c) { AABB r; r.combine(a); r.combine(b); r.combine(c); return r; }
static AABB sweptPoint(const V3& p, const V3& d, double s) { AABB b; b.combine(p); b.combine(p - s * d); return b; }
static AABB sweptEdge(const V3& a, const V3& da, const V3& b, const V3& db, double s) {
    AABB r = sweptPoint(a, da, s); r.combine(sweptPoint(b, db, s)); return r;
}
static AABB sweptTri(const V3* p, const V3* d, double s) {
    AABB r;
    for (int k = 0; k < 3; ++k) r.combine(sweptPoint(p[k], d[k], s));
    return r;
}

// CPUBroadPhaseBVH::build / buildSwept, LBVH.cpp:284-339.
void BroadPhase::build(const Mesh& m) {
    faceBoxes.resize(m.surface.size());
    for (size_t f = 0; f < m.surface.size(); ++f)
        faceBoxes[f] = triBox(m.x[m.surface[f][0]], m.x[m.surface[f][1]], m.x[m.surface[f][2]]);
    edgeBoxes.resize(m.surfEdges.size());
    for (size_t e = 0; e < m.surfEdges.size(); ++e)
        edgeBoxes[e] = edgeBox(m.x[m.surfEdges[e].first], m.x[m.surfEdges[e].second]);
    sweptPointBoxes.clear();
    sweptQueryRadius = 0;
    faceTree.build(faceBoxes);
    edgeTree.build(edgeBoxes);
}

void BroadPhase::buildSwept(const Mesh& m, const std::vector<V3>& dir, double step) {
    sweptPointBoxes.resize(m.surfVerts.size());
    for (size_t s = 0; s < m.surfVerts.size(); ++s) {
        int v = m.surfVerts[s];
        sweptPointBoxes[s] = sweptPoint(m.x[v], dir[v], step);
    }
    faceBoxes.resize(m.surface.size());
    for (size_t f = 0; f < m.surface.size(); ++f) {
        V3 p[3], d[3];
        for (int k = 0; k < 3; ++k) { p[k] = m.x[m.surface[f][k]]; d[k] = dir[m.surface[f][k]]; }
        faceBoxes[f] = sweptTri(p, d, step);
    }
    edgeBoxes.resize(m.surfEdges.size());
    for (size_t e = 0; e < m.surfEdges.size(); ++e) {
        int a = m.surfEdges[e].first, b = m.surfEdges[e].second;
        edgeBoxes[e] = sweptEdge(m.x[a], dir[a], m.x[b], dir[b], step);
    }
    sweptQueryRadius = 0;
    faceTree.build(faceBoxes);
    edgeTree.build(edgeBoxes);
}

// ---------------------------------------------------------------------------
// Active sets, CollisionBroadPhase.cpp:765-1059 and 1076-1092
// ---------------------------------------------------------------------------
void calculateActiveSet(Mesh& m, BroadPhase& bp) {
    double sq = std::sqrt(m.Hhat);
    int ns = (int)m.surfVerts.size(), ne = (int)m.surfEdges.size();
    std::vector<std::vector<Contact>> csPT(ns), csEE(ne);
    std::vector<std::vector<int>> ccdPT(ns), ccdEE(ne);
    const auto& X = m.x;
    for (int svI = 0; svI < ns; ++svI) {
        int vI = m.surfVerts[svI];
        std::vector<int> tri;
        bp.faceTree.query(pointBox(X[vI]), sq, tri);
        AABB pb = pointBox(X[vI]);
        for (int sfI : tri) {
            const I4& f = m.surface[sfI];
            if (isCollider(m.btype[vI]) && isCollider(m.btype[f[0]]) && isCollider(m.btype[f[1]]) && isCollider(m.btype[f[2]])) continue;
            if (vI == f[0] || vI == f[1] || vI == f[2]) continue;
            if (!pb.overlaps(triBox(X[f[0]], X[f[1]], X[f[2]]), sq)) continue;
            ccdPT[svI].push_back(sfI);
            int t = dTypePT(X[vI], X[f[0]], X[f[1]], X[f[2]]);
            double d;
            switch (t) {
            case 0: d = dPP(X[vI], X[f[0]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[0], -1, -1); break;
            case 1: d = dPP(X[vI], X[f[1]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[1], -1, -1); break;
            case 2: d = dPP(X[vI], X[f[2]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[2], -1, -1); break;
            case 3: d = dPE(X[vI], X[f[0]], X[f[1]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[0], f[1], -1); break;
            case 4: d = dPE(X[vI], X[f[1]], X[f[2]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[1], f[2], -1); break;
            case 5: d = dPE(X[vI], X[f[2]], X[f[0]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[2], f[0], -1); break;
            case 6: d = dPT(X[vI], X[f[0]], X[f[1]], X[f[2]]); if (d < m.Hhat) csPT[svI].emplace_back(-vI - 1, f[0], f[1], f[2]); break;
            default: break;
            }
        }
    }
    for (int eI = 0; eI < ne; ++eI) {
        const I2& E = m.surfEdges[eI];
        std::vector<int> edges;
        bp.edgeTree.query(edgeBox(X[E.first], X[E.second]), sq, edges);
        edges.erase(std::remove_if(edges.begin(), edges.end(), [eI](int c) { return c <= eI; }), edges.end());
        AABB b1 = edgeBox(X[E.first], X[E.second]);
        for (int eJ : edges) {
            const I2& F = m.surfEdges[eJ];
            if (isCollider(m.btype[E.first]) && isCollider(m.btype[E.second]) && isCollider(m.btype[F.first]) && isCollider(m.btype[F.second])) continue;
            if (E.first == F.first || E.first == F.second || E.second == F.first || E.second == F.second || eI > eJ) continue;
            if (!b1.overlaps(edgeBox(X[F.first], X[F.second]), sq)) continue;
            ccdEE[eI].push_back(eJ);
            int t = dTypeEE(X[E.first], X[E.second], X[F.first], X[F.second]);
            double cs = crossSqNormEE(X[E.first], X[E.second], X[F.first], X[F.second]);
            double ex = epsX(m, E.first, E.second, F.first, F.second);
            int add_e = (cs < ex) ? -eJ - 2 : -1;
            double d;
            switch (t) {
            case 0: d = dPP(X[E.first], X[F.first]); if (d < m.Hhat) csEE[eI].emplace_back(-E.first - 1, F.first, -1, add_e); break;
            case 1: d = dPP(X[E.first], X[F.second]); if (d < m.Hhat) csEE[eI].emplace_back(-E.first - 1, F.second, -1, add_e); break;
            case 2: d = dPE(X[E.first], X[F.first], X[F.second]); if (d < m.Hhat) csEE[eI].emplace_back(-E.first - 1, F.first, F.second, add_e); break;
            case 3: d = dPP(X[E.second], X[F.first]); if (d < m.Hhat) csEE[eI].emplace_back(-E.second - 1, F.first, -1, add_e); break;
            case 4: d = dPP(X[E.second], X[F.second]); if (d < m.Hhat) csEE[eI].emplace_back(-E.second - 1, F.second, -1, add_e); break;
            case 5: d = dPE(X[E.second], X[F.first], X[F.second]); if (d < m.Hhat) csEE[eI].emplace_back(-E.second - 1, F.first, F.second, add_e); break;
            case 6: d = dPE(X[F.first], X[E.first], X[E.second]); if (d < m.Hhat) csEE[eI].emplace_back(-F.first - 1, E.first, E.second, add_e); break;
            case 7: d = dPE(X[F.second], X[E.first], X[E.second]); if (d < m.Hhat) csEE[eI].emplace_back(-F.second - 1, E.first, E.second, add_e); break;
            case 8:
                d = dEE(X[E.first], X[E.second], X[F.first], X[F.second]);
                if (d < m.Hhat) {
                    if (add_e <= -2) csEE[eI].emplace_back(E.first, E.second, F.first, -F.second - ne - 2);
                    else csEE[eI].emplace_back(E.first, E.second, F.first, F.second);
                }
                break;
            default: break;
            }
        }
    }
    m.selfCCD.clear();
    for (int s = 0; s < ns; ++s) for (int f : ccdPT[s]) m.selfCCD.push_back({-s - 1, f});
    for (int e = 0; e < ne; ++e) for (int f : ccdEE[e]) m.selfCCD.push_back({e, f});
    m.selfActive.clear();
    std::map<Contact, int> counter;
    for (const auto& cs : csPT)
        for (const Contact& c : cs) {
            if (c[3] < 0) ++counter[c];
            else m.selfActive.push_back(c);
        }
    m.selfEE.clear(); m.selfEEeIe.clear();
    for (int eI = 0; eI < ne; ++eI)
        for (const Contact& c : csEE[eI]) {
            if (c[3] >= 0) m.selfActive.push_back(c);
            else if (c[3] == -1) ++counter[c];
            else if (c[3] >= -ne - 1) {
                m.selfEE.emplace_back(c[0], c[1], c[2], -1);
                m.selfEEeIe.push_back({eI, -c[3] - 2});
            } else {
                m.selfEE.emplace_back(c[0], c[1], c[2], -c[3] - ne - 2);
                m.selfEEeIe.push_back({-1, -1});
            }
        }
    for (const auto& kv : counter) m.selfActive.emplace_back(kv.first[0], kv.first[1], kv.first[2], -kv.second);
}

// Ground::calculateActivateSet, CollisionBroadPhase.cpp:1076-1092 (kept in
// surface-vertex order; the reference appends under a mutex).
void groundActiveSet(Mesh& m) {
    m.envActive.clear();
    for (int v : m.surfVerts) {
        double dist = dot(m.groundN, m.x[v]) - m.groundD;
        if (dist * dist < m.Hhat) m.envActive.push_back(v);
    }
}

// buildCollisionSets, IPCSolver.cpp:544-556.
void buildCollisionSets(Mesh& m, BroadPhase& bp, bool rehash) {
    if (m.use_barrier) {
        if (rehash) bp.build(m);
        calculateActiveSet(m, bp);
    }
    groundActiveSet(m);
}

// ---------------------------------------------------------------------------
// Additive CCD, CPU IPC/AdditiveCCD.cpp:1-329
// ---------------------------------------------------------------------------
static double ptDistUnclassified(const V3& p, const V3& t0, const V3& t1, const V3& t2) {
    switch (dTypePT(p, t0, t1, t2)) {
    case 0: return dPP(p, t0);
    case 1: return dPP(p, t1);
    case 2: return dPP(p, t2);
    case 3: return dPE(p, t0, t1);
    case 4: return dPE(p, t1, t2);
    case 5: return dPE(p, t2, t0);
    case 6: return dPT(p, t0, t1, t2);
    default: return std::numeric_limits<double>::max();
    }
}
static double eeDistUnclassified(const V3& a0, const V3& a1, const V3& b0, const V3& b1) {
    switch (dTypeEE(a0, a1, b0, b1)) {
    case 0: return dPP(a0, b0);
    case 1: return dPP(a0, b1);
    case 2: return dPE(a0, b0, b1);
    case 3: return dPP(a1, b0);
    case 4: return dPP(a1, b1);
    case 5: return dPE(a1, b0, b1);
    case 6: return dPE(b0, a0, a1);
    case 7: return dPE(b1, a0, a1);
    case 8: return dEE(a0, a1, b0, b1);
    default: return std::numeric_limits<double>::max();
    }
}

double edgeEdgeCCD(V3 a0, V3 a1, V3 b0, V3 b1, V3 da0, V3 da1, V3 db0, V3 db1, double eta, double th) {
    V3 mov = (da0 + da1 + db0 + db1) / 4;
    da0 -= mov; da1 -= mov; db0 -= mov; db1 -= mov;
    double maxDisp = std::sqrt(std::max(sqnorm(da0), sqnorm(da1))) + std::sqrt(std::max(sqnorm(db0), sqnorm(db1)));
    if (maxDisp == 0) return 1.0;
    double d2 = eeDistUnclassified(a0, a1, b0, b1);
    double dF = d2 - th * th;
    if (dF <= 0) {
        d2 = std::min(std::min(sqnorm(a0 - b0), sqnorm(a0 - b1)), std::min(sqnorm(a1 - b0), sqnorm(a1 - b1)));
        dF = d2 - th * th;
    }
    double dc = std::sqrt(d2);
    double gap = eta * dF / (dc + th);
    double toc = 0.0;
    for (int it = 0; it < 10000; ++it) {
        double lb = (1 - eta) * dF / ((dc + th) * maxDisp);
        if (!std::isfinite(lb) || lb <= 0.0) return std::max(0.0, std::min(toc, 1.0));
        a0 += lb * da0; a1 += lb * da1; b0 += lb * db0; b1 += lb * db1;
        d2 = eeDistUnclassified(a0, a1, b0, b1);
        dF = d2 - th * th;
        if (dF <= 0) {
            d2 = std::min(std::min(sqnorm(a0 - b0), sqnorm(a0 - b1)), std::min(sqnorm(a1 - b0), sqnorm(a1 - b1)));
            dF = d2 - th * th;
        }
        dc = std::sqrt(d2);
        if (toc && (dF / (dc + th) < gap)) break;
        toc += lb;
        if (toc > 1.0) return 1.0;
    }
    return std::max(0.0, std::min(toc, 1.0));
}

double pointTriangleCCD(V3 p, V3 t0, V3 t1, V3 t2, V3 dp, V3 dt0, V3 dt1, V3 dt2, double eta, double th) {
    V3 mov = (dt0 + dt1 + dt2 + dp) / 4;
    dt0 -= mov; dt1 -= mov; dt2 -= mov; dp -= mov;
    double maxDisp = norm(dp) + std::sqrt(std::max(std::max(sqnorm(dt0), sqnorm(dt1)), sqnorm(dt2)));
    if (maxDisp == 0) return 1.0;
    double d2 = ptDistUnclassified(p, t0, t1, t2);
    double dc = std::sqrt(d2);
    double gap = eta * (d2 - th * th) / (dc + th);
    double toc = 0.0;
    for (int it = 0; it < 10000; ++it) {
        double lb = (1 - eta) * (d2 - th * th) / ((dc + th) * maxDisp);
        if (!std::isfinite(lb) || lb <= 0.0) return std::max(0.0, std::min(toc, 1.0));
        p += lb * dp; t0 += lb * dt0; t1 += lb * dt1; t2 += lb * dt2;
        d2 = ptDistUnclassified(p, t0, t1, t2);
        dc = std::sqrt(d2);
        if (toc && ((d2 - th * th) / (dc + th) < gap)) break;
        toc += lb;
        if (toc > 1.0) return 1.0;
    }
    return std::max(0.0, std::min(toc, 1.0));
}

// limitStepByGround, CPU IPC/FeasibleStep.cpp:8-40.
void limitStepByGround(const Mesh& m, const std::vector<V3>& dir, double slack, double& step) {
    if (m.surfVerts.empty()) return;
    double mn = std::numeric_limits<double>::infinity();
    for (int v : m.surfVerts) {
        double r = 1.0;
        double nm = dot(m.groundN, -dir[v]);
        if (nm < 0.0) {
            double dist = dot(m.groundN, m.x[v]) - m.groundD;
            double cand = -dist / nm * slack;
            if (cand >= 0.0) r = cand;
        }
        mn = std::min(mn, r);
    }
    step = std::min(step, mn);
}

// Self_largestFeasibleStepSize, ContactMechanics.cpp:3704-3752.
void selfLargestFeasibleStep(const Mesh& m, const std::vector<V3>& dir, double slack, double& step) {
    if (m.selfCCD.empty()) return;
    double ratio = 1.0 - slack;
    double mn = std::numeric_limits<double>::infinity();
    for (const I2& pr : m.selfCCD) {
        double a;
        if (pr.first < 0) {
            int pt = m.surfVerts[-pr.first - 1];
            const I4& f = m.surface[pr.second];
            a = pointTriangleCCD(m.x[pt], m.x[f[0]], m.x[f[1]], m.x[f[2]], -dir[pt], -dir[f[0]], -dir[f[1]], -dir[f[2]], ratio, 0.0);
        } else {
            const I2& e1 = m.surfEdges[pr.first];
            const I2& e2 = m.surfEdges[pr.second];
            a = edgeEdgeCCD(m.x[e1.first], m.x[e1.second], m.x[e2.first], m.x[e2.second],
                            -dir[e1.first], -dir[e1.second], -dir[e2.first], -dir[e2.second], ratio, 0.0);
        }
        mn = std::min(mn, a);
    }
    step = std::min(step, mn);
}

// Self_largestFeasibleStepSize_CCD, ContactMechanics.cpp:3754-3867.  The
// broad phase must have been built swept with the entry step.
void selfLargestFeasibleStepCCD(const Mesh& m, BroadPhase& bp, const std::vector<V3>& dir, double slack, double& step) {
    double ratio = 1.0 - slack;
    double ptStep = step;
    double mnPT = 1.0;
    bool anyPT = false;
    for (size_t s = 0; s < m.surfVerts.size(); ++s) {
        int vI = m.surfVerts[s];
        double best = 1.0;
        std::vector<int> tri;
        bp.faceTree.query(bp.sweptPointBoxes[s], bp.sweptQueryRadius, tri);
        AABB pb = sweptPoint(m.x[vI], dir[vI], ptStep);
        for (int sfI : tri) {
            const I4& f = m.surface[sfI];
            if (isCollider(m.btype[vI]) && isCollider(m.btype[f[0]]) && isCollider(m.btype[f[1]]) && isCollider(m.btype[f[2]])) continue;
            if (vI == f[0] || vI == f[1] || vI == f[2]) continue;
            V3 p[3] = {m.x[f[0]], m.x[f[1]], m.x[f[2]]}, d[3] = {dir[f[0]], dir[f[1]], dir[f[2]]};
            if (!pb.overlaps(sweptTri(p, d, ptStep))) continue;
            double a = pointTriangleCCD(m.x[vI], p[0], p[1], p[2], -dir[vI], -d[0], -d[1], -d[2], ratio, 0);
            best = std::min(a, best);
        }
        mnPT = anyPT ? std::min(mnPT, best) : best;
        anyPT = true;
    }
    if (anyPT) step = std::min(step, mnPT);
    double eeStep = step;
    double mnEE = 1.0;
    bool anyEE = false;
    for (int eJ = 0; eJ < (int)m.surfEdges.size(); ++eJ) {
        double best = 1.0;
        const I2& EJ = m.surfEdges[eJ];
        std::vector<int> cand;
        bp.edgeTree.query(bp.edgeBoxes[eJ], bp.sweptQueryRadius, cand);
        cand.erase(std::remove_if(cand.begin(), cand.end(), [eJ](int c) { return c <= eJ; }), cand.end());
        AABB b1 = sweptEdge(m.x[EJ.first], dir[EJ.first], m.x[EJ.second], dir[EJ.second], eeStep);
        for (int eI : cand) {
            const I2& EI = m.surfEdges[eI];
            if (isCollider(m.btype[EI.first]) && isCollider(m.btype[EI.second]) && isCollider(m.btype[EJ.first]) && isCollider(m.btype[EJ.second])) continue;
            if (EI.first == EJ.first || EI.first == EJ.second || EI.second == EJ.first || EI.second == EJ.second || eI < eJ) continue;
            AABB b2 = sweptEdge(m.x[EI.first], dir[EI.first], m.x[EI.second], dir[EI.second], eeStep);
            if (!b1.overlaps(b2)) continue;
            double a = edgeEdgeCCD(m.x[EI.first], m.x[EI.second], m.x[EJ.first], m.x[EJ.second],
                                   -dir[EI.first], -dir[EI.second], -dir[EJ.first], -dir[EJ.second], ratio, 0);
            best = std::min(a, best);
        }
        mnEE = anyEE ? std::min(mnEE, best) : best;
        anyEE = true;
    }
    if (anyEE) step = std::min(step, mnEE);
}

// IglUtils::segTriIntersect, ContactMechanics.h:47-71 (Cramer's rule stands
// in for the full-pivot LU solve of the same 3x3 system).  The reference skips
// coplanar pairs (coplanar contact is caught by the distances) but tests only
// exact signs and det == 0; with coplanarTol > 0 a segment whose two plane
// distances are both within coplanarTol of zero (relative to |n| times its
// reach from t0) is taken as coplanar too, so rounding on rotated meshes
// cannot report the edges and triangles of one flat face as intersecting.
// coplanarTol = 0 is the reference's rule exactly.
static bool segTriIntersect(const V3& e0, const V3& e1, const V3& t0, const V3& t1, const V3& t2, double coplanarTol) {
    V3 c0 = t1 - t0, c1 = t2 - t0, c2 = e0 - e1;
    V3 n = cross(c0, c1);
    const double d0 = dot(n, e0 - t0), d1 = dot(n, e1 - t0);
    if (d0 * d1 > 0.0) return false;
    if (coplanarTol > 0.0) {
        const double tol = coplanarTol * norm(n) * std::max(norm(e0 - t0), norm(e1 - t0));
        if (std::fabs(d0) <= tol && std::fabs(d1) <= tol) return false;
    }
    M3 A;
    for (int k = 0; k < 3; ++k) { A.a[k][0] = c0[k]; A.a[k][1] = c1[k]; A.a[k][2] = c2[k]; }
    double det = det3(A);
    if (det == 0.0) return false;
    V3 rhs = e0 - t0;
    M3 A0 = A, A1 = A, A2 = A;
    for (int k = 0; k < 3; ++k) { A0.a[k][0] = rhs[k]; A1.a[k][1] = rhs[k]; A2.a[k][2] = rhs[k]; }
    double u = det3(A0) / det, v = det3(A1) / det, t = det3(A2) / det;
    return u >= 0.0 && v >= 0.0 && u + v <= 1.0 && t >= 0.0 && t <= 1.0;
}

// isIntersected + checkEdgeTriIntersectionIfAny, IPCSolver.cpp:476-542.  The
// ground part only inspects the current environment active set, as in the
// reference.
bool isIntersected(const Mesh& m, BroadPhase& bp) {
    for (int v : m.envActive) {
        double dist = dot(m.groundN, m.x[v]) - m.groundD;
        if (dist * dist <= 0.0) return true;
    }
    for (size_t f = 0; f < m.surface.size(); ++f) {
        const I4& F = m.surface[f];
        std::vector<int> edges;
        bp.edgeTree.query(triBox(m.x[F[0]], m.x[F[1]], m.x[F[2]]), 0.0, edges);
        for (int e : edges) {
            const I2& E = m.surfEdges[e];
            if (E.first == F[0] || E.first == F[1] || E.first == F[2] || E.second == F[0] || E.second == F[1] || E.second == F[2]) continue;
            if (isCollider(m.btype[E.first]) && isCollider(m.btype[E.second]) && isCollider(m.btype[F[0]]) && isCollider(m.btype[F[1]]) && isCollider(m.btype[F[2]])) continue;
            if (segTriIntersect(m.x[E.first], m.x[E.second], m.x[F[0]], m.x[F[1]], m.x[F[2]], m.coplanarTol)) return true;
        }
    }
    return false;
}

}  // namespace oracle
