// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
// anything under oracle/; the shipped library never links it.
//
// Physics terms: rest state, Stable Neo-Hookean, Baraff-Witkin cloth,
// quadratic bending, barrier contact with the EE mollifier, lagged friction,
// soft boundary penalty, energy and the kappa rules.  Each function cites the
// reference function it restates.
#include "oracle_core.h"

#include <cstdio>
#include <map>
#include <set>
#include <stdexcept>
#include <unordered_map>

namespace oracle {

void parallelFor(int n, int threads, const std::function<void(int, int)>& body) {
    if (n <= 0) return;
    if (threads <= 1 || n < 256) { body(0, n); return; }
    int t = std::min(threads, n);
    std::vector<std::thread> pool;
    int chunk = (n + t - 1) / t;
    for (int k = 0; k < t; ++k) {
        int b = k * chunk, e = std::min(n, b + chunk);
        if (b >= e) break;
        pool.emplace_back([&, b, e]() { body(b, e); });
    }
    for (auto& th : pool) th.join();
}

// ---------------------------------------------------------------------------
// Material and rest state
// ---------------------------------------------------------------------------

// updateMaterial, CPU IPC/Simulator.cpp:128-141.
void updateMaterial(Mesh& m) {
    double lengthRateLame = m.E / (2 * (1 + m.nu));
    double volumeRateLame = m.E * m.nu / ((1 + m.nu) * (1 - 2 * m.nu));
    m.lengthRate = 4 * lengthRateLame / 3;
    m.volumeRate = volumeRateLame + 5 * lengthRateLame / 6;
    m.stretchS = m.clothE / (1 - m.nu * m.nu);
    m.shearS = m.shearE / (2 * (1 + m.nu)) / m.thickness;
    m.plateRigidity = m.bendE * std::pow(m.thickness, 3) / (12 * (1 - m.nu * m.nu));
}

static M3 dsTet(const std::vector<V3>& x, const I4& t) {
    // calculateDms3D_double(..., 0), Elasticity.cpp:570-598: columns x1-x0, x2-x0, x3-x0.
    M3 M;
    for (int c = 0; c < 3; ++c) {
        V3 d = x[t[c + 1]] - x[t[0]];
        M.a[0][c] = d.x; M.a[1][c] = d.y; M.a[2][c] = d.z;
    }
    return M;
}

static double tetVolume(const std::vector<V3>& x, const I4& t) {
    // calculateVolum, Elasticity.cpp:535-563.
    V3 OA = x[t[1]] - x[t[0]], OB = x[t[2]] - x[t[0]], OC = x[t[3]] - x[t[0]];
    V3 h = cross(OA, OB);
    double bottom = norm(h);
    h = normalized(h);
    double v = bottom * std::fabs(dot(h, OC)) / 6;
    return v > 0 ? v : -v;
}

static Mat<2, 2> dmTri(const std::vector<V3>& x, const I3& t) {
    // calculateDms2D_double, Elasticity.cpp:610-640: rotate the normal to +y and
    // take (x, z) as the material coordinates.
    V3 v01 = x[t[1]] - x[t[0]], v02 = x[t[2]] - x[t[0]];
    V3 n = normalized(cross(v01, v02));
    V3 target(0, 1, 0);
    V3 vec = cross(n, target);
    double c = dot(n, target);
    M3 R = M3::identity(), K;
    K.a[0][1] = -vec.z; K.a[0][2] = vec.y;
    K.a[1][0] = vec.z; K.a[1][2] = -vec.x;
    K.a[2][0] = -vec.y; K.a[2][1] = vec.x;
    M3 K2 = mul(K, K);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R.a[i][j] += K.a[i][j] + K2.a[i][j] / (1 + c);
    auto rot = [&](const V3& p) {
        return V3(R.a[0][0] * p.x + R.a[0][1] * p.y + R.a[0][2] * p.z,
                  R.a[1][0] * p.x + R.a[1][1] * p.y + R.a[1][2] * p.z,
                  R.a[2][0] * p.x + R.a[2][1] * p.y + R.a[2][2] * p.z);
    };
    V3 r0 = rot(x[t[0]]), r1 = rot(x[t[1]]), r2 = rot(x[t[2]]);
    Mat<2, 2> M;
    M.a[0][0] = r1.x - r0.x; M.a[1][0] = r1.z - r0.z;
    M.a[0][1] = r2.x - r0.x; M.a[1][1] = r2.z - r0.z;
    return M;
}

// initMesh3D, CPU IPC/Elasticity.cpp:1050-1116.
void initRestState(Mesh& m) {
    int nv = m.nv();
    m.mass.assign(nv, 0.0);
    m.DmInv.clear(); m.vol.clear(); m.DmInv2.clear(); m.area.clear();
    double massSum = 0;
    for (size_t i = 0; i < m.tets.size(); ++i) {
        const I4& t = m.tets[i];
        M3 DM = dsTet(m.x, t);
        double vlm = tetVolume(m.x, t);
        for (int k = 0; k < 4; ++k) m.mass[t[k]] += vlm * m.density / 4;
        massSum += vlm * m.density;
        m.DmInv.push_back(inverse3(DM));
        m.vol.push_back(vlm);
    }
    for (size_t i = 0; i < m.tris.size(); ++i) {
        const I3& t = m.tris[i];
        Mat<2, 2> DM = dmTri(m.x, t);
        V3 v01 = m.x[t[1]] - m.x[t[0]], v02 = m.x[t[2]] - m.x[t[0]];
        double a = norm(cross(v01, v02)) * 0.5;
        a *= m.thickness;
        m.area.push_back(a);
        for (int k = 0; k < 3; ++k) m.mass[t[k]] += a * m.cloth_density / 3;
        massSum += a * m.cloth_density;
        double det = DM.a[0][0] * DM.a[1][1] - DM.a[0][1] * DM.a[1][0];
        Mat<2, 2> inv;
        inv.a[0][0] = DM.a[1][1] / det; inv.a[0][1] = -DM.a[0][1] / det;
        inv.a[1][0] = -DM.a[1][0] / det; inv.a[1][1] = DM.a[0][0] / det;
        m.DmInv2.push_back(inv);
    }
    m.meanMass = massSum / nv;
    if (m.tetLen.size() != m.tets.size()) m.tetLen.assign(m.tets.size(), m.lengthRate);
    if (m.tetVolR.size() != m.tets.size()) m.tetVolR.assign(m.tets.size(), m.volumeRate);
}

// prepareQuadraticBending, CPU IPC/Simulator.cpp:48-109.
void prepareQuadraticBending(Mesh& m) {
    m.bend.clear();
    std::unordered_map<int64_t, int> edgeMap;
    for (const I3& tri : m.tris) {
        for (int i = 0; i < 3; ++i) {
            int e0 = tri[i], e1 = tri[(i + 1) % 3];
            int other = tri[(i + 2) % 3];
            if (e0 > e1) std::swap(e0, e1);
            int64_t key = (int64_t(e0) << 32) | e1;
            auto it = edgeMap.find(key);
            if (it == edgeMap.end()) { edgeMap[key] = other; continue; }
            int o1 = it->second, o2 = other;
            V3 v0 = m.x[o1], v1 = m.x[e0], v2 = m.x[e1], v3 = m.x[o2];
            V3 E0 = v2 - v1, E1 = v0 - v1, E2 = v3 - v1, E3 = v0 - v2, E4 = v3 - v2;
            double a0 = 0.5 * norm(cross(E0, E1)), a1 = 0.5 * norm(cross(E0, E2));
            auto cot = [](const V3& p, const V3& q) { return dot(p, q) / norm(cross(p, q)); };
            double c01 = cot(E0, E1), c02 = cot(E0, E2), c03 = cot(-E0, E3), c04 = cot(-E0, E4);
            double K[4] = {c03 + c04, c01 + c02, -c01 - c03, -c02 - c04};
            QuadBend qb;
            qb.v[0] = e0; qb.v[1] = e1; qb.v[2] = o1; qb.v[3] = o2;
            double s = 3.0 / (a0 + a1);
            for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) qb.Q.a[a][b] = s * K[a] * K[b];
            m.bend.push_back(qb);
        }
    }
}

// Hinge list of prepareHingeBending (CPU IPC/Simulator.cpp:111-125) over the
// interior triangle edges of mesh3D::getSurface's edge pass
// (SimulationMesh.cpp:660-705): edges as (min, max) vertex pairs in
// lexicographic order, each with the opposite vertices of its two triangles
// in triangle order; edges on one triangle only carry no hinge.  Weight and
// rest angle follow makeHingeBendingInfo (HingeBending.cpp:45-73).
void prepareHingeBending(Mesh& m) {
    m.hinges.clear();
    std::map<std::pair<int, int>, std::vector<int>> opposite;
    for (const I3& tri : m.tris)
        for (int i = 0; i < 3; ++i) {
            int a = tri[i], b = tri[(i + 1) % 3];
            opposite[{std::min(a, b), std::max(a, b)}].push_back(tri[(i + 2) % 3]);
        }
    for (const auto& kv : opposite) {
        if (kv.second.size() != 2) continue;
        HingeBend hb;
        hb.v[0] = kv.first.first; hb.v[1] = kv.first.second; hb.v[2] = kv.second[0]; hb.v[3] = kv.second[1];
        // called at creation, while x holds the rest positions
        const V3 e = m.x[hb.v[1]] - m.x[hb.v[0]];
        const double l = norm(e);
        const double twiceAreas = norm(cross(e, m.x[hb.v[2]] - m.x[hb.v[0]])) + norm(cross(e, m.x[hb.v[3]] - m.x[hb.v[0]]));
        if (!std::isfinite(l) || !std::isfinite(twiceAreas) || l <= 0.0 || twiceAreas <= 0.0)
            throw std::runtime_error("degenerate rest hinge geometry");
        hb.weight = l * l / twiceAreas;
        hb.rest = hingeAngle(m.x[hb.v[0]], m.x[hb.v[1]], m.x[hb.v[2]], m.x[hb.v[3]], nullptr, nullptr);
        m.hinges.push_back(hb);
    }
}

// Signed dihedral angle about the edge x0 -> x1 between the normals
// n0 = e x (x2 - x0) and n1 = (x3 - x0) x e: zero when the two triangles are
// coplanar and unfolded.  The reference measures the same angle through
// LibShell::angle (Elasticity.cpp:29-150); any convention of the form
// +/- theta + const gives the same hinge energy, since only
// remainder(theta - rest, 2 pi) squared enters it.  Derivatives come from
// second-order jets over the 12 coordinates.
double hingeAngle(const V3& x0, const V3& x1, const V3& x2, const V3& x3, double* g, double* H) {
    typedef Jet<12> J;
    const JV3<12> p0 = jvar<12>(x0, 0), p1 = jvar<12>(x1, 3), p2 = jvar<12>(x2, 6), p3 = jvar<12>(x3, 9);
    const JV3<12> e = jsub(p1, p0);
    const JV3<12> n0 = jcross(e, jsub(p2, p0)), n1 = jcross(jsub(p3, p0), e);
    const J el = jsqrt(jdot(e, e));
    const J th = jatan2(jdot(jcross(n0, n1), e) / el, jdot(n0, n1));
    if (g)
        for (int i = 0; i < 12; ++i) g[i] = th.g[i];
    if (H)
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) H[12 * i + j] = th.h[i][j];
    return th.v;
}

// hingeBendingEnergy / hingeBendingGradientAndHessian (HingeBending.cpp:76-106)
// followed by makePD, as the assembly (IPCSolver.cpp:238-267) applies it.
double hingeEnergy(const HingeBend& hb, const std::vector<V3>& x, double k, double* g, double* H) {
    double tg[12], tH[144];
    const bool deriv = g || H;
    const double th = hingeAngle(x[hb.v[0]], x[hb.v[1]], x[hb.v[2]], x[hb.v[3]], deriv ? tg : nullptr, deriv ? tH : nullptr);
    const double d = std::remainder(th - hb.rest, 6.28318530717958647692);
    const double s = k * hb.weight;
    if (g)
        for (int i = 0; i < 12; ++i) g[i] = s * d * tg[i];
    if (H) {
        Mat<12, 12> M;
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) M.a[i][j] = s * (tg[i] * tg[j] + d * tH[12 * i + j]);
        makePD<12>(M);
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) H[12 * i + j] = M.a[i][j];
    }
    return 0.5 * s * d * d;
}

// mesh3D::getSurface, CPU IPC/SimulationMesh.cpp:364-446.  The reference walks
// an std::unordered_map, so the face order is the standard library's bucket
// order; the same container, hash and insertion sequence reproduce it.
namespace {
struct TriKey {
    uint64_t k[3];
    bool operator==(const TriKey& o) const { return k[0] == o.k[0] && k[1] == o.k[1] && k[2] == o.k[2]; }
};
}  // namespace

void getSurface(Mesh& m) {
    uint64_t length = (uint64_t)m.nv();
    auto hash = [&](const TriKey& t) { return length * (length * t.k[0] + t.k[1]) + t.k[2]; };
    int nt = (int)m.tets.size();
    std::unordered_map<TriKey, uint64_t, decltype(hash)> tri2Tet(4 * nt, hash);
    for (int i = 0; i < nt; ++i) {
        const I4& T = m.tets[i];
        for (int j = 0; j < 4; ++j) {
            uint64_t a = T[j % 4], b = T[(1 + j) % 4], c = T[(2 + j) % 4];
            TriKey perms[6] = {{{a, b, c}}, {{a, c, b}}, {{b, a, c}}, {{b, c, a}}, {{c, a, b}}, {{c, b, a}}};
            bool found = false;
            for (int p = 0; p < 6; ++p) {
                auto it = tri2Tet.find(perms[p]);
                if (it != tri2Tet.end()) { tri2Tet[perms[p]] = (uint64_t)nt + 1; found = true; break; }
            }
            if (!found) tri2Tet[perms[0]] = (uint64_t)i;
        }
    }
    m.surface.clear();
    for (const auto& kv : tri2Tet) {
        uint64_t tetId = kv.second;
        const TriKey& t = kv.first;
        if (tetId < (uint64_t)nt) {
            V3 vec1 = m.x[t.k[1]] - m.x[t.k[0]], vec2 = m.x[t.k[2]] - m.x[t.k[0]];
            int id3 = 0;
            for (int i = 0; i < 4; ++i) {
                int v = m.tets[tetId][i];
                if ((uint64_t)v != t.k[0] && (uint64_t)v != t.k[1] && (uint64_t)v != t.k[2]) { id3 = v; break; }
            }
            V3 vec3 = m.x[id3] - m.x[t.k[0]];
            V3 n = cross(vec1, vec2);
            if (dot(n, vec3) < 0)
                m.surface.push_back({(int)t.k[0], (int)t.k[1], (int)t.k[2], (int)tetId});
            else
                m.surface.push_back({(int)t.k[0], (int)t.k[2], (int)t.k[1], (int)tetId});
        }
    }
    for (const I3& tri : m.tris) m.surface.push_back({tri[0], tri[1], tri[2], 0});
    std::vector<char> flag(m.nv(), 0);
    m.surfVerts.clear();
    for (const I4& f : m.surface)
        for (int i = 0; i < 3; ++i)
            if (!flag[f[i]]) { m.surfVerts.push_back(f[i]); flag[f[i]] = 1; }
    std::set<std::pair<uint64_t, uint64_t>> edges;
    for (const I4& f : m.surface) {
        for (int i = 0; i < 3; ++i) {
            if (edges.find({(uint64_t)f[1], (uint64_t)f[0]}) == edges.end()) edges.insert({(uint64_t)f[0], (uint64_t)f[1]});
            if (edges.find({(uint64_t)f[2], (uint64_t)f[1]}) == edges.end()) edges.insert({(uint64_t)f[1], (uint64_t)f[2]});
            if (edges.find({(uint64_t)f[0], (uint64_t)f[2]}) == edges.end()) edges.insert({(uint64_t)f[2], (uint64_t)f[0]});
        }
    }
    m.surfEdges.clear();
    for (const auto& e : edges) m.surfEdges.push_back({(int)e.first, (int)e.second});
}

// updateInertialTarget, CPU IPC/IPCSolver.cpp:55-70.
void updateInertialTarget(Mesh& m) {
    double g = m.apply_gravity ? -9.8 : 0.0;
    V3 gdt2 = V3(0, g, 0) * m.dt * m.dt;
    m.xtilde.resize(m.nv());
    for (int i = 0; i < m.nv(); ++i) m.xtilde[i] = m.vprev[i] + m.vel[i] * m.dt + gdt2;
}

// ---------------------------------------------------------------------------
// Stable Neo-Hookean (Elasticity.cpp:1144-1170, 1337-1479, 695-727)
// ---------------------------------------------------------------------------

static M3 cofactor(const M3& F) {
    M3 p;
    p.a[0][0] = F.a[1][1] * F.a[2][2] - F.a[1][2] * F.a[2][1];
    p.a[0][1] = F.a[1][2] * F.a[2][0] - F.a[1][0] * F.a[2][2];
    p.a[0][2] = F.a[1][0] * F.a[2][1] - F.a[1][1] * F.a[2][0];
    p.a[1][0] = F.a[2][1] * F.a[0][2] - F.a[2][2] * F.a[0][1];
    p.a[1][1] = F.a[2][2] * F.a[0][0] - F.a[2][0] * F.a[0][2];
    p.a[1][2] = F.a[2][0] * F.a[0][1] - F.a[2][1] * F.a[0][0];
    p.a[2][0] = F.a[0][1] * F.a[1][2] - F.a[1][1] * F.a[0][2];
    p.a[2][1] = F.a[0][2] * F.a[1][0] - F.a[0][0] * F.a[1][2];
    p.a[2][2] = F.a[0][0] * F.a[1][1] - F.a[0][1] * F.a[1][0];
    return p;
}
static double frob2(const M3& F) {
    double s = 0;
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) s += F.a[i][j] * F.a[i][j];
    return s;
}

// computePEPF_StableNHK3D_2_double.  I2 = sum sigma^2 = ||F||_F^2 and the
// signed product of the rotation-aware singular values is det F.
M3 snhPK1(const M3& F, double u, double r) {
    double I3 = det3(F), I2 = frob2(F);
    M3 cof = cofactor(F), P;
    double a = u * (1 - 1 / (I2 + 1));
    double b = r * (I3 - 1 - u * 3 / (r * 4));
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) P.a[i][j] = a * F.a[i][j] + b * cof.a[i][j];
    return P;
}

// project_StabbleNHK_2_H_3D (the live closed-form branch) followed by makePD.
Mat<9, 9> snhHessian(const M3& F, double u, double r) {
    double I3 = det3(F), Ic = frob2(F);
    double mu = u, lambda = r;
    Vec<9> g1, gJ;
    V3 c0(F.a[0][0], F.a[1][0], F.a[2][0]), c1(F.a[0][1], F.a[1][1], F.a[2][1]), c2(F.a[0][2], F.a[1][2], F.a[2][2]);
    V3 cols[3] = {c0, c1, c2};
    for (int c = 0; c < 3; ++c) for (int k = 0; k < 3; ++k) g1[3 * c + k] = 2 * cols[c][k];
    V3 j0 = cross(c1, c2), j1 = cross(c2, c0), j2 = cross(c0, c1);
    V3 js[3] = {j0, j1, j2};
    for (int c = 0; c < 3; ++c) for (int k = 0; k < 3; ++k) gJ[3 * c + k] = js[c][k];
    auto hat = [](const V3& f) {
        M3 h;
        h.a[0][1] = -f.z; h.a[0][2] = f.y;
        h.a[1][0] = f.z; h.a[1][2] = -f.x;
        h.a[2][0] = -f.y; h.a[2][1] = f.x;
        return h;
    };
    M3 f0 = hat(c0), f1 = hat(c1), f2 = hat(c2);
    Mat<9, 9> HJ;
    auto put = [&](int bi, int bj, const M3& B, double s) {
        for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) HJ.a[3 * bi + i][3 * bj + j] = s * B.a[i][j];
    };
    put(0, 1, f2, -1); put(0, 2, f1, 1);
    put(1, 0, f2, 1); put(1, 2, f0, -1);
    put(2, 0, f1, -1); put(2, 1, f0, 1);
    double J = I3;
    double sI = (Ic * mu) / (2 * (Ic + 1));
    double sJ = lambda * (J - 1 - (3 * mu) / (4.0 * lambda));
    double sg = (mu / (2 * (Ic + 1) * (Ic + 1)));
    Mat<9, 9> H;
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j)
            H.a[i][j] = sI * (i == j ? 2.0 : 0.0) + sJ * HJ.a[i][j] + sg * g1[i] * g1[j] + lambda * gJ[i] * gJ[j];
    makePD<9>(H);
    return H;
}

// getObjEnergy_StableNHK2_3D energy density.
double snhEnergyDensity(const M3& F, double u, double r) {
    double I2 = frob2(F), I3 = det3(F);
    double t = I3 - 1 - 3 * u / 4 / r;
    return 0.5 * u * (I2 - 3) + 0.5 * r * t * t - 0.5 * u * std::log(I2 + 1);
}

// computePFPX3D_double, Elasticity.cpp:803-848 (9x12, column-major vec(F)).
static Mat<9, 12> pfpxTet(const M3& Di) {
    Mat<9, 12> P;
    double m = Di.a[0][0], n = Di.a[0][1], o = Di.a[0][2];
    double p = Di.a[1][0], q = Di.a[1][1], r = Di.a[1][2];
    double s = Di.a[2][0], t = Di.a[2][1], u = Di.a[2][2];
    double t1 = -(m + p + s), t2 = -(n + q + t), t3 = -(o + r + u);
    double rows[3][4] = {{t1, m, p, s}, {t2, n, q, t}, {t3, o, r, u}};
    for (int c = 0; c < 3; ++c)
        for (int k = 0; k < 3; ++k)
            for (int v = 0; v < 4; ++v) P.a[3 * c + k][3 * v + k] = rows[c][v];
    return P;
}

// computePFPX32D_double, Elasticity.cpp:851-897 (6x9).
static Mat<6, 9> pfpxTri(const Mat<2, 2>& Di) {
    Mat<6, 9> P;
    double s0 = Di.a[0][0] + Di.a[1][0], s1 = Di.a[0][1] + Di.a[1][1];
    double d0 = Di.a[0][0], d1 = Di.a[1][0], d2 = Di.a[0][1], d3 = Di.a[1][1];
    for (int k = 0; k < 3; ++k) {
        P.a[k][k] = -s0; P.a[3 + k][k] = -s1;
        P.a[k][3 + k] = d0; P.a[3 + k][3 + k] = d2;
        P.a[k][6 + k] = d1; P.a[3 + k][6 + k] = d3;
    }
    return P;
}

static M3 tetF(const std::vector<V3>& x, const I4& t, const M3& Di) { return mul(dsTet(x, t), Di); }

// ---------------------------------------------------------------------------
// Baraff-Witkin membrane (Elasticity.cpp:1174-1205, 1481-1544, 729-771)
// ---------------------------------------------------------------------------
using M32 = Mat<3, 2>;

static M32 bwPK1(const M32& F, double stretchS, double shearS, double s) {
    V3 f0(F.a[0][0], F.a[1][0], F.a[2][0]), f1(F.a[0][1], F.a[1][1], F.a[2][1]);
    double I6 = dot(f0, f1);
    double I5u = dot(f0, f0), I5v = dot(f1, f1);
    double uc = 1.0 - 1 / std::sqrt(I5u), vc = 1.0 - 1 / std::sqrt(I5v);
    if (I5u > 1) uc += 1.5 * s * (std::sqrt(I5u) + 1 / std::sqrt(I5u) - 2);
    if (I5v > 1) vc += 1.5 * s * (std::sqrt(I5v) + 1 / std::sqrt(I5v) - 2);
    M32 P;
    for (int k = 0; k < 3; ++k) {
        double st0 = uc * 2. * f0[k], st1 = vc * 2. * f1[k];
        double sh0 = 2 * (I6 - 0.0) * f1[k], sh1 = 2 * (I6 - 0.0) * f0[k];
        P.a[k][0] = stretchS * st0 + shearS * sh0;
        P.a[k][1] = stretchS * st1 + shearS * sh1;
    }
    return P;
}

static Mat<6, 6> bwHessian(const M32& F, double stretchS, double shearS, double s) {
    Mat<6, 6> finalH;
    V3 f0(F.a[0][0], F.a[1][0], F.a[2][0]), f1(F.a[0][1], F.a[1][1], F.a[2][1]);
    {
        Mat<6, 6> H;
        double I5u = dot(f0, f0), I5v = dot(f1, f1);
        double su = std::sqrt(I5u), sv = std::sqrt(I5v);
        if (su > 1) { double d = 2 * (((su - 1) * (3 * su * s - 3 * s + 2)) / (2 * su)); for (int k = 0; k < 3; ++k) H.a[k][k] = d; }
        if (sv > 1) { double d = 2 * (((sv - 1) * (3 * sv * s - 3 * s + 2)) / (2 * sv)); for (int k = 0; k < 3; ++k) H.a[3 + k][3 + k] = d; }
        V3 fu = normalized(f0), fv = normalized(f1);
        double uC = (su > 1.0) ? (3 * I5u * s - 3 * s + 2) / (std::sqrt(I5u)) : 2.0;
        double vC = (sv > 1.0) ? (3 * I5v * s - 3 * s + 2) / (std::sqrt(I5v)) : 2.0;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                H.a[i][j] += uC * (fu[i] * fu[j]);
                H.a[3 + i][3 + j] += vC * (fv[i] * fv[j]);
            }
        addScaled(finalH, H, stretchS);
    }
    {
        Mat<6, 6> Hs;
        for (int k = 0; k < 3; ++k) { Hs.a[3 + k][k] = 1.0; Hs.a[k][3 + k] = 1.0; }
        double I6 = dot(f0, f1);
        double sign = I6 >= 0 ? 1.0 : -1.0;
        Vec<6> g;
        for (int k = 0; k < 3; ++k) { g[k] = f1[k]; g[3 + k] = f0[k]; }
        double I2 = dot(f0, f0) + dot(f1, f1);
        double l0 = 0.5 * (I2 + std::sqrt(I2 * I2 + 12.0 * I6 * I6));
        Vec<6> Hg = mulv(Hs, g), q0;
        double qn = 0;
        for (int k = 0; k < 6; ++k) { q0[k] = I6 * Hg[k] + l0 * g[k]; qn += q0[k] * q0[k]; }
        qn = std::sqrt(qn);
        if (qn > 0) for (int k = 0; k < 6; ++k) q0[k] /= qn;
        Mat<6, 6> T;
        for (int i = 0; i < 6; ++i) for (int j = 0; j < 6; ++j) T.a[i][j] = 0.5 * ((i == j ? 1.0 : 0.0) + sign * Hs.a[i][j]);
        Vec<6> Tq = mulv(T, q0);
        double nTq = 0;
        for (int k = 0; k < 6; ++k) nTq += Tq[k] * Tq[k];
        Mat<6, 6> Hsh;
        for (int i = 0; i < 6; ++i)
            for (int j = 0; j < 6; ++j)
                Hsh.a[i][j] = 2 * (std::fabs(I6) * (T.a[i][j] - (Tq[i] * Tq[j]) / nTq) + l0 * (q0[i] * q0[j]));
        addScaled(finalH, Hsh, shearS);
    }
    return finalH;
}

static double bwEnergyDensity(const M32& F, double stretchS, double shearS, double s) {
    V3 f0(F.a[0][0], F.a[1][0], F.a[2][0]), f1(F.a[0][1], F.a[1][1], F.a[2][1]);
    double I6 = dot(f0, f1);
    double shear = I6 * I6;
    double I5u = norm(f0), I5v = norm(f1);
    double uc = I5u <= 1 ? 0 : 1, vc = I5v <= 1 ? 0 : 1;
    double st = std::pow(I5u - 1, 2) + uc * s * std::pow(I5u - 1, 3) + std::pow(I5v - 1, 2) + vc * s * std::pow(I5v - 1, 3);
    return stretchS * st + shearS * shear;
}

static M32 triF(const std::vector<V3>& x, const I3& t, const Mat<2, 2>& Di) {
    M32 Ds;
    V3 a = x[t[1]] - x[t[0]], b = x[t[2]] - x[t[0]];
    for (int k = 0; k < 3; ++k) { Ds.a[k][0] = a[k]; Ds.a[k][1] = b[k]; }
    return mul(Ds, Di);
}

// ---------------------------------------------------------------------------
// Distances, classification, barrier (ContactMechanics.cpp:143-316, 678-813)
// ---------------------------------------------------------------------------

// Explicit solve of a 2x2 symmetric system; stands in for the 2x2 ldlt()
// solves of the reference (same solution up to round-off).
static inline void solve2(double m00, double m01, double m11, double r0, double r1, double& x0, double& x1) {
    double det = m00 * m11 - m01 * m01;
    x0 = (m11 * r0 - m01 * r1) / det;
    x1 = (m00 * r1 - m01 * r0) / det;
}

static inline void ptParam(const V3& r0, const V3& nvec, const V3& w, double& p0, double& p1) {
    V3 r1 = cross(r0, nvec);
    solve2(dot(r0, r0), dot(r0, r1), dot(r1, r1), dot(r0, w), dot(r1, w), p0, p1);
}

// dType_PT, ContactMechanics.cpp:143-193.
int dTypePT(const V3& v0, const V3& v1, const V3& v2, const V3& v3) {
    V3 nvec = cross(v2 - v1, v3 - v1);
    double a0, b0, a1, b1, a2, b2;
    ptParam(v2 - v1, nvec, v0 - v1, a0, b0);
    if (a0 > 0.0 && a0 < 1.0 && b0 >= 0.0) return 3;
    ptParam(v3 - v2, nvec, v0 - v2, a1, b1);
    if (a1 > 0.0 && a1 < 1.0 && b1 >= 0.0) return 4;
    ptParam(v1 - v3, nvec, v0 - v3, a2, b2);
    if (a2 > 0.0 && a2 < 1.0 && b2 >= 0.0) return 5;
    if (a0 <= 0.0 && a2 >= 1.0) return 0;
    if (a1 <= 0.0 && a0 >= 1.0) return 1;
    if (a2 <= 0.0 && a1 >= 1.0) return 2;
    return 6;
}

// dType_EE, ContactMechanics.cpp:195-280.
int dTypeEE(const V3& v0, const V3& v1, const V3& v2, const V3& v3) {
    V3 u = v1 - v0, v = v3 - v2, w = v0 - v2;
    double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), e = dot(v, w);
    double D = a * c - b * b;
    double tD = D, sN, tN;
    int defaultCase = 8;
    sN = (b * e - c * d);
    if (sN <= 0.0) { tN = e; tD = c; defaultCase = 2; }
    else if (sN >= D) { tN = e + b; tD = c; defaultCase = 5; }
    else {
        tN = (a * e - b * d);
        V3 uv = cross(u, v);
        if (tN > 0.0 && tN < tD && (dot(uv, w) == 0.0 || sqnorm(uv) < 1.0e-20 * a * c)) {
            if (sN < D / 2) { tN = e; tD = c; defaultCase = 2; }
            else { tN = e + b; tD = c; defaultCase = 5; }
        }
    }
    if (tN <= 0.0) {
        if (-d <= 0.0) return 0;
        else if (-d >= a) return 3;
        else return 6;
    } else if (tN >= tD) {
        if ((-d + b) <= 0.0) return 1;
        else if ((-d + b) >= a) return 4;
        else return 7;
    }
    return defaultCase;
}

double dPP(const V3& a, const V3& b) { return sqnorm(a - b); }
double dPE(const V3& p, const V3& e0, const V3& e1) { return sqnorm(cross(e0 - p, e1 - p)) / sqnorm(e1 - e0); }
double dPT(const V3& p, const V3& t0, const V3& t1, const V3& t2) {
    V3 b = cross(t1 - t0, t2 - t0);
    double aTb = dot(p - t0, b);
    return aTb * aTb / sqnorm(b);
}
double dEE(const V3& a0, const V3& a1, const V3& b0, const V3& b1) {
    V3 b = cross(a1 - a0, b1 - b0);
    double aTb = dot(b0 - a0, b);
    return aTb * aTb / sqnorm(b);
}
double crossSqNormEE(const V3& a0, const V3& a1, const V3& b0, const V3& b1) { return sqnorm(cross(a1 - a0, b1 - b0)); }

// compute_b / compute_g_b / compute_H_b, ContactMechanics.cpp:775-790.
void barrier(double d, double dHat, double& b) { b = -(d - dHat) * (d - dHat) * std::log(d / dHat); }
void barrierG(double d, double dHat, double& g) {
    double t = d - dHat;
    g = t * std::log(d / dHat) * -2.0 - (t * t) / d;
}
void barrierH(double d, double dHat, double& h) {
    double t = d - dHat;
    h = (std::log(d / dHat) * -2.0 - t * 4.0 / d) + 1.0 / (d * d) * (t * t);
}

template <int N>
static void jetOut(const Jet<N>& j, double* g, double* H) {
    for (int i = 0; i < N; ++i) g[i] = j.g[i];
    if (H) for (int i = 0; i < N; ++i) for (int k = 0; k < N; ++k) H[i * N + k] = j.h[i][k];
}

// Exact derivatives of the squared distances (stand-ins for the generated
// g_/H_ functions, ContactMechanics.cpp:792-2476).
void distanceGradHess(int kind, const V3* p, double* g, double* H) {
    switch (kind) {
    case 0: {
        // g_PP / H_PP, ContactMechanics.cpp:792-805
        V3 d = p[0] - p[1];
        V3 d2 = 2.0 * d;
        for (int k = 0; k < 3; ++k) { g[k] = d2[k]; g[3 + k] = -d2[k]; }
        if (H) {
            for (int i = 0; i < 36; ++i) H[i] = 0;
            for (int k = 0; k < 6; ++k) H[k * 6 + k] = 2.0;
            for (int k = 0; k < 3; ++k) { H[k * 6 + 3 + k] = -2.0; H[(3 + k) * 6 + k] = -2.0; }
        }
        return;
    }
    case 1: {
        auto v0 = jvar<9>(p[0], 0), v1 = jvar<9>(p[1], 3), v2 = jvar<9>(p[2], 6);
        auto c = jcross(jsub(v1, v0), jsub(v2, v0));
        auto e = jsub(v2, v1);
        jetOut<9>(jdot(c, c) / jdot(e, e), g, H);
        return;
    }
    case 2: {
        auto v0 = jvar<12>(p[0], 0), v1 = jvar<12>(p[1], 3), v2 = jvar<12>(p[2], 6), v3 = jvar<12>(p[3], 9);
        auto b = jcross(jsub(v2, v1), jsub(v3, v1));
        auto aTb = jdot(jsub(v0, v1), b);
        jetOut<12>((aTb * aTb) / jdot(b, b), g, H);
        return;
    }
    case 3: {
        auto v0 = jvar<12>(p[0], 0), v1 = jvar<12>(p[1], 3), v2 = jvar<12>(p[2], 6), v3 = jvar<12>(p[3], 9);
        auto b = jcross(jsub(v1, v0), jsub(v3, v2));
        auto aTb = jdot(jsub(v2, v0), b);
        jetOut<12>((aTb * aTb) / jdot(b, b), g, H);
        return;
    }
    default: {
        auto v0 = jvar<12>(p[0], 0), v1 = jvar<12>(p[1], 3), v2 = jvar<12>(p[2], 6), v3 = jvar<12>(p[3], 9);
        auto c = jcross(jsub(v1, v0), jsub(v3, v2));
        jetOut<12>(jdot(c, c), g, H);
        return;
    }
    }
}
void crossSqNormGradHess(const V3* p, double* g, double* H) { distanceGradHess(4, p, g, H); }

// SelfConstraintVal, ContactMechanics.cpp:2478-2503.
double selfConstraintVal(const Mesh& m, const Contact& c) {
    const auto& x = m.x;
    if (c[0] >= 0) return dEE(x[c[0]], x[c[1]], x[c[2]], x[c[3]]);
    int v0 = -c[0] - 1;
    if (c[2] < 0) return dPP(x[v0], x[c[1]]);
    if (c[3] < 0) return dPE(x[v0], x[c[1]], x[c[2]]);
    return dPT(x[v0], x[c[1]], x[c[2]], x[c[3]]);
}

// compute_eps_x, ContactMechanics.cpp:758-762 (rest positions).
double epsX(const Mesh& m, int a0, int a1, int b0, int b1) {
    return 1e-3 * sqnorm(m.rest[a0] - m.rest[a1]) * sqnorm(m.rest[b0] - m.rest[b1]);
}

// Mollifier e(x) and its derivatives, ContactMechanics.cpp:678-756.
static void mollifier(const V3* p, double epsx, double& e, double* eg, double* eH) {
    double c = crossSqNormEE(p[0], p[1], p[2], p[3]);
    if (c < epsx) {
        double q = c / epsx;
        e = (-q + 2.0) * q;
        if (eg || eH) {
            double g[12], H[144];
            crossSqNormGradHess(p, g, eH ? H : nullptr);
            double one = 1.0 / epsx;
            double qg = 2.0 * one * (-one * c + 1.0);
            double qH = -2.0 / (epsx * epsx);
            if (eg) for (int i = 0; i < 12; ++i) eg[i] = qg * g[i];
            if (eH) for (int i = 0; i < 12; ++i) for (int j = 0; j < 12; ++j) eH[i * 12 + j] = H[i * 12 + j] * qg + (qH * g[i]) * g[j];
        }
    } else {
        e = 1.0;
        if (eg) for (int i = 0; i < 12; ++i) eg[i] = 0;
        if (eH) for (int i = 0; i < 144; ++i) eH[i] = 0;
    }
}

// ---------------------------------------------------------------------------
// Contact gradient / Hessian (ContactMechanics.cpp:2970-3080, 3466-3700)
// ---------------------------------------------------------------------------

static void contactPoints(const Mesh& m, const Contact& c, int& kind, int idx[4], int& npts) {
    if (c[0] >= 0) { kind = 3; idx[0] = c[0]; idx[1] = c[1]; idx[2] = c[2]; idx[3] = c[3]; npts = 4; return; }
    idx[0] = -c[0] - 1; idx[1] = c[1];
    if (c[2] < 0) { kind = 0; npts = 2; return; }
    idx[2] = c[2];
    if (c[3] < 0) { kind = 1; npts = 3; return; }
    idx[3] = c[3]; kind = 2; npts = 4;
}

// compute_g_dpt: gradient of coef * input[i] * d(x) (x multiplicity for PP/PE).
static int gDPT(const Mesh& m, const std::vector<Contact>& set, const std::vector<double>& input, int offset,
                std::vector<V3>& out, double coef) {
    int ci = offset, count = 0;
    for (const Contact& c : set) {
        int kind, idx[4], np;
        contactPoints(m, c, kind, idx, np);
        V3 p[4];
        for (int k = 0; k < np; ++k) p[k] = m.x[idx[k]];
        double g[12];
        distanceGradHess(kind, p, g, nullptr);
        double s;
        if (kind == 3 || kind == 2) { s = coef * input[ci]; count++; }
        else { s = coef * -c[3] * input[ci]; count += -c[3]; }
        for (int k = 0; k < np; ++k) out[idx[k]] += V3(g[3 * k] * s, g[3 * k + 1] * s, g[3 * k + 2] * s);
        ++ci;
    }
    return count;
}

template <int N>
static Mat<N, N> toMat(const double* H) {
    Mat<N, N> M;
    for (int i = 0; i < N; ++i) for (int j = 0; j < N; ++j) M.a[i][j] = H[i * N + j];
    return M;
}

static void hDPT(const Mesh& m, BHessian& BH, double dHat, double coef) {
    for (const Contact& c : m.selfActive) {
        int kind, idx[4], np;
        contactPoints(m, c, kind, idx, np);
        V3 p[4];
        for (int k = 0; k < np; ++k) p[k] = m.x[idx[k]];
        double d = selfConstraintVal(m, c);
        double g[12], H[144];
        distanceGradHess(kind, p, g, H);
        double gb, hb;
        barrierG(d, dHat, gb);
        barrierH(d, dHat, hb);
        double cf = (kind == 0 || kind == 1) ? coef * -c[3] : coef;
        int n = 3 * np;
        double a = cf * hb, b = cf * gb;
        std::vector<double> M(n * n);
        for (int i = 0; i < n; ++i) for (int j = 0; j < n; ++j) M[i * n + j] = (a * g[i]) * g[j] + b * H[i * n + j];
        if (np == 4) {
            auto B = toMat<12>(M.data()); makePD<12>(B);
            BH.H12.push_back(B); BH.D4.push_back({idx[0], idx[1], idx[2], idx[3]});
        } else if (np == 3) {
            auto B = toMat<9>(M.data()); makePD<9>(B);
            BH.H9.push_back(B); BH.D3.push_back({idx[0], idx[1], idx[2]});
        } else {
            auto B = toMat<6>(M.data()); makePD<6>(B);
            BH.H6.push_back(B); BH.D2.push_back({idx[0], idx[1]});
        }
    }
}

// Points of a mollified entry and its four edge vertices.
static void eeMollifiedGeometry(const Mesh& m, int cI, int quad[4]) {
    const Contact& c = m.selfEE[cI];
    if (c[3] >= 0) { quad[0] = c[0]; quad[1] = c[1]; quad[2] = c[2]; quad[3] = c[3]; return; }
    const I2& eIeJ = m.selfEEeIe[cI];
    const I2& eI = m.surfEdges[eIeJ.first];
    const I2& eJ = m.surfEdges[eIeJ.second];
    quad[0] = eI.first; quad[1] = eI.second; quad[2] = eJ.first; quad[3] = eJ.second;
}

// compute_g_dee, ContactMechanics.cpp:3034-3080.
static void gDEE(const Mesh& m, std::vector<V3>& out, double dHat, double coef) {
    int n = (int)m.selfEE.size();
    std::vector<double> vals(n);
    for (int cI = 0; cI < n; ++cI) vals[cI] = selfConstraintVal(m, m.selfEE[cI]);
    for (int cI = 0; cI < n; ++cI) {
        double b;
        barrier(vals[cI], dHat, b);
        barrierG(vals[cI], dHat, vals[cI]);
        int q[4];
        eeMollifiedGeometry(m, cI, q);
        double ex = epsX(m, q[0], q[1], q[2], q[3]);
        V3 p[4] = {m.x[q[0]], m.x[q[1]], m.x[q[2]], m.x[q[3]]};
        double e, eg[12];
        mollifier(p, ex, e, eg, nullptr);
        double cb = coef * b;
        for (int k = 0; k < 4; ++k) out[q[k]] += V3(cb * eg[3 * k], cb * eg[3 * k + 1], cb * eg[3 * k + 2]);
        vals[cI] *= e;
    }
    gDPT(m, m.selfEE, vals, 0, out, coef);
}

// compute_H_dee, ContactMechanics.cpp:3575-3700.
static void hDEE(const Mesh& m, BHessian& BH, double dHat, double coef) {
    int n = (int)m.selfEE.size();
    for (int cI = 0; cI < n; ++cI) {
        const Contact& c = m.selfEE[cI];
        double d = selfConstraintVal(m, c);
        double b, gb, hb;
        barrier(d, dHat, b); barrierG(d, dHat, gb); barrierH(d, dHat, hb);
        int q[4];
        eeMollifiedGeometry(m, cI, q);
        double ex = epsX(m, q[0], q[1], q[2], q[3]);
        V3 p[4] = {m.x[q[0]], m.x[q[1]], m.x[q[2]], m.x[q[3]]};
        double e, eg[12], eH[144];
        mollifier(p, ex, e, eg, eH);
        double gd[12] = {0}, Hd[144] = {0};
        if (c[3] >= 0) {
            distanceGradHess(3, p, gd, Hd);
        } else {
            int v0 = -c[0] - 1;
            int ind[4] = {q[0], q[1], q[2], q[3]};
            if (c[2] >= 0) {
                V3 pp[3] = {m.x[v0], m.x[c[1]], m.x[c[2]]};
                double g9[9], H9[81];
                distanceGradHess(1, pp, g9, H9);
                int map[3] = {0, 0, 0};
                for (int i = 0; i < 4; ++i) {
                    if (v0 == ind[i]) map[0] = i;
                    else if (c[1] == ind[i]) map[1] = i;
                    else if (c[2] == ind[i]) map[2] = i;
                }
                for (int i = 0; i < 3; ++i) {
                    for (int k = 0; k < 3; ++k) gd[3 * map[i] + k] = g9[3 * i + k];
                    for (int j = 0; j < 3; ++j)
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                Hd[(3 * map[i] + a) * 12 + 3 * map[j] + bb] = H9[(3 * i + a) * 9 + 3 * j + bb];
                }
            } else {
                V3 pp[2] = {m.x[v0], m.x[c[1]]};
                double g6[6], H6[36];
                distanceGradHess(0, pp, g6, H6);
                int map[2] = {0, 0};
                for (int i = 0; i < 4; ++i) {
                    if (v0 == ind[i]) map[0] = i;
                    else if (c[1] == ind[i]) map[1] = i;
                }
                for (int i = 0; i < 2; ++i) {
                    for (int k = 0; k < 3; ++k) gd[3 * map[i] + k] = g6[3 * i + k];
                    for (int j = 0; j < 2; ++j)
                        for (int a = 0; a < 3; ++a)
                            for (int bb = 0; bb < 3; ++bb)
                                Hd[(3 * map[i] + a) * 12 + 3 * map[j] + bb] = H6[(3 * i + a) * 6 + 3 * j + bb];
                }
            }
        }
        Mat<12, 12> PH;
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) {
                double k1 = ((coef * gb) * gd[i]) * eg[j];
                double k1t = ((coef * gb) * gd[j]) * eg[i];
                PH.a[i][j] = k1 + k1t + (coef * b) * eH[i * 12 + j] + ((coef * e * hb) * gd[i]) * gd[j] + (coef * e * gb) * Hd[i * 12 + j];
            }
        makePD<12>(PH);
        BH.H12.push_back(PH);
        BH.D4.push_back({q[0], q[1], q[2], q[3]});
    }
}

// ---------------------------------------------------------------------------
// Friction (Friction.cpp:81-545, FrictionKinematics.h)
// ---------------------------------------------------------------------------
using M32d = Mat<3, 2>;

static M32d basisCols(const V3& a, const V3& b) {
    M32d B;
    for (int k = 0; k < 3; ++k) { B.a[k][0] = a[k]; B.a[k][1] = b[k]; }
    return B;
}
static void tangentAndCoord(const Mesh& m, const Contact& c, std::array<double, 2>& coord, M32d& basis) {
    const auto& x = m.x;
    if (c[0] >= 0) {
        V3 v0 = x[c[0]], v1 = x[c[1]], v2 = x[c[2]], v3 = x[c[3]];
        V3 e20 = v0 - v2, e01 = v1 - v0, e23 = v3 - v2;
        solve2(sqnorm(e01), -dot(e23, e01), sqnorm(e23), -dot(e20, e01), dot(e20, e23), coord[0], coord[1]);
        V3 v01 = v1 - v0;
        basis = basisCols(normalized(v01), normalized(cross(cross(v01, v3 - v2), v01)));
        return;
    }
    int p = -c[0] - 1;
    if (c[2] < 0) {
        coord = {0, 0};
        V3 v01 = x[c[1]] - x[p];
        V3 xc = cross(V3(1, 0, 0), v01), yc = cross(V3(0, 1, 0), v01);
        if (sqnorm(xc) > sqnorm(yc)) basis = basisCols(normalized(xc), normalized(cross(v01, xc)));
        else basis = basisCols(normalized(yc), normalized(cross(v01, yc)));
    } else if (c[3] < 0) {
        V3 e12 = x[c[2]] - x[c[1]];
        coord[0] = dot(x[p] - x[c[1]], e12) / sqnorm(e12);
        coord[1] = 0;
        basis = basisCols(normalized(e12), normalized(cross(e12, x[p] - x[c[1]])));
    } else {
        V3 r0 = x[c[2]] - x[c[1]], r1 = x[c[3]] - x[c[1]], w = x[p] - x[c[1]];
        solve2(dot(r0, r0), dot(r0, r1), dot(r1, r1), dot(r0, w), dot(r1, w), coord[0], coord[1]);
        basis = basisCols(normalized(r0), normalized(cross(cross(r0, r1), r0)));
    }
}

// Friction::initialize, Friction.cpp:81-156.
void frictionInitialize(Mesh& m) {
    int n = (int)m.selfActive.size();
    m.selfLambda.resize(n);
    for (int i = 0; i < n; ++i) {
        double d = selfConstraintVal(m, m.selfActive[i]);
        barrierG(d, m.Hhat, m.selfLambda[i]);
        m.selfLambda[i] *= -m.kappa * 2.0 * std::sqrt(d);
        if (m.selfActive[i][3] < -1) m.selfLambda[i] *= -m.selfActive[i][3];
    }
    m.distCoord.resize(n);
    m.tanBasis.resize(n);
    for (int i = 0; i < n; ++i) tangentAndCoord(m, m.selfActive[i], m.distCoord[i], m.tanBasis[i]);
    m.selfActiveLastH = m.selfActive;
    int ng = (int)m.envActive.size();
    m.envLambda.resize(ng);
    for (int i = 0; i < ng; ++i) {
        double dist = dot(m.groundN, m.x[m.envActive[i]]) - m.groundD;
        double d = dist * dist;
        barrierG(d, m.Hhat, m.envLambda[i]);
        m.envLambda[i] *= -m.kappa * 2.0 * std::sqrt(d);
    }
    m.envActiveLastH = m.envActive;
}

// Relative tangential displacement of a lagged contact (computeRelDX_* then
// projection on the frozen basis).
static void frictionRel(const Mesh& m, int cI, double rel[2], int idx[4], int& np, double w[4]) {
    const Contact& c = m.selfActiveLastH[cI];
    const auto& x = m.x; const auto& vp = m.vprev;
    const auto& co = m.distCoord[cI];
    V3 r;
    if (c[0] >= 0) {
        for (int k = 0; k < 4; ++k) idx[k] = c[k];
        np = 4;
        V3 d0 = x[c[0]] - vp[c[0]], d1 = x[c[1]] - vp[c[1]], d2 = x[c[2]] - vp[c[2]], d3 = x[c[3]] - vp[c[3]];
        r = d0 + co[0] * (d1 - d0) - (d2 + co[1] * (d3 - d2));
        w[0] = 1.0 - co[0]; w[1] = co[0]; w[2] = co[1] - 1.0; w[3] = -co[1];
    } else {
        int p = -c[0] - 1;
        idx[0] = p; idx[1] = c[1];
        V3 d0 = x[p] - vp[p], d1 = x[c[1]] - vp[c[1]];
        if (c[2] < 0) {
            np = 2; r = d0 - d1; w[0] = 1; w[1] = -1;
        } else if (c[3] < 0) {
            np = 3; idx[2] = c[2];
            V3 d2 = x[c[2]] - vp[c[2]];
            r = d0 - (d1 + co[0] * (d2 - d1));
            w[0] = 1; w[1] = co[0] - 1.0; w[2] = -co[0];
        } else {
            np = 4; idx[2] = c[2]; idx[3] = c[3];
            V3 d2 = x[c[2]] - vp[c[2]], d3 = x[c[3]] - vp[c[3]];
            r = d0 - (d1 + co[0] * (d2 - d1) + co[1] * (d3 - d1));
            w[0] = 1; w[1] = -1 + co[0] + co[1]; w[2] = -co[0]; w[3] = -co[1];
        }
    }
    const M32d& B = m.tanBasis[cI];
    rel[0] = r.x * B.a[0][0] + r.y * B.a[1][0] + r.z * B.a[2][0];
    rel[1] = r.x * B.a[0][1] + r.y * B.a[1][1] + r.z * B.a[2][1];
}

static inline double f1DivNorm(double x2, double eps) { return (-std::sqrt(x2) + 2.0 * eps) / (eps * eps); }
static inline double f2SF(double x2, double eps) { return 2.0 * (eps - std::sqrt(x2)) / (eps * eps); }
static inline double f0SF(double x2, double eps) { return x2 * (-std::sqrt(x2) / 3.0 + eps) / (eps * eps) + eps / 3.0; }

// Friction::addGradient, Friction.cpp:159-304.
static void frictionGradient(const Mesh& m, std::vector<V3>& g, double eps2, double coef) {
    double eps = std::sqrt(eps2);
    for (int cI = 0; cI < (int)m.selfActiveLastH.size(); ++cI) {
        double rel[2], w[4];
        int idx[4], np;
        frictionRel(m, cI, rel, idx, np, w);
        double sq = rel[0] * rel[0] + rel[1] * rel[1];
        if (sq > eps2) { double s = std::sqrt(sq); rel[0] /= s; rel[1] /= s; }
        else { double f = f1DivNorm(sq, eps); rel[0] *= f; rel[1] *= f; }
        const M32d& B = m.tanBasis[cI];
        V3 t(B.a[0][0] * rel[0] + B.a[0][1] * rel[1], B.a[1][0] * rel[0] + B.a[1][1] * rel[1], B.a[2][0] * rel[0] + B.a[2][1] * rel[1]);
        double s = coef * m.selfLambda[cI];
        for (int k = 0; k < np; ++k) g[idx[k]] += (w[k] * t) * s;
    }
    for (int i = 0; i < (int)m.envActiveLastH.size(); ++i) {
        int v = m.envActiveLastH[i];
        V3 d = m.x[v] - m.vprev[v];
        V3 pr = d - dot(d, m.groundN) * m.groundN;
        double p2 = sqnorm(pr);
        if (p2 > eps2) g[v] += coef * m.envLambda[i] / std::sqrt(p2) * pr;
        else g[v] += coef * m.envLambda[i] / eps * pr;
    }
}

// Friction::addHessian, Friction.cpp:306-457.
static void frictionHessian(const Mesh& m, BHessian& BH, double eps2, double coef) {
    double eps = std::sqrt(eps2);
    // ground basis (groundTangentBasis, Friction.cpp:66-76)
    V3 n = m.groundN;
    V3 helper = std::fabs(n.x) < 0.9 ? V3(1, 0, 0) : V3(0, 1, 0);
    V3 b0 = normalized(helper - dot(helper, n) * n);
    V3 b1 = normalized(cross(n, b0));
    for (int i = 0; i < (int)m.envActiveLastH.size(); ++i) {
        int v = m.envActiveLastH[i];
        double mult = std::max(0.0, coef * m.envLambda[i]);
        V3 d = m.x[v] - m.vprev[v];
        double r0 = dot(b0, d), r1 = dot(b1, d);
        double nr = std::sqrt(r0 * r0 + r1 * r1);
        M3 H;
        if (mult > 0.0) {
            if (nr > eps) {
                double p0 = r0 / nr, p1 = r1 / nr;
                double q0 = -p1, q1 = p0;
                V3 l = q0 * b0 + q1 * b1;
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H.a[a][b] = (mult / nr) * l[a] * l[b];
            } else {
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H.a[a][b] = (mult / eps) * (b0[a] * b0[b] + b1[a] * b1[b]);
            }
        }
        BH.H3.push_back(H);
        BH.D1.push_back(v);
    }
    for (int cI = 0; cI < (int)m.selfActiveLastH.size(); ++cI) {
        double rel[2], w[4];
        int idx[4], np;
        frictionRel(m, cI, rel, idx, np, w);
        double mult = coef * m.selfLambda[cI];
        double weight = std::max(0.0, mult);
        int n3 = 3 * np;
        std::vector<double> H(n3 * n3, 0.0);
        const M32d& B = m.tanBasis[cI];
        auto addDir = [&](double t0, double t1, double eig) {
            double e = std::max(0.0, eig);
            if (e == 0.0) return;
            V3 t(B.a[0][0] * t0 + B.a[0][1] * t1, B.a[1][0] * t0 + B.a[1][1] * t1, B.a[2][0] * t0 + B.a[2][1] * t1);
            double L[12];
            for (int k = 0; k < np; ++k) for (int a = 0; a < 3; ++a) L[3 * k + a] = w[k] * t[a];
            for (int i = 0; i < n3; ++i) for (int j = 0; j < n3; ++j) H[i * n3 + j] += weight * e * L[i] * L[j];
        };
        if (weight != 0.0) {
            double sq = rel[0] * rel[0] + rel[1] * rel[1];
            double nr = std::sqrt(sq);
            if (nr > 0.0) {
                double p0 = rel[0] / nr, p1 = rel[1] / nr;
                if (nr > eps) addDir(-p1, p0, 1.0 / nr);
                else {
                    double perp = f1DivNorm(sq, eps), par = f2SF(sq, eps);
                    addDir(p0, p1, par);
                    addDir(-p1, p0, perp);
                }
            } else {
                double iso = f1DivNorm(0.0, eps);
                addDir(1, 0, iso);
                addDir(0, 1, iso);
            }
        }
        if (np == 4) { BH.H12.push_back(toMat<12>(H.data())); BH.D4.push_back({idx[0], idx[1], idx[2], idx[3]}); }
        else if (np == 3) { BH.H9.push_back(toMat<9>(H.data())); BH.D3.push_back({idx[0], idx[1], idx[2]}); }
        else { BH.H6.push_back(toMat<6>(H.data())); BH.D2.push_back({idx[0], idx[1]}); }
    }
}

// Friction::energy, Friction.cpp:459-545.
static double frictionEnergy(const Mesh& m) {
    double eps2 = m.Fhat * m.dt * m.dt;
    double eps = std::sqrt(eps2);
    double sum = 0;
    for (int cI = 0; cI < (int)m.selfActiveLastH.size(); ++cI) {
        double rel[2], w[4];
        int idx[4], np;
        frictionRel(m, cI, rel, idx, np, w);
        double sq = rel[0] * rel[0] + rel[1] * rel[1];
        sum += sq > eps2 ? m.selfLambda[cI] * std::sqrt(sq) : m.selfLambda[cI] * f0SF(sq, eps);
    }
    double result = m.friction * sum;
    for (int i = 0; i < (int)m.envActiveLastH.size(); ++i) {
        int v = m.envActiveLastH[i];
        V3 d = m.x[v] - m.vprev[v];
        V3 pr = d - dot(d, m.groundN) * m.groundN;
        double sq = sqnorm(pr);
        double cl = sq > eps2 ? std::sqrt(sq) - 0.5 * eps : 0.5 * sq / eps;
        result += m.friction * m.envLambda[i] * cl;
    }
    return result;
}

// ---------------------------------------------------------------------------
// Assembly (computeGradientAndHessian, IPCSolver.cpp:108-319)
// ---------------------------------------------------------------------------
int computeGradientAndHessian(Mesh& m, std::vector<V3>& grad, BHessian& BH, const SolverOptions& o) {
    int nv = m.nv();
    double dt2 = m.dt * m.dt;
    grad.assign(nv, V3());
    for (int v = 0; v < nv; ++v) grad[v] = m.mass[v] * (m.x[v] - m.xtilde[v]);
    for (int v = 0; v < nv; ++v) grad[v] += (m.drag * m.mass[v] * (m.x[v] - m.vprev[v]));
    // soft boundary (BoundaryConditions.cpp:175-210)
    for (size_t k = 0; k < m.softIdx.size(); ++k) {
        int v = m.softIdx[k];
        grad[v] += m.softW * (m.x[v] - m.softTarget[k]);
        M3 H = M3::identity();
        scale(H, m.softW);
        BH.H3.push_back(H);
        BH.D1.push_back(v);
    }
    // tetrahedra
    int nt = (int)m.tets.size();
    std::vector<Vec<12>> tetG(nt);
    size_t h12base = BH.H12.size();
    BH.H12.resize(h12base + nt);
    parallelFor(nt, o.threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            M3 F = tetF(m.x, m.tets[i], m.DmInv[i]);
            M3 P = snhPK1(F, m.tetLen[i], m.tetVolR[i]);
            Mat<9, 12> PF = pfpxTet(m.DmInv[i]);
            Vec<9> pv;
            for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) pv[3 * c + r] = P.a[r][c];
            Vec<12> f = mulv(transpose(PF), pv);
            for (int k = 0; k < 12; ++k) f[k] = m.vol[i] * f[k];
            tetG[i] = f;
            Mat<9, 9> Hq = snhHessian(F, m.tetLen[i], m.tetVolR[i]);
            Mat<12, 12> H = mul(transpose(PF), mul(Hq, PF));
            scale(H, m.vol[i] * dt2);
            BH.H12[h12base + i] = H;
        }
    });
    for (int i = 0; i < nt; ++i)
        for (int k = 0; k < 4; ++k) {
            int v = m.tets[i][k];
            grad[v] += dt2 * V3(tetG[i][3 * k], tetG[i][3 * k + 1], tetG[i][3 * k + 2]);
        }
    for (int i = 0; i < nt; ++i) BH.D4.push_back(m.tets[i]);
    // cloth triangles
    int nf = (int)m.tris.size();
    std::vector<Vec<9>> triG(nf);
    size_t h9base = BH.H9.size();
    BH.H9.resize(h9base + nf);
    parallelFor(nf, o.threads, [&](int b, int e) {
        for (int i = b; i < e; ++i) {
            M32 F = triF(m.x, m.tris[i], m.DmInv2[i]);
            M32 P = bwPK1(F, m.stretchS, m.shearS, m.strainRate);
            Mat<6, 9> PF = pfpxTri(m.DmInv2[i]);
            Vec<6> pv;
            for (int c = 0; c < 2; ++c) for (int r = 0; r < 3; ++r) pv[3 * c + r] = P.a[r][c];
            Vec<9> f = mulv(transpose(PF), pv);
            for (int k = 0; k < 9; ++k) f[k] = dt2 * m.area[i] * f[k];
            triG[i] = f;
            Mat<6, 6> Hq = bwHessian(F, m.stretchS, m.shearS, m.strainRate);
            Mat<9, 9> H = mul(transpose(PF), mul(Hq, PF));
            scale(H, m.area[i] * dt2);
            BH.H9[h9base + i] = H;
        }
    });
    for (int i = 0; i < nf; ++i)
        for (int k = 0; k < 3; ++k) {
            int v = m.tris[i][k];
            grad[v] += V3(triG[i][3 * k], triG[i][3 * k + 1], triG[i][3 * k + 2]);
        }
    for (int i = 0; i < nf; ++i) BH.D3.push_back(m.tris[i]);
    // quadratic bending (IPCSolver.cpp:197-237)
    double bs = m.plateRigidity * dt2;
    for (const QuadBend& qb : m.bend) {
        for (int a = 0; a < 4; ++a) {
            V3 s;
            for (int b = 0; b < 4; ++b) s += qb.Q.a[a][b] * m.x[qb.v[b]];
            grad[qb.v[a]] += bs * s;
        }
        Mat<12, 12> H;
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) for (int k = 0; k < 3; ++k) H.a[3 * a + k][3 * b + k] = bs * qb.Q.a[a][b];
        BH.H12.push_back(H);
        BH.D4.push_back({qb.v[0], qb.v[1], qb.v[2], qb.v[3]});
    }
    // hinge bending (IPCSolver.cpp:238-267)
    for (const HingeBend& hb : m.hinges) {
        double hg[12], hH[144];
        hingeEnergy(hb, m.x, m.plateRigidity, hg, hH);
        for (int a = 0; a < 4; ++a) grad[hb.v[a]] += dt2 * V3(hg[3 * a], hg[3 * a + 1], hg[3 * a + 2]);
        Mat<12, 12> H;
        for (int i = 0; i < 12; ++i)
            for (int j = 0; j < 12; ++j) H.a[i][j] = dt2 * hH[12 * i + j];
        BH.H12.push_back(H);
        BH.D4.push_back({hb.v[0], hb.v[1], hb.v[2], hb.v[3]});
    }
    // ground barrier (IPCSolver.cpp:270-293)
    for (size_t cI = 0; cI < m.envActive.size(); ++cI) {
        int v = m.envActive[cI];
        double dist = dot(m.groundN, m.x[v]) - m.groundD;
        double d = dist * dist;
        double gb, hb;
        barrierG(d, m.Hhat, gb);
        barrierH(d, m.Hhat, hb);
        grad[v] += m.kappa * gb * 2.0 * dist * m.groundN;
        double param = 4.0 * hb * d + 2.0 * gb;
        if (param > 0) {
            M3 H;
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H.a[a][b] = m.kappa * param * m.groundN[a] * m.groundN[b];
            BH.H3.push_back(H);
            BH.D1.push_back(v);
        }
    }
    // self contact (IPCSolver.cpp:296-307)
    std::vector<double> vals(m.selfActive.size());
    for (size_t i = 0; i < m.selfActive.size(); ++i) {
        double d = selfConstraintVal(m, m.selfActive[i]);
        barrierG(d, m.Hhat, vals[i]);
    }
    int collisions = gDPT(m, m.selfActive, vals, 0, grad, m.kappa);
    gDEE(m, grad, m.Hhat, m.kappa);
    hDPT(m, BH, m.Hhat, m.kappa);
    hDEE(m, BH, m.Hhat, m.kappa);
    // friction (IPCSolver.cpp:309-317)
    frictionGradient(m, grad, m.Fhat * dt2, m.friction);
    frictionHessian(m, BH, m.Fhat * dt2, m.friction);
    return collisions;
}

// computeEnergy, IPCSolver.cpp:322-456.
double computeEnergy(const Mesh& m, double kappa, const SolverOptions& o) {
    int nt = (int)m.tets.size(), nf = (int)m.tris.size();
    int nchunk = std::max(1, o.threads);
    std::vector<double> parts(nchunk, 0.0);
    auto chunked = [&](int n, const std::function<double(int)>& f) {
        std::fill(parts.begin(), parts.end(), 0.0);
        int per = (n + nchunk - 1) / nchunk;
        parallelFor(nchunk, o.threads > 1 && n >= 256 ? o.threads : 1, [&](int b, int e) {
            for (int c = b; c < e; ++c) {
                double s = 0;
                for (int i = c * per; i < std::min(n, (c + 1) * per); ++i) s += f(i);
                parts[c] = s;
            }
        });
        double s = 0;
        for (double p : parts) s += p;
        return s;
    };
    double E = chunked(nt, [&](int i) {
        M3 F = tetF(m.x, m.tets[i], m.DmInv[i]);
        return snhEnergyDensity(F, m.tetLen[i], m.tetVolR[i]) * m.vol[i];
    });
    E += chunked(nf, [&](int i) {
        M32 F = triF(m.x, m.tris[i], m.DmInv2[i]);
        return bwEnergyDensity(F, m.stretchS, m.shearS, m.strainRate) * m.area[i];
    });
    double be = 0;
    for (const QuadBend& qb : m.bend) {
        double s = 0;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) s += qb.Q.a[a][b] * dot(m.x[qb.v[a]], m.x[qb.v[b]]);
        be += s;
    }
    be *= 0.5 * m.plateRigidity;
    E += be;
    for (const HingeBend& hb : m.hinges) E += hingeEnergy(hb, m.x, m.plateRigidity, nullptr, nullptr);
    E *= m.dt * m.dt;
    double dE = 0;
    for (int i = 0; i < m.nv(); ++i) {
        dE += sqnorm(m.x[i] - m.xtilde[i]) * m.mass[i] / 2.0;
        dE += (sqnorm(m.x[i] - m.vprev[i]) * (m.drag) * m.mass[i] / 2.0);
    }
    E += dE;
    double soft = 0;
    for (size_t k = 0; k < m.softIdx.size(); ++k) soft += 0.5 * m.softW * sqnorm(m.x[m.softIdx[k]] - m.softTarget[k]);
    E += soft;
    double bsum = 0;
    for (int v : m.envActive) {
        double dist = dot(m.groundN, m.x[v]) - m.groundD;
        double b;
        barrier(dist * dist, m.Hhat, b);
        bsum += b;
    }
    for (const Contact& c : m.selfActive) {
        double b;
        barrier(selfConstraintVal(m, c), m.Hhat, b);
        if (c[3] < -1) b *= -c[3];
        bsum += b;
    }
    for (int cI = 0; cI < (int)m.selfEE.size(); ++cI) {
        int q[4];
        eeMollifiedGeometry(m, cI, q);
        double ex = epsX(m, q[0], q[1], q[2], q[3]);
        V3 p[4] = {m.x[q[0]], m.x[q[1]], m.x[q[2]], m.x[q[3]]};
        double e;
        mollifier(p, ex, e, nullptr, nullptr);
        double b;
        barrier(selfConstraintVal(m, m.selfEE[cI]), m.Hhat, b);
        bsum += b * e;
    }
    E += kappa * bsum;
    E += frictionEnergy(m);
    return E;
}

// ---------------------------------------------------------------------------
// kappa rules (IPCSolver.cpp:751-869)
// ---------------------------------------------------------------------------
void suggestKappa(double& kappa, double Hhat, double bbox2, double meanMass) {
    double hb;
    barrierH(1.0e-16 * bbox2, Hhat, hb);
    kappa = 1e13 * meanMass / (4.0e-16 * bbox2 * hb);
}
void upperBoundKappa(double& kappa, double Hhat, double bbox2, double meanMass) {
    double hb;
    barrierH(1.0e-16 * bbox2, Hhat, hb);
    double kmax = 100 * 1e13 * meanMass / (4.0e-16 * bbox2 * hb);
    if (kappa > kmax) kappa = kmax;
}

// initKappa: `kappa` may alias m.kappa exactly as in the reference.
void initKappa(Mesh& m, double& kappa) {
    if (m.envActive.size() + m.selfActive.size() == 0) return;
    int nv = m.nv();
    std::vector<V3> gE(nv), gc(nv);
    for (int v = 0; v < nv; ++v) gE[v] += m.mass[v] * (m.x[v] - m.xtilde[v]);
    double dt2 = m.dt * m.dt;
    for (size_t i = 0; i < m.tets.size(); ++i) {
        M3 F = tetF(m.x, m.tets[i], m.DmInv[i]);
        M3 P = snhPK1(F, m.tetLen[i], m.tetVolR[i]);
        Mat<9, 12> PF = pfpxTet(m.DmInv[i]);
        Vec<9> pv;
        for (int c = 0; c < 3; ++c) for (int r = 0; r < 3; ++r) pv[3 * c + r] = P.a[r][c];
        Vec<12> f = mulv(transpose(PF), pv);
        for (int k = 0; k < 4; ++k)
            gE[m.tets[i][k]] += dt2 * V3(m.vol[i] * f[3 * k], m.vol[i] * f[3 * k + 1], m.vol[i] * f[3 * k + 2]);
    }
    for (int v : m.envActive) {
        double dist = dot(m.groundN, m.x[v]) - m.groundD;
        double g;
        barrierG(dist * dist, m.Hhat, g);
        gc[v] += g * 2.0 * dist * m.groundN;
    }
    std::vector<double> vals(m.selfActive.size());
    for (size_t i = 0; i < m.selfActive.size(); ++i) barrierG(selfConstraintVal(m, m.selfActive[i]), m.Hhat, vals[i]);
    gDPT(m, m.selfActive, vals, 0, gc, 1);
    double gsum = 0, gsnorm = 0;
    for (int i = 0; i < nv; ++i) { gsum += dot(gc[i], gE[i]); gsnorm += sqnorm(gc[i]); }
    double minKappa = -gsum / gsnorm;
    if (minKappa > 0.0) kappa = minKappa;
    suggestKappa(minKappa, m.Hhat, m.bboxDiag2, m.meanMass);
    if (kappa < minKappa) kappa = minKappa;
    upperBoundKappa(m.kappa, m.Hhat, m.bboxDiag2, m.meanMass);
}

// postLineSearch, IPCSolver.cpp:811-869.
void postLineSearch(Mesh& m, double& kappa) {
    if (kappa == 0.0) { initKappa(m, kappa); return; }
    bool update = false;
    for (size_t i = 0; i < m.closeID.size(); ++i) {
        double dist = dot(m.groundN, m.x[m.closeID[i]]) - m.groundD;
        if (dist * dist <= m.closeVal[i]) { update = true; break; }
    }
    if (!update)
        for (size_t i = 0; i < m.closeMID.size(); ++i)
            if (selfConstraintVal(m, m.closeMID[i]) <= m.closeMVal[i]) { update = true; break; }
    if (update) {
        kappa *= 2.0;
        upperBoundKappa(m.kappa, m.Hhat, m.bboxDiag2, m.meanMass);
    }
    m.closeID.clear(); m.closeMID.clear(); m.closeVal.clear(); m.closeMVal.clear();
    for (int v : m.envActive) {
        double dist = dot(m.groundN, m.x[v]) - m.groundD;
        double d = dist * dist;
        if (d < m.dTol) { m.closeID.push_back(v); m.closeVal.push_back(d); }
    }
    for (const Contact& c : m.selfActive) {
        double d = selfConstraintVal(m, c);
        if (d < m.dTol) { m.closeMID.push_back(c); m.closeMVal.push_back(d); }
    }
}

// twistingBoundaryDirection, CPU IPC/Simulator.cpp:24-46, with the angular
// rate as a parameter (3.14/5 rad/s in the reference's twisting-mat scene).
V3 motionDirection(int motion, double rate, const V3& x, const V3& rest, double frac, double dt) {
    if (motion != MOTION_TWIST_X) return V3();
    double ang = rate * dt * frac;
    double c = std::cos(ang), s = std::sin(ang);
    if (rest.x < 0.0) return V3(x.x, c * x.y + s * x.z, -s * x.y + c * x.z) - x;
    if (rest.x > 0.0) return V3(x.x, c * x.y - s * x.z, s * x.y + c * x.z) - x;
    return V3();
}

}  // namespace oracle
