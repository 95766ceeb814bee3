// Host-side rest-state set-up of a GPU context: material parameters, lumped
// masses, inverse rest shapes, volumes/areas, quadratic bending hinges and
// the collision surface.  Runs once per context on the CPU; the results are
// uploaded and never recomputed.
//
// Reference: updateMaterial (CPU IPC/Simulator.cpp:128-141), initMesh3D
// (CPU IPC/Elasticity.cpp:1050-1116), prepareQuadraticBending
// (CPU IPC/Simulator.cpp:48-109), mesh3D::getSurface
// (CPU IPC/SimulationMesh.cpp:364-446), buildModels (Simulator.cpp:426-529).
#include "scene_setup.h"
#include "hinge_bending.cuh"

#include <cmath>
#include <cstdint>
#include <set>
#include <stdexcept>
#include <map>
#include <unordered_map>

namespace cipc {

namespace {
struct P3 {
    double x, y, z;
};
inline P3 sub(P3 a, P3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline P3 crs(P3 a, P3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double dt(P3 a, P3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double nrm(P3 a) { return std::sqrt(dt(a, a)); }
inline P3 scl(double s, P3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline P3 at(const std::vector<double>& x, int i) { return {x[3 * i], x[3 * i + 1], x[3 * i + 2]}; }

struct TriKey {
    uint64_t k[3];
    bool operator==(const TriKey& o) const { return k[0] == o.k[0] && k[1] == o.k[1] && k[2] == o.k[2]; }
};
}  // namespace

void materialFromYoung(double E, double nu, double& lengthRate, double& volumeRate) {
    double lengthRateLame = E / (2 * (1 + nu));
    double volumeRateLame = E * nu / ((1 + nu) * (1 - 2 * nu));
    lengthRate = 4 * lengthRateLame / 3;
    volumeRate = volumeRateLame + 5 * lengthRateLame / 6;
}

void setupScene(const SceneInput& in, SceneRest& out) {
    int nv = in.nv;
    const std::vector<double>& x = in.x;
    // material (updateMaterial)
    materialFromYoung(in.E, in.nu, out.lengthRate, out.volumeRate);
    out.stretchS = in.clothE / (1 - in.nu * in.nu);
    out.shearS = in.shearE / (2 * (1 + in.nu)) / in.thickness;
    out.plateRigidity = in.bendE * std::pow(in.thickness, 3) / (12 * (1 - in.nu * in.nu));
    // masses, inverse rest shapes (initMesh3D)
    out.mass.assign(nv, 0.0);
    out.DmInv.assign(9 * (size_t)in.nt, 0.0);
    out.vol.assign(in.nt, 0.0);
    out.tetMu.assign(in.nt, out.lengthRate);
    out.tetLam.assign(in.nt, out.volumeRate);
    double massSum = 0;
    for (int i = 0; i < in.nt; ++i) {
        const int* t = &in.tets[4 * i];
        P3 a = sub(at(x, t[1]), at(x, t[0])), b = sub(at(x, t[2]), at(x, t[0])), c = sub(at(x, t[3]), at(x, t[0]));
        double m[3][3] = {{a.x, b.x, c.x}, {a.y, b.y, c.y}, {a.z, b.z, c.z}};
        P3 h = crs(a, b);
        double bottom = nrm(h);
        double hn = nrm(h);
        if (hn > 0) h = scl(1.0 / hn, h);
        double v = bottom * std::fabs(dt(h, c)) / 6;
        v = v > 0 ? v : -v;
        out.vol[i] = v;
        for (int k = 0; k < 4; ++k) out.mass[t[k]] += v * in.density / 4;
        massSum += v * in.density;
        double c00 = m[1][1] * m[2][2] - m[1][2] * m[2][1], c10 = m[1][2] * m[2][0] - m[1][0] * m[2][2], c20 = m[1][0] * m[2][1] - m[1][1] * m[2][0];
        double det = m[0][0] * c00 + m[0][1] * c10 + m[0][2] * c20;
        if (!(std::fabs(det) > 0)) throw std::invalid_argument("degenerate rest tetrahedron " + std::to_string(i));
        double* D = &out.DmInv[9 * (size_t)i];
        D[0] = c00 / det; D[3] = c10 / det; D[6] = c20 / det;
        D[1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) / det;
        D[4] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) / det;
        D[7] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) / det;
        D[2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) / det;
        D[5] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) / det;
        D[8] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) / det;
        if (!in.tetE.empty()) materialFromYoung(in.tetE[i], in.nu, out.tetMu[i], out.tetLam[i]);
    }
    out.DmInv2.assign(4 * (size_t)in.nf, 0.0);
    out.area.assign(in.nf, 0.0);
    for (int i = 0; i < in.nf; ++i) {
        const int* t = &in.tris[3 * i];
        P3 v01 = sub(at(x, t[1]), at(x, t[0])), v02 = sub(at(x, t[2]), at(x, t[0]));
        P3 n = crs(v01, v02);
        double nn = nrm(n);
        if (nn > 0) n = scl(1.0 / nn, n);
        // rotate the triangle normal onto +y; (x, z) are the material coordinates
        P3 vec = crs(n, P3{0, 1, 0});
        double cs = n.y;
        double K[3][3] = {{0, -vec.z, vec.y}, {vec.z, 0, -vec.x}, {-vec.y, vec.x, 0}};
        double R[3][3];
        for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) {
                double k2 = K[r][0] * K[0][q] + K[r][1] * K[1][q] + K[r][2] * K[2][q];
                R[r][q] = (r == q ? 1.0 : 0.0) + K[r][q] + k2 / (1 + cs);
            }
        auto rot = [&](P3 p) {
            return P3{R[0][0] * p.x + R[0][1] * p.y + R[0][2] * p.z, R[1][0] * p.x + R[1][1] * p.y + R[1][2] * p.z,
                      R[2][0] * p.x + R[2][1] * p.y + R[2][2] * p.z};
        };
        P3 r0 = rot(at(x, t[0])), r1 = rot(at(x, t[1])), r2 = rot(at(x, t[2]));
        double M[2][2] = {{r1.x - r0.x, r2.x - r0.x}, {r1.z - r0.z, r2.z - r0.z}};
        double det = M[0][0] * M[1][1] - M[0][1] * M[1][0];
        if (!(std::fabs(det) > 0)) throw std::invalid_argument("degenerate rest triangle " + std::to_string(i));
        double* D = &out.DmInv2[4 * (size_t)i];
        D[0] = M[1][1] / det; D[1] = -M[0][1] / det; D[2] = -M[1][0] / det; D[3] = M[0][0] / det;
        double a = nrm(crs(v01, v02)) * 0.5 * in.thickness;
        out.area[i] = a;
        for (int k = 0; k < 3; ++k) out.mass[t[k]] += a * in.cloth_density / 3;
        massSum += a * in.cloth_density;
    }
    out.meanMass = massSum / nv;
    // quadratic bending hinges (prepareQuadraticBending)
    out.bendV.clear();
    out.bendQ.clear();
    if (in.quadBending) {
        std::unordered_map<int64_t, int> edgeMap;
        for (int i = 0; i < in.nf; ++i) {
            const int* tri = &in.tris[3 * i];
            for (int e = 0; e < 3; ++e) {
                int e0 = tri[e], e1 = tri[(e + 1) % 3], other = tri[(e + 2) % 3];
                if (e0 > e1) std::swap(e0, e1);
                int64_t key = (int64_t(e0) << 32) | e1;
                auto it = edgeMap.find(key);
                if (it == edgeMap.end()) { edgeMap[key] = other; continue; }
                int o1 = it->second, o2 = other;
                P3 v0 = at(x, o1), v1 = at(x, e0), v2 = at(x, e1), v3 = at(x, o2);
                P3 E0 = sub(v2, v1), E1 = sub(v0, v1), E2 = sub(v3, v1), E3 = sub(v0, v2), E4 = sub(v3, v2);
                double a0 = 0.5 * nrm(crs(E0, E1)), a1 = 0.5 * nrm(crs(E0, E2));
                auto cot = [](P3 p, P3 q) { return dt(p, q) / nrm(crs(p, q)); };
                P3 mE0 = scl(-1.0, E0);
                double c01 = cot(E0, E1), c02 = cot(E0, E2), c03 = cot(mE0, E3), c04 = cot(mE0, E4);
                double K[4] = {c03 + c04, c01 + c02, -c01 - c03, -c02 - c04};
                double s = 3.0 / (a0 + a1);
                out.bendV.insert(out.bendV.end(), {e0, e1, o1, o2});
                for (int p = 0; p < 4; ++p) for (int q = 0; q < 4; ++q) out.bendQ.push_back(s * K[p] * K[q]);
            }
        }
    }
    // dihedral-angle hinges (prepareHingeBending, Simulator.cpp:111-125): the
    // interior triangle edges as (min, max) pairs in lexicographic order, each
    // with the opposite vertices of its two triangles in triangle order
    out.hingeW.clear();
    out.hingeTh0.clear();
    if (in.hingeBending) {
        std::map<std::pair<int, int>, std::vector<int>> opposite;
        for (int i = 0; i < in.nf; ++i) {
            const int* tri = &in.tris[3 * i];
            for (int e = 0; e < 3; ++e) {
                const int a = tri[e], b = tri[(e + 1) % 3];
                opposite[{std::min(a, b), std::max(a, b)}].push_back(tri[(e + 2) % 3]);
            }
        }
        for (const auto& kv : opposite) {
            if (kv.second.size() != 2) continue;
            const int hv[4] = {kv.first.first, kv.first.second, kv.second[0], kv.second[1]};
            double r[12];
            for (int k = 0; k < 4; ++k)
                for (int q = 0; q < 3; ++q) r[3 * k + q] = x[3 * (size_t)hv[k] + q];
            const double w = hinge::restWeight(r);
            if (!std::isfinite(w) || !(w > 0)) throw std::invalid_argument("degenerate rest hinge geometry");
            out.bendV.insert(out.bendV.end(), {hv[0], hv[1], hv[2], hv[3]});
            out.hingeW.push_back(w);
            out.hingeTh0.push_back(hinge::angle(r));
        }
    }
    // collision surface
    if (in.hasSurface) {
        out.faces = in.faces;
        out.surfVerts = in.surfVerts;
        out.edges = in.edges;
    } else {
        // getSurface: tet boundary faces in the standard library's hash-map
        // order (the reference's order on the same library), oriented
        // outward, then the cloth triangles; first-appearance surface
        // vertices; surface edges from an ordered set.
        uint64_t length = (uint64_t)nv;
        auto hash = [&](const TriKey& t) { return length * (length * t.k[0] + t.k[1]) + t.k[2]; };
        std::unordered_map<TriKey, uint64_t, decltype(hash)> tri2Tet(4 * (size_t)in.nt, hash);
        uint64_t nt = (uint64_t)in.nt;
        for (int i = 0; i < in.nt; ++i) {
            const int* T = &in.tets[4 * i];
            for (int j = 0; j < 4; ++j) {
                uint64_t a = T[j % 4], b = T[(1 + j) % 4], c = T[(2 + j) % 4];
                TriKey perms[6] = {{{a, b, c}}, {{a, c, b}}, {{b, a, c}}, {{b, c, a}}, {{c, a, b}}, {{c, b, a}}};
                bool found = false;
                for (int p = 0; p < 6; ++p) {
                    if (tri2Tet.find(perms[p]) != tri2Tet.end()) { tri2Tet[perms[p]] = nt + 1; found = true; break; }
                }
                if (!found) tri2Tet[perms[0]] = (uint64_t)i;
            }
        }
        out.faces.clear();
        for (const auto& kv : tri2Tet) {
            if (kv.second >= nt) continue;
            const TriKey& t = kv.first;
            const int* T = &in.tets[4 * kv.second];
            int id3 = 0;
            for (int q = 0; q < 4; ++q)
                if ((uint64_t)T[q] != t.k[0] && (uint64_t)T[q] != t.k[1] && (uint64_t)T[q] != t.k[2]) { id3 = T[q]; break; }
            P3 n = crs(sub(at(x, (int)t.k[1]), at(x, (int)t.k[0])), sub(at(x, (int)t.k[2]), at(x, (int)t.k[0])));
            if (dt(n, sub(at(x, id3), at(x, (int)t.k[0]))) < 0) out.faces.insert(out.faces.end(), {(int)t.k[0], (int)t.k[1], (int)t.k[2]});
            else out.faces.insert(out.faces.end(), {(int)t.k[0], (int)t.k[2], (int)t.k[1]});
        }
        for (int i = 0; i < in.nf; ++i) out.faces.insert(out.faces.end(), {in.tris[3 * i], in.tris[3 * i + 1], in.tris[3 * i + 2]});
        std::vector<char> flag(nv, 0);
        out.surfVerts.clear();
        for (size_t f = 0; f < out.faces.size(); ++f)
            if (!flag[out.faces[f]]) { out.surfVerts.push_back(out.faces[f]); flag[out.faces[f]] = 1; }
        std::set<std::pair<int, int>> es;
        size_t nfc = out.faces.size() / 3;
        for (size_t f = 0; f < nfc; ++f) {
            const int* F = &out.faces[3 * f];
            for (int rep = 0; rep < 3; ++rep) {
                if (!es.count({F[1], F[0]})) es.insert({F[0], F[1]});
                if (!es.count({F[2], F[1]})) es.insert({F[1], F[2]});
                if (!es.count({F[0], F[2]})) es.insert({F[2], F[0]});
            }
        }
        out.edges.clear();
        for (const auto& e : es) { out.edges.push_back(e.first); out.edges.push_back(e.second); }
    }
    if (out.edges.empty()) throw std::invalid_argument("simulation surface has no edges");
    double len = 0;
    size_t ne = out.edges.size() / 2;
    for (size_t e = 0; e < ne; ++e) len += nrm(sub(at(x, out.edges[2 * e]), at(x, out.edges[2 * e + 1])));
    out.avgEdge = len / (ne * 3);
    // bbox-relative scalars (buildModels)
    double d2 = 0;
    for (int k = 0; k < 3; ++k) d2 += (in.bboxMax[k] - in.bboxMin[k]) * (in.bboxMax[k] - in.bboxMin[k]);
    out.bboxDiag2 = d2;
    out.Hhat = in.relDhat * in.relDhat * d2;
    out.Fhat = 1e-6 * d2;
    out.dTol = 1e-18 * d2;
}

}  // namespace cipc
