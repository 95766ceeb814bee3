// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
// anything under oracle/; the shipped library never links it.
//
// C ABI wrappers.  Scene setup follows FEMSimulator::buildModels
// (CPU IPC/Simulator.cpp:426-529).
#include "oracle_api.h"
#include "oracle_core.h"

#include <cstdio>
#include <cstring>
#include <stdexcept>

using namespace oracle;

namespace {
struct Ctx {
    Mesh m;
    BroadPhase bp;
    SolverOptions o;
    int stepIndex = 0;
};
void setErr(char* err, int len, const char* msg) {
    if (err && len > 0) { std::snprintf(err, len, "%s", msg); }
}
}  // namespace

extern "C" {

void* cipc_oracle_create(const cipc_oracle_scene* s, char* err, int errlen) {
    try {
        auto* c = new Ctx();
        Mesh& m = c->m;
        m.density = s->density; m.cloth_density = s->cloth_density; m.thickness = s->thickness;
        m.E = s->E; m.nu = s->nu; m.clothE = s->clothE; m.shearE = s->shearE; m.bendE = s->bendE;
        m.strainRate = s->strainRate; m.friction = s->friction;
        m.dt = s->dt; m.drag = s->drag; m.newtonThr = s->newtonThr;
        m.use_barrier = s->use_barrier != 0; m.apply_gravity = s->apply_gravity != 0; m.quasi_static = s->quasi_static != 0;
        updateMaterial(m);
        m.x.resize(s->nv);
        for (int i = 0; i < s->nv; ++i) m.x[i] = V3(s->x[3 * i], s->x[3 * i + 1], s->x[3 * i + 2]);
        m.vel.assign(s->nv, V3());
        if (s->vel) for (int i = 0; i < s->nv; ++i) m.vel[i] = V3(s->vel[3 * i], s->vel[3 * i + 1], s->vel[3 * i + 2]);
        m.tets.resize(s->nt);
        for (int i = 0; i < s->nt; ++i) for (int k = 0; k < 4; ++k) m.tets[i][k] = s->tets[4 * i + k];
        m.tris.resize(s->nf);
        for (int i = 0; i < s->nf; ++i) for (int k = 0; k < 3; ++k) m.tris[i][k] = s->tris[3 * i + k];
        m.btype.assign(s->btype, s->btype + s->nv);
        if (s->tetE) {
            m.tetLen.resize(s->nt); m.tetVolR.resize(s->nt);
            for (int i = 0; i < s->nt; ++i) {
                Mesh tmp = Mesh();
                tmp.E = s->tetE[i]; tmp.nu = m.nu; tmp.clothE = m.clothE; tmp.shearE = m.shearE; tmp.thickness = m.thickness; tmp.bendE = m.bendE;
                updateMaterial(tmp);
                m.tetLen[i] = tmp.lengthRate; m.tetVolR[i] = tmp.volumeRate;
            }
        }
        // bending model: 0 none, 1 quadratic (USE_QUADRATIC_BENDING), 2 hinge
        if (s->quad_bending == 1) prepareQuadraticBending(m);
        else if (s->quad_bending == 2) prepareHingeBending(m);
        initRestState(m);
        m.rest = m.x;
        m.vprev = m.x;
        // soft / Dirichlet (BoundaryConditionOps::initialize)
        if (s->nsoft > 0) {
            m.softIdx.assign(s->softIdx, s->softIdx + s->nsoft);
            m.softW = s->softW; m.softMotion = s->softMotion; m.softRate = s->softRate;
            m.softTarget.resize(s->nsoft);
            for (int k = 0; k < s->nsoft; ++k) m.softTarget[k] = m.x[m.softIdx[k]];
        }
        if (s->ndir > 0) {
            m.dirIdx.assign(s->dirIdx, s->dirIdx + s->ndir);
            m.dirMotion = s->dirMotion; m.dirRate = s->dirRate;
        }
        updateInertialTarget(m);
        V3 lo(s->bboxMin[0], s->bboxMin[1], s->bboxMin[2]), hi(s->bboxMax[0], s->bboxMax[1], s->bboxMax[2]);
        m.bboxDiag2 = sqnorm(hi - lo);
        m.Hhat = s->relDhat * s->relDhat * m.bboxDiag2;
        m.Fhat = 1e-6 * m.bboxDiag2;
        m.dTol = 1e-18 * m.bboxDiag2;
        m.kappa = 0;
        getSurface(m);
        if (m.surfEdges.empty()) throw std::runtime_error("simulation surface has no edges");
        double len = 0;
        for (const I2& e : m.surfEdges) len += norm(m.x[e.first] - m.x[e.second]);
        m.avgEdge = len / (m.surfEdges.size() * 3);
        c->o.linear = s->linear;
        c->o.pcgRelTol = s->pcgRelTol > 0 ? s->pcgRelTol : 1e-6;
        c->o.threads = s->threads > 0 ? s->threads : 1;
        buildCollisionSets(m, c->bp, true);
        return c;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return nullptr;
    }
}

void cipc_oracle_destroy(void* h) { delete static_cast<Ctx*>(h); }

int cipc_oracle_step(void* h, cipc_oracle_stats* out, char* err, int errlen) {
    auto* c = static_cast<Ctx*>(h);
    try {
        StepStats st;
        solveIPCStep(c->m, c->bp, st, c->stepIndex, c->o);
        c->stepIndex++;
        if (out) {
            out->frame = st.frame; out->newton = st.newton; out->kappaIters = st.kappaIters; out->backtracks = st.backtracks;
            out->energyBacktracks = st.energyBacktracks; out->intersectionBacktracks = st.intersectionBacktracks;
            out->maxEnergyBacktracksPerNewton = st.maxEnergyBacktracksPerNewton; out->newtonOverTwo = st.newtonOverTwo;
            out->collisions = st.collisions; out->kappa = st.kappa; out->minDist2 = st.minDist2;
            out->acceptedStepSum = st.acceptedStepSum; out->minStep = st.minStep; out->maxStep = st.maxStep;
            out->groundContacts = st.groundContacts; out->selfContacts = st.selfContacts;
            out->mollifiedContacts = st.mollifiedContacts; out->matrixNnz = st.matrixNnz; out->pcgIterations = st.pcgIterations;
            out->linearSolves = st.linearSolves;
        }
        return 0;
    } catch (const std::exception& e) {
        setErr(err, errlen, e.what());
        return 1;
    }
}

void cipc_oracle_info(void* h, long long* counts) {
    auto* c = static_cast<Ctx*>(h);
    counts[0] = c->m.nv(); counts[1] = (long long)c->m.surface.size(); counts[2] = (long long)c->m.surfVerts.size();
    counts[3] = (long long)c->m.surfEdges.size(); counts[4] = (long long)c->m.bend.size();
    counts[5] = (long long)c->m.tets.size(); counts[6] = (long long)c->m.tris.size();
}

void cipc_oracle_scalars(void* h, double* o) {
    const Mesh& m = static_cast<Ctx*>(h)->m;
    double v[14] = {m.kappa, m.Hhat, m.Fhat, m.dTol, m.bboxDiag2, m.meanMass, m.avgEdge, m.lengthRate, m.volumeRate,
                    m.stretchS, m.shearS, m.plateRigidity, m.dt, m.newtonThr};
    std::memcpy(o, v, sizeof(v));
}
void cipc_oracle_set_kappa(void* h, double k) { static_cast<Ctx*>(h)->m.kappa = k; }
void cipc_oracle_set_intersection_rule(void* h, int rule) {
    static_cast<Ctx*>(h)->m.coplanarTol = rule == 1 ? 0.0 : 1e-12;
}

static std::vector<V3>* field(Mesh& m, int which) {
    switch (which) {
    case 0: return &m.x; case 1: return &m.vel; case 2: return &m.vprev; case 3: return &m.xtilde; case 4: return &m.rest;
    default: return nullptr;
    }
}
void cipc_oracle_get(void* h, int which, double* out) {
    Mesh& m = static_cast<Ctx*>(h)->m;
    if (which == 5) { for (int i = 0; i < m.nv(); ++i) out[i] = m.mass[i]; return; }
    auto* f = field(m, which);
    for (size_t i = 0; i < f->size(); ++i) { out[3 * i] = (*f)[i].x; out[3 * i + 1] = (*f)[i].y; out[3 * i + 2] = (*f)[i].z; }
}
void cipc_oracle_set(void* h, int which, const double* in) {
    Mesh& m = static_cast<Ctx*>(h)->m;
    auto* f = field(m, which);
    for (size_t i = 0; i < f->size(); ++i) (*f)[i] = V3(in[3 * i], in[3 * i + 1], in[3 * i + 2]);
}

void cipc_oracle_surface(void* h, int* faces, int* verts, int* edges) {
    const Mesh& m = static_cast<Ctx*>(h)->m;
    for (size_t i = 0; i < m.surface.size(); ++i) for (int k = 0; k < 3; ++k) faces[3 * i + k] = m.surface[i][k];
    for (size_t i = 0; i < m.surfVerts.size(); ++i) verts[i] = m.surfVerts[i];
    for (size_t i = 0; i < m.surfEdges.size(); ++i) { edges[2 * i] = m.surfEdges[i].first; edges[2 * i + 1] = m.surfEdges[i].second; }
}

void cipc_oracle_rest(void* h, double* dminv, double* vol, double* dminv2, double* area, int* bendv, double* bendq) {
    const Mesh& m = static_cast<Ctx*>(h)->m;
    for (size_t i = 0; i < m.tets.size(); ++i) {
        for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) dminv[9 * i + 3 * a + b] = m.DmInv[i].a[a][b];
        vol[i] = m.vol[i];
    }
    for (size_t i = 0; i < m.tris.size(); ++i) {
        for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) dminv2[4 * i + 2 * a + b] = m.DmInv2[i].a[a][b];
        area[i] = m.area[i];
    }
    for (size_t i = 0; i < m.bend.size(); ++i) {
        for (int k = 0; k < 4; ++k) bendv[4 * i + k] = m.bend[i].v[k];
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) bendq[16 * i + 4 * a + b] = m.bend[i].Q.a[a][b];
    }
}

void cipc_oracle_collision_sets(void* h, long long* counts) {
    auto* c = static_cast<Ctx*>(h);
    buildCollisionSets(c->m, c->bp, true);
    counts[0] = (long long)c->m.selfActive.size(); counts[1] = (long long)c->m.selfEE.size();
    counts[2] = (long long)c->m.selfCCD.size(); counts[3] = (long long)c->m.envActive.size();
}

void cipc_oracle_get_sets(void* h, int* sa, int* see, int* eeie, int* ccd, int* gr) {
    const Mesh& m = static_cast<Ctx*>(h)->m;
    for (size_t i = 0; i < m.selfActive.size(); ++i) for (int k = 0; k < 4; ++k) sa[4 * i + k] = m.selfActive[i][k];
    for (size_t i = 0; i < m.selfEE.size(); ++i) {
        for (int k = 0; k < 4; ++k) see[4 * i + k] = m.selfEE[i][k];
        eeie[2 * i] = m.selfEEeIe[i].first; eeie[2 * i + 1] = m.selfEEeIe[i].second;
    }
    for (size_t i = 0; i < m.selfCCD.size(); ++i) { ccd[2 * i] = m.selfCCD[i].first; ccd[2 * i + 1] = m.selfCCD[i].second; }
    for (size_t i = 0; i < m.envActive.size(); ++i) gr[i] = m.envActive[i];
}

void cipc_oracle_friction_init(void* h) { frictionInitialize(static_cast<Ctx*>(h)->m); }

long long cipc_oracle_system(void* h, double* grad, int* rowptr, int* col, double* val, double* rhs) {
    auto* c = static_cast<Ctx*>(h);
    std::vector<V3> g;
    BHessian BH;
    computeGradientAndHessian(c->m, g, BH, c->o);
    LinearSystem ls;
    assembleSystem(c->m, BH, g, ls);
    if (grad) for (int i = 0; i < c->m.nv(); ++i) { grad[3 * i] = g[i].x; grad[3 * i + 1] = g[i].y; grad[3 * i + 2] = g[i].z; }
    if (rowptr) {
        std::memcpy(rowptr, ls.rowPtr.data(), ls.rowPtr.size() * sizeof(int));
        std::memcpy(col, ls.col.data(), ls.col.size() * sizeof(int));
        std::memcpy(val, ls.val.data(), ls.val.size() * sizeof(double));
        if (rhs) std::memcpy(rhs, ls.rhs.data(), ls.rhs.size() * sizeof(double));
    }
    return ls.nnz;
}

double cipc_oracle_energy(void* h, double kappa) {
    auto* c = static_cast<Ctx*>(h);
    return computeEnergy(c->m, kappa, c->o);
}
double cipc_oracle_total_energy(void* h) {
    auto* c = static_cast<Ctx*>(h);
    return computeEnergy(c->m, c->m.kappa, c->o);
}

void cipc_oracle_step_bounds(void* h, const double* dirIn, double alphaIn, double* out) {
    auto* c = static_cast<Ctx*>(h);
    Mesh& m = c->m;
    std::vector<V3> dir(m.nv());
    for (int i = 0; i < m.nv(); ++i) dir[i] = V3(dirIn[3 * i], dirIn[3 * i + 1], dirIn[3 * i + 2]);
    double a = 1.0;
    limitStepByGround(m, dir, 0.8, a);
    out[0] = a;
    double p = alphaIn;
    selfLargestFeasibleStep(m, dir, 0.8, p);
    out[1] = p;
    double mx = 0;
    for (int v : m.surfVerts) mx = std::max(mx, norm(dir[v]));
    out[2] = mx > 0 ? std::sqrt(m.Hhat) / (mx * 2.0) : 1.0;
    double f = alphaIn;
    c->bp.buildSwept(m, dir, f);
    selfLargestFeasibleStepCCD(m, c->bp, dir, 0.8, f);
    out[3] = f;
    c->bp.build(m);
}

int cipc_oracle_intersected(void* h) {
    auto* c = static_cast<Ctx*>(h);
    c->bp.build(c->m);
    return isIntersected(c->m, c->bp) ? 1 : 0;
}

static V3 at(const double* p, int i) { return V3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
double cipc_oracle_pt_ccd(const double* p, const double* d, double eta) {
    return pointTriangleCCD(at(p, 0), at(p, 1), at(p, 2), at(p, 3), at(d, 0), at(d, 1), at(d, 2), at(d, 3), eta, 0.0);
}
double cipc_oracle_ee_ccd(const double* p, const double* d, double eta) {
    return edgeEdgeCCD(at(p, 0), at(p, 1), at(p, 2), at(p, 3), at(d, 0), at(d, 1), at(d, 2), at(d, 3), eta, 0.0);
}

void cipc_oracle_snh(const double* Fin, double u, double r, double* P, double* H, double* psi) {
    M3 F;
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) F.a[a][b] = Fin[3 * a + b];
    M3 p = snhPK1(F, u, r);
    for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) P[3 * a + b] = p.a[a][b];
    Mat<9, 9> h = snhHessian(F, u, r);
    for (int a = 0; a < 9; ++a) for (int b = 0; b < 9; ++b) H[9 * a + b] = h.a[a][b];
    *psi = snhEnergyDensity(F, u, r);
}

// One hinge element: positions x12 and rest positions rest12 of (edge start,
// edge end, first opposite, second opposite); returns 0.5 k w d^2 and fills
// the gradient (12) and the PSD-projected Hessian (144) when given.
double cipc_oracle_hinge(const double* x12, const double* rest12, double k, double* g, double* H) {
    Mesh m;
    for (int i = 0; i < 4; ++i) m.x.push_back(V3(rest12[3 * i], rest12[3 * i + 1], rest12[3 * i + 2]));
    m.tris.push_back({0, 1, 2});
    m.tris.push_back({0, 3, 1});
    prepareHingeBending(m);
    if (m.hinges.size() != 1) return std::nan("");
    std::vector<V3> x;
    for (int i = 0; i < 4; ++i) x.push_back(V3(x12[3 * i], x12[3 * i + 1], x12[3 * i + 2]));
    HingeBend hb = m.hinges[0];
    // keep the caller's vertex order (the hinge list sorts the edge)
    hb.v[0] = 0; hb.v[1] = 1; hb.v[2] = 2; hb.v[3] = 3;
    const double l = norm(m.x[1] - m.x[0]);
    hb.weight = l * l / (norm(cross(m.x[1] - m.x[0], m.x[2] - m.x[0])) + norm(cross(m.x[1] - m.x[0], m.x[3] - m.x[0])));
    hb.rest = hingeAngle(m.x[0], m.x[1], m.x[2], m.x[3], nullptr, nullptr);
    return hingeEnergy(hb, x, k, g, H);
}

double cipc_oracle_distance(int kind, const double* pts, double* g, double* H) {
    V3 p[4];
    int np = kind == 0 ? 2 : (kind == 1 ? 3 : 4);
    for (int i = 0; i < np; ++i) p[i] = at(pts, i);
    distanceGradHess(kind, p, g, H);
    switch (kind) {
    case 0: return dPP(p[0], p[1]);
    case 1: return dPE(p[0], p[1], p[2]);
    case 2: return dPT(p[0], p[1], p[2], p[3]);
    case 3: return dEE(p[0], p[1], p[2], p[3]);
    default: return crossSqNormEE(p[0], p[1], p[2], p[3]);
    }
}

int cipc_oracle_linear_solve(int nv, const int* rowptr, const int* col, const double* val, const double* rhs, double* sol,
                             int method, double tol, int maxIter, int* iters, double* relres, int threads,
                             const double* xyz) {
    try {
        LinearSystem ls;
        int n = 3 * nv;
        ls.rowPtr.assign(rowptr, rowptr + n + 1);
        ls.col.assign(col, col + rowptr[n]);
        ls.val.assign(val, val + rowptr[n]);
        ls.rhs.assign(rhs, rhs + n);
        SolverOptions o;
        o.linear = method; o.pcgRelTol = tol; o.pcgMaxIter = maxIter; o.threads = threads > 0 ? threads : 1;
        solveSystem(ls, nv, o, xyz);
        std::memcpy(sol, ls.sol.data(), n * sizeof(double));
        if (iters) *iters = ls.pcgIters;
        if (relres) *relres = ls.pcgRelResidual;
        return 0;
    } catch (const std::exception&) {
        return 1;
    }
}

}  // extern "C"
