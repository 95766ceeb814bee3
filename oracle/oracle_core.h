// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
// anything under oracle/; the shipped library never links it.
//
// Data model of the oracle.  It restates the reference's mesh3D state
// (CPU IPC/SimulationMesh.h:37-129) field by field with plain std:: types.
#pragma once

#include "oracle_math.h"

#include <array>
#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <thread>
#include <utility>
#include <vector>

namespace oracle {

using I2 = std::pair<int, int>;
using I3 = std::array<int, 3>;
using I4 = std::array<int, 4>;

// Encoded contact, CPU IPC/EncodedContact.h:1-40.  Ordering is lexicographic
// over the four ints, which is what the reference's std::map uses.
struct Contact {
    int c[4];
    Contact() : c{-1, -1, -1, -1} {}
    Contact(int a, int b, int d, int e) : c{a, b, d, e} {}
    int& operator[](int i) { return c[i]; }
    int operator[](int i) const { return c[i]; }
    bool operator<(const Contact& o) const {
        for (int i = 0; i < 4; ++i) {
            if (c[i] < o.c[i]) return true;
            if (c[i] > o.c[i]) return false;
        }
        return false;
    }
    bool operator==(const Contact& o) const {
        return c[0] == o.c[0] && c[1] == o.c[1] && c[2] == o.c[2] && c[3] == o.c[3];
    }
};

// Boundary codes, CPU IPC/BoundaryConditions.h:17-36.
inline bool isFree(int t) { return t == 0; }
inline bool isCollider(int t) { return t >= 2; }

// Quadratic bending hinge, CPU IPC/SimulationMesh.h:17-35.
struct QuadBend {
    int v[4];  // edge0, edge1, opposite of first triangle, opposite of second
    Mat<4, 4> Q;
};

// Dihedral-angle (hinge) bending element, CPU IPC/HingeBending.{h,cpp}: the
// edge (v[0], v[1]) and the opposite vertices of its two triangles, the
// weight l0^2 / (2 A0 + 2 A1) and the rest angle.
struct HingeBend {
    int v[4];
    double weight, rest;
};

// Prescribed boundary motions the scenes use.  The reference stores these as
// std::function callbacks (BoundaryConditions.h:39-69); the oracle keeps the
// two closed forms its scenes need.
enum MotionKind { MOTION_NONE = 0, MOTION_TWIST_X = 1 };

struct Mesh {
    // material and solver scalars (SimulationMesh.h:39-83)
    double density = 1000, cloth_density = 200, thickness = 1e-3;
    double E = 1e4, nu = 0.49, clothE = 1e4, shearE = 1e1, bendE = 1e4, strainRate = 1e2;
    double friction = 0.4;
    double lengthRate = 0, volumeRate = 0, stretchS = 0, shearS = 0, plateRigidity = 0;
    double dt = 0.01, drag = 0, Hhat = 1e-6, Fhat = 1e-6, dTol = 1e-18, kappa = 0;
    double bboxDiag2 = 0, newtonThr = 1e-2, meanMass = 0, avgEdge = 0;
    bool use_barrier = true, apply_gravity = true, quasi_static = false;
    // segment-triangle coplanarity: relative tolerance (1e-12), or 0 for the
    // reference's exact rule (signs and det == 0 only)
    double coplanarTol = 1e-12;

    std::vector<V3> x, rest, vel, vprev, xtilde;
    std::vector<I4> tets;
    std::vector<I3> tris;
    std::vector<M3> DmInv;
    std::vector<Mat<2, 2>> DmInv2;
    std::vector<double> vol, area, mass;
    std::vector<double> tetLen, tetVolR;  // per-tet SNH parameters (uniform in the reference)
    std::vector<QuadBend> bend;
    std::vector<HingeBend> hinges;
    std::vector<I4> surface;  // v0, v1, v2, owning tet (or 0 for cloth)
    std::vector<int> surfVerts;
    std::vector<I2> surfEdges;
    std::vector<int> btype;

    // soft target penalty (BoundaryConditions.h:53-69)
    std::vector<int> softIdx;
    std::vector<V3> softTarget;
    double softW = 0;
    int softMotion = MOTION_NONE;
    double softRate = 0;
    // animated Dirichlet vertices (BoundaryConditions.h:39-51)
    std::vector<int> dirIdx;
    int dirMotion = MOTION_NONE;
    double dirRate = 0;

    // contact sets (SimulationMesh.h:84-98)
    std::vector<int> envActive, envActiveLastH;
    std::vector<Contact> selfActive, selfActiveLastH, selfEE;
    std::vector<I2> selfEEeIe, selfCCD;
    std::vector<double> selfLambda, envLambda;
    std::vector<std::array<double, 2>> distCoord;
    std::vector<Mat<3, 2>> tanBasis;
    std::vector<int> closeID;
    std::vector<Contact> closeMID;
    std::vector<double> closeVal, closeMVal;

    V3 groundN{0, 1, 0};
    double groundD = -1;

    int nv() const { return (int)x.size(); }
};

// Block Hessian lists, CPU IPC/ContactMechanics.h:8-22.
struct BHessian {
    std::vector<int> D1;
    std::vector<std::array<int, 2>> D2;
    std::vector<I3> D3;
    std::vector<I4> D4;
    std::vector<M3> H3;
    std::vector<Mat<6, 6>> H6;
    std::vector<Mat<9, 9>> H9;
    std::vector<Mat<12, 12>> H12;
    void clear() { D1.clear(); D2.clear(); D3.clear(); D4.clear(); H3.clear(); H6.clear(); H9.clear(); H12.clear(); }
};

// Axis-aligned box, CPU IPC/LBVH.h:10-19 and LBVH.cpp:139-161.
struct AABB {
    V3 lo{1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
    V3 hi{-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
    void combine(const V3& p) { lo = vmin(lo, p); hi = vmax(hi, p); }
    void combine(const AABB& b) { lo = vmin(lo, b.lo); hi = vmax(hi, b.hi); }
    V3 center() const { return 0.5 * (lo + hi); }
    bool overlaps(const AABB& b, double gap = 0.0) const {
        return !((b.lo.x - hi.x > gap) || (b.lo.y - hi.y > gap) || (b.lo.z - hi.z > gap)
                 || (lo.x - b.hi.x > gap) || (lo.y - b.hi.y > gap) || (lo.z - b.hi.z > gap));
    }
};

// Linear BVH, CPU IPC/LBVH.cpp:163-282.
struct LBVH {
    struct Node { uint32_t parent = 0xFFFFFFFFu, left = 0xFFFFFFFFu, right = 0xFFFFFFFFu, prim = 0xFFFFFFFFu; };
    std::vector<Node> nodes;
    std::vector<AABB> boxes;
    void build(const std::vector<AABB>& prims);
    void query(const AABB& box, double gap, std::vector<int>& out) const;
};

// Broad phase state (CPU IPC/LBVH.h:51-85, CollisionBroadPhase.h:16-80 with the
// LinearBVH backend).
struct BroadPhase {
    LBVH faceTree, edgeTree;
    std::vector<AABB> sweptPointBoxes, faceBoxes, edgeBoxes;
    double sweptQueryRadius = 0;
    void build(const Mesh& m);
    void buildSwept(const Mesh& m, const std::vector<V3>& dir, double step);
};

// Per-step statistics, CPU IPC/IPCSolver.h:12-44 (the fields the oracle fills).
struct StepStats {
    int frame = 0, newton = 0, kappaIters = 0, backtracks = 0, energyBacktracks = 0, intersectionBacktracks = 0;
    int maxEnergyBacktracksPerNewton = 0, newtonOverTwo = 0;
    double collisions = 0, kappa = 0, minDist2 = -1, acceptedStepSum = 0, minStep = 1, maxStep = 0;
    long long groundContacts = 0, selfContacts = 0, mollifiedContacts = 0, matrixNnz = 0;
    long long pcgIterations = 0;
    long long linearSolves = 0;  // numericFactorizations of IPCStepStats (IPCSolver.cpp:1042)
};

struct MultifrontalCache;  // ordering and symbolic factorisation of the last pattern (oracle_multifrontal.cpp)
struct SolverOptions {
    int linear = 0;           // 0 = envelope Cholesky, 1 = block-Jacobi PCG, 2 = multifrontal Cholesky
    double pcgRelTol = 1e-6;  // LinearSolverOptions.h:15
    int pcgMaxIter = 10000;   // LinearSolverOptions.h:16
    int threads = 1;
    // the multifrontal solve keeps its analysis here and reuses it while the
    // matrix pattern is unchanged, as PARDISO keeps phase 11 (PardisoSolver.cpp:182-248)
    mutable std::shared_ptr<MultifrontalCache> mfCache;
};

// ---- simple deterministic parallel-for over index chunks ----
void parallelFor(int n, int threads, const std::function<void(int, int)>& body);

// ---- physics (oracle_physics.cpp) ----
void updateMaterial(Mesh& m);
void initRestState(Mesh& m);
void prepareQuadraticBending(Mesh& m);
void prepareHingeBending(Mesh& m);
// hinge angle and, when g / H are given, its gradient and Hessian in the
// 12 coordinates (x[v0], x[v1], x[v2], x[v3])
double hingeAngle(const V3& x0, const V3& x1, const V3& x2, const V3& x3, double* g, double* H);
// 0.5 k w remainder(theta - rest, 2 pi)^2, and its gradient and PSD-projected Hessian
double hingeEnergy(const HingeBend& hb, const std::vector<V3>& x, double k, double* g, double* H);
void getSurface(Mesh& m);
void updateInertialTarget(Mesh& m);

M3 snhPK1(const M3& F, double u, double r);
Mat<9, 9> snhHessian(const M3& F, double u, double r);
double snhEnergyDensity(const M3& F, double u, double r);

int dTypePT(const V3& v0, const V3& v1, const V3& v2, const V3& v3);
int dTypeEE(const V3& v0, const V3& v1, const V3& v2, const V3& v3);
double dPP(const V3& a, const V3& b);
double dPE(const V3& p, const V3& e0, const V3& e1);
double dPT(const V3& p, const V3& t0, const V3& t1, const V3& t2);
double dEE(const V3& a0, const V3& a1, const V3& b0, const V3& b1);
double crossSqNormEE(const V3& a0, const V3& a1, const V3& b0, const V3& b1);
void barrier(double d, double dHat, double& b);
void barrierG(double d, double dHat, double& g);
void barrierH(double d, double dHat, double& h);
double selfConstraintVal(const Mesh& m, const Contact& c);
double epsX(const Mesh& m, int a0, int a1, int b0, int b1);

// generic distance derivative (exact via jets); n = 2, 3, or 4 points
void distanceGradHess(int kind, const V3* p, double* g, double* H);  // kind 0 PP, 1 PE, 2 PT, 3 EE, 4 crossSqNorm
void crossSqNormGradHess(const V3* p, double* g, double* H);

int computeGradientAndHessian(Mesh& m, std::vector<V3>& g, BHessian& BH, const SolverOptions& o);
double computeEnergy(const Mesh& m, double kappa, const SolverOptions& o);
void frictionInitialize(Mesh& m);
void initKappa(Mesh& m, double& kappa);
void suggestKappa(double& kappa, double Hhat, double bbox2, double meanMass);
void upperBoundKappa(double& kappa, double Hhat, double bbox2, double meanMass);
void postLineSearch(Mesh& m, double& kappa);
V3 motionDirection(int motion, double rate, const V3& x, const V3& rest, double frac, double dt);

// ---- collision (oracle_collision.cpp) ----
void calculateActiveSet(Mesh& m, BroadPhase& bp);
void groundActiveSet(Mesh& m);
double pointTriangleCCD(V3 p, V3 t0, V3 t1, V3 t2, V3 dp, V3 dt0, V3 dt1, V3 dt2, double eta, double thickness);
double edgeEdgeCCD(V3 a0, V3 a1, V3 b0, V3 b1, V3 da0, V3 da1, V3 db0, V3 db1, double eta, double thickness);
void limitStepByGround(const Mesh& m, const std::vector<V3>& dir, double slack, double& step);
void selfLargestFeasibleStep(const Mesh& m, const std::vector<V3>& dir, double slack, double& step);
void selfLargestFeasibleStepCCD(const Mesh& m, BroadPhase& bp, const std::vector<V3>& dir, double slack, double& step);
bool isIntersected(const Mesh& m, BroadPhase& bp);
void buildCollisionSets(Mesh& m, BroadPhase& bp, bool rehash = true);

// ---- solver (oracle_solver.cpp) ----
struct LinearSystem {
    std::vector<int> rowPtr, col;  // lower CSR of the 3N x 3N system (duplicates summed)
    std::vector<double> val;
    std::vector<double> rhs, sol;
    long long nnz = 0;
    int pcgIters = 0;
    double pcgRelResidual = 0;
};
void assembleSystem(const Mesh& m, const BHessian& BH, const std::vector<V3>& g, LinearSystem& ls);
// xyz (3 nv positions, or null) lets the multifrontal ordering cut by coordinates
void solveSystem(LinearSystem& ls, int nv, const SolverOptions& o, const double* xyz = nullptr);
void multifrontalSolve(LinearSystem& ls, int nv, int threads, const double* xyz, MultifrontalCache* cache = nullptr);
std::shared_ptr<MultifrontalCache> newMultifrontalCache();
int solveIPCStep(Mesh& m, BroadPhase& bp, StepStats& stats, int stepIndex, const SolverOptions& o);

}  // namespace oracle
