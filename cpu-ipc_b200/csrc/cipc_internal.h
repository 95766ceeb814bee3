// Internal state of one GPU simulation context and the launchers each
// translation unit exports.  Not part of the public C ABI (include/cipc_gpu.h).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <chrono>
#include <stdexcept>
#include <cstdint>
#include <string>
#include <vector>

#define CIPC_CUDA(call)                                                                          \
    do {                                                                                         \
        cudaError_t e__ = (call);                                                                \
        if (e__ != cudaSuccess)                                                                  \
            throw cipc::CudaError(std::string(#call) + ": " + cudaGetErrorString(e__));          \
    } while (0)

namespace cipc {

// Number of this library's kernel launches since load (CUB sorts/scans are
// not counted).  Every launch goes through launch() below.
extern long long g_kernelLaunches;

template <class... KArgs, class... Args>
inline void launch(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t stream, Args&&... args) {
    ++g_kernelLaunches;
    kernel<<<grid, block, smem, stream>>>(static_cast<KArgs>(args)...);
}

// Optional CUDA-event timing of one kernel family on the context's stream:
// when enabled, launches of that family are bracketed by events from a
// pool, read back after the timed region.
enum ProfileKind {
    PROF_NONE = 0, PROF_SPMV = 1, PROF_TET = 2, PROF_TRI = 3, PROF_SLOT = 4, PROF_BARRIER = 5, PROF_ACTIVE = 6, PROF_FULLCCD = 7, PROF_PCG = 8
};

struct CudaError : std::runtime_error {
    using std::runtime_error::runtime_error;
};
struct InvalidArgument : std::invalid_argument {
    using std::invalid_argument::invalid_argument;
};

// CIPC_DEBUG_ALLOC=1: every reallocation of a grow-only buffer is timed on
// the host and printed to stderr.
bool debugAlloc();
void reportAlloc(size_t oldBytes, size_t newBytes, double ms);

// Grow-only device buffer.
template <class T>
struct DBuf {
    T* p = nullptr;
    size_t cap = 0;
    // grows to twice the request: buffers sized by contact counts grow for a
    // few steps and then stay (a reallocation costs a device-wide wait and
    // page mapping, tens of milliseconds for the pile's contact buffers)
    void reserve(size_t n) {
        if (n <= cap) return;
        const bool dbg = debugAlloc();
        const auto t0 = dbg ? std::chrono::steady_clock::now() : std::chrono::steady_clock::time_point();
        if (p) cudaFree(p);
        size_t c = n < 64 ? 64 : 2 * n;
        CIPC_CUDA(cudaMalloc(&p, c * sizeof(T)));
        if (dbg) reportAlloc(cap * sizeof(T), c * sizeof(T), std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
        cap = c;
    }
    void free() { if (p) cudaFree(p); p = nullptr; cap = 0; }
    operator T*() const { return p; }
};

// Scalars that kernels read (copied to the device once per change).
struct SimParams {
    double dt, drag, Hhat, Fhat, dTol, kappa, bboxDiag2, newtonThr, meanMass, avgEdge;
    double friction, stretchS, shearS, strainRate, plateRigidity;
    double groundN[3], groundD;
    double softW;
    int useBarrier, applyGravity, quasiStatic;
};

// Device LBVH over primitive boxes (faces or edges).  Node i < n-1 internal,
// n-1 <= i < 2n-1 leaves in Morton order.
struct DevBvh {
    int n = 0;
    DBuf<uint64_t> keys, keysAlt;
    DBuf<int> left, right, parent, leafPrim, flags, escape;
    DBuf<double> lo, hi;       // 3 per node
    DBuf<double> primLo, primHi;  // 3 per primitive
    DBuf<unsigned char> sortTmp;
    DBuf<double> sceneBox;     // 6
    DBuf<double> boxPart;      // 6 per block of the scene-box reduction
    DBuf<float> rec;           // 16 per internal node: both children's boxes (rounded outward) and indices
    DBuf<int> bigCount;        // primitives kept out of the tree (large boxes), tested by every query
    double bigExtent = 0;      // the box width past which a primitive is large
    // spatial-hash backend over the same primitive boxes: (cell key,
    // primitive) pairs sorted by key, and the primitives too large to insert
    int hashPairs = 0;
    DBuf<uint64_t> hashKey, hashKeyAlt;
    DBuf<int> hashPrim, hashPrimAlt, hashCount, hashOffset, hashBig, hashBigFlag;
    DBuf<unsigned char> hashTmp;
};

struct Ctx {
    // sizes
    int nv = 0, nt = 0, nf = 0, nb = 0, nsf = 0, nsv = 0, nse = 0;
    int mixed = 0;             // 0 FP64 Hessian/SpMV, 1 FP32
    int precond = 0;           // 0 block-Jacobi, 1 learned
    int broadPhase = 0;        // CIPC_BROAD_PHASE_LBVH or CIPC_BROAD_PHASE_SPATIAL_HASH
    double pcgTol = 1e-6;
    int pcgMaxIter = 10000;
    SimParams P;
    cudaStream_t s = nullptr;
    std::string lastError;
    int stepIndex = 0;
    // relative coplanarity tolerance of the segment-triangle intersection
    // test (COPLANAR_TOL); 0 selects the reference's exact rule
    double coplanarTol = 1e-12;
    // a tensor-core completion wait timed out: the network's forward pass is
    // refused for the rest of the context's life
    bool tcFault = false;
    long long hostSyncs = 0;  // host waits on the context's stream (hostSync)
    DBuf<double> stepScal;  // device scalars of the chained step bounds
    DBuf<int2> ccdPairs;    // candidate pairs of the full edge-edge CCD (query, candidate)
    DBuf<int> ccdPairCount; // their number (may exceed the buffer: the caller grows it and runs again)
    // hook at the linear-solve seam (NewtonLinearSystem::solve): Adam
    // iterations of the network on every assembled Newton system, and/or a
    // dump of every system to files in dumpDir
    int hookTrainIters = 0, hookTrainProbes = 4;
    double hookTrainLr = 1e-3;
    unsigned long long hookTrainSeed = 0;
    long long hookSystems = 0;  // systems the hook has seen
    std::string dumpDir;

    // host mirrors needed by the driver
    std::vector<int> hBtype, hSoftIdx, hDirIdx;
    int dirMotion = 0, softMotion = 0;
    double dirRate = 0, softRate = 0;

    // state (3*nv doubles unless noted)
    DBuf<double> x, x0, xt, vp, vel, rest, dir, grad, mass, softTarget;
    DBuf<int> btype, softIdx, dirIdx;
    // topology and rest data
    DBuf<int> tets, tris, bendV, faces, surfVerts, edges;
    DBuf<double> DmInv, vol, tetMu, tetLam, DmInv2, area, bendQ;
    DBuf<double> hingeW, hingeTh0;  // dihedral-angle bending: per hinge weight and rest angle (bendQ unused)
    int hinge = 0;                  // bending elements are dihedral-angle hinges

    // static symmetric BSR pattern (elements), full storage
    int nnzb = 0;
    DBuf<int> rowPtr, colIdx, diagSlot;
    std::vector<int> hRowPtr;  // host copy of rowPtr (static pattern)
    DBuf<int> hcPtr, hcIdx;    // per slot: element-block contributions (bit 31 = transpose)
    DBuf<int> gcPtr, gcIdx;    // per vertex: element gradient contributions
    DBuf<double> valD, constD;  // static values (FP64) and the constant bending part
    DBuf<float> valF;
    DBuf<double> elemHD;       // element lower blocks, 9 per block
    DBuf<float> elemHF;
    DBuf<double> elemG;        // element gradient rows, 3 per entry
    int nElemBlocks = 0, nElemGrad = 0;
    DBuf<double> vtxGrad, diagExtra;  // per-vertex accumulators (3 and 9 per vertex)

    // contact sets
    int nSelf = 0, nPT = 0, nEE = 0, nPPE = 0, nMoll = 0, nCcdPT = 0, nCcdEE = 0, nGround = 0;
    long long nPPERaw = 0;
    DBuf<int> selfActive;      // 4 per contact
    DBuf<int> selfEE, eeIe;    // 4 and 2 per mollified contact
    DBuf<uint64_t> ccdPT, ccdEE;
    DBuf<int> ground;
    DBuf<uint64_t> kPT, kEE, kMoll, kPPE, kTmp;
    DBuf<uint64_t> uniq;
    DBuf<int> counts, runs;
    DBuf<int> counters;        // device counters for candidate emission
    // friction (lagged at step start)
    int nFric = 0, nFricG = 0;
    DBuf<int> fricSet, fricGround;
    DBuf<double> fricLambda, fricCoord, fricBasis, fricGLambda;
    // close constraints for the kappa update
    int nCloseG = 0, nCloseS = 0;
    DBuf<int> closeG, closeS;
    DBuf<double> closeGVal, closeSVal;

    // dynamic (contact) contributions
    int nDynG = 0, nDynH = 0, nDynB = 0;
    DBuf<int> dynGKey, dynGKeyAlt, dynGIdx, dynGIdxAlt, dynGStart, dynGEnd;
    DBuf<double> dynGVal;
    DBuf<uint64_t> dynHKey, dynHKeyAlt;
    DBuf<int> dynHIdx, dynHIdxAlt;
    DBuf<double> dynHValD;
    DBuf<float> dynHValF;
    DBuf<int> dynRowStart, dynRowEnd, dynCol, dynSrcStart;
    DBuf<double> dynBD;
    DBuf<float> dynBF;
    DBuf<double> barrierUpper;      // packed upper triangles of the self-contact barrier Hessians (78 per contact)
    DBuf<unsigned char> groundTmp;  // temporary storage of the ground-set selection (runs beside the PP/PE encoding)
    DBuf<unsigned char> sortTmp;

    // PCG
    DBuf<double> rhs, sol, r, z, p, Ap, Dinv, red, corrX, corrR;
    DBuf<float> rF, zF, pF, ApF, xF, DinvF;
    int lastPcgIters = 0;
    double lastPcgRelRes = 0;
    long long pcgItersTotal = 0;

    int lastPcgLaunchIters = 0;
    DBuf<unsigned> pcgBar;              // grid-barrier counters of the persistent PCG
    DBuf<double> pcgPipe, pcgParts;     // pipelined PCG: six recurrence vectors, two sets of partial sums
    // the factor packed for the streaming PCG: lower part (columns <= row) and
    // transposed part (columns >= row, diagonal transposed) of the static
    // slots as compact rows of FP16 blocks (9 halves each); the index lists
    // depend only on the static pattern and are built once
    DBuf<int> gLptr, gLcol, gLslot, gUptr, gUcol, gUslot;
    DBuf<uint16_t> gLval, gUval;
    int nGL = 0, nGU = 0;
    bool factorPacked = false;
    int pcgSliceMax = -1;               // cached pipelined PCG: largest static-slot count of a block's rows
    int pcgSliceRows = 0;               // the block row count pcgSliceMax was computed for
    bool assembled = false;             // a Newton system has been assembled

    // learned preconditioner: network weights (FP32 master, BF16 copy, Adam
    // state), graph features and activations of the current system, and the
    // factor G on the IC(0) pattern (slot-aligned with the static and contact
    // BSR: lower slots G_ij, mirror slots G_ij^T, diagonal slots G_ii)
    DBuf<float> mpW, mpG, mpM, mpV;
    DBuf<unsigned short> mpWb;
    int mpStep = 0;
    bool mpReady = false, mpMirrorReady = false, mpFactorReady = false;
    long long mpFallbacks = 0;
    DBuf<double> mpS;                   // 9 per vertex: inverse Cholesky factor of the diagonal block
    DBuf<double> mpT;                   // PCG temporary (3 per vertex)
    DBuf<float> mpNodeF, mpEdgeF, mpEdgeFD;
    DBuf<int> mpMirS, mpMirD, mpDeg, mpRowS, mpRowE;
    DBuf<float> mpH, mpAgg, mpES, mpED, mpHeadD;
    DBuf<float> mpGS, mpGD;
    DBuf<float> mpVec, mpDGS, mpDGD, mpDH, mpDES, mpDED, mpDAgg, mpDS, mpDSD;
    DBuf<float> mpBD, mpBX, mpPart;     // backward: per-item gradients, second input block, split-K partials
    DBuf<unsigned char> mpLowS, mpLowD; // 1 for lower slots of the static / contact pattern
    DBuf<int> mpFlatS, mpFlatD;         // flat lower-edge lists: slot, row, column (3 arrays each, packed)
    int nFlatS = -1, nFlatD = 0;
    DBuf<int> mpScanTmpI;               // row counts and offsets of the flat lists
    DBuf<unsigned char> mpScanTmp;

    // collision structures
    DevBvh faceTree, edgeTree;
    DBuf<double> sweptPt;     // 6 per surface vertex
    DBuf<double> scratch;     // reduction scratch
    DBuf<double> sums;         // SUM_SLOTS device sums read back together
    DBuf<int> status;
    DBuf<double> scal;        // device scalars
    DBuf<double> energyBuf;

    // kernel-family timing (ProfileKind): event pairs recorded on c.s
    int profKind = PROF_NONE;
    std::vector<cudaEvent_t> profEv;
    int profUsed = 0;
};

inline void profBegin(Ctx& c, int kind) {
    if (c.profKind == kind && c.profUsed + 2 <= (int)c.profEv.size()) cudaEventRecord(c.profEv[c.profUsed], c.s);
}
inline void profEnd(Ctx& c, int kind) {
    if (c.profKind == kind && c.profUsed + 2 <= (int)c.profEv.size()) {
        cudaEventRecord(c.profEv[c.profUsed + 1], c.s);
        c.profUsed += 2;
    }
}

// ---- launchers (elastic.cu) ----
// The host waits for the context's stream (counted: the host round trips of
// the Newton driver).
inline void hostSync(Ctx& c) {
    ++c.hostSyncs;
    CIPC_CUDA(cudaStreamSynchronize(c.s));
}

void buildStaticPattern(Ctx& c, const std::vector<int>& tets, const std::vector<int>& tris, const std::vector<int>& bendV);
void assembleElastic(Ctx& c);          // vtxGrad, diagExtra, element blocks, static BSR values, element gradient
void tetGradient(Ctx& c);              // elemG of the tetrahedra only (no Hessian)
double elasticEnergy(Ctx& c);          // (SNH + BW + bending) * dt^2 + inertia + soft, FP64
void elasticEnergySums(Ctx& c, int slot0);
double elasticEnergyCombine(const Ctx& c, const double* h);
void gatherGradient(Ctx& c);           // grad = vtxGrad + element + dynamic contributions
void initKappaGradE(Ctx& c, double* gE);  // inertia + tet elastic gradient into device buffer gE

// ---- launchers (collision.cu) ----
void buildBvh(Ctx& c, DevBvh& t, int n);
void computeFaceBoxes(Ctx& c, const double* x, const double* d, double step, bool swept, const double* stepPtr = nullptr);
void computeEdgeBoxes(Ctx& c, const double* x, const double* d, double step, bool swept, const double* stepPtr = nullptr);
void buildCollisionSets(Ctx& c, bool rehash);
void groundActiveSet(Ctx& c);
bool isIntersected(Ctx& c);
// Step bounds chained on the device (ground, partial CCD, CFL, full CCD and
// the merge rule of IPCSolver.cpp:943-990) with one read-back.
double stepBoundsDevice(Ctx& c);
void deviceMinTo(Ctx& c, const double* v, int n, double* dst);
void deviceMaxTo(Ctx& c, const double* v, int n, double* dst);
void accdBatch(int n, const int* kind, const double* p, const double* d, double eta, double* toi);  // host arrays
double groundStepBound(Ctx& c);
double partialCCD(Ctx& c, double alpha);
double cflBound(Ctx& c);
double fullCCD(Ctx& c, double alpha);
void dirichletBound(Ctx& c, double& alpha);

// ---- launchers (contact.cu) ----
int contactAssemble(Ctx& c);           // barrier + mollified + friction gradient/Hessian -> dynamic lists; returns collisions
double contactEnergy(Ctx& c, double kappa);
void contactEnergySums(Ctx& c, int slot0);
double contactEnergyCombine(const Ctx& c, double kappa, const double* h);
void frictionInitialize(Ctx& c);
void contactGradientKappa(Ctx& c, double* gc);  // ground + self barrier gradient with coefficient 1
void closeConstraintCheck(Ctx& c, bool& update);
void closeConstraintRecord(Ctx& c);
void constraintMinMax(Ctx& c, double& mn, double& mx, bool& any);
void finalizeDynamic(Ctx& c);          // sort + segment dynamic gradient and Hessian entries

// ---- launchers (pcg.cu) ----
int pcgSolve(Ctx& c);                  // solves A sol = rhs; returns iterations
void spmv(Ctx& c, const double* x, double* y);
void buildRhs(Ctx& c);

// ---- reductions (util.cu) ----
double deviceSum(Ctx& c, const double* v, int n);
constexpr int SUM_SLOTS = 16;
void deviceSumTo(Ctx& c, const double* v, int n, int slot);  // no host sync
void fetchSums(Ctx& c, double* h, int nslots);
double deviceMax(Ctx& c, const double* v, int n);
double deviceMin(Ctx& c, const double* v, int n, double init);
double deviceDot(Ctx& c, const double* a, const double* b, int n);
double deviceInfNorm(Ctx& c, const double* v, int n);
void checkStatus(Ctx& c, const char* stage);

}  // namespace cipc
