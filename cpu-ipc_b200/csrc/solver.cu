// Host driver of the GPU IPC time step and the C ABI (include/cipc_gpu.h).
//
// The control flow mirrors the reference's solver so that iteration counts,
// backtracking decisions and kappa updates follow the same rules:
//   solveIPCStep           CPU IPC/IPCSolver.cpp:1079-1336
//   solveBarrierSubproblem CPU IPC/IPCSolver.cpp:890-1064
//   lineSearch             CPU IPC/IPCSolver.cpp:560-749
//   kappa rules            CPU IPC/IPCSolver.cpp:751-869
// Every numeric stage runs on the GPU (elastic.cu, contact.cu, collision.cu,
// pcg.cu); the host only sequences stages and reads back scalars.
#include "../../include/cipc_gpu.h"
#include "cipc_device.cuh"
#include "cipc_internal.h"
#include "fsai.h"
#include "mpnn.h"
#include "scene_setup.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <string>

namespace cipc {

long long g_kernelLaunches = 0;

double fullCCDDir(Ctx& c, const double* d, double alpha);
void rebuildTrees(Ctx& c);

namespace {

constexpr int TB = 256;
inline int blocksFor(int n) { return std::max(1, std::min((n + TB - 1) / TB, 148 * 16)); }

__global__ void stepForwardKernel(int nv, const double* x0, const double* dir, const int* btype, double alpha, int all, double* x) {
    CIPC_KERNEL_LOOP(v, nv) {
        if (all || btype[v] == 0)
            for (int q = 0; q < 3; ++q) x[3 * v + q] = x0[3 * v + q] - alpha * dir[3 * v + q];
    }
}
__global__ void velocityKernel(int nv, const double* x, double* vp, double* vel, double* xt, double dt, int quasi, double g) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int q = 0; q < 3; ++q) {
            double xv = x[3 * v + q];
            double ve = quasi ? 0.0 : (xv - vp[3 * v + q]) / dt;
            vel[3 * v + q] = ve;
            vp[3 * v + q] = xv;
        }
        double gd[3] = {0.0, g * dt * dt, 0.0};
        for (int q = 0; q < 3; ++q) xt[3 * v + q] = vp[3 * v + q] + vel[3 * v + q] * dt + gd[q];
    }
}
__global__ void inertialTargetKernel(int nv, const double* vp, const double* vel, double* xt, double dt, double g) {
    CIPC_KERNEL_LOOP(v, nv) {
        double gd[3] = {0.0, g * dt * dt, 0.0};
        for (int q = 0; q < 3; ++q) xt[3 * v + q] = vp[3 * v + q] + vel[3 * v + q] * dt + gd[q];
    }
}

// Animated boundary motion (twistingBoundaryDirection, Simulator.cpp:24-46):
// the displacement that rotates x about the x axis by the step's angle,
// clockwise or counter-clockwise by the side of the rest position (cs, sn:
// cosine and sine of the angle, evaluated once on the host).  With
// `target` the kernel writes x - displacement (the soft targets), else the
// displacement itself into out (3 per vertex of the list).
__global__ void motionKernel(int n, const int* idx, const double* x, const double* rest, double cs, double sn, int target, double* out) {
    CIPC_KERNEL_LOOP(k, n) {
        const int v = idx[k];
        const double y = x[3 * v + 1], z = x[3 * v + 2], r0 = rest[3 * v];
        double d1 = 0.0, d2 = 0.0;
        if (r0 < 0.0) { d1 = cs * y + sn * z - y; d2 = -sn * y + cs * z - z; }
        else if (r0 > 0.0) { d1 = cs * y - sn * z - y; d2 = sn * y + cs * z - z; }
        if (target) {
            out[3 * k] = x[3 * v]; out[3 * k + 1] = y - d1; out[3 * k + 2] = z - d2;
        } else {
            out[3 * v] = 0.0; out[3 * v + 1] = d1; out[3 * v + 2] = d2;
        }
    }
}

using Clock = std::chrono::steady_clock;
double ms(Clock::time_point a, Clock::time_point b) { return std::chrono::duration<double, std::milli>(b - a).count(); }

void sync(Ctx& c) { hostSync(c); }

void stepForward(Ctx& c, const double* x0, const double* d, double alpha, bool all = false) {
    launch(stepForwardKernel, blocksFor(c.nv), TB, 0, c.s, c.nv, x0, d, c.btype, alpha, all ? 1 : 0, c.x);
}

// Elastic plus contact energy with one read-back of all term sums.
double totalEnergy(Ctx& c, double kappa) {
    elasticEnergySums(c, 0);
    const bool contact = c.nGround || c.nSelf || c.nMoll || c.nFric || c.nFricG;
    if (contact) contactEnergySums(c, 5);
    double h[10];
    fetchSums(c, h, contact ? 10 : 5);
    return elasticEnergyCombine(c, h) + (contact ? contactEnergyCombine(c, kappa, h + 5) : 0.0);
}

void suggestKappa(double& kappa, double Hhat, double bbox2, double meanMass) {
    double d = 1.0e-16 * bbox2, t = d - Hhat;
    double hb = (std::log(d / Hhat) * -2.0 - t * 4.0 / d) + 1.0 / (d * d) * (t * t);
    kappa = 1e13 * meanMass / (4.0e-16 * bbox2 * hb);
}
void upperBoundKappa(double& kappa, double Hhat, double bbox2, double meanMass) {
    double d = 1.0e-16 * bbox2, t = d - Hhat;
    double hb = (std::log(d / Hhat) * -2.0 - t * 4.0 / d) + 1.0 / (d * d) * (t * t);
    double kmax = 100 * 1e13 * meanMass / (4.0e-16 * bbox2 * hb);
    if (kappa > kmax) kappa = kmax;
}

// initKappa (IPCSolver.cpp:770-809); `kappa` may alias c.P.kappa.
void initKappa(Ctx& c, double& kappa) {
    if (c.nGround + c.nSelf == 0) return;
    tetGradient(c);  // elemG holds the tetrahedral gradient at x
    c.scratch.reserve(8 + 1024);
    DBuf<double>& gE = c.z;
    DBuf<double>& gc = c.Ap;
    gE.reserve(3 * c.nv); gc.reserve(3 * c.nv);
    initKappaGradE(c, gE);
    contactGradientKappa(c, gc);
    double gsum = deviceDot(c, gc, gE, 3 * c.nv);
    double gsnorm = deviceDot(c, gc, gc, 3 * c.nv);
    double minKappa = -gsum / gsnorm;
    if (minKappa > 0.0) kappa = minKappa;
    suggestKappa(minKappa, c.P.Hhat, c.P.bboxDiag2, c.P.meanMass);
    if (kappa < minKappa) kappa = minKappa;
    upperBoundKappa(c.P.kappa, c.P.Hhat, c.P.bboxDiag2, c.P.meanMass);
}

// postLineSearch (IPCSolver.cpp:811-869); kappa is the sub-problem's copy.
void postLineSearch(Ctx& c, double& kappa) {
    if (kappa == 0.0) { initKappa(c, kappa); return; }
    bool update = false;
    closeConstraintCheck(c, update);
    if (update) {
        kappa *= 2.0;
        upperBoundKappa(c.P.kappa, c.P.Hhat, c.P.bboxDiag2, c.P.meanMass);
    }
    closeConstraintRecord(c);
}

struct Stats {
    cipc_step_stats s;
};

// Energy of the point a line search accepted, kept for the next line search
// of the same barrier subproblem: x, the active sets and the lagged friction
// are unchanged in between (assembly, the linear solve and the step bounds
// do not touch them), so the next search starts from the same value it
// would recompute, as long as kappa has not changed.
struct EnergyCache {
    bool valid = false;
    double kappa = 0, E = 0;
};

bool lineSearch(Ctx& c, double& alpha, double kappa, cipc_step_stats& st, EnergyCache& ec) {
    const double E0 = (ec.valid && ec.kappa == kappa) ? ec.E : totalEnergy(c, kappa);
    ec.valid = false;
    double gTp = deviceDot(c, c.grad, c.dir, 3 * c.nv);
    if (!std::isfinite(E0) || !std::isfinite(gTp)) throw std::runtime_error("line search received a non-finite energy or direction");
    CIPC_CUDA(cudaMemcpyAsync(c.x0.p, c.x.p, sizeof(double) * 3 * c.nv, cudaMemcpyDeviceToDevice, c.s));
    stepForward(c, c.x0, c.dir, alpha);
    int nInter = 0;
    if (c.P.useBarrier) {
        rebuildTrees(c);
        while (isIntersected(c)) {
            if (nInter >= 64 || alpha <= std::numeric_limits<double>::epsilon())
                throw std::runtime_error("line search could not find a non-intersecting step");
            nInter++;
            alpha /= 2.0;
            stepForward(c, c.x0, c.dir, alpha);
            rebuildTrees(c);
        }
    }
    buildCollisionSets(c, false);
    double E = totalEnergy(c, kappa);
    int nLS = 0;
    const double LF = alpha;
    auto ok = [&](double e) { return std::isfinite(e) && e < E0; };
    while (!ok(E)) {
        if (nLS >= 64 || alpha <= std::numeric_limits<double>::epsilon() * std::max(1.0, LF)) {
            double thr = c.P.newtonThr * std::sqrt(c.P.bboxDiag2) * c.P.dt;
            if (deviceInfNorm(c, c.dir, 3 * c.nv) < thr) {
                CIPC_CUDA(cudaMemcpyAsync(c.x.p, c.x0.p, sizeof(double) * 3 * c.nv, cudaMemcpyDeviceToDevice, c.s));
                buildCollisionSets(c, true);
                st.energyBacktracks += nLS;
                st.intersectionBacktracks += nInter;
                st.lineSearchBacktracks += nInter + nLS;
                st.maximumEnergyBacktracksPerNewton = std::max(st.maximumEnergyBacktracksPerNewton, nLS);
                if (nLS > 2) ++st.newtonStepsWithMoreThanTwoBacktracks;
                return false;
            }
            throw std::runtime_error("line search failed to find a strict energy decrease");
        }
        alpha *= 0.5;
        ++nLS;
        stepForward(c, c.x0, c.dir, alpha);
        buildCollisionSets(c, true);
        E = totalEnergy(c, kappa);
    }
    bool recomputeAfterE = false;
    if (alpha < LF) {
        bool recompute = false;
        if (c.P.useBarrier) {
            int it = 0;
            while (isIntersected(c)) {
                if (it++ >= 64 || alpha <= std::numeric_limits<double>::epsilon()) throw std::runtime_error("backtracked step remains intersecting");
                alpha /= 2.0;
                nInter++;
                stepForward(c, c.x0, c.dir, alpha);
                rebuildTrees(c);
                recompute = true;
            }
        }
        if (recompute) buildCollisionSets(c, false);
        recomputeAfterE = recompute;
    }
    st.energyBacktracks += nLS;
    st.intersectionBacktracks += nInter;
    st.lineSearchBacktracks += nInter + nLS;
    st.maximumEnergyBacktracksPerNewton = std::max(st.maximumEnergyBacktracksPerNewton, nLS);
    if (nLS > 2) ++st.newtonStepsWithMoreThanTwoBacktracks;
    st.acceptedStepSum += alpha;
    st.minimumAcceptedStep = std::min(st.minimumAcceptedStep, alpha);
    st.maximumAcceptedStep = std::max(st.maximumAcceptedStep, alpha);
    // E was evaluated at the accepted x with the active sets now in place,
    // unless the intersection check moved x afterwards
    if (!recomputeAfterE) {
        ec.valid = true;
        ec.kappa = kappa;
        ec.E = E;
    }
    return true;
}

// Assembly stage: gradient into c.grad, Hessian into the static + contact BSR.
// CIPC_DEBUG_TIMING=1: the assembly's parts timed on the host (with a
// synchronisation after each) and printed to stderr.
static bool debugTiming() {
    static int v = -1;
    if (v < 0) { const char* e = std::getenv("CIPC_DEBUG_TIMING"); v = (e && *e == '1') ? 1 : 0; }
    return v == 1;
}

int assembleAll(Ctx& c) {
    const bool dbg = debugTiming();
    auto t0 = Clock::now();
    assembleElastic(c);
    if (dbg) sync(c);
    auto t1 = Clock::now();
    int coll = contactAssemble(c);
    if (dbg) sync(c);
    auto t2 = Clock::now();
    gatherGradient(c);
    checkStatus(c, "assembly");
    auto t3 = Clock::now();
    if (dbg)
        std::fprintf(stderr, "[assembly] elastic %.3f ms, contact %.3f ms (%d self, %d mollified, %d friction), gradient+status %.3f ms\n", ms(t0, t1),
                     ms(t1, t2), c.nSelf, c.nMoll, c.nFric, ms(t2, t3));
    c.assembled = true;
    return coll;
}

static void requireSystem(const Ctx& c) {
    if (!c.assembled) throw InvalidArgument("no assembled Newton system: step or assemble first");
}

// The Newton system at the solve seam, as a file: magic "CIPCSYS1", then
// int32 nv, nnzb, ndyn, value bytes (4 or 8), frame, Newton index; static
// BSR row pointers (nv+1) and columns (nnzb), values (9 per block), contact
// BSR row starts and ends (nv each), columns (ndyn), values (9 per block);
// FP64 per-vertex diagonal extras (9 nv), right-hand side (3 nv), positions
// (3 nv); int32 boundary types (nv).
static void dumpSystem(Ctx& c, int newton) {
    const int nv = c.nv, nnzb = c.nnzb, ndyn = c.nDynB, vb = c.mixed ? 4 : 8;
    char name[64];
    std::snprintf(name, sizeof(name), "/system_%06d_%03d.bin", c.stepIndex, newton);
    const std::string path = c.dumpDir + name;
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + path);
    auto put = [&](const void* p, size_t bytes) {
        if (bytes && std::fwrite(p, 1, bytes, f) != bytes) { std::fclose(f); throw std::runtime_error("short write to " + path); }
    };
    auto dev = [&](const void* d, size_t bytes) {
        std::vector<char> h(bytes);
        if (bytes) CIPC_CUDA(cudaMemcpy(h.data(), d, bytes, cudaMemcpyDeviceToHost));
        put(h.data(), bytes);
    };
    sync(c);
    const int head[6] = {nv, nnzb, ndyn, vb, c.stepIndex, newton};
    put("CIPCSYS1", 8);
    put(head, sizeof(head));
    dev(c.rowPtr.p, sizeof(int) * (nv + 1));
    dev(c.colIdx.p, sizeof(int) * (size_t)nnzb);
    dev(c.mixed ? (const void*)c.valF.p : (const void*)c.valD.p, (size_t)vb * 9 * nnzb);
    if (ndyn) {
        dev(c.dynRowStart.p, sizeof(int) * nv);
        dev(c.dynRowEnd.p, sizeof(int) * nv);
        dev(c.dynCol.p, sizeof(int) * (size_t)ndyn);
        dev(c.mixed ? (const void*)c.dynBF.p : (const void*)c.dynBD.p, (size_t)vb * 9 * ndyn);
    } else {
        std::vector<int> z(2 * (size_t)nv, 0);
        put(z.data(), sizeof(int) * z.size());
    }
    dev(c.diagExtra.p, sizeof(double) * 9 * nv);
    dev(c.rhs.p, sizeof(double) * 3 * nv);
    dev(c.x.p, sizeof(double) * 3 * nv);
    dev(c.btype.p, sizeof(int) * nv);
    std::fclose(f);
}

void linearSolve(Ctx& c, int newton = 0) {
    buildRhs(c);
    if (c.hookTrainIters > 0 || !c.dumpDir.empty()) {
        if (!c.dumpDir.empty()) dumpSystem(c, newton);
        if (c.hookTrainIters > 0) {
            if (!c.mpReady) mpnnInitWeights(c, 1);
            mpnnPrepare(c);
            for (int it = 0; it < c.hookTrainIters; ++it) {
                mpnnForward(c);
                mpnnLoss(c, c.hookTrainProbes, nullptr, c.hookTrainSeed + 104729ull * (unsigned long long)(c.mpStep + 1), true);
                mpnnAdam(c, c.hookTrainLr);
            }
        }
        ++c.hookSystems;
    }
    pcgSolve(c);
    CIPC_CUDA(cudaMemcpyAsync(c.dir.p, c.sol.p, sizeof(double) * 3 * c.nv, cudaMemcpyDeviceToDevice, c.s));
}

int solveBarrierSubproblem(Ctx& c, double kappa, cipc_step_stats& st) {
    EnergyCache ec;
    int k = 0;
    double beta = 1;
    const int kmin = 6;
    for (; k < 10000; ++k) {
        auto t0 = Clock::now();
        // assembleAll ends with a read of the status word: the stream is idle here
        st.collisions += assembleAll(c);
        auto t1 = Clock::now();
        linearSolve(c, k);
        st.pcgIterations += c.lastPcgIters;
        st.pcgRelativeResidual = std::max(st.pcgRelativeResidual, c.lastPcgRelRes);
        st.matrixBlocks = std::max<long long>(st.matrixBlocks, (long long)c.nnzb + c.nDynB);
        double thr = c.P.newtonThr * std::sqrt(c.P.bboxDiag2) * c.P.dt;
        double dn = deviceInfNorm(c, c.dir, 3 * c.nv);
        auto t2 = Clock::now();
        if (dn < thr) {
            st.assemblyMilliseconds += ms(t0, t1);
            st.linearSolveMilliseconds += ms(t1, t2);
            break;
        }
        // ground bound, partial CCD, CFL bound, full CCD and their merge
        double alpha = stepBoundsDevice(c);
        auto t3 = Clock::now();
        bool accepted = lineSearch(c, alpha, kappa, st, ec);
        sync(c);
        auto t4 = Clock::now();
        if (!accepted) {
            st.assemblyMilliseconds += ms(t0, t1);
            st.linearSolveMilliseconds += ms(t1, t2);
            st.ccdMilliseconds += ms(t2, t3);
            st.lineSearchMilliseconds += ms(t3, t4);
            break;
        }
        // postLineSearch ends with a read-back (its minimum distance): the stream is idle here
        postLineSearch(c, kappa);
        auto t5 = Clock::now();
        st.assemblyMilliseconds += ms(t0, t1);
        st.linearSolveMilliseconds += ms(t1, t2);
        st.ccdMilliseconds += ms(t2, t3);
        st.lineSearchMilliseconds += ms(t3, t4);
        st.postLineSearchMilliseconds += ms(t4, t5);
        if (k + 1 >= kmin) beta = (1 - alpha) * beta;
        if (beta <= thr) break;
    }
    st.newtonIterations += k;
    return k;
}

void solveIPCStep(Ctx& c, cipc_step_stats& st) {
    std::memset(&st, 0, sizeof(st));
    st.frame = c.stepIndex;
    st.minimumAcceptedStep = 1.0;
    st.minConstraintDistance2 = -1.0;
    auto tBegin = Clock::now();
    SimParams& P = c.P;
    upperBoundKappa(P.kappa, P.Hhat, P.bboxDiag2, P.meanMass);
    if (P.kappa < 1e-16) suggestKappa(P.kappa, P.Hhat, P.bboxDiag2, P.meanMass);
    initKappa(c, P.kappa);
    frictionInitialize(c);
    int nv = c.nv;
    // animated boundaries, on the device from the positions at the start of
    // the step (IPCSolver.cpp:1120-1155)
    const int ns = (int)c.hSoftIdx.size(), nd = (int)c.hDirIdx.size();
    if (ns && c.softMotion == CIPC_MOTION_TWIST_X) {
        const double ang = c.softRate * P.dt;
        launch(motionKernel, blocksFor(ns), TB, 0, c.s, ns, (const int*)c.softIdx, (const double*)c.x, (const double*)c.rest, std::cos(ang),
               std::sin(ang), 1, (double*)c.softTarget);
    }
    if (nd && c.dirMotion == CIPC_MOTION_TWIST_X) {
        c.Ap.reserve(3 * (size_t)nv);
        CIPC_CUDA(cudaMemcpyAsync(c.x0.p, c.x.p, sizeof(double) * 3 * nv, cudaMemcpyDeviceToDevice, c.s));
        // the Dirichlet vertices' displacement for the fraction `frac` of the
        // step's rotation (zero elsewhere), from the start-of-step positions x0
        auto dirs = [&](double frac) {
            CIPC_CUDA(cudaMemsetAsync(c.Ap.p, 0, sizeof(double) * 3 * nv, c.s));
            const double ang = c.dirRate * P.dt * frac;
            launch(motionKernel, blocksFor(nd), TB, 0, c.s, nd, (const int*)c.dirIdx, (const double*)c.x0, (const double*)c.rest, std::cos(ang),
                   std::sin(ang), 0, (double*)c.Ap);
        };
        double na = 1;
        dirs(na);
        na = fullCCDDir(c, c.Ap, na);
        dirs(na);
        stepForward(c, c.x0, c.Ap, 1.0, true);
        rebuildTrees(c);
        int ni = 0;
        while (isIntersected(c)) {
            if (ni++ >= 64 || na <= std::numeric_limits<double>::epsilon()) throw std::runtime_error("animated boundary update remains intersecting");
            na /= 2.0;
            dirs(na);
            stepForward(c, c.x0, c.Ap, 1.0, true);
            rebuildTrees(c);
        }
        buildCollisionSets(c, false);
    }
    for (; st.kappaIterations < 64; ++st.kappaIterations) {
        c.nCloseG = c.nCloseS = 0;
        solveBarrierSubproblem(c, P.kappa, st);
        double mn, mx;
        bool any;
        constraintMinMax(c, mn, mx, any);
        if (any) {
            st.minConstraintDistance2 = mn;
            if (mn < P.dTol) break;
            else if (mx < P.Hhat) break;
        } else break;
    }
    if (st.kappaIterations == 64) throw std::runtime_error("IPC kappa loop exceeded its iteration limit");
    ++st.kappaIterations;
    launch(velocityKernel, blocksFor(nv), TB, 0, c.s, nv, c.x, c.vp, c.vel, c.xt, P.dt, P.quasiStatic, P.applyGravity ? -9.8 : 0.0);
    CIPC_CUDA(cudaGetLastError());
    sync(c);
    st.stepMilliseconds = ms(tBegin, Clock::now());
    st.kappa = P.kappa;
    st.groundContacts = c.nGround;
    st.selfContacts = c.nSelf;
    st.mollifiedContacts = c.nMoll;
    c.stepIndex++;
}

template <class T>
void upload(DBuf<T>& d, const std::vector<T>& h) {
    d.reserve(std::max<size_t>(h.size(), 1));
    if (!h.empty()) CIPC_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

Ctx* createContext(const cipc_scene_desc* s, const cipc_linear_options* o) {
    if (!s || s->nv <= 0 || !s->x || !s->btype) throw InvalidArgument("scene needs vertices and boundary types");
    if (s->nt < 0 || s->nf < 0 || (s->nt > 0 && !s->tets) || (s->nf > 0 && !s->tris)) throw InvalidArgument("invalid element arrays");
    if (s->nv >= (1 << 21) - 2) throw InvalidArgument("vertex count exceeds the 2^21 limit of the packed contact keys");
    if (!(s->dt > 0) || !(s->relDhat > 0)) throw InvalidArgument("time step and dHat must be positive");
    if (o && o->backend != CIPC_LINEAR_GPU_PCG) throw InvalidArgument("only the GPU PCG backend is implemented by this library");
    if (s->quad_bending < 0 || s->quad_bending > 2) throw InvalidArgument("bending model must be 0 (none), 1 (quadratic) or 2 (hinge)");
    if (o && o->precision != CIPC_PRECISION_FP64 && o->precision != CIPC_PRECISION_MIXED) throw InvalidArgument("unknown precision");
    if (o && o->preconditioner != CIPC_PRECOND_BLOCK_JACOBI && o->preconditioner != CIPC_PRECOND_LEARNED && o->preconditioner != CIPC_PRECOND_FSAI)
        throw InvalidArgument("unknown preconditioner");
    for (int i = 0; i < 4 * s->nt; ++i)
        if (s->tets[i] < 0 || s->tets[i] >= s->nv) throw InvalidArgument("tetrahedron references an out-of-range vertex");
    for (int i = 0; i < 3 * s->nf; ++i)
        if (s->tris[i] < 0 || s->tris[i] >= s->nv) throw InvalidArgument("triangle references an out-of-range vertex");
    // BoundaryConditionOps::initialize validation (BoundaryConditions.cpp:55-109)
    for (int k = 0; k < s->nsoft; ++k) {
        int v = s->softIdx[k];
        if (v < 0 || v >= s->nv || s->btype[v] != 0) throw InvalidArgument("soft boundary vertices must remain free Newton unknowns");
    }
    if (s->nsoft > 0 && !(s->softW > 0)) throw InvalidArgument("soft boundary weight must be finite and positive");
    for (int k = 0; k < s->ndir; ++k) {
        int v = s->dirIdx[k];
        if (v < 0 || v >= s->nv || s->btype[v] == 0) throw InvalidArgument("animated Dirichlet vertices must be marked constrained");
    }
    int dev = 0;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) throw CudaError("no CUDA device is available");
    CIPC_CUDA(cudaGetDevice(&dev));
    auto c = new Ctx();
    try {
        c->nv = s->nv; c->nt = s->nt; c->nf = s->nf;
        if (o) {
            c->mixed = o->precision == CIPC_PRECISION_MIXED;
            c->precond = o->preconditioner;
            c->pcgTol = o->relativeTolerance > 0 ? o->relativeTolerance : 1e-6;
            c->pcgMaxIter = o->maximumIterations > 0 ? o->maximumIterations : 10000;
        }
        SceneInput in;
        in.nv = s->nv; in.nt = s->nt; in.nf = s->nf;
        in.x.assign(s->x, s->x + 3 * (size_t)s->nv);
        in.tets.assign(s->tets, s->tets + 4 * (size_t)s->nt);
        in.tris.assign(s->tris, s->tris + 3 * (size_t)s->nf);
        if (s->tetE) in.tetE.assign(s->tetE, s->tetE + s->nt);
        in.density = s->density; in.cloth_density = s->cloth_density; in.thickness = s->thickness; in.E = s->E; in.nu = s->nu;
        in.clothE = s->clothE; in.shearE = s->shearE; in.bendE = s->bendE; in.strainRate = s->strainRate; in.relDhat = s->relDhat;
        in.quadBending = s->quad_bending == 1;
        in.hingeBending = s->quad_bending == 2;
        for (int k = 0; k < 3; ++k) { in.bboxMin[k] = s->bboxMin[k]; in.bboxMax[k] = s->bboxMax[k]; }
        if (s->surfFaces && s->surfVerts && s->surfEdges) {
            in.hasSurface = true;
            in.faces.assign(s->surfFaces, s->surfFaces + 3 * (size_t)s->nsf);
            in.surfVerts.assign(s->surfVerts, s->surfVerts + s->nsv);
            in.edges.assign(s->surfEdges, s->surfEdges + 2 * (size_t)s->nse);
        }
        SceneRest r;
        setupScene(in, r);
        c->nb = (int)r.bendV.size() / 4;
        c->nsf = (int)r.faces.size() / 3;
        c->nsv = (int)r.surfVerts.size();
        c->nse = (int)r.edges.size() / 2;
        SimParams& P = c->P;
        std::memset(&P, 0, sizeof(P));
        P.dt = s->dt; P.drag = s->drag; P.Hhat = r.Hhat; P.Fhat = r.Fhat; P.dTol = r.dTol; P.kappa = 0; P.bboxDiag2 = r.bboxDiag2;
        P.newtonThr = s->newtonThr; P.meanMass = r.meanMass; P.avgEdge = r.avgEdge; P.friction = s->friction;
        P.stretchS = r.stretchS; P.shearS = r.shearS; P.strainRate = s->strainRate; P.plateRigidity = r.plateRigidity;
        P.groundN[0] = 0; P.groundN[1] = 1; P.groundN[2] = 0; P.groundD = -1;
        P.softW = s->softW;
        P.useBarrier = s->use_barrier; P.applyGravity = s->apply_gravity; P.quasiStatic = s->quasi_static;
        c->hBtype.assign(s->btype, s->btype + s->nv);
        if (s->nsoft > 0) c->hSoftIdx.assign(s->softIdx, s->softIdx + s->nsoft);
        if (s->ndir > 0) c->hDirIdx.assign(s->dirIdx, s->dirIdx + s->ndir);
        c->softMotion = s->softMotion; c->softRate = s->softRate; c->dirMotion = s->dirMotion; c->dirRate = s->dirRate;
        for (int v : c->hSoftIdx) if (v < 0 || v >= s->nv || c->hBtype[v] != 0) throw InvalidArgument("soft boundary vertices must be free");
        for (int v : c->hDirIdx) if (v < 0 || v >= s->nv || c->hBtype[v] == 0) throw InvalidArgument("animated Dirichlet vertices must be marked constrained");
        CIPC_CUDA(cudaStreamCreateWithFlags(&c->s, cudaStreamNonBlocking));
        size_t n3 = 3 * (size_t)s->nv;
        upload(c->x, in.x); upload(c->rest, in.x); upload(c->vp, in.x);
        c->x0.reserve(n3); c->xt.reserve(n3); c->dir.reserve(n3); c->grad.reserve(n3);
        std::vector<double> vel(n3, 0.0);
        if (s->vel) vel.assign(s->vel, s->vel + n3);
        upload(c->vel, vel);
        upload(c->mass, r.mass);
        upload(c->btype, c->hBtype);
        upload(c->tets, in.tets); upload(c->tris, in.tris);
        upload(c->DmInv, r.DmInv); upload(c->vol, r.vol); upload(c->tetMu, r.tetMu); upload(c->tetLam, r.tetLam);
        upload(c->DmInv2, r.DmInv2); upload(c->area, r.area);
        upload(c->bendV, r.bendV); upload(c->bendQ, r.bendQ);
        c->hinge = in.hingeBending ? 1 : 0;
        if (c->hinge) { upload(c->hingeW, r.hingeW); upload(c->hingeTh0, r.hingeTh0); }
        upload(c->faces, r.faces); upload(c->surfVerts, r.surfVerts); upload(c->edges, r.edges);
        upload(c->softIdx, c->hSoftIdx);
        std::vector<double> tgt;
        for (int v : c->hSoftIdx) for (int q = 0; q < 3; ++q) tgt.push_back(in.x[3 * v + q]);
        upload(c->softTarget, tgt);
        upload(c->dirIdx, c->hDirIdx);
        c->status.reserve(4);
        CIPC_CUDA(cudaMemset(c->status.p, 0, sizeof(int)));
        c->counters.reserve(16);
        c->scratch.reserve(2048);
        buildStaticPattern(*c, in.tets, in.tris, r.bendV);
        launch(inertialTargetKernel, blocksFor(c->nv), TB, 0, c->s, c->nv, c->vp, c->vel, c->xt, P.dt, P.applyGravity ? -9.8 : 0.0);
        CIPC_CUDA(cudaGetLastError());
        // rebuildCollisionSets (Simulator.cpp:532-540)
        buildCollisionSets(*c, true);
        // the learned preconditioner starts from its deterministic initial
        // weights (the first-order factor); hosts load trained ones
        if (c->precond == CIPC_PRECOND_LEARNED) mpnnInitWeights(*c, 1);
        sync(*c);
        return c;
    } catch (...) {
        delete c;
        throw;
    }
}

}  // namespace
}  // namespace cipc

using namespace cipc;

struct cipc_gpu_context {
    Ctx* c;
};

static thread_local std::string g_createError;

template <class F>
static int guarded(cipc_gpu_context* h, F f) {
    if (!h || !h->c) return CIPC_ERR_INVALID_ARGUMENT;
    try {
        f(*h->c);
        return CIPC_OK;
    } catch (const InvalidArgument& e) {
        h->c->lastError = e.what();
        return CIPC_ERR_INVALID_ARGUMENT;
    } catch (const CudaError& e) {
        h->c->lastError = e.what();
        return CIPC_ERR_CUDA;
    } catch (const std::exception& e) {
        h->c->lastError = e.what();
        std::string m = e.what();
        if (m.find("device status") != std::string::npos) return CIPC_ERR_DEVICE_STATUS;
        if (m.find("did not converge") != std::string::npos) return CIPC_ERR_NOT_CONVERGED;
        return CIPC_ERR_RUNTIME;
    }
}

extern "C" {

const char* cipc_gpu_create_error(void) { return g_createError.c_str(); }

int cipc_gpu_create(const cipc_scene_desc* scene, const cipc_linear_options* options, cipc_gpu_context** out) {
    if (!out) return CIPC_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    try {
        Ctx* c = createContext(scene, options);
        *out = new cipc_gpu_context{c};
        g_createError.clear();
        return CIPC_OK;
    } catch (const InvalidArgument& e) {
        g_createError = e.what();
        return CIPC_ERR_INVALID_ARGUMENT;
    } catch (const CudaError& e) {
        g_createError = e.what();
        return CIPC_ERR_CUDA;
    } catch (const std::exception& e) {
        g_createError = e.what();
        return CIPC_ERR_RUNTIME;
    }
}

void cipc_gpu_destroy(cipc_gpu_context* h) {
    if (!h) return;
    if (h->c) {
        if (h->c->s) cudaStreamSynchronize(h->c->s);
        Ctx& c = *h->c;
        DBuf<double>* ds[] = {&c.x, &c.x0, &c.xt, &c.vp, &c.vel, &c.rest, &c.dir, &c.grad, &c.mass, &c.softTarget, &c.DmInv, &c.vol, &c.tetMu,
                              &c.tetLam, &c.DmInv2, &c.area, &c.bendQ, &c.hingeW, &c.hingeTh0, &c.valD, &c.constD, &c.elemHD, &c.elemG, &c.vtxGrad, &c.diagExtra,
                              &c.fricLambda, &c.fricCoord, &c.fricBasis, &c.fricGLambda, &c.closeGVal, &c.closeSVal, &c.dynGVal, &c.dynHValD,
                              &c.dynBD, &c.rhs, &c.sol, &c.r, &c.z, &c.p, &c.Ap, &c.Dinv, &c.red, &c.corrX, &c.corrR, &c.sweptPt, &c.scratch,
                              &c.scal, &c.energyBuf, &c.sums, &c.mpS, &c.mpT, &c.pcgPipe, &c.pcgParts,
                              &c.faceTree.lo, &c.faceTree.hi, &c.faceTree.primLo, &c.faceTree.primHi, &c.faceTree.sceneBox, &c.edgeTree.lo,
                              &c.edgeTree.hi, &c.edgeTree.primLo, &c.edgeTree.primHi, &c.edgeTree.sceneBox, &c.faceTree.boxPart, &c.edgeTree.boxPart};
        for (auto* d : ds) d->free();
        DBuf<float>* fs[] = {&c.valF, &c.elemHF, &c.dynHValF, &c.dynBF, &c.rF, &c.zF, &c.pF, &c.ApF, &c.xF, &c.DinvF, &c.mpW, &c.mpG, &c.mpM, &c.mpV,
                             &c.mpNodeF, &c.mpEdgeF, &c.mpEdgeFD, &c.mpH, &c.mpAgg, &c.mpES, &c.mpED, &c.mpHeadD, &c.mpGS, &c.mpGD,
                             &c.mpVec, &c.mpDGS, &c.mpDGD, &c.mpDH, &c.mpDES, &c.mpDED, &c.mpDAgg, &c.mpDS, &c.mpDSD,
                             &c.mpBD, &c.mpBX, &c.mpPart, &c.faceTree.rec, &c.edgeTree.rec};
        for (auto* d : fs) d->free();
        DBuf<int>* is[] = {&c.btype, &c.softIdx, &c.dirIdx, &c.tets, &c.tris, &c.bendV, &c.faces, &c.surfVerts, &c.edges, &c.rowPtr, &c.colIdx,
                           &c.diagSlot, &c.hcPtr, &c.hcIdx, &c.gcPtr, &c.gcIdx, &c.selfActive, &c.selfEE, &c.eeIe, &c.ground, &c.counts, &c.runs,
                           &c.counters, &c.fricSet, &c.fricGround, &c.closeG, &c.closeS, &c.dynGKey, &c.dynGKeyAlt, &c.dynGIdx, &c.dynGIdxAlt,
                           &c.dynGStart, &c.dynGEnd, &c.dynHIdx, &c.dynHIdxAlt, &c.dynRowStart, &c.dynRowEnd, &c.dynCol, &c.dynSrcStart, &c.status,
                           &c.faceTree.left, &c.faceTree.right, &c.faceTree.parent, &c.faceTree.leafPrim, &c.faceTree.flags, &c.faceTree.escape,
                           &c.edgeTree.left, &c.edgeTree.right, &c.edgeTree.parent, &c.edgeTree.leafPrim, &c.edgeTree.flags, &c.edgeTree.escape, &c.mpMirS, &c.mpMirD, &c.mpDeg,
                           &c.mpRowS, &c.mpRowE};
        for (auto* d : is) d->free();
        c.mpWb.free(); c.mpLowS.free(); c.mpLowD.free(); c.pcgBar.free();
        DBuf<uint64_t>* us[] = {&c.ccdPT, &c.ccdEE, &c.kPT, &c.kEE, &c.kMoll, &c.kPPE, &c.kTmp, &c.uniq, &c.dynHKey, &c.dynHKeyAlt,
                                &c.faceTree.keys, &c.faceTree.keysAlt, &c.edgeTree.keys, &c.edgeTree.keysAlt};
        for (auto* d : us) d->free();
        c.sortTmp.free(); c.groundTmp.free(); c.barrierUpper.free(); c.ccdPairs.free(); c.ccdPairCount.free(); c.stepScal.free(); c.faceTree.sortTmp.free(); c.edgeTree.sortTmp.free();
        c.gLptr.free(); c.gLcol.free(); c.gLslot.free(); c.gUptr.free(); c.gUcol.free(); c.gUslot.free(); c.gLval.free(); c.gUval.free();
        for (DevBvh* t : {&c.faceTree, &c.edgeTree}) {
            t->hashKey.free(); t->hashKeyAlt.free(); t->hashPrim.free(); t->hashPrimAlt.free(); t->hashCount.free(); t->hashOffset.free();
            t->hashBig.free(); t->hashBigFlag.free(); t->hashTmp.free(); t->bigCount.free();
        }
        for (cudaEvent_t e : c.profEv) cudaEventDestroy(e);
        if (c.s) cudaStreamDestroy(c.s);
        delete h->c;
    }
    delete h;
}

const char* cipc_gpu_last_error(const cipc_gpu_context* h) { return (h && h->c) ? h->c->lastError.c_str() : "invalid context"; }

int cipc_gpu_step(cipc_gpu_context* h, cipc_step_stats* stats) {
    return guarded(h, [&](Ctx& c) {
        cipc_step_stats st;
        solveIPCStep(c, st);
        if (stats) *stats = st;
    });
}

static DBuf<double>* stateBuf(Ctx& c, int which) {
    switch (which) {
    case 0: return &c.x; case 1: return &c.vel; case 2: return &c.vp; case 3: return &c.xt; case 4: return &c.rest;
    default: throw InvalidArgument("unknown state field");
    }
}

int cipc_gpu_get_state(cipc_gpu_context* h, int which, double* out) {
    return guarded(h, [&](Ctx& c) {
        if (!out) throw InvalidArgument("null output");
        hostSync(c);
        CIPC_CUDA(cudaMemcpy(out, stateBuf(c, which)->p, sizeof(double) * 3 * c.nv, cudaMemcpyDeviceToHost));
    });
}

int cipc_gpu_set_state(cipc_gpu_context* h, int which, const double* in) {
    return guarded(h, [&](Ctx& c) {
        if (!in) throw InvalidArgument("null input");
        if (which == 4) throw InvalidArgument("rest positions are fixed at creation");
        hostSync(c);
        CIPC_CUDA(cudaMemcpy(stateBuf(c, which)->p, in, sizeof(double) * 3 * c.nv, cudaMemcpyHostToDevice));
    });
}

int cipc_gpu_get_scalars(cipc_gpu_context* h, double* o) {
    return guarded(h, [&](Ctx& c) {
        const SimParams& P = c.P;
        double v[14] = {P.kappa, P.Hhat, P.Fhat, P.dTol, P.bboxDiag2, P.meanMass, P.avgEdge, 0, 0, P.stretchS, P.shearS, P.plateRigidity, P.dt, P.newtonThr};
        if (c.nt > 0) {
            CIPC_CUDA(cudaMemcpy(&v[7], c.tetMu.p, sizeof(double), cudaMemcpyDeviceToHost));
            CIPC_CUDA(cudaMemcpy(&v[8], c.tetLam.p, sizeof(double), cudaMemcpyDeviceToHost));
        }
        std::memcpy(o, v, sizeof(v));
    });
}

int cipc_gpu_set_kappa(cipc_gpu_context* h, double kappa) {
    return guarded(h, [&](Ctx& c) { c.P.kappa = kappa; });
}

int cipc_gpu_set_broad_phase(cipc_gpu_context* h, int backend) {
    return guarded(h, [&](Ctx& c) {
        if (backend != CIPC_BROAD_PHASE_LBVH && backend != CIPC_BROAD_PHASE_SPATIAL_HASH) throw InvalidArgument("unknown broad-phase backend");
        if (backend != c.broadPhase) {
            c.broadPhase = backend;
            rebuildTrees(c);  // the structures the next query reads
            sync(c);
        }
    });
}

int cipc_gpu_set_intersection_rule(cipc_gpu_context* h, int rule) {
    return guarded(h, [&](Ctx& c) {
        if (rule != CIPC_INTERSECT_TOLERANT && rule != CIPC_INTERSECT_REFERENCE) throw InvalidArgument("unknown intersection rule");
        c.coplanarTol = rule == CIPC_INTERSECT_REFERENCE ? 0.0 : 1e-12;
    });
}

int cipc_gpu_get_counts(cipc_gpu_context* h, long long* o) {
    return guarded(h, [&](Ctx& c) {
        o[0] = c.nv; o[1] = c.nsf; o[2] = c.nsv; o[3] = c.nse; o[4] = c.nb; o[5] = c.nt; o[6] = c.nf; o[7] = c.nnzb; o[8] = c.nDynB;
    });
}

int cipc_gpu_get_surface(cipc_gpu_context* h, int* faces, int* verts, int* edges) {
    return guarded(h, [&](Ctx& c) {
        CIPC_CUDA(cudaMemcpy(faces, c.faces.p, sizeof(int) * 3 * c.nsf, cudaMemcpyDeviceToHost));
        CIPC_CUDA(cudaMemcpy(verts, c.surfVerts.p, sizeof(int) * c.nsv, cudaMemcpyDeviceToHost));
        CIPC_CUDA(cudaMemcpy(edges, c.edges.p, sizeof(int) * 2 * c.nse, cudaMemcpyDeviceToHost));
    });
}

int cipc_gpu_build_collision_sets(cipc_gpu_context* h, long long* o) {
    return guarded(h, [&](Ctx& c) {
        buildCollisionSets(c, true);
        sync(c);
        if (o) { o[0] = c.nSelf; o[1] = c.nMoll; o[2] = (long long)c.nCcdPT + c.nCcdEE; o[3] = c.nGround; }
    });
}

int cipc_gpu_get_active_sets(cipc_gpu_context* h, int* sa, int* see, int* eeie, int* ccd, int* gr) {
    return guarded(h, [&](Ctx& c) {
        sync(c);
        if (sa && c.nSelf) CIPC_CUDA(cudaMemcpy(sa, c.selfActive.p, sizeof(int) * 4 * c.nSelf, cudaMemcpyDeviceToHost));
        if (see && c.nMoll) CIPC_CUDA(cudaMemcpy(see, c.selfEE.p, sizeof(int) * 4 * c.nMoll, cudaMemcpyDeviceToHost));
        if (eeie && c.nMoll) CIPC_CUDA(cudaMemcpy(eeie, c.eeIe.p, sizeof(int) * 2 * c.nMoll, cudaMemcpyDeviceToHost));
        if (ccd) {
            std::vector<uint64_t> a(c.nCcdPT), b(c.nCcdEE);
            if (c.nCcdPT) CIPC_CUDA(cudaMemcpy(a.data(), c.ccdPT.p, sizeof(uint64_t) * c.nCcdPT, cudaMemcpyDeviceToHost));
            if (c.nCcdEE) CIPC_CUDA(cudaMemcpy(b.data(), c.ccdEE.p, sizeof(uint64_t) * c.nCcdEE, cudaMemcpyDeviceToHost));
            for (int i = 0; i < c.nCcdPT; ++i) { ccd[2 * i] = -(int)(a[i] >> 32) - 1; ccd[2 * i + 1] = (int)(a[i] & 0xffffffffu); }
            for (int i = 0; i < c.nCcdEE; ++i) {
                ccd[2 * (c.nCcdPT + i)] = (int)(b[i] >> 32);
                ccd[2 * (c.nCcdPT + i) + 1] = (int)(b[i] & 0xffffffffu);
            }
        }
        if (gr && c.nGround) CIPC_CUDA(cudaMemcpy(gr, c.ground.p, sizeof(int) * c.nGround, cudaMemcpyDeviceToHost));
    });
}

int cipc_gpu_friction_init(cipc_gpu_context* h) {
    return guarded(h, [&](Ctx& c) { frictionInitialize(c); sync(c); });
}

int cipc_gpu_assemble(cipc_gpu_context* h, double* grad, int* collisions) {
    return guarded(h, [&](Ctx& c) {
        int coll = assembleAll(c);
        sync(c);
        if (collisions) *collisions = coll;
        if (grad) CIPC_CUDA(cudaMemcpy(grad, c.grad.p, sizeof(double) * 3 * c.nv, cudaMemcpyDeviceToHost));
    });
}

int cipc_gpu_export_matrix(cipc_gpu_context* h, long long* count, int* rows, int* cols, double* vals) {
    return guarded(h, [&](Ctx& c) {
        requireSystem(c);
        sync(c);
        long long n = 9LL * (c.nnzb + c.nDynB + c.nv);
        if (count) *count = n;
        if (!rows) return;
        std::vector<int> rp(c.nv + 1), col(c.nnzb), drs(c.nv), dre(c.nv), dcol(std::max(c.nDynB, 1));
        std::vector<double> val(9 * (size_t)c.nnzb), dval(9 * (size_t)std::max(c.nDynB, 1)), diag(9 * (size_t)c.nv);
        CIPC_CUDA(cudaMemcpy(rp.data(), c.rowPtr.p, sizeof(int) * (c.nv + 1), cudaMemcpyDeviceToHost));
        CIPC_CUDA(cudaMemcpy(col.data(), c.colIdx.p, sizeof(int) * c.nnzb, cudaMemcpyDeviceToHost));
        if (c.mixed) {
            std::vector<float> f(9 * (size_t)c.nnzb);
            CIPC_CUDA(cudaMemcpy(f.data(), c.valF.p, sizeof(float) * f.size(), cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < f.size(); ++i) val[i] = f[i];
        } else {
            CIPC_CUDA(cudaMemcpy(val.data(), c.valD.p, sizeof(double) * val.size(), cudaMemcpyDeviceToHost));
        }
        if (c.nDynB) {
            CIPC_CUDA(cudaMemcpy(drs.data(), c.dynRowStart.p, sizeof(int) * c.nv, cudaMemcpyDeviceToHost));
            CIPC_CUDA(cudaMemcpy(dre.data(), c.dynRowEnd.p, sizeof(int) * c.nv, cudaMemcpyDeviceToHost));
            CIPC_CUDA(cudaMemcpy(dcol.data(), c.dynCol.p, sizeof(int) * c.nDynB, cudaMemcpyDeviceToHost));
            if (c.mixed) {
                std::vector<float> f(9 * (size_t)c.nDynB);
                CIPC_CUDA(cudaMemcpy(f.data(), c.dynBF.p, sizeof(float) * f.size(), cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < f.size(); ++i) dval[i] = f[i];
            } else {
                CIPC_CUDA(cudaMemcpy(dval.data(), c.dynBD.p, sizeof(double) * 9 * c.nDynB, cudaMemcpyDeviceToHost));
            }
        }
        CIPC_CUDA(cudaMemcpy(diag.data(), c.diagExtra.p, sizeof(double) * diag.size(), cudaMemcpyDeviceToHost));
        long long k = 0;
        auto put = [&](int r, int cl, const double* B) {
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) { rows[k] = 3 * r + a; cols[k] = 3 * cl + b; vals[k] = B[3 * a + b]; ++k; }
        };
        for (int r = 0; r < c.nv; ++r) {
            for (int q = rp[r]; q < rp[r + 1]; ++q) put(r, col[q], &val[9 * (size_t)q]);
            if (c.nDynB) for (int q = drs[r]; q < dre[r]; ++q) put(r, dcol[q], &dval[9 * (size_t)q]);
            put(r, r, &diag[9 * (size_t)r]);
        }
        if (count) *count = k;
    });
}

int cipc_gpu_solve(cipc_gpu_context* h, double* direction, int* iterations, double* relRes) {
    return guarded(h, [&](Ctx& c) {
        requireSystem(c);
        linearSolve(c);
        sync(c);
        if (direction) CIPC_CUDA(cudaMemcpy(direction, c.dir.p, sizeof(double) * 3 * c.nv, cudaMemcpyDeviceToHost));
        if (iterations) *iterations = c.lastPcgIters;
        if (relRes) *relRes = c.lastPcgRelRes;
    });
}

int cipc_gpu_energy(cipc_gpu_context* h, double kappa, double* e) {
    return guarded(h, [&](Ctx& c) { *e = totalEnergy(c, kappa); });
}

int cipc_gpu_step_bounds(cipc_gpu_context* h, const double* dir, double alphaIn, double* out) {
    return guarded(h, [&](Ctx& c) {
        CIPC_CUDA(cudaMemcpy(c.dir.p, dir, sizeof(double) * 3 * c.nv, cudaMemcpyHostToDevice));
        out[0] = std::min(1.0, groundStepBound(c));
        out[1] = partialCCD(c, alphaIn);
        out[2] = cflBound(c);
        out[3] = fullCCD(c, alphaIn);
        rebuildTrees(c);
        sync(c);
    });
}

int cipc_gpu_timed_steps(cipc_gpu_context* h, int nsteps, cipc_step_stats* last, double* deviceMs) {
    return guarded(h, [&](Ctx& c) {
        if (nsteps <= 0) throw InvalidArgument("nsteps must be positive");
        cudaEvent_t a, b;
        CIPC_CUDA(cudaEventCreate(&a));
        CIPC_CUDA(cudaEventCreate(&b));
        CIPC_CUDA(cudaEventRecord(a, c.s));
        cipc_step_stats st;
        try {
            for (int k = 0; k < nsteps; ++k) solveIPCStep(c, st);
        } catch (...) {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
            throw;
        }
        CIPC_CUDA(cudaEventRecord(b, c.s));
        CIPC_CUDA(cudaEventSynchronize(b));
        float msf = 0;
        CIPC_CUDA(cudaEventElapsedTime(&msf, a, b));
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        if (last) *last = st;
        if (deviceMs) *deviceMs = msf;
    });
}

int cipc_gpu_profile(cipc_gpu_context* h, int kind, int capacity) {
    return guarded(h, [&](Ctx& c) {
        sync(c);
        for (cudaEvent_t e : c.profEv) cudaEventDestroy(e);
        c.profEv.clear();
        c.profUsed = 0;
        c.profKind = kind;
        if (kind == PROF_NONE) return;
        if (capacity <= 0) throw InvalidArgument("capacity must be positive");
        c.profEv.resize(2 * (size_t)capacity);
        for (auto& e : c.profEv) CIPC_CUDA(cudaEventCreate(&e));
    });
}

int cipc_gpu_profile_read(cipc_gpu_context* h, long long* launches, double* totalMs) {
    return guarded(h, [&](Ctx& c) {
        sync(c);
        double tot = 0;
        for (int i = 0; i + 1 < c.profUsed; i += 2) {
            float m = 0;
            CIPC_CUDA(cudaEventElapsedTime(&m, c.profEv[i], c.profEv[i + 1]));
            tot += m;
        }
        if (launches) *launches = c.profUsed / 2;
        if (totalMs) *totalMs = tot;
    });
}

long long cipc_gpu_kernel_launches(void) { return g_kernelLaunches; }

int cipc_gpu_intersected(cipc_gpu_context* h, int* result) {
    return guarded(h, [&](Ctx& c) {
        rebuildTrees(c);
        *result = isIntersected(c) ? 1 : 0;
    });
}

int cipc_gpu_export_bsr(cipc_gpu_context* h, int* sizes, int* rowPtr, int* col, double* val, int* dynRowStart, int* dynRowEnd, int* dynCol,
                        double* dynVal, double* diagExtra) {
    return guarded(h, [&](Ctx& c) {
        requireSystem(c);
        sync(c);
        if (sizes) { sizes[0] = c.nnzb; sizes[1] = c.nDynB; }
        if (!rowPtr) return;
        int nv = c.nv;
        CIPC_CUDA(cudaMemcpy(rowPtr, c.rowPtr.p, sizeof(int) * (nv + 1), cudaMemcpyDeviceToHost));
        CIPC_CUDA(cudaMemcpy(col, c.colIdx.p, sizeof(int) * c.nnzb, cudaMemcpyDeviceToHost));
        auto blocks = [&](double* out, const DBuf<double>& d, const DBuf<float>& f, size_t n) {
            if (!n) return;
            if (c.mixed) {
                std::vector<float> t(9 * n);
                CIPC_CUDA(cudaMemcpy(t.data(), f.p, sizeof(float) * t.size(), cudaMemcpyDeviceToHost));
                for (size_t i = 0; i < t.size(); ++i) out[i] = t[i];
            } else {
                CIPC_CUDA(cudaMemcpy(out, d.p, sizeof(double) * 9 * n, cudaMemcpyDeviceToHost));
            }
        };
        blocks(val, c.valD, c.valF, c.nnzb);
        if (c.nDynB) {
            CIPC_CUDA(cudaMemcpy(dynRowStart, c.dynRowStart.p, sizeof(int) * nv, cudaMemcpyDeviceToHost));
            CIPC_CUDA(cudaMemcpy(dynRowEnd, c.dynRowEnd.p, sizeof(int) * nv, cudaMemcpyDeviceToHost));
            CIPC_CUDA(cudaMemcpy(dynCol, c.dynCol.p, sizeof(int) * c.nDynB, cudaMemcpyDeviceToHost));
            blocks(dynVal, c.dynBD, c.dynBF, c.nDynB);
        } else {
            for (int i = 0; i < nv; ++i) dynRowStart[i] = dynRowEnd[i] = 0;
        }
        CIPC_CUDA(cudaMemcpy(diagExtra, c.diagExtra.p, sizeof(double) * 9 * nv, cudaMemcpyDeviceToHost));
    });
}

int cipc_gpu_precond_num_params(void) { return MP_NPARAM; }

int cipc_gpu_precond_set_weights(cipc_gpu_context* h, const float* weights, int n) {
    return guarded(h, [&](Ctx& c) {
        if (!weights) throw InvalidArgument("weights pointer is null");
        mpnnSetWeights(c, weights, n);
    });
}

int cipc_gpu_precond_get_weights(cipc_gpu_context* h, float* weights, int n) {
    return guarded(h, [&](Ctx& c) {
        if (!weights || n != MP_NPARAM) throw InvalidArgument("expected a buffer of " + std::to_string(MP_NPARAM) + " parameters");
        if (!c.mpReady) mpnnInitWeights(c, 1);
        mpnnGetWeights(c, weights);
    });
}

int cipc_gpu_precond_loss(cipc_gpu_context* h, int probes, const float* probeVectors, unsigned long long seed, double* loss, float* grad) {
    return guarded(h, [&](Ctx& c) {
        requireSystem(c);
        if (!c.mpReady) mpnnInitWeights(c, 1);
        mpnnPrepare(c);
        mpnnForward(c);
        double l = mpnnLoss(c, probes, probeVectors, seed, grad != nullptr);
        if (loss) *loss = l;
        if (grad) mpnnGetGrad(c, grad);
    });
}

int cipc_gpu_precond_train(cipc_gpu_context* h, int iterations, int probes, double learningRate, unsigned long long seed, double* lossFirst,
                           double* lossLast) {
    return guarded(h, [&](Ctx& c) {
        if (iterations < 1 || probes < 1 || !(learningRate > 0)) throw InvalidArgument("training needs iterations, probes and a positive rate");
        requireSystem(c);
        if (!c.mpReady) mpnnInitWeights(c, 1);
        mpnnPrepare(c);
        for (int it = 0; it < iterations; ++it) {
            mpnnForward(c);
            double l = mpnnLoss(c, probes, nullptr, seed + 104729ull * (unsigned long long)(c.mpStep + 1), true);
            if (it == 0 && lossFirst) *lossFirst = l;
            if (lossLast) *lossLast = l;
            mpnnAdam(c, learningRate);
        }
        sync(c);
    });
}

int cipc_gpu_set_online_training(cipc_gpu_context* h, int iterations, int probes, double learningRate, unsigned long long seed) {
    return guarded(h, [&](Ctx& c) {
        if (iterations < 0 || (iterations > 0 && (probes < 1 || !(learningRate > 0))))
            throw InvalidArgument("online training needs non-negative iterations, probes and a positive rate");
        c.hookTrainIters = iterations;
        c.hookTrainProbes = probes;
        c.hookTrainLr = learningRate;
        c.hookTrainSeed = seed;
    });
}

int cipc_gpu_set_system_dump(cipc_gpu_context* h, const char* directory) {
    return guarded(h, [&](Ctx& c) { c.dumpDir = directory ? directory : ""; });
}

int cipc_gpu_host_syncs(cipc_gpu_context* h, long long* count) {
    return guarded(h, [&](Ctx& c) { *count = c.hostSyncs; });
}

int cipc_gpu_hook_systems(cipc_gpu_context* h, long long* count) {
    return guarded(h, [&](Ctx& c) { *count = c.hookSystems; });
}

int cipc_gpu_precond_factor(cipc_gpu_context* h, int which, float* gStatic, float* gContact) {
    return guarded(h, [&](Ctx& c) {
        requireSystem(c);
        if (which != CIPC_PRECOND_LEARNED && which != CIPC_PRECOND_FSAI) throw InvalidArgument("which must be a factor preconditioner");
        if (which == CIPC_PRECOND_FSAI) {
            mpnnPrepare(c, false);
            fsaiBuild(c);
        } else {
            if (!c.mpReady) mpnnInitWeights(c, 1);
            mpnnPrepare(c);
            mpnnForward(c);
        }
        sync(c);
        if (gStatic) CIPC_CUDA(cudaMemcpy(gStatic, c.mpGS.p, sizeof(float) * 9 * (size_t)c.nnzb, cudaMemcpyDeviceToHost));
        if (gContact && c.nDynB) CIPC_CUDA(cudaMemcpy(gContact, c.mpGD.p, sizeof(float) * 9 * (size_t)c.nDynB, cudaMemcpyDeviceToHost));
    });
}

int cipc_gpu_precond_stats(cipc_gpu_context* h, long long* out) {
    return guarded(h, [&](Ctx& c) {
        out[0] = c.mpFallbacks;
        out[1] = c.mpStep;
        out[2] = c.lastPcgLaunchIters;
    });
}

}  // extern "C"

extern "C" int cipc_gpu_accd(int n, const int* kind, const double* positions, const double* displacements, double eta, double* toi, char* err,
                             int errlen) {
    auto fail = [&](const char* m, int code) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", m);
        return code;
    };
    if (n < 0 || (n > 0 && (!kind || !positions || !displacements || !toi)) || !(eta > 0.0 && eta <= 1.0))
        return fail("invalid arguments", CIPC_ERR_INVALID_ARGUMENT);
    if (n == 0) return CIPC_OK;
    for (int k = 0; k < n; ++k)
        if (kind[k] != 0 && kind[k] != 1) return fail("pair kind must be 0 (point-triangle) or 1 (edge-edge)", CIPC_ERR_INVALID_ARGUMENT);
    try {
        cipc::accdBatch(n, kind, positions, displacements, eta, toi);
    } catch (const cipc::CudaError& e) {
        return fail(e.what(), CIPC_ERR_CUDA);
    } catch (const std::exception& e) {
        return fail(e.what(), CIPC_ERR_RUNTIME);
    }
    return CIPC_OK;
}

extern "C" int cipc_gpu_pcg_bsr(int nv, const int* rowPtr, const int* colIdx, const double* vals, const double* rhs, double* sol,
                                const cipc_linear_options* options, int* iterations, double* relResidual, char* err, int errlen) {
    auto fail = [&](const char* m, int code) {
        if (err && errlen > 0) std::snprintf(err, errlen, "%s", m);
        return code;
    };
    if (nv <= 0 || !rowPtr || !colIdx || !vals || !rhs || !sol) return fail("invalid arguments", CIPC_ERR_INVALID_ARGUMENT);
    Ctx c;
    try {
        c.nv = nv;
        if (options) {
            c.pcgTol = options->relativeTolerance > 0 ? options->relativeTolerance : 1e-6;
            c.pcgMaxIter = options->maximumIterations > 0 ? options->maximumIterations : 10000;
            c.mixed = options->precision == CIPC_PRECISION_MIXED;
        }
        int nnzb = rowPtr[nv];
        if (nnzb < 0 || rowPtr[0] < 0) return fail("row pointers must be non-negative and non-decreasing", CIPC_ERR_INVALID_ARGUMENT);
        c.nnzb = nnzb;
        std::vector<int> rp(rowPtr, rowPtr + nv + 1), ci(colIdx, colIdx + nnzb), diag(nv, -1);
        for (int r = 0; r < nv; ++r) {
            if (rp[r] < 0 || rp[r + 1] < rp[r]) return fail("row pointers must be non-negative and non-decreasing", CIPC_ERR_INVALID_ARGUMENT);
            int nd = 0;
            for (int k = rp[r]; k < rp[r + 1]; ++k) {
                if (ci[k] < 0 || ci[k] >= nv) return fail("column index out of range", CIPC_ERR_INVALID_ARGUMENT);
                if (ci[k] == r) { diag[r] = k; ++nd; }
            }
            // the block-Jacobi inverse needs the row's one diagonal block
            if (nd != 1) return fail("every block row needs exactly one diagonal block", CIPC_ERR_INVALID_ARGUMENT);
        }
        CIPC_CUDA(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        upload(c.rowPtr, rp); upload(c.colIdx, ci); upload(c.diagSlot, diag);
        std::vector<double> v(vals, vals + 9 * (size_t)nnzb);
        if (c.mixed) {
            std::vector<float> f(v.begin(), v.end());
            upload(c.valF, f);
        } else {
            upload(c.valD, v);
        }
        upload(c.diagExtra, std::vector<double>(9 * (size_t)nv, 0.0));
        upload(c.rhs, std::vector<double>(rhs, rhs + 3 * (size_t)nv));
        c.counters.reserve(16);
        c.status.reserve(4);
        int it = pcgSolve(c);
        CIPC_CUDA(cudaMemcpy(sol, c.sol.p, sizeof(double) * 3 * nv, cudaMemcpyDeviceToHost));
        if (iterations) *iterations = it;
        if (relResidual) *relResidual = c.lastPcgRelRes;
    } catch (const std::exception& e) {
        int code = std::string(e.what()).find("did not converge") != std::string::npos ? CIPC_ERR_NOT_CONVERGED : CIPC_ERR_CUDA;
        c.rowPtr.free(); c.colIdx.free(); c.diagSlot.free(); c.valD.free(); c.valF.free(); c.diagExtra.free(); c.rhs.free();
        c.sol.free(); c.r.free(); c.z.free(); c.p.free(); c.Ap.free(); c.Dinv.free(); c.red.free(); c.scal.free(); c.counters.free(); c.status.free();
        if (c.s) cudaStreamDestroy(c.s);
        return fail(e.what(), code);
    }
    c.rowPtr.free(); c.colIdx.free(); c.diagSlot.free(); c.valD.free(); c.valF.free(); c.diagExtra.free(); c.rhs.free();
    c.sol.free(); c.r.free(); c.z.free(); c.p.free(); c.Ap.free(); c.Dinv.free(); c.red.free(); c.scal.free(); c.counters.free(); c.status.free();
    if (c.s) cudaStreamDestroy(c.s);
    return CIPC_OK;
}
