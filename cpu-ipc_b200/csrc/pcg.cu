// Newton linear solve on the GPU: block-Jacobi preconditioned conjugate
// gradients on A = (static element BSR) + (contact BSR) + (per-vertex
// diagonal: mass, ground, soft), replacing NewtonLinearSystem::solve's
// backends (CPU IPC/NewtonLinearSystem.cpp:21-56, 176-207).  The stopping rule
// is Eigen's: ||r||^2 < tol^2 ||b||^2 with x0 = 0.
//
// SpMV: a group of 8 lanes owns one block row; lanes stride over the row's
// 3x3 blocks (contiguous 72-byte FP64 or 36-byte FP32 blocks, so a group reads
// one coalesced run) and combine with shuffles.  Dot products reduce per block
// into partials; the next kernel sums the partials in a fixed order, so no
// host round trip is needed inside an iteration and results are reproducible.
//
// Mixed precision: FP32 blocks, FP32 vectors and FP32 SpMV accumulation in an
// inner PCG, wrapped in FP64 iterative refinement: the outer loop recomputes
// the true residual b - A x in FP64 (FP32 blocks promoted) and stops on the
// same FP64 criterion as the FP64 solver.
#include "cipc_device.cuh"
#include <cuda_fp16.h>
#include "cipc_gpu.h"
#include "cipc_internal.h"
#include "fsai.h"
#include "mpnn.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>

namespace cipc {

namespace {

constexpr int VB = 256;          // threads per block for vector kernels
constexpr int GROUP = 4;         // lanes per block row (measured: 4 lanes, 128 rows per block, one block per SM beat 8 lanes and two blocks per SM by 10 %)
constexpr int MAXPART = 512;
constexpr int PB = 512;          // threads per block of the persistent PCG
constexpr int PIPE_PMAX = 1024;  // partial-sum slots per array of the pipelined PCG (>= its grid)

inline int vecBlocks(int n) { return std::max(1, std::min((n + VB - 1) / VB, MAXPART)); }

template <class MT, class VT>
__device__ __forceinline__ void blockMulAdd(const MT* B, const VT* xv, VT acc[3]) {
    acc[0] += (VT)B[0] * xv[0] + (VT)B[1] * xv[1] + (VT)B[2] * xv[2];
    acc[1] += (VT)B[3] * xv[0] + (VT)B[4] * xv[1] + (VT)B[5] * xv[2];
    acc[2] += (VT)B[6] * xv[0] + (VT)B[7] * xv[1] + (VT)B[8] * xv[2];
}

// acc += B x for a 3x3 block of FP16 values (row-major)
template <class VT>
__device__ __forceinline__ void blockMulAddH(const __half* B, const VT* xv, VT acc[3]) {
    VT b[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) b[e] = (VT)__half2float(B[e]);
    acc[0] += b[0] * xv[0] + b[1] * xv[1] + b[2] * xv[2];
    acc[1] += b[3] * xv[0] + b[4] * xv[1] + b[5] * xv[2];
    acc[2] += b[6] * xv[0] + b[7] * xv[1] + b[8] * xv[2];
}

// y = A x ; partial[block] = sum over the block's rows of x . y (for p.Ap)
template <class MT, class VT>
__global__ void spmvKernel(int nv, const int* rowPtr, const int* col, const MT* val, const int* dRowS, const int* dRowE, const int* dCol,
                           const MT* dVal, const double* diagExtra, const VT* x, VT* y, double* partial, const int* flag) {
    if (flag && *flag) return;
    int gid = blockIdx.x * blockDim.x + threadIdx.x;
    int lane = threadIdx.x & (GROUP - 1);
    int grp = (threadIdx.x & 31) / GROUP;
    const int RPW = 32 / GROUP;  // rows per warp per pass
    int nWarps = gridDim.x * blockDim.x / 32;
    double dotAcc = 0;
    // the loop bound is uniform across a warp, so every lane reaches the shuffles
    for (int base = (gid / 32) * RPW; base < nv; base += nWarps * RPW) {
        int row = base + grp;
        bool active = row < nv;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) {
            for (int k = rowPtr[row] + lane; k < rowPtr[row + 1]; k += GROUP) {
                int c = col[k];
                VT xv[3] = {x[3 * c], x[3 * c + 1], x[3 * c + 2]};
                blockMulAdd(val + (size_t)9 * k, xv, acc);
            }
            if (dRowS) {
                for (int k = dRowS[row] + lane; k < dRowE[row]; k += GROUP) {
                    int c = dCol[k];
                    VT xv[3] = {x[3 * c], x[3 * c + 1], x[3 * c + 2]};
                    blockMulAdd(dVal + (size_t)9 * k, xv, acc);
                }
            }
        }
        for (int o = GROUP / 2; o > 0; o >>= 1)
            for (int q = 0; q < 3; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o, GROUP);
        if (active && lane == 0) {
            VT xv[3] = {x[3 * row], x[3 * row + 1], x[3 * row + 2]};
            const double* D = diagExtra + 9 * row;
            for (int q = 0; q < 3; ++q) acc[q] += (VT)(D[3 * q] * (double)xv[0] + D[3 * q + 1] * (double)xv[1] + D[3 * q + 2] * (double)xv[2]);
            for (int q = 0; q < 3; ++q) {
                y[3 * row + q] = acc[q];
                dotAcc += (double)xv[q] * (double)acc[q];
            }
        }
    }
    if (partial) {
        double s = blockReduce(dotAcc, AddOp(), 0.0);
        if (threadIdx.x == 0) partial[blockIdx.x] = s;
    }
}

__device__ __forceinline__ double sumPartials(const double* p, int n) {
    // every block sums the partials in the same order (deterministic)
    __shared__ double sh;
    double v = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) v += p[i];
    v = blockReduce(v, AddOp(), 0.0);
    if (threadIdx.x == 0) sh = v;
    __syncthreads();
    return sh;
}

// block-Jacobi inverse of the assembled diagonal blocks
template <class MT>
__global__ void dinvKernel(int nv, const int* diagSlot, const MT* val, const int* dRowS, const int* dRowE, const int* dCol, const MT* dVal,
                           const double* diagExtra, double* Dinv) {
    CIPC_KERNEL_LOOP(v, nv) {
        double D[9];
        for (int k = 0; k < 9; ++k) D[k] = diagExtra[9 * v + k];
        int s = diagSlot[v];
        if (s >= 0) for (int k = 0; k < 9; ++k) D[k] += (double)val[(size_t)9 * s + k];
        if (dRowS)
            for (int k = dRowS[v]; k < dRowE[v]; ++k)
                if (dCol[k] == v) for (int q = 0; q < 9; ++q) D[q] += (double)dVal[(size_t)9 * k + q];
        double c00 = D[4] * D[8] - D[5] * D[7], c10 = D[5] * D[6] - D[3] * D[8], c20 = D[3] * D[7] - D[4] * D[6];
        double det = D[0] * c00 + D[1] * c10 + D[2] * c20;
        double* o = Dinv + 9 * v;
        if (det == 0.0 || !isfinite(det)) { for (int k = 0; k < 9; ++k) o[k] = 0.0; continue; }
        o[0] = c00 / det; o[3] = c10 / det; o[6] = c20 / det;
        o[1] = (D[2] * D[7] - D[1] * D[8]) / det;
        o[4] = (D[0] * D[8] - D[2] * D[6]) / det;
        o[7] = (D[1] * D[6] - D[0] * D[7]) / det;
        o[2] = (D[1] * D[5] - D[2] * D[4]) / det;
        o[5] = (D[2] * D[3] - D[0] * D[5]) / det;
        o[8] = (D[0] * D[4] - D[1] * D[3]) / det;
    }
}

template <class VT>
__device__ __forceinline__ void applyDinv(const double* Dinv, const VT* r, VT* z, int v) {
    const double* D = Dinv + 9 * v;
    double r0 = r[3 * v], r1 = r[3 * v + 1], r2 = r[3 * v + 2];
    z[3 * v] = (VT)(D[0] * r0 + D[1] * r1 + D[2] * r2);
    z[3 * v + 1] = (VT)(D[3] * r0 + D[4] * r1 + D[5] * r2);
    z[3 * v + 2] = (VT)(D[6] * r0 + D[7] * r1 + D[8] * r2);
}

// scal layout: 0 rz, 1 beta, 2 thr, 3 rr, 4 iterations, 6 rhs2
template <class VT>
__global__ void pcgInitKernel(int nv, const VT* b, const double* Dinv, VT* x, VT* r, VT* z, VT* p, double* part0, double* part1) {
    double rr = 0, rz = 0;
    CIPC_KERNEL_LOOP(v, nv) {
        for (int q = 0; q < 3; ++q) { x[3 * v + q] = VT(0); r[3 * v + q] = b[3 * v + q]; }
        applyDinv(Dinv, r, z, v);
        for (int q = 0; q < 3; ++q) {
            p[3 * v + q] = z[3 * v + q];
            rr += (double)r[3 * v + q] * (double)r[3 * v + q];
            rz += (double)r[3 * v + q] * (double)z[3 * v + q];
        }
    }
    double a = blockReduce(rr, AddOp(), 0.0);
    __syncthreads();
    double c = blockReduce(rz, AddOp(), 0.0);
    if (threadIdx.x == 0) { part0[blockIdx.x] = a; part1[blockIdx.x] = c; }
}

__global__ void pcgInitScalars(const double* part0, const double* part1, int np, double tol, double* scal, int* flag) {
    double rr = sumPartials(part0, np);
    double rz = sumPartials(part1, np);
    if (threadIdx.x == 0) {
        scal[6] = rr;
        double thr = fmax(tol * tol * rr, 2.2250738585072014e-308);
        scal[2] = thr;
        scal[3] = rr;
        scal[0] = rz;
        scal[4] = 0;
        *flag = (rr == 0.0 || rr < thr) ? 1 : 0;
    }
}

// x += a p ; r -= a Ap ; z = M r ; partials of r.r and r.z
template <class VT>
__global__ void pcgUpdateKernel(int nv, const double* pAp, int np, const double* scal, const double* Dinv, const VT* p, const VT* Ap, VT* x, VT* r,
                                VT* z, double* partRR, double* partRZ, const int* flag) {
    if (*flag) return;
    VT alpha = (VT)(scal[0] / sumPartials(pAp, np));
    double rr = 0, rz = 0;
    CIPC_KERNEL_LOOP(v, nv) {
        for (int q = 0; q < 3; ++q) {
            x[3 * v + q] += alpha * p[3 * v + q];
            r[3 * v + q] -= alpha * Ap[3 * v + q];
        }
        applyDinv(Dinv, r, z, v);
        for (int q = 0; q < 3; ++q) {
            rr += (double)r[3 * v + q] * (double)r[3 * v + q];
            rz += (double)r[3 * v + q] * (double)z[3 * v + q];
        }
    }
    double a = blockReduce(rr, AddOp(), 0.0);
    __syncthreads();
    double c = blockReduce(rz, AddOp(), 0.0);
    if (threadIdx.x == 0) { partRR[blockIdx.x] = a; partRZ[blockIdx.x] = c; }
}

// scalar step: convergence test, beta; one block.
__global__ void pcgScalarKernel(const double* partRR, const double* partRZ, int np, double* scal, int* flag, int maxIter) {
    if (*flag) return;
    double rr = sumPartials(partRR, np);
    double rz = sumPartials(partRZ, np);
    if (threadIdx.x == 0) {
        scal[3] = rr;
        if (rr < scal[2]) { *flag = 1; scal[4] += 1; return; }
        scal[1] = rz / scal[0];  // beta
        scal[0] = rz;
        scal[4] += 1;
        if (scal[4] >= maxIter) *flag = 2;
    }
}

template <class VT>
__global__ void pcgDirKernel(int nv, const double* scal, const VT* z, VT* p, const int* flag) {
    if (*flag == 1) return;
    VT beta = (VT)scal[1];
    CIPC_KERNEL_LOOP(i, 3 * nv) p[i] = z[i] + beta * p[i];
}

__global__ void rhsKernel(int nv, const double* g, const int* btype, double* b) {
    CIPC_KERNEL_LOOP(v, nv) {
        bool fr = btype[v] == 0;
        for (int q = 0; q < 3; ++q) b[3 * v + q] = fr ? g[3 * v + q] : 0.0;
    }
}

// r = b - Ax (FP64), rF = (float) r, partial |r|^2
__global__ void residualKernel(int n3, const double* b, const double* Ax, double* r, float* rF, double* part) {
    double rr = 0;
    CIPC_KERNEL_LOOP(i, n3) {
        double v = b[i] - Ax[i];
        r[i] = v;
        rF[i] = (float)v;
        rr += v * v;
    }
    double s = blockReduce(rr, AddOp(), 0.0);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void accumulateKernel(int n3, const float* d, double* x) {
    CIPC_KERNEL_LOOP(i, n3) x[i] += (double)d[i];
}

// ---------------------------------------------------------------------------
// Persistent PCG: the whole CG loop in one cooperative launch.
//
// Two grid barriers per iteration with block-Jacobi.  The direction update is
// folded into the SpMV phase through A p' = A z + beta A p, so each phase only
// reads vectors that the previous phase finished:
//   phase 1: p = z + beta p, Ap = A z + beta Ap, partial p.Ap     | barrier
//   phase 2: x += alpha p, r -= alpha Ap, z = M r, partial r.r, r.z | barrier
// With the learned factorised approximate inverse M = S^T G^T G S, phase 2
// splits in three (r and S r | t = G S r | z = S^T G^T t), four barriers per
// iteration.  A group of GROUP lanes owns one block row in every phase, so a
// row's x, r, p, Ap are only touched by their owner; z, S r and t are read by
// neighbours after a barrier.  Those reads are plain loads: the barrier's
// acquire (then __syncthreads) orders them after the other blocks' writes
// under the PTX memory model, and they may hit in L1, where the vertices
// that neighbouring rows of one SM share are fetched from L2 once.  Every block sums the
// per-block partials in the same order, so all blocks take the same branch and
// results are reproducible.  The barrier spin is bounded: on timeout it sets
// an error flag and the kernel returns.
// ---------------------------------------------------------------------------
template <class MT, class VT>
struct PcgArgs {
    int nv;
    const int *rowPtr, *col;
    const MT* val;
    const int *dRowS, *dRowE, *dCol;
    const MT* dVal;
    const double* diagExtra;
    const double* Dinv;
    // learned factor (null for block-Jacobi): S 9 per vertex, G slot-aligned
    const double* S;
    const float *gS, *gD;
    // the static part of G packed by rows (null: read gS): lower part and
    // transposed part, FP16 blocks with their columns and row offsets
    const __half *gL, *gU;
    const int *gLptr, *gLcol, *gUptr, *gUcol;
    VT* t;
    const VT* b;
    VT *x, *r, *z, *p, *Ap;
    VT *u, *w, *mA, *mB, *q, *s;  // pipelined variant only
    double *partA, *partB, *partC;
    double* pp;                   // pipelined variant: two sets of three partial arrays, PIPE_PMAX each
    int sliceMax;                 // cached variant: static slots of the largest block row range
    int rowsPerBlock;             // cached variant: rows each block owns (<= ROWS_PER_BLOCK)
    int dynCap;                   // cached variant: contact slots a block's window may hold
    int cacheG;                   // cached variant with a factor: G blocks staged in shared memory
    double* scal;  // out: [3] rr, [4] iterations, [6] rhs2
    int* flag;     // out: 1 converged, 2 iteration cap, 3 barrier timeout
    unsigned* bar;  // BAR_WORDS words: grid-barrier counters and generation
    double tol;
    int maxIter;
};

// Two block sums with one pair of __syncthreads; the result is valid in
// every thread.  Partial sums follow a fixed order (reproducible).
__device__ __forceinline__ void blockReduce2(double& a, double& b) {
    __shared__ double s0[32], s1[32], r2[2];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
    }
    __syncthreads();  // earlier readers of s0/s1/r2 are done
    if (lane == 0) { s0[w] = a; s1[w] = b; }
    __syncthreads();
    if (w == 0) {
        double x = lane < nw ? s0[lane] : 0.0, y = lane < nw ? s1[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_xor_sync(0xffffffffu, x, o);
            y += __shfl_xor_sync(0xffffffffu, y, o);
        }
        if (lane == 0) { r2[0] = x; r2[1] = y; }
    }
    __syncthreads();
    a = r2[0];
    b = r2[1];
}

// Three block sums with one pair of __syncthreads (as blockReduce2).
__device__ __forceinline__ void blockReduce3(double& a, double& b, double& c) {
    __shared__ double s0[32], s1[32], s2[32], r3[3];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, o);
        b += __shfl_xor_sync(0xffffffffu, b, o);
        c += __shfl_xor_sync(0xffffffffu, c, o);
    }
    __syncthreads();
    if (lane == 0) { s0[w] = a; s1[w] = b; s2[w] = c; }
    __syncthreads();
    if (w == 0) {
        double x = lane < nw ? s0[lane] : 0.0, y = lane < nw ? s1[lane] : 0.0, z = lane < nw ? s2[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) {
            x += __shfl_xor_sync(0xffffffffu, x, o);
            y += __shfl_xor_sync(0xffffffffu, y, o);
            z += __shfl_xor_sync(0xffffffffu, z, o);
        }
        if (lane == 0) { r3[0] = x; r3[1] = y; r3[2] = z; }
    }
    __syncthreads();
    a = r3[0];
    b = r3[1];
    c = r3[2];
}

// Grid barrier on one arrival counter that only grows within a launch (it is
// zeroed before the launch): barrier number e is complete when the counter
// reaches e * nblocks.  Thread 0 arrives with an acquire-release atomic after
// the block's __syncthreads, which releases every write the block made before
// the barrier; the spin's acquire loads, followed by __syncthreads, order the
// block's later reads after the other blocks' writes.  One flat counter with
// these semantics measured 1.3 us per barrier on B200 for 148-296 blocks,
// against 2.9 us for a two-level tree of counters with full fences.
// The spin is bounded: on timeout the spinning thread sets flag = 3 and the
// barrier returns false; a block that returns early makes every other block
// time out at its next barrier, so no wait is unbounded.
constexpr int BAR_WORDS = 32;  // the counter, alone on its 128-byte line
constexpr long long BAR_SPIN_MAX = 1ll << 25;

__device__ __forceinline__ unsigned atomAddAcqRelGpu(unsigned* p, unsigned v) {
    unsigned old;
    asm volatile("atom.add.acq_rel.gpu.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
    return old;
}
__device__ __forceinline__ unsigned ldAcquireGpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
// spin (acquire loads) until the counter reaches target; false on timeout
__device__ __forceinline__ bool barrierSpin(const unsigned* bar, int* flag, unsigned target) {
    long long spins = 0;
    while ((int)(ldAcquireGpu(bar) - target) < 0) {
        if (++spins > BAR_SPIN_MAX) { atomicExch(flag, 3); return false; }
    }
    return true;
}

__device__ __forceinline__ bool gridBarrier(unsigned* bar, int* flag, unsigned nblocks, unsigned& epoch) {
    const unsigned target = ++epoch * nblocks;
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int good = 1;
        if (atomAddAcqRelGpu(bar, 1u) + 1 != target) good = barrierSpin(bar, flag, target);
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Grid barrier followed by the sums of K per-block partial arrays (array j at
// P + j * stride, one entry per block, written before the barrier).  Warp 0
// waits (every lane spins with its own acquire loads), reads the partials in
// a fixed order and reduces them with shuffles, so every block gets the same
// bits; one __syncthreads hands the sums to the block.
template <int K>
__device__ __forceinline__ bool gridBarrierSum(unsigned* bar, int* flag, unsigned nblocks, unsigned& epoch, const double* P, size_t stride,
                                               double (&out)[K]) {
    const unsigned target = ++epoch * nblocks;
    __shared__ double res[K];
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        if (lane == 0) atomAddAcqRelGpu(bar, 1u);
        const bool good = __all_sync(0xffffffffu, barrierSpin(bar, flag, target));
        double v[K];
        for (int j = 0; j < K; ++j) v[j] = 0.0;
        if (good)
            for (int i = lane; i < (int)nblocks; i += 32)
                for (int j = 0; j < K; ++j) v[j] += __ldcg(P + j * stride + i);
        for (int o = 16; o > 0; o >>= 1)
            for (int j = 0; j < K; ++j) v[j] += __shfl_xor_sync(0xffffffffu, v[j], o);
        if (lane == 0) {
            for (int j = 0; j < K; ++j) res[j] = v[j];
            ok = good ? 1 : 0;
        }
    }
    __syncthreads();
    for (int j = 0; j < K; ++j) out[j] = res[j];
    return ok != 0;
}

// Row-group iteration shared by every phase: the same (block, lane group)
// owns the same rows in all phases.
struct RowIter {
    int lane, grp, first, stride, limit;
    __device__ RowIter() {
        int gid = blockIdx.x * blockDim.x + threadIdx.x;
        lane = threadIdx.x & (GROUP - 1);
        grp = (threadIdx.x & 31) / GROUP;
        first = (gid / 32) * (32 / GROUP);
        stride = gridDim.x * blockDim.x / 32 * (32 / GROUP);
        limit = 0x7fffffff;
    }
    // single pass over this block's own rows [blockIdx.x * rows, + rows) of nv
    __device__ RowIter(int nv, int rows) {
        lane = threadIdx.x & (GROUP - 1);
        grp = (threadIdx.x & 31) / GROUP;
        const int row0 = blockIdx.x * rows;
        first = row0 + (threadIdx.x / 32) * (32 / GROUP);
        stride = nv;
        limit = min(nv, row0 + rows);
    }
};

template <class VT>
__device__ __forceinline__ void groupReduce3(VT acc[3]) {
    for (int o = GROUP / 2; o > 0; o >>= 1)
        for (int q = 0; q < 3; ++q) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o, GROUP);
}

// acc += (A u)_row over the row's static and contact blocks (lane-strided)
template <class MT, class VT>
__device__ __forceinline__ void rowSpmv(const PcgArgs<MT, VT>& a, int row, int lane, const VT* u, VT acc[3]) {
    for (int k = a.rowPtr[row] + lane; k < a.rowPtr[row + 1]; k += GROUP) {
        int c = a.col[k];
        VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
        blockMulAdd(a.val + (size_t)9 * k, xv, acc);
    }
    if (a.dRowS) {
        for (int k = a.dRowS[row] + lane; k < a.dRowE[row]; k += GROUP) {
            int c = a.dCol[k];
            VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
            blockMulAdd(a.dVal + (size_t)9 * k, xv, acc);
        }
    }
}

// acc += (G u)_row (TR = false: lower slots and the diagonal block) or
// (G^T u)_row (TR = true: mirror slots and the transposed diagonal block)
template <bool TR, class MT, class VT>
__device__ __forceinline__ void rowFactor(const PcgArgs<MT, VT>& a, int row, int lane, const VT* u, VT acc[3]) {
    if (a.gL) {
        // packed rows: only the blocks of this pass, FP16
        const int* ptr = TR ? a.gUptr : a.gLptr;
        const int* cl = TR ? a.gUcol : a.gLcol;
        const __half* G = TR ? a.gU : a.gL;
        // two of the lane's slots per round: both gathers are issued before
        // the products, which stay in slot order
        const int ke = ptr[row + 1];
        for (int k = ptr[row] + lane; k < ke; k += 2 * GROUP) {
            const int k1 = k + GROUP;
            const bool two = k1 < ke;
            const int c0 = cl[k], c1 = two ? cl[k1] : c0;
            const VT x0[3] = {u[3 * c0], u[3 * c0 + 1], u[3 * c0 + 2]};
            const VT x1[3] = {u[3 * c1], u[3 * c1 + 1], u[3 * c1 + 2]};
            blockMulAddH(G + (size_t)9 * k, x0, acc);
            if (two) blockMulAddH(G + (size_t)9 * k1, x1, acc);
        }
    } else for (int k = a.rowPtr[row] + lane; k < a.rowPtr[row + 1]; k += GROUP) {
        int c = a.col[k];
        if (TR ? c < row : c > row) continue;
        VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
        const float* B = a.gS + (size_t)9 * k;
        if (TR && c == row) {
            for (int q = 0; q < 3; ++q) acc[q] += (VT)B[q] * xv[0] + (VT)B[3 + q] * xv[1] + (VT)B[6 + q] * xv[2];
        } else {
            blockMulAdd(B, xv, acc);
        }
    }
    if (a.dRowS) {
        for (int k = a.dRowS[row] + lane; k < a.dRowE[row]; k += GROUP) {
            int c = a.dCol[k];
            if (TR ? c <= row : c >= row) continue;
            VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
            blockMulAdd(a.gD + (size_t)9 * k, xv, acc);
        }
    }
}

// z = M r for the learned factor, phases after r is final: writes S r into
// z, t = G (S r), z = S^T G^T t; returns this thread's r.z contribution
// (valid on lane 0 of each group).  Three barriers; false on barrier timeout.
template <class MT, class VT>
__device__ bool learnedApply(const PcgArgs<MT, VT>& a, const RowIter& it, double& rz, double* partRR, double rrLocal, unsigned& ep) {
    const unsigned nb = gridDim.x;
    for (int base = it.first; base < a.nv; base += it.stride) {
        int row = base + it.grp;
        if (row < a.nv && it.lane == 0) {
            const double* S = a.S + 9 * row;
            double r0 = a.r[3 * row], r1 = a.r[3 * row + 1], r2 = a.r[3 * row + 2];
            a.z[3 * row] = (VT)(S[0] * r0);
            a.z[3 * row + 1] = (VT)(S[3] * r0 + S[4] * r1);
            a.z[3 * row + 2] = (VT)(S[6] * r0 + S[7] * r1 + S[8] * r2);
        }
    }
    {
        double dummy = 0;
        blockReduce2(rrLocal, dummy);
        if (threadIdx.x == 0) partRR[blockIdx.x] = rrLocal;
    }
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return false;
    for (int base = it.first; base < a.nv; base += it.stride) {
        int row = base + it.grp;
        bool active = row < a.nv;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) rowFactor<false>(a, row, it.lane, (const VT*)a.z, acc);
        groupReduce3(acc);
        if (active && it.lane == 0)
            for (int q = 0; q < 3; ++q) a.t[3 * row + q] = acc[q];
    }
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return false;
    rz = 0;
    for (int base = it.first; base < a.nv; base += it.stride) {
        int row = base + it.grp;
        bool active = row < a.nv;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) rowFactor<true>(a, row, it.lane, (const VT*)a.t, acc);
        groupReduce3(acc);
        if (active && it.lane == 0) {
            const double* S = a.S + 9 * row;
            double y0 = acc[0], y1 = acc[1], y2 = acc[2];
            VT z0 = (VT)(S[0] * y0 + S[3] * y1 + S[6] * y2);
            VT z1 = (VT)(S[4] * y1 + S[7] * y2);
            VT z2 = (VT)(S[8] * y2);
            a.z[3 * row] = z0; a.z[3 * row + 1] = z1; a.z[3 * row + 2] = z2;
            rz += (double)a.r[3 * row] * (double)z0 + (double)a.r[3 * row + 1] * (double)z1 + (double)a.r[3 * row + 2] * (double)z2;
        }
    }
    return true;
}

template <class MT, class VT, bool LEARNED>
__global__ void __launch_bounds__(PB) pcgPersistentKernel(PcgArgs<MT, VT> a) {
    const unsigned nb = gridDim.x;
    unsigned ep = 0;
    const int nv = a.nv;
    const RowIter it;
    // init: x = 0, r = b, z = M r, p = 0, Ap = 0 (the first beta is 0)
    double rr = 0, rz = 0;
    for (int base = it.first; base < nv; base += it.stride) {
        int row = base + it.grp;
        if (row < nv && it.lane == 0) {
            for (int q = 0; q < 3; ++q) {
                a.x[3 * row + q] = VT(0); a.p[3 * row + q] = VT(0); a.Ap[3 * row + q] = VT(0);
                a.r[3 * row + q] = a.b[3 * row + q];
                rr += (double)a.r[3 * row + q] * (double)a.r[3 * row + q];
            }
            if (!LEARNED) {
                applyDinv(a.Dinv, a.r, a.z, row);
                for (int q = 0; q < 3; ++q) rz += (double)a.r[3 * row + q] * (double)a.z[3 * row + q];
            }
        }
    }
    if (LEARNED) {
        if (!learnedApply(a, it, rz, a.partA, rr, ep)) return;
        double dummy = 0;
        blockReduce2(rz, dummy);
        if (threadIdx.x == 0) a.partB[blockIdx.x] = rz;
    } else {
        blockReduce2(rr, rz);
        if (threadIdx.x == 0) { a.partA[blockIdx.x] = rr; a.partB[blockIdx.x] = rz; }
    }
    {
        double sums[2];
        if (!gridBarrierSum<2>(a.bar, a.flag, nb, ep, a.partA, a.partB - a.partA, sums)) return;
        rr = sums[0]; rz = sums[1];
    }
    const double rhs2 = rr;
    const double thr = fmax(a.tol * a.tol * rr, 2.2250738585072014e-308);
    int iter = 0;
    int status = (rr == 0.0 || rr < thr) ? 1 : 0;
    VT beta = VT(0);
    while (status == 0) {
        // phase 1: p = z + beta p ; Ap = A z + beta Ap ; p . Ap
        double d = 0;
        for (int base = it.first; base < nv; base += it.stride) {
            int row = base + it.grp;
            bool active = row < nv;
            VT acc[3] = {VT(0), VT(0), VT(0)};
            if (active) rowSpmv(a, row, it.lane, (const VT*)a.z, acc);
            groupReduce3(acc);
            if (active && it.lane == 0) {
                const double* D = a.diagExtra + 9 * row;
                VT zv[3] = {a.z[3 * row], a.z[3 * row + 1], a.z[3 * row + 2]};
                for (int q = 0; q < 3; ++q) acc[q] += (VT)(D[3 * q] * (double)zv[0] + D[3 * q + 1] * (double)zv[1] + D[3 * q + 2] * (double)zv[2]);
                for (int q = 0; q < 3; ++q) {
                    VT pv = zv[q] + beta * a.p[3 * row + q];
                    VT apv = acc[q] + beta * a.Ap[3 * row + q];
                    a.p[3 * row + q] = pv;
                    a.Ap[3 * row + q] = apv;
                    d += (double)pv * (double)apv;
                }
            }
        }
        {
            double dummy = 0;
            blockReduce2(d, dummy);
            if (threadIdx.x == 0) a.partC[blockIdx.x] = d;
        }
        double pAp[1];
        if (!gridBarrierSum<1>(a.bar, a.flag, nb, ep, a.partC, 0, pAp)) return;
        VT alpha = (VT)(rz / pAp[0]);
        // phase 2: x += alpha p ; r -= alpha Ap ; z = M r
        double lrr = 0, lrz = 0;
        for (int base = it.first; base < nv; base += it.stride) {
            int row = base + it.grp;
            if (row < nv && it.lane == 0) {
                for (int q = 0; q < 3; ++q) {
                    a.x[3 * row + q] += alpha * a.p[3 * row + q];
                    a.r[3 * row + q] -= alpha * a.Ap[3 * row + q];
                    lrr += (double)a.r[3 * row + q] * (double)a.r[3 * row + q];
                }
                if (!LEARNED) {
                    applyDinv(a.Dinv, a.r, a.z, row);
                    for (int q = 0; q < 3; ++q) lrz += (double)a.r[3 * row + q] * (double)a.z[3 * row + q];
                }
            }
        }
        if (LEARNED) {
            if (!learnedApply(a, it, lrz, a.partA, lrr, ep)) return;
            double dummy = 0;
            blockReduce2(lrz, dummy);
            if (threadIdx.x == 0) a.partB[blockIdx.x] = lrz;
        } else {
            blockReduce2(lrr, lrz);
            if (threadIdx.x == 0) { a.partA[blockIdx.x] = lrr; a.partB[blockIdx.x] = lrz; }
        }
        double sums[2];
        if (!gridBarrierSum<2>(a.bar, a.flag, nb, ep, a.partA, a.partB - a.partA, sums)) return;
        rr = sums[0];
        const double rzNew = sums[1];
        ++iter;
        if (rr < thr) { status = 1; break; }
        if (iter >= a.maxIter) { status = 2; break; }
        beta = (VT)(rzNew / rz);
        rz = rzNew;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.scal[3] = rr;
        a.scal[4] = iter;
        a.scal[6] = rhs2;
        atomicCAS(a.flag, 0, status);  // a barrier timeout (3) stands
    }
}

// ---------------------------------------------------------------------------
// Pipelined PCG (Ghysels and Vanroose's recurrences): the dot products of an
// iteration are formed in the same pass as its vector updates, and the
// preconditioned direction's product n = A m is carried by recurrences, so
// one iteration is one pass over the rows and ONE grid barrier with
// block-Jacobi (three with a factor: S w | G (S w) | S^T G^T t).
//   gamma = (r,u), delta = (w,u);  beta = gamma/gamma_old,
//   alpha = gamma / (delta - beta gamma / alpha_old)
//   n = A m;  z = n + beta z;  q = m + beta q;  s = w + beta s;  p = u + beta p
//   x += alpha p;  r -= alpha s;  u -= alpha q;  w -= alpha z;  m = M w
// With block-Jacobi the new m is written to the other of two buffers, since
// neighbours read the current one in the same pass; the partial sums also
// alternate between two sets, so a set is rewritten only two barriers after
// its last read.  The recurrences drift from the true residual in finite
// precision; the callers decide every solve on the true FP64 residual.
// ---------------------------------------------------------------------------
// Rows a block owns in a single-pass launch (PB / GROUP consecutive rows),
// staged once per solve in shared memory: the static slots (column and
// block, and with a factor its G block), the rows' contact blocks when the
// block's contact window fits, the diagonal extras, the 3x3 Jacobi inverse
// or the factor's scaling S, and the rows' recurrence vectors.  Every
// iteration then reads the matrix rows from shared memory and only the
// gathered vectors from L2.
constexpr int ROWS_PER_BLOCK = PB / GROUP;
constexpr int STATE_VECS = 9;  // x r u w z q s p, and the row's own m

struct SmemLayout {
    size_t dex, blk, val, gval, col, rp, drs, dval, dgval, dcol, state, total;
};
__host__ __device__ inline size_t alignUp16(size_t v) { return (v + 15) / 16 * 16; }
// offsets (16-byte aligned) of the cached arrays for a block of
// ROWS_PER_BLOCK rows with at most sliceMax static and dynCap contact slots
__host__ __device__ inline SmemLayout smemLayout(int sliceMax, int dynCap, bool cacheG, int msz, int vsz) {
    SmemLayout L{};
    size_t o = 0;
    L.dex = o;   o = alignUp16(o + (size_t)ROWS_PER_BLOCK * 9 * sizeof(double));
    L.blk = o;   o = alignUp16(o + (size_t)ROWS_PER_BLOCK * 9 * sizeof(double));
    L.val = o;   o = alignUp16(o + (size_t)sliceMax * 9 * msz);
    L.gval = o;  o = alignUp16(o + (cacheG ? (size_t)sliceMax * 9 * sizeof(float) : 0));
    L.col = o;   o = alignUp16(o + (size_t)sliceMax * sizeof(int));
    L.rp = o;    o = alignUp16(o + (size_t)(ROWS_PER_BLOCK + 1) * sizeof(int));
    L.drs = o;   o = alignUp16(o + (size_t)ROWS_PER_BLOCK * 2 * sizeof(int));
    L.dval = o;  o = alignUp16(o + (size_t)dynCap * 9 * msz);
    L.dgval = o; o = alignUp16(o + (cacheG ? (size_t)dynCap * 9 * sizeof(float) : 0));
    L.dcol = o;  o = alignUp16(o + (size_t)dynCap * sizeof(int));
    L.state = o; o = alignUp16(o + (size_t)STATE_VECS * ROWS_PER_BLOCK * 3 * vsz);
    L.total = o;
    return L;
}

template <class MT>
struct RowCache {
    int row0, s0;
    int d0;              // global index of the first cached contact slot; -1: contact blocks are read from global memory
    const int* rp;       // ROWS_PER_BLOCK + 1 static slot offsets (global slot indices)
    const int* col;
    const MT* val;
    const float* gval;   // factor blocks of the static slots (null: read from global memory)
    const int* drs;      // contact slot range [start, end) per row (global slot indices)
    const int* dcol;
    const MT* dval;
    const float* dgval;  // factor blocks of the cached contact slots (null: global)
    const double* dex;   // diagonal extras, 9 per row
    const double* blk;   // 9 per row: the Jacobi inverse, or the factor's scaling S
};

template <class MT, class VT, bool LEARNED>
__device__ RowCache<MT> loadRowCache(const PcgArgs<MT, VT>& a, unsigned char* smem) {
    const bool cacheG = LEARNED && a.cacheG != 0;
    const SmemLayout L = smemLayout(a.sliceMax, a.dynCap, cacheG, (int)sizeof(MT), (int)sizeof(VT));
    double* dex = reinterpret_cast<double*>(smem + L.dex);
    double* blk = reinterpret_cast<double*>(smem + L.blk);
    MT* val = reinterpret_cast<MT*>(smem + L.val);
    float* gval = reinterpret_cast<float*>(smem + L.gval);
    int* col = reinterpret_cast<int*>(smem + L.col);
    int* rp = reinterpret_cast<int*>(smem + L.rp);
    int* drs = reinterpret_cast<int*>(smem + L.drs);
    MT* dval = reinterpret_cast<MT*>(smem + L.dval);
    float* dgval = reinterpret_cast<float*>(smem + L.dgval);
    int* dcol = reinterpret_cast<int*>(smem + L.dcol);
    __shared__ int dlo, dhi;
    RowCache<MT> rc;
    rc.row0 = blockIdx.x * a.rowsPerBlock;
    const int nrows = min(a.rowsPerBlock, a.nv - rc.row0);  // >= 1: the grid is ceil(nv / rowsPerBlock)
    if (threadIdx.x == 0) { dlo = 0x7fffffff; dhi = 0; }
    for (int i = threadIdx.x; i <= nrows; i += blockDim.x) rp[i] = a.rowPtr[rc.row0 + i];
    __syncthreads();
    for (int i = threadIdx.x; i < nrows; i += blockDim.x) {
        int s = 0, e = 0;
        if (a.dRowS) { s = a.dRowS[rc.row0 + i]; e = a.dRowE[rc.row0 + i]; }
        drs[2 * i] = s;
        drs[2 * i + 1] = e;
        if (e > s) { atomicMin(&dlo, s); atomicMax(&dhi, e); }
    }
    rc.s0 = rp[0];
    const int ns = rp[nrows] - rc.s0;  // <= sliceMax (host-computed maximum over blocks)
    for (int k = threadIdx.x; k < ns; k += blockDim.x) col[k] = a.col[rc.s0 + k];
    for (int k = threadIdx.x; k < 9 * ns; k += blockDim.x) val[k] = a.val[(size_t)9 * rc.s0 + k];
    if (cacheG)
        for (int k = threadIdx.x; k < 9 * ns; k += blockDim.x) gval[k] = a.gS[(size_t)9 * rc.s0 + k];
    const double* srcBlk = LEARNED ? a.S : a.Dinv;
    for (int k = threadIdx.x; k < 9 * nrows; k += blockDim.x) {
        dex[k] = a.diagExtra[(size_t)9 * rc.row0 + k];
        blk[k] = srcBlk[(size_t)9 * rc.row0 + k];
    }
    __syncthreads();  // dlo / dhi complete
    // the rows' contact slots are one contiguous window (row-sorted)
    const int nd = dhi > dlo ? dhi - dlo : 0;
    rc.d0 = (nd > 0 && nd <= a.dynCap) ? dlo : -1;
    if (rc.d0 >= 0) {
        for (int k = threadIdx.x; k < nd; k += blockDim.x) dcol[k] = a.dCol[dlo + k];
        for (int k = threadIdx.x; k < 9 * nd; k += blockDim.x) dval[k] = a.dVal[(size_t)9 * dlo + k];
        if (cacheG)
            for (int k = threadIdx.x; k < 9 * nd; k += blockDim.x) dgval[k] = a.gD[(size_t)9 * dlo + k];
    }
    __syncthreads();
    rc.rp = rp; rc.col = col; rc.val = val; rc.gval = cacheG ? gval : nullptr;
    rc.drs = drs; rc.dcol = dcol; rc.dval = dval; rc.dgval = cacheG ? dgval : nullptr;
    rc.dex = dex; rc.blk = blk;
    return rc;
}

// acc = (A u)_row without the diagonal extras, from the cache; every lane of
// the row's group gets the sum
template <class MT, class VT>
__device__ __forceinline__ void rowAxCached(const PcgArgs<MT, VT>& a, const RowCache<MT>& rc, const RowIter& it, int row, const VT* u,
                                            VT acc[3]) {
    const int lr = row - rc.row0;
    if (row < it.limit) {
        const int kb = rc.rp[lr] - rc.s0, ke = rc.rp[lr + 1] - rc.s0;
        // two of the lane's slots per round: both gathers are issued before
        // the products, which stay in slot order
        for (int kk = kb + it.lane; kk < ke; kk += 2 * GROUP) {
            const int k1 = kk + GROUP;
            const bool two = k1 < ke;
            const int c0 = rc.col[kk], c1 = two ? rc.col[k1] : c0;
            const VT x0[3] = {u[3 * c0], u[3 * c0 + 1], u[3 * c0 + 2]};
            const VT x1[3] = {u[3 * c1], u[3 * c1 + 1], u[3 * c1 + 2]};
            blockMulAdd(rc.val + (size_t)9 * kk, x0, acc);
            if (two) blockMulAdd(rc.val + (size_t)9 * k1, x1, acc);
        }
        const int ds = rc.drs[2 * lr], de = rc.drs[2 * lr + 1];
        if (rc.d0 >= 0) {
            for (int k = ds + it.lane; k < de; k += GROUP) {
                int kk = k - rc.d0;
                int c = rc.dcol[kk];
                VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
                blockMulAdd(rc.dval + (size_t)9 * kk, xv, acc);
            }
        } else {
            for (int k = ds + it.lane; k < de; k += GROUP) {
                int c = a.dCol[k];
                VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
                blockMulAdd(a.dVal + (size_t)9 * k, xv, acc);
            }
        }
    }
    groupReduce3(acc);
}

// (G u)_row (TR false) or (G^T u)_row (TR true) from the cache, as rowFactor
template <bool TR, class MT, class VT>
__device__ __forceinline__ void rowFactorCached(const PcgArgs<MT, VT>& a, const RowCache<MT>& rc, const RowIter& it, int row, const VT* u,
                                                VT acc[3]) {
    const int lr = row - rc.row0;
    const int kb = rc.rp[lr] - rc.s0, ke = rc.rp[lr + 1] - rc.s0;
    // the factor block of slot kk (transposed on the diagonal of G^T)
    auto slotMulAdd = [&](int kk, int c, const VT* xv) {
        const float* B = rc.gval ? rc.gval + (size_t)9 * kk : a.gS + (size_t)9 * (kk + rc.s0);
        if (TR && c == row) {
            for (int q = 0; q < 3; ++q) acc[q] += (VT)B[q] * xv[0] + (VT)B[3 + q] * xv[1] + (VT)B[6 + q] * xv[2];
        } else {
            blockMulAdd(B, xv, acc);
        }
    };
    // two of the lane's slots per round, as rowAxCached; slots outside this
    // pass's triangle are skipped
    for (int kk = kb + it.lane; kk < ke; kk += 2 * GROUP) {
        const int k1 = kk + GROUP;
        const int c0 = rc.col[kk], c1 = k1 < ke ? rc.col[k1] : row;
        const bool on0 = !(TR ? c0 < row : c0 > row), on1 = k1 < ke && !(TR ? c1 < row : c1 > row);
        const int g0 = on0 ? c0 : row, g1 = on1 ? c1 : row;
        const VT x0[3] = {u[3 * g0], u[3 * g0 + 1], u[3 * g0 + 2]};
        const VT x1[3] = {u[3 * g1], u[3 * g1 + 1], u[3 * g1 + 2]};
        if (on0) slotMulAdd(kk, c0, x0);
        if (on1) slotMulAdd(k1, c1, x1);
    }
    const int ds = rc.drs[2 * lr], de = rc.drs[2 * lr + 1];
    for (int k = ds + it.lane; k < de; k += GROUP) {
        const bool cached = rc.d0 >= 0;
        int c = cached ? rc.dcol[k - rc.d0] : a.dCol[k];
        if (TR ? c <= row : c >= row) continue;
        VT xv[3] = {u[3 * c], u[3 * c + 1], u[3 * c + 2]};
        blockMulAdd((cached && rc.dgval) ? rc.dgval + (size_t)9 * (k - rc.d0) : a.gD + (size_t)9 * k, xv, acc);
    }
}

// out = S^T G^T G tmp for the factor, where tmp = S w was written by the
// rows' owners before the call: barrier, t = G tmp, barrier, out = S^T G^T t
// into outG (gathered by neighbours) and into the owner's shared copy
// own[3 * local row + q].  Ends without a barrier; false on timeout.
template <class MT, class VT>
__device__ bool factorCachedPasses(const PcgArgs<MT, VT>& a, const RowCache<MT>& rc, const RowIter& it, const VT* tmp, VT* outG, VT* own,
                                   unsigned& ep) {
    const unsigned nb = gridDim.x;
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return false;
    for (int base = it.first; base < it.limit; base += it.stride) {
        int row = base + it.grp;
        bool active = row < it.limit;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) rowFactorCached<false>(a, rc, it, row, tmp, acc);
        groupReduce3(acc);
        // lanes 0, 1, 2 of the group store components 0, 1, 2
        const int q = it.lane;
        if (active && q < 3) a.t[3 * row + q] = q == 0 ? acc[0] : (q == 1 ? acc[1] : acc[2]);
    }
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return false;
    for (int base = it.first; base < it.limit; base += it.stride) {
        int row = base + it.grp;
        bool active = row < it.limit;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) rowFactorCached<true>(a, rc, it, row, (const VT*)a.t, acc);
        groupReduce3(acc);
        const int q = it.lane;
        if (active && q < 3) {
            // component q of S^T y (S lower triangular)
            const int lr = row - rc.row0;
            const double* S = rc.blk + 9 * lr;
            const double y0 = acc[0], y1 = acc[1], y2 = acc[2];
            const VT o = (VT)(q == 0 ? S[0] * y0 + S[3] * y1 + S[6] * y2 : (q == 1 ? S[4] * y1 + S[7] * y2 : S[8] * y2));
            outG[3 * row + q] = o;
            own[3 * lr + q] = o;
        }
    }
    return true;
}

// acc = (A u)_row without the diagonal extras; every lane of the group gets the sum
template <class MT, class VT>
__device__ __forceinline__ void rowAx(const PcgArgs<MT, VT>& a, const RowIter& it, int row, const VT* u, VT acc[3]) {
    if (row < a.nv) rowSpmv(a, row, it.lane, u, acc);
    groupReduce3(acc);
}

// out = M^-1 w for the factor, with tmp = S w already written by the rows'
// owners in the pass before: barrier, t = G tmp, barrier, out = S^T G^T t.
// Ends without a barrier; false on timeout.
template <class MT, class VT>
__device__ bool factorPasses(const PcgArgs<MT, VT>& a, const RowIter& it, const VT* tmp, VT* out, unsigned& ep) {
    const unsigned nb = gridDim.x;
    const int q = it.lane;
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return false;
    for (int base = it.first; base < a.nv; base += it.stride) {
        int row = base + it.grp;
        bool active = row < a.nv;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) rowFactor<false>(a, row, it.lane, tmp, acc);
        groupReduce3(acc);
        // lanes 0, 1, 2 of the group store components 0, 1, 2
        if (active && q < 3) a.t[3 * row + q] = q == 0 ? acc[0] : (q == 1 ? acc[1] : acc[2]);
    }
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return false;
    for (int base = it.first; base < a.nv; base += it.stride) {
        int row = base + it.grp;
        bool active = row < a.nv;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        if (active) rowFactor<true>(a, row, it.lane, (const VT*)a.t, acc);
        groupReduce3(acc);
        if (active && q < 3) {
            // component q of S^T y (S lower triangular)
            const double* S = a.S + 9 * (size_t)row;
            const double y0 = acc[0], y1 = acc[1], y2 = acc[2];
            out[3 * row + q] = (VT)(q == 0 ? S[0] * y0 + S[3] * y1 + S[6] * y2 : (q == 1 ? S[4] * y1 + S[7] * y2 : S[8] * y2));
        }
    }
    return true;
}

// MINB: blocks per SM the compiler must fit (registers: 64 per thread for
// 2, the build of the single-pass kernel and of the two-block streaming
// kernel); 3 and 4 for the streaming builds that trade register spills for
// 48 or 64 resident warps
template <class MT, class VT, bool LEARNED, bool CACHED, int MINB = 2>
__global__ void __launch_bounds__(PB, MINB) pcgPipelinedKernel(PcgArgs<MT, VT> a) {
    extern __shared__ __align__(16) unsigned char pipeSmem[];
    // In a single-pass launch (CACHED) the block's matrix rows and its rows'
    // recurrence vectors live in shared memory: only the gathered vectors
    // (u once; m, and with a factor S w and t, every iteration), the partial
    // sums and the solution at the end touch global memory.  Lanes 0, 1, 2
    // of a row's group update components 0, 1, 2 of the row's vectors.
    const unsigned nb = gridDim.x;
    unsigned ep = 0;
    const int nv = a.nv;
    const RowIter it = CACHED ? RowIter(a.nv, a.rowsPerBlock) : RowIter();
    const int rEnd = CACHED ? it.limit : a.nv;  // rows this thread's loops cover end here
    const int q = it.lane;  // the component this lane updates (q < 3)
    RowCache<MT> rc{};
    VT* sv = nullptr;
    if (CACHED) {
        rc = loadRowCache<MT, VT, LEARNED>(a, pipeSmem);
        const bool cacheG = LEARNED && a.cacheG != 0;
        sv = reinterpret_cast<VT*>(pipeSmem + smemLayout(a.sliceMax, a.dynCap, cacheG, (int)sizeof(MT), (int)sizeof(VT)).state);
    }
    // component q of own-row vector k (0 x, 1 r, 2 u, 3 w, 4 z, 5 q, 6 s, 7 p)
    auto V = [&](int k, int row) -> VT& {
        if (CACHED) return sv[(k * ROWS_PER_BLOCK + (row - rc.row0)) * 3 + q];
        VT* g = k == 0 ? a.x : k == 1 ? a.r : k == 2 ? a.u : k == 3 ? a.w : k == 4 ? a.z : k == 5 ? a.q : k == 6 ? a.s : a.p;
        return g[3 * row + q];
    };
    VT* const ownM = CACHED ? sv + 8 * ROWS_PER_BLOCK * 3 : nullptr;  // the rows' own m (shared copy)
    VT* const ownU = CACHED ? sv + 2 * ROWS_PER_BLOCK * 3 : nullptr;
    auto Ax = [&](int row, const VT* u, VT acc[3]) {
        if (CACHED) rowAxCached(a, rc, it, row, u, acc);
        else rowAx(a, it, row, u, acc);
    };
    auto pick = [&](const VT v[3]) { return q == 0 ? v[0] : (q == 1 ? v[1] : v[2]); };
    // component q of D v for a row's 3x3 block D (row-major), v given whole
    auto rowDot = [&](const double* D, const VT v[3]) {
        return (VT)(D[3 * q] * (double)v[0] + D[3 * q + 1] * (double)v[1] + D[3 * q + 2] * (double)v[2]);
    };
    auto dexRow = [&](int row) { return CACHED ? rc.dex + 9 * (row - rc.row0) : a.diagExtra + 9 * (size_t)row; };
    auto blkRow = [&](int row) { return CACHED ? rc.blk + 9 * (row - rc.row0) : a.Dinv + 9 * (size_t)row; };
    // the group's three components of v (held by lanes 0, 1, 2); every lane calls
    auto share3 = [&](VT v, VT out[3]) {
        out[0] = __shfl_sync(0xffffffffu, v, 0, GROUP);
        out[1] = __shfl_sync(0xffffffffu, v, 1, GROUP);
        out[2] = __shfl_sync(0xffffffffu, v, 2, GROUP);
    };
    VT* sw = a.Ap;  // S w, gathered by the factor's first pass
    // the row's M-related output from the group's three components of v:
    // block-Jacobi m = Dinv v into mOut (and the shared copy), or with a
    // factor S v into sw, the input of the factor's first pass; lanes q < 3
    // of active rows store
    auto precondRow = [&](int row, bool active, const VT v[3], VT* mOut) {
        if (!active || q >= 3) return;
        if (!LEARNED) {
            const VT mq = rowDot(blkRow(row), v);
            mOut[3 * row + q] = mq;
            if (CACHED) ownM[3 * (row - rc.row0) + q] = mq;
        } else {
            // lower triangular
            const double* S = CACHED ? rc.blk + 9 * (row - rc.row0) : a.S + 9 * (size_t)row;
            const double v0 = v[0], v1 = v[1], v2 = v[2];
            sw[3 * row + q] = (VT)(q == 0 ? S[0] * v0 : (q == 1 ? S[3] * v0 + S[4] * v1 : S[6] * v0 + S[7] * v1 + S[8] * v2));
        }
    };
    auto part = [&](int set, int k) { return a.pp + (size_t)(3 * set + k) * PIPE_PMAX; };
    // x = 0, r = b, u = M r; the recurrence vectors start at 0
    double rr = 0;
    for (int base = it.first; base < rEnd; base += it.stride) {
        const int row = base + it.grp;
        const bool active = row < rEnd;
        VT rq = VT(0);
        if (active && q < 3) {
            V(0, row) = VT(0); V(4, row) = VT(0); V(5, row) = VT(0); V(6, row) = VT(0); V(7, row) = VT(0);
            rq = a.b[3 * row + q];
            V(1, row) = rq;
            rr += (double)rq * (double)rq;
        }
        VT rv[3];
        share3(rq, rv);
        if (!LEARNED) {
            if (active && q < 3) {
                const VT uq = rowDot(blkRow(row), rv);
                V(2, row) = uq;
                a.u[3 * row + q] = uq;
            }
        } else {
            precondRow(row, active, rv, nullptr);
        }
    }
    if (LEARNED) {
        if (CACHED) {
            if (!factorCachedPasses(a, rc, it, (const VT*)sw, a.u, ownU, ep)) return;
        } else if (!factorPasses(a, it, (const VT*)sw, a.u, ep)) {
            return;
        }
    }
    if (!gridBarrier(a.bar, a.flag, nb, ep)) return;
    // w = A u, m = M w, gamma = (r,u), delta = (w,u)
    double g = 0, dl = 0;
    for (int base = it.first; base < rEnd; base += it.stride) {
        const int row = base + it.grp;
        const bool active = row < rEnd;
        VT acc[3] = {VT(0), VT(0), VT(0)};
        Ax(row, (const VT*)a.u, acc);
        VT wq = VT(0);
        if (active && q < 3) {
            const VT* uOwn = CACHED ? ownU + 3 * (row - rc.row0) : a.u + 3 * row;
            const VT uo[3] = {uOwn[0], uOwn[1], uOwn[2]};
            wq = pick(acc) + rowDot(dexRow(row), uo);
            V(3, row) = wq;
            const VT uq = V(2, row);
            g += (double)V(1, row) * (double)uq;
            dl += (double)wq * (double)uq;
        }
        VT wv[3];
        share3(wq, wv);
        precondRow(row, active, wv, a.mA);
    }
    blockReduce3(rr, g, dl);
    if (threadIdx.x == 0) { part(0, 0)[blockIdx.x] = rr; part(0, 1)[blockIdx.x] = g; part(0, 2)[blockIdx.x] = dl; }
    if (LEARNED) {
        if (CACHED) {
            if (!factorCachedPasses(a, rc, it, (const VT*)sw, a.mA, ownM, ep)) return;
        } else if (!factorPasses(a, it, (const VT*)sw, a.mA, ep)) {
            return;
        }
    }
    {
        double sums[3];
        if (!gridBarrierSum<3>(a.bar, a.flag, nb, ep, part(0, 0), PIPE_PMAX, sums)) return;
        rr = sums[0]; g = sums[1]; dl = sums[2];
    }
    const double rhs2 = rr;
    const double thr = fmax(a.tol * a.tol * rr, 2.2250738585072014e-308);
    int iter = 0;
    int status = (rr == 0.0 || rr < thr) ? 1 : 0;
    double gPrev = 1.0, alphaPrev = 1.0;
    while (status == 0) {
        double beta = iter == 0 ? 0.0 : g / gPrev;
        double den = iter == 0 ? dl : dl - beta * g / alphaPrev;
        if (!(den != 0.0) || !isfinite(den)) { status = 2; break; }  // breakdown: the caller's true residual decides
        double alpha = g / den;
        const VT* mCur = (LEARNED || (iter & 1) == 0) ? a.mA : a.mB;
        VT* mNext = LEARNED ? a.mA : ((iter & 1) == 0 ? a.mB : a.mA);
        const VT bt = (VT)beta, al = (VT)alpha;
        double lrr = 0, lg = 0, ld = 0;
        for (int base = it.first; base < rEnd; base += it.stride) {
            const int row = base + it.grp;
            const bool active = row < rEnd;
            VT acc[3] = {VT(0), VT(0), VT(0)};
            Ax(row, mCur, acc);
            VT wq = VT(0);
            if (active && q < 3) {
                const VT* mOwn = CACHED ? ownM + 3 * (row - rc.row0) : mCur + 3 * row;
                const VT mo[3] = {mOwn[0], mOwn[1], mOwn[2]};
                const VT zv = pick(acc) + rowDot(dexRow(row), mo) + bt * V(4, row);
                const VT qv = pick(mo) + bt * V(5, row);
                const VT sq = V(3, row) + bt * V(6, row);
                const VT pv = V(2, row) + bt * V(7, row);
                V(4, row) = zv; V(5, row) = qv; V(6, row) = sq; V(7, row) = pv;
                V(0, row) += al * pv;
                const VT rv = V(1, row) - al * sq;
                const VT uv = V(2, row) - al * qv;
                wq = V(3, row) - al * zv;
                V(1, row) = rv; V(2, row) = uv; V(3, row) = wq;
                lrr += (double)rv * (double)rv;
                lg += (double)rv * (double)uv;
                ld += (double)wq * (double)uv;
            }
            VT wv[3];
            share3(wq, wv);
            precondRow(row, active, wv, mNext);
        }
        const int set = (iter + 1) & 1;
        blockReduce3(lrr, lg, ld);
        if (threadIdx.x == 0) { part(set, 0)[blockIdx.x] = lrr; part(set, 1)[blockIdx.x] = lg; part(set, 2)[blockIdx.x] = ld; }
        // the factor's m is replaced only in its last pass, two barriers
        // after every row read it
        if (LEARNED) {
            if (CACHED) {
                if (!factorCachedPasses(a, rc, it, (const VT*)sw, mNext, ownM, ep)) return;
            } else if (!factorPasses(a, it, (const VT*)sw, mNext, ep)) {
                return;
            }
        }
        double sums[3];
        if (!gridBarrierSum<3>(a.bar, a.flag, nb, ep, part(set, 0), PIPE_PMAX, sums)) return;
        gPrev = g;
        alphaPrev = alpha;
        rr = sums[0]; g = sums[1]; dl = sums[2];
        ++iter;
        if (rr < thr) { status = 1; break; }
        if (iter >= a.maxIter || !isfinite(rr)) { status = 2; break; }
    }
    if (CACHED) {
        // the solution leaves shared memory
        for (int base = it.first; base < rEnd; base += it.stride) {
            const int row = base + it.grp;
            if (row < rEnd && q < 3) a.x[3 * row + q] = V(0, row);
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.scal[3] = rr;
        a.scal[4] = iter;
        a.scal[6] = rhs2;
        atomicCAS(a.flag, 0, status);  // a barrier timeout (3) stands
    }
}

__global__ void accumulateKernelD(int n3, const double* d, double* x) {
    CIPC_KERNEL_LOOP(i, n3) x[i] += d[i];
}

__global__ void zeroKernel(int n3, double* x) {
    CIPC_KERNEL_LOOP(i, n3) x[i] = 0.0;
}

}  // namespace

// packed[k] = the FP16 block of slot slot[k] of G (transposed where the
// slot is stored as ~slot: the diagonal blocks of the transposed part)
__global__ void packFactorKernel(int n, const int* slot, const float* gS, __half* out) {
    CIPC_KERNEL_LOOP(i, 9 * n) {
        const int k = i / 9, e = i - 9 * k;
        const int s = slot[k];
        const bool tr = s < 0;
        const int src = tr ? 3 * (e % 3) + e / 3 : e;
        out[i] = __float2half_rn(gS[(size_t)9 * (tr ? ~s : s) + src]);
    }
}

// The factor's static blocks in the packed layout the streaming PCG reads
// (rowFactor): per row the slots with column <= row (G), then those with
// column >= row (G^T: the mirror slots, and the diagonal transposed).  The
// index lists follow the static pattern and are built on the first call.
static void packFactor(Ctx& c) {
    const int nv = c.nv;
    if (c.nGL == 0) {
        std::vector<int> col(c.nnzb);
        CIPC_CUDA(cudaMemcpy(col.data(), c.colIdx.p, sizeof(int) * c.nnzb, cudaMemcpyDeviceToHost));
        std::vector<int> lp(nv + 1, 0), lc, ls, up(nv + 1, 0), uc, us;
        lc.reserve(c.nnzb / 2 + nv); ls.reserve(c.nnzb / 2 + nv); uc.reserve(c.nnzb / 2 + nv); us.reserve(c.nnzb / 2 + nv);
        for (int r = 0; r < nv; ++r) {
            for (int k = c.hRowPtr[r]; k < c.hRowPtr[r + 1]; ++k) {
                const int cl = col[k];
                if (cl <= r) { lc.push_back(cl); ls.push_back(k); }
                if (cl >= r) { uc.push_back(cl); us.push_back(cl == r ? ~k : k); }
            }
            lp[r + 1] = (int)lc.size();
            up[r + 1] = (int)uc.size();
        }
        auto up_ = [&](DBuf<int>& d, const std::vector<int>& h) {
            d.reserve(std::max<size_t>(h.size(), 1));
            if (!h.empty()) CIPC_CUDA(cudaMemcpy(d.p, h.data(), sizeof(int) * h.size(), cudaMemcpyHostToDevice));
        };
        up_(c.gLptr, lp); up_(c.gLcol, lc); up_(c.gLslot, ls); up_(c.gUptr, up); up_(c.gUcol, uc); up_(c.gUslot, us);
        c.nGL = (int)lc.size();
        c.nGU = (int)uc.size();
        c.gLval.reserve(9 * (size_t)std::max(1, c.nGL));
        c.gUval.reserve(9 * (size_t)std::max(1, c.nGU));
    }
    const int vb = std::max(1, std::min((9 * c.nGL + VB - 1) / VB, 148 * 16));
    launch(packFactorKernel, vb, VB, 0, c.s, c.nGL, (const int*)c.gLslot, (const float*)c.mpGS, reinterpret_cast<__half*>(c.gLval.p));
    const int ub = std::max(1, std::min((9 * c.nGU + VB - 1) / VB, 148 * 16));
    launch(packFactorKernel, ub, VB, 0, c.s, c.nGU, (const int*)c.gUslot, (const float*)c.mpGS, reinterpret_cast<__half*>(c.gUval.p));
    CIPC_CUDA(cudaGetLastError());
}

void buildRhs(Ctx& c) {
    c.rhs.reserve(3 * c.nv);
    launch(rhsKernel, vecBlocks(c.nv), VB, 0, c.s, c.nv, c.grad, c.btype, c.rhs);
    CIPC_CUDA(cudaGetLastError());
}

template <class MT, class VT>
static void spmvT(Ctx& c, const MT* val, const MT* dval, const VT* x, VT* y, double* partial, const int* flag, int nblk) {
    bool dyn = c.nDynB > 0;
    launch(spmvKernel<MT, VT>, nblk, VB, 0, c.s, c.nv, c.rowPtr, c.colIdx, val, dyn ? c.dynRowStart.p : nullptr, dyn ? c.dynRowEnd.p : nullptr,
           dyn ? c.dynCol.p : nullptr, dval, c.diagExtra, x, y, partial, flag);
}

static int spmvBlocks(Ctx& c) { return std::max(1, std::min((c.nv * GROUP + VB - 1) / VB, MAXPART)); }

void spmv(Ctx& c, const double* x, double* y) {
    if (c.mixed) spmvT<float, double>(c, c.valF, c.dynBF, x, y, nullptr, nullptr, spmvBlocks(c));
    else spmvT<double, double>(c, c.valD, c.dynBD, x, y, nullptr, nullptr, spmvBlocks(c));
    CIPC_CUDA(cudaGetLastError());
}

static void computeDinv(Ctx& c) {
    int nv = c.nv;
    bool dyn = c.nDynB > 0;
    c.Dinv.reserve(9 * (size_t)nv);
    if (c.mixed)
        launch(dinvKernel<float>, vecBlocks(nv), VB, 0, c.s, nv, c.diagSlot, c.valF, dyn ? c.dynRowStart.p : nullptr, dyn ? c.dynRowEnd.p : nullptr,
               dyn ? c.dynCol.p : nullptr, c.dynBF, c.diagExtra, c.Dinv);
    else
        launch(dinvKernel<double>, vecBlocks(nv), VB, 0, c.s, nv, c.diagSlot, c.valD, dyn ? c.dynRowStart.p : nullptr, dyn ? c.dynRowEnd.p : nullptr,
               dyn ? c.dynCol.p : nullptr, c.dynBD, c.diagExtra, c.Dinv);
}

// PCG on A x = b with vectors of type VT and blocks of type MT.  Returns the
// iteration count; *relRes gets sqrt(rr/rhs2) of the last recursive residual.
template <class MT, class VT>
static int runPcg(Ctx& c, const MT* val, const MT* dval, const VT* b, VT* x, VT* r, VT* z, VT* p, VT* Ap, double tol, int maxIter,
                  int& flagOut, double& relRes) {
    int nv = c.nv;
    int vb = vecBlocks(nv), sb = spmvBlocks(c);
    double* partA = c.red.p;
    double* partB = c.red.p + MAXPART;
    double* partC = c.red.p + 2 * MAXPART;
    int* flag = c.counters.p + 10;
    launch(pcgInitKernel<VT>, vb, VB, 0, c.s, nv, b, c.Dinv, x, r, z, p, partA, partB);
    launch(pcgInitScalars, 1, VB, 0, c.s, partA, partB, vb, tol, c.scal, flag);
    CIPC_CUDA(cudaGetLastError());
    const int chunk = 16;
    int it = 0;
    int hflag = 0;
    double hs[8];
    while (true) {
        for (int k = 0; k < chunk; ++k) {
            profBegin(c, PROF_SPMV);
            spmvT<MT, VT>(c, val, dval, p, Ap, partC, flag, sb);
            profEnd(c, PROF_SPMV);
            launch(pcgUpdateKernel<VT>, vb, VB, 0, c.s, nv, partC, sb, c.scal, c.Dinv, p, Ap, x, r, z, partA, partB, flag);
            launch(pcgScalarKernel, 1, VB, 0, c.s, partA, partB, vb, c.scal, flag, maxIter);
            launch(pcgDirKernel<VT>, vb, VB, 0, c.s, nv, c.scal, z, p, flag);
        }
        CIPC_CUDA(cudaGetLastError());
        CIPC_CUDA(cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        CIPC_CUDA(cudaMemcpyAsync(hs, c.scal.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
        hostSync(c);
        it = (int)hs[4];
        if (hflag) break;
    }
    flagOut = hflag;
    relRes = hs[6] > 0 ? std::sqrt(hs[3] / hs[6]) : 0.0;
    return it;
}

constexpr int PMAX = 1024;  // max blocks of the persistent PCG

// Blocks per SM of the persistent PCG: CIPC_PCG_BLOCKS_PER_SM (1-8) or 2.
static int pcgBlocksPerSm() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("CIPC_PCG_BLOCKS_PER_SM");
        int k = e ? std::atoi(e) : 2;
        v = std::min(8, std::max(1, k));
    }
    return v;
}

// CIPC_PCG_CLASSIC=1 selects the textbook recurrences (two barriers per
// iteration with block-Jacobi); the default is the pipelined kernel.
static bool pcgClassic() {
    static int v = -1;
    if (v < 0) { const char* e = std::getenv("CIPC_PCG_CLASSIC"); v = (e && *e == '1') ? 1 : 0; }
    return v == 1;
}

// Blocks per SM of the streaming kernel's build: 3 by default (48 resident
// warps for a few register spills: measured 10-24 % faster per solve on the
// pile than two blocks per SM); CIPC_PCG_OCC=2 or 4 selects the other builds.
static int pcgOcc() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("CIPC_PCG_OCC");
        v = e ? std::atoi(e) : 3;
        if (v != 2 && v != 4) v = 3;
    }
    return v;
}

// CIPC_PCG_NOPACK=1 keeps the streaming kernel on the slot-aligned FP32 factor.
static bool pcgNoPack() {
    static int v = -1;
    if (v < 0) { const char* e = std::getenv("CIPC_PCG_NOPACK"); v = (e && *e == '1') ? 1 : 0; }
    return v == 1;
}

// CIPC_PCG_NOCACHE=1 keeps the pipelined kernel's matrix rows in global memory.
static bool pcgNoCache() {
    static int v = -1;
    if (v < 0) { const char* e = std::getenv("CIPC_PCG_NOCACHE"); v = (e && *e == '1') ? 1 : 0; }
    return v == 1;
}

// Largest number of static slots over the row ranges the cached kernel's
// blocks own (computed once per context from the static pattern).
// CIPC_DEBUG_PCG=1 prints every inner solve and fallback to stderr.
static bool debugPcg() {
    static int v = -1;
    if (v < 0) { const char* e = std::getenv("CIPC_DEBUG_PCG"); v = (e && *e == '1') ? 1 : 0; }
    return v == 1;
}

// largest static-slot count of `rows` consecutive rows starting at a multiple of rows
static int pcgSliceMax(Ctx& c, int rows) {
    if (c.pcgSliceMax < 0 || c.pcgSliceRows != rows) {
        int m = 0;
        for (int r0 = 0; r0 < c.nv; r0 += rows) {
            int r1 = std::min(c.nv, r0 + rows);
            m = std::max(m, c.hRowPtr[r1] - c.hRowPtr[r0]);
        }
        c.pcgSliceMax = m;
        c.pcgSliceRows = rows;
    }
    return c.pcgSliceMax;
}

template <class MT, class VT, bool LEARNED>
static void launchPersistent(Ctx& c, PcgArgs<MT, VT>& a, int smCount, bool classic) {
    int needed = std::max(1, (c.nv * GROUP + PB - 1) / PB);
    int cap = std::min(PMAX, PIPE_PMAX);
    void* args[] = {&a};
    a.dynCap = 0;
    a.cacheG = 0;
    if (!classic && !pcgNoCache() && !c.hRowPtr.empty() && needed <= cap) {
        // single-pass launch: each block owns ROWS_PER_BLOCK rows for the whole
        // solve and stages them in shared memory.  The largest configuration
        // that keeps every block resident is taken: the factor's blocks
        // cached or not, a contact window of 512 down to 0 slots.
        // rows spread evenly over at least one block per SM
        const int rows = (c.nv + std::max(needed, smCount) - 1) / std::max(needed, smCount);
        const int nbRows = (c.nv + rows - 1) / rows;
        a.rowsPerBlock = rows;
        a.sliceMax = pcgSliceMax(c, rows);
        const void* fn = (const void*)pcgPipelinedKernel<MT, VT, LEARNED, true>;
        int maxOptin = 0, dev = 0;
        CIPC_CUDA(cudaGetDevice(&dev));
        CIPC_CUDA(cudaDeviceGetAttribute(&maxOptin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
        const bool dyn = a.dRowS != nullptr;
        static const int dynCaps[] = {512, 256, 128, 0};
        for (int cg = LEARNED ? 1 : 0; cg >= 0; --cg) {
            for (int dc : dynCaps) {
                if (!dyn && dc > 0) continue;
                size_t smem = smemLayout(a.sliceMax, dc, cg != 0, (int)sizeof(MT), (int)sizeof(VT)).total;
                if (smem + 4096 > (size_t)maxOptin) continue;
                CIPC_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
                int perSM = 0;
                CIPC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, PB, smem));
                if (perSM >= 1 && nbRows <= perSM * smCount && nbRows <= cap) {
                    a.dynCap = dc;
                    a.cacheG = cg;
                    if (debugPcg())
                        std::fprintf(stderr, "[pcg] single-pass launch: %d blocks of %d rows, slice %d, contact window %d, factor cached %d, %zu B shared\n",
                                     nbRows, rows, a.sliceMax, dc, cg, smem);
                    ++g_kernelLaunches;
                    CIPC_CUDA(cudaLaunchCooperativeKernel(fn, dim3(nbRows), dim3(PB), args, smem, c.s));
                    return;
                }
            }
        }
    }
    a.sliceMax = 0;
    a.rowsPerBlock = 0;
    const int occ = classic ? 0 : pcgOcc();
    const void* fn = classic ? (const void*)pcgPersistentKernel<MT, VT, LEARNED>
                   : occ == 4 ? (const void*)pcgPipelinedKernel<MT, VT, LEARNED, false, 4>
                   : occ == 3 ? (const void*)pcgPipelinedKernel<MT, VT, LEARNED, false, 3>
                              : (const void*)pcgPipelinedKernel<MT, VT, LEARNED, false>;
    int perSM = 0;
    CIPC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, PB, 0));
    if (perSM < 1) throw std::runtime_error("persistent PCG kernel does not fit on an SM");
    int grid = std::max(1, std::min(std::min(std::min(perSM, occ >= 3 ? occ : pcgBlocksPerSm()) * smCount, needed), cap));
    ++g_kernelLaunches;
    CIPC_CUDA(cudaLaunchCooperativeKernel(fn, dim3(grid), dim3(PB), args, 0, c.s));
}

// Whole PCG in one cooperative launch (grid sized to what is co-resident).
// learned: apply the factor in c.mpS / c.mpGS / c.mpGD instead of block-Jacobi.
template <class MT, class VT>
static int runPcgPersistent(Ctx& c, const MT* val, const MT* dval, const VT* b, VT* x, VT* r, VT* z, VT* p, VT* Ap, double tol, int maxIter,
                            int& flagOut, double& relRes, bool learned = false, bool classic = false) {
    static int smCount = 0, coop = -1;
    if (coop < 0) {
        int dev = 0;
        CIPC_CUDA(cudaGetDevice(&dev));
        CIPC_CUDA(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, dev));
        CIPC_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    }
    if (!coop) {
        if (learned) throw std::runtime_error("the learned preconditioner needs cooperative launch support");
        return runPcg<MT, VT>(c, val, dval, b, x, r, z, p, Ap, tol, maxIter, flagOut, relRes);
    }
    bool dyn = c.nDynB > 0;
    PcgArgs<MT, VT> a;
    a.nv = c.nv; a.rowPtr = c.rowPtr; a.col = c.colIdx; a.val = val;
    a.dRowS = dyn ? c.dynRowStart.p : nullptr; a.dRowE = dyn ? c.dynRowEnd.p : nullptr; a.dCol = dyn ? c.dynCol.p : nullptr; a.dVal = dval;
    a.diagExtra = c.diagExtra; a.Dinv = c.Dinv; a.b = b; a.x = x; a.r = r; a.z = z; a.p = p; a.Ap = Ap;
    a.S = nullptr; a.gS = nullptr; a.gD = nullptr; a.t = nullptr;
    a.gL = a.gU = nullptr; a.gLptr = a.gLcol = a.gUptr = a.gUcol = nullptr;
    if (learned) {
        c.mpT.reserve(3 * (size_t)c.nv);
        a.S = c.mpS.p; a.gS = c.mpGS.p; a.gD = c.mpGD.p; a.t = reinterpret_cast<VT*>(c.mpT.p);
        if (c.factorPacked) {
            a.gL = reinterpret_cast<const __half*>(c.gLval.p); a.gU = reinterpret_cast<const __half*>(c.gUval.p);
            a.gLptr = c.gLptr.p; a.gLcol = c.gLcol.p; a.gUptr = c.gUptr.p; a.gUcol = c.gUcol.p;
        }
    }
    a.partA = c.red.p; a.partB = c.red.p + PMAX; a.partC = c.red.p + 2 * PMAX;
    // pipelined kernel: six more vectors and two sets of partial sums
    size_t n3 = 3 * (size_t)c.nv;
    c.pcgPipe.reserve(6 * n3 * sizeof(VT) / sizeof(double) + 6);
    VT* pv = reinterpret_cast<VT*>(c.pcgPipe.p);
    a.u = pv; a.w = pv + n3; a.mA = pv + 2 * n3; a.mB = pv + 3 * n3; a.q = pv + 4 * n3; a.s = pv + 5 * n3;
    c.pcgParts.reserve(6 * (size_t)PIPE_PMAX);
    a.pp = c.pcgParts.p;
    a.scal = c.scal.p; a.flag = c.counters.p + 10;
    c.pcgBar.reserve(BAR_WORDS);
    a.bar = c.pcgBar.p;
    a.tol = tol; a.maxIter = maxIter;
    CIPC_CUDA(cudaMemsetAsync(c.counters.p + 10, 0, sizeof(int), c.s));
    CIPC_CUDA(cudaMemsetAsync(c.pcgBar.p, 0, BAR_WORDS * sizeof(unsigned), c.s));
    profBegin(c, PROF_PCG);
    classic = classic || pcgClassic();
    if (learned) launchPersistent<MT, VT, true>(c, a, smCount, classic);
    else launchPersistent<MT, VT, false>(c, a, smCount, classic);
    profEnd(c, PROF_PCG);
    int hflag = 0;
    double hs[8];
    CIPC_CUDA(cudaMemcpyAsync(&hflag, a.flag, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    CIPC_CUDA(cudaMemcpyAsync(hs, c.scal.p, 8 * sizeof(double), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    if (hflag == 3) throw std::runtime_error("device status in PCG: grid barrier timed out");
    flagOut = hflag;
    relRes = hs[6] > 0 ? std::sqrt(hs[3] / hs[6]) : 0.0;
    c.lastPcgLaunchIters = (int)hs[4];
    return (int)hs[4];
}

static void reservePcg(Ctx& c) {
    size_t n3 = 3 * (size_t)c.nv;
    c.sol.reserve(n3); c.r.reserve(n3); c.z.reserve(n3); c.p.reserve(n3); c.Ap.reserve(n3);
    c.red.reserve(4 * PMAX + 16);
    c.scal.reserve(16);
    c.counters.reserve(16);
}

// Builds the factor for the current system (network forward, or the exact
// FSAI); false when block-Jacobi is selected.
static bool prepareLearned(Ctx& c) {
    c.factorPacked = false;
    if (c.precond == CIPC_PRECOND_FSAI) {
        mpnnPrepare(c, false);
        fsaiBuild(c);
    } else if (c.precond == CIPC_PRECOND_LEARNED) {
        if (!c.mpReady) mpnnInitWeights(c, 1);
        mpnnPrepare(c);
        mpnnForward(c);
    } else {
        return false;
    }
    // the streaming kernel (systems too large for the single-pass cache)
    // reads the factor's static part packed by rows in FP16
    if (!pcgNoPack()) {
        packFactor(c);
        c.factorPacked = true;
    }
    return true;
}

// ||rhs - A sol||^2 in FP64 (FP32 blocks promoted in mixed mode)
static double trueResidual2(Ctx& c) {
    int nv = c.nv, n3 = 3 * nv;
    c.rF.reserve(n3);
    double* part = c.red.p + 3 * MAXPART;
    if (c.mixed) spmvT<float, double>(c, c.valF, c.dynBF, c.sol.p, c.Ap.p, nullptr, nullptr, spmvBlocks(c));
    else spmvT<double, double>(c, c.valD, c.dynBD, c.sol.p, c.Ap.p, nullptr, nullptr, spmvBlocks(c));
    int nb = vecBlocks(nv);
    launch(residualKernel, nb, VB, 0, c.s, n3, c.rhs.p, c.Ap.p, c.r.p, c.rF.p, part);
    return deviceSum(c, part, nb);
}

// Iteration cap of one solve with a factor preconditioner before block-Jacobi
// takes over (CIPC_FACTOR_CAP, default 1000): a factor that does not reach
// the inner tolerance within it is rejected rather than iterated further.
static int factorCap() {
    static int v = -1;
    if (v < 0) {
        const char* e = std::getenv("CIPC_FACTOR_CAP");
        v = e ? std::max(10, std::atoi(e)) : 1000;
    }
    return v;
}

static int pcgSolve64(Ctx& c) {
    reservePcg(c);
    computeDinv(c);
    bool learned = prepareLearned(c);
    int n3 = 3 * c.nv;
    int flag = 0;
    double rel = 0;
    // the pipelined recurrences are asked for no more than 1e-8 relative
    // (their attainable accuracy); tighter tolerances are reached by the
    // corrections below
    int it = runPcgPersistent<double, double>(c, c.valD, c.dynBD, c.rhs.p, c.sol.p, c.r.p, c.z.p, c.p.p, c.Ap.p,
                                              pcgClassic() ? c.pcgTol : std::max(c.pcgTol, 1e-8),
                                              learned ? std::min(c.pcgMaxIter, factorCap()) : c.pcgMaxIter, flag, rel, learned);
    // the true FP64 residual decides every solve; corrections restart from
    // the current iterate (residual replacement) with the textbook
    // recurrences, block-Jacobi taking over from a rejected factor
    double rhs2 = deviceDot(c, c.rhs, c.rhs, n3);
    double thr = std::max(c.pcgTol * c.pcgTol * rhs2, 2.2250738585072014e-308);
    double tr2 = trueResidual2(c);
    if (debugPcg()) std::fprintf(stderr, "[pcg] fp64 it %d flag %d true rr/b2 %.3e factor %d\n", it, flag, tr2 / rhs2, (int)learned);
    if (learned && (flag != 1 || !(tr2 < thr))) {
        c.mpFallbacks++;
        learned = false;
    }
    c.corrX.reserve(n3); c.corrR.reserve(n3);
    for (int k = 0; k < 8 && !(tr2 < thr) && it < c.pcgMaxIter; ++k) {
        int f2 = 0;
        int it2 = runPcgPersistent<double, double>(c, c.valD, c.dynBD, c.r.p, c.corrX.p, c.corrR.p, c.z.p, c.p.p, c.Ap.p,
                                                   0.5 * std::sqrt(thr / tr2), c.pcgMaxIter - it, f2, rel, learned, true);
        it += it2;
        launch(accumulateKernelD, vecBlocks(c.nv + 1), VB, 0, c.s, n3, (const double*)c.corrX.p, c.sol.p);
        tr2 = trueResidual2(c);
        if (debugPcg()) std::fprintf(stderr, "[pcg] fp64 correction it %d flag %d true rr/b2 %.3e\n", it2, f2, tr2 / rhs2);
    }
    c.lastPcgIters = it;
    c.lastPcgRelRes = rhs2 > 0 ? std::sqrt(tr2 / rhs2) : 0.0;
    c.pcgItersTotal += it;
    if (!(tr2 < thr) && rhs2 > 0) throw std::runtime_error("GPU PCG did not converge within " + std::to_string(c.pcgMaxIter) + " iterations");
    return it;
}

// r = b - A sol in FP64 (FP32 blocks promoted), bF = (float) r; returns |r|^2
static double mixedResidual(Ctx& c, float* bF) {
    int nv = c.nv, n3 = 3 * nv;
    double* part = c.red.p + 3 * MAXPART;
    spmvT<float, double>(c, c.valF, c.dynBF, c.sol.p, c.Ap.p, nullptr, nullptr, spmvBlocks(c));
    int nb = vecBlocks(nv);
    launch(residualKernel, nb, VB, 0, c.s, n3, c.rhs.p, c.Ap.p, c.r.p, bF, part);
    return deviceSum(c, part, nb);
}

// FP32 inner PCG + FP64 iterative refinement on the true residual, starting
// from the current c.sol.  Returns false when a factor preconditioner was
// rejected (inner solve over its cap, or the true residual not reached).
static bool refineMixed(Ctx& c, bool learned, double thr, double rhs2, int& total, double& rr) {
    int nv = c.nv, n3 = 3 * nv;
    float* bF = c.DinvF.p;  // FP32 copy of the current residual (right-hand side of the correction)
    int vb = vecBlocks(nv + 1);
    const double innerTol = 1e-3;
    double prevRR = 1e308;
    rr = mixedResidual(c, bF);
    // The pipelined kernel's recurrences stagnate with FP32 vectors on these
    // systems (measured), so with it the corrections run FP64 vectors over
    // the FP32 blocks below; the FP32-vector inner loop serves the classic
    // kernel.
    const int outerMax = pcgClassic() ? 40 : 0;
    for (int outer = 0; outer < outerMax && !(rr < thr); ++outer) {
        if (!(rr < 0.25 * prevRR) && outer > 2) break;  // refinement stagnates: finish in FP64 below
        prevRR = rr;
        int budget = c.pcgMaxIter - total;
        if (budget <= 0) break;
        int cap = learned ? std::min(budget, factorCap()) : budget;
        int flag = 0;
        double rel = 0;
        int it = runPcgPersistent<float, float>(c, c.valF, c.dynBF, bF, c.xF.p, c.rF.p, c.zF.p, c.pF.p, c.ApF.p,
                                                std::max(innerTol, 0.5 * std::sqrt(thr / rr)), cap, flag, rel, learned);
        total += it;
        launch(accumulateKernel, vb, VB, 0, c.s, n3, c.xF.p, c.sol.p);
        rr = mixedResidual(c, bF);
        if (debugPcg()) std::fprintf(stderr, "[pcg] mixed outer %d inner it %d flag %d rel %.3e -> rr/b2 %.3e learned %d\n", outer, it, flag, rel, rr / rhs2,
                                     (int)learned);
        if (learned && flag != 1) return false;
    }
    // FP64-vector PCG on the true residual (FP32 blocks promoted), repeated
    // as residual replacement until the true FP64 residual passes; the
    // repeats use the textbook recurrences, free of pipelining drift
    c.corrX.reserve(n3); c.corrR.reserve(n3);
    for (int k = 0; k < 8 && !(rr < thr) && total < c.pcgMaxIter; ++k) {
        int budget = c.pcgMaxIter - total;
        int flag = 0;
        double rel = 0;
        double tol = 0.5 * std::sqrt(thr / rr);
        if (k == 0 && !pcgClassic()) tol = std::max(tol, 1e-8);
        int it = runPcgPersistent<float, double>(c, c.valF, c.dynBF, c.r.p, c.corrX.p, c.corrR.p, c.z.p, c.p.p, c.Ap.p, tol,
                                                 learned ? std::min(budget, factorCap()) : budget, flag, rel, learned, k > 0);
        total += it;
        launch(accumulateKernelD, vb, VB, 0, c.s, n3, c.corrX.p, c.sol.p);
        rr = mixedResidual(c, bF);
        if (debugPcg()) std::fprintf(stderr, "[pcg] mixed FP64-vector run it %d flag %d -> rr/b2 %.3e learned %d\n", it, flag, rr / rhs2, (int)learned);
        if (learned && flag != 1) return false;
    }
    return !learned || rr < thr;
}

static int pcgSolveMixed(Ctx& c, bool learned) {
    int nv = c.nv;
    int n3 = 3 * nv;
    c.rF.reserve(n3); c.zF.reserve(n3); c.pF.reserve(n3); c.ApF.reserve(n3); c.xF.reserve(n3); c.DinvF.reserve(n3);
    launch(zeroKernel, vecBlocks(nv + 1), VB, 0, c.s, n3, c.sol.p);
    double rhs2 = deviceDot(c, c.rhs, c.rhs, n3);
    c.lastPcgIters = 0;
    if (rhs2 == 0.0) { c.lastPcgRelRes = 0; return 0; }
    double thr = std::max(c.pcgTol * c.pcgTol * rhs2, 2.2250738585072014e-308);
    int total = 0;
    double rr = rhs2;
    if (!refineMixed(c, learned, thr, rhs2, total, rr)) {
        // the factor was rejected (cap or true FP64 residual): block-Jacobi
        // continues the refinement from the current iterate
        c.mpFallbacks++;
        if (debugPcg()) std::fprintf(stderr, "[pcg] factor rejected after %d iterations (rr/b2 %.3e): block-Jacobi\n", total, rr / rhs2);
        refineMixed(c, false, thr, rhs2, total, rr);
    }
    if (!(rr < thr)) throw std::runtime_error("GPU PCG did not converge within " + std::to_string(c.pcgMaxIter) + " iterations");
    c.lastPcgIters = total;
    c.lastPcgRelRes = std::sqrt(rr / rhs2);
    c.pcgItersTotal += total;
    return total;
}

static int pcgSolveMixed(Ctx& c) {
    reservePcg(c);
    computeDinv(c);
    bool learned = prepareLearned(c);
    return pcgSolveMixed(c, learned);
}

int pcgSolve(Ctx& c) { return c.mixed ? pcgSolveMixed(c) : pcgSolve64(c); }

}  // namespace cipc

// ---------------------------------------------------------------------------
// Allocation-free stand-alone PCG.
//
// For callers that must not allocate device memory: code running where
// cudaMalloc is forbidden or unwanted, e.g. a host whose device memory is
// owned by its own allocator (a framework's caching allocator, a pre-sized
// arena) or a loop that must not pay allocation latency.  The caller passes
// device pointers for the matrix, right-hand side and solution; every scratch
// vector lives in the file-scope array below.  The array is sized for at
// most CIPC_NOALLOC_MAX_ROWS block rows (NOALLOC_DOUBLES doubles: 8,008,064
// bytes, 7.6 MiB) and every GPU that loads this library keeps it until the
// process exits.  All calls share it and it keeps the last call's contents,
// so calls that overlap on the GPU (two streams, two host threads) race;
// serialise them.
// ---------------------------------------------------------------------------
namespace {
constexpr int NOALLOC_MAX_ROWS = 32768;
constexpr int NOALLOC_PARTS = 3 * 512;
// r, z, p, Ap (3 per row each), Dinv and a zero diagonal term (9 per row
// each), partial sums, scalars, then int storage (flag words, diagonal slots).
constexpr size_t NOALLOC_VEC = 3 * (size_t)NOALLOC_MAX_ROWS;
constexpr size_t NOALLOC_DOUBLES = 4 * NOALLOC_VEC + 18 * (size_t)NOALLOC_MAX_ROWS + NOALLOC_PARTS + 16 + (NOALLOC_MAX_ROWS + 64) / 2;
static_assert(NOALLOC_DOUBLES * sizeof(double) == 8008064, "the documented scratch size");
}  // namespace

static __device__ __align__(256) double g_noallocScratch[NOALLOC_DOUBLES];

namespace {
double* g_noallocAddr[256] = {nullptr};  // device address of the scratch, per device id

// Checks the caller's block-CSR structure while locating the diagonal blocks:
// row pointers non-negative and non-decreasing, column indices in range, and
// exactly one diagonal block per row (an SPD matrix has a nonsingular
// diagonal block in every row; the block-Jacobi inverse needs it).  A failure
// sets a bit of *bad; the caller then reads no block.
__global__ void noallocDiagKernel(int nv, const int* rowPtr, const int* colIdx, int* diagSlot, double* zeroDiag, int* bad) {
    CIPC_KERNEL_LOOP(r, nv) {
        const int b = rowPtr[r], e = rowPtr[r + 1];
        int s = -1, nd = 0;
        if (b < 0 || e < b) {
            atomicOr(bad, 1);
        } else {
            for (int k = b; k < e; ++k) {
                const int cl = colIdx[k];
                if (cl < 0 || cl >= nv) { atomicOr(bad, 2); break; }
                if (cl == r) { s = k; ++nd; }
            }
            if (nd != 1) atomicOr(bad, 4);
        }
        diagSlot[r] = s;
        for (int q = 0; q < 9; ++q) zeroDiag[9 * r + q] = 0.0;
    }
}
}  // namespace

extern "C" int cipc_gpu_pcg_bsr_noalloc(int nv, const int* rowPtr, const int* colIdx, const double* vals, const double* rhs, double* sol,
                                        double relativeTolerance, int maximumIterations, void* stream, int* iterations, double* relResidual) {
    using namespace cipc;
    if (nv <= 0 || !rowPtr || !colIdx || !vals || !rhs || !sol) return CIPC_ERR_INVALID_ARGUMENT;
    if (nv > NOALLOC_MAX_ROWS) return CIPC_ERR_INVALID_ARGUMENT;
    if (!(relativeTolerance > 0) || maximumIterations <= 0) return CIPC_ERR_INVALID_ARGUMENT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 256) return CIPC_ERR_CUDA;
    if (!g_noallocAddr[dev]) {
        // first call on this device: resolve the array's device address with
        // this device current (the host symbol itself is not a device address)
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noallocScratch) != cudaSuccess || !p) return CIPC_ERR_CUDA;
        g_noallocAddr[dev] = static_cast<double*>(p);
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double* base = g_noallocAddr[dev];
    double* r = base;
    double* z = r + NOALLOC_VEC;
    double* p = z + NOALLOC_VEC;
    double* Ap = p + NOALLOC_VEC;
    double* Dinv = Ap + NOALLOC_VEC;
    double* zeroDiag = Dinv + 9 * (size_t)NOALLOC_MAX_ROWS;
    double* parts = zeroDiag + 9 * (size_t)NOALLOC_MAX_ROWS;
    double* scal = parts + NOALLOC_PARTS;
    int* ints = reinterpret_cast<int*>(scal + 16);
    int* flag = ints;
    int* bad = ints + 1;
    int* diagSlot = ints + 64;
    double* partA = parts;
    double* partB = parts + 512;
    double* partC = parts + 1024;
    int vb = vecBlocks(nv);
    int sb = std::max(1, std::min((nv * GROUP + VB - 1) / VB, MAXPART));
    // the structure check runs (and is read back) before any kernel reads a
    // block through the caller's column indices
    int hbad = 0;
    if (cudaMemsetAsync(bad, 0, sizeof(int), s) != cudaSuccess) return CIPC_ERR_CUDA;
    launch(noallocDiagKernel, vb, VB, 0, s, nv, rowPtr, colIdx, diagSlot, zeroDiag, bad);
    if (cudaGetLastError() != cudaSuccess) return CIPC_ERR_CUDA;
    if (cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CIPC_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return CIPC_ERR_CUDA;
    if (hbad) return CIPC_ERR_INVALID_ARGUMENT;
    launch(dinvKernel<double>, vb, VB, 0, s, nv, diagSlot, vals, (const int*)nullptr, (const int*)nullptr, (const int*)nullptr,
           (const double*)nullptr, zeroDiag, Dinv);
    launch(pcgInitKernel<double>, vb, VB, 0, s, nv, rhs, Dinv, sol, r, z, p, partA, partB);
    launch(pcgInitScalars, 1, VB, 0, s, partA, partB, vb, relativeTolerance, scal, flag);
    if (cudaGetLastError() != cudaSuccess) return CIPC_ERR_CUDA;
    int hflag = 0;
    double hs[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int guard = 0; guard < maximumIterations / 16 + 2; ++guard) {
        for (int k = 0; k < 16; ++k) {
            launch(spmvKernel<double, double>, sb, VB, 0, s, nv, rowPtr, colIdx, vals, (const int*)nullptr, (const int*)nullptr, (const int*)nullptr,
                   (const double*)nullptr, zeroDiag, p, Ap, partC, flag);
            launch(pcgUpdateKernel<double>, vb, VB, 0, s, nv, partC, sb, scal, Dinv, p, Ap, sol, r, z, partA, partB, flag);
            launch(pcgScalarKernel, 1, VB, 0, s, partA, partB, vb, scal, flag, maximumIterations);
            launch(pcgDirKernel<double>, vb, VB, 0, s, nv, scal, z, p, flag);
        }
        if (cudaGetLastError() != cudaSuccess) return CIPC_ERR_CUDA;
        if (cudaMemcpyAsync(&hflag, flag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CIPC_ERR_CUDA;
        if (cudaMemcpyAsync(hs, scal, 8 * sizeof(double), cudaMemcpyDeviceToHost, s) != cudaSuccess) return CIPC_ERR_CUDA;
        if (cudaStreamSynchronize(s) != cudaSuccess) return CIPC_ERR_CUDA;
        if (hflag) break;
    }
    if (iterations) *iterations = (int)hs[4];
    if (relResidual) *relResidual = hs[6] > 0 ? std::sqrt(hs[3] / hs[6]) : 0.0;
    return hflag == 1 ? CIPC_OK : CIPC_ERR_NOT_CONVERGED;
}
