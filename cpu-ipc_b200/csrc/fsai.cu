// Factorised sparse approximate inverse (FSAI) on the IC(0) block pattern:
// the exact minimiser of the Kaporin condition number of G Â G^T over lower
// block-triangular G with the pattern of the matrix's own lower blocks
// (Kolotilina and Yeremin's construction, applied to the block-Jacobi-scaled
// matrix Â = S A S^T).  It is what the learned network's loss targets, built
// here directly: for block row i with pattern P = {i} + its lower neighbours,
//     Â_PP Y = E_i        (3|P| x 3, one dense SPD solve per row)
//     Y_ii = U U^T        (U upper triangular)
//     G_{i,P} = U^-1 Y^T  (so G_ii = U^T is lower triangular and (G Â G^T)_ii = I).
// One warp owns one block row: it gathers Â_PP into shared memory (block
// lookups by binary search in the sorted static and contact rows), factors
// it (Cholesky, lanes over rows) and writes G into the same slot-aligned
// storage the learned factor uses, so the persistent PCG applies either.
// Rows with more than FS_MAXM - 1 lower neighbours keep the first ones by
// column; Dirichlet vertices keep G_ii = I and no off-diagonal block.
//
// No counterpart in CPU-IPC (its preconditioned option is Eigen's
// IncompleteCholesky, CPU IPC/NewtonLinearSystem.cpp:186-192).
#include "cipc_device.cuh"
#include "cipc_internal.h"
#include "fsai.h"

#include <algorithm>
#include <climits>

namespace cipc {

namespace {

constexpr int FS_MAXM = 16;            // blocks per pattern row (i and 15 neighbours)
constexpr int FS_N = 3 * FS_MAXM;      // dense system order
constexpr int FS_WARPS = 2;            // warps per CTA (shared memory: 2 x 18 KB)

__device__ __forceinline__ int findCol(const int* col, int lo, int hi, int c) {
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (col[mid] < c) lo = mid + 1; else hi = mid;
    }
    return lo;  // caller checks lo < end and col[lo] == c
}

template <class MT>
__device__ void rawBlock(int a, int b, const int* rowPtr, const int* col, const MT* val, const int* dRowS, const int* dRowE, const int* dCol,
                         const MT* dVal, double B[9]) {
    for (int q = 0; q < 9; ++q) B[q] = 0.0;
    int lo = rowPtr[a], hi = rowPtr[a + 1];
    int k = findCol(col, lo, hi, b);
    if (k < hi && col[k] == b)
        for (int q = 0; q < 9; ++q) B[q] += (double)val[(size_t)9 * k + q];
    if (dRowS) {
        lo = dRowS[a]; hi = dRowE[a];
        k = findCol(dCol, lo, hi, b);
        if (k < hi && dCol[k] == b)
            for (int q = 0; q < 9; ++q) B[q] += (double)dVal[(size_t)9 * k + q];
    }
}

template <class MT>
__global__ void __launch_bounds__(32 * FS_WARPS) fsaiKernel(int nv, const int* rowPtr, const int* col, const MT* val, const int* dRowS,
                                                             const int* dRowE, const int* dCol, const MT* dVal, const int* diagSlot, const int* mirS,
                                                             const int* mirD, const int* btype, const double* S, float* gS, float* gD,
                                                             int* truncated) {
    __shared__ double Ksh[FS_WARPS][FS_N * FS_N];
    __shared__ double Ysh[FS_WARPS][FS_N * 3];
    __shared__ int Psh[FS_WARPS][FS_MAXM], sSlot[FS_WARPS][FS_MAXM], dSlot[FS_WARPS][FS_MAXM];
    __shared__ int mSh[FS_WARPS], okSh[FS_WARPS];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double* K = Ksh[w];
    double* Y = Ysh[w];
    int* P = Psh[w];
    const int warpsTotal = gridDim.x * FS_WARPS;
    for (int i = blockIdx.x * FS_WARPS + w; i < nv; i += warpsTotal) {
        if (btype[i] != 0) {
            if (lane < 9) gS[(size_t)9 * diagSlot[i] + lane] = (lane % 4 == 0) ? 1.f : 0.f;
            continue;
        }
        // pattern: i, then the free lower neighbours (static and contact merged by column)
        if (lane == 0) {
            int m = 0;
            P[m] = i; sSlot[w][m] = diagSlot[i]; dSlot[w][m] = -1; ++m;
            int ks = rowPtr[i], ke = rowPtr[i + 1];
            int kd = dRowS ? dRowS[i] : 0, kde = dRowS ? dRowE[i] : 0;
            bool cut = false;
            while (true) {
                int cs = (ks < ke && col[ks] < i) ? col[ks] : INT_MAX;
                int cd = (kd < kde && dCol[kd] < i) ? dCol[kd] : INT_MAX;
                int c = min(cs, cd);
                if (c == INT_MAX) break;
                int ss = -1, ds = -1;
                if (cs == c) ss = ks++;
                if (cd == c) ds = kd++;
                if (btype[c] != 0) continue;
                if (m == FS_MAXM) { cut = true; break; }
                P[m] = c; sSlot[w][m] = ss; dSlot[w][m] = ds; ++m;
            }
            if (cut) atomicAdd(truncated, 1);
            mSh[w] = m;
            okSh[w] = 1;
        }
        __syncwarp();
        const int m = mSh[w], n = 3 * m;
        // gather Â_PP (identity diagonal blocks)
        for (int q = lane; q < m * m; q += 32) {
            int a = q / m, b = q % m;
            double O[9];
            if (a == b) {
                for (int t = 0; t < 9; ++t) O[t] = (t % 4 == 0) ? 1.0 : 0.0;
            } else {
                double B[9];
                rawBlock(P[a], P[b], rowPtr, col, val, dRowS, dRowE, dCol, dVal, B);
                const double* Sa = S + 9 * P[a];
                const double* Sb = S + 9 * P[b];
                double T[9];
                for (int r = 0; r < 3; ++r)
                    for (int s = 0; s < 3; ++s) T[3 * r + s] = Sa[3 * r] * B[s] + Sa[3 * r + 1] * B[3 + s] + Sa[3 * r + 2] * B[6 + s];
                for (int r = 0; r < 3; ++r)
                    for (int s = 0; s < 3; ++s) O[3 * r + s] = T[3 * r] * Sb[3 * s] + T[3 * r + 1] * Sb[3 * s + 1] + T[3 * r + 2] * Sb[3 * s + 2];
            }
            for (int r = 0; r < 3; ++r)
                for (int s = 0; s < 3; ++s) K[(3 * a + r) * FS_N + 3 * b + s] = O[3 * r + s];
        }
        __syncwarp();
        // Cholesky K = L L^T in place (lower triangle)
        for (int k = 0; k < n; ++k) {
            if (lane == 0) {
                double d = K[k * FS_N + k];
                if (!(d > 0.0)) { okSh[w] = 0; d = 1.0; }
                K[k * FS_N + k] = sqrt(d);
            }
            __syncwarp();
            double lkk = K[k * FS_N + k];
            for (int r = k + 1 + lane; r < n; r += 32) K[r * FS_N + k] /= lkk;
            __syncwarp();
            for (int r = k + 1 + lane; r < n; r += 32) {
                double lrk = K[r * FS_N + k];
                for (int c2 = k + 1; c2 <= r; ++c2) K[r * FS_N + c2] -= lrk * K[c2 * FS_N + k];
            }
            __syncwarp();
        }
        // Y = K^-1 E_0: lanes 0..2 solve one right-hand side each
        if (lane < 3) {
            for (int r = 0; r < n; ++r) {
                double s = (r == lane) ? 1.0 : 0.0;
                for (int c2 = 0; c2 < r; ++c2) s -= K[r * FS_N + c2] * Y[c2 * 3 + lane];
                Y[r * 3 + lane] = s / K[r * FS_N + r];
            }
            for (int r = n - 1; r >= 0; --r) {
                double s = Y[r * 3 + lane];
                for (int c2 = r + 1; c2 < n; ++c2) s -= K[c2 * FS_N + r] * Y[c2 * 3 + lane];
                Y[r * 3 + lane] = s / K[r * FS_N + r];
            }
        }
        __syncwarp();
        // U upper with Y_ii = U U^T, then G_{i,t} = U^-1 Y_t^T
        double Ui[9];
        bool ok = okSh[w] != 0;
        {
            double y00 = Y[0], y01 = 0.5 * (Y[1] + Y[3]), y02 = 0.5 * (Y[2] + Y[6]);
            double y11 = Y[4], y12 = 0.5 * (Y[5] + Y[7]), y22 = Y[8];
            double u22 = y22 > 0 ? sqrt(y22) : 0.0;
            double u12 = u22 > 0 ? y12 / u22 : 0.0, u02 = u22 > 0 ? y02 / u22 : 0.0;
            double t11 = y11 - u12 * u12;
            double u11 = t11 > 0 ? sqrt(t11) : 0.0;
            double u01 = u11 > 0 ? (y01 - u02 * u12) / u11 : 0.0;
            double t00 = y00 - u01 * u01 - u02 * u02;
            double u00 = t00 > 0 ? sqrt(t00) : 0.0;
            ok = ok && u00 > 0 && u11 > 0 && u22 > 0 && isfinite(u00 + u01 + u02 + u11 + u12 + u22);
            if (ok) {
                // inverse of the upper-triangular U
                Ui[0] = 1 / u00; Ui[4] = 1 / u11; Ui[8] = 1 / u22;
                Ui[1] = -u01 / (u00 * u11);
                Ui[5] = -u12 / (u11 * u22);
                Ui[2] = (u01 * u12 - u02 * u11) / (u00 * u11 * u22);
                Ui[3] = Ui[6] = Ui[7] = 0.0;
            }
        }
        for (int t = lane; t < m; t += 32) {
            float G[9];
            if (!ok) {
                // this row falls back to block-Jacobi
                for (int q = 0; q < 9; ++q) G[q] = (t == 0 && q % 4 == 0) ? 1.f : 0.f;
            } else {
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) {
                        double s = 0;
                        for (int c2 = 0; c2 < 3; ++c2) s += Ui[3 * a + c2] * Y[(3 * t + b) * 3 + c2];
                        G[3 * a + b] = (float)s;
                    }
                if (t == 0) { G[1] = G[2] = G[5] = 0.f; }
            }
            if (t == 0) {
                for (int q = 0; q < 9; ++q) gS[(size_t)9 * diagSlot[i] + q] = G[q];
                continue;
            }
            int ss = sSlot[w][t], ds = dSlot[w][t];
            float* dst = ss >= 0 ? gS + (size_t)9 * ss : gD + (size_t)9 * ds;
            int mir = ss >= 0 ? mirS[ss] : mirD[ds];
            float* dstT = mir >= 0 ? (ss >= 0 ? gS : gD) + (size_t)9 * mir : nullptr;
            for (int q = 0; q < 9; ++q) dst[q] = G[q];
            if (dstT)
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) dstT[3 * a + b] = G[3 * b + a];
        }
        __syncwarp();
    }
}

__global__ void zeroFactorKernel(size_t n, float* a) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)blockDim.x * gridDim.x) a[i] = 0.f;
}

}  // namespace

template <class MT>
static void buildT(Ctx& c, const MT* val, const MT* dval) {
    int nv = c.nv;
    bool dyn = c.nDynB > 0;
    size_t es = (size_t)std::max(c.nnzb, 1), ed = (size_t)std::max(c.nDynB, 1);
    c.mpGS.reserve(9 * es);
    c.mpGD.reserve(9 * ed);
    launch(zeroFactorKernel, 1024, 256, 0, c.s, 9 * es, c.mpGS.p);
    launch(zeroFactorKernel, 1024, 256, 0, c.s, 9 * ed, c.mpGD.p);
    c.counters.reserve(16);
    CIPC_CUDA(cudaMemsetAsync(c.counters.p + 13, 0, sizeof(int), c.s));
    int grid = std::max(1, std::min((nv + FS_WARPS - 1) / FS_WARPS, 148 * 16));
    launch(fsaiKernel<MT>, grid, 32 * FS_WARPS, 0, c.s, nv, (const int*)c.rowPtr.p, (const int*)c.colIdx.p, val, dyn ? (const int*)c.dynRowStart.p : nullptr,
           dyn ? (const int*)c.dynRowEnd.p : nullptr, dyn ? (const int*)c.dynCol.p : nullptr, dval, (const int*)c.diagSlot.p, (const int*)c.mpMirS.p,
           (const int*)c.mpMirD.p, (const int*)c.btype.p, (const double*)c.mpS.p, c.mpGS.p, c.mpGD.p, c.counters.p + 13);
    CIPC_CUDA(cudaGetLastError());
    c.mpFactorReady = true;
}

void fsaiBuild(Ctx& c) {
    if (c.mixed) buildT<float>(c, c.valF.p, c.dynBF.p);
    else buildT<double>(c, c.valD.p, c.dynBD.p);
}

}  // namespace cipc
