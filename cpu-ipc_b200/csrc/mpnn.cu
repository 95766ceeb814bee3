// Learned preconditioner: a message-passing network over the Newton
// matrix's 3x3-block graph that emits a lower block-triangular factor G on
// the IC(0) pattern (the lower block pattern of the matrix itself) of the
// block-Jacobi-scaled matrix
//     Â = S A S^T,  S_i = L_i^-1,  D_i = L_i L_i^T (assembled diagonal block),
// used as a factorised sparse approximate inverse
//     M^-1 = S^T G^T G S        (G = I gives block-Jacobi exactly),
// so applying it is two sparse products over the existing block pattern.
// G is lower triangular with a positive diagonal (softplus), so M^-1 is SPD
// for any weights.
//
// Training minimises the Kaporin condition number of B = G Â G^T,
//     L = log(tr(B)/n) - (2/n) sum_q log G_qq,
// with tr(B)/n estimated from probe vectors w as mean w^T B w / w^T w; the
// minimiser of L over the pattern is the factorised sparse approximate
// inverse of that pattern.  Forward and backward kernels are hand-written;
// the weights are used in BF16 with FP32 accumulation, FP32 masters are
// updated by Adam.
//
// Graph: nodes are vertices; edges are the lower off-diagonal block slots
// (col < row) of the static BSR and of the contact BSR.  Each edge keeps its
// factor block in its own slot and the transpose in the mirror slot (row and
// column swapped), so G x and G^T x are both row-wise products.
//
// No counterpart in CPU-IPC; the closest is the Eigen IncompleteCholesky
// option of NewtonLinearSystem::solve (CPU IPC/NewtonLinearSystem.cpp:186-192).
#include "cipc_device.cuh"
#include "cipc_internal.h"
#include "mpnn.h"
#include "dense_tc.cuh"

#include <cuda_bf16.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

namespace cipc {

namespace {

constexpr int TB = 128;
inline int blocksFor(int n, int tb = TB) { return std::max(1, std::min((n + tb - 1) / tb, 148 * 32)); }

typedef __nv_bfloat16 bf16;
__device__ __forceinline__ float W(const bf16* w, int i) { return __bfloat162float(w[i]); }
__device__ __forceinline__ float relu(float x) { return x > 0.f ? x : 0.f; }
__device__ __forceinline__ float softplus(float x) { return x > 20.f ? x : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoidf(float x) { return 1.f / (1.f + expf(-x)); }

// ---------------------------------------------------------------------------
// scaling and features
// ---------------------------------------------------------------------------
template <class MT>
__device__ void diagBlock(int v, const int* diagSlot, const MT* val, const int* dRowS, const int* dRowE, const int* dCol, const MT* dVal,
                          const double* diagExtra, double D[9], double C[9]) {
    for (int k = 0; k < 9; ++k) { D[k] = diagExtra[9 * v + k]; C[k] = 0.0; }
    int s = diagSlot[v];
    if (s >= 0) for (int k = 0; k < 9; ++k) D[k] += (double)val[(size_t)9 * s + k];
    if (dRowS)
        for (int k = dRowS[v]; k < dRowE[v]; ++k)
            if (dCol[k] == v)
                for (int q = 0; q < 9; ++q) { D[q] += (double)dVal[(size_t)9 * k + q]; C[q] += (double)dVal[(size_t)9 * k + q]; }
}

// S = L^-1 of the Cholesky factor of D (lower entries used); diagonal
// scaling if D is not positive definite.
__device__ void invChol(const double D[9], double S[9]) {
    for (int k = 0; k < 9; ++k) S[k] = 0.0;
    double a00 = D[0], a10 = D[3], a11 = D[4], a20 = D[6], a21 = D[7], a22 = D[8];
    bool ok = a00 > 0;
    double l00 = 0, l10 = 0, l20 = 0, l11 = 0, l21 = 0, l22 = 0;
    if (ok) { l00 = sqrt(a00); l10 = a10 / l00; l20 = a20 / l00; double t = a11 - l10 * l10; ok = t > 0; if (ok) l11 = sqrt(t); }
    if (ok) { l21 = (a21 - l20 * l10) / l11; double t = a22 - l20 * l20 - l21 * l21; ok = t > 0; if (ok) l22 = sqrt(t); }
    if (ok && isfinite(l22)) {
        S[0] = 1 / l00; S[4] = 1 / l11; S[8] = 1 / l22;
        S[3] = -l10 / (l00 * l11);
        S[7] = -l21 / (l11 * l22);
        S[6] = (l10 * l21 - l11 * l20) / (l00 * l11 * l22);
    } else {
        for (int q = 0; q < 3; ++q) S[4 * q] = D[4 * q] > 0 ? 1.0 / sqrt(D[4 * q]) : 1.0;
    }
}

// out = S_i B S_j^T (B row-major 3x3, S lower-triangular row-major)
template <class MT>
__device__ __forceinline__ void scaleBlock(const double* Si, const MT* B, const double* Sj, double out[9]) {
    double T[9];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) T[3 * a + b] = Si[3 * a] * (double)B[b] + Si[3 * a + 1] * (double)B[3 + b] + Si[3 * a + 2] * (double)B[6 + b];
    for (int a = 0; a < 3; ++a)
        for (int d = 0; d < 3; ++d) out[3 * a + d] = T[3 * a] * Sj[3 * d] + T[3 * a + 1] * Sj[3 * d + 1] + T[3 * a + 2] * Sj[3 * d + 2];
}

template <class MT>
__global__ void scaleKernel(int nv, const int* diagSlot, const MT* val, const int* dRowS, const int* dRowE, const int* dCol, const MT* dVal,
                            const double* diagExtra, double* S, float* f5) {
    CIPC_KERNEL_LOOP(v, nv) {
        double D[9], C[9], Sv[9];
        diagBlock(v, diagSlot, val, dRowS, dRowE, dCol, dVal, diagExtra, D, C);
        invChol(D, Sv);
        for (int k = 0; k < 9; ++k) S[9 * v + k] = Sv[k];
        double sc[9];
        scaleBlock(Sv, C, Sv, sc);
        f5[v] = (float)((sc[0] + sc[4] + sc[8]) / 3.0);
    }
}

// per row: sums / max / counts of |Â_vc|_F over off-diagonal slots
template <class MT>
__global__ void nodeFeatKernel(int nv, const int* rowPtr, const int* col, const MT* val, const int* dRowS, const int* dRowE, const int* dCol,
                               const MT* dVal, const double* S, const float* f5, float* f) {
    CIPC_KERNEL_LOOP(v, nv) {
        double sumS = 0, sumD = 0, mx = 0;
        int degS = 0, degD = 0;
        for (int k = rowPtr[v]; k < rowPtr[v + 1]; ++k) {
            int c = col[k];
            if (c == v) continue;
            double b[9];
            scaleBlock(S + 9 * v, val + (size_t)9 * k, S + 9 * c, b);
            double n = 0;
            for (int q = 0; q < 9; ++q) n += b[q] * b[q];
            n = sqrt(n);
            sumS += n; mx = fmax(mx, n); ++degS;
        }
        if (dRowS)
            for (int k = dRowS[v]; k < dRowE[v]; ++k) {
                int c = dCol[k];
                if (c == v) continue;
                double b[9];
                scaleBlock(S + 9 * v, dVal + (size_t)9 * k, S + 9 * c, b);
                double n = 0;
                for (int q = 0; q < 9; ++q) n += b[q] * b[q];
                n = sqrt(n);
                sumD += n; mx = fmax(mx, n); ++degD;
            }
        float* o = f + MPNN_NF * v;
        o[0] = (float)sumS; o[1] = (float)sumD; o[2] = (float)mx;
        o[3] = log1pf((float)degS); o[4] = log1pf((float)degD); o[5] = f5[v];
    }
}

// edge features Â_ij (9, row-major) for lower slots of a row-ranged pattern
template <class MT>
__global__ void edgeFeatKernel(int nv, const int* rowS, const int* rowE, const int* col, const MT* val, const double* S, float* g) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) {
            int c = col[k];
            if (c >= v) continue;
            double b[9];
            scaleBlock(S + 9 * v, val + (size_t)9 * k, S + 9 * c, b);
            for (int q = 0; q < 9; ++q) g[(size_t)9 * k + q] = (float)b[q];
        }
    }
}

// mirror slot of (row, col) = slot of (col, row) in a column-sorted pattern
__global__ void mirrorKernel(int nv, const int* rowS, const int* rowE, const int* col, int* mirror) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) {
            int c = col[k];
            int lo = rowS[c], hi = rowE[c];
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (col[mid] < v) lo = mid + 1; else hi = mid;
            }
            mirror[k] = (lo < rowE[c] && col[lo] == v) ? lo : -1;
        }
    }
}
__global__ void rowRangeKernel(int nv, const int* rowPtr, int* rs, int* re) {
    CIPC_KERNEL_LOOP(v, nv) { rs[v] = rowPtr[v]; re[v] = rowPtr[v + 1]; }
}

__global__ void degreeKernel(int nv, const int* rowPtr, const int* col, const int* mirS, const int* dRowS, const int* dRowE, const int* dCol,
                             const int* mirD, int* deg) {
    CIPC_KERNEL_LOOP(v, nv) {
        int d = 0;
        for (int k = rowPtr[v]; k < rowPtr[v + 1]; ++k) {
            int c = col[k];
            if (c != v && (c < v || mirS[k] >= 0)) ++d;
        }
        if (dRowS)
            for (int k = dRowS[v]; k < dRowE[v]; ++k) {
                int c = dCol[k];
                if (c != v && (c < v || mirD[k] >= 0)) ++d;
            }
        deg[v] = d;
    }
}

// mean of incident edge states; an edge is read at its lower slot
// Mean of the incident edges' features, one warp per vertex: lane t sums
// feature t over the row's static slots, then its contact slots, in slot
// order (one coalesced 128-byte row per edge).  Each lane first resolves one
// slot of the row (its lower-slot index, or -1 for the diagonal and for
// blocks without an edge), and the warp walks them with shuffles.
__device__ __forceinline__ float aggregateRange(float a, int v, int k0, int k1, const int* col, const int* mir, const float* e, int lane) {
    for (int c0 = k0; c0 < k1; c0 += 32) {
        const int k = c0 + lane;
        int slot = -1;
        if (k < k1) {
            const int c = col[k];
            slot = c == v ? -1 : (c < v ? k : mir[k]);
        }
        const int m = min(32, k1 - c0);
        for (int j = 0; j < m; ++j) {
            const int sj = __shfl_sync(0xffffffffu, slot, j);
            if (sj >= 0) a += e[(size_t)MPNN_H * sj + lane];
        }
    }
    return a;
}

__global__ void aggregateKernel(int nv, const int* rowPtr, const int* col, const int* mirS, const float* eS, const int* dRowS, const int* dRowE,
                                const int* dCol, const int* mirD, const float* eD, const int* deg, float* agg) {
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * blockDim.x / 32;
    for (int v = (blockIdx.x * blockDim.x + threadIdx.x) / 32; v < nv; v += warps) {
        float a = aggregateRange(0.f, v, rowPtr[v], rowPtr[v + 1], col, mirS, eS, lane);
        if (dRowS) a = aggregateRange(a, v, dRowS[v], dRowE[v], dCol, mirD, eD, lane);
        const float inv = deg[v] > 0 ? 1.f / deg[v] : 0.f;
        agg[(size_t)MPNN_H * v + lane] = a * inv;
    }
}

// ---------------------------------------------------------------------------
// Tiled dense layers of the forward pass.  A CTA stages one weight matrix
// (transposed, FP32 from the BF16 copy) and a tile of DT_ITEMS input rows in
// shared memory; two threads per item split the outputs and accumulate in
// FP32 registers.  Items are nodes or the lower edges of a flat edge list;
// gather and emit functors read the layer's inputs and write its outputs.
// ---------------------------------------------------------------------------
constexpr int DT_ITEMS = 64;
constexpr int DT_THREADS = 2 * DT_ITEMS;

template <int IN, int OUT, class G, class E>
__global__ void __launch_bounds__(DT_THREADS) denseTiledKernel(int n, G gather, E emit, const bf16* Wm, const bf16* bias) {
    constexpr int HALF = (OUT + 1) / 2;
    __shared__ float sW[IN][OUT + 1];
    __shared__ float sB[OUT];
    __shared__ float sX[DT_ITEMS][IN + 1];
    for (int t = threadIdx.x; t < IN * OUT; t += DT_THREADS) sW[t % IN][t / IN] = W(Wm, t);
    for (int t = threadIdx.x; t < OUT; t += DT_THREADS) sB[t] = W(bias, t);
    for (int base = blockIdx.x * DT_ITEMS; base < n; base += gridDim.x * DT_ITEMS) {
        __syncthreads();
        for (int t = threadIdx.x; t < DT_ITEMS * IN; t += DT_THREADS) {
            int r = t / IN, i = t % IN, item = base + r;
            sX[r][i] = item < n ? gather(item, i) : 0.f;
        }
        __syncthreads();
        const int r = threadIdx.x >> 1, h = threadIdx.x & 1, item = base + r;
        float acc[HALF];
#pragma unroll
        for (int q = 0; q < HALF; ++q) {
            int o = h * HALF + q;
            acc[q] = o < OUT ? sB[o] : 0.f;
        }
        for (int i = 0; i < IN; ++i) {
            float x = sX[r][i];
#pragma unroll
            for (int q = 0; q < HALF; ++q) {
                int o = h * HALF + q;
                if (o < OUT) acc[q] += sW[i][o] * x;
            }
        }
        if (item < n) {
#pragma unroll
            for (int q = 0; q < HALF; ++q) {
                int o = h * HALF + q;
                if (o < OUT) emit(item, o, acc[q]);
            }
        }
    }
}

// flat list of the lower edges of a row-ranged pattern
__global__ void lowerCountKernel(int nv, const int* rowS, const int* rowE, const int* col, int* cnt) {
    CIPC_KERNEL_LOOP(v, nv) {
        int k = 0;
        for (int s = rowS[v]; s < rowE[v]; ++s) k += col[s] < v;
        cnt[v] = k;
    }
}
__global__ void lowerFillKernel(int nv, const int* rowS, const int* rowE, const int* col, const int* off, int* eSlot, int* eI, int* eJ) {
    CIPC_KERNEL_LOOP(v, nv) {
        int o = off[v];
        for (int s = rowS[v]; s < rowE[v]; ++s)
            if (col[s] < v) { eSlot[o] = s; eI[o] = v; eJ[o] = col[s]; ++o; }
    }
}

struct NodeFeatGather {
    const float* f;
    __device__ float operator()(int v, int i) const { return f[MPNN_NF * v + i]; }
};
struct EdgeFeatGather {
    const int* slot;
    const float* g;
    __device__ float operator()(int e, int i) const { return g[(size_t)9 * slot[e] + i]; }
};
struct EdgeLayerGather {  // [e_l ; h_i + h_j]
    const int *slot, *ei, *ej;
    const float *e, *h;
    // tensor-core layer: an edge's slot and end vertices, and its inputs
    // lane and MPNN_H + lane
    struct Idx {
        int s, i, j;
    };
    __device__ Idx index(int k) const { return Idx{slot[k], ei[k], ej[k]}; }
    __device__ static Idx shfl(const Idx& x, int src) {
        return Idx{__shfl_sync(0xffffffffu, x.s, src), __shfl_sync(0xffffffffu, x.i, src), __shfl_sync(0xffffffffu, x.j, src)};
    }
    __device__ float2 pair(const Idx& x, int lane) const {
        return make_float2(e[(size_t)MPNN_H * x.s + lane], h[(size_t)MPNN_H * x.i + lane] + h[(size_t)MPNN_H * x.j + lane]);
    }
};
struct NodeLayerGather {  // [h ; agg]
    const float *h, *agg;
    struct Idx {
        int v;
    };
    __device__ Idx index(int v) const { return Idx{v}; }
    __device__ static Idx shfl(const Idx& x, int src) { return Idx{__shfl_sync(0xffffffffu, x.v, src)}; }
    __device__ float2 pair(const Idx& x, int lane) const {
        return make_float2(h[(size_t)MPNN_H * x.v + lane], agg[(size_t)MPNN_H * x.v + lane]);
    }
};
struct HeadEdgeGather {  // [e_L ; g]
    const int* slot;
    const float *e, *g;
    __device__ float operator()(int k, int i) const {
        return i < MPNN_H ? e[(size_t)MPNN_H * slot[k] + i] : g[(size_t)9 * slot[k] + i - MPNN_H];
    }
};
struct NodeHiddenGather {
    const float* h;
    __device__ float operator()(int v, int i) const { return h[(size_t)MPNN_H * v + i]; }
};

__device__ __forceinline__ void reluStore32(float* dst, const float v[32]) {
    float4* p = reinterpret_cast<float4*>(dst);
#pragma unroll
    for (int o = 0; o < 8; ++o) p[o] = make_float4(relu(v[4 * o]), relu(v[4 * o + 1]), relu(v[4 * o + 2]), relu(v[4 * o + 3]));
}
struct ReluEmitNode {
    float* out;
    __device__ void operator()(int v, int o, float a) const { out[(size_t)MPNN_H * v + o] = relu(a); }
    __device__ void emit32(int v, const float a[32]) const { reluStore32(out + (size_t)MPNN_H * v, a); }
};
struct ReluEmitEdge {
    const int* slot;
    float* out;
    __device__ void operator()(int k, int o, float a) const { out[(size_t)MPNN_H * slot[k] + o] = relu(a); }
    __device__ void emit32(int k, const float a[32]) const { reluStore32(out + (size_t)MPNN_H * slot[k], a); }
};
// G_ij into the lower slot and G_ij^T into its mirror; no block touches a
// Dirichlet vertex
struct HeadEdgeEmit {
    const int *slot, *ei, *ej, *mirror, *btype;
    float* gOut;
    __device__ void operator()(int k, int o, float a) const {
        const int s = slot[k];
        const float v = (btype[ei[k]] == 0 && btype[ej[k]] == 0) ? a : 0.f;
        gOut[(size_t)9 * s + o] = v;
        const int m = mirror[s];
        if (m >= 0) gOut[(size_t)9 * m + 3 * (o % 3) + o / 3] = v;
    }
};
// G_ii: lower triangle, softplus diagonal; Dirichlet vertices keep I
struct HeadDiagEmit {
    const int *diagSlot, *btype;
    float *gS, *headD;
    __device__ void operator()(int v, int o, float a) const {
        headD[6 * v + o] = a;
        float* G = gS + (size_t)9 * diagSlot[v];
        const bool fixedV = btype[v] != 0;
        const int pos[6] = {0, 4, 8, 3, 6, 7};
        float val = o < 3 ? softplus(a) : a;
        if (fixedV) val = o < 3 ? 1.f : 0.f;
        G[pos[o]] = val;
        if (o == 0) { G[1] = 0.f; G[2] = 0.f; G[5] = 0.f; }
    }
};

// ---------------------------------------------------------------------------
// factor and scaled operator products (FP32 vectors, one thread per row)
// ---------------------------------------------------------------------------
// y = G u (transpose = 0: lower slots + diagonal) or y = G^T u (mirror slots + transposed diagonal)
__global__ void factorApplyKernel(int nv, int transpose, const int* rowPtr, const int* col, const float* gS, const int* dRowS, const int* dRowE,
                                  const int* dCol, const float* gD, const float* u, float* y) {
    CIPC_KERNEL_LOOP(v, nv) {
        float acc[3] = {0.f, 0.f, 0.f};
        for (int k = rowPtr[v]; k < rowPtr[v + 1]; ++k) {
            int c = col[k];
            if (transpose ? c < v : c > v) continue;
            const float* B = gS + (size_t)9 * k;
            float x0 = u[3 * c], x1 = u[3 * c + 1], x2 = u[3 * c + 2];
            if (transpose && c == v)
                for (int a = 0; a < 3; ++a) acc[a] += B[a] * x0 + B[3 + a] * x1 + B[6 + a] * x2;
            else
                for (int a = 0; a < 3; ++a) acc[a] += B[3 * a] * x0 + B[3 * a + 1] * x1 + B[3 * a + 2] * x2;
        }
        if (dRowS)
            for (int k = dRowS[v]; k < dRowE[v]; ++k) {
                int c = dCol[k];
                if (transpose ? c <= v : c >= v) continue;
                const float* B = gD + (size_t)9 * k;
                float x0 = u[3 * c], x1 = u[3 * c + 1], x2 = u[3 * c + 2];
                for (int a = 0; a < 3; ++a) acc[a] += B[3 * a] * x0 + B[3 * a + 1] * x1 + B[3 * a + 2] * x2;
            }
        for (int a = 0; a < 3; ++a) y[3 * v + a] = acc[a];
    }
}

// y = Â u = S A S^T u
template <class MT>
__global__ void scaledSpmvKernel(int nv, const int* rowPtr, const int* col, const MT* val, const int* dRowS, const int* dRowE, const int* dCol,
                                 const MT* dVal, const double* diagExtra, const double* S, const float* u, float* y) {
    CIPC_KERNEL_LOOP(v, nv) {
        double acc[3] = {0, 0, 0};
        auto stu = [&](int c, double x[3]) {
            // S_c^T u_c (S_c lower triangular)
            const double* Sc = S + 9 * c;
            double u0 = u[3 * c], u1 = u[3 * c + 1], u2 = u[3 * c + 2];
            x[0] = Sc[0] * u0 + Sc[3] * u1 + Sc[6] * u2;
            x[1] = Sc[4] * u1 + Sc[7] * u2;
            x[2] = Sc[8] * u2;
        };
        for (int k = rowPtr[v]; k < rowPtr[v + 1]; ++k) {
            double x[3];
            stu(col[k], x);
            const MT* B = val + (size_t)9 * k;
            for (int a = 0; a < 3; ++a) acc[a] += (double)B[3 * a] * x[0] + (double)B[3 * a + 1] * x[1] + (double)B[3 * a + 2] * x[2];
        }
        if (dRowS)
            for (int k = dRowS[v]; k < dRowE[v]; ++k) {
                double x[3];
                stu(dCol[k], x);
                const MT* B = dVal + (size_t)9 * k;
                for (int a = 0; a < 3; ++a) acc[a] += (double)B[3 * a] * x[0] + (double)B[3 * a + 1] * x[1] + (double)B[3 * a + 2] * x[2];
            }
        {
            double x[3];
            stu(v, x);
            const double* B = diagExtra + 9 * v;
            for (int a = 0; a < 3; ++a) acc[a] += B[3 * a] * x[0] + B[3 * a + 1] * x[1] + B[3 * a + 2] * x[2];
        }
        const double* Sv = S + 9 * v;
        y[3 * v] = (float)(Sv[0] * acc[0]);
        y[3 * v + 1] = (float)(Sv[3] * acc[0] + Sv[4] * acc[1]);
        y[3 * v + 2] = (float)(Sv[6] * acc[0] + Sv[7] * acc[1] + Sv[8] * acc[2]);
    }
}

// probe vectors: four summed uniforms from a splitmix64 stream, unit variance
__global__ void probeKernel(int n, unsigned long long seed, float* w) {
    CIPC_KERNEL_LOOP(i, n) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ull * (unsigned long long)(i + 1);
        float s = 0.f;
        for (int k = 0; k < 4; ++k) {
            z ^= z >> 30; z *= 0xBF58476D1CE4E5B9ull; z ^= z >> 27; z *= 0x94D049BB133111EBull; z ^= z >> 31;
            s += (float)(z >> 40) * (1.0f / 16777216.0f) - 0.5f;
        }
        w[i] = s * 1.7320508f;
    }
}

// partials of u.v and w.w
__global__ void probeDotsKernel(int n, const float* u, const float* v, const float* w, double* part) {
    double uv = 0, ww = 0;
    CIPC_KERNEL_LOOP(i, n) {
        uv += (double)u[i] * (double)v[i];
        ww += (double)w[i] * (double)w[i];
    }
    double a = blockReduce(uv, AddOp(), 0.0);
    __syncthreads();
    double b = blockReduce(ww, AddOp(), 0.0);
    if (threadIdx.x == 0) { part[2 * blockIdx.x] = a; part[2 * blockIdx.x + 1] = b; }
}

// partial sums of log G_qq over the diagonal blocks
__global__ void logDiagKernel(int nv, const int* diagSlot, const float* gS, double* part) {
    double s = 0;
    CIPC_KERNEL_LOOP(v, nv) {
        const float* G = gS + (size_t)9 * diagSlot[v];
        s += log((double)G[0]) + log((double)G[4]) + log((double)G[8]);
    }
    double a = blockReduce(s, AddOp(), 0.0);
    if (threadIdx.x == 0) part[blockIdx.x] = a;
}

// dG_ij += scale * w_i v_j^T for lower slots and the lower triangle of the
// diagonal slot (static: dyn = 0); contact slots: lower only
__global__ void factorGradKernel(int nv, const int* rowS, const int* rowE, const int* col, int dyn, const int* btype, const float* w, const float* vv,
                                 float scale, float* dG) {
    CIPC_KERNEL_LOOP(i, nv) {
        if (btype[i] != 0) continue;
        for (int k = rowS[i]; k < rowE[i]; ++k) {
            int j = col[k];
            if (j > i || (dyn && j == i) || btype[j] != 0) continue;
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) {
                    if (j == i && b > a) continue;
                    dG[(size_t)9 * k + 3 * a + b] += scale * w[3 * i + a] * vv[3 * j + b];
                }
        }
    }
}

// dG /= T on the slots; on static diagonal slots also subtract (2/n) / G_qq
__global__ void gradScaleKernel(size_t n, float invT, float* dG) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)blockDim.x * gridDim.x) dG[i] *= invT;
}
__global__ void gradDiagKernel(int nv, const int* diagSlot, const int* btype, const float* gS, float coef, float* dG) {
    CIPC_KERNEL_LOOP(v, nv) {
        if (btype[v] != 0) continue;
        size_t s = (size_t)9 * diagSlot[v];
        for (int q = 0; q < 3; ++q) dG[s + 4 * q] -= coef / gS[s + 4 * q];
    }
}

// ---------------------------------------------------------------------------
// backward
//
// Each layer's backward runs in two parts.  An item kernel (one thread per
// node, or per row over its lower slots) forms the pre-activation gradient
// d (written to D[item][OUT], zero for masked items) and propagates W^T d to
// the layer's inputs.  The weight gradient dW = D^T X and db = sum D is then
// a split-K reduction over the items: each CTA stages TI items of D and X in
// shared memory and accumulates its share of the OUT x IN outputs in
// registers, writes one partial per output, and a second kernel sums the
// partials in CTA order - deterministic and free of atomics.
// ---------------------------------------------------------------------------
constexpr int WG_TI = 32;        // items per shared-memory tile
constexpr int WG_THREADS = 256;
constexpr int WG_GRID = 296;     // CTAs of the split-K reduction (2 per SM)

// X = [X1 (ld1, IN1 columns) ; X2 (ld2, IN2 columns)] per item; mask may be
// null (all items active).  partial[cta][OUT*(IN1+IN2) + OUT].  The heads
// and the embeddings (the tensor-core layers use weightGradTcKernel).
template <int OUT, int IN1, int IN2>
__global__ void __launch_bounds__(WG_THREADS) weightGradKernel(int items, const float* D, const float* X1, const float* X2, const unsigned char* mask,
                                                               float* partial) {
    constexpr int IN = IN1 + IN2;
    constexpr int NW = OUT * IN + OUT;
    constexpr int PER = (NW + WG_THREADS - 1) / WG_THREADS;
    __shared__ float sD[WG_TI][OUT];
    __shared__ float sX[WG_TI][IN + 1];
    float acc[PER];
    for (int q = 0; q < PER; ++q) acc[q] = 0.f;
    for (int base = blockIdx.x * WG_TI; base < items; base += gridDim.x * WG_TI) {
        __syncthreads();
        for (int t = threadIdx.x; t < WG_TI * OUT; t += WG_THREADS) {
            int it = base + t / OUT, o = t % OUT;
            bool on = it < items && (!mask || mask[it]);
            sD[t / OUT][o] = on ? D[(size_t)it * OUT + o] : 0.f;
        }
        for (int t = threadIdx.x; t < WG_TI * IN; t += WG_THREADS) {
            int r = t / IN, i = t % IN, it = base + r;
            bool on = it < items && (!mask || mask[it]);
            float v = 0.f;
            if (on) v = i < IN1 ? X1[(size_t)it * IN1 + i] : X2[(size_t)it * IN2 + (i - IN1)];
            sX[r][i] = v;
        }
        __syncthreads();
        for (int q = 0; q < PER; ++q) {
            int idx = threadIdx.x + q * WG_THREADS;
            if (idx >= NW) break;
            float s = 0.f;
            if (idx < OUT * IN) {
                int o = idx / IN, i = idx % IN;
#pragma unroll 8
                for (int r = 0; r < WG_TI; ++r) s += sD[r][o] * sX[r][i];
            } else {
                int o = idx - OUT * IN;
#pragma unroll 8
                for (int r = 0; r < WG_TI; ++r) s += sD[r][o];
            }
            acc[q] += s;
        }
    }
    for (int q = 0; q < PER; ++q) {
        int idx = threadIdx.x + q * WG_THREADS;
        if (idx < NW) partial[(size_t)blockIdx.x * NW + idx] = acc[q];
    }
}

// gW[w] += sum over CTAs of partial (weights at wOff, biases at bOff)
__global__ void weightGradReduceKernel(int nw, int out, int ctas, const float* partial, float* gW, float* gB) {
    CIPC_KERNEL_LOOP(idx, nw) {
        float s = 0.f;
        for (int g = 0; g < ctas; ++g) s += partial[(size_t)g * nw + idx];
        if (idx < nw - out) gW[idx] += s;
        else gB[idx - (nw - out)] += s;
    }
}

__global__ void headDiagBackKernel(int nv, const float* headD, const int* diagSlot, const float* dGS, const bf16* w, float* D6, float* dhL) {
    CIPC_KERNEL_LOOP(v, nv) {
        const float* dB = dGS + (size_t)9 * diagSlot[v];
        const float* o = headD + 6 * v;
        float d[6] = {dB[0] * sigmoidf(o[0]), dB[4] * sigmoidf(o[1]), dB[8] * sigmoidf(o[2]), dB[3], dB[6], dB[7]};
        float dh[MPNN_H];
        for (int t = 0; t < MPNN_H; ++t) dh[t] = 0.f;
        for (int q = 0; q < 6; ++q) {
            D6[6 * v + q] = d[q];
            for (int t = 0; t < MPNN_H; ++t) dh[t] += d[q] * W(w + MP_WD, q * MPNN_H + t);
        }
        for (int t = 0; t < MPNN_H; ++t) dhL[(size_t)MPNN_H * v + t] = dh[t];
    }
}

__global__ void headEdgeBackKernel(int nv, const int* rowS, const int* rowE, const int* col, const float* dG, const bf16* w, float* D9, float* deL) {
    constexpr int IN = MPNN_H + MPNN_EF;
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) {
            if (col[k] >= v) continue;
            const float* d = dG + (size_t)9 * k;
            float dh[MPNN_H];
            for (int t = 0; t < MPNN_H; ++t) dh[t] = 0.f;
            for (int q = 0; q < 9; ++q) {
                D9[(size_t)9 * k + q] = d[q];
                const bf16* Wr = w + MP_WO + q * IN;
                for (int t = 0; t < MPNN_H; ++t) dh[t] += d[q] * W(Wr, t);
            }
            for (int t = 0; t < MPNN_H; ++t) deL[(size_t)MPNN_H * k + t] = dh[t];
        }
    }
}

// node layer backward: h' = relu(Wh [h; agg] + b)
__global__ void nodeLayerBackKernel(int nv, const float* hNext, const float* dhNext, const bf16* Wm, float* D32, float* dhPrev, float* dagg) {
    CIPC_KERNEL_LOOP(v, nv) {
        float dpre[MPNN_H];
        for (int t = 0; t < MPNN_H; ++t) {
            dpre[t] = hNext[(size_t)MPNN_H * v + t] > 0.f ? dhNext[(size_t)MPNN_H * v + t] : 0.f;
            D32[(size_t)MPNN_H * v + t] = dpre[t];
        }
        for (int i = 0; i < 2 * MPNN_H; ++i) {
            float s = 0.f;
            for (int o = 0; o < MPNN_H; ++o) s += W(Wm, o * 2 * MPNN_H + i) * dpre[o];
            if (i < MPNN_H) dhPrev[(size_t)MPNN_H * v + i] += s;
            else dagg[(size_t)MPNN_H * v + i - MPNN_H] = s;
        }
    }
}

// d e_k += dagg_i / deg_i + dagg_j / deg_j for the edge k = (i, j)
__global__ void aggBackKernel(int nv, const int* rowS, const int* rowE, const int* col, const float* dagg, const int* deg, float* de) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) {
            int c = col[k];
            if (c >= v) continue;
            float iv = deg[v] > 0 ? 1.f / deg[v] : 0.f, ic = deg[c] > 0 ? 1.f / deg[c] : 0.f;
            for (int t = 0; t < MPNN_H; ++t) de[(size_t)MPNN_H * k + t] += dagg[(size_t)MPNN_H * v + t] * iv + dagg[(size_t)MPNN_H * c + t] * ic;
        }
    }
}

// edge layer backward: e' = relu(We [e; h_i + h_j] + b); adds to de^l,
// writes ds_k (the gradient with respect to h_i + h_j), the pre-activation
// gradient and the summed endpoint states (the second input block)
__global__ void edgeLayerBackKernel(int nv, const int* rowS, const int* rowE, const int* col, const float* hPrev, const float* eNext,
                                    const float* deNext, const bf16* Wm, float* D32, float* hsum, float* dePrev, float* ds) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) {
            int c = col[k];
            if (c >= v) continue;
            float dpre[MPNN_H];
            for (int t = 0; t < MPNN_H; ++t) {
                dpre[t] = eNext[(size_t)MPNN_H * k + t] > 0.f ? deNext[(size_t)MPNN_H * k + t] : 0.f;
                D32[(size_t)MPNN_H * k + t] = dpre[t];
                hsum[(size_t)MPNN_H * k + t] = hPrev[(size_t)MPNN_H * v + t] + hPrev[(size_t)MPNN_H * c + t];
            }
            for (int i = 0; i < 2 * MPNN_H; ++i) {
                float s = 0.f;
                for (int o = 0; o < MPNN_H; ++o) s += W(Wm, o * 2 * MPNN_H + i) * dpre[o];
                if (i < MPNN_H) dePrev[(size_t)MPNN_H * k + i] += s;
                else ds[(size_t)MPNN_H * k + i - MPNN_H] = s;
            }
        }
    }
}

// dh_v += sum of ds over the edges incident to v (read at their lower slot)
__global__ void dsGatherKernel(int nv, const int* rowPtr, const int* col, const int* mirS, const float* dsS, const int* dRowS, const int* dRowE,
                               const int* dCol, const int* mirD, const float* dsD, float* dh) {
    CIPC_KERNEL_LOOP(v, nv) {
        float s[MPNN_H];
        for (int t = 0; t < MPNN_H; ++t) s[t] = 0.f;
        for (int k = rowPtr[v]; k < rowPtr[v + 1]; ++k) {
            int c = col[k];
            if (c == v) continue;
            int slot = c < v ? k : mirS[k];
            if (slot < 0) continue;
            for (int t = 0; t < MPNN_H; ++t) s[t] += dsS[(size_t)MPNN_H * slot + t];
        }
        if (dRowS)
            for (int k = dRowS[v]; k < dRowE[v]; ++k) {
                int c = dCol[k];
                if (c == v) continue;
                int slot = c < v ? k : mirD[k];
                if (slot < 0) continue;
                for (int t = 0; t < MPNN_H; ++t) s[t] += dsD[(size_t)MPNN_H * slot + t];
            }
        for (int t = 0; t < MPNN_H; ++t) dh[(size_t)MPNN_H * v + t] += s[t];
    }
}

// pre-activation gradient of an embedding (relu): items are nodes or, with
// row ranges, the lower slots of a pattern
__global__ void reluGradNodeKernel(int nv, const float* y, const float* dy, float* D32) {
    CIPC_KERNEL_LOOP(i, nv * MPNN_H) D32[i] = y[i] > 0.f ? dy[i] : 0.f;
}
__global__ void reluGradEdgeKernel(int nv, const int* rowS, const int* rowE, const int* col, const float* y, const float* dy, float* D32) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) {
            if (col[k] >= v) continue;
            for (int t = 0; t < MPNN_H; ++t) D32[(size_t)MPNN_H * k + t] = y[(size_t)MPNN_H * k + t] > 0.f ? dy[(size_t)MPNN_H * k + t] : 0.f;
        }
    }
}

// 1 for lower slots (col < row) of a row-ranged pattern, else 0
__global__ void lowerMaskKernel(int nv, const int* rowS, const int* rowE, const int* col, unsigned char* mask) {
    CIPC_KERNEL_LOOP(v, nv) {
        for (int k = rowS[v]; k < rowE[v]; ++k) mask[k] = col[k] < v ? 1 : 0;
    }
}

__global__ void toBf16Kernel(int n, const float* w, bf16* o) {
    CIPC_KERNEL_LOOP(i, n) o[i] = __float2bfloat16_rn(w[i]);
}

__global__ void adamKernel(int n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2, float eps, float c1, float c2, float clip) {
    CIPC_KERNEL_LOOP(i, n) {
        float gi = fmaxf(-clip, fminf(clip, g[i]));
        m[i] = b1 * m[i] + (1.f - b1) * gi;
        v[i] = b2 * v[i] + (1.f - b2) * gi * gi;
        w[i] -= lr * (m[i] / c1) / (sqrtf(v[i] / c2) + eps);
    }
}

__global__ void zeroFloatKernel(size_t n, float* a) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)blockDim.x * gridDim.x) a[i] = 0.f;
}

struct DynView {
    const int *rs, *re, *col;
    bool on;
};
DynView dynView(Ctx& c) {
    bool on = c.nDynB > 0;
    return {on ? c.dynRowStart.p : nullptr, on ? c.dynRowEnd.p : nullptr, on ? c.dynCol.p : nullptr, on};
}

void zeroF(Ctx& c, float* p, size_t n) {
    if (n) launch(zeroFloatKernel, (unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, c.s, n, p);
}
const bf16* wbf(Ctx& c) { return reinterpret_cast<const bf16*>(c.mpWb.p); }

}  // namespace

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
void mpnnInitWeights(Ctx& c, unsigned long long seed) {
    std::vector<float> w(MP_NPARAM, 0.f);
    unsigned long long z = seed;
    auto rnd = [&]() {
        z += 0x9E3779B97F4A7C15ull;
        unsigned long long t = z;
        t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
        t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
        t ^= t >> 31;
        return (double)(t >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
    };
    auto fill = [&](int off, int fanOut, int fanIn) {
        double s = std::sqrt(6.0 / (fanIn + fanOut));
        for (int i = 0; i < fanOut * fanIn; ++i) w[off + i] = (float)(s * rnd());
    };
    fill(MP_WN0, MPNN_H, MPNN_NF);
    fill(MP_WE0, MPNN_H, MPNN_EF);
    for (int l = 0; l < MPNN_L; ++l) { fill(mpWe(l), MPNN_H, 2 * MPNN_H); fill(mpWh(l), MPNN_H, 2 * MPNN_H); }
    // heads start at the first-order factor G = I - strict_lower(Â)
    const float inv = (float)std::log(std::exp(1.0) - 1.0);  // softplus^-1(1)
    w[MP_BD + 0] = w[MP_BD + 1] = w[MP_BD + 2] = inv;
    for (int q = 0; q < 9; ++q) w[MP_WO + q * (MPNN_H + MPNN_EF) + MPNN_H + q] = -1.f;
    mpnnSetWeights(c, w.data(), MP_NPARAM);
}

void mpnnSetWeights(Ctx& c, const float* w, int n) {
    if (n != MP_NPARAM) throw InvalidArgument("expected " + std::to_string(MP_NPARAM) + " network parameters, got " + std::to_string(n));
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(w[i])) throw InvalidArgument("network parameter " + std::to_string(i) + " is not finite");
    c.mpW.reserve(MP_NPARAM); c.mpWb.reserve(MP_NPARAM); c.mpG.reserve(MP_NPARAM); c.mpM.reserve(MP_NPARAM); c.mpV.reserve(MP_NPARAM);
    CIPC_CUDA(cudaMemcpyAsync(c.mpW.p, w, sizeof(float) * MP_NPARAM, cudaMemcpyHostToDevice, c.s));
    zeroF(c, c.mpM.p, MP_NPARAM);
    zeroF(c, c.mpV.p, MP_NPARAM);
    zeroF(c, c.mpG.p, MP_NPARAM);
    launch(toBf16Kernel, blocksFor(MP_NPARAM), TB, 0, c.s, MP_NPARAM, (const float*)c.mpW.p, reinterpret_cast<bf16*>(c.mpWb.p));
    hostSync(c);
    c.mpStep = 0;
    c.mpReady = true;
    c.mpFactorReady = false;
}

void mpnnGetWeights(Ctx& c, float* w) {
    if (!c.mpReady) throw InvalidArgument("no network weights set");
    CIPC_CUDA(cudaMemcpyAsync(w, c.mpW.p, sizeof(float) * MP_NPARAM, cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
}

void mpnnGetGrad(Ctx& c, float* g) {
    if (!c.mpReady) throw InvalidArgument("no network weights set");
    CIPC_CUDA(cudaMemcpyAsync(g, c.mpG.p, sizeof(float) * MP_NPARAM, cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
}

// Flat list of the lower edges of a row-ranged pattern: three arrays of
// `count` ints (slot, row, column) packed in `out`.  Returns the count.
static int buildLowerList(Ctx& c, const int* rowS, const int* rowE, const int* col, DBuf<int>& out) {
    int nv = c.nv;
    c.mpScanTmpI.reserve(2 * (size_t)nv + 2);
    int* cnt = c.mpScanTmpI.p;
    int* off = cnt + nv + 1;
    launch(lowerCountKernel, blocksFor(nv), TB, 0, c.s, nv, rowS, rowE, col, cnt);
    CIPC_CUDA(cudaMemsetAsync(cnt + nv, 0, sizeof(int), c.s));
    size_t bytes = 0;
    CIPC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, cnt, off, nv + 1, c.s));
    c.mpScanTmp.reserve(bytes + 16);
    CIPC_CUDA(cub::DeviceScan::ExclusiveSum(c.mpScanTmp.p, bytes, cnt, off, nv + 1, c.s));
    int n = 0;
    CIPC_CUDA(cudaMemcpyAsync(&n, off + nv, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    out.reserve(3 * (size_t)std::max(n, 1));
    if (n > 0) launch(lowerFillKernel, blocksFor(nv), TB, 0, c.s, nv, rowS, rowE, col, (const int*)off, out.p, out.p + n, out.p + 2 * (size_t)n);
    return n;
}

template <class MT>
static void prepareT(Ctx& c, const MT* val, const MT* dval, bool features) {
    int nv = c.nv;
    DynView d = dynView(c);
    size_t es = (size_t)std::max(c.nnzb, 1), ed = (size_t)std::max(c.nDynB, 1);
    c.mpS.reserve(9 * (size_t)nv);
    c.mpNodeF.reserve(MPNN_NF * (size_t)nv + nv);
    float* f5 = c.mpNodeF.p + MPNN_NF * (size_t)nv;
    launch(scaleKernel<MT>, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.diagSlot.p, val, d.rs, d.re, d.col, dval, (const double*)c.diagExtra.p,
           c.mpS.p, f5);
    if (features)
        launch(nodeFeatKernel<MT>, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.rowPtr.p, (const int*)c.colIdx.p, val, d.rs, d.re, d.col, dval,
               (const double*)c.mpS.p, (const float*)f5, c.mpNodeF.p);
    if (!c.mpMirrorReady) {
        c.mpMirS.reserve(es);
        c.mpRowS.reserve(nv); c.mpRowE.reserve(nv);
        launch(rowRangeKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.rowPtr.p, c.mpRowS.p, c.mpRowE.p);
        launch(mirrorKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.mpRowS.p, (const int*)c.mpRowE.p, (const int*)c.colIdx.p, c.mpMirS.p);
        c.mpLowS.reserve(es);
        launch(lowerMaskKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.mpRowS.p, (const int*)c.mpRowE.p, (const int*)c.colIdx.p, c.mpLowS.p);
        c.mpMirrorReady = true;
    }
    c.mpEdgeF.reserve(9 * es);
    if (features)
        launch(edgeFeatKernel<MT>, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.mpRowS.p, (const int*)c.mpRowE.p, (const int*)c.colIdx.p, val,
               (const double*)c.mpS.p, c.mpEdgeF.p);
    c.mpMirD.reserve(ed);
    c.mpEdgeFD.reserve(9 * ed);
    c.mpLowD.reserve(ed);
    if (d.on) {
        launch(mirrorKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, c.mpMirD.p);
        launch(lowerMaskKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, c.mpLowD.p);
        if (features) launch(edgeFeatKernel<MT>, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, dval, (const double*)c.mpS.p, c.mpEdgeFD.p);
    }
    if (features) {  // the network's flat edge lists
        if (c.nFlatS < 0) c.nFlatS = buildLowerList(c, (const int*)c.mpRowS.p, (const int*)c.mpRowE.p, (const int*)c.colIdx.p, c.mpFlatS);
        c.nFlatD = d.on ? buildLowerList(c, d.rs, d.re, d.col, c.mpFlatD) : 0;
    }
    c.mpDeg.reserve(nv);
    launch(degreeKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.rowPtr.p, (const int*)c.colIdx.p, (const int*)c.mpMirS.p, d.rs, d.re, d.col,
           (const int*)c.mpMirD.p, c.mpDeg.p);
    CIPC_CUDA(cudaGetLastError());
    c.mpFactorReady = false;
}

void mpnnPrepare(Ctx& c, bool features) {
    if (c.mixed) prepareT<float>(c, c.valF.p, c.dynBF.p, features);
    else prepareT<double>(c, c.valD.p, c.dynBD.p, features);
}

static_assert(mpWe(0) % 8 == 0 && mpWh(0) % 8 == 0 && MP_LAYER % 8 == 0,
              "tensor-core layer weights start on 16-byte boundaries");

void mpnnForward(Ctx& c) {
    if (!c.mpReady) throw InvalidArgument("no network weights set");
    if (c.tcFault) throw std::runtime_error("a tensor-core wait timed out earlier on this context; recreate it to use the learned preconditioner");
    int nv = c.nv;
    DynView d = dynView(c);
    size_t es = (size_t)std::max(c.nnzb, 1), ed = (size_t)std::max(c.nDynB, 1);
    c.mpH.reserve((size_t)(MPNN_L + 1) * MPNN_H * nv);
    c.mpAgg.reserve((size_t)MPNN_L * MPNN_H * nv);
    c.mpES.reserve((size_t)(MPNN_L + 1) * MPNN_H * es);
    c.mpED.reserve((size_t)(MPNN_L + 1) * MPNN_H * ed);
    c.mpGS.reserve(9 * es);
    c.mpGD.reserve(9 * ed);
    c.mpHeadD.reserve(6 * (size_t)nv);
    const bf16* w = wbf(c);
    auto H = [&](int l) { return c.mpH.p + (size_t)l * MPNN_H * nv; };
    auto ES = [&](int l) { return c.mpES.p + (size_t)l * MPNN_H * es; };
    auto ED = [&](int l) { return c.mpED.p + (size_t)l * MPNN_H * ed; };
    const int nS = c.nFlatS, nD = d.on ? c.nFlatD : 0;
    const int *sSlot = c.mpFlatS.p, *sI = sSlot + nS, *sJ = sSlot + 2 * (size_t)nS;
    const int *dSlot = c.mpFlatD.p, *dI = dSlot + nD, *dJ = dSlot + 2 * (size_t)nD;
    auto grid = [](int n) { return std::max(1, std::min((n + DT_ITEMS - 1) / DT_ITEMS, 148 * 16)); };
    // embeddings
    launch(denseTiledKernel<MPNN_NF, MPNN_H, NodeFeatGather, ReluEmitNode>, grid(nv), DT_THREADS, 0, c.s, nv, NodeFeatGather{c.mpNodeF.p},
           ReluEmitNode{H(0)}, w + MP_WN0, w + MP_BN0);
    if (nS) launch(denseTiledKernel<MPNN_EF, MPNN_H, EdgeFeatGather, ReluEmitEdge>, grid(nS), DT_THREADS, 0, c.s, nS,
                   EdgeFeatGather{sSlot, c.mpEdgeF.p}, ReluEmitEdge{sSlot, ES(0)}, w + MP_WE0, w + MP_BE0);
    if (nD) launch(denseTiledKernel<MPNN_EF, MPNN_H, EdgeFeatGather, ReluEmitEdge>, grid(nD), DT_THREADS, 0, c.s, nD,
                   EdgeFeatGather{dSlot, c.mpEdgeFD.p}, ReluEmitEdge{dSlot, ED(0)}, w + MP_WE0, w + MP_BE0);
    // the 64 -> 32 message-passing layers run on the tensor cores
    auto tcGrid = [](int n) { return std::max(1, std::min((n + tc::M - 1) / tc::M, 148 * 4)); };
    for (int l = 0; l < MPNN_L; ++l) {
        if (nS) launch(tc::denseTcKernel<EdgeLayerGather, ReluEmitEdge>, tcGrid(nS), tc::THREADS, 0, c.s, nS, EdgeLayerGather{sSlot, sI, sJ, ES(l), H(l)},
                       ReluEmitEdge{sSlot, ES(l + 1)}, w + mpWe(l), w + mpBe(l), c.status.p, (int)CIPC_ST_TC_TIMEOUT);
        if (nD) launch(tc::denseTcKernel<EdgeLayerGather, ReluEmitEdge>, tcGrid(nD), tc::THREADS, 0, c.s, nD, EdgeLayerGather{dSlot, dI, dJ, ED(l), H(l)},
                       ReluEmitEdge{dSlot, ED(l + 1)}, w + mpWe(l), w + mpBe(l), c.status.p, (int)CIPC_ST_TC_TIMEOUT);
        float* agg = c.mpAgg.p + (size_t)l * MPNN_H * nv;
        launch(aggregateKernel, blocksFor(32 * nv), TB, 0, c.s, nv, (const int*)c.rowPtr.p, (const int*)c.colIdx.p, (const int*)c.mpMirS.p,
               (const float*)ES(l + 1), d.rs, d.re, d.col, (const int*)c.mpMirD.p, (const float*)ED(l + 1), (const int*)c.mpDeg.p, agg);
        launch(tc::denseTcKernel<NodeLayerGather, ReluEmitNode>, tcGrid(nv), tc::THREADS, 0, c.s, nv, NodeLayerGather{H(l), agg}, ReluEmitNode{H(l + 1)},
               w + mpWh(l), w + mpBh(l), c.status.p, (int)CIPC_ST_TC_TIMEOUT);
    }
    // heads: contact diagonal slots carry no factor part
    if (d.on) CIPC_CUDA(cudaMemsetAsync(c.mpGD.p, 0, sizeof(float) * 9 * (size_t)c.nDynB, c.s));
    if (nS) launch(denseTiledKernel<MPNN_H + MPNN_EF, 9, HeadEdgeGather, HeadEdgeEmit>, grid(nS), DT_THREADS, 0, c.s, nS,
                   HeadEdgeGather{sSlot, ES(MPNN_L), c.mpEdgeF.p}, HeadEdgeEmit{sSlot, sI, sJ, c.mpMirS.p, c.btype.p, c.mpGS.p}, w + MP_WO, w + MP_BO);
    if (nD) launch(denseTiledKernel<MPNN_H + MPNN_EF, 9, HeadEdgeGather, HeadEdgeEmit>, grid(nD), DT_THREADS, 0, c.s, nD,
                   HeadEdgeGather{dSlot, ED(MPNN_L), c.mpEdgeFD.p}, HeadEdgeEmit{dSlot, dI, dJ, c.mpMirD.p, c.btype.p, c.mpGD.p}, w + MP_WO, w + MP_BO);
    launch(denseTiledKernel<MPNN_H, 6, NodeHiddenGather, HeadDiagEmit>, grid(nv), DT_THREADS, 0, c.s, nv, NodeHiddenGather{H(MPNN_L)},
           HeadDiagEmit{c.diagSlot.p, c.btype.p, c.mpGS.p, c.mpHeadD.p}, w + MP_WD, w + MP_BD);
    CIPC_CUDA(cudaGetLastError());
    c.mpFactorReady = true;
}

template <class MT>
static double lossT(Ctx& c, const MT* val, const MT* dval, int nprobes, const float* hostProbes, unsigned long long seed, bool backward) {
    int nv = c.nv, n3 = 3 * nv;
    DynView d = dynView(c);
    size_t es = (size_t)std::max(c.nnzb, 1), ed = (size_t)std::max(c.nDynB, 1);
    c.mpVec.reserve(3 * (size_t)n3);
    float* w = c.mpVec.p;
    float* u = w + n3;   // G^T w
    float* vv = u + n3;  // Â G^T w
    if (backward) {
        c.mpDGS.reserve(9 * es);
        c.mpDGD.reserve(9 * ed);
        zeroF(c, c.mpDGS.p, 9 * es);
        zeroF(c, c.mpDGD.p, 9 * ed);
    }
    int nb = std::min(1024, std::max(1, (n3 + 255) / 256));
    c.red.reserve(2 * 1024 + 16);
    std::vector<double> part(2 * nb + 2 * 1024);
    double T = 0;
    for (int pr = 0; pr < nprobes; ++pr) {
        if (hostProbes)
            CIPC_CUDA(cudaMemcpyAsync(w, hostProbes + (size_t)pr * n3, sizeof(float) * n3, cudaMemcpyHostToDevice, c.s));
        else
            launch(probeKernel, blocksFor(n3), TB, 0, c.s, n3, seed + 7919ull * pr, w);
        launch(factorApplyKernel, blocksFor(nv), TB, 0, c.s, nv, 1, (const int*)c.rowPtr.p, (const int*)c.colIdx.p, (const float*)c.mpGS.p, d.rs, d.re,
               d.col, (const float*)c.mpGD.p, (const float*)w, u);
        launch(scaledSpmvKernel<MT>, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.rowPtr.p, (const int*)c.colIdx.p, val, d.rs, d.re, d.col, dval,
               (const double*)c.diagExtra.p, (const double*)c.mpS.p, (const float*)u, vv);
        launch(probeDotsKernel, nb, 256, 0, c.s, n3, (const float*)u, (const float*)vv, (const float*)w, c.red.p);
        CIPC_CUDA(cudaMemcpyAsync(part.data(), c.red.p, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, c.s));
        hostSync(c);
        double uv = 0, ww = 0;
        for (int k = 0; k < nb; ++k) { uv += part[2 * k]; ww += part[2 * k + 1]; }
        if (!(ww > 0)) throw InvalidArgument("probe vector is zero");
        T += uv / ww / nprobes;
        if (backward) {
            float scale = (float)(2.0 / ww / nprobes);
            launch(factorGradKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.mpRowS.p, (const int*)c.mpRowE.p, (const int*)c.colIdx.p, 0,
                   (const int*)c.btype.p, (const float*)w, (const float*)vv, scale, c.mpDGS.p);
            if (d.on)
                launch(factorGradKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, 1, (const int*)c.btype.p, (const float*)w, (const float*)vv,
                       scale, c.mpDGD.p);
        }
    }
    int nb2 = std::min(1024, std::max(1, (nv + 255) / 256));
    launch(logDiagKernel, nb2, 256, 0, c.s, nv, (const int*)c.diagSlot.p, (const float*)c.mpGS.p, c.red.p);
    CIPC_CUDA(cudaMemcpyAsync(part.data(), c.red.p, sizeof(double) * nb2, cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    double logDiag = 0;
    for (int k = 0; k < nb2; ++k) logDiag += part[k];
    if (!(T > 0) || !std::isfinite(T) || !std::isfinite(logDiag)) throw std::runtime_error("learned preconditioner loss is not finite");
    double loss = std::log(T) - 2.0 / n3 * logDiag;
    if (!backward) return loss;

    launch(gradScaleKernel, 1024, 256, 0, c.s, 9 * es, (float)(1.0 / T), c.mpDGS.p);
    if (d.on) launch(gradScaleKernel, 1024, 256, 0, c.s, 9 * ed, (float)(1.0 / T), c.mpDGD.p);
    launch(gradDiagKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.diagSlot.p, (const int*)c.btype.p, (const float*)c.mpGS.p, (float)(2.0 / n3),
           c.mpDGS.p);

    const bf16* wb = wbf(c);
    float* gW = c.mpG.p;
    zeroF(c, gW, MP_NPARAM);
    size_t items = std::max(std::max(es, ed), (size_t)nv);
    c.mpDH.reserve((size_t)(MPNN_L + 1) * MPNN_H * nv);
    c.mpDES.reserve((size_t)(MPNN_L + 1) * MPNN_H * es);
    c.mpDED.reserve((size_t)(MPNN_L + 1) * MPNN_H * ed);
    c.mpDAgg.reserve((size_t)MPNN_H * nv);
    c.mpDS.reserve((size_t)MPNN_H * es);
    c.mpDSD.reserve((size_t)MPNN_H * ed);
    c.mpBD.reserve((size_t)MPNN_H * items);
    c.mpBX.reserve((size_t)MPNN_H * items);
    c.mpPart.reserve((size_t)WG_GRID * (MPNN_H * 2 * MPNN_H + MPNN_H));
    zeroF(c, c.mpDH.p, (size_t)(MPNN_L + 1) * MPNN_H * nv);
    zeroF(c, c.mpDES.p, (size_t)(MPNN_L + 1) * MPNN_H * es);
    zeroF(c, c.mpDED.p, (size_t)(MPNN_L + 1) * MPNN_H * ed);
    auto H = [&](int l) { return c.mpH.p + (size_t)l * MPNN_H * nv; };
    auto DH = [&](int l) { return c.mpDH.p + (size_t)l * MPNN_H * nv; };
    auto ES = [&](int l) { return c.mpES.p + (size_t)l * MPNN_H * es; };
    auto ED = [&](int l) { return c.mpED.p + (size_t)l * MPNN_H * ed; };
    auto DES = [&](int l) { return c.mpDES.p + (size_t)l * MPNN_H * es; };
    auto DED = [&](int l) { return c.mpDED.p + (size_t)l * MPNN_H * ed; };
    const int *rs = c.mpRowS.p, *re = c.mpRowE.p, *col = c.colIdx.p;
    float* BD = c.mpBD.p;
    float* BX = c.mpBX.p;
    // dW += D^T [X1 X2], db += sum D over `n` items (split-K, deterministic)
    auto wgrad = [&](auto kernel, int out, int in, int n, const float* X1, const float* X2, const unsigned char* mask, int wOff, int bOff) {
        if (n <= 0) return;
        int nw = out * in + out;
        int grid = std::max(1, std::min(WG_GRID, (n + WG_TI - 1) / WG_TI));
        launch(kernel, grid, WG_THREADS, 0, c.s, n, (const float*)BD, X1, X2, mask, c.mpPart.p);
        launch(weightGradReduceKernel, blocksFor(nw), TB, 0, c.s, nw, out, grid, (const float*)c.mpPart.p, gW + wOff, gW + bOff);
    };
    // the 64 -> 32 message-passing layers: the same contraction on the tensor cores
    auto wgradTc = [&](int n, const float* X1, const float* X2, const unsigned char* mask, int wOff, int bOff) {
        if (n <= 0) return;
        static bool attr = false;
        if (!attr) {
            CIPC_CUDA(cudaFuncSetAttribute(tc::weightGradTcKernel, cudaFuncAttributeMaxDynamicSharedMemorySize, tc::WG_SMEM));
            attr = true;
        }
        const int nw = MPNN_H * 2 * MPNN_H + MPNN_H;
        const int grid = std::max(1, std::min(WG_GRID, (n + tc::WG_K - 1) / tc::WG_K));
        launch(tc::weightGradTcKernel, grid, tc::THREADS, tc::WG_SMEM, c.s, n, (const float*)BD, X1, X2, mask, c.mpPart.p, c.status.p,
               (int)CIPC_ST_TC_TIMEOUT);
        launch(weightGradReduceKernel, blocksFor(nw), TB, 0, c.s, nw, MPNN_H, grid, (const float*)c.mpPart.p, gW + wOff, gW + bOff);
    };
    int nd = d.on ? c.nDynB : 0;
    // heads
    launch(headDiagBackKernel, blocksFor(nv), TB, 0, c.s, nv, (const float*)c.mpHeadD.p, (const int*)c.diagSlot.p, (const float*)c.mpDGS.p, wb, BD,
           DH(MPNN_L));
    wgrad(weightGradKernel<6, MPNN_H, 0>, 6, MPNN_H, nv, (const float*)H(MPNN_L), (const float*)nullptr, (const unsigned char*)nullptr, MP_WD, MP_BD);
    launch(headEdgeBackKernel, blocksFor(nv), TB, 0, c.s, nv, rs, re, col, (const float*)c.mpDGS.p, wb, BD, DES(MPNN_L));
    wgrad(weightGradKernel<9, MPNN_H, MPNN_EF>, 9, MPNN_H + MPNN_EF, c.nnzb, (const float*)ES(MPNN_L), (const float*)c.mpEdgeF.p,
          (const unsigned char*)c.mpLowS.p, MP_WO, MP_BO);
    if (d.on) {
        launch(headEdgeBackKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, (const float*)c.mpDGD.p, wb, BD, DED(MPNN_L));
        wgrad(weightGradKernel<9, MPNN_H, MPNN_EF>, 9, MPNN_H + MPNN_EF, nd, (const float*)ED(MPNN_L), (const float*)c.mpEdgeFD.p,
              (const unsigned char*)c.mpLowD.p, MP_WO, MP_BO);
    }
    for (int l = MPNN_L - 1; l >= 0; --l) {
        const float* agg = c.mpAgg.p + (size_t)l * MPNN_H * nv;
        launch(nodeLayerBackKernel, blocksFor(nv), TB, 0, c.s, nv, (const float*)H(l + 1), (const float*)DH(l + 1), wb + mpWh(l), BD, DH(l), c.mpDAgg.p);
        wgradTc(nv, (const float*)H(l), agg, (const unsigned char*)nullptr, mpWh(l), mpBh(l));
        launch(aggBackKernel, blocksFor(nv), TB, 0, c.s, nv, rs, re, col, (const float*)c.mpDAgg.p, (const int*)c.mpDeg.p, DES(l + 1));
        if (d.on) launch(aggBackKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, (const float*)c.mpDAgg.p, (const int*)c.mpDeg.p, DED(l + 1));
        launch(edgeLayerBackKernel, blocksFor(nv), TB, 0, c.s, nv, rs, re, col, (const float*)H(l), (const float*)ES(l + 1), (const float*)DES(l + 1),
               wb + mpWe(l), BD, BX, DES(l), c.mpDS.p);
        wgradTc(c.nnzb, (const float*)ES(l), (const float*)BX, (const unsigned char*)c.mpLowS.p, mpWe(l), mpBe(l));
        if (d.on) {
            launch(edgeLayerBackKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, (const float*)H(l), (const float*)ED(l + 1),
                   (const float*)DED(l + 1), wb + mpWe(l), BD, BX, DED(l), c.mpDSD.p);
            wgradTc(nd, (const float*)ED(l), (const float*)BX, (const unsigned char*)c.mpLowD.p, mpWe(l), mpBe(l));
        }
        launch(dsGatherKernel, blocksFor(nv), TB, 0, c.s, nv, (const int*)c.rowPtr.p, col, (const int*)c.mpMirS.p, (const float*)c.mpDS.p, d.rs, d.re,
               d.col, (const int*)c.mpMirD.p, (const float*)c.mpDSD.p, DH(l));
    }
    // embeddings
    launch(reluGradNodeKernel, blocksFor(nv * MPNN_H), TB, 0, c.s, nv, (const float*)H(0), (const float*)DH(0), BD);
    wgrad(weightGradKernel<MPNN_H, MPNN_NF, 0>, MPNN_H, MPNN_NF, nv, (const float*)c.mpNodeF.p, (const float*)nullptr, (const unsigned char*)nullptr,
          MP_WN0, MP_BN0);
    launch(reluGradEdgeKernel, blocksFor(nv), TB, 0, c.s, nv, rs, re, col, (const float*)ES(0), (const float*)DES(0), BD);
    wgrad(weightGradKernel<MPNN_H, MPNN_EF, 0>, MPNN_H, MPNN_EF, c.nnzb, (const float*)c.mpEdgeF.p, (const float*)nullptr, (const unsigned char*)c.mpLowS.p,
          MP_WE0, MP_BE0);
    if (d.on) {
        launch(reluGradEdgeKernel, blocksFor(nv), TB, 0, c.s, nv, d.rs, d.re, d.col, (const float*)ED(0), (const float*)DED(0), BD);
        wgrad(weightGradKernel<MPNN_H, MPNN_EF, 0>, MPNN_H, MPNN_EF, nd, (const float*)c.mpEdgeFD.p, (const float*)nullptr, (const unsigned char*)c.mpLowD.p,
              MP_WE0, MP_BE0);
    }
    CIPC_CUDA(cudaGetLastError());
    return loss;
}

double mpnnLoss(Ctx& c, int nprobes, const float* probes, unsigned long long seed, bool backward) {
    if (!c.mpFactorReady) throw InvalidArgument("no factor: run the network forward on an assembled system first");
    if (nprobes < 1) throw InvalidArgument("need at least one probe vector");
    if (c.mixed) return lossT<float>(c, c.valF.p, c.dynBF.p, nprobes, probes, seed, backward);
    return lossT<double>(c, c.valD.p, c.dynBD.p, nprobes, probes, seed, backward);
}

void mpnnAdam(Ctx& c, double lr) {
    c.mpStep++;
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.f - std::pow(b1, (float)c.mpStep), c2 = 1.f - std::pow(b2, (float)c.mpStep);
    launch(adamKernel, blocksFor(MP_NPARAM), TB, 0, c.s, MP_NPARAM, c.mpW.p, (const float*)c.mpG.p, c.mpM.p, c.mpV.p, (float)lr, b1, b2, 1e-8f, c1,
           c2, 1.0f);
    launch(toBf16Kernel, blocksFor(MP_NPARAM), TB, 0, c.s, MP_NPARAM, (const float*)c.mpW.p, reinterpret_cast<bf16*>(c.mpWb.p));
    CIPC_CUDA(cudaGetLastError());
    c.mpFactorReady = false;
}

}  // namespace cipc
