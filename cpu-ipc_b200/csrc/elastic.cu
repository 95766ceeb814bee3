// Elastic assembly on the GPU: inertia/drag/soft per vertex, Stable
// Neo-Hookean tetrahedra, Baraff-Witkin cloth triangles and quadratic bending
// hinges.  Every element writes its gradient rows and lower-triangular 3x3
// Hessian blocks to private slots; per-vertex and per-BSR-slot gathers then
// sum them in a fixed order (no atomics, deterministic).
//
// Reference: computeGradientAndHessian, CPU IPC/IPCSolver.cpp:108-237;
// Elasticity.cpp:1144-1205 (PK1), 1337-1544 (Hessians), 695-771 (energies).
#include "cipc_device.cuh"
#include "cipc_internal.h"
#include "hinge_bending.cuh"

#include <algorithm>
#include <numeric>

namespace cipc {

namespace {

constexpr int TB = 128;
inline int blocksFor(int n, int tb = TB) { return std::max(1, std::min((n + tb - 1) / tb, 148 * 16)); }

// Lower-block index of local pair (a, b), a >= b.
__host__ __device__ __forceinline__ int lowerIdx(int a, int b) { return a * (a + 1) / 2 + b; }

__global__ void vertexInitKernel(int nv, const double* x, const double* xt, const double* vp, const double* mass, double drag,
                                 double* vtxGrad, double* diagExtra) {
    CIPC_KERNEL_LOOP(v, nv) {
        double m = mass[v];
        for (int k = 0; k < 3; ++k) {
            double g = m * (x[3 * v + k] - xt[3 * v + k]);
            g += drag * m * (x[3 * v + k] - vp[3 * v + k]);
            vtxGrad[3 * v + k] = g;
        }
        double d = m * (1.0 + drag);
        for (int k = 0; k < 9; ++k) diagExtra[9 * v + k] = (k % 4 == 0) ? d : 0.0;
    }
}

__global__ void softKernel(int ns, const int* idx, const double* target, double w, const double* x, double* vtxGrad, double* diagExtra) {
    CIPC_KERNEL_LOOP(k, ns) {
        int v = idx[k];
        for (int d = 0; d < 3; ++d) vtxGrad[3 * v + d] += w * (x[3 * v + d] - target[3 * k + d]);
        diagExtra[9 * v + 0] += w; diagExtra[9 * v + 4] += w; diagExtra[9 * v + 8] += w;
    }
}

// Stable Neo-Hookean tetrahedra (PK1 Elasticity.cpp:1144-1170, Hessian and
// makePD 1337-1479, scatter IPCSolver.cpp:139-164), tiled in two phases.
//
// Phase 1, one thread per tetrahedron: F = Ds Dm^-1, the gradient
// vol dt^2 P(F) G^T, and the Hessian's analytic eigensystem in F space - the
// rotation-aware SVD F = U diag(s) V^T, 3 scaling modes (a 3x3 eigenproblem
// in the singular-value basis) and 3 twist + 3 flip modes with closed-form
// eigenvalues mu Ic/(Ic+1) +/- lambda (J - alpha) s_k.  Each mode m with
// eigenvalue e_m > 0 leaves w_m[a] = sqrt(vol dt^2 e_m) Q_m G_a (3 values per
// vertex a) in shared memory, so that the projected 12x12 Hessian is
// sum_m w_m w_m^T (the PSD projection of project_StabbleNHK_2_H_3D's 9x9
// matrix pulled back through PFPX).
//
// Phase 2, the CTA's threads over (tetrahedron, lower block, block row):
// each forms 3 entries of one lower 3x3 block, sum_m w_m[a][r] w_m[b][q],
// and stores them next to its neighbours' (the tile's element blocks are one
// contiguous range of elemH, 90 values per tetrahedron).  Blocks touching a
// constrained vertex are zeroed as the reference drops them.
// ---------------------------------------------------------------------------
template <class T>
struct TetTile;
template <>
struct TetTile<float> { static constexpr int N = 128; };
template <>
struct TetTile<double> { static constexpr int N = 64; };
constexpr int TET_W = 109;  // 9 modes x 4 vertices x 3, padded to an odd stride (bank spread)

// mode m (0..8) of the SNH Hessian eigensystem: eigenvalue and Q_m (3x3)
template <class T>
__device__ __forceinline__ T snhMode(int m, const T U[3][3], const T V[3][3], const T W[3][3], const T A[3][3], const T s[3], T Ut, T lJ,
                                     T Q[3][3]) {
    if (m < 3) {
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = 0; c < 3; ++c) Q[r][c] = U[r][0] * W[0][m] * V[c][0] + U[r][1] * W[1][m] * V[c][1] + U[r][2] * W[2][m] * V[c][2];
        return A[m][m];
    }
    const int t = (m - 3) % 3;
    const int i = t == 2 ? 1 : 0, j = t == 0 ? 1 : 2, k = 3 - i - j;
    const bool twist = m < 6;
    const T sg = twist ? T(-1) : T(1);
    const T isq2 = T(0.70710678118654752440);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) Q[r][c] = isq2 * (U[r][i] * V[c][j] + sg * U[r][j] * V[c][i]);
    return twist ? Ut + lJ * s[k] : Ut - lJ * s[k];
}

template <class T, bool HESS>
__global__ void __launch_bounds__(TetTile<T>::N) tetKernel(int nt, const int* tets, const double* x, const double* DmInv, const double* vol,
                                                           const double* tmu, const double* tlam, const int* btype, double dt2, double* elemG,
                                                           T* elemH) {
    constexpr int N = TetTile<T>::N;
    // dynamic shared memory (tetSmemBytes): gradients, modes, free flags
    extern __shared__ __align__(16) unsigned char tetSmem[];
    double* sg = reinterpret_cast<double*>(tetSmem);
    T* sw = reinterpret_cast<T*>(tetSmem + sizeof(double) * 12 * N);
    unsigned char* sfree = tetSmem + sizeof(double) * 12 * N + (HESS ? sizeof(T) * TET_W * N : 0);
    const int tid = threadIdx.x;
    for (int base = blockIdx.x * N; base < nt; base += gridDim.x * N) {
        const int cnt = min(N, nt - base);
        if (tid < cnt) {
            const int i = base + tid;
            int v[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) v[a] = tets[4 * i + a];
            double Di[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) Di[k] = DmInv[9 * (size_t)i + k];
            const d3 x0 = ld3(x, v[0]);
            const d3 e1 = ld3(x, v[1]) - x0, e2 = ld3(x, v[2]) - x0, e3 = ld3(x, v[3]) - x0;
            const double Ds[3][3] = {{e1.x, e2.x, e3.x}, {e1.y, e2.y, e3.y}, {e1.z, e2.z, e3.z}};
            double F[3][3];
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) F[r][c] = Ds[r][0] * Di[c] + Ds[r][1] * Di[3 + c] + Ds[r][2] * Di[6 + c];
            const double u = tmu[i], lr = tlam[i];
            double I2 = 0;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) I2 += F[r][c] * F[r][c];
            double cof[3][3];
            cof[0][0] = F[1][1] * F[2][2] - F[1][2] * F[2][1];
            cof[0][1] = F[1][2] * F[2][0] - F[1][0] * F[2][2];
            cof[0][2] = F[1][0] * F[2][1] - F[1][1] * F[2][0];
            cof[1][0] = F[2][1] * F[0][2] - F[2][2] * F[0][1];
            cof[1][1] = F[2][2] * F[0][0] - F[2][0] * F[0][2];
            cof[1][2] = F[2][0] * F[0][1] - F[2][1] * F[0][0];
            cof[2][0] = F[0][1] * F[1][2] - F[1][1] * F[0][2];
            cof[2][1] = F[0][2] * F[1][0] - F[0][0] * F[1][2];
            cof[2][2] = F[0][0] * F[1][1] - F[0][1] * F[1][0];
            const double J = F[0][0] * cof[0][0] + F[0][1] * cof[0][1] + F[0][2] * cof[0][2];
            const double ca = u * (1 - 1 / (I2 + 1)), cb = lr * (J - 1 - u * 3 / (lr * 4));
            // G rows: dF/dx_a = G[a][c] (column c of F)
            double G[4][3];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                G[1][c] = Di[c]; G[2][c] = Di[3 + c]; G[3][c] = Di[6 + c];
                G[0][c] = -(G[1][c] + G[2][c] + G[3][c]);
            }
            const double sc = vol[i] * dt2;
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int r = 0; r < 3; ++r) {
                    double f = 0;
#pragma unroll
                    for (int c = 0; c < 3; ++c) f += (ca * F[r][c] + cb * cof[r][c]) * G[a][c];
                    sg[12 * tid + 3 * a + r] = sc * f;
                }
            if (HESS) {
                unsigned char fr = 0;
#pragma unroll
                for (int a = 0; a < 4; ++a) fr |= (btype[v[a]] == 0 ? 1 : 0) << a;
                sfree[tid] = fr;
                T Ft[3][3], U[3][3], V[3][3], s[3];
#pragma unroll
                for (int r = 0; r < 3; ++r)
#pragma unroll
                    for (int c = 0; c < 3; ++c) Ft[r][c] = T(F[r][c]);
                svd3<T>(Ft, U, s, V);
                const T Ic = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
                const T Jt = s[0] * s[1] * s[2];
                const T Ut = T(u) * Ic / (Ic + T(1));
                const T lJ = T(lr) * (Jt - T(1) - T(3) * T(u) / (T(4) * T(lr)));
                const T gC = T(u) / (T(2) * (Ic + T(1)) * (Ic + T(1)));
                const T cf[3] = {s[1] * s[2], s[0] * s[2], s[0] * s[1]};
                T A[3][3];
#pragma unroll
                for (int p = 0; p < 3; ++p)
#pragma unroll
                    for (int q = 0; q < 3; ++q) {
                        A[p][q] = gC * T(4) * s[p] * s[q] + T(lr) * cf[p] * cf[q];
                        if (p == q) A[p][q] += Ut;
                        else A[p][q] += lJ * s[3 - p - q];
                    }
                T W[3][3];
                jacobiSym3<T>(A, W);
                T* w = sw + TET_W * tid;
#pragma unroll
                for (int m = 0; m < 9; ++m) {
                    T Q[3][3];
                    const T ev = snhMode<T>(m, U, V, W, A, s, Ut, lJ, Q);
                    const T coef = ev > T(0) ? sqrt(T(sc) * ev) : T(0);
#pragma unroll
                    for (int a = 0; a < 4; ++a)
#pragma unroll
                        for (int r = 0; r < 3; ++r)
                            w[12 * m + 3 * a + r] = coef * (Q[r][0] * T(G[a][0]) + Q[r][1] * T(G[a][1]) + Q[r][2] * T(G[a][2]));
                }
            }
        }
        __syncthreads();
        // the tile's gradients: 12 consecutive doubles per tetrahedron
        for (int o = tid; o < 12 * cnt; o += N) elemG[(size_t)12 * base + o] = sg[o];
        if (HESS) {
            // (tetrahedron, lower block, block row) items: 3 consecutive
            // entries of elemH each, consecutive items consecutive in memory
            T* out = elemH + (size_t)90 * base;
            for (int it = tid; it < 30 * cnt; it += N) {
                const int t = it / 30, rest = it - 30 * t;
                const int blk = rest / 3, r = rest - 3 * blk;
                const int a = blk >= 6 ? 3 : (blk >= 3 ? 2 : (blk >= 1 ? 1 : 0));
                const int b = blk - a * (a + 1) / 2;  // lowerIdx(a, b) = blk
                const T* w = sw + TET_W * t;
                T h0 = T(0), h1 = T(0), h2 = T(0);
#pragma unroll
                for (int m = 0; m < 9; ++m) {
                    const T wa = w[12 * m + 3 * a + r];
                    h0 += wa * w[12 * m + 3 * b];
                    h1 += wa * w[12 * m + 3 * b + 1];
                    h2 += wa * w[12 * m + 3 * b + 2];
                }
                const unsigned fr = sfree[t];
                const bool keep = ((fr >> a) & 1u) && ((fr >> b) & 1u);
                T* o = out + 90 * t + 9 * blk + 3 * r;
                o[0] = keep ? h0 : T(0);
                o[1] = keep ? h1 : T(0);
                o[2] = keep ? h2 : T(0);
            }
        }
        __syncthreads();
    }
}

template <class T, bool HESS>
constexpr size_t tetSmemBytes() {
    return sizeof(double) * 12 * TetTile<T>::N + (HESS ? sizeof(T) * TET_W * TetTile<T>::N : 0) + TetTile<T>::N;
}

// Launch of the tiled tetrahedron kernel: one tile of N tetrahedra per CTA
// pass, grid-stride over the tiles.  The dynamic shared memory exceeds the
// 48 KB default, so the limit is raised once per instantiation.
template <class T, bool HESS>
void launchTet(Ctx& c, double dt2, T* elemH) {
    constexpr int N = TetTile<T>::N;
    constexpr size_t smem = tetSmemBytes<T, HESS>();
    static bool attr = false;
    if (!attr) {
        CIPC_CUDA(cudaFuncSetAttribute(tetKernel<T, HESS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    const int tiles = (c.nt + N - 1) / N;
    launch(tetKernel<T, HESS>, std::max(1, std::min(tiles, 148 * 16)), N, smem, c.s, c.nt, c.tets, c.x, c.DmInv, c.vol, c.tetMu, c.tetLam,
           c.btype, dt2, c.elemG, elemH);
}

// Baraff-Witkin membrane, project_baraffwitkint_H_3D + computePEPF_baraffwitkin_double.
template <class T>
__global__ void triKernel(int nf, const int* tris, const double* x, const double* DmInv2, const double* area, const int* btype,
                          double stretchS, double shearS, double sr, double dt2, double* elemG, T* elemH, int blockBase,
                          int gradBase) {
    CIPC_KERNEL_LOOP(i, nf) {
        int v[3] = {tris[3 * i], tris[3 * i + 1], tris[3 * i + 2]};
        const double* D = DmInv2 + 4 * i;
        d3 x0 = ld3(x, v[0]);
        d3 a1 = ld3(x, v[1]) - x0, a2 = ld3(x, v[2]) - x0;
        d3 f0 = D[0] * a1 + D[2] * a2;  // column 0: D(0,0), D(1,0)
        d3 f1 = D[1] * a1 + D[3] * a2;  // column 1: D(0,1), D(1,1)
        double Gt[3][2] = {{-(D[0] + D[2]), -(D[1] + D[3])}, {D[0], D[1]}, {D[2], D[3]}};
        double I6 = dot(f0, f1), I5u = dot(f0, f0), I5v = dot(f1, f1);
        double uc = 1.0 - 1 / sqrt(I5u), vc = 1.0 - 1 / sqrt(I5v);
        if (I5u > 1) uc += 1.5 * sr * (sqrt(I5u) + 1 / sqrt(I5u) - 2);
        if (I5v > 1) vc += 1.5 * sr * (sqrt(I5v) + 1 / sqrt(I5v) - 2);
        double P[3][2];
        for (int k = 0; k < 3; ++k) {
            P[k][0] = stretchS * (uc * 2. * comp(f0, k)) + shearS * (2 * I6 * comp(f1, k));
            P[k][1] = stretchS * (vc * 2. * comp(f1, k)) + shearS * (2 * I6 * comp(f0, k));
        }
        double sc = dt2 * area[i];
        for (int a = 0; a < 3; ++a)
            for (int r = 0; r < 3; ++r) elemG[3 * (gradBase + 3 * i + a) + r] = sc * (P[r][0] * Gt[a][0] + P[r][1] * Gt[a][1]);
        // 6x6 Hessian in T
        T H[6][6];
        for (int p = 0; p < 6; ++p) for (int q = 0; q < 6; ++q) H[p][q] = T(0);
        {
            T su = sqrt(T(I5u)), sv = sqrt(T(I5v));
            T s = T(sr);
            if (su > T(1)) { T d = T(2) * (((su - T(1)) * (T(3) * su * s - T(3) * s + T(2))) / (T(2) * su)); H[0][0] = H[1][1] = H[2][2] = d; }
            if (sv > T(1)) { T d = T(2) * (((sv - T(1)) * (T(3) * sv * s - T(3) * s + T(2))) / (T(2) * sv)); H[3][3] = H[4][4] = H[5][5] = d; }
            T nu = sqrt(T(I5u)), nvv = sqrt(T(I5v));
            T fu[3] = {T(f0.x) / nu, T(f0.y) / nu, T(f0.z) / nu}, fv[3] = {T(f1.x) / nvv, T(f1.y) / nvv, T(f1.z) / nvv};
            T uC = (su > T(1)) ? (T(3) * T(I5u) * s - T(3) * s + T(2)) / sqrt(T(I5u)) : T(2);
            T vC = (sv > T(1)) ? (T(3) * T(I5v) * s - T(3) * s + T(2)) / sqrt(T(I5v)) : T(2);
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) { H[p][q] += uC * (fu[p] * fu[q]); H[3 + p][3 + q] += vC * (fv[p] * fv[q]); }
            for (int p = 0; p < 6; ++p) for (int q = 0; q < 6; ++q) H[p][q] *= T(stretchS);
        }
        {
            T sign = I6 >= 0 ? T(1) : T(-1);
            T g[6] = {T(f1.x), T(f1.y), T(f1.z), T(f0.x), T(f0.y), T(f0.z)};
            T Hg[6] = {g[3], g[4], g[5], g[0], g[1], g[2]};
            T I2 = T(I5u + I5v);
            T i6 = T(I6);
            T l0 = T(0.5) * (I2 + sqrt(I2 * I2 + T(12) * i6 * i6));
            T q0[6];
            T qn = T(0);
            for (int k = 0; k < 6; ++k) { q0[k] = i6 * Hg[k] + l0 * g[k]; qn += q0[k] * q0[k]; }
            qn = sqrt(qn);
            if (qn > T(0)) for (int k = 0; k < 6; ++k) q0[k] /= qn;
            // T = 0.5 (I + sign * Hs), Hs swaps the two 3-blocks
            T Tq[6];
            for (int k = 0; k < 6; ++k) Tq[k] = T(0.5) * (q0[k] + sign * q0[(k + 3) % 6]);
            T nTq = T(0);
            for (int k = 0; k < 6; ++k) nTq += Tq[k] * Tq[k];
            T ai6 = fabs(i6);
            for (int p = 0; p < 6; ++p)
                for (int q = 0; q < 6; ++q) {
                    T Tpq = T(0.5) * ((p == q ? T(1) : T(0)) + ((q == (p + 3) % 6) ? sign : T(0)));
                    H[p][q] += T(shearS) * T(2) * (ai6 * (Tpq - (Tq[p] * Tq[q]) / nTq) + l0 * (q0[p] * q0[q]));
                }
        }
        T* out = elemH + (size_t)9 * (blockBase + 6 * i);
        T scT = T(sc);
        bool fr[3] = {btype[v[0]] == 0, btype[v[1]] == 0, btype[v[2]] == 0};
        for (int a = 0; a < 3; ++a)
            for (int b = 0; b <= a; ++b) {
                T* blk = out + 9 * lowerIdx(a, b);
                for (int r = 0; r < 3; ++r)
                    for (int q = 0; q < 3; ++q) {
                        T s = T(0);
                        for (int c = 0; c < 2; ++c)
                            for (int d = 0; d < 2; ++d) s += T(Gt[a][c]) * H[3 * c + r][3 * d + q] * T(Gt[b][d]);
                        blk[3 * r + q] = (fr[a] && fr[b]) ? scT * s : T(0);
                    }
            }
    }
}

template <class T>
__global__ void bendKernel(int nb, const int* bv, const double* Q, const double* x, const int* btype, double bs, double* elemG,
                           T* elemH, int blockBase, int gradBase) {
    CIPC_KERNEL_LOOP(i, nb) {
        int v[4];
        for (int a = 0; a < 4; ++a) v[a] = bv[4 * i + a];
        const double* q = Q + 16 * i;
        d3 p[4];
        for (int a = 0; a < 4; ++a) p[a] = ld3(x, v[a]);
        for (int a = 0; a < 4; ++a) {
            d3 s = mk(0, 0, 0);
            for (int b = 0; b < 4; ++b) s = s + q[4 * a + b] * p[b];
            st3(elemG, gradBase + 4 * i + a, bs * s);
        }
        T* out = elemH + (size_t)9 * (blockBase + 10 * i);
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b <= a; ++b) {
                T* blk = out + 9 * lowerIdx(a, b);
                bool ok = btype[v[a]] == 0 && btype[v[b]] == 0;
                T d = ok ? T(bs * q[4 * a + b]) : T(0);
                for (int e = 0; e < 9; ++e) blk[e] = (e % 4 == 0) ? d : T(0);
            }
    }
}

// Dihedral-angle bending (hingeBendingGradientAndHessian + makePD,
// HingeBending.cpp:88-106, IPCSolver.cpp:238-267), one warp per hinge as the
// contact kernels: every lane forms the angle's gradient in closed form,
// lanes 0-11 one column each of its Hessian, the warp projects the 12 x 12
// Hessian onto the PSD cone in shared memory, and the 10 lower 3 x 3 blocks
// go to the hinge's element slots as bendKernel writes them (blocks touching
// a constrained vertex zeroed).  scale = plateRigidity * dt^2.
constexpr int HINGE_WPB = 4;
template <class T>
__global__ void __launch_bounds__(HINGE_WPB * 32) hingeKernel(int nb, const int* bv, const double* hw, const double* th0, const double* x,
                                                              const int* btype, double k, double dt2, double* elemG, T* elemH, int blockBase,
                                                              int gradBase, int* status) {
    __shared__ JacobiSmem sm[HINGE_WPB];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    JacobiSmem& S = sm[w];
    for (int i = blockIdx.x * HINGE_WPB + w; i < nb; i += gridDim.x * HINGE_WPB) {
        int v[4];
        double xs[12];
        for (int a = 0; a < 4; ++a) {
            v[a] = bv[4 * i + a];
            for (int q = 0; q < 3; ++q) xs[3 * a + q] = x[3 * (size_t)v[a] + q];
        }
        const double s = k * hw[i];
        const double d = remainder(hinge::angle(xs) - th0[i], 6.28318530717958647692);
        hinge::Vec3<double> gr[4];
        hinge::angleGrad(hinge::Vec3<double>{xs[0], xs[1], xs[2]}, hinge::Vec3<double>{xs[3], xs[4], xs[5]},
                         hinge::Vec3<double>{xs[6], xs[7], xs[8]}, hinge::Vec3<double>{xs[9], xs[10], xs[11]}, gr);
        double tg[12];
        for (int a = 0; a < 4; ++a) { tg[3 * a] = gr[a].x; tg[3 * a + 1] = gr[a].y; tg[3 * a + 2] = gr[a].z; }
        if (!isfinite(d) && lane == 0) raiseStatus(status, CIPC_ST_NONFINITE);
        if (lane < 12) {
            double col[12];
            hinge::angleHessColumn(xs, lane, col);
            double tl = tg[0];
            for (int r = 1; r < 12; ++r) tl = r == lane ? tg[r] : tl;
            for (int r = 0; r < 12; ++r) S.A[12 * r + lane] = s * (tg[r] * tl + d * col[r]);
        }
        if (lane < 4) st3(elemG, gradBase + 4 * i + lane, mk(dt2 * s * d * tg[3 * lane], dt2 * s * d * tg[3 * lane + 1], dt2 * s * d * tg[3 * lane + 2]));
        __syncwarp();
        if (!warpPsdProject(S, 12, lane) && lane == 0) raiseStatus(status, CIPC_ST_JACOBI_CAP);
        T* out = elemH + (size_t)9 * (blockBase + 10 * i);
        for (int e = lane; e < 90; e += 32) {
            const int blk = e / 9, ent = e % 9;
            const int a = blk >= 6 ? 3 : (blk >= 3 ? 2 : (blk >= 1 ? 1 : 0));
            const int b = blk - a * (a + 1) / 2;  // lowerIdx(a, b) = blk
            const bool ok = btype[v[a]] == 0 && btype[v[b]] == 0;
            out[e] = ok ? T(dt2 * S.A[12 * (3 * a + ent / 3) + 3 * b + ent % 3]) : T(0);
        }
        __syncwarp();
    }
}

// w * remainder(theta - theta0, 2 pi)^2 per hinge (the energy sums it with 0.5 k)
__global__ void hingeEnergyKernel(int nb, const int* bv, const double* hw, const double* th0, const double* x, double* out) {
    CIPC_KERNEL_LOOP(i, nb) {
        double xs[12];
        for (int a = 0; a < 4; ++a)
            for (int q = 0; q < 3; ++q) xs[3 * a + q] = x[3 * (size_t)bv[4 * i + a] + q];
        const double d = remainder(hinge::angle(xs) - th0[i], 6.28318530717958647692);
        out[i] = hw[i] * d * d;
    }
}

template <class T>
__global__ void slotReduceKernel(int nnzb, const int* hcPtr, const int* hcIdx, const T* elemH, T* val) {
    CIPC_KERNEL_LOOP(sl, nnzb) {
        T acc[9];
        for (int e = 0; e < 9; ++e) acc[e] = T(0);
        for (int k = hcPtr[sl]; k < hcPtr[sl + 1]; ++k) {
            int code = hcIdx[k];
            bool tr = code < 0;
            int b = tr ? ~code : code;
            const T* blk = elemH + (size_t)9 * b;
            if (tr) {
                for (int r = 0; r < 3; ++r) for (int q = 0; q < 3; ++q) acc[3 * r + q] += blk[3 * q + r];
            } else {
                for (int e = 0; e < 9; ++e) acc[e] += blk[e];
            }
        }
        for (int e = 0; e < 9; ++e) val[(size_t)9 * sl + e] = acc[e];
    }
}

// Per-vertex gradient: vertex terms plus the vertex's element and contact
// contributions.  GG lanes share a vertex: each sums a fixed stride of the
// contribution list, then the group adds the lanes' sums in a fixed order
// (deterministic).
constexpr int GG = 8;
__global__ void gatherGradKernel(int nv, const double* vtxGrad, const int* gcPtr, const int* gcIdx, const double* elemG,
                                 const int* dynStart, const int* dynEnd, const int* dynIdx, const double* dynVal, double* grad) {
    const int lane = threadIdx.x % GG;
    const int stride = gridDim.x * blockDim.x / GG;
    // the loop bound is the warp's first vertex, so that all 32 lanes take
    // part in every shuffle (blockDim is a multiple of 32)
    const int warpFirst = (blockIdx.x * blockDim.x + (threadIdx.x & ~31)) / GG;
    for (int w0 = warpFirst; w0 < nv; w0 += stride) {
        const int v = w0 + (threadIdx.x & 31) / GG;
        const bool active = v < nv;
        double g[3] = {0.0, 0.0, 0.0};
        if (active) for (int k = gcPtr[v] + lane; k < gcPtr[v + 1]; k += GG) {
            const int e = gcIdx[k];
            g[0] += elemG[3 * e]; g[1] += elemG[3 * e + 1]; g[2] += elemG[3 * e + 2];
        }
        if (dynStart && active) {
            for (int k = dynStart[v] + lane; k < dynEnd[v]; k += GG) {
                const int e = dynIdx[k];
                g[0] += dynVal[3 * e]; g[1] += dynVal[3 * e + 1]; g[2] += dynVal[3 * e + 2];
            }
        }
#pragma unroll
        for (int o = GG / 2; o > 0; o >>= 1)
#pragma unroll
            for (int q = 0; q < 3; ++q) g[q] += __shfl_down_sync(0xffffffffu, g[q], o, GG);
        if (active && lane == 0) {
            grad[3 * v] = vtxGrad[3 * v] + g[0];
            grad[3 * v + 1] = vtxGrad[3 * v + 1] + g[1];
            grad[3 * v + 2] = vtxGrad[3 * v + 2] + g[2];
        }
    }
}

// ---- energies ----
__global__ void tetEnergyKernel(int nt, const int* tets, const double* x, const double* DmInv, const double* vol, const double* tmu,
                                const double* tlam, double* out) {
    CIPC_KERNEL_LOOP(i, nt) {
        const double* Di = DmInv + 9 * i;
        d3 x0 = ld3(x, tets[4 * i]);
        d3 e1 = ld3(x, tets[4 * i + 1]) - x0, e2 = ld3(x, tets[4 * i + 2]) - x0, e3 = ld3(x, tets[4 * i + 3]) - x0;
        double F[3][3];
        double Ds[3][3] = {{e1.x, e2.x, e3.x}, {e1.y, e2.y, e3.y}, {e1.z, e2.z, e3.z}};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) F[r][c] = Ds[r][0] * Di[c] + Ds[r][1] * Di[3 + c] + Ds[r][2] * Di[6 + c];
        double I2 = 0;
        for (int r = 0; r < 3; ++r) for (int c = 0; c < 3; ++c) I2 += F[r][c] * F[r][c];
        double J = F[0][0] * (F[1][1] * F[2][2] - F[1][2] * F[2][1]) - F[0][1] * (F[1][0] * F[2][2] - F[1][2] * F[2][0]) +
                   F[0][2] * (F[1][0] * F[2][1] - F[1][1] * F[2][0]);
        double u = tmu[i], r = tlam[i];
        double t = J - 1 - 3 * u / 4 / r;
        out[i] = (0.5 * u * (I2 - 3) + 0.5 * r * t * t - 0.5 * u * log(I2 + 1)) * vol[i];
    }
}

__global__ void triEnergyKernel(int nf, const int* tris, const double* x, const double* DmInv2, const double* area, double stretchS,
                                double shearS, double sr, double* out) {
    CIPC_KERNEL_LOOP(i, nf) {
        const double* D = DmInv2 + 4 * i;
        d3 x0 = ld3(x, tris[3 * i]);
        d3 a1 = ld3(x, tris[3 * i + 1]) - x0, a2 = ld3(x, tris[3 * i + 2]) - x0;
        d3 f0 = D[0] * a1 + D[2] * a2, f1 = D[1] * a1 + D[3] * a2;
        double I6 = dot(f0, f1);
        double u = sqrt(dot(f0, f0)), v = sqrt(dot(f1, f1));
        double uc = u <= 1 ? 0 : 1, vc = v <= 1 ? 0 : 1;
        double st = (u - 1) * (u - 1) + uc * sr * (u - 1) * (u - 1) * (u - 1) + (v - 1) * (v - 1) + vc * sr * (v - 1) * (v - 1) * (v - 1);
        out[i] = (stretchS * st + shearS * I6 * I6) * area[i];
    }
}

__global__ void bendEnergyKernel(int nb, const int* bv, const double* Q, const double* x, double* out) {
    CIPC_KERNEL_LOOP(i, nb) {
        const double* q = Q + 16 * i;
        d3 p[4];
        for (int a = 0; a < 4; ++a) p[a] = ld3(x, bv[4 * i + a]);
        double s = 0;
        for (int a = 0; a < 4; ++a) for (int b = 0; b < 4; ++b) s += q[4 * a + b] * dot(p[a], p[b]);
        out[i] = s;
    }
}

__global__ void inertiaEnergyKernel(int nv, const double* x, const double* xt, const double* vp, const double* mass, double drag, double* out) {
    CIPC_KERNEL_LOOP(v, nv) {
        d3 a = ld3(x, v) - ld3(xt, v), b = ld3(x, v) - ld3(vp, v);
        out[v] = sqn(a) * mass[v] / 2.0 + sqn(b) * drag * mass[v] / 2.0;
    }
}

__global__ void softEnergyKernel(int ns, const int* idx, const double* target, double w, const double* x, double* out) {
    CIPC_KERNEL_LOOP(k, ns) {
        int v = idx[k];
        d3 d = ld3(x, v) - ld3(target, k);
        out[k] = 0.5 * w * sqn(d);
    }
}

}  // namespace

void buildStaticPattern(Ctx& c, const std::vector<int>& tets, const std::vector<int>& tris, const std::vector<int>& bendV) {
    int nv = c.nv;
    struct Contrib { long long key; int code; };
    std::vector<Contrib> hc;
    std::vector<std::pair<int, int>> gc;  // (vertex, element gradient index)
    hc.reserve((size_t)16 * c.nt + 9 * (size_t)c.nf + 16 * (size_t)c.nb);
    int blockBase = 0, gradBase = 0;
    auto addElem = [&](const int* vs, int k, int bBase, int gBase) {
        for (int a = 0; a < k; ++a) {
            gc.push_back({vs[a], gBase + a});
            for (int b = 0; b < k; ++b) {
                long long key = (long long)vs[a] * nv + vs[b];
                int code = a >= b ? (bBase + lowerIdx(a, b)) : ~(bBase + lowerIdx(b, a));
                hc.push_back({key, code});
            }
        }
    };
    for (int i = 0; i < c.nt; ++i) addElem(&tets[4 * i], 4, blockBase + 10 * i, gradBase + 4 * i);
    blockBase += 10 * c.nt; gradBase += 4 * c.nt;
    for (int i = 0; i < c.nf; ++i) addElem(&tris[3 * i], 3, blockBase + 6 * i, gradBase + 3 * i);
    blockBase += 6 * c.nf; gradBase += 3 * c.nf;
    for (int i = 0; i < c.nb; ++i) addElem(&bendV[4 * i], 4, blockBase + 10 * i, gradBase + 4 * i);
    blockBase += 10 * c.nb; gradBase += 4 * c.nb;
    // every vertex owns a diagonal slot even without elements
    for (int v = 0; v < nv; ++v) hc.push_back({(long long)v * nv + v, INT32_MIN});
    c.nElemBlocks = blockBase;
    c.nElemGrad = gradBase;
    std::stable_sort(hc.begin(), hc.end(), [](const Contrib& a, const Contrib& b) { return a.key < b.key; });
    std::vector<int> rowPtr(nv + 1, 0), col, hcPtr, hcIdx, diag(nv, -1);
    hcPtr.push_back(0);
    for (size_t k = 0; k < hc.size();) {
        size_t e = k;
        while (e < hc.size() && hc[e].key == hc[k].key) {
            if (hc[e].code != INT32_MIN) hcIdx.push_back(hc[e].code);
            ++e;
        }
        int r = (int)(hc[k].key / nv), cl = (int)(hc[k].key % nv);
        if (r == cl) diag[r] = (int)col.size();
        col.push_back(cl);
        rowPtr[r + 1]++;
        hcPtr.push_back((int)hcIdx.size());
        k = e;
    }
    for (int r = 0; r < nv; ++r) rowPtr[r + 1] += rowPtr[r];
    c.nnzb = (int)col.size();
    std::stable_sort(gc.begin(), gc.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
    std::vector<int> gcPtr(nv + 1, 0), gcIdx(gc.size());
    for (size_t k = 0; k < gc.size(); ++k) { gcPtr[gc[k].first + 1]++; gcIdx[k] = gc[k].second; }
    for (int v = 0; v < nv; ++v) gcPtr[v + 1] += gcPtr[v];
    auto up = [&](DBuf<int>& d, const std::vector<int>& h) {
        d.reserve(std::max<size_t>(h.size(), 1));
        if (!h.empty()) CIPC_CUDA(cudaMemcpy(d.p, h.data(), h.size() * sizeof(int), cudaMemcpyHostToDevice));
    };
    up(c.rowPtr, rowPtr); up(c.colIdx, col); up(c.diagSlot, diag); up(c.hcPtr, hcPtr); up(c.hcIdx, hcIdx);
    c.hRowPtr = rowPtr;
    up(c.gcPtr, gcPtr); up(c.gcIdx, gcIdx);
    c.valD.reserve((size_t)9 * c.nnzb);
    c.valF.reserve((size_t)9 * c.nnzb);
    c.elemG.reserve((size_t)3 * std::max(1, c.nElemGrad));
    c.elemHD.reserve((size_t)9 * std::max(1, c.nElemBlocks));
    c.elemHF.reserve((size_t)9 * std::max(1, c.nElemBlocks));
    c.vtxGrad.reserve((size_t)3 * nv);
    c.diagExtra.reserve((size_t)9 * nv);
}

template <class T>
static void assembleElasticT(Ctx& c, T* elemH, T* val) {
    const SimParams& P = c.P;
    double dt2 = P.dt * P.dt;
    if (c.nt) {
        profBegin(c, PROF_TET);
        launchTet<T, true>(c, dt2, elemH);
        profEnd(c, PROF_TET);
    }
    profBegin(c, PROF_TRI);
    int bBase = 10 * c.nt, gBase = 4 * c.nt;
    if (c.nf)
        launch(triKernel<T>, blocksFor(c.nf), TB, 0, c.s, c.nf, c.tris, c.x, c.DmInv2, c.area, c.btype, P.stretchS, P.shearS, P.strainRate, dt2,
                                                       c.elemG, elemH, bBase, gBase);
    profEnd(c, PROF_TRI);
    bBase += 6 * c.nf; gBase += 3 * c.nf;
    if (c.nb && c.hinge)
        launch(hingeKernel<T>, std::max(1, std::min((c.nb + HINGE_WPB - 1) / HINGE_WPB, 148 * 64)), HINGE_WPB * 32, 0, c.s, c.nb, c.bendV,
               (const double*)c.hingeW, (const double*)c.hingeTh0, c.x, c.btype, P.plateRigidity, dt2, c.elemG, elemH, bBase, gBase, c.status.p);
    else if (c.nb)
        launch(bendKernel<T>, blocksFor(c.nb), TB, 0, c.s, c.nb, c.bendV, c.bendQ, c.x, c.btype, P.plateRigidity * dt2, c.elemG, elemH, bBase, gBase);
    profBegin(c, PROF_SLOT);
    launch(slotReduceKernel<T>, blocksFor(c.nnzb), TB, 0, c.s, c.nnzb, c.hcPtr, c.hcIdx, elemH, val);
    profEnd(c, PROF_SLOT);
}

void assembleElastic(Ctx& c) {
    launch(vertexInitKernel, blocksFor(c.nv), TB, 0, c.s, c.nv, c.x, c.xt, c.vp, c.mass, c.P.drag, c.vtxGrad, c.diagExtra);
    int ns = (int)c.hSoftIdx.size();
    if (ns) launch(softKernel, blocksFor(ns), TB, 0, c.s, ns, c.softIdx, c.softTarget, c.P.softW, c.x, c.vtxGrad, c.diagExtra);
    if (c.mixed) assembleElasticT<float>(c, c.elemHF, c.valF);
    else assembleElasticT<double>(c, c.elemHD, c.valD);
    CIPC_CUDA(cudaGetLastError());
}

void gatherGradient(Ctx& c) {
    bool dyn = c.nDynG > 0;
    launch(gatherGradKernel, blocksFor(GG * c.nv), TB, 0, c.s, c.nv, c.vtxGrad, c.gcPtr, c.gcIdx, c.elemG, dyn ? c.dynGStart.p : nullptr,
                                                      dyn ? c.dynGEnd.p : nullptr, dyn ? c.dynGIdx.p : nullptr, c.dynGVal, c.grad);
    CIPC_CUDA(cudaGetLastError());
}

// The elastic energy's term sums into device slots slot0 .. slot0 + 4 (no
// host synchronisation); elasticEnergyCombine adds them in a fixed order.
void elasticEnergySums(Ctx& c, int slot0) {
    const SimParams& P = c.P;
    int n = std::max(std::max(c.nt, c.nf), std::max(c.nb, c.nv));
    c.energyBuf.reserve(std::max(n, 1));
    const int ns = (int)c.hSoftIdx.size();
    if (c.nt) {
        launch(tetEnergyKernel, blocksFor(c.nt), TB, 0, c.s, c.nt, c.tets, c.x, c.DmInv, c.vol, c.tetMu, c.tetLam, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nt, slot0 + 0);
    }
    if (c.nf) {
        launch(triEnergyKernel, blocksFor(c.nf), TB, 0, c.s, c.nf, c.tris, c.x, c.DmInv2, c.area, P.stretchS, P.shearS, P.strainRate, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nf, slot0 + 1);
    }
    if (c.nb) {
        if (c.hinge)
            launch(hingeEnergyKernel, blocksFor(c.nb), TB, 0, c.s, c.nb, c.bendV, (const double*)c.hingeW, (const double*)c.hingeTh0, c.x, c.energyBuf);
        else
            launch(bendEnergyKernel, blocksFor(c.nb), TB, 0, c.s, c.nb, c.bendV, c.bendQ, c.x, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nb, slot0 + 2);
    }
    launch(inertiaEnergyKernel, blocksFor(c.nv), TB, 0, c.s, c.nv, c.x, c.xt, c.vp, c.mass, P.drag, c.energyBuf);
    deviceSumTo(c, c.energyBuf, c.nv, slot0 + 3);
    if (ns) {
        launch(softEnergyKernel, blocksFor(ns), TB, 0, c.s, ns, c.softIdx, c.softTarget, P.softW, c.x, c.energyBuf);
        deviceSumTo(c, c.energyBuf, ns, slot0 + 4);
    }
}

double elasticEnergyCombine(const Ctx& c, const double* h) {
    const SimParams& P = c.P;
    double E = 0;
    if (c.nt) E += h[0];
    if (c.nf) E += h[1];
    if (c.nb) E += 0.5 * P.plateRigidity * h[2];
    E *= P.dt * P.dt;
    E += h[3];
    if (!c.hSoftIdx.empty()) E += h[4];
    return E;
}

double elasticEnergy(Ctx& c) {
    elasticEnergySums(c, 0);
    double h[5];
    fetchSums(c, h, 5);
    return elasticEnergyCombine(c, h);
}

namespace {
__global__ void gradEKernel(int nv, const double* x, const double* xt, const double* mass, const int* gcPtr, const int* gcIdx,
                            const double* elemG, int ntGrad, double* gE) {
    CIPC_KERNEL_LOOP(v, nv) {
        double g[3];
        for (int k = 0; k < 3; ++k) g[k] = mass[v] * (x[3 * v + k] - xt[3 * v + k]);
        for (int k = gcPtr[v]; k < gcPtr[v + 1]; ++k) {
            int e = gcIdx[k];
            if (e >= ntGrad) continue;  // tetrahedra only
            g[0] += elemG[3 * e]; g[1] += elemG[3 * e + 1]; g[2] += elemG[3 * e + 2];
        }
        gE[3 * v] = g[0]; gE[3 * v + 1] = g[1]; gE[3 * v + 2] = g[2];
    }
}
}  // namespace

// The tetrahedra's elastic gradients alone (elemG), for the kappa
// initialisation: no Hessian work.
void tetGradient(Ctx& c) {
    if (c.nt) launchTet<float, false>(c, c.P.dt * c.P.dt, (float*)nullptr);
    CIPC_CUDA(cudaGetLastError());
}

// computeEGradient (IPCSolver.cpp:72-106): inertia (no drag) plus the
// tetrahedral elastic gradient.  Requires elemG from assembleElastic or
// tetGradient at x.
void initKappaGradE(Ctx& c, double* gE) {
    launch(gradEKernel, blocksFor(c.nv), TB, 0, c.s, c.nv, c.x, c.xt, c.mass, c.gcPtr, c.gcIdx, c.elemG, 4 * c.nt, gE);
    CIPC_CUDA(cudaGetLastError());
}

}  // namespace cipc
