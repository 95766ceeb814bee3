// Device-side building blocks shared by the IPC kernels: small vector math,
// the status word, deterministic block reductions, the warp-parallel Jacobi
// PSD projection of contact Hessian blocks and the rotation-aware 3x3 SVD.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define CIPC_HD __host__ __device__ __forceinline__

// Status bits written by kernels; the host reads them after each stage.
enum CipcStatusBits {
    CIPC_ST_NONFINITE = 1,
    CIPC_ST_STACK_OVERFLOW = 2,
    CIPC_ST_CAPACITY = 4,
    CIPC_ST_CCD_CAP = 8,
    CIPC_ST_JACOBI_CAP = 16,
    CIPC_ST_TC_TIMEOUT = 32,
};

template <class T>
CIPC_HD T cipc_pow_int(T x, int n) {
    return n == 2 ? x * x : (n == -2 ? T(1) / (x * x) : x);
}

struct d3 {
    double x, y, z;
};
CIPC_HD d3 mk(double a, double b, double c) { return d3{a, b, c}; }
CIPC_HD d3 operator+(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
CIPC_HD d3 operator-(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
CIPC_HD d3 operator-(d3 a) { return mk(-a.x, -a.y, -a.z); }
CIPC_HD d3 operator*(double s, d3 a) { return mk(s * a.x, s * a.y, s * a.z); }
CIPC_HD d3 operator/(d3 a, double s) { return mk(a.x / s, a.y / s, a.z / s); }
CIPC_HD double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
CIPC_HD d3 cross(d3 a, d3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
CIPC_HD double sqn(d3 a) { return dot(a, a); }
CIPC_HD double comp(d3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

__device__ __forceinline__ d3 ld3(const double* p, int i) { return mk(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }
__device__ __forceinline__ void st3(double* p, int i, d3 v) { p[3 * i] = v.x; p[3 * i + 1] = v.y; p[3 * i + 2] = v.z; }

__device__ __forceinline__ void raiseStatus(int* status, int bit) { atomicOr(status, bit); }

// Grid-stride helper.
#define CIPC_KERNEL_LOOP(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += blockDim.x * gridDim.x)

// ---------------------------------------------------------------------------
// Block reductions (fixed order for a fixed launch shape => deterministic)
// ---------------------------------------------------------------------------
template <class T, class Op>
__device__ __forceinline__ T warpReduce(T v, Op op) {
    for (int o = 16; o > 0; o >>= 1) v = op(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
struct AddOp { template <class T> __device__ T operator()(T a, T b) const { return a + b; } };
struct MinOp { template <class T> __device__ T operator()(T a, T b) const { return a < b ? a : b; } };
struct MaxOp { template <class T> __device__ T operator()(T a, T b) const { return a > b ? a : b; } };

// Reduces one value per thread to one value per block (result valid in thread 0).
template <class T, class Op>
__device__ T blockReduce(T v, Op op, T identity) {
    __shared__ T sh[32];
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    v = warpReduce(v, op);
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    int nw = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nw) ? sh[threadIdx.x] : identity;
    if (w == 0) v = warpReduce(v, op);
    return v;
}

// ---------------------------------------------------------------------------
// Warp-parallel cyclic Jacobi for symmetric n x n (n even, n <= 12) blocks.
// One warp owns the matrix in shared memory; each round rotates n/2 disjoint
// index pairs (round-robin schedule), so every entry update is independent.
// ---------------------------------------------------------------------------
struct JacobiSmem {
    double A[144], B[144], V[144], W[144], O[144];
    double cs[12], sn[12];
    int partner[12];
    double red;
};

__device__ __forceinline__ void rrPair(int n, int round, int k, int& p, int& q) {
    int m = n - 1;
    if (k == 0) { p = m; q = round; }
    else { p = (round + k) % m; q = (round - k + m) % m; }
    if (p > q) { int t = p; p = q; q = t; }
}

// Projects the symmetric matrix in S.A (row-major, leading dim n) onto the PSD
// cone following makePD: unchanged if already PSD, else negative eigenvalues
// set to zero.  Result left in S.A.  Returns false if the sweep cap was hit.
__device__ inline bool warpPsdProject(JacobiSmem& S, int n, int lane) {
    int nn = n * n;
    for (int e = lane; e < nn; e += 32) {
        S.O[e] = S.A[e];
        S.V[e] = (e / n == e % n) ? 1.0 : 0.0;
    }
    __syncwarp();
    bool converged = false;
    for (int sweep = 0; sweep < 40 && !converged; ++sweep) {
        double off = 0, diag = 0;
        for (int e = lane; e < nn; e += 32) {
            int i = e / n, j = e % n;
            double a = S.A[e];
            if (i == j) diag += a * a; else off += a * a;
        }
        off = warpReduce(off, AddOp());
        diag = warpReduce(diag, AddOp());
        // relative off-diagonal Frobenius norm below ~1e-15: rounding keeps
        // re-creating off-diagonal terms of order eps * ||A||, so a tighter
        // bound need not be reachable
        if (off <= 1e-30 * diag || off == 0.0 || !(diag < 1e300)) { converged = true; break; }
        for (int round = 0; round < n - 1; ++round) {
            if (lane < n / 2) {
                int p, q;
                rrPair(n, round, lane, p, q);
                double apq = S.A[p * n + q];
                double c = 1.0, s = 0.0;
                if (apq != 0.0) {
                    double app = S.A[p * n + p], aqq = S.A[q * n + q];
                    double theta = (aqq - app) / (2.0 * apq);
                    double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(t * t + 1.0);
                    s = t * c;
                }
                // column p' = c col_p - s col_q ; column q' = s col_p + c col_q
                S.partner[p] = q; S.cs[p] = c; S.sn[p] = -s;
                S.partner[q] = p; S.cs[q] = c; S.sn[q] = s;
            }
            __syncwarp();
            for (int e = lane; e < nn; e += 32) {
                int i = e / n, j = e % n;
                int pi = S.partner[i], pj = S.partner[j];
                double ci = S.cs[i], si = S.sn[i], cj = S.cs[j], sj = S.sn[j];
                S.B[e] = ci * cj * S.A[i * n + j] + ci * sj * S.A[i * n + pj] + si * cj * S.A[pi * n + j] + si * sj * S.A[pi * n + pj];
                S.W[e] = cj * S.V[i * n + j] + sj * S.V[i * n + pj];
            }
            __syncwarp();
            for (int e = lane; e < nn; e += 32) { S.A[e] = S.B[e]; S.V[e] = S.W[e]; }
            __syncwarp();
        }
    }
    double mn = 1e300;
    for (int i = lane; i < n; i += 32) mn = fmin(mn, S.A[i * n + i]);
    mn = warpReduce(mn, MinOp());
    __syncwarp();
    if (mn >= 0.0) {
        for (int e = lane; e < nn; e += 32) S.A[e] = S.O[e];
        __syncwarp();
        return converged;
    }
    for (int k = lane; k < n; k += 32) S.cs[k] = fmax(S.A[k * n + k], 0.0);
    __syncwarp();
    for (int e = lane; e < nn; e += 32) {
        int i = e / n, j = e % n;
        double s = 0;
        for (int k = 0; k < n; ++k) s += S.cs[k] * S.V[i * n + k] * S.V[j * n + k];
        S.B[e] = s;
    }
    __syncwarp();
    for (int e = lane; e < nn; e += 32) S.A[e] = S.B[e];
    __syncwarp();
    return converged;
}

// ---------------------------------------------------------------------------
// The same projection for a 12 x 12 matrix held in registers by the 16 lanes
// of a half warp, by one-sided (Hestenes) Jacobi on B = A + mu I with
// mu = ||A||_F, which is positive semidefinite, so that its singular vectors
// are the eigenvectors of A.  Lane j holds column j of W (B V as the sweeps
// proceed) and of V (lanes 12-15 hold nothing).  A rotation of columns p, q
// needs only those two columns: each round takes the partner's columns by
// shuffle and updates its own, with no row operations, so the round's code
// is the same for every round and no register is indexed by the lane.  At
// the end lambda_j = w_j . v_j - mu.  Two matrices share a warp.  Smaller
// contacts are zero-padded to 12: a padded column never rotates (its inner
// product with every other column is zero) and adds the eigenvalue 0, so the
// projection of the leading block is unchanged.
// ---------------------------------------------------------------------------

// partner of index i in round r of the round-robin schedule over m + 1 indices
// (m odd): index m meets r, the others pair up as i + i' = 2r (mod m)
__host__ __device__ constexpr int rrPartner(int m, int r, int i) {
    return i == m ? r : (i == r ? m : (2 * r - i + m) % m);
}

// Projects the symmetric 12 x 12 matrix A (shared memory, row-major) onto
// the PSD cone as warpPsdProject does: A is left unchanged when no
// eigenvalue is negative, else replaced by V max(L, 0) V^T (formed from the
// upper triangle of each product, so exactly symmetric).  V (144 doubles)
// and lam (12) are shared scratch of the same half warp.  Every lane of the
// warp calls it; `active` is false on a half without a matrix.  A sweep
// rotates every pair whose columns are not orthogonal to 1e-15 (relative);
// the sweeps stop after one whose largest relative inner product was at most
// 1e-8 (quadratic convergence leaves about 1e-16).  Returns false if the
// sweep cap was hit.
__device__ inline bool halfWarpPsdProject12(double* A, double* V, double* lam, int hl, bool active) {
    constexpr int N = 12, M = N - 1;
    constexpr unsigned FULL = 0xffffffffu;
    const int j = hl;
    const bool own = active && j < N;
    double w[N], v[N];
    double fro = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        w[k] = own ? A[k * N + j] : 0.0;
        fro += w[k] * w[k];
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) fro += __shfl_xor_sync(FULL, fro, o, 16);
    const double mu = sqrt(fro);
#pragma unroll
    for (int k = 0; k < N; ++k) {
        if (k == j) w[k] += mu;
        v[k] = (k == j) ? 1.0 : 0.0;
    }
    // a zero or non-finite matrix is left as it is
    bool done = !active || !(mu > 0.0 && mu < 1e300);
    bool converged = done;
    for (int sweep = 0; sweep < 40; ++sweep) {
        if (__all_sync(FULL, done)) break;
        double mx = 0.0;
        for (int r = 0; r < M; ++r) {
            const int P = j < N ? rrPartner(M, r, j) : j;
            const bool lower = j < P;
            double wp[N];
            double gam = 0.0, nn = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                wp[k] = __shfl_sync(FULL, w[k], P, 16);
                gam += w[k] * wp[k];
                nn += w[k] * w[k];
            }
            const double np = __shfl_sync(FULL, nn, P, 16);
            // alpha = |w_p|^2, beta = |w_q|^2 for the pair p < q (both lanes
            // form the same gamma: the same products in the same order)
            const double al = lower ? nn : np, be = lower ? np : nn;
            double c = 1.0, s = 0.0;
            if (!done && P != j && gam != 0.0) {
                const double rel = fabs(gam) / (sqrt(al) * sqrt(be));
                mx = fmax(mx, rel);
                if (rel > 1e-15) {
                    const double z = (be - al) / (2.0 * gam);
                    const double t = (z >= 0 ? 1.0 : -1.0) / (fabs(z) + sqrt(1.0 + z * z));
                    c = 1.0 / sqrt(1.0 + t * t);
                    s = c * t;
                }
            }
            // w_p' = c w_p - s w_q, w_q' = s w_p + c w_q, and the same for V
            const double sj = lower ? -s : s;
#pragma unroll
            for (int k = 0; k < N; ++k) w[k] = c * w[k] + sj * wp[k];
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const double o = __shfl_sync(FULL, v[k], P, 16);
                v[k] = c * v[k] + sj * o;
            }
        }
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, o, 16));
        if (!done && mx <= 1e-8) { done = true; converged = true; }
    }
    double lj = 0.0;
#pragma unroll
    for (int k = 0; k < N; ++k) lj += w[k] * v[k];
    lj -= mu;
    double mn = own ? lj : 1e300;
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) mn = fmin(mn, __shfl_xor_sync(FULL, mn, o, 16));
    const bool project = active && converged && mn < 0.0 && mu < 1e300;
    if (project && j < N) {
        lam[j] = fmax(lj, 0.0);
#pragma unroll
        for (int k = 0; k < N; ++k) V[k * N + j] = v[k];
    }
    __syncwarp();
    if (project && j < N) {
        // column j of V max(L, 0) V^T; entry (i, j) from rows min(i, j) and max(i, j)
#pragma unroll
        for (int i = 0; i < N; ++i) {
            const int rl = i < j ? i : j, rh = i < j ? j : i;
            double acc = 0.0;
#pragma unroll
            for (int k = 0; k < N; ++k) acc += (lam[k] * V[rl * N + k]) * V[rh * N + k];
            A[i * N + j] = acc;
        }
    }
    __syncwarp();
    return converged;
}

// ---------------------------------------------------------------------------
// Rotation-aware SVD of a 3x3 matrix: F = U diag(s) V^T with U, V proper
// rotations and s[2] carrying the sign of det F.  V from a cyclic Jacobi
// eigen-solve of F^T F (eigenvalues sorted descending), U and s from a Givens
// QR of F V.
// ---------------------------------------------------------------------------
template <class T>
CIPC_HD void jacobiSym3(T S[3][3], T V[3][3]) {
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) V[i][j] = (i == j) ? T(1) : T(0);
    for (int sweep = 0; sweep < 20; ++sweep) {
        T off = S[0][1] * S[0][1] + S[0][2] * S[0][2] + S[1][2] * S[1][2];
        T dg = S[0][0] * S[0][0] + S[1][1] * S[1][1] + S[2][2] * S[2][2];
        if (off <= T(1e-34) * dg || off == T(0)) break;
#pragma unroll
        for (int pq = 0; pq < 3; ++pq) {
            int p = pq == 2 ? 1 : 0, q = pq == 0 ? 1 : 2;
            T apq = S[p][q];
            if (apq == T(0)) continue;
            T theta = (S[q][q] - S[p][p]) / (T(2) * apq);
            T t = (theta >= T(0) ? T(1) : T(-1)) / (fabs(theta) + sqrt(theta * theta + T(1)));
            T c = T(1) / sqrt(t * t + T(1)), s = t * c;
            for (int k = 0; k < 3; ++k) {
                T akp = S[k][p], akq = S[k][q];
                S[k][p] = c * akp - s * akq;
                S[k][q] = s * akp + c * akq;
            }
            for (int k = 0; k < 3; ++k) {
                T apk = S[p][k], aqk = S[q][k];
                S[p][k] = c * apk - s * aqk;
                S[q][k] = s * apk + c * aqk;
            }
            for (int k = 0; k < 3; ++k) {
                T vkp = V[k][p], vkq = V[k][q];
                V[k][p] = c * vkp - s * vkq;
                V[k][q] = s * vkp + c * vkq;
            }
        }
    }
}

template <class T>
CIPC_HD void svd3(const T F[3][3], T U[3][3], T s[3], T V[3][3]) {
    T S[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) S[i][j] = F[0][i] * F[0][j] + F[1][i] * F[1][j] + F[2][i] * F[2][j];
    jacobiSym3(S, V);
    T ev[3] = {S[0][0], S[1][1], S[2][2]};
    // sort descending with V columns
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 2 - a; ++b)
            if (ev[b] < ev[b + 1]) {
                T t = ev[b]; ev[b] = ev[b + 1]; ev[b + 1] = t;
                for (int k = 0; k < 3; ++k) { T u = V[k][b]; V[k][b] = V[k][b + 1]; V[k][b + 1] = u; }
            }
    T detV = V[0][0] * (V[1][1] * V[2][2] - V[1][2] * V[2][1]) - V[0][1] * (V[1][0] * V[2][2] - V[1][2] * V[2][0]) +
             V[0][2] * (V[1][0] * V[2][1] - V[1][1] * V[2][0]);
    if (detV < T(0)) for (int k = 0; k < 3; ++k) V[k][2] = -V[k][2];
    T R[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) R[i][j] = F[i][0] * V[0][j] + F[i][1] * V[1][j] + F[i][2] * V[2][j];
    T Q[3][3];
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) Q[i][j] = (i == j) ? T(1) : T(0);
#pragma unroll
    for (int g = 0; g < 3; ++g) {
        const int i = g == 0 ? 1 : 2, j = g == 2 ? 1 : 0;  // (1,0), (2,0), (2,1)
        T a = R[j][j], b = R[i][j];
        T r = sqrt(a * a + b * b);
        T c = T(1), sn = T(0);
        if (r > T(0)) { c = a / r; sn = b / r; }
        for (int k = 0; k < 3; ++k) {
            T rj = R[j][k], ri = R[i][k];
            R[j][k] = c * rj + sn * ri;
            R[i][k] = -sn * rj + c * ri;
        }
        // Q <- Q G^T so that F V = Q R holds
        for (int k = 0; k < 3; ++k) {
            T qj = Q[k][j], qi = Q[k][i];
            Q[k][j] = c * qj + sn * qi;
            Q[k][i] = -sn * qj + c * qi;
        }
    }
    for (int i = 0; i < 3; ++i) for (int j = 0; j < 3; ++j) U[i][j] = Q[i][j];
    s[0] = R[0][0]; s[1] = R[1][1]; s[2] = R[2][2];
}
