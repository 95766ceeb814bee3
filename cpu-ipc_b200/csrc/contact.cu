// Contact terms on the GPU: log-barrier (PP/PE/PT/EE), the mollified
// nearly-parallel edge-edge term, the ground barrier and lagged friction.
//
// Each self contact is handled by one half warp: lane 0 of the half
// evaluates the distance and gradient, each of the first 3 x points lanes one
// row of the distance Hessian, the half projects the (zero-padded) 12 x 12
// barrier Hessian onto the PSD cone with a register-resident parallel Jacobi
// sweep, then writes its gradient rows and all vertex-pair 3x3 blocks as
// keyed entries.  The nearly-parallel edge-edge term keeps one warp per
// contact and the shared-memory sweep.  The entries
// are radix-sorted by (vertex) and (row, col) and summed per segment, so the
// result is deterministic and needs no floating-point atomics.
//
// Reference: compute_g_dpt / compute_g_dee / compute_H_dpt / compute_H_dee,
// CPU IPC/ContactMechanics.cpp:2970-3080, 3466-3700; ground barrier
// IPCSolver.cpp:270-293; Friction::initialize/addGradient/addHessian/energy,
// CPU IPC/Friction.cpp:81-545; computeEnergy barrier part IPCSolver.cpp:398-451.
#include "cipc_internal.h"
#include "distance_derivs.cuh"
#include "geometry.cuh"

#include <cub/cub.cuh>

#include <algorithm>

namespace cipc {

namespace {

constexpr int TB = 128;
constexpr int WPB = 4;  // warps per block in the warp-per-contact kernels
inline int blocksFor(int n, int tb = TB) { return std::max(1, std::min((n + tb - 1) / tb, 148 * 32)); }
inline int warpBlocksFor(int n) { return std::max(1, std::min((n + WPB - 1) / WPB, 148 * 64)); }
inline int halfWarpBlocksFor(int n) { return std::max(1, std::min((n + 2 * WPB - 1) / (2 * WPB), 148 * 64)); }

constexpr int GSENT = 0x7fffffff;
constexpr uint64_t HSENT = 0xffffffffffffffffull;

__device__ __forceinline__ void barrierB(double d, double dHat, double& b) { b = -(d - dHat) * (d - dHat) * log(d / dHat); }
__device__ __forceinline__ void barrierG(double d, double dHat, double& g) {
    double t = d - dHat;
    g = t * log(d / dHat) * -2.0 - (t * t) / d;
}
__device__ __forceinline__ void barrierH(double d, double dHat, double& h) {
    double t = d - dHat;
    h = (log(d / dHat) * -2.0 - t * 4.0 / d) + 1.0 / (d * d) * (t * t);
}

// Decode an encoded contact: kind 0 PP, 1 PE, 2 PT, 3 EE; idx the vertices.
__device__ __forceinline__ int decode(const int* c, int idx[4]) {
    if (c[0] >= 0) { idx[0] = c[0]; idx[1] = c[1]; idx[2] = c[2]; idx[3] = c[3]; return 3; }
    idx[0] = -c[0] - 1; idx[1] = c[1];
    if (c[2] < 0) return 0;
    idx[2] = c[2];
    if (c[3] < 0) return 1;
    idx[3] = c[3];
    return 2;
}
__device__ __forceinline__ int npts(int kind) { return kind == 0 ? 2 : (kind == 1 ? 3 : 4); }

__device__ __forceinline__ double distVal(int kind, const d3* p) {
    switch (kind) {
    case 0: return dPP(p[0], p[1]);
    case 1: return dPE(p[0], p[1], p[2]);
    case 2: return dPT(p[0], p[1], p[2], p[3]);
    default: return dEE(p[0], p[1], p[2], p[3]);
    }
}

// Gradient and (optionally) Hessian of the squared distance of a contact kind.
__device__ void distDerivs(int kind, const d3* p, double* g, double* H) {
    double v[12];
    int np = npts(kind);
    for (int k = 0; k < np; ++k) { v[3 * k] = p[k].x; v[3 * k + 1] = p[k].y; v[3 * k + 2] = p[k].z; }
    switch (kind) {
    case 0: {
        for (int k = 0; k < 3; ++k) { g[k] = 2.0 * (v[k] - v[3 + k]); g[3 + k] = -g[k]; }
        if (H) {
            for (int i = 0; i < 36; ++i) H[i] = 0.0;
            for (int k = 0; k < 6; ++k) H[7 * k] = 2.0;
            for (int k = 0; k < 3; ++k) { H[k * 6 + 3 + k] = -2.0; H[(3 + k) * 6 + k] = -2.0; }
        }
        return;
    }
    case 1: g_PE<double>(v, g); if (H) H_PE<double>(v, H); return;
    case 2: g_PT<double>(v, g); if (H) H_PT<double>(v, H); return;
    default: g_EE<double>(v, g); if (H) H_EE<double>(v, H); return;
    }
}

struct DynOut {
    int* gKey;
    double* gVal;
    uint64_t* hKey;
    void* hVal;
    int mixed;
};

__device__ __forceinline__ void putH(const DynOut& o, size_t e, int k, double v) {
    if (o.mixed) ((float*)o.hVal)[9 * e + k] = (float)v;
    else ((double*)o.hVal)[9 * e + k] = v;
}

// Writes the projected n x n matrix (leading dimension ld) as 16 block
// entries on vertices idx[0..np-1]; unused or non-free entries get the
// sentinel key.  `step` lanes (a warp or a half warp) share the entries.
__device__ void writeBlocks(const DynOut& o, size_t hBase, const double* A, int ld, const int* idx, int np, const int* btype, int lane,
                            int step = 32) {
    for (int e = lane; e < 16 * 9; e += step) {
        int blk = e / 9, k = e % 9;
        int a = blk / 4, b = blk % 4;
        size_t slot = hBase + blk;
        bool valid = a < np && b < np && btype[idx[a]] == 0 && btype[idx[b]] == 0;
        if (k == 0) o.hKey[slot] = valid ? (((uint64_t)(uint32_t)idx[a] << 32) | (uint32_t)idx[b]) : HSENT;
        double v = valid ? A[(3 * a + k / 3) * ld + 3 * b + k % 3] : 0.0;
        putH(o, slot, k, v);
    }
}

// shared scratch of one contact in the half-warp projection kernel
struct HalfSmem {
    double A[144], V[144], lam[12];
};

// index of entry (lo, hi), lo <= hi < 12, in a packed upper triangle (78)
__host__ __device__ constexpr int upperIndex(int lo, int hi) { return lo * 12 - lo * (lo - 1) / 2 + (hi - lo); }

// Self-contact barrier, one thread per contact: the gradient entries
// kappa*b'(d)*grad d (x multiplicity for PP/PE) and, withHessian, the upper
// triangle of kappa*(b'' g g^T + b' H) zero-padded to 12 x 12, 78 values per
// contact at upper + 78 i, for the projection kernel.  Every entry (r, q) is
// formed once, so the matrix the eigen-solver gets is exactly symmetric.
__global__ void selfBarrierKernel(int n, const int* active, const double* x, double Hhat, double kappa, DynOut o, size_t gBase,
                                  int withHessian, double* upper, int* status) {
    CIPC_KERNEL_LOOP(i, n) {
        int idx[4] = {0, 0, 0, 0};
        const int kind = decode(active + 4 * i, idx);
        const int np = npts(kind), nd = 3 * np;
        d3 p[4];
        for (int k = 0; k < np; ++k) p[k] = ld3(x, idx[k]);
        const double d = distVal(kind, p);
        double gb, hb;
        barrierG(d, Hhat, gb);
        barrierH(d, Hhat, hb);
        const double cf = (kind <= 1) ? kappa * -active[4 * i + 3] : kappa;
        if (!isfinite(d)) raiseStatus(status, CIPC_ST_NONFINITE);
        double g[12], H[144];
        distDerivs(kind, p, g, withHessian ? H : nullptr);
        for (int a = 0; a < 4; ++a) {
            const size_t slot = gBase + 4 * (size_t)i + a;
            const bool valid = a < np;
            o.gKey[slot] = valid ? idx[a] : GSENT;
            for (int k = 0; k < 3; ++k) o.gVal[3 * slot + k] = valid ? cf * gb * g[3 * a + k] : 0.0;
        }
        if (withHessian) {
            const double ca = cf * hb, cb = cf * gb;
            double* U = upper + 78 * (size_t)i;
            for (int lo = 0; lo < 12; ++lo)
                for (int hi = lo; hi < 12; ++hi)
                    U[upperIndex(lo, hi)] = (hi < nd) ? (ca * g[lo]) * g[hi] + cb * H[lo * nd + hi] : 0.0;
        }
    }
}

// PSD projection of the self-contact barrier Hessians, one half warp per
// contact (two per warp): the packed upper triangle is unfolded into a
// symmetric 12 x 12 in shared memory, projected by the register-resident
// Jacobi sweep and written as the contact's 16 vertex-pair blocks.  Three
// blocks per SM: 168 registers (the columns of the matrix and of its
// eigenvectors stay in registers) for 12 resident warps.
__global__ void __launch_bounds__(32 * WPB, 3) selfBarrierPsdKernel(int n, const int* active, const int* btype, const double* upper, DynOut o, size_t hBase, int* status) {
    __shared__ HalfSmem sm[2 * WPB];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, half = lane >> 4, hl = lane & 15;
    HalfSmem& S = sm[2 * w + half];
    for (int i0 = 2 * (blockIdx.x * WPB + w); i0 < n; i0 += 2 * gridDim.x * WPB) {
        const int i = i0 + half;
        const bool act = i < n;
        if (act) {
            const double* U = upper + 78 * (size_t)i;
            for (int e = hl; e < 144; e += 16) {
                const int r = e / 12, q = e - r * 12;
                S.A[e] = U[r <= q ? upperIndex(r, q) : upperIndex(q, r)];
            }
        }
        __syncwarp();
        if (!halfWarpPsdProject12(S.A, S.V, S.lam, hl, act) && act && hl == 0) raiseStatus(status, CIPC_ST_JACOBI_CAP);
        if (act) {
            int idx[4] = {0, 0, 0, 0};
            const int np = npts(decode(active + 4 * i, idx));
            writeBlocks(o, hBase + 16 * (size_t)i, S.A, 12, idx, np, btype, hl, 16);
        }
        __syncwarp();
    }
}

__device__ __forceinline__ void edgeQuad(const int* see, const int* eeIe, const int* edges, int i, int q[4]) {
    const int* c = see + 4 * i;
    if (c[3] >= 0) { q[0] = c[0]; q[1] = c[1]; q[2] = c[2]; q[3] = c[3]; return; }
    int eI = eeIe[2 * i], eJ = eeIe[2 * i + 1];
    q[0] = edges[2 * eI]; q[1] = edges[2 * eI + 1]; q[2] = edges[2 * eJ]; q[3] = edges[2 * eJ + 1];
}

// Mollified nearly-parallel edge-edge term kappa * e(x) * b(d(x)).
__global__ void mollifiedKernel(int n, const int* see, const int* eeIe, const int* edges, const double* x, const double* rest, const int* btype,
                                double Hhat, double kappa, DynOut o, size_t gBase, size_t hBase, int* status) {
    __shared__ JacobiSmem sm[WPB];
    int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    JacobiSmem& S = sm[w];
    for (int i = blockIdx.x * WPB + w; i < n; i += gridDim.x * WPB) {
        int q[4];
        edgeQuad(see, eeIe, edges, i, q);
        if (lane == 0) {
            const int* c = see + 4 * i;
            int cidx[4] = {0, 0, 0, 0};
            int kind = decode(c, cidx);
            int np = npts(kind);
            d3 p[4], pc[4];
            for (int k = 0; k < 4; ++k) p[k] = ld3(x, q[k]);
            for (int k = 0; k < np; ++k) pc[k] = ld3(x, cidx[k]);
            double d = distVal(kind, pc);
            double b, gb, hb;
            barrierB(d, Hhat, b); barrierG(d, Hhat, gb); barrierH(d, Hhat, hb);
            double ex = 1e-3 * sqn(ld3(rest, q[0]) - ld3(rest, q[1])) * sqn(ld3(rest, q[2]) - ld3(rest, q[3]));
            double v[12];
            for (int k = 0; k < 4; ++k) { v[3 * k] = p[k].x; v[3 * k + 1] = p[k].y; v[3 * k + 2] = p[k].z; }
            double cs = crossSqNormEE(p[0], p[1], p[2], p[3]);
            double e = 1.0;
            double* eg = S.cs;   // 12
            double* eH = S.O;    // 144
            double* gd = S.W;    // 12 (first 12 entries)
            double* Hd = S.B;    // 144
            for (int k = 0; k < 12; ++k) { eg[k] = 0.0; gd[k] = 0.0; }
            for (int k = 0; k < 144; ++k) { eH[k] = 0.0; Hd[k] = 0.0; }
            if (cs < ex) {
                double qq = cs / ex;
                e = (-qq + 2.0) * qq;
                double one = 1.0 / ex;
                double qg = 2.0 * one * (-one * cs + 1.0);
                double qH = -2.0 / (ex * ex);
                double cg[12];
                g_EECross<double>(v, cg);
                H_EECross<double>(v, eH);
                for (int r = 0; r < 12; ++r) {
                    for (int s = 0; s < 12; ++s) eH[r * 12 + s] = eH[r * 12 + s] * qg + (qH * cg[r]) * cg[s];
                    eg[r] = qg * cg[r];
                }
            }
            // distance derivatives scattered onto the edge quad
            double g9[12], H9[144];
            distDerivs(kind, pc, g9, H9);
            int map[4] = {0, 1, 2, 3};
            if (kind != 3) {
                for (int a = 0; a < np; ++a)
                    for (int k = 0; k < 4; ++k)
                        if (q[k] == cidx[a]) { map[a] = k; break; }
            }
            int nd = 3 * np;
            for (int a = 0; a < np; ++a)
                for (int r = 0; r < 3; ++r) {
                    gd[3 * map[a] + r] = g9[3 * a + r];
                    for (int bb = 0; bb < np; ++bb)
                        for (int s = 0; s < 3; ++s) Hd[(3 * map[a] + r) * 12 + 3 * map[bb] + s] = H9[(3 * a + r) * nd + 3 * bb + s];
                }
            for (int r = 0; r < 12; ++r) S.V[r] = kappa * b * eg[r] + kappa * (e * gb) * gd[r];
            for (int r = 0; r < 12; ++r)
                for (int s = 0; s < 12; ++s) {
                    double k1 = ((kappa * gb) * gd[r]) * eg[s];
                    double k1t = ((kappa * gb) * gd[s]) * eg[r];
                    S.A[r * 12 + s] = k1 + k1t + (kappa * b) * eH[r * 12 + s] + ((kappa * e * hb) * gd[r]) * gd[s] + (kappa * e * gb) * Hd[r * 12 + s];
                }
            if (!isfinite(d)) raiseStatus(status, CIPC_ST_NONFINITE);
        }
        __syncwarp();
        if (lane < 4) {
            size_t slot = gBase + 4 * (size_t)i + lane;
            o.gKey[slot] = q[lane];
            for (int k = 0; k < 3; ++k) o.gVal[3 * slot + k] = S.V[3 * lane + k];
        }
        __syncwarp();
        if (!warpPsdProject(S, 12, lane) && lane == 0) raiseStatus(status, CIPC_ST_JACOBI_CAP);
        writeBlocks(o, hBase + 16 * (size_t)i, S.A, 12, q, 4, btype, lane);
        __syncwarp();
    }
}

__global__ void groundBarrierKernel(int n, const int* ground, const double* x, const int* btype, double nx, double ny, double nz, double D,
                                    double Hhat, double kappa, double* vtxGrad, double* diagExtra) {
    CIPC_KERNEL_LOOP(i, n) {
        int v = ground[i];
        d3 p = ld3(x, v);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        double d = dist * dist;
        double gb, hb;
        barrierG(d, Hhat, gb);
        barrierH(d, Hhat, hb);
        double s = kappa * gb * 2.0 * dist;
        vtxGrad[3 * v] += s * nx; vtxGrad[3 * v + 1] += s * ny; vtxGrad[3 * v + 2] += s * nz;
        double param = 4.0 * hb * d + 2.0 * gb;
        if (param > 0 && btype[v] == 0) {
            double n3[3] = {nx, ny, nz};
            for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) diagExtra[9 * v + 3 * a + b] += kappa * param * n3[a] * n3[b];
        }
    }
}

// ---- friction ----
__device__ __forceinline__ d3 nrm(d3 a) { double n = sqrt(sqn(a)); return n > 0 ? a / n : a; }

__global__ void frictionInitKernel(int n, const int* active, const double* x, double Hhat, double kappa, int* fset, double* lambda, double* coord,
                                   double* basis) {
    CIPC_KERNEL_LOOP(i, n) {
        const int* c = active + 4 * i;
        for (int k = 0; k < 4; ++k) fset[4 * i + k] = c[k];
        int idx[4] = {0, 0, 0, 0};
        int kind = decode(c, idx);
        d3 p[4];
        for (int k = 0; k < npts(kind); ++k) p[k] = ld3(x, idx[k]);
        double d = distVal(kind, p);
        double gb;
        barrierG(d, Hhat, gb);
        double lam = gb * (-kappa * 2.0 * sqrt(d));
        if (c[3] < -1) lam *= -c[3];
        lambda[i] = lam;
        double c0 = 0, c1 = 0;
        d3 b0, b1;
        if (kind == 3) {
            d3 e20 = p[0] - p[2], e01 = p[1] - p[0], e23 = p[3] - p[2];
            solve2(sqn(e01), -dot(e23, e01), sqn(e23), -dot(e20, e01), dot(e20, e23), c0, c1);
            b0 = nrm(e01);
            b1 = nrm(cross(cross(e01, e23), e01));
        } else if (kind == 0) {
            d3 v01 = p[1] - p[0];
            d3 xc = cross(mk(1, 0, 0), v01), yc = cross(mk(0, 1, 0), v01);
            if (sqn(xc) > sqn(yc)) { b0 = nrm(xc); b1 = nrm(cross(v01, xc)); }
            else { b0 = nrm(yc); b1 = nrm(cross(v01, yc)); }
        } else if (kind == 1) {
            d3 e12 = p[2] - p[1];
            c0 = dot(p[0] - p[1], e12) / sqn(e12);
            b0 = nrm(e12);
            b1 = nrm(cross(e12, p[0] - p[1]));
        } else {
            d3 r0 = p[2] - p[1], r1 = p[3] - p[1], w = p[0] - p[1];
            solve2(dot(r0, r0), dot(r0, r1), dot(r1, r1), dot(r0, w), dot(r1, w), c0, c1);
            b0 = nrm(r0);
            b1 = nrm(cross(cross(r0, r1), r0));
        }
        coord[2 * i] = c0; coord[2 * i + 1] = c1;
        double* B = basis + 6 * i;
        B[0] = b0.x; B[1] = b1.x; B[2] = b0.y; B[3] = b1.y; B[4] = b0.z; B[5] = b1.z;
    }
}

__global__ void frictionGroundInitKernel(int n, const int* ground, const double* x, double nx, double ny, double nz, double D, double Hhat,
                                         double kappa, int* fg, double* lambda) {
    CIPC_KERNEL_LOOP(i, n) {
        int v = ground[i];
        fg[i] = v;
        d3 p = ld3(x, v);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        double d = dist * dist;
        double gb;
        barrierG(d, Hhat, gb);
        lambda[i] = gb * (-kappa * 2.0 * sqrt(d));
    }
}

// Relative tangential displacement and lift weights of a lagged contact.
__device__ __forceinline__ int frictionRel(const int* c, const double* x, const double* vp, const double* co, const double* B, int idx[4], double w[4],
                                           double rel[2]) {
    int kind = decode(c, idx);
    int np = npts(kind);
    d3 dd[4];
    for (int k = 0; k < np; ++k) dd[k] = ld3(x, idx[k]) - ld3(vp, idx[k]);
    d3 r;
    if (kind == 3) {
        r = dd[0] + co[0] * (dd[1] - dd[0]) - (dd[2] + co[1] * (dd[3] - dd[2]));
        w[0] = 1.0 - co[0]; w[1] = co[0]; w[2] = co[1] - 1.0; w[3] = -co[1];
    } else if (kind == 0) {
        r = dd[0] - dd[1]; w[0] = 1; w[1] = -1;
    } else if (kind == 1) {
        r = dd[0] - (dd[1] + co[0] * (dd[2] - dd[1]));
        w[0] = 1; w[1] = co[0] - 1.0; w[2] = -co[0];
    } else {
        r = dd[0] - (dd[1] + co[0] * (dd[2] - dd[1]) + co[1] * (dd[3] - dd[1]));
        w[0] = 1; w[1] = -1 + co[0] + co[1]; w[2] = -co[0]; w[3] = -co[1];
    }
    rel[0] = r.x * B[0] + r.y * B[2] + r.z * B[4];
    rel[1] = r.x * B[1] + r.y * B[3] + r.z * B[5];
    return np;
}

__device__ __forceinline__ double f1DivNorm(double x2, double eps) { return (-sqrt(x2) + 2.0 * eps) / (eps * eps); }
__device__ __forceinline__ double f2SF(double x2, double eps) { return 2.0 * (eps - sqrt(x2)) / (eps * eps); }
__device__ __forceinline__ double f0SF(double x2, double eps) { return x2 * (-sqrt(x2) / 3.0 + eps) / (eps * eps) + eps / 3.0; }

__global__ void frictionSelfKernel(int n, const int* fset, const double* x, const double* vp, const double* coord, const double* basis,
                                   const double* lambda, const int* btype, double eps2, double coef, DynOut o, size_t gBase, size_t hBase) {
    CIPC_KERNEL_LOOP(i, n) {
        int idx[4] = {0, 0, 0, 0};
        double w[4], rel[2];
        const double* B = basis + 6 * i;
        int np = frictionRel(fset + 4 * i, x, vp, coord + 2 * i, B, idx, w, rel);
        double eps = sqrt(eps2);
        double sq = rel[0] * rel[0] + rel[1] * rel[1];
        double u0 = rel[0], u1 = rel[1];
        if (sq > eps2) { double s = sqrt(sq); u0 /= s; u1 /= s; }
        else { double f = f1DivNorm(sq, eps); u0 *= f; u1 *= f; }
        d3 t = mk(B[0] * u0 + B[1] * u1, B[2] * u0 + B[3] * u1, B[4] * u0 + B[5] * u1);
        double s = coef * lambda[i];
        for (int k = 0; k < 4; ++k) {
            size_t slot = gBase + 4 * (size_t)i + k;
            bool valid = k < np;
            o.gKey[slot] = valid ? idx[k] : GSENT;
            d3 g = (w[k] * s) * t;
            o.gVal[3 * slot] = valid ? g.x : 0.0; o.gVal[3 * slot + 1] = valid ? g.y : 0.0; o.gVal[3 * slot + 2] = valid ? g.z : 0.0;
        }
        // analytic PSD Hessian: rank <= 2 in the tangent plane
        double weight = fmax(0.0, coef * lambda[i]);
        double dirs[2][2] = {{0, 0}, {0, 0}}, eig[2] = {0, 0};
        if (weight != 0.0) {
            double nr = sqrt(sq);
            if (nr > 0.0) {
                double p0 = rel[0] / nr, p1 = rel[1] / nr;
                if (nr > eps) { dirs[0][0] = -p1; dirs[0][1] = p0; eig[0] = 1.0 / nr; }
                else {
                    dirs[0][0] = p0; dirs[0][1] = p1; eig[0] = f2SF(sq, eps);
                    dirs[1][0] = -p1; dirs[1][1] = p0; eig[1] = f1DivNorm(sq, eps);
                }
            } else {
                double iso = f1DivNorm(0.0, eps);
                dirs[0][0] = 1; eig[0] = iso;
                dirs[1][1] = 1; eig[1] = iso;
            }
        }
        d3 L[2];
        double lw[2];
        for (int m = 0; m < 2; ++m) {
            L[m] = mk(B[0] * dirs[m][0] + B[1] * dirs[m][1], B[2] * dirs[m][0] + B[3] * dirs[m][1], B[4] * dirs[m][0] + B[5] * dirs[m][1]);
            lw[m] = weight * fmax(0.0, eig[m]);
        }
        for (int blk = 0; blk < 16; ++blk) {
            int a = blk / 4, b = blk % 4;
            size_t slot = hBase + 16 * (size_t)i + blk;
            bool valid = a < np && b < np && btype[idx[a]] == 0 && btype[idx[b]] == 0;
            o.hKey[slot] = valid ? (((uint64_t)(uint32_t)idx[a] << 32) | (uint32_t)idx[b]) : HSENT;
            for (int r = 0; r < 3; ++r)
                for (int q = 0; q < 3; ++q) {
                    double v = 0;
                    for (int m = 0; m < 2; ++m) v += lw[m] * (w[a] * comp(L[m], r)) * (w[b] * comp(L[m], q));
                    putH(o, slot, 3 * r + q, valid ? v : 0.0);
                }
        }
    }
}

__global__ void frictionGroundKernel(int n, const int* fg, const double* lambda, const double* x, const double* vp, const int* btype, double nx,
                                     double ny, double nz, double eps2, double coef, double* vtxGrad, double* diagExtra) {
    CIPC_KERNEL_LOOP(i, n) {
        int v = fg[i];
        d3 N = mk(nx, ny, nz);
        d3 d = ld3(x, v) - ld3(vp, v);
        d3 pr = d - dot(d, N) * N;
        double p2 = sqn(pr);
        double eps = sqrt(eps2);
        d3 g = p2 > eps2 ? (coef * lambda[i] / sqrt(p2)) * pr : (coef * lambda[i] / eps) * pr;
        vtxGrad[3 * v] += g.x; vtxGrad[3 * v + 1] += g.y; vtxGrad[3 * v + 2] += g.z;
        // groundTangentBasis (Friction.cpp:66-76)
        d3 helper = fabs(nx) < 0.9 ? mk(1, 0, 0) : mk(0, 1, 0);
        d3 b0 = nrm(helper - dot(helper, N) * N);
        d3 b1 = nrm(cross(N, b0));
        double mult = fmax(0.0, coef * lambda[i]);
        if (mult > 0.0 && btype[v] == 0) {
            double r0 = dot(b0, d), r1 = dot(b1, d);
            double nr = sqrt(r0 * r0 + r1 * r1);
            double H[9];
            if (nr > eps) {
                double p0 = r0 / nr, p1 = r1 / nr;
                d3 l = (-p1) * b0 + p0 * b1;
                for (int a = 0; a < 3; ++a) for (int b = 0; b < 3; ++b) H[3 * a + b] = (mult / nr) * comp(l, a) * comp(l, b);
            } else {
                for (int a = 0; a < 3; ++a)
                    for (int b = 0; b < 3; ++b) H[3 * a + b] = (mult / eps) * (comp(b0, a) * comp(b0, b) + comp(b1, a) * comp(b1, b));
            }
            for (int k = 0; k < 9; ++k) diagExtra[9 * v + k] += H[k];
        }
    }
}

// ---- energies ----
__global__ void groundEnergyKernel(int n, const int* ground, const double* x, double nx, double ny, double nz, double D, double Hhat, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        d3 p = ld3(x, ground[i]);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        double b;
        barrierB(dist * dist, Hhat, b);
        out[i] = b;
    }
}
__global__ void selfEnergyKernel(int n, const int* active, const double* x, double Hhat, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        int idx[4] = {0, 0, 0, 0};
        const int* c = active + 4 * i;
        int kind = decode(c, idx);
        d3 p[4];
        for (int k = 0; k < npts(kind); ++k) p[k] = ld3(x, idx[k]);
        double b;
        barrierB(distVal(kind, p), Hhat, b);
        if (c[3] < -1) b *= -c[3];
        out[i] = b;
    }
}
__global__ void mollEnergyKernel(int n, const int* see, const int* eeIe, const int* edges, const double* x, const double* rest, double Hhat, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        int q[4];
        edgeQuad(see, eeIe, edges, i, q);
        int idx[4] = {0, 0, 0, 0};
        int kind = decode(see + 4 * i, idx);
        d3 p[4];
        for (int k = 0; k < npts(kind); ++k) p[k] = ld3(x, idx[k]);
        double b;
        barrierB(distVal(kind, p), Hhat, b);
        double ex = 1e-3 * sqn(ld3(rest, q[0]) - ld3(rest, q[1])) * sqn(ld3(rest, q[2]) - ld3(rest, q[3]));
        double cs = crossSqNormEE(ld3(x, q[0]), ld3(x, q[1]), ld3(x, q[2]), ld3(x, q[3]));
        double e = 1.0;
        if (cs < ex) { double qq = cs / ex; e = (-qq + 2.0) * qq; }
        out[i] = b * e;
    }
}
__global__ void frictionEnergyKernel(int n, const int* fset, const double* x, const double* vp, const double* coord, const double* basis,
                                     const double* lambda, double eps2, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        int idx[4];
        double w[4], rel[2];
        frictionRel(fset + 4 * i, x, vp, coord + 2 * i, basis + 6 * i, idx, w, rel);
        double sq = rel[0] * rel[0] + rel[1] * rel[1];
        double eps = sqrt(eps2);
        out[i] = sq > eps2 ? lambda[i] * sqrt(sq) : lambda[i] * f0SF(sq, eps);
    }
}
__global__ void frictionGroundEnergyKernel(int n, const int* fg, const double* lambda, const double* x, const double* vp, double nx, double ny,
                                           double nz, double eps2, double friction, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        int v = fg[i];
        d3 N = mk(nx, ny, nz);
        d3 d = ld3(x, v) - ld3(vp, v);
        d3 pr = d - dot(d, N) * N;
        double sq = sqn(pr);
        double eps = sqrt(eps2);
        double cl = sq > eps2 ? sqrt(sq) - 0.5 * eps : 0.5 * sq / eps;
        out[i] = friction * lambda[i] * cl;
    }
}

// ---- dynamic segment bookkeeping ----
__global__ void gradSegKernel(int n, const int* keys, int* start, int* end) {
    CIPC_KERNEL_LOOP(i, n) {
        int k = keys[i];
        if (k == GSENT) continue;
        if (i == 0 || keys[i - 1] != k) start[k] = i;
        if (i == n - 1 || keys[i + 1] != k) end[k] = i + 1;
    }
}
__global__ void headFlagKernel(int n, const uint64_t* keys, int* flags) {
    CIPC_KERNEL_LOOP(i, n) {
        uint64_t k = keys[i];
        flags[i] = (k != HSENT && (i == 0 || keys[i - 1] != k)) ? 1 : 0;
    }
}
__global__ void uniqueKernel(int n, const uint64_t* keys, const int* flags, const int* pos, int* col, int* srcStart) {
    CIPC_KERNEL_LOOP(i, n) {
        if (!flags[i]) continue;
        int u = pos[i];
        col[u] = (int)(keys[i] & 0xffffffffu);
        srcStart[u] = i;
    }
}
// Number of non-sentinel entries in a sorted key array (sentinels sort last).
__global__ void validCountKernel(int n, const uint64_t* keys, int* out) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (keys[mid] == HSENT) hi = mid; else lo = mid + 1;
    }
    *out = lo;
}
__global__ void rowBoundsKernel(int nu, const int* srcStart, const uint64_t* keys, int* rowStart, int* rowEnd) {
    CIPC_KERNEL_LOOP(u, nu) {
        int r = (int)(keys[srcStart[u]] >> 32);
        int rPrev = u > 0 ? (int)(keys[srcStart[u - 1]] >> 32) : -1;
        int rNext = u + 1 < nu ? (int)(keys[srcStart[u + 1]] >> 32) : -1;
        if (r != rPrev) rowStart[r] = u;
        if (r != rNext) rowEnd[r] = u + 1;
    }
}
template <class T>
__global__ void dynReduceKernel(int nu, int nValid, const int* srcStart, const int* order, const T* vals, T* out) {
    CIPC_KERNEL_LOOP(u, nu) {
        int b = srcStart[u], e = u + 1 < nu ? srcStart[u + 1] : nValid;
        T acc[9];
        for (int k = 0; k < 9; ++k) acc[k] = T(0);
        for (int j = b; j < e; ++j) {
            const T* v = vals + (size_t)9 * order[j];
            for (int k = 0; k < 9; ++k) acc[k] += v[k];
        }
        for (int k = 0; k < 9; ++k) out[(size_t)9 * u + k] = acc[k];
    }
}
__global__ void iotaKernel(int n, int* a) { CIPC_KERNEL_LOOP(i, n) a[i] = i; }

}  // namespace

static DynOut dynOut(Ctx& c) {
    DynOut o;
    o.gKey = c.dynGKey; o.gVal = c.dynGVal; o.hKey = c.dynHKey;
    o.hVal = c.mixed ? (void*)c.dynHValF.p : (void*)c.dynHValD.p;
    o.mixed = c.mixed;
    return o;
}

static void reserveDyn(Ctx& c, int nContacts) {
    size_t ng = 4 * (size_t)std::max(nContacts, 1), nh = 16 * (size_t)std::max(nContacts, 1);
    c.dynGKey.reserve(ng); c.dynGKeyAlt.reserve(ng); c.dynGIdx.reserve(ng); c.dynGIdxAlt.reserve(ng); c.dynGVal.reserve(3 * ng);
    c.dynHKey.reserve(nh); c.dynHKeyAlt.reserve(nh); c.dynHIdx.reserve(nh); c.dynHIdxAlt.reserve(nh);
    if (c.mixed) c.dynHValF.reserve(9 * nh); else c.dynHValD.reserve(9 * nh);
}

// Gradient/Hessian of all contact terms at the current x (barrier with
// kappa = P.kappa, friction with the lagged sets).  Ground terms go straight
// to the per-vertex accumulators; self terms become keyed entries.
int contactAssemble(Ctx& c) {
    const SimParams& P = c.P;
    if (c.nGround)
        launch(groundBarrierKernel, blocksFor(c.nGround), TB, 0, c.s, c.nGround, c.ground, c.x, c.btype, P.groundN[0], P.groundN[1], P.groundN[2],
                                                                 P.groundD, P.Hhat, P.kappa, c.vtxGrad, c.diagExtra);
    int nTot = c.nSelf + c.nMoll + c.nFric;
    reserveDyn(c, nTot);
    DynOut o = dynOut(c);
    size_t g = 0, h = 0;
    if (c.nSelf) {
        profBegin(c, PROF_BARRIER);
        c.barrierUpper.reserve(78 * (size_t)c.nSelf);
        launch(selfBarrierKernel, blocksFor(c.nSelf), TB, 0, c.s, c.nSelf, c.selfActive, c.x, P.Hhat, P.kappa, o, g, 1, c.barrierUpper.p, c.status);
        launch(selfBarrierPsdKernel, halfWarpBlocksFor(c.nSelf), 32 * WPB, 0, c.s, c.nSelf, c.selfActive, c.btype, c.barrierUpper.p, o, h, c.status);
        profEnd(c, PROF_BARRIER);
    }
    g += 4 * (size_t)c.nSelf; h += 16 * (size_t)c.nSelf;
    if (c.nMoll)
        launch(mollifiedKernel, warpBlocksFor(c.nMoll), 32 * WPB, 0, c.s, c.nMoll, c.selfEE, c.eeIe, c.edges, c.x, c.rest, c.btype, P.Hhat, P.kappa, o,
                                                                     g, h, c.status);
    g += 4 * (size_t)c.nMoll; h += 16 * (size_t)c.nMoll;
    double eps2 = P.Fhat * P.dt * P.dt;
    if (c.nFric)
        launch(frictionSelfKernel, blocksFor(c.nFric), TB, 0, c.s, c.nFric, c.fricSet, c.x, c.vp, c.fricCoord, c.fricBasis, c.fricLambda, c.btype, eps2,
                                                               P.friction, o, g, h);
    g += 4 * (size_t)c.nFric; h += 16 * (size_t)c.nFric;
    if (c.nFricG)
        launch(frictionGroundKernel, blocksFor(c.nFricG), TB, 0, c.s, c.nFricG, c.fricGround, c.fricGLambda, c.x, c.vp, c.btype, P.groundN[0], P.groundN[1],
                                                                  P.groundN[2], eps2, P.friction, c.vtxGrad, c.diagExtra);
    c.nDynG = (int)g;
    c.nDynH = (int)h;
    CIPC_CUDA(cudaGetLastError());
    finalizeDynamic(c);
    return c.nPT + c.nEE + (int)c.nPPERaw;
}

void finalizeDynamic(Ctx& c) {
    int ng = c.nDynG, nh = c.nDynH;
    c.dynGStart.reserve(c.nv); c.dynGEnd.reserve(c.nv);
    CIPC_CUDA(cudaMemsetAsync(c.dynGStart.p, 0, sizeof(int) * c.nv, c.s));
    CIPC_CUDA(cudaMemsetAsync(c.dynGEnd.p, 0, sizeof(int) * c.nv, c.s));
    c.dynRowStart.reserve(c.nv); c.dynRowEnd.reserve(c.nv);
    CIPC_CUDA(cudaMemsetAsync(c.dynRowStart.p, 0, sizeof(int) * c.nv, c.s));
    CIPC_CUDA(cudaMemsetAsync(c.dynRowEnd.p, 0, sizeof(int) * c.nv, c.s));
    c.nDynB = 0;
    if (ng > 0) {
        launch(iotaKernel, blocksFor(ng), TB, 0, c.s, ng, c.dynGIdxAlt);
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, c.dynGKey.p, c.dynGKeyAlt.p, c.dynGIdxAlt.p, c.dynGIdx.p, ng, 0, 32, c.s);
        c.sortTmp.reserve(bytes + 16);
        CIPC_CUDA(cub::DeviceRadixSort::SortPairs(c.sortTmp.p, bytes, c.dynGKey.p, c.dynGKeyAlt.p, c.dynGIdxAlt.p, c.dynGIdx.p, ng, 0, 32, c.s));
        launch(gradSegKernel, blocksFor(ng), TB, 0, c.s, ng, c.dynGKeyAlt, c.dynGStart, c.dynGEnd);
    }
    if (nh > 0) {
        launch(iotaKernel, blocksFor(nh), TB, 0, c.s, nh, c.dynHIdxAlt);
        size_t bytes = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, bytes, c.dynHKey.p, c.dynHKeyAlt.p, c.dynHIdxAlt.p, c.dynHIdx.p, nh, 0, 64, c.s);
        c.sortTmp.reserve(bytes + 16);
        CIPC_CUDA(cub::DeviceRadixSort::SortPairs(c.sortTmp.p, bytes, c.dynHKey.p, c.dynHKeyAlt.p, c.dynHIdxAlt.p, c.dynHIdx.p, nh, 0, 64, c.s));
        c.counts.reserve(nh + 1);
        c.runs.reserve(nh + 1);
        launch(headFlagKernel, blocksFor(nh), TB, 0, c.s, nh, c.dynHKeyAlt, c.counts);
        size_t b2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, b2, c.counts.p, c.runs.p, nh + 1, c.s);
        c.sortTmp.reserve(b2 + 16);
        // flags[nh] must be 0 so that runs[nh] is the unique count
        CIPC_CUDA(cudaMemsetAsync(c.counts.p + nh, 0, sizeof(int), c.s));
        CIPC_CUDA(cub::DeviceScan::ExclusiveSum(c.sortTmp.p, b2, c.counts.p, c.runs.p, nh + 1, c.s));
        int nu = 0;
        CIPC_CUDA(cudaMemcpyAsync(&nu, c.runs.p + nh, sizeof(int), cudaMemcpyDeviceToHost, c.s));
        hostSync(c);
        c.nDynB = nu;
        if (nu > 0) {
            c.dynCol.reserve(nu); c.dynSrcStart.reserve(nu);
            launch(uniqueKernel, blocksFor(nh), TB, 0, c.s, nh, c.dynHKeyAlt, c.counts, c.runs, c.dynCol, c.dynSrcStart);
            launch(rowBoundsKernel, blocksFor(nu), TB, 0, c.s, nu, c.dynSrcStart, c.dynHKeyAlt, c.dynRowStart, c.dynRowEnd);
            c.counters.reserve(16);
            launch(validCountKernel, 1, 1, 0, c.s, nh, c.dynHKeyAlt, c.counters.p + 9);
            int nValid = 0;
            CIPC_CUDA(cudaMemcpyAsync(&nValid, c.counters.p + 9, sizeof(int), cudaMemcpyDeviceToHost, c.s));
            hostSync(c);
            if (c.mixed) {
                c.dynBF.reserve((size_t)9 * nu);
                launch(dynReduceKernel<float>, blocksFor(nu), TB, 0, c.s, nu, nValid, c.dynSrcStart, c.dynHIdx, c.dynHValF, c.dynBF);
            } else {
                c.dynBD.reserve((size_t)9 * nu);
                launch(dynReduceKernel<double>, blocksFor(nu), TB, 0, c.s, nu, nValid, c.dynSrcStart, c.dynHIdx, c.dynHValD, c.dynBD);
            }
        }
    }
    CIPC_CUDA(cudaGetLastError());
}

// The contact energy's term sums into device slots slot0 .. slot0 + 4 (no
// host synchronisation); contactEnergyCombine adds them in a fixed order.
void contactEnergySums(Ctx& c, int slot0) {
    const SimParams& P = c.P;
    int n = std::max(std::max(c.nGround, c.nSelf), std::max(c.nMoll, std::max(c.nFric, c.nFricG)));
    c.energyBuf.reserve(std::max(n, 1));
    if (c.nGround) {
        launch(groundEnergyKernel, blocksFor(c.nGround), TB, 0, c.s, c.nGround, c.ground, c.x, P.groundN[0], P.groundN[1], P.groundN[2], P.groundD, P.Hhat,
                                                                c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nGround, slot0 + 0);
    }
    if (c.nSelf) {
        launch(selfEnergyKernel, blocksFor(c.nSelf), TB, 0, c.s, c.nSelf, c.selfActive, c.x, P.Hhat, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nSelf, slot0 + 1);
    }
    if (c.nMoll) {
        launch(mollEnergyKernel, blocksFor(c.nMoll), TB, 0, c.s, c.nMoll, c.selfEE, c.eeIe, c.edges, c.x, c.rest, P.Hhat, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nMoll, slot0 + 2);
    }
    double eps2 = P.Fhat * P.dt * P.dt;
    if (c.nFric) {
        launch(frictionEnergyKernel, blocksFor(c.nFric), TB, 0, c.s, c.nFric, c.fricSet, c.x, c.vp, c.fricCoord, c.fricBasis, c.fricLambda, eps2, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nFric, slot0 + 3);
    }
    if (c.nFricG) {
        launch(frictionGroundEnergyKernel, blocksFor(c.nFricG), TB, 0, c.s, c.nFricG, c.fricGround, c.fricGLambda, c.x, c.vp, P.groundN[0], P.groundN[1],
                                                                        P.groundN[2], eps2, P.friction, c.energyBuf);
        deviceSumTo(c, c.energyBuf, c.nFricG, slot0 + 4);
    }
}

double contactEnergyCombine(const Ctx& c, double kappa, const double* h) {
    if (!(c.nGround || c.nSelf || c.nMoll || c.nFric || c.nFricG)) return 0.0;
    double bsum = 0;
    if (c.nGround) bsum += h[0];
    if (c.nSelf) bsum += h[1];
    if (c.nMoll) bsum += h[2];
    double E = kappa * bsum;
    if (c.nFric) E += c.P.friction * h[3];
    if (c.nFricG) E += h[4];
    return E;
}

double contactEnergy(Ctx& c, double kappa) {
    if (!(c.nGround || c.nSelf || c.nMoll || c.nFric || c.nFricG)) return 0.0;
    contactEnergySums(c, 0);
    double h[5];
    fetchSums(c, h, 5);
    return contactEnergyCombine(c, kappa, h);
}

// Friction::initialize at the current x with kappa = P.kappa.
void frictionInitialize(Ctx& c) {
    const SimParams& P = c.P;
    c.nFric = c.nSelf;
    c.fricSet.reserve(4 * std::max(c.nFric, 1));
    c.fricLambda.reserve(std::max(c.nFric, 1));
    c.fricCoord.reserve(2 * std::max(c.nFric, 1));
    c.fricBasis.reserve(6 * std::max(c.nFric, 1));
    if (c.nFric)
        launch(frictionInitKernel, blocksFor(c.nFric), TB, 0, c.s, c.nFric, c.selfActive, c.x, P.Hhat, P.kappa, c.fricSet, c.fricLambda, c.fricCoord,
                                                               c.fricBasis);
    c.nFricG = c.nGround;
    c.fricGround.reserve(std::max(c.nFricG, 1));
    c.fricGLambda.reserve(std::max(c.nFricG, 1));
    if (c.nFricG)
        launch(frictionGroundInitKernel, blocksFor(c.nFricG), TB, 0, c.s, c.nFricG, c.ground, c.x, P.groundN[0], P.groundN[1], P.groundN[2], P.groundD,
                                                                      P.Hhat, P.kappa, c.fricGround, c.fricGLambda);
    CIPC_CUDA(cudaGetLastError());
}

namespace {
__global__ void gatherDynOnly(int nv, const int* start, const int* end, const int* idx, const double* val, double* out) {
    CIPC_KERNEL_LOOP(v, nv) {
        double g[3] = {out[3 * v], out[3 * v + 1], out[3 * v + 2]};
        for (int k = start[v]; k < end[v]; ++k) {
            int e = idx[k];
            g[0] += val[3 * e]; g[1] += val[3 * e + 1]; g[2] += val[3 * e + 2];
        }
        out[3 * v] = g[0]; out[3 * v + 1] = g[1]; out[3 * v + 2] = g[2];
    }
}
__global__ void groundGradOnly(int n, const int* ground, const double* x, double nx, double ny, double nz, double D, double Hhat, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        int v = ground[i];
        d3 p = ld3(x, v);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        double gb;
        barrierG(dist * dist, Hhat, gb);
        double s = gb * 2.0 * dist;
        out[3 * v] += s * nx; out[3 * v + 1] += s * ny; out[3 * v + 2] += s * nz;
    }
}
}  // namespace

// Constraint gradient with coefficient 1 (ground + self PT/EE/PP/PE, no
// mollified term), as initKappa uses it (IPCSolver.cpp:782-797).
void contactGradientKappa(Ctx& c, double* gc) {
    const SimParams& P = c.P;
    CIPC_CUDA(cudaMemsetAsync(gc, 0, sizeof(double) * 3 * c.nv, c.s));
    if (c.nGround)
        launch(groundGradOnly, blocksFor(c.nGround), TB, 0, c.s, c.nGround, c.ground, c.x, P.groundN[0], P.groundN[1], P.groundN[2], P.groundD, P.Hhat, gc);
    if (c.nSelf) {
        reserveDyn(c, c.nSelf);
        DynOut o = dynOut(c);
        launch(selfBarrierKernel, blocksFor(c.nSelf), TB, 0, c.s, c.nSelf, c.selfActive, c.x, P.Hhat, 1.0, o, (size_t)0, 0, (double*)nullptr, c.status);
        c.nDynG = 4 * c.nSelf;
        c.nDynH = 0;
        finalizeDynamic(c);
        launch(gatherDynOnly, blocksFor(c.nv), TB, 0, c.s, c.nv, c.dynGStart, c.dynGEnd, c.dynGIdx, c.dynGVal, gc);
        c.nDynG = 0;
    }
    CIPC_CUDA(cudaGetLastError());
}

namespace {
__global__ void groundDistKernel(int n, const int* ground, const double* x, double nx, double ny, double nz, double D, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        d3 p = ld3(x, ground[i]);
        double dist = nx * p.x + ny * p.y + nz * p.z - D;
        out[i] = dist * dist;
    }
}
__global__ void selfDistKernel(int n, const int* active, const double* x, double* out) {
    CIPC_KERNEL_LOOP(i, n) {
        int idx[4] = {0, 0, 0, 0};
        int kind = decode(active + 4 * i, idx);
        d3 p[4];
        for (int k = 0; k < npts(kind); ++k) p[k] = ld3(x, idx[k]);
        out[i] = distVal(kind, p);
    }
}
__global__ void closeCheckKernel(int ng, const int* cg, const double* cgv, int ns, const int* cs, const double* csv, const double* x, double nx,
                                 double ny, double nz, double D, int* flag) {
    CIPC_KERNEL_LOOP(i, ng + ns) {
        if (i < ng) {
            d3 p = ld3(x, cg[i]);
            double dist = nx * p.x + ny * p.y + nz * p.z - D;
            if (dist * dist <= cgv[i]) atomicOr(flag, 1);
        } else {
            int j = i - ng;
            int idx[4] = {0, 0, 0, 0};
            int kind = decode(cs + 4 * j, idx);
            d3 p[4];
            for (int k = 0; k < npts(kind); ++k) p[k] = ld3(x, idx[k]);
            if (distVal(kind, p) <= csv[j]) atomicOr(flag, 1);
        }
    }
}
}  // namespace

void constraintMinMax(Ctx& c, double& mn, double& mx, bool& any) {
    const SimParams& P = c.P;
    int n = c.nGround + c.nSelf;
    any = n > 0;
    mn = 1e308; mx = -1e308;
    if (!any) return;
    c.energyBuf.reserve(n);
    if (c.nGround)
        launch(groundDistKernel, blocksFor(c.nGround), TB, 0, c.s, c.nGround, c.ground, c.x, P.groundN[0], P.groundN[1], P.groundN[2], P.groundD, c.energyBuf);
    if (c.nSelf) launch(selfDistKernel, blocksFor(c.nSelf), TB, 0, c.s, c.nSelf, c.selfActive, c.x, c.energyBuf.p + c.nGround);
    mn = deviceMin(c, c.energyBuf, n, 1e308);
    mx = deviceMax(c, c.energyBuf, n);
}

// postLineSearch part 1: has any recorded close constraint moved closer?
void closeConstraintCheck(Ctx& c, bool& update) {
    const SimParams& P = c.P;
    update = false;
    if (c.nCloseG + c.nCloseS == 0) return;
    c.counters.reserve(16);
    CIPC_CUDA(cudaMemsetAsync(c.counters.p + 8, 0, sizeof(int), c.s));
    launch(closeCheckKernel, blocksFor(c.nCloseG + c.nCloseS), TB, 0, c.s, c.nCloseG, c.closeG, c.closeGVal, c.nCloseS, c.closeS, c.closeSVal, c.x,
                                                                       P.groundN[0], P.groundN[1], P.groundN[2], P.groundD, c.counters.p + 8);
    int f = 0;
    CIPC_CUDA(cudaMemcpyAsync(&f, c.counters.p + 8, sizeof(int), cudaMemcpyDeviceToHost, c.s));
    hostSync(c);
    update = f != 0;
}

// postLineSearch part 2: record constraints with d < dTol (host-side
// compaction; dTol = 1e-18 * bbox^2 makes these lists tiny or empty).
void closeConstraintRecord(Ctx& c) {
    const SimParams& P = c.P;
    int n = c.nGround + c.nSelf;
    c.nCloseG = c.nCloseS = 0;
    if (n == 0) return;
    c.energyBuf.reserve(n);
    if (c.nGround)
        launch(groundDistKernel, blocksFor(c.nGround), TB, 0, c.s, c.nGround, c.ground, c.x, P.groundN[0], P.groundN[1], P.groundN[2], P.groundD, c.energyBuf);
    if (c.nSelf) launch(selfDistKernel, blocksFor(c.nSelf), TB, 0, c.s, c.nSelf, c.selfActive, c.x, c.energyBuf.p + c.nGround);
    double mn = deviceMin(c, c.energyBuf, n, 1e308);
    if (!(mn < P.dTol)) return;
    std::vector<double> d(n);
    CIPC_CUDA(cudaMemcpy(d.data(), c.energyBuf.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    std::vector<int> g(std::max(c.nGround, 1)), s(4 * std::max(c.nSelf, 1));
    if (c.nGround) CIPC_CUDA(cudaMemcpy(g.data(), c.ground.p, c.nGround * sizeof(int), cudaMemcpyDeviceToHost));
    if (c.nSelf) CIPC_CUDA(cudaMemcpy(s.data(), c.selfActive.p, 4 * c.nSelf * sizeof(int), cudaMemcpyDeviceToHost));
    std::vector<int> cg, cs;
    std::vector<double> cgv, csv;
    for (int i = 0; i < c.nGround; ++i) if (d[i] < P.dTol) { cg.push_back(g[i]); cgv.push_back(d[i]); }
    for (int i = 0; i < c.nSelf; ++i)
        if (d[c.nGround + i] < P.dTol) { for (int k = 0; k < 4; ++k) cs.push_back(s[4 * i + k]); csv.push_back(d[c.nGround + i]); }
    c.nCloseG = (int)cg.size(); c.nCloseS = (int)csv.size();
    c.closeG.reserve(std::max(c.nCloseG, 1)); c.closeGVal.reserve(std::max(c.nCloseG, 1));
    c.closeS.reserve(4 * std::max(c.nCloseS, 1)); c.closeSVal.reserve(std::max(c.nCloseS, 1));
    if (c.nCloseG) {
        CIPC_CUDA(cudaMemcpy(c.closeG.p, cg.data(), cg.size() * sizeof(int), cudaMemcpyHostToDevice));
        CIPC_CUDA(cudaMemcpy(c.closeGVal.p, cgv.data(), cgv.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
    if (c.nCloseS) {
        CIPC_CUDA(cudaMemcpy(c.closeS.p, cs.data(), cs.size() * sizeof(int), cudaMemcpyHostToDevice));
        CIPC_CUDA(cudaMemcpy(c.closeSVal.p, csv.data(), csv.size() * sizeof(double), cudaMemcpyHostToDevice));
    }
}

}  // namespace cipc
