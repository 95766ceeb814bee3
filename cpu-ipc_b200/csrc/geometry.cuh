// Contact geometry shared by the broad-phase, CCD and barrier kernels:
// closest-feature classification, squared distances, additive CCD and the
// segment-triangle intersection test.  Compiled without FMA contraction in
// the collision unit so that set-defining decisions (box overlap,
// classification, distance < dHat) round exactly like the oracle.
//
// Reference: dType_PT / dType_EE / d_* (CPU IPC/ContactMechanics.cpp:143-316,
// 764-813), point_triangle_ccd / edge_edge_ccd (CPU IPC/AdditiveCCD.cpp),
// IglUtils::segTriIntersect (CPU IPC/ContactMechanics.h:47-71).
#pragma once

#include "cipc_device.cuh"

namespace cipc {

// Explicit solution of a 2x2 symmetric system (stands in for the 2x2 LDLT of
// the reference; same formula as the oracle).
__device__ __forceinline__ void solve2(double m00, double m01, double m11, double r0, double r1, double& x0, double& x1) {
    double det = m00 * m11 - m01 * m01;
    x0 = (m11 * r0 - m01 * r1) / det;
    x1 = (m00 * r1 - m01 * r0) / det;
}
__device__ __forceinline__ void ptParam(d3 r0, d3 nvec, d3 w, double& p0, double& p1) {
    d3 r1 = cross(r0, nvec);
    solve2(dot(r0, r0), dot(r0, r1), dot(r1, r1), dot(r0, w), dot(r1, w), p0, p1);
}

__device__ __forceinline__ int dTypePT(d3 v0, d3 v1, d3 v2, d3 v3) {
    d3 nvec = cross(v2 - v1, v3 - v1);
    double a0, b0, a1, b1, a2, b2;
    ptParam(v2 - v1, nvec, v0 - v1, a0, b0);
    if (a0 > 0.0 && a0 < 1.0 && b0 >= 0.0) return 3;
    ptParam(v3 - v2, nvec, v0 - v2, a1, b1);
    if (a1 > 0.0 && a1 < 1.0 && b1 >= 0.0) return 4;
    ptParam(v1 - v3, nvec, v0 - v3, a2, b2);
    if (a2 > 0.0 && a2 < 1.0 && b2 >= 0.0) return 5;
    if (a0 <= 0.0 && a2 >= 1.0) return 0;
    if (a1 <= 0.0 && a0 >= 1.0) return 1;
    if (a2 <= 0.0 && a1 >= 1.0) return 2;
    return 6;
}

__device__ __forceinline__ int dTypeEE(d3 v0, d3 v1, d3 v2, d3 v3) {
    d3 u = v1 - v0, v = v3 - v2, w = v0 - v2;
    double a = dot(u, u), b = dot(u, v), c = dot(v, v), d = dot(u, w), e = dot(v, w);
    double D = a * c - b * b;
    double tD = D, sN, tN;
    int def = 8;
    sN = (b * e - c * d);
    if (sN <= 0.0) { tN = e; tD = c; def = 2; }
    else if (sN >= D) { tN = e + b; tD = c; def = 5; }
    else {
        tN = (a * e - b * d);
        d3 uv = cross(u, v);
        if (tN > 0.0 && tN < tD && (dot(uv, w) == 0.0 || sqn(uv) < 1.0e-20 * a * c)) {
            if (sN < D / 2) { tN = e; tD = c; def = 2; }
            else { tN = e + b; tD = c; def = 5; }
        }
    }
    if (tN <= 0.0) {
        if (-d <= 0.0) return 0;
        else if (-d >= a) return 3;
        else return 6;
    } else if (tN >= tD) {
        if ((-d + b) <= 0.0) return 1;
        else if ((-d + b) >= a) return 4;
        else return 7;
    }
    return def;
}

__device__ __forceinline__ double dPP(d3 a, d3 b) { return sqn(a - b); }
__device__ __forceinline__ double dPE(d3 p, d3 e0, d3 e1) { return sqn(cross(e0 - p, e1 - p)) / sqn(e1 - e0); }
__device__ __forceinline__ double dPT(d3 p, d3 t0, d3 t1, d3 t2) {
    d3 b = cross(t1 - t0, t2 - t0);
    double aTb = dot(p - t0, b);
    return aTb * aTb / sqn(b);
}
__device__ __forceinline__ double dEE(d3 a0, d3 a1, d3 b0, d3 b1) {
    d3 b = cross(a1 - a0, b1 - b0);
    double aTb = dot(b0 - a0, b);
    return aTb * aTb / sqn(b);
}
__device__ __forceinline__ double crossSqNormEE(d3 a0, d3 a1, d3 b0, d3 b1) { return sqn(cross(a1 - a0, b1 - b0)); }

__device__ __forceinline__ double ptDistU(d3 p, d3 t0, d3 t1, d3 t2) {
    switch (dTypePT(p, t0, t1, t2)) {
    case 0: return dPP(p, t0);
    case 1: return dPP(p, t1);
    case 2: return dPP(p, t2);
    case 3: return dPE(p, t0, t1);
    case 4: return dPE(p, t1, t2);
    case 5: return dPE(p, t2, t0);
    default: return dPT(p, t0, t1, t2);
    }
}
__device__ __forceinline__ double eeDistU(d3 a0, d3 a1, d3 b0, d3 b1) {
    switch (dTypeEE(a0, a1, b0, b1)) {
    case 0: return dPP(a0, b0);
    case 1: return dPP(a0, b1);
    case 2: return dPE(a0, b0, b1);
    case 3: return dPP(a1, b0);
    case 4: return dPP(a1, b1);
    case 5: return dPE(a1, b0, b1);
    case 6: return dPE(b0, a0, a1);
    case 7: return dPE(b1, a0, a1);
    default: return dEE(a0, a1, b0, b1);
    }
}

// Additive CCD, conservative time of impact in [0, 1] (eta = 1 - slackness).
// The iteration cap (10000) of the reference is kept; hitting it raises a
// status bit instead of looping on.
__device__ inline double edgeEdgeCCD(d3 a0, d3 a1, d3 b0, d3 b1, d3 da0, d3 da1, d3 db0, d3 db1, double eta, int* status) {
    const double th = 0.0;
    d3 mov = (da0 + da1 + db0 + db1) / 4;
    da0 = da0 - mov; da1 = da1 - mov; db0 = db0 - mov; db1 = db1 - mov;
    double maxDisp = sqrt(fmax(sqn(da0), sqn(da1))) + sqrt(fmax(sqn(db0), sqn(db1)));
    if (maxDisp == 0) return 1.0;
    double d2 = eeDistU(a0, a1, b0, b1);
    double dF = d2 - th * th;
    if (dF <= 0) {
        d2 = fmin(fmin(sqn(a0 - b0), sqn(a0 - b1)), fmin(sqn(a1 - b0), sqn(a1 - b1)));
        dF = d2 - th * th;
    }
    double dc = sqrt(d2);
    double gap = eta * dF / (dc + th);
    double toc = 0.0;
    for (int it = 0; it < 10000; ++it) {
        double lb = (1 - eta) * dF / ((dc + th) * maxDisp);
        if (!isfinite(lb) || lb <= 0.0) return fmax(0.0, fmin(toc, 1.0));
        a0 = a0 + lb * da0; a1 = a1 + lb * da1; b0 = b0 + lb * db0; b1 = b1 + lb * db1;
        d2 = eeDistU(a0, a1, b0, b1);
        dF = d2 - th * th;
        if (dF <= 0) {
            d2 = fmin(fmin(sqn(a0 - b0), sqn(a0 - b1)), fmin(sqn(a1 - b0), sqn(a1 - b1)));
            dF = d2 - th * th;
        }
        dc = sqrt(d2);
        if (toc != 0.0 && (dF / (dc + th) < gap)) return fmax(0.0, fmin(toc, 1.0));
        toc += lb;
        if (toc > 1.0) return 1.0;
    }
    if (status) raiseStatus(status, CIPC_ST_CCD_CAP);
    return fmax(0.0, fmin(toc, 1.0));
}

__device__ inline double pointTriangleCCD(d3 p, d3 t0, d3 t1, d3 t2, d3 dp, d3 dt0, d3 dt1, d3 dt2, double eta, int* status) {
    const double th = 0.0;
    d3 mov = (dt0 + dt1 + dt2 + dp) / 4;
    dt0 = dt0 - mov; dt1 = dt1 - mov; dt2 = dt2 - mov; dp = dp - mov;
    double maxDisp = sqrt(sqn(dp)) + sqrt(fmax(fmax(sqn(dt0), sqn(dt1)), sqn(dt2)));
    if (maxDisp == 0) return 1.0;
    double d2 = ptDistU(p, t0, t1, t2);
    double dc = sqrt(d2);
    double gap = eta * (d2 - th * th) / (dc + th);
    double toc = 0.0;
    for (int it = 0; it < 10000; ++it) {
        double lb = (1 - eta) * (d2 - th * th) / ((dc + th) * maxDisp);
        if (!isfinite(lb) || lb <= 0.0) return fmax(0.0, fmin(toc, 1.0));
        p = p + lb * dp; t0 = t0 + lb * dt0; t1 = t1 + lb * dt1; t2 = t2 + lb * dt2;
        d2 = ptDistU(p, t0, t1, t2);
        dc = sqrt(d2);
        if (toc != 0.0 && ((d2 - th * th) / (dc + th) < gap)) return fmax(0.0, fmin(toc, 1.0));
        toc += lb;
        if (toc > 1.0) return 1.0;
    }
    if (status) raiseStatus(status, CIPC_ST_CCD_CAP);
    return fmax(0.0, fmin(toc, 1.0));
}

__device__ __forceinline__ double det3c(d3 c0, d3 c1, d3 c2) {
    // determinant of the matrix with columns c0, c1, c2
    return c0.x * (c1.y * c2.z - c2.y * c1.z) - c1.x * (c0.y * c2.z - c2.y * c0.z) + c2.x * (c0.y * c1.z - c1.y * c0.z);
}

// Coplanar pairs are skipped as in the reference (IglUtils::segTriIntersect).
// With coplanarTol > 0 so is a segment whose two plane distances are both
// within coplanarTol of zero relative to |n| times its reach from t0:
// rounding on rotated meshes must not report the edges and triangles of one
// flat face as intersecting.  coplanarTol = 0 is the reference's exact rule
// (signs of the plane distances and det == 0 only).
constexpr double COPLANAR_TOL = 1e-12;
__device__ __forceinline__ bool segTriIntersect(d3 e0, d3 e1, d3 t0, d3 t1, d3 t2, double coplanarTol) {
    d3 c0 = t1 - t0, c1 = t2 - t0, c2 = e0 - e1;
    d3 n = cross(c0, c1);
    const double d0 = dot(n, e0 - t0), d1 = dot(n, e1 - t0);
    if (d0 * d1 > 0.0) return false;
    if (coplanarTol > 0.0) {
        const double tol = coplanarTol * sqrt(sqn(n)) * fmax(sqrt(sqn(e0 - t0)), sqrt(sqn(e1 - t0)));
        if (fabs(d0) <= tol && fabs(d1) <= tol) return false;
    }
    double det = det3c(c0, c1, c2);
    if (det == 0.0) return false;
    d3 rhs = e0 - t0;
    double u = det3c(rhs, c1, c2) / det, v = det3c(c0, rhs, c2) / det, t = det3c(c0, c1, rhs) / det;
    return u >= 0.0 && v >= 0.0 && u + v <= 1.0 && t >= 0.0 && t <= 1.0;
}

}  // namespace cipc
