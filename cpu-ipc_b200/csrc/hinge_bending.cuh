// Dihedral-angle (hinge) bending element math, host and device: the bending
// model of the reference's build without USE_QUADRATIC_BENDING
// (CPU IPC/HingeBending.cpp:45-106, angle derivatives CPU IPC/Elasticity.cpp:
// 12-150).  Energy 0.5 k w d^2 with d = remainder(theta - theta0, 2 pi),
// w = l0^2 / (2 A0 + 2 A1) from the rest shape; gradient k w d grad(theta);
// Hessian k w (grad(theta) grad(theta)^T + d hess(theta)) before the PSD
// projection the caller applies.
//
// theta is the signed angle about the edge x0 -> x1 between the normals
// n0 = e x (x2 - x0) and n1 = (x3 - x0) x e (zero for two coplanar, unfolded
// triangles).  Its gradient is the closed form of the classical bending
// force directions: the opposite vertices move along their triangle's normal
// with magnitude 1 / (distance to the edge), the edge vertices take the
// negated combination weighted by where the opposite vertices project onto
// the edge.  The Hessian is the forward-mode derivative of that closed form
// (12 directional derivatives carried with every value).
#pragma once

#include <cmath>

#if defined(__CUDACC__)
#define HINGE_HD __host__ __device__ __forceinline__
#else
#define HINGE_HD inline
#endif

namespace cipc {
namespace hinge {

// value with its derivatives along the 12 coordinates (x0, x1, x2, x3)
struct Dual {
    double v;
    double d[12];
};
HINGE_HD Dual dconst(double c) {
    Dual r;
    r.v = c;
    for (int i = 0; i < 12; ++i) r.d[i] = 0.0;
    return r;
}
HINGE_HD Dual operator+(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v + b.v;
    for (int i = 0; i < 12; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
HINGE_HD Dual operator-(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v - b.v;
    for (int i = 0; i < 12; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
HINGE_HD Dual operator-(const Dual& a) {
    Dual r;
    r.v = -a.v;
    for (int i = 0; i < 12; ++i) r.d[i] = -a.d[i];
    return r;
}
HINGE_HD Dual operator*(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v * b.v;
    for (int i = 0; i < 12; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
HINGE_HD Dual operator/(const Dual& a, const Dual& b) {
    Dual r;
    r.v = a.v / b.v;
    for (int i = 0; i < 12; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) / b.v;
    return r;
}
HINGE_HD Dual dsqrt(const Dual& a) {
    Dual r;
    r.v = sqrt(a.v);
    for (int i = 0; i < 12; ++i) r.d[i] = a.d[i] / (2.0 * r.v);
    return r;
}
HINGE_HD Dual datan2(const Dual& y, const Dual& x) {
    Dual r;
    r.v = atan2(y.v, x.v);
    const double q = x.v * x.v + y.v * y.v;
    for (int i = 0; i < 12; ++i) r.d[i] = (x.v * y.d[i] - y.v * x.d[i]) / q;
    return r;
}

// value with its derivative along one coordinate: a GPU kernel gives each
// of 12 lanes one coordinate and gets one Hessian column per lane
struct Dual1 {
    double v, d;
};
HINGE_HD Dual1 operator+(const Dual1& a, const Dual1& b) { return {a.v + b.v, a.d + b.d}; }
HINGE_HD Dual1 operator-(const Dual1& a, const Dual1& b) { return {a.v - b.v, a.d - b.d}; }
HINGE_HD Dual1 operator-(const Dual1& a) { return {-a.v, -a.d}; }
HINGE_HD Dual1 operator*(const Dual1& a, const Dual1& b) { return {a.v * b.v, a.d * b.v + a.v * b.d}; }
HINGE_HD Dual1 operator/(const Dual1& a, const Dual1& b) {
    const double q = a.v / b.v;
    return {q, (a.d - q * b.d) / b.v};
}

HINGE_HD double sqrtT(double a) { return sqrt(a); }
HINGE_HD Dual sqrtT(const Dual& a) { return dsqrt(a); }
HINGE_HD Dual1 sqrtT(const Dual1& a) {
    const double r = sqrt(a.v);
    return {r, a.d / (2.0 * r)};
}
HINGE_HD double constT(double, double c) { return c; }
HINGE_HD Dual constT(const Dual&, double c) { return dconst(c); }
HINGE_HD Dual1 constT(const Dual1&, double c) { return {c, 0.0}; }

template <class T>
struct Vec3 {
    T x, y, z;
};
template <class T>
HINGE_HD Vec3<T> vsub(const Vec3<T>& a, const Vec3<T>& b) {
    return {a.x - b.x, a.y - b.y, a.z - b.z};
}
template <class T>
HINGE_HD Vec3<T> vadd(const Vec3<T>& a, const Vec3<T>& b) {
    return {a.x + b.x, a.y + b.y, a.z + b.z};
}
template <class T>
HINGE_HD Vec3<T> vneg(const Vec3<T>& a) {
    return {-a.x, -a.y, -a.z};
}
template <class T>
HINGE_HD Vec3<T> vscale(const T& s, const Vec3<T>& a) {
    return {s * a.x, s * a.y, s * a.z};
}
template <class T>
HINGE_HD T vdot(const Vec3<T>& a, const Vec3<T>& b) {
    return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <class T>
HINGE_HD Vec3<T> vcross(const Vec3<T>& a, const Vec3<T>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

// theta (value only); x holds x0, x1, x2, x3
HINGE_HD double angle(const double* x) {
    const Vec3<double> p0{x[0], x[1], x[2]}, p1{x[3], x[4], x[5]}, p2{x[6], x[7], x[8]}, p3{x[9], x[10], x[11]};
    const Vec3<double> e = vsub(p1, p0);
    const Vec3<double> n0 = vcross(e, vsub(p2, p0)), n1 = vcross(vsub(p3, p0), e);
    return atan2(vdot(vcross(n0, n1), e) / sqrt(vdot(e, e)), vdot(n0, n1));
}

// grad(theta) in closed form, for T = double, or Dual (whose derivatives then
// give the rows of hess(theta)); out[k] is the gradient at vertex k
template <class T>
HINGE_HD void angleGrad(const Vec3<T>& p0, const Vec3<T>& p1, const Vec3<T>& p2, const Vec3<T>& p3, Vec3<T> out[4]) {
    const Vec3<T> e = vsub(p1, p0), a = vsub(p2, p0), b = vsub(p3, p0);
    const Vec3<T> n0 = vcross(e, a), n1 = vcross(b, e);
    const T ee = vdot(e, e);
    const T el = sqrtT(ee);
    // an opposite vertex turns its triangle about the edge: moving it along
    // the triangle's normal by h changes theta by -h / (its distance to the
    // edge), the distance being |n| / |e|
    out[2] = vscale(-el / vdot(n0, n0), n0);
    out[3] = vscale(-el / vdot(n1, n1), n1);
    // the edge vertices take the rest, split by where the opposite vertices
    // project onto the edge (t = 0 at x0, 1 at x1)
    const T t2 = vdot(a, e) / ee, t3 = vdot(b, e) / ee;
    const T one = constT(ee, 1.0);
    out[1] = vneg(vadd(vscale(t2, out[2]), vscale(t3, out[3])));
    out[0] = vneg(vadd(vscale(one - t2, out[2]), vscale(one - t3, out[3])));
}

// column j of hess(theta) (= row j, the Hessian being symmetric): the
// derivative of the closed-form gradient along coordinate j
HINGE_HD void angleHessColumn(const double* x, int j, double* col) {
    Vec3<Dual1> p[4];
    for (int v = 0; v < 4; ++v) {
        Dual1 c[3];
        for (int q = 0; q < 3; ++q) c[q] = Dual1{x[3 * v + q], 3 * v + q == j ? 1.0 : 0.0};
        p[v] = Vec3<Dual1>{c[0], c[1], c[2]};
    }
    Vec3<Dual1> gr[4];
    angleGrad(p[0], p[1], p[2], p[3], gr);
    for (int v = 0; v < 4; ++v) {
        col[3 * v] = gr[v].x.d;
        col[3 * v + 1] = gr[v].y.d;
        col[3 * v + 2] = gr[v].z.d;
    }
}

// rest weight l0^2 / (2 A0 + 2 A1) of a hinge given its rest positions
HINGE_HD double restWeight(const double* r) {
    const Vec3<double> p0{r[0], r[1], r[2]}, p1{r[3], r[4], r[5]}, p2{r[6], r[7], r[8]}, p3{r[9], r[10], r[11]};
    const Vec3<double> e = vsub(p1, p0);
    const Vec3<double> c0 = vcross(e, vsub(p2, p0)), c1 = vcross(e, vsub(p3, p0));
    return vdot(e, e) / (sqrt(vdot(c0, c0)) + sqrt(vdot(c1, c1)));
}

// energy 0.5 k w d^2; g (12) = k w d grad(theta); H (144, row-major, not yet
// projected) = k w (grad grad^T + d hess(theta))
HINGE_HD double energyGradHess(const double* x, double w, double theta0, double k, double* g, double* H) {
    Vec3<Dual> p[4];
    for (int v = 0; v < 4; ++v) {
        Dual c[3];
        for (int q = 0; q < 3; ++q) {
            c[q] = dconst(x[3 * v + q]);
            c[q].d[3 * v + q] = 1.0;
        }
        p[v] = Vec3<Dual>{c[0], c[1], c[2]};
    }
    Vec3<Dual> gr[4];
    angleGrad(p[0], p[1], p[2], p[3], gr);
    const double d = remainder(angle(x) - theta0, 6.28318530717958647692);
    const double s = k * w;
    double tg[12];
    for (int v = 0; v < 4; ++v) {
        tg[3 * v] = gr[v].x.v;
        tg[3 * v + 1] = gr[v].y.v;
        tg[3 * v + 2] = gr[v].z.v;
    }
    if (g)
        for (int i = 0; i < 12; ++i) g[i] = s * d * tg[i];
    if (H)
        for (int v = 0; v < 4; ++v)
            for (int q = 0; q < 3; ++q) {
                const Dual& c = q == 0 ? gr[v].x : (q == 1 ? gr[v].y : gr[v].z);
                const int i = 3 * v + q;
                for (int j = 0; j < 12; ++j) H[12 * i + j] = s * (tg[i] * tg[j] + d * c.d[j]);
            }
    return 0.5 * s * d * d;
}

}  // namespace hinge
}  // namespace cipc
