// Test infrastructure only: the FP64 CPU oracle for the IPC Newton pipeline.
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use
// anything under oracle/; the shipped library never links it.
//
// Small fixed-size linear algebra used by the oracle.  Everything is plain
// IEEE double arithmetic compiled with -ffp-contract=off so that operation
// order is reproducible.
#pragma once

#include <array>
#include <cmath>
#include <cstring>
#include <algorithm>

namespace oracle {

struct V3 {
    double x = 0, y = 0, z = 0;
    V3() = default;
    V3(double a, double b, double c) : x(a), y(b), z(c) {}
    double& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
    double operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
};
inline V3 operator+(const V3& a, const V3& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 operator-(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 operator-(const V3& a) { return {-a.x, -a.y, -a.z}; }
inline V3 operator*(double s, const V3& a) { return {s * a.x, s * a.y, s * a.z}; }
inline V3 operator*(const V3& a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 operator/(const V3& a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline V3& operator+=(V3& a, const V3& b) { a.x += b.x; a.y += b.y; a.z += b.z; return a; }
inline V3& operator-=(V3& a, const V3& b) { a.x -= b.x; a.y -= b.y; a.z -= b.z; return a; }
inline double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(const V3& a, const V3& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
inline double sqnorm(const V3& a) { return dot(a, a); }
inline double norm(const V3& a) { return std::sqrt(sqnorm(a)); }
inline V3 normalized(const V3& a) { double n = norm(a); return n > 0 ? a / n : a; }
inline V3 vmin(const V3& a, const V3& b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
inline V3 vmax(const V3& a, const V3& b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }

// Row-major dense matrix with compile-time shape.
template <int R, int C>
struct Mat {
    double a[R][C];
    Mat() { std::memset(a, 0, sizeof(a)); }
    double& operator()(int i, int j) { return a[i][j]; }
    double operator()(int i, int j) const { return a[i][j]; }
    static Mat zero() { return Mat(); }
    static Mat identity() { Mat m; for (int i = 0; i < std::min(R, C); ++i) m.a[i][i] = 1; return m; }
};
template <int N>
struct Vec {
    double v[N];
    Vec() { for (int i = 0; i < N; ++i) v[i] = 0; }
    double& operator[](int i) { return v[i]; }
    double operator[](int i) const { return v[i]; }
};

template <int R, int K, int C>
inline Mat<R, C> mul(const Mat<R, K>& A, const Mat<K, C>& B) {
    Mat<R, C> out;
    for (int i = 0; i < R; ++i)
        for (int j = 0; j < C; ++j) {
            double s = 0;
            for (int k = 0; k < K; ++k) s += A.a[i][k] * B.a[k][j];
            out.a[i][j] = s;
        }
    return out;
}
template <int R, int C>
inline Mat<C, R> transpose(const Mat<R, C>& A) {
    Mat<C, R> out;
    for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) out.a[j][i] = A.a[i][j];
    return out;
}
template <int R, int C>
inline Vec<R> mulv(const Mat<R, C>& A, const Vec<C>& v) {
    Vec<R> out;
    for (int i = 0; i < R; ++i) { double s = 0; for (int k = 0; k < C; ++k) s += A.a[i][k] * v[k]; out[i] = s; }
    return out;
}
template <int N>
inline Mat<N, N> outer(const Vec<N>& u, const Vec<N>& v, double s = 1.0) {
    Mat<N, N> out;
    for (int i = 0; i < N; ++i) for (int j = 0; j < N; ++j) out.a[i][j] = s * u[i] * v[j];
    return out;
}
template <int R, int C>
inline void addScaled(Mat<R, C>& A, const Mat<R, C>& B, double s) {
    for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) A.a[i][j] += s * B.a[i][j];
}
template <int R, int C>
inline void scale(Mat<R, C>& A, double s) {
    for (int i = 0; i < R; ++i) for (int j = 0; j < C; ++j) A.a[i][j] *= s;
}

using M3 = Mat<3, 3>;
inline double det3(const M3& F) {
    return F.a[0][0] * (F.a[1][1] * F.a[2][2] - F.a[1][2] * F.a[2][1])
         - F.a[0][1] * (F.a[1][0] * F.a[2][2] - F.a[1][2] * F.a[2][0])
         + F.a[0][2] * (F.a[1][0] * F.a[2][1] - F.a[1][1] * F.a[2][0]);
}
// Inverse by cofactors (the closed form a 3x3 fixed-size inverse uses).
inline M3 inverse3(const M3& m) {
    M3 inv;
    double c00 = m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1];
    double c10 = m.a[1][2] * m.a[2][0] - m.a[1][0] * m.a[2][2];
    double c20 = m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0];
    double det = m.a[0][0] * c00 + m.a[0][1] * c10 + m.a[0][2] * c20;
    inv.a[0][0] = c00 / det;
    inv.a[1][0] = c10 / det;
    inv.a[2][0] = c20 / det;
    inv.a[0][1] = (m.a[0][2] * m.a[2][1] - m.a[0][1] * m.a[2][2]) / det;
    inv.a[1][1] = (m.a[0][0] * m.a[2][2] - m.a[0][2] * m.a[2][0]) / det;
    inv.a[2][1] = (m.a[0][1] * m.a[2][0] - m.a[0][0] * m.a[2][1]) / det;
    inv.a[0][2] = (m.a[0][1] * m.a[1][2] - m.a[0][2] * m.a[1][1]) / det;
    inv.a[1][2] = (m.a[0][2] * m.a[1][0] - m.a[0][0] * m.a[1][2]) / det;
    inv.a[2][2] = (m.a[0][0] * m.a[1][1] - m.a[0][1] * m.a[1][0]) / det;
    return inv;
}

// Cyclic Jacobi eigen-decomposition of a symmetric N x N matrix.  Used to
// restate the PSD projection of a symmetric block (negative eigenvalues set to
// zero, V D V^T rebuilt).  The projection onto the PSD cone is unique, so any
// accurate eigen-solver reproduces it to round-off.
template <int N>
inline void jacobiEigen(const Mat<N, N>& Ain, Vec<N>& w, Mat<N, N>& V) {
    Mat<N, N> A = Ain;
    V = Mat<N, N>::identity();
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0, diag = 0;
        for (int i = 0; i < N; ++i) {
            diag += A.a[i][i] * A.a[i][i];
            for (int j = i + 1; j < N; ++j) off += A.a[i][j] * A.a[i][j];
        }
        if (off <= 1e-32 * diag || off == 0.0) break;
        for (int p = 0; p < N - 1; ++p)
            for (int q = p + 1; q < N; ++q) {
                double apq = A.a[p][q];
                if (apq == 0.0) continue;
                double app = A.a[p][p], aqq = A.a[q][q];
                double theta = (aqq - app) / (2.0 * apq);
                double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
                double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < N; ++k) {
                    double akp = A.a[k][p], akq = A.a[k][q];
                    A.a[k][p] = c * akp - s * akq;
                    A.a[k][q] = s * akp + c * akq;
                }
                for (int k = 0; k < N; ++k) {
                    double apk = A.a[p][k], aqk = A.a[q][k];
                    A.a[p][k] = c * apk - s * aqk;
                    A.a[q][k] = s * apk + c * aqk;
                }
                for (int k = 0; k < N; ++k) {
                    double vkp = V.a[k][p], vkq = V.a[k][q];
                    V.a[k][p] = c * vkp - s * vkq;
                    V.a[k][q] = s * vkp + c * vkq;
                }
            }
    }
    for (int i = 0; i < N; ++i) w[i] = A.a[i][i];
}

// PSD projection: follows IglUtils::makePD (ContactMechanics.h:27-45): if the
// smallest eigenvalue is non-negative the block is returned unchanged,
// otherwise every negative eigenvalue is clamped to zero.
template <int N>
inline void makePD(Mat<N, N>& H) {
    Vec<N> w; Mat<N, N> V;
    jacobiEigen<N>(H, w, V);
    double wmin = w[0];
    for (int i = 1; i < N; ++i) wmin = std::min(wmin, w[i]);
    if (wmin >= 0.0) return;
    Mat<N, N> out;
    for (int k = 0; k < N; ++k) {
        double lk = w[k] < 0.0 ? 0.0 : w[k];
        if (lk == 0.0) continue;
        for (int i = 0; i < N; ++i) {
            double vik = lk * V.a[i][k];
            for (int j = 0; j < N; ++j) out.a[i][j] += vik * V.a[j][k];
        }
    }
    H = out;
}

// Second-order forward-mode jet: value, gradient and Hessian with respect to
// N independent variables.  The oracle differentiates the plain squared
// distance formulas with it, so its derivatives are exact up to round-off and
// independent of any closed-form derivative code.
template <int N>
struct Jet {
    double v = 0;
    double g[N];
    double h[N][N];
    Jet() { std::memset(g, 0, sizeof(g)); std::memset(h, 0, sizeof(h)); }
    explicit Jet(double c) : Jet() { v = c; }
    static Jet var(double value, int i) { Jet j; j.v = value; j.g[i] = 1.0; return j; }
};
template <int N> inline Jet<N> operator+(const Jet<N>& a, const Jet<N>& b) {
    Jet<N> r; r.v = a.v + b.v;
    for (int i = 0; i < N; ++i) { r.g[i] = a.g[i] + b.g[i]; for (int j = 0; j < N; ++j) r.h[i][j] = a.h[i][j] + b.h[i][j]; }
    return r;
}
template <int N> inline Jet<N> operator-(const Jet<N>& a, const Jet<N>& b) {
    Jet<N> r; r.v = a.v - b.v;
    for (int i = 0; i < N; ++i) { r.g[i] = a.g[i] - b.g[i]; for (int j = 0; j < N; ++j) r.h[i][j] = a.h[i][j] - b.h[i][j]; }
    return r;
}
template <int N> inline Jet<N> operator*(const Jet<N>& a, const Jet<N>& b) {
    Jet<N> r; r.v = a.v * b.v;
    for (int i = 0; i < N; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            r.h[i][j] = a.h[i][j] * b.v + a.v * b.h[i][j] + a.g[i] * b.g[j] + a.g[j] * b.g[i];
    return r;
}
template <int N> inline Jet<N> operator/(const Jet<N>& a, const Jet<N>& b) {
    Jet<N> r; r.v = a.v / b.v;
    for (int i = 0; i < N; ++i) r.g[i] = (a.g[i] - r.v * b.g[i]) / b.v;
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            r.h[i][j] = (a.h[i][j] - r.g[i] * b.g[j] - b.g[i] * r.g[j] - r.v * b.h[i][j]) / b.v;
    return r;
}
template <int N> inline Jet<N> jsqrt(const Jet<N>& a) {
    Jet<N> r; r.v = std::sqrt(a.v);
    for (int i = 0; i < N; ++i) r.g[i] = a.g[i] / (2.0 * r.v);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) r.h[i][j] = a.h[i][j] / (2.0 * r.v) - a.g[i] * a.g[j] / (4.0 * a.v * r.v);
    return r;
}
// atan2(y, x) with its first and second partial derivatives chained in
template <int N> inline Jet<N> jatan2(const Jet<N>& y, const Jet<N>& x) {
    Jet<N> r; r.v = std::atan2(y.v, x.v);
    const double r2 = x.v * x.v + y.v * y.v, r4 = r2 * r2;
    const double ty = x.v / r2, tx = -y.v / r2;                       // d/dy, d/dx
    const double tyy = -2.0 * x.v * y.v / r4, txx = 2.0 * x.v * y.v / r4, txy = (y.v * y.v - x.v * x.v) / r4;
    for (int i = 0; i < N; ++i) r.g[i] = ty * y.g[i] + tx * x.g[i];
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            r.h[i][j] = ty * y.h[i][j] + tx * x.h[i][j] + tyy * y.g[i] * y.g[j] + txx * x.g[i] * x.g[j] +
                        txy * (x.g[i] * y.g[j] + y.g[i] * x.g[j]);
    return r;
}
template <int N> struct JV3 { Jet<N> x, y, z; };
template <int N> inline JV3<N> jsub(const JV3<N>& a, const JV3<N>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <int N> inline Jet<N> jdot(const JV3<N>& a, const JV3<N>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <int N> inline JV3<N> jcross(const JV3<N>& a, const JV3<N>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <int N> inline JV3<N> jvar(const V3& p, int base) {
    return {Jet<N>::var(p.x, base), Jet<N>::var(p.y, base + 1), Jet<N>::var(p.z, base + 2)};
}

}  // namespace oracle
