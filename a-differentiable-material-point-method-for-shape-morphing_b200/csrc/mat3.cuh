// mat3.cuh -- 3x3 register-resident matrix helpers and the cubic B-spline
// kernel shared by every stage.  Host+device so the same arithmetic can be
// unit-tested on the CPU.
#pragma once
#include <cmath>
#include <cuda_runtime.h>

#define DMPM_HD __host__ __device__ __forceinline__

namespace dmpm {

// std::numeric_limits<float>::epsilon(): the node-mass threshold of the
// reference (ForwardSimulation.cpp:55, BackPropagation.cpp:55), kept in every
// precision.
constexpr double kFltEps = 1.1920928955078125e-07;

template <class T> struct m3 {
    T a[3][3];  // a[row][col]
    DMPM_HD T& operator()(int i, int j) { return a[i][j]; }
    DMPM_HD const T& operator()(int i, int j) const { return a[i][j]; }
};

template <class T> DMPM_HD m3<T> m3_zero() {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = T(0);
    return r;
}
template <class T> DMPM_HD m3<T> m3_eye() {
    m3<T> r = m3_zero<T>();
    r.a[0][0] = r.a[1][1] = r.a[2][2] = T(1);
    return r;
}
template <class To, class Ti> DMPM_HD m3<To> m3_cast(const m3<Ti>& A) {
    m3<To> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = (To)A.a[i][j];
    return r;
}
template <class T> DMPM_HD m3<T> operator+(const m3<T>& A, const m3<T>& B) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = A.a[i][j] + B.a[i][j];
    return r;
}
template <class T> DMPM_HD m3<T> operator-(const m3<T>& A, const m3<T>& B) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = A.a[i][j] - B.a[i][j];
    return r;
}
template <class T> DMPM_HD m3<T> operator*(T s, const m3<T>& A) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = s * A.a[i][j];
    return r;
}
template <class T> DMPM_HD m3<T> operator*(const m3<T>& A, const m3<T>& B) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = A.a[i][0] * B.a[0][j] + A.a[i][1] * B.a[1][j] + A.a[i][2] * B.a[2][j];
    return r;
}
// A^T B without forming A^T
template <class T> DMPM_HD m3<T> mtm(const m3<T>& A, const m3<T>& B) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = A.a[0][i] * B.a[0][j] + A.a[1][i] * B.a[1][j] + A.a[2][i] * B.a[2][j];
    return r;
}
// A B^T
template <class T> DMPM_HD m3<T> mmt(const m3<T>& A, const m3<T>& B) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = A.a[i][0] * B.a[j][0] + A.a[i][1] * B.a[j][1] + A.a[i][2] * B.a[j][2];
    return r;
}
template <class T> DMPM_HD m3<T> transpose(const m3<T>& A) {
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = A.a[j][i];
    return r;
}
template <class T> DMPM_HD T ddot(const m3<T>& A, const m3<T>& B) {
    T s = T(0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) s += A.a[i][j] * B.a[i][j];
    return s;
}
// y = A x
template <class T> DMPM_HD void mv(const m3<T>& A, const T* x, T* y) {
#pragma unroll
    for (int i = 0; i < 3; i++) y[i] = A.a[i][0] * x[0] + A.a[i][1] * x[1] + A.a[i][2] * x[2];
}
// y = A^T x
template <class T> DMPM_HD void mtv(const m3<T>& A, const T* x, T* y) {
#pragma unroll
    for (int i = 0; i < 3; i++) y[i] = A.a[0][i] * x[0] + A.a[1][i] * x[1] + A.a[2][i] * x[2];
}

// Cofactor-expansion determinant and inverse in the operation order of
// Eigen's fixed-size 3x3 paths, which the reference uses for F.determinant()
// and F.inverse() (Eigen LU/Determinant.h, LU/InverseImpl.h).
template <class T> DMPM_HD T det3(const m3<T>& m) {
    return m.a[0][0] * (m.a[1][1] * m.a[2][2] - m.a[1][2] * m.a[2][1]) -
           m.a[0][1] * (m.a[1][0] * m.a[2][2] - m.a[1][2] * m.a[2][0]) +
           m.a[0][2] * (m.a[1][0] * m.a[2][1] - m.a[1][1] * m.a[2][0]);
}
template <class T> DMPM_HD T cof3(const m3<T>& m, int i, int j) {
    const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m.a[i1][j1] * m.a[i2][j2] - m.a[i1][j2] * m.a[i2][j1];
}
// F^{-T} = cof(F) / det(F) with det from the first-column cofactors.
template <class T> DMPM_HD m3<T> inv_transpose3(const m3<T>& m) {
    const T c00 = cof3(m, 0, 0), c10 = cof3(m, 1, 0), c20 = cof3(m, 2, 0);
    const T det = c00 * m.a[0][0] + c10 * m.a[1][0] + c20 * m.a[2][0];
    const T id = T(1) / det;
    m3<T> r;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) r.a[i][j] = cof3(m, i, j) * id;  // (F^{-1})_{ji} = cof_{ij} / det
    return r;
}

// ---------------------------------------------------------------- B-spline
// Cubic B-spline N(x) and N'(x) (Interpolation.h:5-30).  The stencil of a point
// is the 4x4x4 block of nodes starting at floor(x_rel / dx) - 1.
template <class T> DMPM_HD T bspline(T x) {
    T ax = x < T(0) ? -x : x;
    if (ax < T(1)) return T(0.5) * ax * ax * ax - ax * ax + T(2) / T(3);
    if (ax < T(2)) return (T(2) - ax) * (T(2) - ax) * (T(2) - ax) / T(6);
    return T(0);
}
template <class T> DMPM_HD T bspline_slope(T x) {
    T ax = x < T(0) ? -x : x;
    if (ax < T(1)) return T(1.5) * x * ax - T(2) * x;
    if (ax < T(2)) return -x * ax / T(2) + T(2) * x - T(2) * x / ax;
    return T(0);
}

// Weights of one axis: for the 4 stencil nodes base+0..3 of a point at
// relative coordinate r (lattice units), the node offsets d_k = (base+k)*dx +
// min - x  and N(d_k/dx), N'(d_k/dx).
template <class T> struct axis_w {
    T d[4], n[4], s[4];
};

// floor(x_rel / dx) - 1 by division, as the reference computes it
// (stencil_base_lattice: floor(r) - 1 of a lattice coordinate r).  The
// result is clamped to [-4, dim]: a stencil starting outside that range has
// no node inside the grid either way, and the clamp keeps all later index
// arithmetic (tile extents, node indices) bounded for any input, including
// non-finite positions.
template <class T> DMPM_HD int stencil_base_lattice(T r, int dim) {
    const T q = floor(r);
    int b;
    if (!(q > T(-8))) b = -8;                    // also catches NaN
    else if (q > T(dim + 8)) b = dim + 8;
    else b = (int)q;
    b -= 1;
    return b < -4 ? -4 : (b > dim ? dim : b);
}
template <class T> DMPM_HD int stencil_base(T xrel, T dx, int dim) { return stencil_base_lattice<T>(xrel / dx, dim); }

template <class T> DMPM_HD void axis_weights(T x, T mn, T dx, int base, axis_w<T>& w, bool slopes) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const T xg = mn + (T)(base + k) * dx;
        const T d = xg - x;
        const T q = d / dx;
        w.d[k] = d;
        w.n[k] = bspline(q);
        w.s[k] = slopes ? bspline_slope(q) : T(0);
    }
}
// the same from the lattice coordinate t = (x - mn) / dx - base: d_k = (k - t) dx
template <class T> DMPM_HD void axis_weights_lattice(T t, T dx, axis_w<T>& w, bool slopes) {
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const T q = (T)k - t;
        w.d[k] = q * dx;
        w.n[k] = bspline(q);
        w.s[k] = slopes ? bspline_slope(q) : T(0);
    }
}

}  // namespace dmpm
