// svd3.cuh -- 3x3 singular value and polar decompositions in registers.
//
// Method: the implicit-shifted symmetric QR SVD for 3x3 matrices of Gast, Fu,
// Jiang and Teran (UCLA technical report, 2016), the method the reference uses
// through include/qrsvd/ImplicitQRSVD.h (polarDecomposition, :863-877):
//   1. Givens rotations reduce A to upper bidiagonal B = U^T A V;
//   2. implicit QR sweeps with a Wilkinson shift taken from the trailing 2x2
//      block of B^T B, each sweep chasing the bulge back to bidiagonal form,
//      until one super-diagonal or diagonal entry of B is negligible;
//   3. the remaining coupled 2x2 block is diagonalised by a 2x2 SVD (a Givens
//      rotation that makes the block symmetric, then a Jacobi rotation);
//   4. singular values are ordered by decreasing magnitude.
// Convention (the reference's "rotation variant"): U and V are rotations,
// |s0| >= |s1| >= |s2|, s0 and s1 are non-negative, and s2 carries the sign
// of det(A).  With that convention R = U V^T and S = V diag(s) V^T are unique
// for distinct |s_i|, so they match the reference's polar factors up to
// rounding whatever path the iteration took.
//
// Givens rotation convention used throughout: g = (c, s) acts on rows (i, k)
// as  row_i <- c row_i - s row_k,  row_k <- s row_i + c row_k,  and on columns
// (i, k) the same way.  givens(a, b) returns c = a/r, s = -b/r so that the
// rotation maps (a, b) to (r, 0).
#pragma once
#include "mat3.cuh"

namespace dmpm {

template <class T> struct givens_t { T c, s; };

template <class T> DMPM_HD givens_t<T> givens(T a, T b) {
    givens_t<T> g{T(1), T(0)};
    const T d = a * a + b * b;
    if (d != T(0)) {
        const T t = T(1) / sqrt(d);
        g.c = a * t;
        g.s = -b * t;
    }
    return g;
}
// Rotation mapping (a, b) to (0, r): c = b/r, s = a/r.
template <class T> DMPM_HD givens_t<T> givens_to_zero_first(T a, T b) {
    givens_t<T> g{T(0), T(1)};
    const T d = a * a + b * b;
    if (d != T(0)) {
        const T t = T(1) / sqrt(d);
        g.s = a * t;
        g.c = b * t;
    }
    return g;
}
template <class T> DMPM_HD void rot_rows(m3<T>& A, int i, int k, givens_t<T> g) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const T x = A.a[i][j], y = A.a[k][j];
        A.a[i][j] = g.c * x - g.s * y;
        A.a[k][j] = g.s * x + g.c * y;
    }
}
template <class T> DMPM_HD void rot_cols(m3<T>& A, int i, int k, givens_t<T> g) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const T x = A.a[j][i], y = A.a[j][k];
        A.a[j][i] = g.c * x - g.s * y;
        A.a[j][k] = g.s * x + g.c * y;
    }
}

// Chase a bidiagonal matrix whose only off-pattern entry is B(1,0) back to
// upper bidiagonal form (B(2,0) must already be zero).  Row rotations are
// accumulated into U, column rotations into V, keeping A = U B V^T.
template <class T> DMPM_HD void chase_to_bidiagonal(m3<T>& B, m3<T>& U, m3<T>& V) {
    givens_t<T> g = givens(B.a[0][0], B.a[1][0]);  // zero B(1,0); fills B(0,2)
    rot_rows(B, 0, 1, g);
    rot_cols(U, 0, 1, g);
    g = givens(B.a[0][1], B.a[0][2]);               // zero B(0,2); fills B(2,1)
    rot_cols(B, 1, 2, g);
    rot_cols(V, 1, 2, g);
    g = givens(B.a[1][1], B.a[2][1]);               // zero B(2,1)
    rot_rows(B, 1, 2, g);
    rot_cols(U, 1, 2, g);
    B.a[1][0] = T(0);
    B.a[0][2] = T(0);
    B.a[2][1] = T(0);
}

// 2x2 SVD of M = [[a, b], [c, d]] = Ru diag(s0, s1) Rv^T with Ru, Rv
// rotations, |s0| >= |s1|, s0 >= 0.  Returned as Givens pairs in the
// rot_cols convention (applying rot_cols(X, i, k, gu) post-multiplies X by Ru).
template <class T> DMPM_HD void svd2(T a, T b, T c, T d, givens_t<T>& gu, T& s0, T& s1, givens_t<T>& gv) {
    // Rotation Q with Q^T M symmetric: (cos, sin) proportional to (a + d, c - b).
    T x = a + d, y = c - b;
    T r = sqrt(x * x + y * y);
    T cq = T(1), sq = T(0);
    if (r != T(0)) { cq = x / r; sq = y / r; }
    // S = Q^T M with Q = [[cq, -sq], [sq, cq]]
    const T s00 = cq * a + sq * c, s01 = cq * b + sq * d, s11 = -sq * b + cq * d;
    // symmetric eigen-decomposition S = W diag(e0, e1) W^T
    T cw = T(1), sw = T(0), e0 = s00, e1 = s11;
    if (s01 != T(0)) {
        const T tau = T(0.5) * (s00 - s11);
        const T w = sqrt(tau * tau + s01 * s01);
        const T t = (tau > T(0)) ? s01 / (tau + w) : s01 / (tau - w);
        cw = T(1) / sqrt(t * t + T(1));
        sw = -t * cw;
        const T c2 = cw * cw, s2 = sw * sw, csy = T(2) * cw * sw * s01;
        e0 = c2 * s00 - csy + s2 * s11;
        e1 = s2 * s00 + csy + c2 * s11;
    }
    // W = [[cw, sw], [-sw, cw]] diagonalises S with the values above.
    // Order by magnitude; the polar step already placed any negative sign on
    // the smaller value.
    T w00 = cw, w01 = sw, w10 = -sw, w11 = cw;
    if (fabs(e0) < fabs(e1) || (fabs(e0) == fabs(e1) && e0 < e1)) {
        T t = e0; e0 = e1; e1 = t;
        // swap columns and negate the new second column (keeps det = +1)
        T n00 = w01, n10 = w11, n01 = -w00, n11 = -w10;
        w00 = n00; w10 = n10; w01 = n01; w11 = n11;
    }
    if (e0 < T(0)) { e0 = -e0; e1 = -e1; w00 = -w00; w10 = -w10; w01 = -w01; w11 = -w11;  // U = Q W D, D = -I
        // V = W, U = Q W (-I): keep both rotations by moving the sign into U
        // only when needed below.
        cq = -cq; sq = -sq; }
    // Rv = W; Ru = Q W.  Express as Givens pairs: a rotation matrix
    // [[c, s], [-s, c]] in rot_cols convention has (c, s) = (m00, m01).
    gv.c = w00; gv.s = w01;
    const T u00 = cq * w00 - sq * w10, u01 = cq * w01 - sq * w11;
    gu.c = u00; gu.s = u01;
    s0 = e0; s1 = e1;
}

// Swap columns i and k of X and negate the new column k (keeps det X).
template <class T> DMPM_HD void swap_cols_keep_det(m3<T>& X, int i, int k) {
#pragma unroll
    for (int j = 0; j < 3; j++) {
        const T t = X.a[j][i];
        X.a[j][i] = X.a[j][k];
        X.a[j][k] = -t;
    }
}
template <class T> DMPM_HD void negate_col(m3<T>& X, int i) {
#pragma unroll
    for (int j = 0; j < 3; j++) X.a[j][i] = -X.a[j][i];
}

template <class T> DMPM_HD void svd3(const m3<T>& A, m3<T>& U, T sig[3], m3<T>& V) {
    m3<T> B = A;
    U = m3_eye<T>();
    V = m3_eye<T>();
    // 1. upper bidiagonal: zero B(2,0), then chase.
    {
        givens_t<T> g = givens(B.a[1][0], B.a[2][0]);
        rot_rows(B, 1, 2, g);
        rot_cols(U, 1, 2, g);
        B.a[2][0] = T(0);
        chase_to_bidiagonal(B, U, V);
    }
    const T eps = sizeof(T) == 4 ? T(1.1920928955078125e-07) : T(2.220446049250313e-16);
    T a1 = B.a[0][0], b1 = B.a[0][1], a2 = B.a[1][1], b2 = B.a[1][2], a3 = B.a[2][2];
    T tol = T(128) * eps;
    {
        T sc = T(0.5) * sqrt(a1 * a1 + a2 * a2 + a3 * a3 + b1 * b1 + b2 * b2);
        tol *= (sc > T(1) ? sc : T(1));
    }
    // 2. implicit-shift QR sweeps
    for (int it = 0; it < 64; it++) {
        if (!(fabs(b2) > tol && fabs(b1) > tol && fabs(a1) > tol && fabs(a2) > tol && fabs(a3) > tol)) break;
        // Wilkinson shift of [[a2^2 + b1^2, a2 b2], [a2 b2, a3^2 + b2^2]]
        const T t11 = a2 * a2 + b1 * b1, t12 = a2 * b2, t22 = a3 * a3 + b2 * b2;
        const T dd = T(0.5) * (t11 - t22);
        const T bs = t12 * t12;
        const T mu = t22 - copysign(bs / (fabs(dd) + sqrt(dd * dd + bs)), dd);
        givens_t<T> g = givens(a1 * a1 - mu, a1 * b1);
        rot_cols(B, 0, 1, g);
        rot_cols(V, 0, 1, g);
        chase_to_bidiagonal(B, U, V);
        a1 = B.a[0][0]; b1 = B.a[0][1]; a2 = B.a[1][1]; b2 = B.a[1][2]; a3 = B.a[2][2];
    }
    // 3. deflation
    int block;  // top-left row/col of the coupled 2x2 block (0 or 1)
    if (fabs(b2) <= tol) {
        block = 0;
    } else if (fabs(b1) <= tol) {
        block = 1;
    } else if (fabs(a2) <= tol) {
        // zero row 1: rotate rows (1,2) to kill B(1,2); row 1 becomes zero
        givens_t<T> g = givens_to_zero_first(B.a[1][2], B.a[2][2]);
        rot_rows(B, 1, 2, g);
        rot_cols(U, 1, 2, g);
        block = 0;
    } else if (fabs(a3) <= tol) {
        // zero column 2: kill B(1,2) with columns (1,2), then B(0,2) with (0,2)
        givens_t<T> g = givens(B.a[1][1], B.a[1][2]);
        rot_cols(B, 1, 2, g);
        rot_cols(V, 1, 2, g);
        g = givens(B.a[0][0], B.a[0][2]);
        rot_cols(B, 0, 2, g);
        rot_cols(V, 0, 2, g);
        block = 0;
    } else {
        // |a1| small: zero row 0 with rows (0,1) then (0,2)
        givens_t<T> g = givens_to_zero_first(B.a[0][1], B.a[1][1]);
        rot_rows(B, 0, 1, g);
        rot_cols(U, 0, 1, g);
        g = givens_to_zero_first(B.a[0][2], B.a[2][2]);
        rot_rows(B, 0, 2, g);
        rot_cols(U, 0, 2, g);
        block = 1;
    }
    {
        // two explicit branches keep every matrix index a compile-time constant
        givens_t<T> gu, gv;
        T s0, s1;
        if (block == 0) {
            svd2(B.a[0][0], B.a[0][1], B.a[1][0], B.a[1][1], gu, s0, s1, gv);
            rot_cols(U, 0, 1, gu);
            rot_cols(V, 0, 1, gv);
            sig[0] = s0;
            sig[1] = s1;
            sig[2] = B.a[2][2];
        } else {
            svd2(B.a[1][1], B.a[1][2], B.a[2][1], B.a[2][2], gu, s0, s1, gv);
            rot_cols(U, 1, 2, gu);
            rot_cols(V, 1, 2, gv);
            sig[1] = s0;
            sig[2] = s1;
            sig[0] = B.a[0][0];
        }
    }
    // 4. order by decreasing magnitude (swaps keep U, V rotations)
#pragma unroll
    for (int pass = 0; pass < 2; pass++) {
#pragma unroll
        for (int i = 0; i < 2; i++) {
            if (fabs(sig[i]) < fabs(sig[i + 1])) {
                const T t = sig[i]; sig[i] = sig[i + 1]; sig[i + 1] = t;
                swap_cols_keep_det(U, i, i + 1);
                swap_cols_keep_det(V, i, i + 1);
            }
        }
    }
    // signs: s0, s1 >= 0; the sign of det A ends on s2
#pragma unroll
    for (int i = 0; i < 2; i++) {
        if (sig[i] < T(0)) {
            sig[i] = -sig[i];
            sig[2] = -sig[2];
            negate_col(U, i);
            negate_col(U, 2);
        }
    }
}

// polarDecomposition: F = R S with R = U V^T a rotation and S = V diag(s) V^T.
template <class T> DMPM_HD void polar3(const m3<T>& F, m3<T>& R, m3<T>& S) {
    m3<T> U, V;
    T s[3];
    svd3(F, U, s, V);
    R = mmt(U, V);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++)
            S.a[i][j] = V.a[i][0] * s[0] * V.a[j][0] + V.a[i][1] * s[1] * V.a[j][1] + V.a[i][2] * s[2] * V.a[j][2];
}

// one scaled Newton step X <- (z X + c X^-T) / 2, c = cbrt(det X), z = 1 / c;
// true when the squared change is at most tol times the squared norm
template <class T> DMPM_HD bool newton_step(m3<T>& X, T tol) {
    const m3<T> Xit = inv_transpose3(X);
    const T c = cbrt(det3(X));
    const T z = T(1) / c;
    T diff = T(0), nrm = T(0);
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const T y = T(0.5) * (z * X.a[i][j] + c * Xit.a[i][j]);
            diff += (y - X.a[i][j]) * (y - X.a[i][j]);
            nrm += y * y;
            X.a[i][j] = y;
        }
    return diff <= tol * nrm;
}


// Polar decomposition F = R S of a matrix with det F > 0 by the scaled Newton
// iteration  X <- (z X + X^{-T} / z) / 2,  z = det(X)^{-1/3}  (Higham 1986,
// determinant scaling), which converges quadratically to the rotation of the
// polar decomposition -- for det F > 0 the same R that polar3 obtains from
// the SVD -- in a few inverse-transposes instead of an SVD.  Returns false,
// leaving R and S unset, when det F is not comfortably positive or the
// iteration has not converged in 24 steps; the caller then uses polar3, whose
// rotation-variant convention the reference relies on for inverted F.
template <class T> DMPM_HD bool polar_newton(const m3<T>& F, m3<T>& R, m3<T>& S) {
    if (!(det3(F) > T(1e-6))) return false;
    m3<T> X = F;
    bool done = false;
    // Near convergence the iteration is quadratic: a step that changes X by a relative
    // delta leaves an error of about delta^2, so once a step changes X by less than
    // 1e-9 (squared: 1e-18) X is within FP64 rounding of R.
    for (int it = 0; it < 24 && !done; it++) done = newton_step<T>(X, T(1e-18));
    if (!done) return false;
    R = X;
    const m3<T> M = mtm(R, F);  // R^T F, symmetric up to rounding
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) S.a[i][j] = T(0.5) * (M.a[i][j] + M.a[j][i]);
    return true;
}

}  // namespace dmpm
