// elasticity.cuh -- fixed-corotated first Piola-Kirchhoff stress and its
// derivative applied to a direction, in registers.
//
//   P(F)        = 2 mu (F - R) + lam (J - 1) J F^{-T},  J = max(det F, 1e-6)
//                 (PK_FixedCorotatedElasticity, Elasticity.cpp:88-98)
//   dP(F)[dF]   = 2 mu (dF - dR) + lam (J F^{-T} : dF) J F^{-T}
//                 + lam (J - 1) d(J F^{-T})[dF]
//                 (d2_FCE_psi_dF2_mult_by_dF, Elasticity.cpp:100-178)
// dR comes from the polar factors: with X = R^T dR skew, X S + S X =
// R^T dF - dF^T R, a 3x3 linear system in the axial vector of X whose rows and
// unknown order are those of Elasticity.cpp:138-171.
//
// Two variants of d(J F^{-T})[dF]:
//   REFCOMPAT: the reference's central finite differences of J F^{-T} with
//              delta = 1e-6 (d_JFit_dF_FD, Elasticity.cpp:7-72), and its
//              conditioning guard (log|det A| > 20 => A += 1e-4 I, :155-159);
//   EXACT:     the analytic J [(F^{-T}:dF) F^{-T} - F^{-T} dF^T F^{-T}] (zero
//              derivative of J where the clamp is active), no guard.
// Because P is the gradient of an energy, dP/dF is self-adjoint, so applying
// it to dL/dP gives dL/dF; the reference relies on the same identity.
#pragma once
#include "svd3.cuh"

namespace dmpm {

template <class T> DMPM_HD m3<T> pk_from_polar(const m3<T>& F, const m3<T>& R, T lam, T mu) {
    T J = det3(F);
    J = J > T(1e-6) ? J : T(1e-6);
    const m3<T> Fit = inv_transpose3(F);
    const T c = lam * (J - T(1)) * J;
    m3<T> P;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) P.a[i][j] = T(2) * mu * (F.a[i][j] - R.a[i][j]) + c * Fit.a[i][j];
    return P;
}

template <class T> DMPM_HD m3<T> pk_stress(const m3<T>& F, T lam, T mu) {
    m3<T> R, S;
    polar3(F, R, S);
    return pk_from_polar(F, R, lam, mu);
}

// dR = R X,  X = [x]_x,  A x = b  (Cramer's rule).
template <class T> DMPM_HD m3<T> rotation_derivative(const m3<T>& R, const m3<T>& S, const m3<T>& dF, bool guard) {
    m3<T> A;
    A.a[0][0] = S.a[0][2]; A.a[0][1] = S.a[1][2]; A.a[0][2] = -(S.a[0][0] + S.a[1][1]);
    A.a[1][0] = -S.a[0][1]; A.a[1][1] = S.a[0][0] + S.a[2][2]; A.a[1][2] = -S.a[1][2];
    A.a[2][0] = -(S.a[1][1] + S.a[2][2]); A.a[2][1] = S.a[0][1]; A.a[2][2] = S.a[0][2];
    T D = det3(A);
    if (guard && log(fabs(D)) > T(20)) {
        A.a[0][0] += T(1e-4); A.a[1][1] += T(1e-4); A.a[2][2] += T(1e-4);
        D = det3(A);
    }
    const m3<T> t = mtm(R, dF) - mtm(dF, R);  // R^T dF - dF^T R
    const T b[3] = {t.a[0][1], t.a[0][2], t.a[1][2]};
    T x[3];
    const T id = T(1) / D;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        m3<T> M = A;
#pragma unroll
        for (int i = 0; i < 3; i++) M.a[i][c] = b[i];
        x[c] = det3(M) * id;
    }
    m3<T> X = m3_zero<T>();
    X.a[0][1] = -x[2]; X.a[0][2] = x[1];
    X.a[1][0] = x[2];  X.a[1][2] = -x[0];
    X.a[2][0] = -x[1]; X.a[2][1] = x[0];
    return R * X;
}

// sum_ij d(J F^{-T})_ab / dF_ij dF_ij by central differences, delta = 1e-6.
template <class T> DMPM_HD m3<T> djfit_fd_mult(const m3<T>& F, const m3<T>& dF) {
    const T delta = T(1e-6);
    m3<T> acc = m3_zero<T>();
    m3<T> G = F;
#pragma unroll
    for (int ij = 0; ij < 9; ij++) {
        const int i = ij / 3, j = ij % 3;  // row-major sweep and contraction order, as Elasticity.cpp:126-140
        const T orig = G.a[i][j];
        G.a[i][j] = orig + delta;
        const T Jp = det3(G);
        const m3<T> fwd = Jp * inv_transpose3(G);
        G.a[i][j] = orig - delta;
        const T Jm = det3(G);
        const m3<T> bwd = Jm * inv_transpose3(G);
        G.a[i][j] = orig;
        const T w = dF.a[i][j];
#pragma unroll
        for (int a = 0; a < 3; a++)
#pragma unroll
            for (int b = 0; b < 3; b++) acc.a[a][b] += (T)((fwd.a[a][b] - bwd.a[a][b]) / (T(2) * delta)) * w;
    }
    return acc;
}

template <bool EXACT, class T>
DMPM_HD m3<T> d2_mult_from_polar(const m3<T>& F, const m3<T>& R, const m3<T>& S, T lam, T mu, const m3<T>& dF) {
    const T detF = det3(F);
    const m3<T> Fit = inv_transpose3(F);
    m3<T> ret = (T(2) * mu) * dF;
    if (!EXACT) {
        const T J = detF > T(1e-6) ? detF : T(1e-6);
        ret = ret + (lam * J * ddot(J * Fit, dF)) * Fit;
        ret = ret + (lam * (J - T(1))) * djfit_fd_mult(F, dF);
        ret = ret - (T(2) * mu) * rotation_derivative(R, S, dF, true);
    } else {
        const bool clamped = !(detF > T(1e-6));
        const T J = clamped ? T(1e-6) : detF;
        const m3<T> FdF = Fit * mtm(dF, Fit);  // F^{-T} dF^T F^{-T}
        if (!clamped) {
            const T c = ddot(Fit, dF);
            ret = ret + (lam * J * J * c) * Fit;
            ret = ret + (lam * (J - T(1)) * J) * (c * Fit - FdF);
        } else {
            ret = ret - (lam * (J - T(1)) * J) * FdF;
        }
        ret = ret - (T(2) * mu) * rotation_derivative(R, S, dF, false);
    }
    return ret;
}

template <bool EXACT, class T> DMPM_HD m3<T> d2_mult(const m3<T>& F, T lam, T mu, const m3<T>& dF) {
    m3<T> R, S;
    polar3(F, R, S);
    return d2_mult_from_polar<EXACT>(F, R, S, lam, mu, dF);
}

}  // namespace dmpm
