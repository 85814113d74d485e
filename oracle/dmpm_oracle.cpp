// dmpm_oracle.cpp -- CPU restatement of the reference's hot path, used ONLY as a
// test checker (tests/, __graft_entry__.smoke(), and bench.py's CPU-baseline
// leg).  The product never links or calls this file.
//
// It restates, in plain serial C++ templated on the scalar type T (float or
// double), the algorithm of DiffMPMLib3D (paths relative to the reference
// project):
//   Interpolation.h:5-30            cubic B-spline N(x) and N'(x)
//   Elasticity.cpp:88-98            fixed-corotated first Piola-Kirchhoff stress
//   Elasticity.cpp:7-72,100-178     dP/dF : dF with the finite-difference
//                                   d(J F^-T)/dF and the polar-derivative solve
//   ForwardSimulation.cpp:6-124     P_op_1, P2G, G_op, G2P, P_op_2 (+ smoothing)
//   ForwardSimulation.cpp:262-290   CalculatePointCloudVolumes
//   CompGraph.cpp:7-17,110-267      SetUpCompGraph, EndLayerMassLoss,
//                                   ComputeForwardPass, ComputeBackwardPass
//   BackPropagation.cpp:6-125       Back_Timestep
// plus an "exact" adjoint (the true derivative of the same forward map; see
// back_timestep) that differs from the reference's in the terms the reference
// gets wrong.
//
// Matrices are 3x3 column-major (element (i,j) at a[i + 3*j]), the storage of
// the reference's Eigen::Matrix3f, so arrays cross the C ABI unchanged.
//
// The polar decomposition uses an independent method (one-sided Jacobi SVD in
// long double) rather than the reference's implicit-shift QR; for non-degenerate
// F both give the same R and S up to rounding.  Its sign convention is the
// reference's (JIXIE, include/qrsvd/ImplicitQRSVD.h:687-877): U and V are
// rotations, singular values sorted by decreasing magnitude, and only the last
// may be negative.
//
// Parity pin: tests/test_oracle_pin.py checks this file against golden vectors
// produced by the reference itself (tests/golden/make_golden.py).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

namespace oracle {

typedef long double LD;
static const double kFltEps = 1.1920928955078125e-07;  // std::numeric_limits<float>::epsilon()

// ---------------------------------------------------------------- B-spline
// Interpolation.h:5-17
template <class T> T bspline(T x) {
    x = std::fabs(x);
    if (T(0) <= x && x < T(1)) return T(0.5) * x * x * x - x * x + T(2) / T(3);
    if (T(1) <= x && x < T(2)) return (T(2) - x) * (T(2) - x) * (T(2) - x) / T(6);
    return T(0);
}
// Interpolation.h:19-30
template <class T> T bspline_slope(T x) {
    T ax = std::fabs(x);
    if (T(0) <= ax && ax < T(1)) return T(1.5) * x * ax - T(2) * x;
    if (T(1) <= ax && ax < T(2)) return -x * ax / T(2) + T(2) * x - T(2) * x / ax;
    return T(0);
}

// ---------------------------------------------------------------- 3x3 helpers
template <class T> struct M3 {
    T a[9];
    T& operator()(int i, int j) { return a[i + 3 * j]; }
    T operator()(int i, int j) const { return a[i + 3 * j]; }
    static M3 zero() { M3 m; for (int k = 0; k < 9; k++) m.a[k] = T(0); return m; }
    static M3 eye() { M3 m = zero(); m(0, 0) = m(1, 1) = m(2, 2) = T(1); return m; }
    static M3 load(const T* p) { M3 m; std::memcpy(m.a, p, sizeof(T) * 9); return m; }
    void store(T* p) const { std::memcpy(p, a, sizeof(T) * 9); }
};
template <class T> M3<T> operator+(const M3<T>& A, const M3<T>& B) { M3<T> C; for (int k = 0; k < 9; k++) C.a[k] = A.a[k] + B.a[k]; return C; }
template <class T> M3<T> operator-(const M3<T>& A, const M3<T>& B) { M3<T> C; for (int k = 0; k < 9; k++) C.a[k] = A.a[k] - B.a[k]; return C; }
template <class T> M3<T> operator*(T s, const M3<T>& A) { M3<T> C; for (int k = 0; k < 9; k++) C.a[k] = s * A.a[k]; return C; }
template <class T> M3<T> operator*(const M3<T>& A, const M3<T>& B) {
    M3<T> C;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) C(i, j) = A(i, 0) * B(0, j) + A(i, 1) * B(1, j) + A(i, 2) * B(2, j);
    return C;
}
template <class T> M3<T> tr(const M3<T>& A) { M3<T> C; for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) C(i, j) = A(j, i); return C; }
template <class T> T inner(const M3<T>& A, const M3<T>& B) { T s = 0; for (int k = 0; k < 9; k++) s += A.a[k] * B.a[k]; return s; }
template <class T> void mv(const M3<T>& A, const T* x, T* y) {
    for (int i = 0; i < 3; i++) y[i] = A(i, 0) * x[0] + A(i, 1) * x[1] + A(i, 2) * x[2];
}

// Determinant and inverse with the cofactor expansions of Eigen 3.4's fixed
// 3x3 paths (LU/Determinant.h:56-65, LU/InverseImpl.h:127-176), which the
// reference uses through Mat3::determinant() / Mat3::inverse().
template <class T> T det3(const M3<T>& m) {
    auto h = [&](int a, int b, int c) { return m(0, a) * (m(1, b) * m(2, c) - m(1, c) * m(2, b)); };
    return h(0, 1, 2) - h(1, 0, 2) + h(2, 0, 1);
}
template <class T> T cof(const M3<T>& m, int i, int j) {
    int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
    return m(i1, j1) * m(i2, j2) - m(i1, j2) * m(i2, j1);
}
template <class T> M3<T> inv3(const M3<T>& m) {
    T c0[3] = {cof(m, 0, 0), cof(m, 1, 0), cof(m, 2, 0)};
    T det = c0[0] * m(0, 0) + c0[1] * m(1, 0) + c0[2] * m(2, 0);
    T id = T(1) / det;
    M3<T> r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r(i, j) = cof(m, j, i) * id;
    return r;
}

// ---------------------------------------------------------------- SVD / polar
// One-sided (Hestenes) Jacobi SVD in long double, then the reference's
// convention (rotations U, V; |s0| >= |s1| >= |s2|; only s2 may be negative).
inline void svd_ld(const LD A[3][3], LD U[3][3], LD s[3], LD V[3][3]) {
    LD B[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) { B[i][j] = A[i][j]; V[i][j] = (i == j) ? 1 : 0; }
    const int pairs[3][2] = {{0, 1}, {0, 2}, {1, 2}};
    for (int sweep = 0; sweep < 100; sweep++) {
        bool rotated = false;
        for (auto& pr : pairs) {
            int i = pr[0], j = pr[1];
            LD al = 0, be = 0, ga = 0;
            for (int k = 0; k < 3; k++) { al += B[k][i] * B[k][i]; be += B[k][j] * B[k][j]; ga += B[k][i] * B[k][j]; }
            if (ga == 0 || std::fabs(ga) <= 1e-19L * std::sqrt(al * be)) continue;
            rotated = true;
            LD zeta = (be - al) / (2 * ga);
            LD t = (zeta >= 0 ? 1 : -1) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
            LD c = 1 / std::sqrt(1 + t * t), sn = c * t;
            for (int k = 0; k < 3; k++) {
                LD bi = B[k][i], bj = B[k][j];
                B[k][i] = c * bi - sn * bj; B[k][j] = sn * bi + c * bj;
                LD vi = V[k][i], vj = V[k][j];
                V[k][i] = c * vi - sn * vj; V[k][j] = sn * vi + c * vj;
            }
        }
        if (!rotated) break;
    }
    for (int j = 0; j < 3; j++) s[j] = std::sqrt(B[0][j] * B[0][j] + B[1][j] * B[1][j] + B[2][j] * B[2][j]);
    // sort columns by decreasing singular value
    int ord[3] = {0, 1, 2};
    std::sort(ord, ord + 3, [&](int a, int b) { return s[a] > s[b]; });
    LD Bs[3][3], Vs[3][3], ss[3];
    for (int j = 0; j < 3; j++) {
        ss[j] = s[ord[j]];
        for (int k = 0; k < 3; k++) { Bs[k][j] = B[k][ord[j]]; Vs[k][j] = V[k][ord[j]]; }
    }
    LD scale = std::max(ss[0], (LD)1e-300L);
    for (int j = 0; j < 3; j++) {
        s[j] = ss[j];
        for (int k = 0; k < 3; k++) V[k][j] = Vs[k][j];
    }
    // U columns; complete rank-deficient cases with cross products
    for (int j = 0; j < 2; j++) {
        if (ss[j] > 1e-30L * scale) for (int k = 0; k < 3; k++) U[k][j] = Bs[k][j] / ss[j];
        else {
            // any unit vector orthogonal to the previous columns
            LD e[3] = {1, 0, 0};
            if (j == 1 && std::fabs(U[0][0]) > 0.9L) { e[0] = 0; e[1] = 1; }
            if (j == 1) {
                LD d = e[0] * U[0][0] + e[1] * U[1][0] + e[2] * U[2][0];
                for (int k = 0; k < 3; k++) e[k] -= d * U[k][0];
            }
            LD n = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
            for (int k = 0; k < 3; k++) U[k][j] = e[k] / n;
        }
    }
    if (ss[2] > 1e-30L * scale) for (int k = 0; k < 3; k++) U[k][2] = Bs[k][2] / ss[2];
    else {
        U[0][2] = U[1][0] * U[2][1] - U[2][0] * U[1][1];
        U[1][2] = U[2][0] * U[0][1] - U[0][0] * U[2][1];
        U[2][2] = U[0][0] * U[1][1] - U[1][0] * U[0][1];
    }
    auto detl = [](LD M[3][3]) {
        return M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
               M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
    };
    if (detl(V) < 0) for (int k = 0; k < 3; k++) { V[k][2] = -V[k][2]; U[k][2] = -U[k][2]; }
    if (detl(U) < 0) { for (int k = 0; k < 3; k++) U[k][2] = -U[k][2]; s[2] = -s[2]; }
}

template <class T> void svd(const M3<T>& F, M3<T>& U, T sig[3], M3<T>& V) {
    LD A[3][3], Ul[3][3], sl[3], Vl[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) A[i][j] = F(i, j);
    svd_ld(A, Ul, sl, Vl);
    for (int i = 0; i < 3; i++) {
        sig[i] = (T)sl[i];
        for (int j = 0; j < 3; j++) { U(i, j) = (T)Ul[i][j]; V(i, j) = (T)Vl[i][j]; }
    }
}

// polarDecomposition (ImplicitQRSVD.h:863-877): R = U V^T, S = V diag(s) V^T.
template <class T> void polar(const M3<T>& F, M3<T>& R, M3<T>& S) {
    LD A[3][3], U[3][3], s[3], V[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) A[i][j] = F(i, j);
    svd_ld(A, U, s, V);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            LD r = 0, sy = 0;
            for (int k = 0; k < 3; k++) { r += U[i][k] * V[j][k]; sy += V[i][k] * s[k] * V[j][k]; }
            R(i, j) = (T)r;
            S(i, j) = (T)sy;
        }
}

// ---------------------------------------------------------------- elasticity
// PK_FixedCorotatedElasticity, Elasticity.cpp:88-98
template <class T> M3<T> pk(const M3<T>& F, T lam, T mu) {
    M3<T> R, S;
    polar(F, R, S);
    T J = std::max(det3(F), T(1e-6));
    return T(2) * mu * (F - R) + (lam * (J - T(1)) * J) * tr(inv3(F));
}

// FixedCorotatedElasticity, Elasticity.cpp:74-86
template <class T> T energy(const M3<T>& F, T lam, T mu) {
    M3<T> U, V; T s[3];
    svd(F, U, s, V);
    T ss = (s[0] - 1) * (s[0] - 1) + (s[1] - 1) * (s[1] - 1) + (s[2] - 1) * (s[2] - 1);
    T J = std::max(det3(F), T(1e-6));
    return mu * ss + T(0.5) * lam * (J - 1) * (J - 1);
}

// Rotation derivative: solve X S + S X = R^T dF - dF^T R for skew X = [x]_x,
// return R X.  The 3x3 system and its unknown ordering follow
// Elasticity.cpp:138-171.  `guard` reproduces the reference's conditioning
// guard (log|det A| > 20 => A += 1e-4 I, Elasticity.cpp:155-159).
template <class T> M3<T> rotation_derivative(const M3<T>& R, const M3<T>& S, const M3<T>& dF, bool guard) {
    M3<T> A;
    A(0, 0) = S(0, 2); A(0, 1) = S(1, 2); A(0, 2) = -(S(0, 0) + S(1, 1));
    A(1, 0) = -S(0, 1); A(1, 1) = S(0, 0) + S(2, 2); A(1, 2) = -S(1, 2);
    A(2, 0) = -(S(1, 1) + S(2, 2)); A(2, 1) = S(0, 1); A(2, 2) = S(0, 2);
    if (guard) {
        LD dA = 0;
        {
            LD m[3][3];
            for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) m[i][j] = A(i, j);
            dA = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
                 m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
        }
        if (std::log(std::fabs(dA)) > 20.0L) for (int i = 0; i < 3; i++) A(i, i) += T(1e-4);
    }
    M3<T> t = tr(R) * dF - tr(dF) * R;
    LD b[3] = {t(0, 1), t(0, 2), t(1, 2)};
    // Cramer's rule in long double
    LD a[3][3];
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) a[i][j] = A(i, j);
    auto d3 = [](LD m[3][3]) {
        return m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    };
    LD D = d3(a), x[3];
    for (int c = 0; c < 3; c++) {
        LD m[3][3];
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) m[i][j] = (j == c) ? b[i] : a[i][j];
        x[c] = d3(m) / D;
    }
    M3<T> X = M3<T>::zero();
    X(0, 1) = (T)-x[2]; X(0, 2) = (T)x[1];
    X(1, 0) = (T)x[2];  X(1, 2) = (T)-x[0];
    X(2, 0) = (T)-x[1]; X(2, 1) = (T)x[0];
    return R * X;
}

// d_JFit_dF_FD contracted with dF (Elasticity.cpp:7-72, 126-140): central
// differences of J F^-T with delta = 1e-6 in the working precision.
template <class T> M3<T> djfit_fd_mult(const M3<T>& F, const M3<T>& dF) {
    auto jfit = [](const M3<T>& G) { T J = det3(G); return J * tr(inv3(G)); };
    T delta = T(1e-6);
    M3<T> tf = F;
    T tens[3][3][9];  // [a][b][i + 3 j]
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            T orig = tf(i, j);
            tf(i, j) = orig + delta;
            M3<T> fw = jfit(tf);
            tf(i, j) = orig - delta;
            M3<T> bw = jfit(tf);
            tf(i, j) = orig;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) {
                    T l1 = fw(a, b), l2 = bw(a, b);
                    tens[a][b][i + 3 * j] = (T)((l1 - l2) / (2.0 * (double)delta));
                }
        }
    M3<T> term;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            T acc = 0;
            for (int ij = 0; ij < 9; ij++) {
                int i = ij / 3, j = ij % 3;
                acc += tens[a][b][i + 3 * j] * dF(i, j);
            }
            term(a, b) = acc;
        }
    return term;
}

// d2_FCE_psi_dF2_mult_by_dF, Elasticity.cpp:100-178 (reference-compatible).
template <class T> M3<T> d2_ref(const M3<T>& F, T lam, T mu, const M3<T>& dF) {
    M3<T> R, S;
    polar(F, R, S);
    T J = det3(F);
    M3<T> Fit = tr(inv3(F));
    J = std::max(J, T(1e-6));
    M3<T> ret = T(2) * mu * dF;
    ret = ret + (lam * J * inner(J * Fit, dF)) * Fit;
    ret = ret + (lam * (J - T(1))) * djfit_fd_mult(F, dF);
    ret = ret - T(2) * mu * rotation_derivative(R, S, dF, true);
    return ret;
}

// Exact dP/dF : dF of the same P (analytic d(J F^-T), no guard).
//   unclamped: dP = 2mu(dF - dR) + lam (JF^-T:dF) JF^-T + lam (J-1) J[(F^-T:dF)F^-T - F^-T dF^T F^-T]
//   clamped (det F < 1e-6, J const): dP = 2mu(dF - dR) - lam (J-1) J F^-T dF^T F^-T
template <class T> M3<T> d2_exact(const M3<T>& F, T lam, T mu, const M3<T>& dF) {
    M3<T> R, S;
    polar(F, R, S);
    T detF = det3(F);
    bool clamped = !(detF > T(1e-6));
    T J = clamped ? T(1e-6) : detF;
    M3<T> Fit = tr(inv3(F));
    M3<T> FdF = Fit * tr(dF) * Fit;
    M3<T> ret = T(2) * mu * dF;
    if (!clamped) {
        T c = inner(Fit, dF);
        ret = ret + (lam * J * J * c) * Fit;
        ret = ret + (lam * (J - T(1)) * J) * (c * Fit - FdF);
    } else {
        ret = ret - (lam * (J - T(1)) * J) * FdF;
    }
    ret = ret - T(2) * mu * rotation_derivative(R, S, dF, false);
    return ret;
}

// ---------------------------------------------------------------- graph
enum Mode { REFCOMPAT = 0, EXACT = 1 };

template <class T> struct Layer {
    std::vector<T> x, v, F, C, P, dFc;
    std::vector<T> dLdx, dLdv, dLdF, dLdC, dLdP, dLdv_next, dLdC_next, dLdFe;
    std::vector<T> gm, gv, gp;              // grid mass, velocity, momentum
    std::vector<T> gdLdv, gdLdp, gdLdm;     // grid adjoints
};

template <class T> struct Graph {
    int n = 0, dim[3] = {0, 0, 0};
    T dx = 1, mn[3] = {0, 0, 0};
    std::vector<T> m, vol, lam, mu, target;
    T dt = T(1.0 / 120.0), drag = T(0.5), fext[3] = {0, 0, 0}, s = T(0.1);
    std::vector<Layer<T>> layers;

    size_t G() const { return (size_t)dim[0] * dim[1] * dim[2]; }

    void alloc_layer(Layer<T>& L) {
        L.x.assign(3 * n, 0); L.v.assign(3 * n, 0); L.F.assign(9 * n, 0); L.C.assign(9 * n, 0);
        L.P.assign(9 * n, 0); L.dFc.assign(9 * n, 0);
        L.dLdx.assign(3 * n, 0); L.dLdv.assign(3 * n, 0); L.dLdF.assign(9 * n, 0); L.dLdC.assign(9 * n, 0);
        L.dLdP.assign(9 * n, 0); L.dLdv_next.assign(3 * n, 0); L.dLdC_next.assign(9 * n, 0); L.dLdFe.assign(9 * n, 0);
        L.gm.assign(G(), 0); L.gv.assign(3 * G(), 0); L.gp.assign(3 * G(), 0);
        L.gdLdv.assign(3 * G(), 0); L.gdLdp.assign(3 * G(), 0); L.gdLdm.assign(G(), 0);
    }

    // stencil iteration shared by every stage: base = floor((x-min)/dx) - 1 by
    // division (ForwardSimulation.cpp:17-20), node (i,j,k) = idx/16, idx%16/4,
    // idx%4, bounds-skip (ForwardSimulation.cpp:22-36), node.x = min + ijk*dx
    // (Grid.cpp:22).
    template <class Fn> void stencil(const T* xp, Fn fn) const {
        int base[3];
        for (int a = 0; a < 3; a++) base[a] = (int)std::floor((xp[a] - mn[a]) / dx) - 1;
        for (int idx = 0; idx < 64; idx++) {
            int ii[3] = {base[0] + idx / 16, base[1] + (idx % 16) / 4, base[2] + idx % 4};
            if (ii[0] < 0 || ii[0] >= dim[0] || ii[1] < 0 || ii[1] >= dim[1] || ii[2] < 0 || ii[2] >= dim[2]) continue;
            size_t g = ((size_t)ii[0] * dim[1] + ii[1]) * dim[2] + ii[2];
            T d[3], nd[3], ns[3];
            for (int a = 0; a < 3; a++) {
                T xg = mn[a] + (T)ii[a] * dx;
                d[a] = xg - xp[a];
                nd[a] = bspline(d[a] / dx);
                ns[a] = bspline_slope(d[a] / dx);
            }
            T w = nd[0] * nd[1] * nd[2];
            T gw[3] = {-T(1) / dx * (ns[0] * nd[1] * nd[2]), -T(1) / dx * (nd[0] * ns[1] * nd[2]),
                       -T(1) / dx * (nd[0] * nd[1] * ns[2])};
            fn(g, d, w, gw);
        }
    }

    // SingleThreadMPM::P2G (ForwardSimulation.cpp:11-51, 174-182)
    void p2g(const Layer<T>& L, std::vector<T>& gm, std::vector<T>& gp, T dt_, T drag_) const {
        std::fill(gm.begin(), gm.end(), T(0));
        std::fill(gp.begin(), gp.end(), T(0));
        for (int p = 0; p < n; p++) {
            M3<T> Fe = M3<T>::load(&L.F[9 * p]) + M3<T>::load(&L.dFc[9 * p]);
            M3<T> G = (-T(3) / (dx * dx) * dt_ * vol[p]) * M3<T>::load(&L.P[9 * p]) * tr(Fe) +
                      m[p] * M3<T>::load(&L.C[9 * p]);
            T mvd[3];
            for (int a = 0; a < 3; a++) mvd[a] = m[p] * L.v[3 * p + a] * (T(1) - dt_ * drag_);
            stencil(&L.x[3 * p], [&](size_t g, const T* d, T w, const T*) {
                gm[g] += w * m[p];
                T Gd[3];
                mv(G, d, Gd);
                for (int a = 0; a < 3; a++) gp[3 * g + a] += w * (mvd[a] + Gd[a]);
            });
        }
    }

    // SingleThreadMPM::ForwardTimeStep with smoothing (ForwardSimulation.cpp:136-157)
    void forward_step(int i) {
        Layer<T>& L = layers[i];
        Layer<T>& N = layers[i + 1];
        for (int p = 0; p < n; p++) {  // P_op_1
            M3<T> Fe = M3<T>::load(&L.F[9 * p]) + M3<T>::load(&L.dFc[9 * p]);
            pk(Fe, lam[p], mu[p]).store(&L.P[9 * p]);
        }
        p2g(L, L.gm, L.gp, dt, drag);  // G_Reset + P2G
        std::fill(L.gv.begin(), L.gv.end(), T(0));
        for (size_t g = 0; g < G(); g++)  // G_op (ForwardSimulation.cpp:53-58)
            if (std::fabs(L.gm[g]) > T(kFltEps))
                for (int a = 0; a < 3; a++) L.gv[3 * g + a] = L.gp[3 * g + a] / L.gm[g] + dt * fext[a];
        for (int p = 0; p < n; p++) {  // G2P (ForwardSimulation.cpp:60-106) + P_op_2 (118-124)
            T vn[3] = {0, 0, 0};
            M3<T> Cn = M3<T>::zero();
            stencil(&L.x[3 * p], [&](size_t g, const T* d, T w, const T*) {
                for (int a = 0; a < 3; a++) vn[a] += w * L.gv[3 * g + a];
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) Cn(a, b) += T(3) / (dx * dx) * w * L.gv[3 * g + a] * d[b];
            });
            for (int a = 0; a < 3; a++) N.v[3 * p + a] = vn[a];
            Cn.store(&N.C[9 * p]);
            M3<T> F = M3<T>::load(&L.F[9 * p]);
            M3<T> Fe = F + M3<T>::load(&L.dFc[9 * p]);
            M3<T> Fn = (M3<T>::eye() + dt * Cn) * Fe;
            Fn = (T(1) - s) * Fn + s * F;
            Fn.store(&N.F[9 * p]);
            for (int a = 0; a < 3; a++) N.x[3 * p + a] = L.x[3 * p + a] + dt * vn[a];
        }
    }

    void setup(int num_layers) {  // SetUpCompGraph (CompGraph.cpp:7-17)
        Layer<T> first = layers[0];
        layers.assign(num_layers, first);
    }

    void forward(int start) {
        for (int i = start; i + 1 < (int)layers.size(); i++) forward_step(i);
    }

    // EndLayerMassLoss (CompGraph.cpp:110-244).  The loss is accumulated in
    // double whatever T is.
    double loss() {
        Layer<T>& L = layers.back();
        p2g(L, L.gm, L.gp, T(0), T(0));
        const T eps = T(1e-4), min_mass = T(1e-3), w_pen = T(10);
        double Ls = 0;
        for (size_t g = 0; g < G(); g++) {
            T cm = L.gm[g], tm = target[g];
            T clog = std::log(cm + T(1) + eps) - std::log(tm + T(1) + eps);
            Ls += (double)(T(0.5) * clog * clog);
            L.gdLdm[g] = clog / (cm + T(1) + eps);
            if (cm < min_mass) {
                T diff = min_mass - cm;
                Ls += (double)(w_pen * diff * diff);
                L.gdLdm[g] += -T(2) * w_pen * diff;
            }
        }
        for (int p = 0; p < n; p++) {
            T acc[3] = {0, 0, 0};
            stencil(&L.x[3 * p], [&](size_t g, const T*, T, const T* gw) {
                for (int a = 0; a < 3; a++) acc[a] += m[p] * L.gdLdm[g] * gw[a];
            });
            for (int a = 0; a < 3; a++) { L.dLdx[3 * p + a] = acc[a]; L.dLdv[3 * p + a] = 0; }
            for (int k = 0; k < 9; k++) { L.dLdF[9 * p + k] = 0; L.dLdC[9 * p + k] = 0; }
        }
        return Ls;
    }

    void reset_gradients(Layer<T>& L) {  // PointCloud/Grid::ResetGradients
        std::fill(L.dLdx.begin(), L.dLdx.end(), T(0)); std::fill(L.dLdv.begin(), L.dLdv.end(), T(0));
        std::fill(L.dLdF.begin(), L.dLdF.end(), T(0)); std::fill(L.dLdC.begin(), L.dLdC.end(), T(0));
        std::fill(L.dLdP.begin(), L.dLdP.end(), T(0)); std::fill(L.dLdv_next.begin(), L.dLdv_next.end(), T(0));
        std::fill(L.dLdC_next.begin(), L.dLdC_next.end(), T(0)); std::fill(L.dLdFe.begin(), L.dLdFe.end(), T(0));
        std::fill(L.gdLdv.begin(), L.gdLdv.end(), T(0)); std::fill(L.gdLdp.begin(), L.gdLdp.end(), T(0));
        std::fill(L.gdLdm.begin(), L.gdLdm.end(), T(0));
    }

    // Back_Timestep (BackPropagation.cpp:6-125).  REFCOMPAT reproduces it term
    // by term.  EXACT is the true adjoint of forward_step:
    //   dLdC_next carries (1-s) on dt dLdF' Fe^T,
    //   no second (I + dt C')^T dLdF' transport term,
    //   the grad-w momentum term keeps (1 - dt drag),
    //   dLdm uses p/m^2 = (v - dt f_ext)/m,
    //   dP/dF : dF is analytic (no finite differences, no guard),
    //   and dLdFe (= dL/d dFc of this layer) is stored separately from dLdF.
    void back_timestep(int i, int mode) {
        Layer<T>& Nx = layers[i + 1];
        Layer<T>& L = layers[i];
        const bool ex = (mode == EXACT);
        const T k3 = T(3) / (dx * dx);
        for (int p = 0; p < n; p++) {  // adjoint P_op_2 (BackPropagation.cpp:14-25)
            M3<T> Cn = M3<T>::load(&Nx.C[9 * p]);
            M3<T> dFn = M3<T>::load(&Nx.dLdF[9 * p]);
            M3<T> Fe = M3<T>::load(&L.F[9 * p]) + M3<T>::load(&L.dFc[9 * p]);
            M3<T> dF = tr(M3<T>::eye() + dt * Cn) * dFn;
            dF = (T(1) - s) * dF + s * dFn;
            dF.store(&L.dLdF[9 * p]);
            for (int a = 0; a < 3; a++) L.dLdv_next[3 * p + a] = dt * Nx.dLdx[3 * p + a] + Nx.dLdv[3 * p + a];
            M3<T> dCn = (ex ? (T(1) - s) * dt : dt) * dFn * tr(Fe) + M3<T>::load(&Nx.dLdC[9 * p]);
            dCn.store(&L.dLdC_next[9 * p]);
        }
        for (int p = 0; p < n; p++) {  // adjoint G2P (BackPropagation.cpp:27-44)
            M3<T> dCn = M3<T>::load(&L.dLdC_next[9 * p]);
            stencil(&L.x[3 * p], [&](size_t g, const T* d, T w, const T*) {
                T cd[3];
                mv(dCn, d, cd);
                for (int a = 0; a < 3; a++) L.gdLdv[3 * g + a] += L.dLdv_next[3 * p + a] * w + k3 * w * cd[a];
            });
        }
        for (size_t g = 0; g < G(); g++) {  // adjoint G_op (BackPropagation.cpp:46-59)
            if (std::fabs(L.gm[g]) > T(kFltEps)) {
                T dot = 0;
                for (int a = 0; a < 3; a++) {
                    L.gdLdp[3 * g + a] = L.gdLdv[3 * g + a] / L.gm[g];
                    T vv = ex ? (L.gv[3 * g + a] - dt * fext[a]) : L.gv[3 * g + a];
                    dot += vv * L.gdLdv[3 * g + a];
                }
                L.gdLdm[g] = -T(1) / L.gm[g] * dot;
            }
        }
        for (int p = 0; p < n; p++) {  // adjoint P2G + P_op_1 (BackPropagation.cpp:61-124)
            const T* xp = &L.x[3 * p];
            M3<T> Fe = M3<T>::load(&L.F[9 * p]) + M3<T>::load(&L.dFc[9 * p]);
            M3<T> FeT = tr(Fe);
            M3<T> P = M3<T>::load(&L.P[9 * p]);
            M3<T> G = (-k3 * dt * vol[p]) * P * FeT + m[p] * M3<T>::load(&L.C[9 * p]);
            M3<T> GT = tr(G);
            M3<T> dP = M3<T>::load(&L.dLdP[9 * p]);
            M3<T> dF = M3<T>::load(&L.dLdF[9 * p]);
            M3<T> dC = M3<T>::load(&L.dLdC[9 * p]);
            M3<T> dCn = M3<T>::load(&L.dLdC_next[9 * p]);
            T dx_[3], dv_[3];
            for (int a = 0; a < 3; a++) { dx_[a] = L.dLdx[3 * p + a]; dv_[a] = L.dLdv[3 * p + a]; }
            const T* vp = &L.v[3 * p];
            const T* vnx = &L.dLdv_next[3 * p];
            const T mvf = ex ? (T(1) - dt * drag) : T(1);
            M3<T> dFe_stress = M3<T>::zero();
            stencil(xp, [&](size_t g, const T* d, T w, const T* gw) {
                const T* dLdp = &L.gdLdp[3 * g];
                const T dLdm = L.gdLdm[g];
                const T* vg = &L.gv[3 * g];
                T FtD[3], PtDp[3];
                mv(FeT, d, FtD);
                mv(tr(P), dLdp, PtDp);
                for (int a = 0; a < 3; a++)
                    for (int b = 0; b < 3; b++) {
                        dP(a, b) -= w * k3 * dt * vol[p] * dLdp[a] * FtD[b];
                        T t = w * k3 * dt * vol[p] * d[a] * PtDp[b];
                        if (ex) dFe_stress(a, b) -= t; else dF(a, b) -= t;
                        dC(a, b) += w * m[p] * dLdp[a] * d[b];
                    }
                for (int a = 0; a < 3; a++) dx_[a] += m[p] * dLdm * gw[a];
                T Gd[3], GtDp[3];
                mv(G, d, Gd);
                mv(GT, dLdp, GtDp);
                T q = 0;
                for (int a = 0; a < 3; a++) q += (m[p] * vp[a] * mvf + Gd[a]) * dLdp[a];
                for (int a = 0; a < 3; a++) dx_[a] += gw[a] * q - w * GtDp[a];
                T vdot = vg[0] * vnx[0] + vg[1] * vnx[1] + vg[2] * vnx[2];
                for (int a = 0; a < 3; a++) dx_[a] += gw[a] * vdot;
                T ip = 0;
                for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++) ip += dCn(a, b) * vg[a] * d[b];
                T cv[3];
                mv(tr(dCn), vg, cv);
                for (int a = 0; a < 3; a++) dx_[a] += k3 * (ip * gw[a] - w * cv[a]);
                for (int a = 0; a < 3; a++) dv_[a] += w * m[p] * (T(1) - dt * drag) * dLdp[a];
            });
            M3<T> Cn = M3<T>::load(&Nx.C[9 * p]);
            M3<T> dFn = M3<T>::load(&Nx.dLdF[9 * p]);
            if (!ex) {
                dF = dF + tr(M3<T>::eye() + dt * Cn) * dFn;
                dF = dF + d2_ref(Fe, lam[p], mu[p], dP);
                dF.store(&L.dLdF[9 * p]);
                dF.store(&L.dLdFe[9 * p]);
            } else {
                // dL/dFe = (1-s)(I + dt C')^T dLdF' + stress term + dP/dFe : dLdP
                M3<T> dFe = (T(1) - s) * (tr(M3<T>::eye() + dt * Cn) * dFn) + dFe_stress +
                            d2_exact(Fe, lam[p], mu[p], dP);
                dFe.store(&L.dLdFe[9 * p]);
                (dFe + s * dFn).store(&L.dLdF[9 * p]);
            }
            for (int a = 0; a < 3; a++) { dx_[a] += Nx.dLdx[3 * p + a]; L.dLdx[3 * p + a] = dx_[a]; L.dLdv[3 * p + a] = dv_[a]; }
            dP.store(&L.dLdP[9 * p]);
            dC.store(&L.dLdC[9 * p]);
        }
    }

    void backward(int control_layer, int mode) {  // ComputeBackwardPass (CompGraph.cpp:258-267)
        for (int i = (int)layers.size() - 2; i >= control_layer; i--) {
            reset_gradients(layers[i]);
            back_timestep(i, mode);
        }
    }
};

// CalculatePointCloudVolumes (ForwardSimulation.cpp:262-290) with a fresh grid.
template <class T> void calc_volumes(Graph<T>& g) {
    Layer<T>& L = g.layers[0];
    std::vector<T> gm(g.G()), gp(3 * g.G());
    g.p2g(L, gm, gp, T(0), T(0));
    for (int p = 0; p < g.n; p++) {
        T mg = 0;
        g.stencil(&L.x[3 * p], [&](size_t gi, const T*, T w, const T*) { mg += w * gm[gi]; });
        g.vol[p] = (std::fabs(mg) > T(kFltEps)) ? (g.m[p] / mg) : T(0);
    }
}

}  // namespace oracle

// ====================================================================== C ABI
using namespace oracle;

#define ORACLE_API(T, SFX)                                                                                    \
    extern "C" T or_bspline_##SFX(T x) { return bspline<T>(x); }                                              \
    extern "C" T or_bspline_slope_##SFX(T x) { return bspline_slope<T>(x); }                                  \
    extern "C" void or_svd_##SFX(const T* F, T* U, T* s, T* V) {                                              \
        M3<T> Um, Vm; svd(M3<T>::load(F), Um, s, Vm); Um.store(U); Vm.store(V); }                            \
    extern "C" void or_polar_##SFX(const T* F, T* R, T* S) {                                                  \
        M3<T> Rm, Sm; polar(M3<T>::load(F), Rm, Sm); Rm.store(R); Sm.store(S); }                             \
    extern "C" void or_pk_##SFX(const T* F, T lam, T mu, T* P) { pk(M3<T>::load(F), lam, mu).store(P); }     \
    extern "C" T or_energy_##SFX(const T* F, T lam, T mu) { return energy(M3<T>::load(F), lam, mu); }        \
    extern "C" void or_d2_ref_##SFX(const T* F, T lam, T mu, const T* dF, T* out) {                           \
        d2_ref(M3<T>::load(F), lam, mu, M3<T>::load(dF)).store(out); }                                       \
    extern "C" void or_d2_exact_##SFX(const T* F, T lam, T mu, const T* dF, T* out) {                         \
        d2_exact(M3<T>::load(F), lam, mu, M3<T>::load(dF)).store(out); }                                     \
    extern "C" void* or_graph_create_##SFX(int n, const T* x, const T* v, const T* F, const T* C,             \
                                           const T* dFc, const T* m, const T* vol, const T* lam,               \
                                           const T* mu, int dx_, int dy_, int dz_, T h, const T* mn,           \
                                           const T* target) {                                                  \
        Graph<T>* g = new Graph<T>();                                                                          \
        g->n = n; g->dim[0] = dx_; g->dim[1] = dy_; g->dim[2] = dz_; g->dx = h;                               \
        for (int a = 0; a < 3; a++) g->mn[a] = mn[a];                                                          \
        g->m.assign(m, m + n); g->vol.assign(vol, vol + n); g->lam.assign(lam, lam + n);                       \
        g->mu.assign(mu, mu + n);                                                                              \
        g->target.assign(g->G(), T(0));                                                                        \
        if (target) g->target.assign(target, target + g->G());                                                 \
        g->layers.resize(1); g->alloc_layer(g->layers[0]);                                                     \
        Layer<T>& L = g->layers[0];                                                                            \
        std::memcpy(L.x.data(), x, sizeof(T) * 3 * n); std::memcpy(L.v.data(), v, sizeof(T) * 3 * n);        \
        std::memcpy(L.F.data(), F, sizeof(T) * 9 * n); std::memcpy(L.C.data(), C, sizeof(T) * 9 * n);        \
        std::memcpy(L.dFc.data(), dFc, sizeof(T) * 9 * n);                                                     \
        return g; }                                                                                            \
    extern "C" void or_graph_destroy_##SFX(void* h) { delete (Graph<T>*)h; }                                  \
    extern "C" void or_graph_calc_volumes_##SFX(void* h, T* vol_out) {                                        \
        Graph<T>* g = (Graph<T>*)h; calc_volumes(*g);                                                          \
        if (vol_out) std::memcpy(vol_out, g->vol.data(), sizeof(T) * g->n); }                                 \
    extern "C" void or_graph_setup_##SFX(void* h, int L, T dt, T drag, const T* f, T s) {                     \
        Graph<T>* g = (Graph<T>*)h; g->dt = dt; g->drag = drag; g->s = s;                                      \
        for (int a = 0; a < 3; a++) g->fext[a] = f[a];                                                         \
        g->setup(L); }                                                                                         \
    extern "C" void or_graph_forward_##SFX(void* h, int start) { ((Graph<T>*)h)->forward(start); }            \
    extern "C" double or_graph_loss_##SFX(void* h) { return ((Graph<T>*)h)->loss(); }                         \
    extern "C" void or_graph_backward_##SFX(void* h, int control, int mode) {                                 \
        ((Graph<T>*)h)->backward(control, mode); }                                                             \
    extern "C" int or_graph_get_##SFX(void* h, int layer, const char* name, T* out) {                         \
        Graph<T>* g = (Graph<T>*)h; Layer<T>& L = g->layers[layer];                                            \
        const std::vector<T>* src = nullptr;                                                                   \
        std::string k(name);                                                                                   \
        if (k == "x") src = &L.x; else if (k == "v") src = &L.v; else if (k == "F") src = &L.F;              \
        else if (k == "C") src = &L.C; else if (k == "P") src = &L.P; else if (k == "dFc") src = &L.dFc;     \
        else if (k == "dLdx") src = &L.dLdx; else if (k == "dLdv") src = &L.dLdv;                             \
        else if (k == "dLdF") src = &L.dLdF; else if (k == "dLdC") src = &L.dLdC;                             \
        else if (k == "dLdP") src = &L.dLdP; else if (k == "dLdFe") src = &L.dLdFe;                           \
        else if (k == "dLdv_next") src = &L.dLdv_next; else if (k == "dLdC_next") src = &L.dLdC_next;         \
        else if (k == "grid_m") src = &L.gm; else if (k == "grid_v") src = &L.gv;                             \
        else if (k == "grid_p") src = &L.gp; else if (k == "grid_dLdv") src = &L.gdLdv;                       \
        else if (k == "grid_dLdp") src = &L.gdLdp; else if (k == "grid_dLdm") src = &L.gdLdm;                 \
        else if (k == "vol") src = &g->vol;                                                                    \
        if (!src) return -1;                                                                                   \
        std::memcpy(out, src->data(), sizeof(T) * src->size()); return (int)src->size(); }                    \
    extern "C" int or_graph_set_##SFX(void* h, int layer, const char* name, const T* in) {                    \
        Graph<T>* g = (Graph<T>*)h; Layer<T>& L = g->layers[layer];                                            \
        std::vector<T>* dst = nullptr;                                                                         \
        std::string k(name);                                                                                   \
        if (k == "x") dst = &L.x; else if (k == "v") dst = &L.v; else if (k == "F") dst = &L.F;              \
        else if (k == "C") dst = &L.C; else if (k == "dFc") dst = &L.dFc;                                     \
        if (!dst) return -1;                                                                                   \
        std::memcpy(dst->data(), in, sizeof(T) * dst->size()); return (int)dst->size(); }                     \
    extern "C" void or_p2g_mass_##SFX(int n, const T* x, T mp, int dx_, int dy_, int dz_, T h, const T* mn,   \
                                      T* out) {                                                                \
        Graph<T> g; g.n = n; g.dim[0] = dx_; g.dim[1] = dy_; g.dim[2] = dz_; g.dx = h;                        \
        for (int a = 0; a < 3; a++) g.mn[a] = mn[a];                                                           \
        std::fill(out, out + g.G(), T(0));                                                                     \
        for (int p = 0; p < n; p++)                                                                            \
            g.stencil(x + 3 * p, [&](size_t gi, const T*, T w, const T*) { out[gi] += w * mp; }); }

#include <string>
ORACLE_API(float, f32)
ORACLE_API(double, f64)
