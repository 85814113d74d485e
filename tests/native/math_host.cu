// math_host.cu -- host instantiations of the engine's device math
// (csrc/mat3.cuh, svd3.cuh, elasticity.cuh) for CPU unit tests against the
// oracle.  Test infrastructure only; built by tests/conftest.py.
#include "elasticity.cuh"

using namespace dmpm;

template <class T> static m3<T> ld(const T* a) {  // column-major in
    m3<T> m;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) m.a[i][j] = a[i + 3 * j];
    return m;
}
template <class T> static void st(const m3<T>& m, T* a) {
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) a[i + 3 * j] = m.a[i][j];
}

#define MATH_API(T, SFX)                                                                              \
    extern "C" T mh_bspline_##SFX(T x) { return bspline<T>(x); }                                      \
    extern "C" T mh_bspline_slope_##SFX(T x) { return bspline_slope<T>(x); }                          \
    extern "C" void mh_svd_##SFX(const T* F, T* U, T* s, T* V) {                                      \
        m3<T> Um, Vm; svd3(ld(F), Um, s, Vm); st(Um, U); st(Vm, V); }                                 \
    extern "C" void mh_polar_##SFX(const T* F, T* R, T* S) {                                          \
        m3<T> Rm, Sm; polar3(ld(F), Rm, Sm); st(Rm, R); st(Sm, S); }                                  \
    extern "C" int mh_polar_newton_##SFX(const T* F, T* R, T* S) {                                    \
        m3<T> Rm, Sm; const bool ok = polar_newton(ld(F), Rm, Sm); if (ok) { st(Rm, R); st(Sm, S); }   \
        return ok ? 1 : 0; }                                                                          \
    extern "C" void mh_pk_##SFX(const T* F, T lam, T mu, T* P) { st(pk_stress(ld(F), lam, mu), P); } \
    extern "C" void mh_d2_##SFX(const T* F, T lam, T mu, const T* dF, int exact, T* out) {            \
        st(exact ? d2_mult<true>(ld(F), lam, mu, ld(dF)) : d2_mult<false>(ld(F), lam, mu, ld(dF)), out); }

MATH_API(float, f32)
MATH_API(double, f64)
