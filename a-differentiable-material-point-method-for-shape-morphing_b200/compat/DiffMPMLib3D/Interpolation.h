// Interpolation.h -- the cubic B-spline weight and its slope (Interpolation.h:5-30),
// inline on the host for callers of the reference's API.  The products and sums are
// formed in the reference's order, so the float results are the reference's bit for
// bit; the engine's kernels evaluate the same polynomials in their own order.
#pragma once
#include <cmath>

#include "pch.h"

namespace DiffMPMLib3D {

inline float CubicBSpline(float x) {
    const float a = std::fabs(x);
    if (a < 1.f) return 0.5f * a * a * a - a * a + 2.f / 3.f;
    if (a < 2.f) return (2.f - a) * (2.f - a) * (2.f - a) / 6.f;
    return 0.f;
}

inline float CubicBSplineSlope(float x) {
    const float a = std::fabs(x);
    if (a < 1.f) return 1.5f * x * a - 2.f * x;
    if (a < 2.f) return -x * a / 2.f + 2.f * x - 2.f * x / a;
    return 0.f;
}

}  // namespace DiffMPMLib3D
