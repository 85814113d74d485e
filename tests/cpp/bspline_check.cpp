// Prints CubicBSpline(x) and CubicBSplineSlope(x) of the compat API for each x read
// from stdin (count first), as the reference's callers evaluate them.
#include <cstdio>

#include "DiffMPMLib3D/Interpolation.h"

int main() {
    int n = 0;
    if (std::scanf("%d", &n) != 1) return 1;
    for (int k = 0; k < n; k++) {
        float x;
        if (std::scanf("%f", &x) != 1) return 1;
        std::printf("%.9g %.9g\n", DiffMPMLib3D::CubicBSpline(x), DiffMPMLib3D::CubicBSplineSlope(x));
    }
    return 0;
}
