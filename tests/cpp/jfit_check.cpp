// A caller of the compat Elasticity API's d(J F^-T)/dF functions, used as the
// reference's callers would: reads `n` and n matrices F (row-major, 9 numbers each)
// from stdin and prints, per matrix, the 81 entries T[a][b](i, j) of d_JFit_dF_FD(F)
// and then of d_JFit_dF(J, F^-T), with J and F^-T formed by the caller.
#include <cstdio>

#include "DiffMPMLib3D/Elasticity.h"

using namespace DiffMPMLib3D;

static void print(const Tensor3x3x3x3& t) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) std::printf("%.9g\n", t[a][b](i, j));
}

int main() {
    int n = 0;
    if (std::scanf("%d", &n) != 1) return 1;
    for (int k = 0; k < n; k++) {
        double f[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                if (std::scanf("%lf", &f[i][j]) != 1) return 1;
        Mat3 F;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) F(i, j) = (float)f[i][j];
        // J and F^-T of the float matrix, in double: the cofactors over the determinant
        double g[3][3], cof[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) g[i][j] = F(i, j);
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) {
                const int a1 = (a + 1) % 3, a2 = (a + 2) % 3, b1 = (b + 1) % 3, b2 = (b + 2) % 3;
                cof[a][b] = g[a1][b1] * g[a2][b2] - g[a1][b2] * g[a2][b1];
            }
        const double J = g[0][0] * cof[0][0] + g[0][1] * cof[0][1] + g[0][2] * cof[0][2];
        Mat3 Fit;
        for (int a = 0; a < 3; a++)
            for (int b = 0; b < 3; b++) Fit(a, b) = (float)(cof[a][b] / J);
        print(d_JFit_dF_FD(F));
        print(d_JFit_dF((float)J, Fit));
    }
    return 0;
}
