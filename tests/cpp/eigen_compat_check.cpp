// A caller of the reference's C++ API that does Eigen arithmetic on the
// API's types, compiled against the compat headers with Eigen on the include
// path (Vec3 / Mat3 are then Eigen::Vector3f / Eigen::Matrix3f) and linked
// with libdmpm_compat_eigen.so.  Host-side parts only (no GPU needed): the
// optimiser step PointCloud::Descend_Adam checked against the same update
// written by the caller with Eigen array expressions, InnerProduct, transposes
// of MaterialPoint fields, Grid node positions and the B-spline.
#include <cmath>
#include <cstdio>
#include <random>
#include <type_traits>

#include "DiffMPMLib3D/Grid.h"
#include "DiffMPMLib3D/Interpolation.h"
#include "DiffMPMLib3D/PointCloud.h"

using namespace DiffMPMLib3D;

static_assert(std::is_same<Vec3, Eigen::Vector3f>::value, "Vec3 is Eigen::Vector3f");
static_assert(std::is_same<Mat3, Eigen::Matrix3f>::value, "Mat3 is Eigen::Matrix3f");
static_assert(sizeof(MaterialPoint) == 472 && sizeof(GridNode) == 80, "reference layouts");

static int fails = 0;
static void expect(bool ok, const char* what) {
    if (!ok) {
        std::printf("FAIL %s\n", what);
        fails++;
    }
}

int main() {
    std::mt19937 rng(7);
    std::normal_distribution<float> nd(0.f, 1.f);
    PointCloud pc;
    pc.points.resize(97);
    for (MaterialPoint& p : pc.points) {
        for (int q = 0; q < 9; q++) {
            p.dLdF.data()[q] = nd(rng);
            p.dFc.data()[q] = 1e-3f * nd(rng);
        }
        p.x = Vec3(nd(rng), nd(rng), nd(rng));
    }
    // the caller's own norm with Eigen expressions on the fields
    float sq = 0.f;
    for (const MaterialPoint& p : pc.points) sq += InnerProduct(p.dLdF, p.dLdF);
    const float gnorm = pc.Compute_dLdF_Norm();
    expect(std::fabs(gnorm - std::sqrt(sq)) <= 1e-5f * gnorm, "Compute_dLdF_Norm vs InnerProduct");
    expect(std::fabs(InnerProduct(pc.points[0].dLdF, pc.points[1].dLdF) -
                     (pc.points[0].dLdF.transpose() * pc.points[1].dLdF).trace()) <= 1e-5f,
           "InnerProduct = trace(A^T B)");

    // one Adam step, written by the caller with Eigen array arithmetic
    const float lr = 1e-2f, b1 = 0.9f, b2 = 0.999f, eps = 1e-5f;
    std::vector<Mat3> want(pc.points.size());
    for (size_t i = 0; i < pc.points.size(); i++) {
        const MaterialPoint& p = pc.points[i];
        const Mat3 g = p.dLdF / gnorm;
        const Mat3 m = (1.f - b1) * g;
        const Mat3 v = (1.f - b2) * g.array().square().matrix();
        const Mat3 mh = m / (1.f - b1), vh = v / (1.f - b2);
        want[i] = p.dFc - lr * (mh.array() / (vh.array().sqrt() + eps)).matrix();
    }
    pc.Descend_Adam(lr, gnorm, b1, b2, eps, 1);
    float worst = 0.f;
    for (size_t i = 0; i < pc.points.size(); i++)
        worst = std::max(worst, (pc.points[i].dFc - want[i]).cwiseAbs().maxCoeff() / (lr + 1e-12f));
    expect(worst <= 1e-5f, "Descend_Adam vs the caller's Eigen expression");

    // symmetric part of a field, positions as Eigen vectors
    const Mat3 sym = 0.5f * (pc.points[3].dFc + pc.points[3].dFc.transpose());
    expect((sym - sym.transpose()).norm() == 0.f, "transpose of a MaterialPoint field");
    const std::vector<Vec3> xs = pc.GetPointPositions();
    expect((xs[5] - pc.points[5].x).norm() == 0.f, "GetPointPositions");

    // grid node positions min + (i, j, k) dx
    Grid grid(4, 5, 6, 0.25f, Vec3(1.f, 2.f, 3.f));
    const Vec3 want_x = Vec3(1.f, 2.f, 3.f) + Vec3(3.f, 4.f, 5.f) * 0.25f;
    expect((grid.nodes[3][4][5].x - want_x).norm() == 0.f, "Grid node position");
    expect(grid.nodes[1][1][1].v.isZero(0.f) && grid.nodes[2][3][4].m == 0.f, "Grid nodes start at zero");

    expect(CubicBSpline(0.f) == 2.f / 3.f && CubicBSpline(2.5f) == 0.f, "CubicBSpline");
    if (fails == 0) std::printf("eigen compat ok\n");
    return fails == 0 ? 0 : 1;
}
