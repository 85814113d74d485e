// Uses the DiffMPMLib3D-compatible C++ API the way the reference's callers do
// (MPMPolyscope.cpp:59-167 scene load, CompGraph.cpp:391-405 first pass,
// DiffMPMAnimator3D.cpp:212-243 gradient check) and writes the results as raw
// doubles for the Python test to compare with the reference's golden vectors.
//   compgraph_check <cloud.mpmbin> <target.mpmbin> <out.bin> <precision> <dim> <layers> <dt> <drag> <s> <fx> <fy> <fz>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>
#include "DiffMPMLib3D/BackPropagation.h"
#include "DiffMPMLib3D/CompGraph.h"
#include "DiffMPMLib3D/Elasticity.h"
#include "DiffMPMLib3D/ForwardSimulation.h"
#include "dmpm.h"

using namespace DiffMPMLib3D;

static void put(std::FILE* f, double v) { std::fwrite(&v, sizeof(double), 1, f); }

int main(int argc, char** argv) {
    if (argc < 13 || argc > 15) return 2;
    const bool det = argc >= 14 && std::atoi(argv[13]) != 0;      // integer node sums (repeatable bits)
    const bool reorder = argc == 15 && std::atoi(argv[14]) != 0;  // cloud stored in cell order on the device
    const int precision = std::atoi(argv[4]), dim = std::atoi(argv[5]), L = std::atoi(argv[6]);
    const float dt = std::atof(argv[7]), drag = std::atof(argv[8]), s = std::atof(argv[9]);
    const Vec3 f_ext(std::atof(argv[10]), std::atof(argv[11]), std::atof(argv[12]));
    auto pc = std::make_shared<PointCloud>();
    auto tpc = std::make_shared<PointCloud>();
    if (!pc->ReadEntirePointCloudFromBinaryFile(argv[1]) || !tpc->ReadEntirePointCloudFromBinaryFile(argv[2])) return 3;
    SingleThreadMPM::SetEnginePrecision(precision);
    SingleThreadMPM::SetEngineDeterministic(det);
    auto grid = std::make_shared<Grid>(dim, dim, dim, 1.0f, Vec3(0, 0, 0));
    SingleThreadMPM::CalculatePointCloudVolumes(*pc, *grid);
    auto target = std::make_shared<Grid>(*grid);
    target->ResetValues();
    SingleThreadMPM::P2G(*tpc, *target, 0.f, 0.f);

    CompGraph cg(pc, grid, target);
    cg.SetSimulationParameters(dt, drag, f_ext, s);
    cg.SetEngineOptions(precision, DMPM_ADJ_REFCOMPAT);
    cg.SetDeterministic(det);
    cg.SetReorderParticles(reorder);
    cg.SetUpCompGraph(L);
    cg.ComputeForwardPass(0);
    const float loss = cg.EndLayerMassLoss();
    cg.ComputeBackwardPass(0);

    // standalone stage functions on the same layers
    PointCloud next = *cg.layers[0].point_cloud;
    PointCloud curr = *cg.layers[0].point_cloud;
    Grid g0 = *grid;
    SingleThreadMPM::ForwardTimeStep(next, curr, g0, s, dt, drag, f_ext);
    CompGraphLayer lo{std::make_shared<PointCloud>(*cg.layers[0].point_cloud), std::make_shared<Grid>(g0)};
    CompGraphLayer hi{std::make_shared<PointCloud>(*cg.layers[1].point_cloud), std::make_shared<Grid>(g0)};
    lo.point_cloud->ResetGradients();
    Back_Timestep(hi, lo, drag, dt, s);

    // CheckGradients fixture (DiffMPMAnimator3D.cpp:212-243): F = 0.8 Rx(45 deg)
    const float th = 3.14159265358979f / 4.f;
    Mat3 F = Mat3::Zero();
    F(0, 0) = 0.8f;
    F(1, 1) = 0.8f * std::cos(th); F(1, 2) = -0.8f * std::sin(th);
    F(2, 1) = 0.8f * std::sin(th); F(2, 2) = 0.8f * std::cos(th);
    const Tensor3x3x3x3 tfd = d2_FCE_psi_dF2_FD(F, 58333.0f, 38888.9f);
    const Tensor3x3x3x3 ttr = d2_FCE_psi_dF2_mult_trick(F, 58333.0f, 38888.9f);
    double l2 = 0.0, ref = 0.0;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int k = 0; k < 9; k++) {
                const double d = tfd[a][b].d[k] - ttr[a][b].d[k];
                l2 += d * d;
                ref += (double)ttr[a][b].d[k] * ttr[a][b].d[k];
            }

    std::FILE* f = std::fopen(argv[3], "wb");
    const size_t n = pc->points.size();
    put(f, (double)n);
    put(f, loss);
    for (size_t p = 0; p < n; p++) put(f, cg.layers[0].point_cloud->points[p].vol);
    for (size_t p = 0; p < n; p++) for (int c = 0; c < 3; c++) put(f, cg.layers[L - 1].point_cloud->points[p].x[c]);
    for (size_t p = 0; p < n; p++) for (int k = 0; k < 9; k++) put(f, cg.layers[0].point_cloud->points[p].dLdF.d[k]);
    for (size_t p = 0; p < n; p++) for (int c = 0; c < 3; c++) put(f, cg.layers[0].point_cloud->points[p].dLdx[c]);
    for (size_t p = 0; p < n; p++) for (int c = 0; c < 3; c++) put(f, next.points[p].x[c]);
    for (size_t p = 0; p < n; p++) for (int k = 0; k < 9; k++) put(f, lo.point_cloud->points[p].dLdF.d[k]);
    for (size_t p = 0; p < n; p++) for (int k = 0; k < 9; k++) put(f, cg.layers[0].point_cloud->points[p].P.d[k]);
    put(f, std::sqrt(l2 / ref));
    put(f, cg.layers.front().point_cloud->Compute_dLdF_Norm());
    std::fclose(f);
    std::printf("ok n=%zu loss=%.9g\n", n, loss);
    return 0;
}
