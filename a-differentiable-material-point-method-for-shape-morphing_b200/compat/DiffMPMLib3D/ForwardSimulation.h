// ForwardSimulation.h -- the reference's SingleThreadMPM entry points
// (ForwardSimulation.h:7-45) that operate on whole clouds and grids, each run
// on the GPU through the engine.
#pragma once
#include "Grid.h"
#include "PointCloud.h"

namespace DiffMPMLib3D {
namespace SingleThreadMPM {

void ForwardTimeStep(PointCloud& next_point_cloud, PointCloud& curr_point_cloud, Grid& grid, float dt, float drag,
                     Vec3 f_ext);
void ForwardTimeStep(PointCloud& next_point_cloud, PointCloud& curr_point_cloud, Grid& grid, float smoothing_factor,
                     float dt, float drag, Vec3 f_ext);
void P_op_1(PointCloud& curr_point_cloud);
void G_Reset(Grid& grid);
void P2G(const PointCloud& curr_point_cloud, Grid& grid, float dt, float drag);
void CalculatePointCloudVolumes(PointCloud& curr_point_cloud, Grid& grid);

// Engine path for the functions above (DMPM_FP32_MIXED by default, or DMPM_FP64).
void SetEnginePrecision(int precision);

}  // namespace SingleThreadMPM
}  // namespace DiffMPMLib3D
