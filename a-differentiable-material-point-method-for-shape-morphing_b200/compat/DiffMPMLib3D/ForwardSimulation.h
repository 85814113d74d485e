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
// the remaining stages, each one GPU launch over the caller's grid / clouds (dmpm_stage_*)
void G_op(Grid& grid, float dt, Vec3 f_ext);
void G_op(Grid& grid, float dt, Vec3 gravity_point, float gravity_mag);
void G2P(PointCloud& next_point_cloud, const PointCloud& curr_point_cloud, Grid& grid);
void P_op_2(PointCloud& next_point_cloud, const PointCloud& curr_point_cloud, float dt);
void P_op_2(PointCloud& next_point_cloud, const PointCloud& curr_point_cloud, float smoothing_factor, float dt);
void CalculatePointCloudVolumes(PointCloud& curr_point_cloud, Grid& grid);

// Engine path for the functions above (DMPM_FP32_MIXED by default, or DMPM_FP64).
void SetEnginePrecision(int precision);
// FP32-mixed path: node sums as integers (dmpm_params::deterministic), so the
// functions above give the same bits on every call with the same inputs.
void SetEngineDeterministic(bool on);

// Mass transfer for headless surfacing (float on the GPU, dmpm_surface_*):
// node masses of `grid` from points of mass mp_m (ForwardSimulation.cpp:292-327)
void P2G_Mass(const std::vector<Vec3> points, Grid& grid, float mp_m);
// grid_2's node masses interpolated from grid_1's (ForwardSimulation.cpp:329-367)
void G2G_Mass(Grid& grid_1, Grid& grid_2);

}  // namespace SingleThreadMPM
}  // namespace DiffMPMLib3D
