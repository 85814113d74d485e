// MultiThreadForwardSimulation.h -- the reference's MultiThreadMPM::ForwardTimeStep
// (MultiThreadForwardSimulation.h:7-8, MultiThreadForwardSimulation.cpp:7-154).  The
// reference splits the step over std::threads with one proxy grid per thread; on the
// GPU the step is SingleThreadMPM::ForwardTimeStep without smoothing (the multi-threaded
// step has none), and proxy_grids are accepted and left unused.
#pragma once
#include <memory>
#include <vector>
#include "Grid.h"
#include "PointCloud.h"

namespace DiffMPMLib3D {
namespace MultiThreadMPM {

void ForwardTimeStep(PointCloud& next_point_cloud, PointCloud& curr_point_cloud, Grid& main_grid,
                     std::vector<std::shared_ptr<Grid>>& proxy_grids, float dt, float drag, Vec3 f_ext);

}  // namespace MultiThreadMPM
}  // namespace DiffMPMLib3D
