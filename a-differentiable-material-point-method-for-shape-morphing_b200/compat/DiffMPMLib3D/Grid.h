// Grid.h -- the reference's uniform grid (Grid.h:7-57, Grid.cpp:3-28,337-362):
// nodes[i][j][k] with node.x = min_point + (i, j, k) * dx.
#pragma once
#include <vector>
#include "GridNode.h"

namespace DiffMPMLib3D {

struct Grid {
    Grid(int dim_x, int dim_y, int dim_z, float dx, Vec3 min_point);
    Grid(const Grid& grid) = default;

    std::vector<Vec3> GetNodePositions() const;
    std::vector<float> GetNodeMasses() const;
    std::vector<Vec3> GetNodeVelocities() const;

    void ResetGradients();
    void ResetValues();

    int dim_x;
    int dim_y;
    int dim_z;
    float dx;
    Vec3 min_point = Vec3::Zero();
    std::vector<std::vector<std::vector<GridNode>>> nodes;
};

}  // namespace DiffMPMLib3D
