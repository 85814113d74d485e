// Grid.h -- the reference's uniform grid (Grid.h:7-57, Grid.cpp:3-28,337-362):
// nodes[i][j][k] with node.x = min_point + (i, j, k) * dx.
#pragma once
#include <array>
#include <functional>
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

    // The grid nodes within interpolation range of a point (Grid.cpp:40-81):
    // the 4 x 4 x 4 block from floor((point - min_point) / dx) - 1 (division, as
    // the reference forms it), i outermost, nodes outside the grid left out;
    // their (i, j, k) are appended to *indices when it is given.
    std::vector<std::reference_wrapper<GridNode>> QueryPoint_CubicBSpline(
        Vec3 point, std::vector<std::array<int, 3>>* indices = nullptr);
    std::vector<std::reference_wrapper<const GridNode>> QueryPointConst_CubicBSpline(
        Vec3 point, std::vector<std::array<int, 3>>* indices = nullptr) const;
    // nodes as one vector in the order (i * dim_y + j) * dim_z + k, and back (Grid.h:22-40)
    std::vector<GridNode> flatten() const;
    void unflatten(const std::vector<GridNode>& flat_nodes);

    int dim_x;
    int dim_y;
    int dim_z;
    float dx;
    Vec3 min_point = Vec3::Zero();
    std::vector<std::vector<std::vector<GridNode>>> nodes;
};

}  // namespace DiffMPMLib3D
