// SphereUnionSurfacing.h -- the reference's SphereUnionMarchingCubesSurfaceFromPointCloud
// (SphereUnionSurfacing.h:4-14, SphereUnionSurfacing.cpp:7-128) on the GPU: the
// sphere-union field of the points (bit-identical to the reference's), then its
// iso_mass level set as a triangle mesh (marching tetrahedra; the reference uses
// libigl's marching cubes, which triangulates the same level set differently).
// mcV / mcF are any matrix types with resize(rows, cols) and (i, j) -- Eigen's
// MatrixXf / MatrixXi as the reference passes them, or TriMatrixOut below.
#pragma once
#include <vector>
#include "pch.h"

namespace DiffMPMLib3D {

// V: 3 floats per vertex, F: 3 indices per triangle
void SphereUnionSurfaceArrays(const std::vector<Vec3>& points, float radius, float grid_dx, float iso_mass,
                              int blur_iterations, Vec3 grid_min_point, Vec3 grid_max_point, std::vector<float>& V,
                              std::vector<int>& F);

template <class MatV, class MatF>
void SphereUnionMarchingCubesSurfaceFromPointCloud(const std::vector<Vec3>& points, float radius, float grid_dx,
                                                    float iso_mass, int blur_iterations, Vec3 grid_min_point,
                                                    Vec3 grid_max_point, MatV& mcV, MatF& mcF) {
    std::vector<float> V;
    std::vector<int> F;
    SphereUnionSurfaceArrays(points, radius, grid_dx, iso_mass, blur_iterations, grid_min_point, grid_max_point, V, F);
    mcV.resize((long)(V.size() / 3), 3);
    mcF.resize((long)(F.size() / 3), 3);
    for (size_t i = 0; i < V.size() / 3; i++)
        for (int c = 0; c < 3; c++) mcV((long)i, c) = V[3 * i + c];
    for (size_t i = 0; i < F.size() / 3; i++)
        for (int c = 0; c < 3; c++) mcF((long)i, c) = F[3 * i + c];
}

// Row-major #rows x 3 storage with the two members the template above uses.
template <class T>
struct TriMatrixOut {
    std::vector<T> a;
    long rows = 0;
    void resize(long r, long) {
        rows = r;
        a.assign((size_t)r * 3, T());
    }
    T& operator()(long i, int c) { return a[(size_t)3 * i + c]; }
};

}  // namespace DiffMPMLib3D
