// GeometryLoading.h -- the reference's mesh-to-point-cloud sampler
// (GeometryLoading.h:8-14, GeometryLoading.cpp:10-83) over the GPU lattice
// sampler dmpm_mesh_lattice_points: the points min_point + sampling_dx (i, j, k)
// inside the watertight mesh (V, F), in the reference's lattice order.
//
// V is any #V x 3 float matrix and F any #F x 3 int matrix with rows() and
// operator()(i, j) -- Eigen::MatrixXf / Eigen::MatrixXi as the reference passes
// them, or the TriMatrix views below.  Throws std::runtime_error on a bad
// index, size or CUDA error.
#pragma once
#include <vector>
#include "pch.h"

namespace DiffMPMLib3D {
namespace GeometryLoading {

// V: nv x 3 floats row by row, F: nf x 3 vertex indices row by row.
std::vector<Vec3> GeneratePointCloudFromTriangleArrays(const float* V, int nv, const int* F, int nf, Vec3 min_point,
                                                       Vec3 max_point, float sampling_dx);

template <class MatV, class MatF>
std::vector<Vec3> GeneratePointCloudFromWatertightTriangleMesh(const MatV& V, const MatF& F, Vec3 min_point,
                                                               Vec3 max_point, float sampling_dx) {
    const int nv = (int)V.rows(), nf = (int)F.rows();
    std::vector<float> v((size_t)nv * 3);
    std::vector<int> f((size_t)nf * 3);
    for (int i = 0; i < nv; i++)
        for (int c = 0; c < 3; c++) v[(size_t)3 * i + c] = (float)V(i, c);
    for (int i = 0; i < nf; i++)
        for (int c = 0; c < 3; c++) f[(size_t)3 * i + c] = (int)F(i, c);
    return GeneratePointCloudFromTriangleArrays(v.data(), nv, f.data(), nf, min_point, max_point, sampling_dx);
}

// Row-major #rows x 3 view with the two members the template above uses.
template <class T>
struct TriMatrix {
    const std::vector<T>* a;
    long rows() const { return (long)(a->size() / 3); }
    T operator()(long i, int c) const { return (*a)[(size_t)3 * i + c]; }
};

}  // namespace GeometryLoading
}  // namespace DiffMPMLib3D
