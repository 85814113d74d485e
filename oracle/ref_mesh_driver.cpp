// ref_mesh_driver.cpp -- runs the reference's mesh-to-point-cloud sampler
// (GeometryLoading::GeneratePointCloudFromWatertightTriangleMesh,
// GeometryLoading.cpp:10-83) on an OBJ file the way LoadMPMPointCloudFromObj
// (MPMPolyscope.cpp:10-60) calls it -- bounding box of the vertices, lattice
// spacing point_dx -- and writes the kept points as float32 triples.
// Test infrastructure (builds golden vectors); see oracle/build_ref_mesh.sh.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "GeometryLoading.h"
#include "igl/readOBJ.h"

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s mesh.obj point_dx out.f32\n", argv[0]);
        return 2;
    }
    Eigen::MatrixXf V;
    Eigen::MatrixXi F;
    if (!igl::readOBJ(argv[1], V, F)) return 1;
    const float point_dx = std::strtof(argv[2], nullptr);
    DiffMPMLib3D::Vec3 mn(DBL_MAX, DBL_MAX, DBL_MAX), mx(-DBL_MAX, -DBL_MAX, -DBL_MAX);
    for (int i = 0; i < (int)V.rows(); i++)
        for (int j = 0; j < 3; j++) {
            mn[j] = std::fmin(mn[j], V(i, j));
            mx[j] = std::fmax(mx[j], V(i, j));
        }
    std::vector<DiffMPMLib3D::Vec3> pts =
        DiffMPMLib3D::GeometryLoading::GeneratePointCloudFromWatertightTriangleMesh(V, F, mn, mx, point_dx);
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 1;
    for (const auto& p : pts) std::fwrite(p.data(), sizeof(float), 3, f);
    std::fclose(f);
    return 0;
}
