// surface_check.cpp -- the compat headless-surfacing API used as the reference's
// GUI uses the reference's: MarchingCubesPointCloud's mass grids
// (DiffMPMAnimator3D.cpp:488-514: P2G_Mass with unit mass, G2G_Mass onto a grid
// refined by `quality`) and SphereUnionMarchingCubesSurfaceFromPointCloud.
// Usage: surface_check <points.f32> <grid_dx> <quality> <radius> <sphere_dx> <iso> <blur> <out.bin>
// Writes <int64 n><n float fine masses><int64 nv><3 nv floats><int64 nf><3 nf ints>.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "DiffMPMLib3D/ForwardSimulation.h"
#include "DiffMPMLib3D/SphereUnionSurfacing.h"

using namespace DiffMPMLib3D;

template <class T> static void put(FILE* f, const T* p, int64_t n) {
    std::fwrite(&n, 8, 1, f);
    std::fwrite(p, sizeof(T), (size_t)n, f);
}

int main(int argc, char** argv) {
    if (argc != 9) return 2;
    FILE* in = std::fopen(argv[1], "rb");
    if (!in) return 3;
    std::vector<float> raw;
    float v;
    while (std::fread(&v, 4, 1, in) == 1) raw.push_back(v);
    std::fclose(in);
    std::vector<Vec3> pts(raw.size() / 3);
    for (size_t i = 0; i < pts.size(); i++) pts[i] = Vec3(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
    const float grid_dx = std::strtof(argv[2], nullptr), quality = std::strtof(argv[3], nullptr);
    const Vec3 mn(-1.f, -1.f, -1.f), mx(1.f, 1.f, 1.f);
    const int d = (int)std::ceil((mx[0] - mn[0]) / grid_dx);
    Grid coarse(d, d, d, grid_dx, mn);
    SingleThreadMPM::P2G_Mass(pts, coarse, 1.0f);
    Grid fine(d * quality, d * quality, d * quality, grid_dx / quality, mn);
    SingleThreadMPM::G2G_Mass(coarse, fine);
    TriMatrixOut<float> V;
    TriMatrixOut<int> F;
    SphereUnionMarchingCubesSurfaceFromPointCloud(pts, std::strtof(argv[4], nullptr), std::strtof(argv[5], nullptr),
                                                  std::strtof(argv[6], nullptr), std::atoi(argv[7]), mn, mx, V, F);
    FILE* out = std::fopen(argv[8], "wb");
    if (!out) return 4;
    const std::vector<float> m = fine.GetNodeMasses();
    put(out, m.data(), (int64_t)m.size());
    put(out, V.a.data(), (int64_t)V.a.size());
    put(out, F.a.data(), (int64_t)F.a.size());
    std::fclose(out);
    return 0;
}
