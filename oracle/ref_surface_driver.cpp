// ref_surface_driver.cpp -- runs the reference's headless surfacing code on a
// point cloud and writes what it produces, as golden vectors for the GPU
// surfacing functions (include/dmpm.h, "surfaces").  Test infrastructure;
// built by oracle/build_ref_mesh.sh into oracle/_ref/ref_surface.
//
//   mass    MarchingCubesPointCloud (DiffMPMAnimator3D.cpp:488-514): coarse grid
//           of ceil((max_x - min_x) / dx) nodes per axis, SingleThreadMPM::P2G_Mass
//           (ForwardSimulation.cpp:292-327), a grid refined by `quality`,
//           SingleThreadMPM::G2G_Mass (ForwardSimulation.cpp:329-367), then
//           igl::marching_cubes of the fine masses at iso (the GUI's iso_mass).  Writes the coarse and
//           fine masses (node order (i * dim_y + j) * dim_z + k) and the mesh.
//   spheres SphereUnionMarchingCubesSurfaceFromPointCloud (SphereUnionSurfacing.cpp:7-128)
//           with the given radius, dx, iso, blur iterations and box.  Writes the mesh.
//   mc      igl::marching_cubes, as SphereUnionSurfacing.cpp:125 calls it, of a field
//           given in a file (n^3 nodes in the order above, positions min + dx (i, j, k),
//           values widened to double as there).
//
// File formats (little endian): points and fields are raw float32; outputs are
// a sequence of blocks <int64 count><count values> (float32 or int32).
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "ForwardSimulation.h"
#include "Grid.h"
#include "SphereUnionSurfacing.h"
#include "igl/marching_cubes.h"

using namespace DiffMPMLib3D;

static std::vector<float> read_f32(const char* path) {
    std::vector<float> v;
    FILE* f = std::fopen(path, "rb");
    if (!f) return v;
    std::fseek(f, 0, SEEK_END);
    const long bytes = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    v.resize((size_t)bytes / 4);
    if (std::fread(v.data(), 4, v.size(), f) != v.size()) v.clear();
    std::fclose(f);
    return v;
}

template <class T> static void put(FILE* f, const T* p, int64_t count) {
    std::fwrite(&count, 8, 1, f);
    std::fwrite(p, sizeof(T), (size_t)count, f);
}

static void put_mesh(FILE* f, const Eigen::MatrixXf& V, const Eigen::MatrixXi& F) {
    std::vector<float> v((size_t)V.rows() * 3);
    std::vector<int> t((size_t)F.rows() * 3);
    for (int i = 0; i < V.rows(); i++)
        for (int c = 0; c < 3; c++) v[(size_t)3 * i + c] = V(i, c);
    for (int i = 0; i < F.rows(); i++)
        for (int c = 0; c < 3; c++) t[(size_t)3 * i + c] = F(i, c);
    put(f, v.data(), (int64_t)v.size());
    put(f, t.data(), (int64_t)t.size());
}

static std::vector<Vec3> as_points(const std::vector<float>& raw) {
    std::vector<Vec3> p(raw.size() / 3);
    for (size_t i = 0; i < p.size(); i++) p[i] = Vec3(raw[3 * i], raw[3 * i + 1], raw[3 * i + 2]);
    return p;
}

static float arg(char** argv, int i) { return std::strtof(argv[i], nullptr); }

int main(int argc, char** argv) {
    if (argc < 2) return 2;
    const std::string mode = argv[1];
    if (mode == "mass" && argc == 14) {
        // mass points mp_m dx quality iso minx miny minz maxx maxy maxz out
        const std::vector<Vec3> pts = as_points(read_f32(argv[2]));
        const float mp_m = arg(argv, 3), dx = arg(argv, 4), quality = arg(argv, 5), iso = arg(argv, 6);
        const Vec3 mn(arg(argv, 7), arg(argv, 8), arg(argv, 9)), mx(arg(argv, 10), arg(argv, 11), arg(argv, 12));
        int dims[3];
        for (int i = 0; i < 3; i++) dims[i] = (int)std::ceil((mx[0] - mn[0]) / dx);
        Grid coarse(dims[0], dims[1], dims[2], dx, mn);
        SingleThreadMPM::P2G_Mass(pts, coarse, mp_m);
        Grid fine(dims[0] * quality, dims[1] * quality, dims[2] * quality, dx / quality, mn);
        SingleThreadMPM::G2G_Mass(coarse, fine);
        Eigen::MatrixXf GV;
        Eigen::VectorXf Gf;
        fine.GetMassSDF(GV, Gf);
        Eigen::MatrixXf V;
        Eigen::MatrixXi F;
        igl::marching_cubes(Gf, GV, fine.dim_x, fine.dim_y, fine.dim_z, iso, V, F);
        FILE* f = std::fopen(argv[13], "wb");
        if (!f) return 3;
        const int64_t cd[3] = {coarse.dim_x, coarse.dim_y, coarse.dim_z}, fd[3] = {fine.dim_x, fine.dim_y, fine.dim_z};
        put(f, cd, 3);
        std::vector<float> m;
        for (int i = 0; i < coarse.dim_x; i++)
            for (int j = 0; j < coarse.dim_y; j++)
                for (int k = 0; k < coarse.dim_z; k++) m.push_back(coarse.nodes[i][j][k].m);
        put(f, m.data(), (int64_t)m.size());
        put(f, fd, 3);
        put(f, Gf.data(), (int64_t)Gf.size());
        put_mesh(f, V, F);
        std::fclose(f);
        return 0;
    }
    if (mode == "spheres" && argc == 14) {
        // spheres points radius dx iso blur minx miny minz maxx maxy maxz out
        const std::vector<Vec3> pts = as_points(read_f32(argv[2]));
        const float radius = arg(argv, 3), dx = arg(argv, 4), iso = arg(argv, 5);
        const int blur = std::atoi(argv[6]);
        const Vec3 mn(arg(argv, 7), arg(argv, 8), arg(argv, 9)), mx(arg(argv, 10), arg(argv, 11), arg(argv, 12));
        Eigen::MatrixXf V;
        Eigen::MatrixXi F;
        SphereUnionMarchingCubesSurfaceFromPointCloud(pts, radius, dx, iso, blur, mn, mx, V, F);
        FILE* f = std::fopen(argv[13], "wb");
        if (!f) return 3;
        put_mesh(f, V, F);
        std::fclose(f);
        return 0;
    }
    if (mode == "mc" && argc == 10) {
        // mc field n dx iso minx miny minz out: field of n^3 nodes, node (i, j, k) at min + dx (i, j, k)
        const std::vector<float> field = read_f32(argv[2]);
        const int n = std::atoi(argv[3]);
        const float dx = arg(argv, 4), iso = arg(argv, 5);
        const Vec3 mn(arg(argv, 6), arg(argv, 7), arg(argv, 8));
        if ((long)field.size() != (long)n * n * n) return 5;
        Eigen::MatrixXf GV((long)n * n * n, 3);
        Eigen::VectorXd Gf((long)n * n * n);  // as SphereUnionSurfacing.cpp:112 (double values)
        long ind = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < n; j++)
                for (int k = 0; k < n; k++) {
                    GV.row(ind) = mn + dx * Vec3(i, j, k);
                    Gf(ind) = field[ind];
                    ind++;
                }
        Eigen::MatrixXf V;
        Eigen::MatrixXi F;
        igl::marching_cubes(Gf, GV, n, n, n, (double)iso, V, F);
        FILE* f = std::fopen(argv[9], "wb");
        if (!f) return 3;
        put_mesh(f, V, F);
        std::fclose(f);
        return 0;
    }
    return 2;
}
