// make_opt_input.cpp -- writes golden OptInput JSON files with cereal's own
// JSON archive (the reference's serialiser, DiffMPMAnimator3D.cpp:252-281),
// for the Python reader/writer in optinput.py.  The struct below lists the
// reference OptInput's fields with their names, types and order
// (MPMPolyscope.h:16-83); Vec3 goes through the reference's cereal_eigen.h.
// Test infrastructure; built and run by tests/golden/make_opt_input.sh.
#include <fstream>
#include <string>

#include <Eigen/Core>

#include "cereal/archives/json.hpp"
#include "cereal/types/string.hpp"
#include "cereal_eigen.h"

using Vec3 = Eigen::Vector3f;

struct Opt {
    std::string mpm_input_mesh_path = "experiments\\big_sca_demo\\input\\bob.obj";
    std::string mpm_target_mesh_path = "experiments\\big_sca_demo\\input\\spot.obj";
    float grid_dx = 1.0f;
    int points_per_cell_cuberoot = 2;
    Vec3 grid_min_point = Vec3(-16.f, -16.f, -16.f);
    Vec3 grid_max_point = Vec3(16.f, 16.f, 16.f);
    float lam = 58333.0f;
    float mu = 38888.9f;
    float p_density = 40.0f;
    float dt = 1.f / 120.0f;
    float drag = 0.5f;
    Vec3 f_ext = Vec3(0.f, 0.f, 0.f);
    int num_animations = 40;
    int num_timesteps = 30;
    int control_stride = 10;
    int max_gd_iters = 25;
    int max_ls_iters = 15;
    float initial_alpha = 0.1f;
    float gd_tol = 1e-3f;
    float smoothing_factor = 0.1f;
    template <class A> void serialize(A& ar) {
        ar(CEREAL_NVP(mpm_input_mesh_path), CEREAL_NVP(mpm_target_mesh_path), CEREAL_NVP(grid_dx),
           CEREAL_NVP(points_per_cell_cuberoot), CEREAL_NVP(grid_min_point), CEREAL_NVP(grid_max_point), CEREAL_NVP(lam),
           CEREAL_NVP(mu), CEREAL_NVP(p_density), CEREAL_NVP(dt), CEREAL_NVP(drag), CEREAL_NVP(f_ext),
           CEREAL_NVP(num_animations), CEREAL_NVP(num_timesteps), CEREAL_NVP(control_stride), CEREAL_NVP(max_gd_iters),
           CEREAL_NVP(max_ls_iters), CEREAL_NVP(initial_alpha), CEREAL_NVP(gd_tol), CEREAL_NVP(smoothing_factor));
    }
};

static void write(const Opt& o, const char* path) {
    std::ofstream ofs(path);
    cereal::JSONOutputArchive ar(ofs);
    ar(o);
}

int main(int argc, char** argv) {
    if (argc == 4) {  // read argv[1] with cereal, write it back to argv[3] ("roundtrip" in argv[2])
        Opt o;
        {
            std::ifstream ifs(argv[1]);
            cereal::JSONInputArchive ar(ifs);
            ar(o);
        }
        write(o, argv[3]);
        return 0;
    }
    const std::string dir = argc > 1 ? argv[1] : ".";
    write(Opt{}, (dir + "/opt_input_default.json").c_str());
    Opt c;
    c.mpm_input_mesh_path = "meshes/sphere.obj";
    c.mpm_target_mesh_path = "meshes/torus.obj";
    c.grid_dx = 0.5f;
    c.points_per_cell_cuberoot = 3;
    c.grid_min_point = Vec3(-1.f, -2.f, -3.f);
    c.grid_max_point = Vec3(4.f, 5.f, 6.f);
    c.lam = 1000.f;
    c.mu = 500.f;
    c.p_density = 2.5f;
    c.dt = 1e-3f;
    c.drag = 0.25f;
    c.f_ext = Vec3(0.f, -9.8f, 0.f);
    c.num_animations = 3;
    c.num_timesteps = 7;
    c.control_stride = 5;
    c.max_gd_iters = 11;
    c.max_ls_iters = 4;
    c.initial_alpha = 0.05f;
    c.gd_tol = 1e-4f;
    c.smoothing_factor = 0.2f;
    write(c, (dir + "/opt_input_custom.json").c_str());
    return 0;
}
