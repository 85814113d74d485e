// ref_driver.cpp -- flat C ABI over the reference's own hot-path C++ API
// (DiffMPMLib3D: CompGraph, SingleThreadMPM, MultiThreadMPM, Back_Timestep,
// Elasticity).  TEST INFRASTRUCTURE: compiled by oracle/build_ref.sh together
// with the unmodified (FP32) or mechanically retyped (FP64) reference sources
// into oracle/_ref/.  Used by tests/golden/make_golden.py to produce golden
// vectors and by bench.py's CPU-baseline leg; never linked by the product.
//
// REAL is float for the shipped reference and double for the retyped build.
// All 3x3 matrices cross this ABI column-major (Eigen's storage order), i.e.
// element (i, j) of particle p sits at [p*9 + i + 3*j].
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <iostream>
#include <limits>
#include <memory>
#include <vector>
#include <omp.h>

#include "pch.h"
#include "PointCloud.h"
#include "Grid.h"
// CompGraph keeps dt / drag / f_ext / smoothing_factor private and only sets
// them inside OptimizeDefGradControlSequence (CompGraph.h:54-58).  Opening the
// class here lets the driver run exactly the initial forward / loss / backward
// sequence of CompGraph.cpp:391-405 with chosen parameters.
#define private public
#include "CompGraph.h"
#undef private
#include "ForwardSimulation.h"
#include "MultiThreadForwardSimulation.h"
#include "BackPropagation.h"
#include "Elasticity.h"
#include "Interpolation.h"
#include "qrsvd/ImplicitQRSVD.h"

#ifndef REF_REAL
#define REF_REAL float
#endif
typedef REF_REAL real;
using namespace DiffMPMLib3D;

namespace {

struct Scene {
    std::shared_ptr<PointCloud> pc;
    std::shared_ptr<Grid> grid;
    std::shared_ptr<Grid> target;
    std::unique_ptr<CompGraph> graph;
};

enum ParticleField {
    PF_X = 0, PF_V, PF_F, PF_C, PF_P, PF_M, PF_VOL, PF_LAM, PF_MU, PF_DFC,
    PF_DLDX, PF_DLDV, PF_DLDF, PF_DLDC, PF_DLDP, PF_DLDV_NEXT, PF_DLDC_NEXT,
    PF_MOMENTUM, PF_VECTOR
};
enum GridField { GF_M = 0, GF_V, GF_P, GF_DLDV, GF_DLDP, GF_DLDM, GF_X };

int particle_field_width(int f) {
    switch (f) {
    case PF_X: case PF_V: case PF_DLDX: case PF_DLDV: case PF_DLDV_NEXT: return 3;
    case PF_M: case PF_VOL: case PF_LAM: case PF_MU: return 1;
    default: return 9;
    }
}

real* particle_field_ptr(MaterialPoint& mp, int f) {
    switch (f) {
    case PF_X: return mp.x.data();
    case PF_V: return mp.v.data();
    case PF_F: return mp.F.data();
    case PF_C: return mp.C.data();
    case PF_P: return mp.P.data();
    case PF_M: return &mp.m;
    case PF_VOL: return &mp.vol;
    case PF_LAM: return &mp.lam;
    case PF_MU: return &mp.mu;
    case PF_DFC: return mp.dFc.data();
    case PF_DLDX: return mp.dLdx.data();
    case PF_DLDV: return mp.dLdv.data();
    case PF_DLDF: return mp.dLdF.data();
    case PF_DLDC: return mp.dLdC.data();
    case PF_DLDP: return mp.dLdP.data();
    case PF_DLDV_NEXT: return mp.dLdv_next.data();
    case PF_DLDC_NEXT: return mp.dLdC_next.data();
    case PF_MOMENTUM: return mp.momentum.data();
    case PF_VECTOR: return mp.vector.data();
    }
    return nullptr;
}

int grid_field_width(int f) { return (f == GF_M || f == GF_DLDM) ? 1 : 3; }

real* grid_field_ptr(GridNode& n, int f) {
    switch (f) {
    case GF_M: return &n.m;
    case GF_V: return n.v.data();
    case GF_P: return n.p.data();
    case GF_DLDV: return n.dLdv.data();
    case GF_DLDP: return n.dLdp.data();
    case GF_DLDM: return &n.dLdm;
    case GF_X: return n.x.data();
    }
    return nullptr;
}

void copy_out_particles(const PointCloud& pc, int f, real* out) {
    const int w = particle_field_width(f);
    for (size_t p = 0; p < pc.points.size(); p++) {
        MaterialPoint& mp = const_cast<MaterialPoint&>(pc.points[p]);
        std::memcpy(out + p * w, particle_field_ptr(mp, f), sizeof(real) * w);
    }
}

void copy_in_particles(PointCloud& pc, int f, const real* in) {
    const int w = particle_field_width(f);
    for (size_t p = 0; p < pc.points.size(); p++)
        std::memcpy(particle_field_ptr(pc.points[p], f), in + p * w, sizeof(real) * w);
}

void copy_out_grid(const Grid& g, int f, real* out) {
    const int w = grid_field_width(f);
    size_t idx = 0;
    for (int i = 0; i < g.dim_x; i++)
        for (int j = 0; j < g.dim_y; j++)
            for (int k = 0; k < g.dim_z; k++, idx++) {
                GridNode& n = const_cast<GridNode&>(g.nodes[i][j][k]);
                std::memcpy(out + idx * w, grid_field_ptr(n, f), sizeof(real) * w);
            }
}

Mat3 load_mat(const real* a) { Mat3 M; std::memcpy(M.data(), a, sizeof(real) * 9); return M; }
void store_mat(const Mat3& M, real* a) { std::memcpy(a, M.data(), sizeof(real) * 9); }

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

extern "C" {

int ref_real_size() { return (int)sizeof(real); }

void* ref_scene_create(int n, const real* x, const real* v, const real* F, const real* C,
                       const real* dFc, const real* m, const real* vol, const real* lam,
                       const real* mu, int dim_x, int dim_y, int dim_z, real dx,
                       const real* min_point) {
    auto* s = new Scene();
    s->pc = std::make_shared<PointCloud>();
    s->pc->points.resize(n);
    for (int p = 0; p < n; p++) {
        MaterialPoint& mp = s->pc->points[p];
        std::memcpy(mp.x.data(), x + 3 * p, sizeof(real) * 3);
        std::memcpy(mp.v.data(), v + 3 * p, sizeof(real) * 3);
        std::memcpy(mp.F.data(), F + 9 * p, sizeof(real) * 9);
        std::memcpy(mp.C.data(), C + 9 * p, sizeof(real) * 9);
        std::memcpy(mp.dFc.data(), dFc + 9 * p, sizeof(real) * 9);
        mp.m = m[p];
        mp.vol = vol[p];
        mp.lam = lam[p];
        mp.mu = mu[p];
    }
    Vec3 mn(min_point[0], min_point[1], min_point[2]);
    s->grid = std::make_shared<Grid>(dim_x, dim_y, dim_z, dx, mn);
    s->target = std::make_shared<Grid>(*s->grid);
    s->target->ResetValues();
    return s;
}

void ref_scene_destroy(void* h) { delete static_cast<Scene*>(h); }

// Target raster from an explicit mass field (flat index i*dy*dz + j*dz + k).
void ref_scene_set_target_mass(void* h, const real* tm) {
    Scene* s = static_cast<Scene*>(h);
    s->target->ResetValues();
    size_t idx = 0;
    for (int i = 0; i < s->target->dim_x; i++)
        for (int j = 0; j < s->target->dim_y; j++)
            for (int k = 0; k < s->target->dim_z; k++, idx++)
                s->target->nodes[i][j][k].m = tm[idx];
}

// Target raster as in LoadCompGraph (MPMPolyscope.cpp:155-160): ResetValues,
// then P2G of target sample points of mass mp with dt = drag = 0.
void ref_scene_target_from_points(void* h, int n, const real* x, real mp) {
    Scene* s = static_cast<Scene*>(h);
    PointCloud tpc;
    tpc.points.resize(n);
    for (int p = 0; p < n; p++) {
        std::memcpy(tpc.points[p].x.data(), x + 3 * p, sizeof(real) * 3);
        tpc.points[p].m = mp;
    }
    s->target->ResetValues();
    SingleThreadMPM::P2G(tpc, *s->target, 0.0, 0.0);
}

void ref_scene_get_target_mass(void* h, real* out) {
    copy_out_grid(*static_cast<Scene*>(h)->target, GF_M, out);
}

// CalculatePointCloudVolumes (ForwardSimulation.cpp:262-290) on a fresh grid.
void ref_scene_calc_volumes(void* h) {
    Scene* s = static_cast<Scene*>(h);
    s->grid->ResetValues();
    SingleThreadMPM::CalculatePointCloudVolumes(*s->pc, *s->grid);
}

// PointCloud::WriteEntirePointCloudToBinaryFile (PointCloud.cpp:334-346): the
// reference's own .mpmbin writer, for pinning the on-disk format.
void ref_scene_write_mpmbin(void* h, const char* path) {
    static_cast<Scene*>(h)->pc->WriteEntirePointCloudToBinaryFile(path);
}

void ref_scene_get_particles(void* h, int field, real* out) {
    copy_out_particles(*static_cast<Scene*>(h)->pc, field, out);
}

// CompGraph(initial_point_cloud, grid, target) + SetUpCompGraph(num_layers)
// with the simulation parameters that OptimizeDefGradControlSequence sets.
void ref_graph_setup(void* h, int num_layers, real dt, real drag, const real* f_ext, real smoothing) {
    Scene* s = static_cast<Scene*>(h);
    s->graph.reset(new CompGraph(s->pc, s->grid, s->target));
    s->graph->dt = dt;
    s->graph->drag = drag;
    s->graph->f_ext = Vec3(f_ext[0], f_ext[1], f_ext[2]);
    s->graph->smoothing_factor = smoothing;
    s->graph->SetUpCompGraph(num_layers);
}

int ref_graph_num_layers(void* h) { return (int)static_cast<Scene*>(h)->graph->layers.size(); }

void ref_graph_forward(void* h, int start_layer) { static_cast<Scene*>(h)->graph->ComputeForwardPass(start_layer); }

real ref_graph_loss(void* h) { return static_cast<Scene*>(h)->graph->EndLayerMassLoss(); }

void ref_graph_backward(void* h, int control_layer) { static_cast<Scene*>(h)->graph->ComputeBackwardPass(control_layer); }

real ref_graph_dldf_norm(void* h) { return static_cast<Scene*>(h)->graph->layers.front().point_cloud->Compute_dLdF_Norm(); }

void ref_graph_get_particles(void* h, int layer, int field, real* out) {
    copy_out_particles(*static_cast<Scene*>(h)->graph->layers[layer].point_cloud, field, out);
}

void ref_graph_set_particles(void* h, int layer, int field, const real* in) {
    copy_in_particles(*static_cast<Scene*>(h)->graph->layers[layer].point_cloud, field, in);
}

void ref_graph_get_grid(void* h, int layer, int field, real* out) {
    copy_out_grid(*static_cast<Scene*>(h)->graph->layers[layer].grid, field, out);
}

// PointCloud's descent rules on one layer (PointCloud.cpp:83-204).
void ref_graph_descend_adam(void* h, int layer, real alpha, real gnorm, real b1, real b2, real eps, int t) {
    static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Descend_Adam(alpha, gnorm, b1, b2, eps, t);
}
void ref_graph_descend_amsgrad(void* h, int layer, real alpha, real gnorm, real b1, real b2, real eps, int t) {
    static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Descend_AMSGrad(alpha, gnorm, b1, b2, eps, t);
}
void ref_graph_descend_lion(void* h, int layer, real alpha, real beta, real gnorm) {
    static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Descend_Lion(alpha, beta, gnorm);
}
void ref_graph_descend_gd(void* h, int layer, real alpha, real gnorm) {
    static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Descend_GradientDescent(alpha, gnorm);
}
void ref_graph_descend_dldf(void* h, int layer, real alpha, real gnorm) {
    static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Descend_dLdF(alpha, gnorm);
}
// The minibatch variants (PointCloud.cpp:51-82) on the given indices.
real ref_graph_dldf_norm_stochastic(void* h, int layer, const int* idx, int nidx) {
    const std::vector<int> mb(idx, idx + nidx);
    return static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Compute_dLdF_Norm_Stochastic(mb);
}
void ref_graph_descend_adam_stochastic(void* h, int layer, real alpha, real gnorm, real b1, real b2, real eps, int t,
                                       const int* idx, int nidx) {
    const std::vector<int> mb(idx, idx + nidx);
    static_cast<Scene*>(h)->graph->layers[layer].point_cloud->Descend_Adam_Stochastic(alpha, gnorm, b1, b2, eps, t, mb);
}

// Timed forward of layers [0, steps) with MultiThreadMPM::ForwardTimeStep
// (MultiThreadForwardSimulation.cpp:7-154) using `threads` proxy grids.
// Requires a graph set up with at least steps + 1 layers.  Returns seconds.
double ref_time_forward_multithread(void* h, int steps, int threads) {
    Scene* s = static_cast<Scene*>(h);
    CompGraph& g = *s->graph;
    std::vector<std::shared_ptr<Grid>> proxies;
    for (int t = 0; t < threads; t++) proxies.push_back(std::make_shared<Grid>(*g.layers[0].grid));
    double t0 = now_s();
    for (int i = 0; i < steps; i++)
        MultiThreadMPM::ForwardTimeStep(*g.layers[i + 1].point_cloud, *g.layers[i].point_cloud,
                                        *g.layers[i].grid, proxies, g.dt, g.drag, g.f_ext);
    return now_s() - t0;
}

// Timed EndLayerMassLoss + ComputeBackwardPass(0) (serial build).  Seconds.
double ref_time_loss_backward(void* h, real* loss_out) {
    Scene* s = static_cast<Scene*>(h);
    double t0 = now_s();
    real L = s->graph->EndLayerMassLoss();
    s->graph->ComputeBackwardPass(0);
    double t1 = now_s();
    if (loss_out) *loss_out = L;
    return t1 - t0;
}

// ---- elementary functions (Interpolation.h, Elasticity.cpp, ImplicitQRSVD.h) ----
real ref_bspline(real x) { return CubicBSpline(x); }
real ref_bspline_slope(real x) { return CubicBSplineSlope(x); }

void ref_pk(const real* F, real lam, real mu, real* P) { store_mat(PK_FixedCorotatedElasticity(load_mat(F), lam, mu), P); }

real ref_energy(const real* F, real lam, real mu) { return FixedCorotatedElasticity(load_mat(F), lam, mu); }

void ref_polar(const real* F, real* R, real* S) {
    Mat3 Rm, Sm;
    JIXIE::polarDecomposition(load_mat(F), Rm, Sm);
    store_mat(Rm, R);
    store_mat(Sm, S);
}

void ref_svd(const real* F, real* U, real* sigma, real* V) {
    Mat3 Um, Vm;
    Vec3 s;
    JIXIE::singularValueDecomposition(load_mat(F), Um, s, Vm);
    store_mat(Um, U);
    store_mat(Vm, V);
    sigma[0] = s[0]; sigma[1] = s[1]; sigma[2] = s[2];
}

void ref_d2(const real* F, real lam, real mu, const real* dF, real* out) {
    store_mat(d2_FCE_psi_dF2_mult_by_dF(load_mat(F), lam, mu, load_mat(dF)), out);
}

// Full 81-entry tensors: out[((a*3+b)*3+i)*3+j] = T[a][b](i, j).
static void store_tensor(const Tensor3x3x3x3& T, real* out) {
    for (int a = 0; a < 3; a++) for (int b = 0; b < 3; b++)
        for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
            out[((a * 3 + b) * 3 + i) * 3 + j] = T[a][b](i, j);
}
void ref_d2_tensor_fd(const real* F, real lam, real mu, real* out) { store_tensor(d2_FCE_psi_dF2_FD(load_mat(F), lam, mu), out); }
void ref_d2_tensor_trick(const real* F, real lam, real mu, real* out) { store_tensor(d2_FCE_psi_dF2_mult_trick(load_mat(F), lam, mu), out); }
void ref_djfit_fd(const real* F, real* out) { store_tensor(d_JFit_dF_FD(load_mat(F)), out); }

void ref_lame(real E, real nu, real* lam, real* mu) { CalculateLameParameters(E, nu, *lam, *mu); }

}  // extern "C"
