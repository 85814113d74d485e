// dmpm_compat.cpp -- the DiffMPMLib3D-compatible C++ API (compat/DiffMPMLib3D/*.h)
// implemented over the engine's C ABI (include/dmpm.h).  Every simulation
// stage runs on the GPU; the host side holds the reference's data structures
// (PointCloud / Grid / CompGraph::layers) and moves them to and from the engine.
// Optimiser steps, file IO and gradient norms are host code, as in the
// reference (PointCloud.cpp).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <limits>
#include <random>
#include <stdexcept>
#include <string>

#include "DiffMPMLib3D/BackPropagation.h"
#include "DiffMPMLib3D/CompGraph.h"
#include "DiffMPMLib3D/Elasticity.h"
#include "DiffMPMLib3D/ForwardSimulation.h"
#include "DiffMPMLib3D/GeometryLoading.h"
#include "DiffMPMLib3D/MultiThreadForwardSimulation.h"
#include "DiffMPMLib3D/SphereUnionSurfacing.h"
#include "dmpm.h"

namespace DiffMPMLib3D {

namespace {

void check(dmpm_ctx* ctx, int st, const char* what) {
    if (st == DMPM_OK || st == DMPM_ERR_NONFINITE) return;  // NaN propagates silently, as in the reference
    std::string msg = std::string(what) + " failed (status " + std::to_string(st) + ")";
    if (ctx) msg += ": " + std::string(dmpm_last_error(ctx));
    throw std::runtime_error(msg);
}

struct Ctx {  // RAII context for the stage functions
    dmpm_ctx* h = nullptr;
    explicit Ctx(int precision, int device = 0) { check(nullptr, dmpm_create(device, precision, &h), "dmpm_create"); }
    ~Ctx() { if (h) dmpm_destroy(h); }
};

size_t num_nodes(const Grid& g) { return (size_t)g.dim_x * g.dim_y * g.dim_z; }

template <class Fn> void for_nodes(Grid& g, Fn fn) {
    size_t idx = 0;
    for (int i = 0; i < g.dim_x; i++)
        for (int j = 0; j < g.dim_y; j++)
            for (int k = 0; k < g.dim_z; k++, idx++) fn(g.nodes[i][j][k], idx);
}
template <class Fn> void for_nodes(const Grid& g, Fn fn) {
    size_t idx = 0;
    for (int i = 0; i < g.dim_x; i++)
        for (int j = 0; j < g.dim_y; j++)
            for (int k = 0; k < g.dim_z; k++, idx++) fn(g.nodes[i][j][k], idx);
}

void set_grid(dmpm_ctx* h, const Grid& g) {
    const double mn[3] = {g.min_point[0], g.min_point[1], g.min_point[2]};
    check(h, dmpm_set_grid(h, g.dim_x, g.dim_y, g.dim_z, g.dx, mn), "dmpm_set_grid");
}

int g_stage_precision = DMPM_FP32_MIXED;
int g_stage_deterministic = 0;

// det < 0: the stage functions' setting (SingleThreadMPM::SetEngineDeterministic)
void set_params(dmpm_ctx* h, float dt, float drag, Vec3 f, float s, int adjoint, int keep_adj, int keep_int,
                int det = -1, int reorder = 0) {
    dmpm_params p;
    dmpm_default_params(&p);
    p.deterministic = det < 0 ? g_stage_deterministic : det;
    p.reorder_particles = reorder;
    p.dt = dt;
    p.drag = drag;
    p.f_ext[0] = f[0]; p.f_ext[1] = f[1]; p.f_ext[2] = f[2];
    p.smoothing = s;
    p.adjoint_mode = adjoint;
    p.control_mode = DMPM_CTRL_PER_LAYER;
    p.loss_kind = DMPM_LOSS_REF_LOGMASS;
    p.checkpoint_every = 1;
    p.keep_adjoints = keep_adj;
    p.keep_intermediates = keep_int;
    check(h, dmpm_set_params(h, &p), "dmpm_set_params");
}

// per-particle field <-> column-major double arrays
void put_field(dmpm_ctx* h, int layer, int field, const std::vector<MaterialPoint>& pts) {
    const int w = (field == DMPM_F_X || field == DMPM_F_V || field == DMPM_F_DLDX || field == DMPM_F_DLDV) ? 3 : 9;
    std::vector<double> a(pts.size() * w);
    for (size_t p = 0; p < pts.size(); p++) {
        const float* src = nullptr;
        switch (field) {
            case DMPM_F_X: src = pts[p].x.data(); break;
            case DMPM_F_V: src = pts[p].v.data(); break;
            case DMPM_F_F: src = pts[p].F.data(); break;
            case DMPM_F_C: src = pts[p].C.data(); break;
            case DMPM_F_DFC: src = pts[p].dFc.data(); break;
            case DMPM_F_DLDX: src = pts[p].dLdx.data(); break;
            case DMPM_F_DLDV: src = pts[p].dLdv.data(); break;
            case DMPM_F_DLDF: src = pts[p].dLdF.data(); break;
            case DMPM_F_DLDC: src = pts[p].dLdC.data(); break;
        }
        for (int q = 0; q < w; q++) a[p * w + q] = src[q];
    }
    check(h, dmpm_set_layer_particles(h, layer, field, a.data()), "dmpm_set_layer_particles");
}

void get_field(dmpm_ctx* h, int layer, int field, std::vector<MaterialPoint>& pts) {
    const int w = (field == DMPM_F_X || field == DMPM_F_V || field == DMPM_F_DLDX || field == DMPM_F_DLDV ||
                   field == DMPM_F_DLDV_NEXT) ? 3 : 9;
    std::vector<double> a(pts.size() * w);
    check(h, dmpm_get_particles(h, layer, field, a.data()), "dmpm_get_particles");
    for (size_t p = 0; p < pts.size(); p++) {
        float* dst = nullptr;
        switch (field) {
            case DMPM_F_P: dst = pts[p].P.data(); break;
            case DMPM_F_DLDX: dst = pts[p].dLdx.data(); break;
            case DMPM_F_DLDV: dst = pts[p].dLdv.data(); break;
            case DMPM_F_DLDF: dst = pts[p].dLdF.data(); break;
            case DMPM_F_DLDC: dst = pts[p].dLdC.data(); break;
            case DMPM_F_DLDP: dst = pts[p].dLdP.data(); break;
            case DMPM_F_DLDV_NEXT: dst = pts[p].dLdv_next.data(); break;
            case DMPM_F_DLDC_NEXT: dst = pts[p].dLdC_next.data(); break;
        }
        for (int q = 0; q < w; q++) dst[q] = (float)a[p * w + q];
    }
}

void get_grid_into(dmpm_ctx* h, int layer, Grid& g, bool values, bool adjoints) {
    const size_t G = num_nodes(g);
    std::vector<double> a(3 * G);
    if (values) {
        check(h, dmpm_get_grid(h, layer, DMPM_G_M, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { n.m = (float)a[i]; });
        check(h, dmpm_get_grid(h, layer, DMPM_G_V, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { for (int c = 0; c < 3; c++) n.v[c] = (float)a[3 * i + c]; });
        check(h, dmpm_get_grid(h, layer, DMPM_G_P, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { for (int c = 0; c < 3; c++) n.p[c] = (float)a[3 * i + c]; });
    }
    if (adjoints) {
        check(h, dmpm_get_grid(h, layer, DMPM_G_DLDV, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { for (int c = 0; c < 3; c++) n.dLdv[c] = (float)a[3 * i + c]; });
        check(h, dmpm_get_grid(h, layer, DMPM_G_DLDP, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { for (int c = 0; c < 3; c++) n.dLdp[c] = (float)a[3 * i + c]; });
        check(h, dmpm_get_grid(h, layer, DMPM_G_DLDM, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { n.dLdm = (float)a[i]; });
    }
}

std::vector<double> to_cm_doubles(const std::vector<Mat3>& M) {
    std::vector<double> a(M.size() * 9);
    for (size_t p = 0; p < M.size(); p++)
        for (int q = 0; q < 9; q++) a[9 * p + q] = M[p].data()[q];
    return a;
}

}  // namespace

// ====================================================================== structs
void MaterialPoint::ResetGradients() {
    dLdx.setZero();
    dLdv.setZero();
    dLdF.setZero();
    dLdC.setZero();
    dLdP.setZero();
    dLdv_next.setZero();
    dLdC_next.setZero();
}

void GridNode::ResetGradients() {
    dLdx.setZero();
    dLdv.setZero();
    dLdp.setZero();
    dLdm = 0.f;
}

Grid::Grid(int _dim_x, int _dim_y, int _dim_z, float _dx, Vec3 _min_point)
    : dim_x(_dim_x), dim_y(_dim_y), dim_z(_dim_z), dx(_dx), min_point(_min_point) {
    nodes.assign(dim_x, std::vector<std::vector<GridNode>>(dim_y, std::vector<GridNode>(dim_z)));
    for (int i = 0; i < dim_x; i++)
        for (int j = 0; j < dim_y; j++)
            for (int k = 0; k < dim_z; k++)
                nodes[i][j][k].x = min_point + Vec3((float)i, (float)j, (float)k) * dx;
}

namespace {
template <class G, class Node>
std::vector<std::reference_wrapper<Node>> query_stencil(G& grid, const Vec3& point,
                                                        std::vector<std::array<int, 3>>* indices) {
    std::vector<std::reference_wrapper<Node>> ret;
    int b[3];
    for (int a = 0; a < 3; a++) b[a] = (int)std::floor((point[a] - grid.min_point[a]) / grid.dx) - 1;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++) {
                const int n[3] = {b[0] + i, b[1] + j, b[2] + k};
                if (n[0] < 0 || n[0] >= grid.dim_x || n[1] < 0 || n[1] >= grid.dim_y || n[2] < 0 || n[2] >= grid.dim_z)
                    continue;
                ret.push_back(std::ref(grid.nodes[n[0]][n[1]][n[2]]));
                if (indices) indices->push_back({n[0], n[1], n[2]});
            }
    return ret;
}
}  // namespace

std::vector<std::reference_wrapper<GridNode>> Grid::QueryPoint_CubicBSpline(Vec3 point,
                                                                          std::vector<std::array<int, 3>>* indices) {
    return query_stencil<Grid, GridNode>(*this, point, indices);
}
std::vector<std::reference_wrapper<const GridNode>> Grid::QueryPointConst_CubicBSpline(
    Vec3 point, std::vector<std::array<int, 3>>* indices) const {
    return query_stencil<const Grid, const GridNode>(*this, point, indices);
}

std::vector<GridNode> Grid::flatten() const {
    std::vector<GridNode> flat;
    flat.reserve(num_nodes(*this));
    for_nodes(*this, [&](const GridNode& n, size_t) { flat.push_back(n); });
    return flat;
}

void Grid::unflatten(const std::vector<GridNode>& flat) {
    nodes.assign(dim_x, std::vector<std::vector<GridNode>>(dim_y, std::vector<GridNode>(dim_z)));
    for_nodes(*this, [&](GridNode& n, size_t i) {
        if (i < flat.size()) n = flat[i];
    });
}

std::vector<Vec3> Grid::GetNodePositions() const {
    std::vector<Vec3> r(num_nodes(*this));
    for_nodes(*this, [&](const GridNode& n, size_t i) { r[i] = n.x; });
    return r;
}
std::vector<float> Grid::GetNodeMasses() const {
    std::vector<float> r(num_nodes(*this));
    for_nodes(*this, [&](const GridNode& n, size_t i) { r[i] = n.m; });
    return r;
}
std::vector<Vec3> Grid::GetNodeVelocities() const {
    std::vector<Vec3> r(num_nodes(*this));
    for_nodes(*this, [&](const GridNode& n, size_t i) { r[i] = n.v; });
    return r;
}
void Grid::ResetGradients() {
    for_nodes(*this, [&](GridNode& n, size_t) { n.ResetGradients(); });
}
void Grid::ResetValues() {
    for_nodes(*this, [&](GridNode& n, size_t) {
        n.m = 0.f;
        n.v.setZero();
        n.p.setZero();
    });
}

// ====================================================================== PointCloud (host, PointCloud.cpp)
void PointCloud::ResetGradients() {
    for (auto& p : points) p.ResetGradients();
}

float PointCloud::Compute_dLdF_Norm() {
    float norm = 0.f;
    for (auto& p : points) norm += p.dLdF.squaredNorm();
    return std::sqrt(norm);
}

void PointCloud::Descend_dLdF(float alpha, float gradient_norm) {
    const float momentum_factor = 0.9f, min_clip = 1e-3f, max_clip = 1.0f;
    for (auto& p : points) {
        Mat3 dir = p.dLdF * (1.f / gradient_norm);
        for (int q = 0; q < 9; q++) {
            float& v = dir.data()[q];
            if (v > max_clip) v = max_clip;
            else if (v < -max_clip) v = -max_clip;
            else if (std::fabs(v) < min_clip) v = v < 0 ? -min_clip : min_clip;
        }
        p.momentum = p.momentum * momentum_factor + dir * alpha;
        p.dFc = p.dFc - p.momentum;
    }
}

void PointCloud::Descend_Adam(float alpha, float gradient_norm, float beta1, float beta2, float epsilon, int t) {
    const float c1 = 1.f - std::pow(beta1, (float)t), c2 = 1.f - std::pow(beta2, (float)t);
    for (auto& p : points) {
        for (int k = 0; k < 9; k++) {
            const float g = p.dLdF.data()[k] / gradient_norm;
            p.momentum.data()[k] = beta1 * p.momentum.data()[k] + (1.f - beta1) * g;
            p.vector.data()[k] = beta2 * p.vector.data()[k] + (1.f - beta2) * g * g;
            const float mh = p.momentum.data()[k] / c1, vh = p.vector.data()[k] / c2;
            p.dFc.data()[k] -= alpha * (mh / (std::sqrt(vh) + epsilon));
        }
    }
}

void PointCloud::Descend_AMSGrad(float alpha, float gradient_norm, float beta1, float beta2, float epsilon, int t) {
    const float c1 = 1.f - std::pow(beta1, (float)t), c2 = 1.f - std::pow(beta2, (float)t);
    for (auto& p : points) {
        for (int k = 0; k < 9; k++) {
            const float g = p.dLdF.data()[k] / gradient_norm;
            p.momentum.data()[k] = beta1 * p.momentum.data()[k] + (1.f - beta1) * g;
            p.vector.data()[k] = beta2 * p.vector.data()[k] + (1.f - beta2) * g * g;
            const float mh = p.momentum.data()[k] / c1, vh = p.vector.data()[k] / c2;
            p.vector_max.data()[k] = std::max(p.vector_max.data()[k], vh);
            p.dFc.data()[k] -= alpha * (mh / (std::sqrt(p.vector_max.data()[k]) + epsilon));
        }
    }
}

std::vector<int> PointCloud::generateMinibatchIndices(int total_size, int minibatch_size) {
    std::vector<int> idx((size_t)std::max(0, total_size));
    for (int i = 0; i < total_size; i++) idx[(size_t)i] = i;
    std::mt19937 rng((unsigned)std::chrono::system_clock::now().time_since_epoch().count());
    std::shuffle(idx.begin(), idx.end(), rng);
    idx.resize((size_t)std::max(0, std::min(minibatch_size, total_size)));
    return idx;
}

float PointCloud::Compute_dLdF_Norm_Stochastic(const std::vector<int>& minibatch_indices) {
    float norm = 0.f;
    for (int i : minibatch_indices) norm += points[(size_t)i].dLdF.squaredNorm();
    return std::sqrt(norm);
}

void PointCloud::Descend_Adam_Stochastic(float alpha, float gradient_norm, float beta1, float beta2, float epsilon,
                                         int timestep, const std::vector<int>& minibatch_indices) {
    const float c1 = 1.f - std::pow(beta1, (float)(timestep + 1)), c2 = 1.f - std::pow(beta2, (float)(timestep + 1));
    for (int i : minibatch_indices) {
        MaterialPoint& p = points[(size_t)i];
        for (int k = 0; k < 9; k++) {
            const float g = p.dLdF.data()[k] / gradient_norm;
            p.momentum.data()[k] = beta1 * p.momentum.data()[k] + (1.f - beta1) * g;
            p.vector.data()[k] = beta2 * p.vector.data()[k] + (1.f - beta2) * g * g;
            const float mh = p.momentum.data()[k] / c1, vh = p.vector.data()[k] / c2;
            p.dFc.data()[k] -= alpha * (mh / (std::sqrt(vh) + epsilon));
        }
    }
}

void PointCloud::Descend_GradientDescent(float alpha, float gradient_norm) {
    for (auto& p : points)
        for (int k = 0; k < 9; k++) p.dFc.data()[k] -= alpha * p.dLdF.data()[k] / gradient_norm;
}

void PointCloud::Descend_Lion(float alpha, float beta, float gradient_norm) {
    for (auto& p : points) {
        for (int k = 0; k < 9; k++) {
            const float g = p.dLdF.data()[k] / gradient_norm;
            const float sg = g > 0.f ? 1.f : (g < 0.f ? -1.f : 0.f);
            p.momentum.data()[k] = beta * p.momentum.data()[k] + (1.f - beta) * sg;
            p.dFc.data()[k] -= alpha * p.momentum.data()[k];
        }
    }
}

bool PointCloud::ReadFromOBJ(std::string obj_path, float point_mass) {
    points.clear();
    std::ifstream ifs(obj_path);
    if (!ifs.good()) {
        std::cout << "couldn't open file: " << obj_path << std::endl;
        return false;
    }
    std::string junk;
    float x, y, z;
    while (ifs >> junk >> x >> y >> z) {
        MaterialPoint mp;
        mp.x = Vec3(x, y, z);
        mp.m = point_mass;
        points.push_back(mp);
    }
    return true;
}

void PointCloud::WriteToOBJ(std::string obj_path) {
    std::ofstream ofs(obj_path);
    if (!ofs) {
        std::cerr << "Could not open file for writing: " << obj_path << std::endl;
        return;
    }
    for (auto& p : points) ofs << "v " << p.x[0] << " " << p.x[1] << " " << p.x[2] << "\n";
}

namespace {
// cereal binary archive pieces (little-endian, as cereal writes on x86)
void w_i32(std::ostream& o, int32_t v) { o.write((const char*)&v, 4); }
void w_f32(std::ostream& o, float v) { o.write((const char*)&v, 4); }
void w_vec(std::ostream& o, const Vec3& v) { w_i32(o, 3); for (int i = 0; i < 3; i++) w_f32(o, v[i]); }
void w_mat(std::ostream& o, const Mat3& m) {
    w_i32(o, 3);
    w_i32(o, 3);
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) w_f32(o, m(i, j));
}
bool r_i32(std::istream& s, int32_t& v) { return (bool)s.read((char*)&v, 4); }
bool r_f32(std::istream& s, float& v) { return (bool)s.read((char*)&v, 4); }
bool r_vec(std::istream& s, Vec3& v) {
    int32_t rows;
    if (!r_i32(s, rows) || rows != 3) return false;
    for (int i = 0; i < 3; i++) if (!r_f32(s, v[i])) return false;
    return true;
}
bool r_mat(std::istream& s, Mat3& m) {
    int32_t rows, cols;
    if (!r_i32(s, rows) || !r_i32(s, cols) || rows != 3 || cols != 3) return false;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) if (!r_f32(s, m(i, j))) return false;
    return true;
}
}  // namespace

void PointCloud::WriteEntirePointCloudToBinaryFile(std::string file_path) {
    std::ofstream ofs(file_path, std::ios::binary);
    if (!ofs.good()) return;
    const uint64_t n = points.size();
    ofs.write((const char*)&n, 8);
    for (const auto& p : points) {
        w_vec(ofs, p.x); w_vec(ofs, p.v); w_mat(ofs, p.F); w_mat(ofs, p.C); w_mat(ofs, p.P);
        w_f32(ofs, p.m); w_f32(ofs, p.vol); w_f32(ofs, p.lam); w_f32(ofs, p.mu);
        w_mat(ofs, p.dFc); w_vec(ofs, p.dLdx); w_vec(ofs, p.dLdv); w_mat(ofs, p.dLdF);
        w_mat(ofs, p.momentum); w_mat(ofs, p.vector); w_mat(ofs, p.vector_max);
    }
}

bool PointCloud::ReadEntirePointCloudFromBinaryFile(std::string file_path) {
    std::ifstream ifs(file_path, std::ios::binary);
    if (!ifs.good()) {
        std::cout << "couldn't read file: " << file_path << std::endl;
        return false;
    }
    uint64_t n = 0;
    if (!ifs.read((char*)&n, 8)) return false;
    std::vector<MaterialPoint> pts(n);
    for (auto& p : pts) {
        if (!(r_vec(ifs, p.x) && r_vec(ifs, p.v) && r_mat(ifs, p.F) && r_mat(ifs, p.C) && r_mat(ifs, p.P) &&
              r_f32(ifs, p.m) && r_f32(ifs, p.vol) && r_f32(ifs, p.lam) && r_f32(ifs, p.mu) && r_mat(ifs, p.dFc) &&
              r_vec(ifs, p.dLdx) && r_vec(ifs, p.dLdv) && r_mat(ifs, p.dLdF) && r_mat(ifs, p.momentum) &&
              r_mat(ifs, p.vector) && r_mat(ifs, p.vector_max)))
            return false;
    }
    points.swap(pts);
    return true;
}

bool PointCloud::IsEqualToOtherPointCloud(const PointCloud& o) {
    if (o.points.size() != points.size()) return false;
    for (size_t i = 0; i < points.size(); i++) {
        const MaterialPoint &a = points[i], &b = o.points[i];
        if (std::memcmp(a.x.data(), b.x.data(), 12) || std::memcmp(a.v.data(), b.v.data(), 12) ||
            std::memcmp(a.F.data(), b.F.data(), 36) || std::memcmp(a.C.data(), b.C.data(), 36) ||
            std::memcmp(a.P.data(), b.P.data(), 36) || a.m != b.m || a.vol != b.vol || a.lam != b.lam || a.mu != b.mu) {
            std::cout << "Not equal at point " << i << std::endl;
            return false;
        }
    }
    std::cout << "Point clouds are equal" << std::endl;
    return true;
}

std::vector<Vec3> PointCloud::GetPointPositions() const {
    std::vector<Vec3> r(points.size());
    for (size_t i = 0; i < points.size(); i++) r[i] = points[i].x;
    return r;
}
std::vector<float> PointCloud::GetPointMasses() const {
    std::vector<float> r(points.size());
    for (size_t i = 0; i < points.size(); i++) r[i] = points[i].m;
    return r;
}
std::vector<float> PointCloud::GetPointVolumes() const {
    std::vector<float> r(points.size());
    for (size_t i = 0; i < points.size(); i++) r[i] = points[i].vol;
    return r;
}
std::vector<Mat3> PointCloud::GetPointDefGrads() const {
    std::vector<Mat3> r(points.size());
    for (size_t i = 0; i < points.size(); i++) r[i] = points[i].F;
    return r;
}
std::vector<float> PointCloud::GetPointDeterminants() const {
    std::vector<float> r(points.size());
    for (size_t i = 0; i < points.size(); i++) {
        const Mat3& F = points[i].F;
        r[i] = F(0, 0) * (F(1, 1) * F(2, 2) - F(1, 2) * F(2, 1)) - F(0, 1) * (F(1, 0) * F(2, 2) - F(1, 2) * F(2, 0)) +
               F(0, 2) * (F(1, 0) * F(2, 1) - F(1, 1) * F(2, 0));
    }
    return r;
}

// ====================================================================== Elasticity (GPU, FP64)
namespace {
std::vector<Mat3> elementary_batch(int kind, const std::vector<Mat3>& F, float lam, float mu,
                                   const std::vector<Mat3>* dF) {
    const int n = (int)F.size();
    std::vector<double> a = to_cm_doubles(F), l(n, lam), m(n, mu), out((size_t)n * 9);
    std::vector<double> b = dF ? to_cm_doubles(*dF) : std::vector<double>();
    check(nullptr, dmpm_elementary(kind, n, a.data(), l.data(), m.data(), dF ? b.data() : nullptr, out.data()),
          "dmpm_elementary");
    std::vector<Mat3> r(n);
    for (int p = 0; p < n; p++)
        for (int q = 0; q < 9; q++) r[p].data()[q] = (float)out[9 * (size_t)p + q];
    return r;
}
}  // namespace

std::vector<Mat3> PK_FixedCorotatedElasticityBatch(const std::vector<Mat3>& F, float lam, float mu) {
    return elementary_batch(DMPM_ELEM_PK, F, lam, mu, nullptr);
}
std::vector<Mat3> d2_FCE_psi_dF2_mult_by_dF_Batch(const std::vector<Mat3>& F, float lam, float mu,
                                                  const std::vector<Mat3>& dF, bool exact) {
    return elementary_batch(exact ? DMPM_ELEM_D2_EXACT : DMPM_ELEM_D2_REFCOMPAT, F, lam, mu, &dF);
}
Mat3 PK_FixedCorotatedElasticity(const Mat3& F, float lam, float mu) {
    return PK_FixedCorotatedElasticityBatch({F}, lam, mu)[0];
}
Mat3 d2_FCE_psi_dF2_mult_by_dF(const Mat3& F, float lam, float mu, const Mat3& dF) {
    return d2_FCE_psi_dF2_mult_by_dF_Batch({F}, lam, mu, {dF})[0];
}
float FixedCorotatedElasticity(const Mat3& F, float lam, float mu) {
    std::vector<double> a = to_cm_doubles({F}), l(1, lam), m(1, mu), out(1);
    check(nullptr, dmpm_elementary(DMPM_ELEM_ENERGY, 1, a.data(), l.data(), m.data(), nullptr, out.data()),
          "dmpm_elementary");
    return (float)out[0];
}
// [a][b](i, j) = dP_ab / dF_ij, from dP/dF : E_ij (Elasticity.cpp:181-229)
Tensor3x3x3x3 d2_FCE_psi_dF2_mult_trick(const Mat3& F, float lam, float mu) {
    std::vector<Mat3> Fs(9, F), E(9);
    for (int k = 0; k < 9; k++) E[k](k / 3, k % 3) = 1.f;
    std::vector<Mat3> r = d2_FCE_psi_dF2_mult_by_dF_Batch(Fs, lam, mu, E, false);
    Tensor3x3x3x3 t;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) t[a][b] = r[a * 3 + b];
    return t;
}
Tensor3x3x3x3 d2_FCE_psi_dF2_FD(const Mat3& F, float lam, float mu) {
    const float delta = 1e-6f;
    std::vector<Mat3> Fs;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            Mat3 Fp = F, Fm = F;
            Fp(i, j) += delta;
            Fm(i, j) -= delta;
            Fs.push_back(Fp);
            Fs.push_back(Fm);
        }
    std::vector<Mat3> P = PK_FixedCorotatedElasticityBatch(Fs, lam, mu);
    Tensor3x3x3x3 t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const Mat3& Pp = P[2 * (i * 3 + j)];
            const Mat3& Pm = P[2 * (i * 3 + j) + 1];
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) t[a][b](i, j) = (Pp(a, b) - Pm(a, b)) / (2.f * delta);
        }
    return t;
}
namespace {
// J F^-T of a 3x3 matrix in FP64: the cofactor matrix (J F^-T = cof(F))
void jfit_d(const double F[3][3], double out[3][3]) {
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++) {
            const int a1 = (a + 1) % 3, a2 = (a + 2) % 3, b1 = (b + 1) % 3, b2 = (b + 2) % 3;
            out[a][b] = F[a1][b1] * F[a2][b2] - F[a1][b2] * F[a2][b1];
        }
}
}  // namespace

Tensor3x3x3x3 d_JFit_dF_FD(const Mat3& F) {
    const double delta = 1e-6;
    double G[3][3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) G[i][j] = F(i, j);
    Tensor3x3x3x3 t;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const double orig = G[i][j];
            double fwd[3][3], bwd[3][3];
            G[i][j] = orig + delta;
            jfit_d(G, fwd);
            G[i][j] = orig - delta;
            jfit_d(G, bwd);
            G[i][j] = orig;
            for (int a = 0; a < 3; a++)
                for (int b = 0; b < 3; b++) t[a][b](i, j) = (float)((fwd[a][b] - bwd[a][b]) / (2.0 * delta));
        }
    return t;
}

// d(J F^-T)_ab / dF_ij = J (F^-T_ab F^-T_ij - F^-T_aj F^-T_ib)  (dJ/dF = J F^-T, dF^-T = -F^-T dF^T F^-T)
Tensor3x3x3x3 d_JFit_dF(float J, const Mat3& Fit) {
    Tensor3x3x3x3 t;
    for (int a = 0; a < 3; a++)
        for (int b = 0; b < 3; b++)
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++)
                    t[a][b](i, j) = (float)((double)J * ((double)Fit(a, b) * Fit(i, j) - (double)Fit(a, j) * Fit(i, b)));
    return t;
}

void CalculateLameParameters(float young_mod, float poisson, float& lam, float& mu) {
    lam = young_mod * poisson / ((1.f + poisson) * (1.f - 2.f * poisson));
    mu = young_mod / (2.f + 2.f * poisson);
}

// ====================================================================== SingleThreadMPM (GPU)
namespace SingleThreadMPM {

void ForwardTimeStep(PointCloud& next, PointCloud& curr, Grid& grid, float dt, float drag, Vec3 f_ext) {
    ForwardTimeStep(next, curr, grid, 0.f, dt, drag, f_ext);
}

void ForwardTimeStep(PointCloud& next, PointCloud& curr, Grid& grid, float s, float dt, float drag, Vec3 f_ext) {
    Ctx c(g_stage_precision);
    set_grid(c.h, grid);
    check(c.h, dmpm_set_points_ref(c.h, curr.points.data(), (int)curr.points.size()), "dmpm_set_points_ref");
    std::vector<double> zeros(num_nodes(grid), 0.0);
    check(c.h, dmpm_set_target_mass(c.h, zeros.data()), "dmpm_set_target_mass");
    set_params(c.h, dt, drag, f_ext, s, DMPM_ADJ_REFCOMPAT, 0, 0);
    check(c.h, dmpm_setup(c.h, 2), "dmpm_setup");
    check(c.h, dmpm_forward(c.h, 0), "dmpm_forward");
    get_field(c.h, 0, DMPM_F_P, curr.points);  // P_op_1 writes P into the current cloud
    if (next.points.size() != curr.points.size()) next.points = curr.points;
    check(c.h, dmpm_get_points_ref(c.h, 1, next.points.data()), "dmpm_get_points_ref");
    get_grid_into(c.h, 0, grid, true, false);
}

void P_op_1(PointCloud& pc) {
    std::vector<Mat3> Fe(pc.points.size());
    for (size_t p = 0; p < pc.points.size(); p++) Fe[p] = pc.points[p].F + pc.points[p].dFc;
    if (pc.points.empty()) return;
    // per-particle lam / mu
    const int n = (int)Fe.size();
    std::vector<double> a = to_cm_doubles(Fe), l(n), m(n), out((size_t)n * 9);
    for (int p = 0; p < n; p++) { l[p] = pc.points[p].lam; m[p] = pc.points[p].mu; }
    check(nullptr, dmpm_elementary(DMPM_ELEM_PK, n, a.data(), l.data(), m.data(), nullptr, out.data()),
          "dmpm_elementary");
    for (int p = 0; p < n; p++)
        for (int q = 0; q < 9; q++) pc.points[p].P.data()[q] = (float)out[9 * (size_t)p + q];
}

void G_Reset(Grid& grid) { grid.ResetValues(); }

void SetEnginePrecision(int precision) { g_stage_precision = precision; }
void SetEngineDeterministic(bool on) { g_stage_deterministic = on ? 1 : 0; }

// Adds this cloud's P2G mass and momentum to the grid (the reference
// accumulates without resetting, ForwardSimulation.cpp:174-182).  The stress
// term uses P of F + dFc, evaluated by the engine.  Always on the FP64 path,
// which keeps the momentum (the FP32 path's grid update overwrites it with v).
void P2G(const PointCloud& pc, Grid& grid, float dt, float drag) {
    if (pc.points.empty()) return;
    Ctx c(DMPM_FP64);
    set_grid(c.h, grid);
    check(c.h, dmpm_set_points_ref(c.h, pc.points.data(), (int)pc.points.size()), "dmpm_set_points_ref");
    std::vector<double> zeros(num_nodes(grid), 0.0);
    check(c.h, dmpm_set_target_mass(c.h, zeros.data()), "dmpm_set_target_mass");
    set_params(c.h, dt, drag, Vec3::Zero(), 0.f, DMPM_ADJ_REFCOMPAT, 0, 0);
    check(c.h, dmpm_setup(c.h, 2), "dmpm_setup");
    check(c.h, dmpm_forward(c.h, 0), "dmpm_forward");
    const size_t G = num_nodes(grid);
    std::vector<double> m(G), p(3 * G);
    check(c.h, dmpm_get_grid(c.h, 0, DMPM_G_M, m.data()), "dmpm_get_grid");
    check(c.h, dmpm_get_grid(c.h, 0, DMPM_G_P, p.data()), "dmpm_get_grid");
    for_nodes(grid, [&](GridNode& nd, size_t i) {
        nd.m += (float)m[i];
        for (int k = 0; k < 3; k++) nd.p[k] += (float)p[3 * i + k];
    });
}

namespace {
void grid_arrays(const Grid& g, std::vector<float>& m, std::vector<float>& p, std::vector<float>& v) {
    const size_t G = num_nodes(g);
    m.resize(G);
    p.resize(3 * G);
    v.resize(3 * G);
    for_nodes(g, [&](const GridNode& nd, size_t i) {
        m[i] = nd.m;
        for (int k = 0; k < 3; k++) {
            p[3 * i + k] = nd.p[k];
            v[3 * i + k] = nd.v[k];
        }
    });
}
void g_op(Grid& grid, float dt, const float* f, const float* gp, float gmag) {
    std::vector<float> m, p, v;
    grid_arrays(grid, m, p, v);
    check(nullptr, dmpm_stage_g_op(grid.dim_x, grid.dim_y, grid.dim_z, grid.dx, grid.min_point.data(), m.data(),
                                   p.data(), dt, f, gp, gmag, v.data()),
          "dmpm_stage_g_op");
    for_nodes(grid, [&](GridNode& nd, size_t i) {
        for (int k = 0; k < 3; k++) nd.v[k] = v[3 * i + k];
    });
}
}  // namespace

void G_op(Grid& grid, float dt, Vec3 f_ext) { g_op(grid, dt, f_ext.data(), nullptr, 0.f); }

void G_op(Grid& grid, float dt, Vec3 gravity_point, float gravity_mag) {
    g_op(grid, dt, nullptr, gravity_point.data(), gravity_mag);
}

void G2P(PointCloud& next, const PointCloud& curr, Grid& grid) {
    const size_t n = curr.points.size();
    if (n == 0) return;
    if (next.points.size() != n) next.points = curr.points;
    std::vector<float> x(3 * n), gv(3 * num_nodes(grid)), v(3 * n), C(9 * n);
    for (size_t p = 0; p < n; p++)
        for (int k = 0; k < 3; k++) x[3 * p + k] = curr.points[p].x[k];
    for_nodes(grid, [&](const GridNode& nd, size_t i) {
        for (int k = 0; k < 3; k++) gv[3 * i + k] = nd.v[k];
    });
    check(nullptr, dmpm_stage_g2p((int)n, x.data(), grid.dim_x, grid.dim_y, grid.dim_z, grid.dx,
                                  grid.min_point.data(), gv.data(), v.data(), C.data()),
          "dmpm_stage_g2p");
    for (size_t p = 0; p < n; p++) {
        for (int k = 0; k < 3; k++) next.points[p].v[k] = v[3 * p + k];
        for (int k = 0; k < 9; k++) next.points[p].C.data()[k] = C[9 * p + k];
    }
}

void P_op_2(PointCloud& next, const PointCloud& curr, float dt) { P_op_2(next, curr, 0.f, dt); }

void P_op_2(PointCloud& next, const PointCloud& curr, float s, float dt) {
    const size_t n = next.points.size();
    if (n == 0) return;
    std::vector<float> x(3 * n), F(9 * n), D(9 * n), v(3 * n), C(9 * n), xo(3 * n), Fo(9 * n);
    for (size_t p = 0; p < n; p++) {
        const MaterialPoint& c = curr.points[p];
        const MaterialPoint& q = next.points[p];
        for (int k = 0; k < 3; k++) {
            x[3 * p + k] = c.x[k];
            v[3 * p + k] = q.v[k];
        }
        for (int k = 0; k < 9; k++) {
            F[9 * p + k] = c.F.data()[k];
            D[9 * p + k] = c.dFc.data()[k];
            C[9 * p + k] = q.C.data()[k];
        }
    }
    check(nullptr, dmpm_stage_p_op_2((int)n, x.data(), F.data(), D.data(), v.data(), C.data(), dt, s, xo.data(),
                                     Fo.data()),
          "dmpm_stage_p_op_2");
    for (size_t p = 0; p < n; p++) {
        for (int k = 0; k < 3; k++) next.points[p].x[k] = xo[3 * p + k];
        for (int k = 0; k < 9; k++) next.points[p].F.data()[k] = Fo[9 * p + k];
    }
}

void CalculatePointCloudVolumes(PointCloud& pc, Grid& grid) {
    if (pc.points.empty()) return;
    P2G(pc, grid, 0.f, 0.f);
    Ctx c(g_stage_precision);
    set_grid(c.h, grid);
    check(c.h, dmpm_set_points_ref(c.h, pc.points.data(), (int)pc.points.size()), "dmpm_set_points_ref");
    set_params(c.h, 0.f, 0.f, Vec3::Zero(), 0.f, DMPM_ADJ_REFCOMPAT, 0, 0);  // before: the raster reads the mode
    check(c.h, dmpm_compute_volumes(c.h), "dmpm_compute_volumes");
    check(c.h, dmpm_setup(c.h, 1), "dmpm_setup");
    std::vector<double> vol(pc.points.size());
    check(c.h, dmpm_get_particles(c.h, 0, DMPM_F_VOL, vol.data()), "dmpm_get_particles");
    for (size_t p = 0; p < pc.points.size(); p++) pc.points[p].vol = (float)vol[p];
}

}  // namespace SingleThreadMPM

void MultiThreadMPM::ForwardTimeStep(PointCloud& next, PointCloud& curr, Grid& main_grid,
                                     std::vector<std::shared_ptr<Grid>>& proxy_grids, float dt, float drag,
                                     Vec3 f_ext) {
    (void)proxy_grids;  // per-thread scratch of the CPU version
    SingleThreadMPM::ForwardTimeStep(next, curr, main_grid, 0.f, dt, drag, f_ext);
}

// ====================================================================== Back_Timestep (GPU)
// The engine recomputes layer n's grid from layer n's cloud, which needs the
// external force the forward step used; Back_Timestep's signature does not
// carry it, so it is recovered from the grid the forward step left in
// layer_n (v = p/m + dt f_ext on any node with |m| > FLT_EPSILON).
void Back_Timestep(CompGraphLayer& layer_nplus1, CompGraphLayer& layer_n, float drag, float dt, float s) {
    PointCloud& pc_prev = *layer_n.point_cloud;
    const PointCloud& pc = *layer_nplus1.point_cloud;
    Grid& grid = *layer_n.grid;
    Vec3 f_ext = Vec3::Zero();
    if (dt != 0.f) {
        bool found = false;
        for_nodes(grid, [&](GridNode& nd, size_t) {
            if (!found && std::fabs(nd.m) > std::numeric_limits<float>::epsilon()) {
                for (int k = 0; k < 3; k++) f_ext[k] = (nd.v[k] - nd.p[k] / nd.m) / dt;
                found = true;
            }
        });
    }
    Ctx c(g_stage_precision);
    set_grid(c.h, grid);
    check(c.h, dmpm_set_points_ref(c.h, pc_prev.points.data(), (int)pc_prev.points.size()), "dmpm_set_points_ref");
    std::vector<double> zeros(num_nodes(grid), 0.0);
    check(c.h, dmpm_set_target_mass(c.h, zeros.data()), "dmpm_set_target_mass");
    set_params(c.h, dt, drag, f_ext, s, DMPM_ADJ_REFCOMPAT, 1, 1);
    check(c.h, dmpm_setup(c.h, 2), "dmpm_setup");
    check(c.h, dmpm_forward(c.h, 0), "dmpm_forward");
    put_field(c.h, 1, DMPM_F_DLDX, pc.points);
    put_field(c.h, 1, DMPM_F_DLDV, pc.points);
    put_field(c.h, 1, DMPM_F_DLDF, pc.points);
    put_field(c.h, 1, DMPM_F_DLDC, pc.points);
    check(c.h, dmpm_backward_range(c.h, 1, 0), "dmpm_backward_range");
    for (int f : {DMPM_F_DLDX, DMPM_F_DLDV, DMPM_F_DLDF, DMPM_F_DLDC, DMPM_F_DLDP, DMPM_F_DLDV_NEXT, DMPM_F_DLDC_NEXT})
        get_field(c.h, 0, f, pc_prev.points);
    get_grid_into(c.h, 0, grid, false, true);
}

// ====================================================================== CompGraph
CompGraph::CompGraph(std::shared_ptr<PointCloud> initial_point_cloud, std::shared_ptr<Grid> grid,
                     std::shared_ptr<const Grid> _target_grid) {
    layers.resize(1);
    layers[0].point_cloud = std::make_shared<PointCloud>(*initial_point_cloud);
    layers[0].grid = std::make_shared<Grid>(*grid);
    target_grid = _target_grid;
}

CompGraph::~CompGraph() {
    if (ctx_) dmpm_destroy(ctx_);
}

void CompGraph::SetSimulationParameters(float _dt, float _drag, Vec3 _f_ext, float s) {
    dt = _dt;
    drag = _drag;
    f_ext = _f_ext;
    smoothing_factor = s;
}

void CompGraph::SetEngineOptions(int precision, int adjoint_mode, int device) {
    if (ctx_ && (precision != precision_ || device != device_)) {
        dmpm_destroy(ctx_);
        ctx_ = nullptr;
    }
    precision_ = precision;
    adjoint_mode_ = adjoint_mode;
    device_ = device;
    ctx_layers_ = 0;
}

void CompGraph::SetDeterministic(bool on) {
    deterministic_ = on;
    ctx_layers_ = 0;  // the next pass sets the graph up again with the mode
}

void CompGraph::SetReorderParticles(bool on) {
    reorder_ = on;
    ctx_layers_ = 0;
}

void CompGraph::EnsureEngine() {
    if (!ctx_) check(nullptr, dmpm_create(device_, precision_, &ctx_), "dmpm_create");
}

// CompGraph.cpp:7-17, plus uploading the graph to the engine
void CompGraph::SetUpCompGraph(int num_layers) {
    if (num_layers <= 0) throw std::invalid_argument("SetUpCompGraph: num_layers must be > 0");
    layers.resize(num_layers);
    for (int i = 1; i < num_layers; i++) {
        layers[i].point_cloud = std::make_shared<PointCloud>(*layers.front().point_cloud);
        layers[i].grid = std::make_shared<Grid>(*layers.front().grid);
    }
    EnsureEngine();
    const Grid& g = *layers.front().grid;
    set_grid(ctx_, g);
    auto& pts = layers.front().point_cloud->points;
    check(ctx_, dmpm_set_points_ref(ctx_, pts.data(), (int)pts.size()), "dmpm_set_points_ref");
    std::vector<double> tm(num_nodes(*target_grid));
    for_nodes(*target_grid, [&](const GridNode& n, size_t i) { tm[i] = n.m; });
    check(ctx_, dmpm_set_target_mass(ctx_, tm.data()), "dmpm_set_target_mass");
    set_params(ctx_, dt, drag, f_ext, smoothing_factor, adjoint_mode_, 1, 0, deterministic_ ? 1 : 0,
               reorder_ && precision_ == DMPM_FP32_MIXED ? 1 : 0);
    check(ctx_, dmpm_setup(ctx_, num_layers), "dmpm_setup");
    ctx_layers_ = num_layers;
}

void CompGraph::PushLayer0AndControls(size_t start) {
    if (!ctx_ || ctx_layers_ != (int)layers.size()) SetUpCompGraph((int)layers.size());
    const auto& ps = layers[start].point_cloud->points;
    for (int f : {DMPM_F_X, DMPM_F_V, DMPM_F_F, DMPM_F_C}) put_field(ctx_, (int)start, f, ps);
    for (size_t l = start; l < layers.size(); l++) put_field(ctx_, (int)l, DMPM_F_DFC, layers[l].point_cloud->points);
}

void CompGraph::PullStates(size_t first, size_t last) {
    for (size_t l = first; l <= last && l < layers.size(); l++) {
        auto& pts = layers[l].point_cloud->points;
        check(ctx_, dmpm_get_points_ref(ctx_, (int)l, pts.data()), "dmpm_get_points_ref");
    }
}

void CompGraph::PullGrid(size_t l) { get_grid_into(ctx_, (int)l, *layers[l].grid, true, false); }

void CompGraph::PullAdjoints(size_t first, size_t last) {
    for (size_t l = first; l <= last && l < layers.size(); l++)
        for (int f : {DMPM_F_DLDX, DMPM_F_DLDV, DMPM_F_DLDF, DMPM_F_DLDC})
            get_field(ctx_, (int)l, f, layers[l].point_cloud->points);
}

// CompGraph.cpp:246-256
void CompGraph::ComputeForwardPass(size_t start_layer) {
    if (layers.size() < 2) return;
    PushLayer0AndControls(start_layer);
    check(ctx_, dmpm_forward(ctx_, (int)start_layer), "dmpm_forward");
    PullStates(start_layer + 1, layers.size() - 1);
    if (sync_grids)
        for (size_t l = start_layer; l + 1 < layers.size(); l++) {
            get_field(ctx_, (int)l, DMPM_F_P, layers[l].point_cloud->points);
            PullGrid(l);
        }
}

// CompGraph.cpp:110-244
float CompGraph::EndLayerMassLoss() {
    if (!ctx_ || ctx_layers_ != (int)layers.size()) SetUpCompGraph((int)layers.size());
    if (layers.size() == 1) {
        PushLayer0AndControls(0);
        check(ctx_, dmpm_forward(ctx_, 0), "dmpm_forward");
    }
    double L = 0.0;
    check(ctx_, dmpm_loss(ctx_, &L), "dmpm_loss");
    const size_t last = layers.size() - 1;
    auto& pts = layers[last].point_cloud->points;
    get_field(ctx_, (int)last, DMPM_F_DLDX, pts);
    for (auto& p : pts) {
        p.dLdF.setZero();
        p.dLdv.setZero();
        p.dLdC.setZero();
    }
    if (sync_grids) {
        Grid& g = *layers[last].grid;
        const size_t G = num_nodes(g);
        std::vector<double> a(G);
        check(ctx_, dmpm_get_grid(ctx_, (int)last, DMPM_G_M, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { n.m = (float)a[i]; n.v.setZero(); });
        check(ctx_, dmpm_get_grid(ctx_, (int)last, DMPM_G_DLDM, a.data()), "dmpm_get_grid");
        for_nodes(g, [&](GridNode& n, size_t i) { n.dLdm = (float)a[i]; });
    }
    return (float)L;
}

// CompGraph.cpp:258-267
void CompGraph::ComputeBackwardPass(size_t control_layer) {
    if (layers.size() < 2) return;
    for (size_t l = control_layer; l + 1 < layers.size(); l++) {
        layers[l].grid->ResetGradients();
        layers[l].point_cloud->ResetGradients();
    }
    check(ctx_, dmpm_backward(ctx_, (int)control_layer), "dmpm_backward");
    PullAdjoints(control_layer, layers.size() - 2);
}

// CompGraph.cpp:457-504 (including its delta = 1e-9f and its perturbation of F)
void CompGraph::FiniteDifferencesGradientTest(int num_steps, size_t particle_id) {
    std::streamsize prev = std::cout.precision(6);
    std::cout << "FINITE DIFFERENCES TEST: dLdF" << std::endl;
    SetUpCompGraph(num_steps);
    ComputeForwardPass(0);
    float initial_loss = EndLayerMassLoss();
    std::cout << "initial loss = " << initial_loss << std::endl;
    ComputeBackwardPass(0);
    MaterialPoint& mp = layers.front().point_cloud->points[particle_id];
    const Mat3 analytic = mp.dLdF;
    Mat3 fd;
    const float delta = 1e-9f;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const float orig = mp.F(i, j);
            mp.F(i, j) = orig + delta;
            ComputeForwardPass(0);
            const float l1 = EndLayerMassLoss();
            mp.F(i, j) = orig - delta;
            ComputeForwardPass(0);
            const float l2 = EndLayerMassLoss();
            fd(i, j) = (l1 - l2) / (2.f * delta);
            mp.F(i, j) = orig;
        }
    const float diff = (fd - analytic).norm();
    std::cout << "gradient difference = " << diff << std::endl;
    std::cout << "gradient difference percentage = " << 100.f * diff / fd.norm() << std::endl;
    std::cout.precision(prev);
}

// CompGraph.cpp:280-454: the reference's control-sequence optimisation loop
// (line-searched Adam + Lion steps on one control layer at a time).
void CompGraph::OptimizeDefGradControlSequence(int num_steps, float _dt, float _drag, Vec3 _f_ext,
                                               int control_stride, int max_gd_iters, int max_line_search_iters,
                                               float initial_alpha, float gd_tol, float _smoothing_factor) {
    dt = _dt;
    drag = _drag;
    f_ext = _f_ext;
    smoothing_factor = _smoothing_factor;
    SetUpCompGraph(num_steps);
    ComputeForwardPass(0);
    const float initial_loss = EndLayerMassLoss();
    std::cout << "initial loss = " << initial_loss << std::endl;
    ComputeBackwardPass(0);
    const float initial_norm = layers.front().point_cloud->Compute_dLdF_Norm();
    std::cout << "initial norm = " << initial_norm << std::endl;
    const float beta1 = 0.9f, beta2 = 0.999f, epsilon = 1e-5f;
    const int total_temporal_iterations = 5;
    float gradient_norm = 0.f;
    for (int temporal = 0; temporal < total_temporal_iterations; temporal++) {
        for (int cf = 0; cf < (int)layers.size() - 1; cf += std::max(1, control_stride)) {
            float alpha = initial_alpha;
            for (int gd = 0; gd < max_gd_iters; gd++) {
                ComputeForwardPass(cf);
                const float gd_loss = EndLayerMassLoss();
                ComputeBackwardPass(cf);
                gradient_norm = layers.front().point_cloud->Compute_dLdF_Norm();
                gradientNormHistory.push_back(gradient_norm);
                if (gradient_norm < gd_tol * initial_norm) break;
                bool decrease = false;
                for (int ls = 0; ls < max_line_search_iters; ls++) {
                    PointCloud& pc = *layers[cf].point_cloud;
                    pc.Descend_Adam(alpha, gradient_norm, beta1, beta2, epsilon, timestep);
                    pc.Descend_Lion(alpha, beta1, gradient_norm);
                    ComputeForwardPass(cf);
                    const float ls_loss = EndLayerMassLoss();
                    if (ls_loss < gd_loss) {
                        decrease = true;
                        break;
                    }
                    pc.Descend_Adam(-alpha, gradient_norm, beta1, beta2, epsilon, timestep);
                    pc.Descend_Lion(-alpha, beta1, gradient_norm);
                    alpha /= 2.f;
                }
                if (!decrease) break;
                timestep += 1;
            }
        }
    }
    const float final_loss = EndLayerMassLoss();
    std::cout << "Initial loss = " << initial_loss << std::endl;
    std::cout << "Final loss = " << final_loss << std::endl;
    std::ofstream ofs("gradient_norm_log.csv");
    for (size_t i = 0; i < gradientNormHistory.size(); i++) ofs << i << "," << gradientNormHistory[i] << "\n";
}

// ---- GeometryLoading (GeometryLoading.cpp:10-83) ----

std::vector<Vec3> GeometryLoading::GeneratePointCloudFromTriangleArrays(const float* V, int nv, const int* F, int nf,
                                                                        Vec3 min_point, Vec3 max_point,
                                                                        float sampling_dx) {
    int dims[3];
    check(nullptr, dmpm_mesh_lattice_dims(min_point.data(), max_point.data(), sampling_dx, dims),
          "dmpm_mesh_lattice_dims");
    const int64_t cap = (int64_t)dims[0] * dims[1] * dims[2];
    std::vector<float> buf((size_t)cap * 3);
    int64_t n = 0;
    check(nullptr, dmpm_mesh_lattice_points(V, nv, F, nf, min_point.data(), max_point.data(), sampling_dx,
                                            buf.data(), cap, &n),
          "dmpm_mesh_lattice_points");
    std::vector<Vec3> pts((size_t)n);
    for (int64_t i = 0; i < n; i++) pts[(size_t)i] = Vec3(buf[3 * i], buf[3 * i + 1], buf[3 * i + 2]);
    return pts;
}

// ---- headless surfacing (ForwardSimulation.cpp:292-367, SphereUnionSurfacing.cpp:7-128) ----

namespace {
std::vector<float> grid_masses(const Grid& g) {
    std::vector<float> m((size_t)g.dim_x * g.dim_y * g.dim_z);
    size_t q = 0;
    for (int i = 0; i < g.dim_x; i++)
        for (int j = 0; j < g.dim_y; j++)
            for (int k = 0; k < g.dim_z; k++) m[q++] = g.nodes[i][j][k].m;
    return m;
}
void set_grid_masses(Grid& g, const std::vector<float>& m) {
    size_t q = 0;
    for (int i = 0; i < g.dim_x; i++)
        for (int j = 0; j < g.dim_y; j++)
            for (int k = 0; k < g.dim_z; k++) g.nodes[i][j][k].m = m[q++];
}
}  // namespace

void SingleThreadMPM::P2G_Mass(const std::vector<Vec3> points, Grid& grid, float mp_m) {
    std::vector<float> flat(points.size() * 3);
    for (size_t i = 0; i < points.size(); i++)
        for (int c = 0; c < 3; c++) flat[3 * i + c] = points[i][c];
    const int dims[3] = {grid.dim_x, grid.dim_y, grid.dim_z};
    std::vector<float> m((size_t)grid.dim_x * grid.dim_y * grid.dim_z);
    check(nullptr, dmpm_surface_p2g_mass(flat.data(), (int64_t)points.size(), mp_m, dims, grid.dx,
                                         grid.min_point.data(), m.data()),
          "dmpm_surface_p2g_mass");
    set_grid_masses(grid, m);
}

void SingleThreadMPM::G2G_Mass(Grid& grid_1, Grid& grid_2) {
    const std::vector<float> m1 = grid_masses(grid_1);
    const int d1[3] = {grid_1.dim_x, grid_1.dim_y, grid_1.dim_z}, d2[3] = {grid_2.dim_x, grid_2.dim_y, grid_2.dim_z};
    std::vector<float> m2((size_t)grid_2.dim_x * grid_2.dim_y * grid_2.dim_z);
    check(nullptr, dmpm_surface_g2g_mass(m1.data(), d1, grid_1.dx, grid_1.min_point.data(), d2, grid_2.dx,
                                         grid_2.min_point.data(), m2.data()),
          "dmpm_surface_g2g_mass");
    set_grid_masses(grid_2, m2);
}

void SphereUnionSurfaceArrays(const std::vector<Vec3>& points, float radius, float grid_dx, float iso_mass,
                              int blur_iterations, Vec3 grid_min_point, Vec3 grid_max_point, std::vector<float>& V,
                              std::vector<int>& F) {
    int dims[3];
    check(nullptr, dmpm_surface_grid_dims(grid_min_point.data(), grid_max_point.data(), grid_dx, dims),
          "dmpm_surface_grid_dims");
    std::vector<float> flat(points.size() * 3);
    for (size_t i = 0; i < points.size(); i++)
        for (int c = 0; c < 3; c++) flat[3 * i + c] = points[i][c];
    std::vector<float> field((size_t)dims[0] * dims[1] * dims[2]);
    check(nullptr, dmpm_surface_sphere_field(flat.data(), (int64_t)points.size(), radius, blur_iterations, dims,
                                             grid_dx, grid_min_point.data(), field.data()),
          "dmpm_surface_sphere_field");
    int64_t nv = 0, nf = 0;
    const int st = dmpm_surface_extract(field.data(), dims, grid_dx, grid_min_point.data(), iso_mass, nullptr, 0,
                                        nullptr, 0, &nv, &nf);
    if (st != DMPM_OK && st != DMPM_ERR_TOO_LARGE) check(nullptr, st, "dmpm_surface_extract");
    V.assign((size_t)nv * 3, 0.f);
    F.assign((size_t)nf * 3, 0);
    check(nullptr, dmpm_surface_extract(field.data(), dims, grid_dx, grid_min_point.data(), iso_mass, V.data(), nv,
                                        F.data(), nf, &nv, &nf),
          "dmpm_surface_extract");
}

}  // namespace DiffMPMLib3D
