// PointCloud.h -- the reference's particle container (PointCloud.h:8-66) with
// its gradient utilities, optimiser steps (PointCloud.cpp:16-204) and the
// .mpmbin binary archive (PointCloud.cpp:334-362: a cereal binary archive of
// the vector of points; each MaterialPoint serialises x, v, F, C, P, m, vol,
// lam, mu, dFc, dLdx, dLdv, dLdF, momentum, vector, vector_max in that order,
// vectors as <int32 rows><rows floats>, matrices as <int32 rows><int32 cols>
// followed by the coefficients in row order).
#pragma once
#include <string>
#include <vector>
#include "MaterialPoint.h"

namespace DiffMPMLib3D {

struct PointCloud {
    void ResetGradients();
    float Compute_dLdF_Norm();
    void Descend_dLdF(float alpha, float gradient_norm);
    void Descend_Adam(float alpha, float gradient_norm, float beta1, float beta2, float epsilon, int timestep);
    void Descend_AMSGrad(float alpha, float gradient_norm, float beta1, float beta2, float epsilon, int timestep);
    void Descend_GradientDescent(float alpha, float gradient_norm);
    void Descend_Lion(float alpha, float beta, float gradient_norm);

    // Minibatch variants (PointCloud.cpp:37-82): a random subset of
    // minibatch_size distinct indices (shuffled with a clock-seeded mt19937, as
    // the reference does), the gradient norm over those points, and an Adam
    // step on them only, whose bias correction uses timestep + 1.
    std::vector<int> generateMinibatchIndices(int total_size, int minibatch_size);
    float Compute_dLdF_Norm_Stochastic(const std::vector<int>& minibatch_indices);
    void Descend_Adam_Stochastic(float alpha, float gradient_norm, float beta1, float beta2, float epsilon,
                                 int timestep, const std::vector<int>& minibatch_indices);

    bool ReadFromOBJ(std::string obj_path, float point_mass);
    void WriteToOBJ(std::string obj_path);
    void WriteEntirePointCloudToBinaryFile(std::string file_path);
    bool ReadEntirePointCloudFromBinaryFile(std::string file_path);
    bool IsEqualToOtherPointCloud(const PointCloud& other_pc);

    std::vector<Vec3> GetPointPositions() const;
    std::vector<float> GetPointMasses() const;
    std::vector<float> GetPointVolumes() const;
    std::vector<Mat3> GetPointDefGrads() const;
    std::vector<float> GetPointDeterminants() const;

    std::vector<MaterialPoint> points;
};

}  // namespace DiffMPMLib3D
