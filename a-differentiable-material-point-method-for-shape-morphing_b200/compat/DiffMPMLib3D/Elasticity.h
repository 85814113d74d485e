// Elasticity.h -- the reference's fixed-corotated elasticity functions
// (Elasticity.h:6-23), evaluated on the GPU in FP64 (dmpm_elementary).
#pragma once
#include <array>
#include "pch.h"

namespace DiffMPMLib3D {

typedef std::array<std::array<Mat3, 3>, 3> Tensor3x3x3x3;  // Tensor3x3x3x3.h:5

float FixedCorotatedElasticity(const Mat3& F, float lam, float mu);
Mat3 PK_FixedCorotatedElasticity(const Mat3& F, float lam, float mu);
Mat3 d2_FCE_psi_dF2_mult_by_dF(const Mat3& F, float lam, float mu, const Mat3& dF);
Tensor3x3x3x3 d2_FCE_psi_dF2_mult_trick(const Mat3& F, float lam, float mu);
Tensor3x3x3x3 d2_FCE_psi_dF2_FD(const Mat3& F, float lam, float mu);
void CalculateLameParameters(float young_mod, float poisson, float& lam, float& mu);

// d(J F^-T)/dF as T[a][b](i, j) = d(J F^-T)_ab / dF_ij: by central differences with
// delta = 1e-6 (d_JFit_dF_FD, Elasticity.cpp:7-72) and in closed form from J and
// F^-T (d_JFit_dF, declared at Elasticity.h:20; the reference defines no body).  Small
// host utilities off the hot path, evaluated in FP64 and rounded to float.
Tensor3x3x3x3 d_JFit_dF_FD(const Mat3& F);
Tensor3x3x3x3 d_JFit_dF(float J, const Mat3& Fit);

// Batched forms: one GPU launch for many matrices (n = size of the vectors).
std::vector<Mat3> PK_FixedCorotatedElasticityBatch(const std::vector<Mat3>& F, float lam, float mu);
std::vector<Mat3> d2_FCE_psi_dF2_mult_by_dF_Batch(const std::vector<Mat3>& F, float lam, float mu,
                                                  const std::vector<Mat3>& dF, bool exact = false);

}  // namespace DiffMPMLib3D
