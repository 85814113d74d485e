// MaterialPoint.h -- the reference's particle record (MaterialPoint.h:8-75):
// same fields, order and defaults, 118 floats = 472 bytes, so arrays of it can
// be handed to dmpm_set_points_ref / dmpm_get_points_ref unchanged.
#pragma once
#include "pch.h"

namespace DiffMPMLib3D {

struct MaterialPoint {
    void ResetGradients();

    Vec3 x = Vec3::Zero();
    Vec3 v = Vec3::Zero();
    Mat3 F = Mat3::Identity();
    Mat3 C = Mat3::Zero();
    Mat3 P = Mat3::Zero();

    float m = 0.f;
    float vol = 0.f;

    float lam = 0.f;
    float mu = 0.f;

    Mat3 dFc = Mat3::Zero();  // control: added to F at every step

    Vec3 dLdx = Vec3::Zero();
    Vec3 dLdv = Vec3::Zero();
    Mat3 dLdF = Mat3::Zero();
    Mat3 dLdC = Mat3::Zero();
    Mat3 dLdP = Mat3::Zero();

    Vec3 dLdv_next = Vec3::Zero();
    Mat3 dLdC_next = Mat3::Zero();

    Mat3 momentum = Mat3::Zero();
    Mat3 vector = Mat3::Zero();
    Mat3 vector_max = Mat3::Zero();
};

static_assert(sizeof(MaterialPoint) == 472, "reference MaterialPoint layout");

}  // namespace DiffMPMLib3D
