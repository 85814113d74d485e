// GridNode.h -- the reference's grid node (GridNode.h:5-24), 80 bytes.
#pragma once
#include "pch.h"

namespace DiffMPMLib3D {

struct GridNode {
    void ResetGradients();

    Vec3 x = Vec3::Zero();
    Vec3 v = Vec3::Zero();
    Vec3 p = Vec3::Zero();
    float m = 0.f;

    Vec3 dLdx = Vec3::Zero();
    Vec3 dLdv = Vec3::Zero();
    Vec3 dLdp = Vec3::Zero();
    float dLdm = 0.f;
};

static_assert(sizeof(GridNode) == 80, "reference GridNode layout");

}  // namespace DiffMPMLib3D
