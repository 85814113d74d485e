// BackPropagation.h -- the reference's adjoint time step (BackPropagation.h:7),
// run on the GPU: fills layer_n's adjoint fields (dLdx, dLdv, dLdF, dLdC,
// dLdP) and layer_n's grid adjoints from layer_nplus1's adjoint.
#pragma once
#include "CompGraph.h"

namespace DiffMPMLib3D {

void Back_Timestep(CompGraphLayer& layer_nplus1, CompGraphLayer& layer_n, float drag, float dt, float smoothing_factor);

}  // namespace DiffMPMLib3D
