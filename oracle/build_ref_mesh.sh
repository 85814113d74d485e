#!/bin/bash
# Builds the reference's mesh sampler (GeometryLoading.cpp, compiled where it
# lies, with the reference's vendored libigl and Eigen) and the driver
# oracle/ref_mesh_driver.cpp into oracle/_ref/ref_mesh, and its headless
# surfacing code (SphereUnionSurfacing.cpp, SingleThreadMPM::P2G_Mass /
# G2G_Mass of ForwardSimulation.cpp, Grid.cpp, with their dependencies) and
# oracle/ref_surface_driver.cpp into oracle/_ref/ref_surface.  Serial builds
# (no -fopenmp), as for the hot path.  $1: reference tree.
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_ref"
g++ -std=c++17 -O2 -fpermissive -w -I "$REF/include" -I "$REF/DiffMPMLib3D" -I /usr/local/cuda/include \
    -o "$HERE/_ref/ref_mesh.tmp" "$REF/DiffMPMLib3D/GeometryLoading.cpp" "$HERE/ref_mesh_driver.cpp"
mv "$HERE/_ref/ref_mesh.tmp" "$HERE/_ref/ref_mesh"
echo "built $HERE/_ref/ref_mesh"
S="$REF/DiffMPMLib3D"
g++ -std=c++17 -O2 -fpermissive -w -I "$REF/include" -I "$S" -I /usr/local/cuda/include \
    -o "$HERE/_ref/ref_surface.tmp" "$S/SphereUnionSurfacing.cpp" "$S/ForwardSimulation.cpp" "$S/Grid.cpp" \
    "$S/GridNode.cpp" "$S/MaterialPoint.cpp" "$S/Elasticity.cpp" "$S/Tensor3x3x3x3.cpp" "$S/PointCloud.cpp" \
    "$HERE/ref_surface_driver.cpp"
mv "$HERE/_ref/ref_surface.tmp" "$HERE/_ref/ref_surface"
echo "built $HERE/_ref/ref_surface"
