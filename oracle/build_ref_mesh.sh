#!/bin/bash
# Builds the reference's mesh sampler (GeometryLoading.cpp, compiled where it
# lies, with the reference's vendored libigl and Eigen) and the driver
# oracle/ref_mesh_driver.cpp into oracle/_ref/ref_mesh.  $1: reference tree.
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
mkdir -p "$HERE/_ref"
g++ -std=c++17 -O2 -fpermissive -w -I "$REF/include" -I "$REF/DiffMPMLib3D" -I /usr/local/cuda/include \
    -o "$HERE/_ref/ref_mesh.tmp" "$REF/DiffMPMLib3D/GeometryLoading.cpp" "$HERE/ref_mesh_driver.cpp"
mv "$HERE/_ref/ref_mesh.tmp" "$HERE/_ref/ref_mesh"
echo "built $HERE/_ref/ref_mesh"
