#!/usr/bin/env bash
# Builds the reference's own CPU implementation of the hot path (DiffMPMLib3D,
# unmodified sources) into oracle/_ref/ for use as a test checker and as the
# timed CPU baseline.  Test infrastructure only: nothing in the product links it.
#
#   oracle/_ref/libref_fp32.so  unmodified sources, serial (no -fopenmp: the
#                               OpenMP build races and GCC rejects three of its
#                               collapse clauses), g++ -O2, FP32 as shipped.
#   oracle/_ref/libref_fp64.so  the same sources mechanically retyped to FP64 in
#                               a temporary directory (float -> double, Eigen
#                               ...f -> ...d, f-suffix literals stripped, and the
#                               FLT_EPSILON thresholds kept as the FP32 constant).
#
# Both libraries add oracle/ref_driver.cpp (this repository's code), which
# drives CompGraph / SingleThreadMPM / MultiThreadMPM / Back_Timestep through
# their public C++ API and exports a flat C ABI for ctypes.
#
# Usage: oracle/build_ref.sh [REFERENCE_ROOT]   (default /root/reference)
set -euo pipefail
REF="${1:-/root/reference}"
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
OUT="$HERE/_ref"
SRC="$REF/DiffMPMLib3D"
if [ ! -d "$SRC" ]; then
  echo "build_ref.sh: reference sources not found at $SRC" >&2
  exit 2
fi
mkdir -p "$OUT"
UNITS="BackPropagation CompGraph Elasticity ForwardSimulation Grid GridNode MaterialPoint MultiThreadForwardSimulation PointCloud Tensor3x3x3x3"
CXXFLAGS="-std=c++17 -O2 -fPIC -fpermissive -w -pthread"
INC_COMMON="-I$REF/include -I/usr/local/cuda/include"

build_one() {  # $1 = source dir, $2 = REAL type, $3 = output .so, $4 = object dir
  local sdir="$1" real="$2" so="$3" odir="$4"
  mkdir -p "$odir"
  local pids=()
  for u in $UNITS; do
    g++ $CXXFLAGS $INC_COMMON -I"$sdir" -c "$sdir/$u.cpp" -o "$odir/$u.o" &
    pids+=($!)
  done
  g++ $CXXFLAGS $INC_COMMON -I"$sdir" -DREF_REAL="$real" -c "$HERE/ref_driver.cpp" -o "$odir/ref_driver.o" &
  pids+=($!)
  local rc=0
  for p in "${pids[@]}"; do wait "$p" || rc=1; done
  if [ "$rc" != 0 ]; then echo "build_ref.sh: compile failed for $so" >&2; return 1; fi
  g++ -shared -pthread -o "$so" "$odir"/*.o -lgomp
}

TMP="$(mktemp -d /tmp/dmpm_ref_build.XXXXXX)"
trap 'rm -rf "$TMP"' EXIT

# FP32: the sources exactly as shipped.
build_one "$SRC" float "$OUT/libref_fp32.so" "$TMP/obj32"

# FP64: retyped copy (only in the temporary directory, never in the repository).
mkdir -p "$TMP/src64"
cp "$SRC"/*.h "$SRC"/*.cuh "$SRC"/*.cpp "$TMP/src64/"
for f in "$TMP/src64"/*.h "$TMP/src64"/*.cuh "$TMP/src64"/*.cpp; do
  sed -E -i \
    -e 's/std::numeric_limits<float>::epsilon\(\)/1.1920928955078125e-07/g' \
    -e 's/\bfloat\b/double/g' \
    -e 's/\b(Vector3|Matrix3|MatrixX|VectorX)f\b/\1d/g' \
    -e 's/\b([0-9]+\.[0-9]*([eE][-+]?[0-9]+)?)f\b/\1/g' \
    -e 's/(^|[^0-9A-Za-z_.])(\.[0-9]+([eE][-+]?[0-9]+)?)f\b/\1\2/g' \
    -e 's/\b([0-9]+[eE][-+]?[0-9]+)f\b/\1/g' \
    "$f"
done
build_one "$TMP/src64" double "$OUT/libref_fp64.so" "$TMP/obj64"
echo "built $OUT/libref_fp32.so $OUT/libref_fp64.so"
