#!/bin/bash
# Builds make_opt_input.cpp against the reference's vendored cereal and Eigen
# (where they lie under the reference tree given as $1) and writes the golden
# OptInput JSON files next to this script; with a JSON file as $2, instead
# reads it with cereal and writes what cereal writes back to $3.
set -e
REF=${1:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
BIN=${TMPDIR:-/tmp}/make_opt_input_$$
g++ -std=c++17 -O1 -I "$REF/include" -I "$REF/DiffMPMLib3D" -o "$BIN" "$HERE/make_opt_input.cpp"
if [ -n "$2" ]; then "$BIN" "$2" roundtrip "$3"; else "$BIN" "$HERE"; fi
rm -f "$BIN"
