#!/bin/sh
# Builds, from the reference's own sources where they lie (read-only), for the
# known-answer tests of the oracle (the built libraries travel with the
# repository snapshot; the reference checkout is needed only here):
#   oracle/_ref/libref_kat.so   kernel, eigen-solver and Johnson-Cook functions
#                               (ref_kat_shim.cpp; g++, __device__ defined empty)
#   oracle/_ref/libref_host.so  the scene setup: mesh readers, vertex normals,
#                               triangle grid, tool construction (ref_host_shim.cpp;
#                               host code compiled by nvcc, which the reference's
#                               headers need for Thrust, linked with the CUDA runtime
#                               its mesh upload calls, never called here)
# Usage: oracle/build_ref.sh [reference_root]
#        (default: $MFREE_REFERENCE_ROOT, else ../reference beside the repository)
set -e
here=$(cd "$(dirname "$0")" && pwd)
ref=${1:-${MFREE_REFERENCE_ROOT:-$(dirname "$(dirname "$here")")/reference}}
cuda=${CUDA_HOME:-/usr/local/cuda}
[ -f "$ref/src/kernels.cuh" ] || { echo "reference sources not found under $ref" >&2; exit 1; }
mkdir -p "$here/_ref"
g++ -std=c++14 -O2 -fPIC -shared -w \
    -D__device__= -D__host__= \
    -I"$here/ref_include" -I"$ref/src" -I"$cuda/include" \
    "$here/ref_kat_shim.cpp" -o "$here/_ref/libref_kat.so"
echo "built $here/_ref/libref_kat.so"
nvcc=${cuda}/bin/nvcc
$nvcc -std=c++17 -O2 -Xcompiler -fPIC -shared -w -x cu -gencode arch=compute_100a,code=sm_100a \
    -include "$here/ref_include/ref_prelude.h" -I"$here/ref_include" -I"$ref/src" \
    "$here/ref_host_shim.cpp" "$ref/src/json_reader.cpp" "$ref/src/ldynak_reader.cpp" \
    "$ref/src/surface_tri_mesh.cpp" "$ref/src/grid_cpu_tri.cpp" "$ref/src/tool_3d.cpp" \
    "$ref/src/geometry_utils.cpp" "$ref/src/types.cpp" \
    -Xlinker --no-undefined -o "$here/_ref/libref_host.so"
echo "built $here/_ref/libref_host.so"
