#!/bin/sh
# Builds oracle/_ref/libref_kat.so from the reference's own sources where they
# lie (read-only), for the known-answer tests of the oracle.  Needs the
# reference checkout; the built library travels with the repository snapshot.
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
