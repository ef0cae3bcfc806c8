#!/bin/sh
# Builds the comparator: the reference's own GPU step (iwf_mfree_gpu_3d,
# leap_frog::step, src/leap_frog.cu:121-195) for sm_100a, linked with the
# scene driver ref_step_main.cu, into baseline/_ref/ref_step_<variant>.
#
# The reference is a CUDA 8 program and does not build with CUDA 12 as it is.
# The patch is the smallest one that keeps its behaviour, and it is applied to
# a temporary copy outside the repository (the reference stays read-only and
# its sources never enter the repository):
#   * texture references (removed in CUDA 12), src/interactions_gpu.cu:41-57:
#     each `texture<T, 1, mode> name;` becomes `__device__ ref_texture<T, 1,
#     mode> name;`; ref_compat.h (forced include) gives tex1Dfetch /
#     cudaBindTexture / cudaUnbindTexture their old meaning with __ldg loads;
#   * GLM (not installed, not vendored): oracle/ref_include/glm/glm.hpp, a
#     project-written GLM-compatible header;
#   * the compile-time physics switches of src/types.h:100-105, per variant:
#       brookshaw  Brookshaw conduction, no CSPM (the reference's default)
#       cspm_pse   CSPM on, PSE conduction instead of Brookshaw
#   * flags: the reference's Release flags (-O3, relocatable device code, no
#     NDEBUG, Release/src/subdir.mk:84-85) with -gencode for sm_100a.
# Usage: baseline/build_ref_gpu.sh [reference_root] [variant ...]
#        (reference_root: $MFREE_REFERENCE_ROOT, else ../reference beside the
#        repository)
set -e
here=$(cd "$(dirname "$0")" && pwd)
root=$(dirname "$here")
ref=${1:-${MFREE_REFERENCE_ROOT:-$(dirname "$root")/reference}}
[ $# -gt 0 ] && shift
variants=${*:-"brookshaw cspm_pse"}
[ -n "$ref" ] && [ -f "$ref/src/leap_frog.cu" ] || { echo "reference sources not found (argument or MFREE_REFERENCE_ROOT)" >&2; exit 1; }
cuda=${CUDA_HOME:-/usr/local/cuda}
nvcc="$cuda/bin/nvcc"
out="$here/_ref"
mkdir -p "$out"
tmp=$(mktemp -d /tmp/mfree_refgpu.XXXXXX)
trap 'rm -rf "$tmp"' EXIT

# the translation units of the step (the CLI main, the scene setups, VTK I/O and
# the unused "rothlin" grid are left out)
units="actions_gpu.cu eigen_solver.cu grid_gpu_base.cu grid_gpu_green.cu interactions_gpu.cu leap_frog.cu
particle_gpu.cu tool_3d_gpu.cu blanking.cpp constants_structs.cpp geometry_utils.cpp grid_cpu_tri.cpp
json_reader.cpp ldynak_reader.cpp surface_tri_mesh.cpp tool_3d.cpp types.cpp"

for v in $variants; do
    src="$tmp/$v/src"
    obj="$tmp/$v/obj"
    mkdir -p "$src" "$obj"
    cp "$ref"/src/*.h "$ref"/src/*.cuh "$src"/
    for u in $units; do cp "$ref/src/$u" "$src/"; done
    sed -i 's/^texture<\(.*\)> *\([A-Za-z_][A-Za-z_0-9]*\);/__device__ ref_texture<\1> \2;/' "$src/interactions_gpu.cu"
    case $v in
        brookshaw) ;;
        cspm_pse)
            sed -i -e 's|^//#define CSPM|#define CSPM|' \
                   -e 's|^#define Thermal_Conduction_Brookshaw|//#define Thermal_Conduction_Brookshaw|' \
                   -e 's|^//#define Thermal_Conduction_PSE|#define Thermal_Conduction_PSE|' "$src/types.h" ;;
        *) echo "unknown variant $v" >&2; exit 1 ;;
    esac
    flags="-O3 -std=c++17 -rdc=true -gencode arch=compute_100a,code=sm_100a -w -include $here/ref_compat.h -I$root/oracle/ref_include -I$src"
    # (ref_compat.h includes oracle/ref_include/ref_prelude.h)
    for u in $units; do echo "$src/$u"; done > "$tmp/$v/list"
    echo "$here/ref_step_main.cu" >> "$tmp/$v/list"
    # every unit is compiled (in parallel) before a failure is reported
    if ! xargs -P 8 -I{} sh -c "$nvcc $flags -x cu -c {} -o $obj/\$(basename {}).o" < "$tmp/$v/list"; then
        echo "compile failed ($v)" >&2
        exit 1
    fi
    $nvcc -O3 -rdc=true -gencode arch=compute_100a,code=sm_100a -o "$out/ref_step_$v" "$obj"/*.o
    echo "built $out/ref_step_$v"
done
