#!/usr/bin/env bash
# Builds the checkers under oracle/ (test infrastructure, never the product):
#   oracle/liblbm_oracle.so      the C restatement (lbm_oracle.c), always;
#   oracle/_ref/libref_cpu.so    the reference's own stl_loader.cpp + voxelize.cpp
#                                + band BFS (sim_runner.hpp), with a GLM shim;
#   oracle/_ref/libref_cuda.so   the reference's own CUDA solvers for sm_100a.
# The _ref libraries are built only where the reference sources exist
# (REF_ROOT, default /root/reference); elsewhere the prebuilt files are used.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_ROOT="${REF_ROOT:-/root/reference}"
NVCC="${NVCC:-nvcc}"
CUDA_INC="$(dirname "$(command -v "$NVCC")")/../include"

# The oracle: -ffp-contract=off keeps float operations uncontracted (the
# reference's geometry is compiled by a default x86-64 g++, which has no FMA).
gcc -O2 -fPIC -shared -std=c11 -ffp-contract=off -fopenmp -Wall -Wno-unused-function \
    -o "$HERE/liblbm_oracle.so" "$HERE/lbm_oracle.c" -lm

if [ ! -d "$REF_ROOT/src" ]; then
    echo "[build_ref] reference sources not present; keeping prebuilt oracle/_ref" >&2
    exit 0
fi
mkdir -p "$HERE/_ref"
SRC="$REF_ROOT/src"

g++ -O2 -fPIC -shared -std=c++17 -ffp-contract=off -w \
    -I"$HERE/ref_shim" -I"$SRC" -I"$CUDA_INC" \
    -o "$HERE/_ref/libref_cpu.so" \
    "$SRC/geom/stl_loader.cpp" "$SRC/geom/voxelize.cpp" "$HERE/ref_cpu_driver.cpp"

"$NVCC" -O3 -std=c++17 -shared -Xcompiler -fPIC -w \
    -gencode arch=compute_100a,code=sm_100a \
    -I"$SRC" -o "$HERE/_ref/libref_cuda.so" \
    "$SRC/lbm/lbm3d_legacy.cu" "$SRC/lbm/lbm3d_home.cu" "$SRC/lbm/lbm3d_hybrid.cu" \
    "$SRC/lbm/lbm_reinit.cu" "$SRC/fields/field_ops.cu" "$SRC/fields/init_profiles.cu" \
    "$SRC/moment_vtk_writer.cu" "$HERE/ref_cuda_driver.cu"
echo "[build_ref] ok"
