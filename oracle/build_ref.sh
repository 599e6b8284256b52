#!/usr/bin/env bash
# Builds the checkers under oracle/ (test infrastructure, never the product):
#   oracle/liblbm_oracle.so      the C restatement (lbm_oracle.c), always;
#   oracle/_ref/libref_cpu.so    the reference's own stl_loader.cpp + voxelize.cpp
#                                + band BFS (sim_runner.hpp), with a GLM shim;
#   oracle/_ref/libref_cuda.so   the reference's own CUDA solvers for sm_100a;
#   oracle/_ref/bin/fluidsim_{legacy,home,hybrid,tgv}
#                                the reference's own headless command-line
#                                tools (its main_*.cpp with its solvers,
#                                geometry and VTK writer), for the CLI tests.
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
mkdir -p "$HERE/_ref/bin"
SRC="$REF_ROOT/src"
# skip when every output is newer than this script and the drivers
STAMP="$HERE/_ref/.stamp"
if [ -f "$STAMP" ] && [ "$STAMP" -nt "$0" ] && [ "$STAMP" -nt "$HERE/ref_cpu_driver.cpp" ] \
   && [ "$STAMP" -nt "$HERE/ref_cuda_driver.cu" ] && [ "$STAMP" -nt "$HERE/ref_shim/glm/glm.hpp" ]; then
    echo "[build_ref] up to date"
    exit 0
fi

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
# the reference's command-line tools, linked from objects built in a scratch folder
OBJ="$(mktemp -d)"
trap 'rm -rf "$OBJ"' EXIT
for f in lbm/lbm3d_legacy lbm/lbm3d_home lbm/lbm3d_hybrid lbm/lbm_reinit fields/field_ops \
         fields/init_profiles moment_vtk_writer; do
    "$NVCC" -O2 -std=c++17 -w -gencode arch=compute_100a,code=sm_100a -I"$SRC" \
        -c "$SRC/$f.cu" -o "$OBJ/$(basename "$f").o" &
done
for f in geom/stl_loader geom/voxelize apps/main_legacy apps/main_home apps/main_hybrid \
         bench/main_taylor_green; do
    g++ -O2 -std=c++17 -w -ffp-contract=off -I"$HERE/ref_shim" -I"$SRC" -I"$CUDA_INC" \
        -c "$SRC/$f.cpp" -o "$OBJ/$(basename "$f").o" &
done
wait
COMMON="$OBJ/lbm_reinit.o $OBJ/field_ops.o $OBJ/moment_vtk_writer.o"
GEOM="$OBJ/stl_loader.o $OBJ/voxelize.o $OBJ/init_profiles.o"
ARCH="-gencode arch=compute_100a,code=sm_100a"
for m in legacy home hybrid; do
    "$NVCC" $ARCH -o "$HERE/_ref/bin/fluidsim_$m" "$OBJ/main_$m.o" "$OBJ/lbm3d_$m.o" $GEOM $COMMON
done
"$NVCC" $ARCH -o "$HERE/_ref/bin/fluidsim_tgv" "$OBJ/main_taylor_green.o" "$OBJ/lbm3d_legacy.o" \
    "$OBJ/lbm3d_home.o" $COMMON
touch "$STAMP"
echo "[build_ref] ok"
