#!/bin/bash
# Builds the reference pieces that compile on their own, from the reference
# tree, into oracle/_ref/ (binaries only; oracle/_ref/ is git-ignored).
# TEST INFRASTRUCTURE: the outputs only check the oracle.
#
#   ref_cpu  particles_sort + the chain-mesh recursion + cloud4 +
#            apply_laplacian, extracted verbatim from src/particles.cpp,
#            src/chainmesh.cpp and src/gravity_long.cpp (into a temporary
#            directory) and driven by oracle/ref_harness_cpu.cpp
#   ref_gpu  src/kick_pme.cu and src/gravity_short.cu compiled whole for
#            sm_100a, linked with oracle/ref_harness_gpu.cu
#
# The reference's own build (CMake + HPX, Boost, FFTW, GSL, MPI) is not used.
set -euo pipefail
REF=${REF:-/root/reference}
HERE=$(cd "$(dirname "$0")" && pwd)
OUT=$HERE/_ref
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
[ -d "$REF/src" ] || { echo "reference tree not found at $REF" >&2; exit 1; }
mkdir -p "$OUT"
TMP=$(mktemp -d)
trap 'rm -rf "$TMP"' EXIT

extract() {  # extract <file> <first line regex> <out>: the function from its header to the first '}' in column 0
  awk -v pat="$2" 'found == 0 && $0 ~ pat {found = 1} found == 1 {print} found == 1 && /^}/ {exit}' "$1" > "$3"
  [ -s "$3" ] || { echo "could not extract $2 from $1" >&2; exit 1; }
}
extract "$REF/src/particles.cpp" '^int particles_sort\(int begin, int end, double xm, int xdim\)' "$TMP/particles_sort.inc"
extract "$REF/src/chainmesh.cpp" '^static void sort\(const range<int> chain_box, int pbegin, int pend\) \{' "$TMP/chainmesh_sort.inc"
extract "$REF/src/gravity_long.cpp" '^double cloud4\(double x\)' "$TMP/cloud4.inc"
extract "$REF/src/gravity_long.cpp" '^void apply_laplacian\(gravity_long_type type\)' "$TMP/apply_laplacian.inc"
# initial conditions: the power-spectrum table, its sigma8 normalisation and
# the growth factor (src/initialize.cpp:10-66,76-83,182-211)
awk '/^struct power_spectrum_function \{/ {f = 1} f == 1 {print} f == 1 && /^};/ {exit}' "$REF/src/initialize.cpp" > "$TMP/power_spectrum.inc"
[ -s "$TMP/power_spectrum.inc" ] || { echo "could not extract power_spectrum_function" >&2; exit 1; }
extract "$REF/src/initialize.cpp" '^double growth_factor\(double omega_m, float a\)' "$TMP/growth_factor.inc"
extract "$REF/src/initialize.cpp" '^static power_spectrum_function read_power_spectrum\(\) \{' "$TMP/read_power_spectrum.inc"

# nvcc (host code) so that tigerpm/tigerpm.hpp skips its HPX include
ARCH="-gencode arch=compute_100a,code=sm_100a"
"$NVCC" $ARCH -std=c++17 -O2 -DNDEBUG -x cu -I"$REF" -I"$TMP" -include string "$HERE/ref_harness_cpu.cpp" -o "$OUT/ref_cpu"
"$NVCC" $ARCH -std=c++17 -O3 -DNDEBUG -rdc=true -I"$REF" -include string -c "$REF/src/kick_pme.cu" -o "$TMP/kick_pme.o"
"$NVCC" $ARCH -std=c++17 -O3 -DNDEBUG -rdc=true -I"$REF" -include string -c "$REF/src/gravity_short.cu" -o "$TMP/gravity_short.o"
"$NVCC" $ARCH -std=c++17 -O3 -DNDEBUG -rdc=true -I"$REF" -include string -c "$HERE/ref_harness_gpu.cu" -o "$TMP/harness.o"
"$NVCC" $ARCH -rdc=true "$TMP/kick_pme.o" "$TMP/gravity_short.o" "$TMP/harness.o" -o "$OUT/ref_gpu" -lcudart
echo "built $OUT/ref_cpu $OUT/ref_gpu"
