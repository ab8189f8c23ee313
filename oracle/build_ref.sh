#!/bin/bash
# Builds the reference's CPU code from its own sources into oracle/_ref/.
#   ref_harness_exact  reference headers + oracle/ref_harness.cpp, no
#                      fast-math, no FMA contraction (golden vectors)
#   ref_harness_fast   same, with the flags of the reference's compile_omp.sh
#                      (timed CPU baseline for generated inputs)
#   testDensitySubGrid_omp  the reference's own OpenMP driver, compile_omp.sh
#                      flags plus -DMEANING_OF_HASTE (timed CPU baseline, C1)
#   testDensitySubGrid_omp_files  the same driver with its result files
#                      switched on (-DMM_FILE -DBIN_FILE: neutral_fractions.dat
#                      and .bin), no fast-math (golden output files)
#   testDensitySubGrid_omp_dust  the reference's dust driver (forced first
#                      scattering, peel-off image.dat), no fast-math (statistical
#                      golden image of the dust path)
# Deviations from compile_omp.sh, all needed to build on this image:
#   -march=x86-64-v3 instead of -march=native (the binary runs on another host),
#   -include cstdint (CommandLineOption.hpp uses int_fast32_t without it),
#   no -Werror (GCC 13 -Wcatch-value in Utilities.hpp),
#   oracle/hdf5_stub on the include path (HDF5 is not installed).
# Reads REF_DIR (default /root/reference); never writes there.
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF_DIR="${REF_DIR:-/root/reference}"
OUT="$HERE/_ref"
if [ ! -f "$REF_DIR/DensitySubGrid.hpp" ]; then
  echo "reference sources not found in $REF_DIR" >&2
  exit 3
fi
CXX=g++
mkdir -p "$OUT"
make -s -C "$HERE" libcmi_oracle.so
COMMON="-std=c++11 -fopenmp -I$REF_DIR -I$HERE -Wall -Wno-unused-variable -Wno-unused-but-set-variable -Wno-catch-value"
LINK="-L$HERE -lcmi_oracle -Wl,-rpath,\$ORIGIN/.. -lm"
$CXX $COMMON -O2 -ffp-contract=off -fno-fast-math -o "$OUT/ref_harness_exact" \
  "$HERE/ref_harness.cpp" $LINK
$CXX $COMMON -march=x86-64-v3 -O3 -ftree-vectorize -funroll-loops -ffast-math \
  -o "$OUT/ref_harness_fast" "$HERE/ref_harness.cpp" $LINK
TMP="$(mktemp -d)"
for f in testDensitySubGrid_omp.cpp CommandLineOption.cpp CommandLineParser.cpp; do
  $CXX -std=c++11 -fopenmp -march=x86-64-v3 -Wall -Wno-catch-value -Wignored-qualifiers \
    -O3 -ftree-vectorize -funroll-loops -ffast-math -DMEANING_OF_HASTE \
    -include cstdint -I"$HERE/hdf5_stub" -I"$REF_DIR" -c "$REF_DIR/$f" -o "$TMP/${f%.cpp}.o" \
    2> "$TMP/${f%.cpp}.log" || { cat "$TMP/${f%.cpp}.log" >&2; exit 1; }
done
$CXX -fopenmp -o "$OUT/testDensitySubGrid_omp" "$TMP"/*.o
rm -f "$TMP"/*.o
for f in testDensitySubGrid_omp.cpp CommandLineOption.cpp CommandLineParser.cpp; do
  $CXX -std=c++11 -fopenmp -Wall -Wno-catch-value -O2 -ffp-contract=off -fno-fast-math \
    -DMM_FILE -DBIN_FILE -include cstdint -I"$HERE/hdf5_stub" -I"$REF_DIR" \
    -c "$REF_DIR/$f" -o "$TMP/${f%.cpp}.o" 2> "$TMP/${f%.cpp}.log" || { cat "$TMP/${f%.cpp}.log" >&2; exit 1; }
done
$CXX -fopenmp -o "$OUT/testDensitySubGrid_omp_files" "$TMP"/*.o
rm -f "$TMP"/*.o
for f in testDensitySubGrid_omp_dust.cpp CommandLineOption.cpp CommandLineParser.cpp; do
  $CXX -std=c++11 -fopenmp -Wall -Wno-catch-value -O2 -ffp-contract=off -fno-fast-math \
    -include cstdint -I"$HERE/hdf5_stub" -I"$REF_DIR" \
    -c "$REF_DIR/$f" -o "$TMP/${f%.cpp}.o" 2> "$TMP/${f%.cpp}.log" || { cat "$TMP/${f%.cpp}.log" >&2; exit 1; }
done
$CXX -fopenmp -o "$OUT/testDensitySubGrid_omp_dust" "$TMP"/*.o
rm -rf "$TMP"
echo "built: $(ls "$OUT" | tr '\n' ' ')"
