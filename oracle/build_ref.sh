#!/bin/bash
# Compiles the reference's own particle path (its headers, unmodified, where
# they lie) with the MPI stand-in into oracle/_ref/: a double build and a
# -DSINGLE build of ref_driver.cpp.  Test infrastructure only.
set -e
HERE="$(cd "$(dirname "$0")" && pwd)"
REF="${LF2_REFERENCE_DIR:-/root/reference}"
if [ ! -f "$REF/LATfield2.hpp" ]; then
  echo "reference sources not found at $REF; skipping oracle/_ref" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
CXX="${CXX:-g++}"
FLAGS="-std=c++14 -O2 -ffp-contract=off -w -I$HERE/mpi_shim -I$REF"
# The FFT build adds the FFTW-interface stand-in (oracle/fftw_shim) and -DFFT3D,
# which brings in the reference's PlanFFT.
for v in double single; do
  out="$HERE/_ref/lf2_ref_driver_$v"
  extra="-DFFT3D -I$HERE/fftw_shim"
  [ "$v" = single ] && extra="$extra -DSINGLE"
  if [ ! -x "$out" ] || [ "$HERE/ref_driver.cpp" -nt "$out" ] || [ "$HERE/mpi_shim/mpi.h" -nt "$out" ] ||
     [ "$HERE/fftw_shim/fftw3.h" -nt "$out" ]; then
    $CXX $FLAGS $extra -o "$out" "$HERE/ref_driver.cpp"
  fi
done
echo "built $HERE/_ref"
