#!/usr/bin/env bash
# Compiles the reference IPPI-LBM sources, where they lie, into checker
# libraries oracle/_ref/libippi_ref_<variant>.so (test infrastructure only).
# The reference's own CMake build is not used: its two translation units are
# compiled directly with g++ -O3 (the flags of its CMakeLists.txt), with
#   -include ref_shim/ref_config.h  in place of Parameter.h (operator/precision)
#   -I ref_shim                     for <mpi.h>, <torch/script.h>, <ATen/Parallel.h>
# and linked with ref_driver.cpp and the oracle library (for the net forward).
# Usage: oracle/build_ref.sh [reference-root]   (default /root/reference)
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
REFROOT=${1:-${IPPI_REFERENCE_DIR:-/root/reference}}
SRC=$REFROOT/IPPI-LBM
OUT=$HERE/_ref
if [ ! -f "$SRC/mesh.cpp" ]; then
  echo "build_ref: reference sources not found under $REFROOT; nothing built"
  exit 0
fi
make -s -C "$HERE"
mkdir -p "$OUT"
CXX=${IPPI_REF_CXX:-/usr/bin/g++}  # system g++: the libstdc++ must be the shared one the host process uses
build() {
  local name=$1; shift
  local lib=$OUT/libippi_ref_$name.so
  if [ "$lib" -nt "$HERE/ref_driver.cpp" ] && [ "$lib" -nt "$SRC/mesh.cpp" ] && \
     [ "$lib" -nt "$HERE/ref_shim/mpi.h" ] && [ "$lib" -nt "$HERE/ref_shim/ref_config.h" ] && \
     [ "$lib" -nt "$HERE/_build/libippi_oracle.so" ]; then
    return 0
  fi
  "$CXX" -O3 -std=c++17 -fPIC -shared -w -pthread "$@" \
    -include "$HERE/ref_shim/ref_config.h" -I "$HERE/ref_shim" -I "$SRC" \
    "$SRC/mesh.cpp" "$SRC/NodeAndLattice.cpp" "$HERE/ref_driver.cpp" \
    -L "$HERE/_build" -lippi_oracle -Wl,-rpath,'$ORIGIN/../_build' \
    -o "$lib"
  echo "build_ref: $lib"
}
build srt
build srt_peskin -DIPPI_REF_PESKIN
build mrt -DIPPI_REF_MRT
build rr -DIPPI_REF_RR
build srt_f32 -DIPPI_REF_SINGLE
build mrt_f32 -DIPPI_REF_MRT -DIPPI_REF_SINGLE
