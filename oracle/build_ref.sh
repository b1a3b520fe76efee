#!/usr/bin/env bash
# Compiles the reference IPPI-LBM sources, where they lie, into checker
# libraries oracle/_ref/libippi_ref_<variant>.so (test infrastructure only).
# The reference's own CMake build is not used: its two translation units are
# compiled directly with g++ -O3 (the flags of its CMakeLists.txt), with
#   -include ref_shim/ref_config.h  in place of Parameter.h (operator/precision)
#   -I ref_shim                     for <mpi.h>, <torch/script.h>, <ATen/Parallel.h>
# and linked with ref_driver.cpp and the oracle library (for the net forward).
# The *_torch variants compile the same sources against the libtorch that the
# torch wheel ships (headers and libraries), with ref_torch/ mapping the
# reference's archive path to IPPI_REF_PT_DIR: the boundary nets then run
# through libtorch itself, on the shipped TorchScript archives, which are
# copied next to the libraries (oracle/_ref/nn/, git-ignored).
# Usage: oracle/build_ref.sh [reference-root]   (default: $IPPI_REFERENCE_DIR;
# the reference's mount point in the build container when that is unset)
set -euo pipefail
HERE=$(cd "$(dirname "$0")" && pwd)
REFROOT=${1:-${IPPI_REFERENCE_DIR:-/root/reference}}  # the reference's mount point
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
build_torch() {
  local name=$1; shift
  local lib=$OUT/libippi_ref_$name.so
  local torch
  torch=$(python3 -c "import torch, os; print(os.path.dirname(torch.__file__))" 2>/dev/null) || return 0
  [ -f "$torch/include/torch/script.h" ] || return 0
  mkdir -p "$OUT/nn"
  for t in 1 3 5 7; do
    [ -f "$REFROOT/NNmodel/AutoT0$t.pt" ] && cp -p "$REFROOT/NNmodel/AutoT0$t.pt" "$OUT/nn/"
  done
  if [ "$lib" -nt "$HERE/ref_driver.cpp" ] && [ "$lib" -nt "$SRC/mesh.cpp" ] && \
     [ "$lib" -nt "$HERE/ref_shim/mpi.h" ] && [ "$lib" -nt "$HERE/ref_shim/ref_config.h" ] && \
     [ "$lib" -nt "$HERE/ref_torch/torch/script.h" ] && [ "$lib" -nt "$HERE/_build/libippi_oracle.so" ]; then
    return 0
  fi
  "$CXX" -O3 -std=c++17 -fPIC -shared -w -pthread -DIPPI_REF_TORCH "$@" \
    -include "$HERE/ref_shim/ref_config.h" -I "$HERE/ref_torch" -I "$torch/include" \
    -I "$torch/include/torch/csrc/api/include" -I "$HERE/ref_shim" -I "$SRC" \
    "$SRC/mesh.cpp" "$SRC/NodeAndLattice.cpp" "$HERE/ref_driver.cpp" \
    -L "$HERE/_build" -lippi_oracle -Wl,-rpath,'$ORIGIN/../_build' \
    -L "$torch/lib" -ltorch -ltorch_cpu -lc10 -Wl,-rpath,"$torch/lib" \
    -o "$lib"
  echo "build_ref: $lib"
}
build srt
build srt_peskin -DIPPI_REF_PESKIN
build mrt -DIPPI_REF_MRT
build rr -DIPPI_REF_RR
build srt_f32 -DIPPI_REF_SINGLE
build mrt_f32 -DIPPI_REF_MRT -DIPPI_REF_SINGLE
build_torch srt_torch
build_torch srt_f32_torch -DIPPI_REF_SINGLE
