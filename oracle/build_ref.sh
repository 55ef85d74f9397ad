#!/usr/bin/env bash
# Compiles the reference's own CUDA solver from its sources where they lie
# (read-only) into oracle/_ref/ra_ref, for sm_100a, with the device shim
# above, and its host-only SCC tools (SCC_CONTRACT/scc_contract.cpp,
# convert_test_to_scc.cpp, split_queries_by_scc.cpp) into oracle/_ref/.
# Nothing is copied out of the reference tree; the only outputs are the
# executables.  Test infrastructure only: the engine never runs them.
#   usage: oracle/build_ref.sh REFERENCE_ROOT   (or MF_REFERENCE_ROOT set)
set -euo pipefail
HERE="$(cd "$(dirname "${BASH_SOURCE[0]}")" && pwd)"
REF="${1:-${MF_REFERENCE_ROOT:-}}"
if [ -z "$REF" ]; then
  echo "build_ref: give the reference project's root (argument or MF_REFERENCE_ROOT)" >&2
  exit 0
fi
SRC="$REF/Region_Aware_PR_with_Pruning_BoundaryCore.cu"
if [ ! -f "$SRC" ]; then
  echo "build_ref: $SRC not found; keeping any prebuilt oracle/_ref/ra_ref" >&2
  exit 0
fi
mkdir -p "$HERE/_ref"
NVCC="${NVCC:-nvcc}"
"$NVCC" -O3 -gencode arch=compute_100a,code=sm_100a -cudart shared \
  -o "$HERE/_ref/ra_ref" "$SRC" "$HERE/ref_device_shim.c" -ldl
echo "build_ref: built $HERE/_ref/ra_ref"
for tool in scc_contract convert_test_to_scc split_queries_by_scc; do
  TSRC="$REF/SCC_CONTRACT/$tool.cpp"
  if [ -f "$TSRC" ]; then
    "${CXX:-g++}" -O3 -std=c++17 -o "$HERE/_ref/$tool" "$TSRC"
    echo "build_ref: built $HERE/_ref/$tool"
  fi
done
