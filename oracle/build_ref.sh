#!/bin/sh
# Compiles the reference's own Galerkin coefficient code (host C++, no CUDA, no GSL)
# from its sources in place, plus the C-ABI shim, into oracle/_ref/libref_coeff.so.
# Test infrastructure only: used to pin the oracle's and the library's tables.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
# usage: sh oracle/build_ref.sh <reference root>   (or SDC_REFERENCE=<root>)
ROOT=${1:-$SDC_REFERENCE}
REF="$ROOT/gpu_flow/code/util"
if [ -z "$ROOT" ] || [ ! -f "$REF/coeff.cu" ]; then
    echo "reference sources not given or not present; skipping oracle/_ref" >&2
    exit 0
fi
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -fPIC -shared -I"$REF" -x c++ "$REF/coeff.cu" -x none "$HERE/ref_coeff_shim.cpp" \
    -o "$HERE/_ref/libref_coeff.so"
echo "built $HERE/_ref/libref_coeff.so"
