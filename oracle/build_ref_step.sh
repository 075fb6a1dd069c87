#!/bin/sh
# Builds the reference's OWN FP64 Boussinesq step (its sources compiled where they lie,
# -DPRECISION_DOUBLE, for sm_100a, with cuFFT) plus the test-only driver ref_step_main.cu
# into oracle/_ref/ref_step. GSL, which the reference's operator constructors call for a
# few small LU inverses, is not installed here: the project-written stand-in headers in
# oracle/gsl_standin/ take its place. The nonlinear operator is compiled through
# ref_nonlinear_fp64.cu, which reconciles one float/double spelling that keeps the
# shipped FP64 build from compiling. Test infrastructure only (golden step fixtures).
#
# usage: sh oracle/build_ref_step.sh <reference root>   (or SDC_REFERENCE=<root>)
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
ROOT=${1:-$SDC_REFERENCE}
if [ -z "$ROOT" ] || [ ! -f "$ROOT/gpu_flow/code/operator/nonlinear_operator_rayleigh_noslip.cu" ]; then
    echo "reference sources not given or not present; skipping oracle/_ref/ref_step" >&2
    exit 0
fi
CODE="$ROOT/gpu_flow/code"
NVCC=${NVCC:-/usr/local/cuda/bin/nvcc}
mkdir -p "$HERE/_ref"
"$NVCC" -std=c++14 -O3 -DPRECISION_DOUBLE -gencode arch=compute_100a,code=sm_100a -w \
    -I"$HERE/gsl_standin" -I"$CODE" \
    "$CODE/util/coeff.cu" "$CODE/util/util.cu" \
    "$CODE/matrix/matrix_device.cu" "$CODE/matrix/matrix_folder.cu" "$CODE/matrix/matrix_host.cu" \
    "$CODE/matrix/matrix_host_iterator.cu" \
    "$CODE/operator/linear_implicit_operator.cu" "$CODE/operator/inverse_B_matrix.cu" \
    "$HERE/ref_nonlinear_fp64.cu" \
    "$CODE/timestepping/implicit_explicit_stepping.cu" \
    "$HERE/ref_step_main.cu" -lcufft -o "$HERE/_ref/ref_step"
echo "built $HERE/_ref/ref_step"
