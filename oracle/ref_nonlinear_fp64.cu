// Test infrastructure: compiles the reference's nonlinear operator
// (gpu_flow/code/operator/nonlinear_operator_rayleigh_noslip.cu) for its FP64 build.
// That file defines init_operator with a `cufftReal` (float) penalization argument while
// its header declares CUDA_FLOAT_REAL (double under PRECISION_DOUBLE), so the FP64 build
// does not compile as shipped. The argument is unused without PENALIZED; mapping the one
// spelling to CUDA_FLOAT_REAL after cufft.h has been read makes definition and
// declaration agree and changes nothing else (the file has no other use of cufftReal).
#include "cuda_defines.h"
#define cufftReal CUDA_FLOAT_REAL
#include "operator/nonlinear_operator_rayleigh_noslip.cu"
