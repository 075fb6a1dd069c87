// solver_internal.h -- library-internal access to a solver handle's device state, used by
// the surrogate (fno.cu). Not part of the C ABI. Every function runs on the handle's
// current stream, sets the handle's last error and returns a status on failure.
#pragma once
#include "rbc.h"
#include <cuda_runtime.h>
#include <cstddef>

namespace rbcint {

struct GridDesc {
    int nx, ny, L, ckeep, device;
    double lx, ly, dt, ra, pr;
    bool mixed;
};
GridDesc grid(const rbc_handle* h);
cudaStream_t stream(const rbc_handle* h);

// Gauss-Legendre collocation tables on the device, [nq][3][L] (C, C', S at z_q) and the
// least-squares inverses [2][L][nq] (Ps, Pc); built by the caller (fno.cu) once.
// Collocation fields of the current state: out[p][4 nq] (p = y Nx + x; channel
// field * nq + q for field theta, u, v, w), FP32, on the device.
rbc_status colloc_encode(rbc_handle* h, int nq, const double* d_basis, float* d_out);

// state += the projection of the collocation increment d_delta[p][4 nq] onto the
// Galerkin state (theta, f, g, F, G); scratch: colloc_scratch_bytes() of device memory.
// Dealiased, Hermitian on the kx = 0 column; the next step is an Euler step.
size_t colloc_scratch_bytes(const rbc_handle* h);
rbc_status colloc_add(rbc_handle* h, int nq, const double* d_proj, const float* d_delta, void* d_scratch);

// Device copy of the whole spectral state (theta, f, g, F, G) in and out.
size_t state_bytes(const rbc_handle* h);
rbc_status state_save(rbc_handle* h, void* d_dst);
rbc_status state_load(rbc_handle* h, const void* d_src); // next step is an Euler step

// Nu_wall of the current state (1 - sum_k (k+1) pi Re theta_k(q=0)).
rbc_status nu_wall(rbc_handle* h, double* nu);

void set_error(rbc_handle* h, const char* msg);

} // namespace rbcint
