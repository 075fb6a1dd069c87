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
unsigned long long uid(const rbc_handle* h); // unique per handle in the process
bool has_tracers(const rbc_handle* h);
void state_changed(rbc_handle* h);           // the next step is an Euler step

// Gauss-Legendre collocation tables on the device, [nq][3][L] (C, C', S at z_q) and the
// least-squares inverses [2][L][nq] (Ps, Pc); built by the caller (fno.cu) once.
// Collocation fields of the current state: out[p][4 nq] (p = y Nx + x; channel
// field * nq + q for field theta, u, v, w), FP32, on the device.
rbc_status colloc_encode(rbc_handle* h, int nq, const double* d_basis, float* d_out);

// colloc_encode plus the mean-mode forcing of the same state (the solver's nonlinear
// operator): d_g[3L] = (2 Re N_theta_k(q=0), 2 Pr NF_k, 2 Pr NG_k), d_y0[3L] = the mean
// modes (Re theta_k(q=0), F_k, G_k) of the state.
rbc_status colloc_encode_forcing(rbc_handle* h, int nq, const double* d_basis, float* d_out, double* d_g,
                                 double* d_y0);
// The mean modes advanced from d_y0 by nsub plain-step recursions (AB2 + implicit Euler,
// the update kernel's q = 0 arithmetic) with forcing linear in time through d_g0 and d_gp
// (NULL: constant forcing), written into the state; the next step is an Euler step.
rbc_status mean_advance(rbc_handle* h, const double* d_y0, const double* d_g0, const double* d_gp, int nsub);

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
// The same value written to device memory on the handle's stream (no host wait).
rbc_status nu_wall_record(rbc_handle* h, double* d_out);

void set_error(rbc_handle* h, const char* msg);

} // namespace rbcint
