// tracer_kernel.cuh -- passive tracer advance (sm_100a, FP64 positions).
//
// Reference: particle_tracer::step_particles (gpu_flow/code/particle/particle_tracer.cu:141-212)
// builds u, v, w on an Nx x Ny x 128 grid (calculate_velocity_operator.cu:106-147, 426-488;
// levels z_l = linspace(-zmax, zmax, 128), zmax = 0.5f - 1e-3) and advances each particle
// with RK4 on that frozen field with trilinear interpolation (vel_interpolate :508-607,
// PERIODIC wrap), then reflects z at +-zmax (periodic_boundaries :722-764).
// Here the grid is never materialised: the velocity at a grid node (x, y, z_l) is
// evaluated when needed from the 5 L synthesised values u11, u21, u31, u12, u22 of that
// node (one contiguous record per node, written by the contraction kernel that reads
// them anyway), with the same sums as compose_u_from_derivs:
//   u = sum_i C'_i(z_l) u11_i + S_i(z_l) u12_i,  v = sum_i C'_i u21_i + S_i u22_i,
//   w = sum_i C_i(z_l) u31_i.
#pragma once
#include "common.cuh"

namespace rbck {

constexpr int kZNum = 128;

struct TracerArgs {
    const void* nv;       // [Ny*Nx][NodeRec] (R): u11, u21, u31, u12, u22 per grid point
    const double* zbasis; // [128][3][L]: C_i(z_l), S_i(z_l), C'_i(z_l)
    double* pos;          // [3][n] x, y, z
    int n, nx, ny, L;
    double lx, ly, dt, zmax;
};

// Velocity (u, v, w) at the grid node xy on the levels z0 and z1 from the node record.
template <typename R, int L>
RBC_D void node_velocity(const R* __restrict__ nv, size_t xy, const double* zb0, const double* zb1,
                         double (&u0)[3], double (&u1)[3])
{
    constexpr int NR = (5 * L + 1) & ~1;
    typedef typename cplx_t<R>::type R2;
    R rec[NR];
    const R2* src = reinterpret_cast<const R2*>(nv + xy * NR);
#pragma unroll
    for (int q = 0; q < NR / 2; ++q) {
        const R2 v = __ldg(src + q);
        rec[2 * q] = v.x;
        rec[2 * q + 1] = v.y;
    }
    double a0 = 0, b0 = 0, c0 = 0, a1 = 0, b1 = 0, c1 = 0;
#pragma unroll
    for (int i = 0; i < L; ++i) {
        const double v11 = rec[i], v21 = rec[L + i], v31 = rec[2 * L + i], v12 = rec[3 * L + i], v22 = rec[4 * L + i];
        const double C0 = zb0[i], S0 = zb0[L + i], D0 = zb0[2 * L + i];
        const double C1 = zb1[i], S1 = zb1[L + i], D1 = zb1[2 * L + i];
        a0 += D0 * v11 + S0 * v12;
        b0 += D0 * v21 + S0 * v22;
        c0 += C0 * v31;
        a1 += D1 * v11 + S1 * v12;
        b1 += D1 * v21 + S1 * v22;
        c1 += C1 * v31;
    }
    u0[0] = a0; u0[1] = b0; u0[2] = c0;
    u1[0] = a1; u1[1] = b1; u1[2] = c1;
}

template <typename R, int L>
RBC_D void vel_interp(const TracerArgs& A, const double* zb, double x, double y, double z, double& rx, double& ry, double& rz)
{
    const R* nv = reinterpret_cast<const R*>(A.nv);
    const int xs = A.nx, ys = A.ny;
    double xg = x * xs / A.lx;
    double yg = y * ys / A.ly;
    double zg = (A.zmax + z) / (2 * A.zmax) * (kZNum - 1);
    xg -= floor(xg / xs) * xs;
    yg -= floor(yg / ys) * ys;
    // __float2int_rd of the double: round to float, then down
    int ix0 = __float2int_rd((float)xg), iy0 = __float2int_rd((float)yg), iz0 = __float2int_rd((float)zg);
    if (ix0 < 0 || ix0 >= xs) ix0 = 0;
    if (iy0 < 0 || iy0 >= ys) iy0 = 0;
    if (iz0 < 0) iz0 = 0;
    else if (iz0 >= kZNum) iz0 = kZNum - 1;
    const int ix1 = (ix0 + 1 >= xs) ? 0 : ix0 + 1;
    const int iy1 = (iy0 + 1 >= ys) ? 0 : iy0 + 1;
    const int iz1 = (iz0 + 1 >= kZNum) ? iz0 : iz0 + 1;
    const double* zb0 = zb + (size_t)iz0 * 3 * L;
    const double* zb1 = zb + (size_t)iz1 * 3 * L;
    double v00[2][3], v10[2][3], v01[2][3], v11[2][3]; // [z level][component], corners (x, y)
    node_velocity<R, L>(nv, (size_t)iy0 * xs + ix0, zb0, zb1, v00[0], v00[1]);
    node_velocity<R, L>(nv, (size_t)iy0 * xs + ix1, zb0, zb1, v10[0], v10[1]);
    node_velocity<R, L>(nv, (size_t)iy1 * xs + ix0, zb0, zb1, v01[0], v01[1]);
    node_velocity<R, L>(nv, (size_t)iy1 * xs + ix1, zb0, zb1, v11[0], v11[1]);
    double wR = xg - (double)ix0, wL = 1 - wR;
    double cz0y0[3], cz0y1[3], cz1y0[3], cz1y1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        cz0y0[d] = wL * v00[0][d] + wR * v10[0][d];
        cz0y1[d] = wL * v01[0][d] + wR * v11[0][d];
        cz1y0[d] = wL * v00[1][d] + wR * v10[1][d];
        cz1y1[d] = wL * v01[1][d] + wR * v11[1][d];
    }
    wR = yg - (double)iy0;
    wL = 1 - wR;
    double c0[3], c1[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        c0[d] = wL * cz0y0[d] + wR * cz0y1[d];
        c1[d] = wL * cz1y0[d] + wR * cz1y1[d];
    }
    wR = zg - (double)iz0;
    wL = 1 - wR;
    rx = wL * c0[0] + wR * c1[0];
    ry = wL * c0[1] + wR * c1[1];
    rz = wL * c0[2] + wR * c1[2];
}

template <typename R, int L>
__global__ void __launch_bounds__(128) k_tracers(TracerArgs A)
{
    __shared__ double zb[kZNum * 3 * L];
    for (int e = threadIdx.x; e < kZNum * 3 * L; e += blockDim.x) zb[e] = A.zbasis[e];
    __syncthreads();
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= A.n) return;
    double x = A.pos[t], y = A.pos[A.n + t], z = A.pos[2 * A.n + t];
    const double dt = A.dt;
    double vx, vy, vz;
    vel_interp<R, L>(A, zb, x, y, z, vx, vy, vz);
    const double dx1 = dt * vx, dy1 = dt * vy, dz1 = dt * vz;
    vel_interp<R, L>(A, zb, x + 0.5 * dx1, y + 0.5 * dy1, z + 0.5 * dz1, vx, vy, vz);
    const double dx2 = dt * vx, dy2 = dt * vy, dz2 = dt * vz;
    vel_interp<R, L>(A, zb, x + 0.5 * dx2, y + 0.5 * dy2, z + 0.5 * dz2, vx, vy, vz);
    const double dx3 = dt * vx, dy3 = dt * vy, dz3 = dt * vz;
    vel_interp<R, L>(A, zb, x + dx3, y + dy3, z + dz3, vx, vy, vz);
    const double dx4 = dt * vx, dy4 = dt * vy, dz4 = dt * vz;
    x += (dx1 + 2 * (dx2 + dx3) + dx4) / 6.;
    y += (dy1 + 2 * (dy2 + dy3) + dy4) / 6.;
    z += (dz1 + 2 * (dz2 + dz3) + dz4) / 6.;
    const double zm = A.zmax;
    if (!(z <= zm)) z = (z < 2 * zm) ? 2 * zm - z : zm;  // also sends NaN to the lid
    else if (z < -zm) z = (z > -2 * zm) ? -2 * zm - z : -zm;
    A.pos[t] = x;
    A.pos[A.n + t] = y;
    A.pos[2 * A.n + t] = z;
}

} // namespace rbck
