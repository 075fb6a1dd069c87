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
#include "splitmix.h"

namespace rbck {

constexpr int kZNum = 128;

struct TracerArgs {
    const void* nv;       // [Ny*Nx][NodeRec] (R): u11, u21, u31, u12, u22 per grid point
    const double* zbasis; // [128][3][L]: C_i(z_l), S_i(z_l), C'_i(z_l)
    double* pos;          // [3][n] x, y, z
    int n, nx, ny, L;
    double lx, ly, dt, zmax;
    // grid-coordinate scales, precomputed on the host: nx / lx, ny / ly,
    // (128 - 1) / (2 zmax), 1 / nx, 1 / ny (one multiply each where the reference divides)
    double sx, sy, sz, inx, iny;
    const double* set_sigma;          // [sets] sqrt(2 D dt) of each tracer set (0: no diffusion)
    int per_set;                      // tracers per set (consecutive ranges)
    unsigned long long noise_seed;
    const long long* step_counter;    // completed fluid steps = step m of the new positions
    float* track;                     // [track_cap][3][n] FP32 frames, or null
    int track_cap, track_period;
};

template <int L> struct NodeRecLen { static constexpr int value = (5 * L + 1) & ~1; };

// Loads the node record of grid point xy into registers.
template <typename R, int L>
RBC_D void load_record(const R* __restrict__ nv, size_t xy, R (&rec)[NodeRecLen<L>::value])
{
    constexpr int NR = NodeRecLen<L>::value;
    typedef typename cplx_t<R>::type R2;
    const R2* src = reinterpret_cast<const R2*>(nv + xy * NR);
#pragma unroll
    for (int q = 0; q < NR / 2; ++q) {
        const R2 v = __ldg(src + q);
        rec[2 * q] = v.x;
        rec[2 * q + 1] = v.y;
    }
}

// Velocity (u, v, w) of a node on the levels z0 and z1 from its record.
template <typename R, int L>
RBC_D void node_velocity(const R* rec, const double* zb0, const double* zb1, double (&u0)[3], double (&u1)[3])
{
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

// Cell of (x, y, z) as the reference's vel_interpolate finds it, for corner lane q of a team
// of 4 (lane q takes the xy corner (q & 1, q >> 1)): the corner's node, the two bracketing
// levels and the lane's trilinear weights.
struct Corner {
    int node, iz0, iz1;
    double w, wz0, wz1;
};
RBC_D Corner find_corner(const TracerArgs& A, int q, double x, double y, double z)
{
    const int xs = A.nx, ys = A.ny;
    // the reference's x Nx / Lx, (zmax + z) / (2 zmax) (Nz - 1) and periodic wrap, with the
    // divisions replaced by multiplies with host-computed factors (equal to rounding)
    double xg = x * A.sx;
    double yg = y * A.sy;
    double zg = (A.zmax + z) * A.sz;
    xg -= floor(xg * A.inx) * xs;
    yg -= floor(yg * A.iny) * ys;
    // __float2int_rd of the double: round to float, then down
    int ix0 = __float2int_rd((float)xg), iy0 = __float2int_rd((float)yg), iz0 = __float2int_rd((float)zg);
    if (ix0 < 0 || ix0 >= xs) ix0 = 0;
    if (iy0 < 0 || iy0 >= ys) iy0 = 0;
    if (iz0 < 0) iz0 = 0;
    else if (iz0 >= kZNum) iz0 = kZNum - 1;
    const int ix1 = (ix0 + 1 >= xs) ? 0 : ix0 + 1;
    const int iy1 = (iy0 + 1 >= ys) ? 0 : iy0 + 1;
    Corner c;
    c.iz0 = iz0;
    c.iz1 = (iz0 + 1 >= kZNum) ? iz0 : iz0 + 1;
    const double wx1 = xg - (double)ix0, wx0 = 1 - wx1;
    const double wy1 = yg - (double)iy0, wy0 = 1 - wy1;
    c.wz1 = zg - (double)iz0;
    c.wz0 = 1 - c.wz1;
    const int ix = (q & 1) ? ix1 : ix0, iy = (q >> 1) ? iy1 : iy0;
    c.w = ((q & 1) ? wx1 : wx0) * ((q >> 1) ? wy1 : wy0);
    c.node = iy * xs + ix;
    return c;
}

// The team's interpolated velocity from this lane's corner record: the node evaluated at
// the two levels, weighted, and the 4 contributions added with two shuffle rounds; every
// lane of the team returns the sum.
template <typename R, int L>
RBC_D void team_velocity(const Corner& c, const R* rec, const double* zb, double& rx, double& ry, double& rz)
{
    double u0[3], u1[3];
    node_velocity<R, L>(rec, zb + (size_t)c.iz0 * 3 * L, zb + (size_t)c.iz1 * 3 * L, u0, u1);
    double v[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        v[d] = c.w * (c.wz0 * u0[d] + c.wz1 * u1[d]);
        v[d] += __shfl_xor_sync(0xffffffffu, v[d], 1, 4);
        v[d] += __shfl_xor_sync(0xffffffffu, v[d], 2, 4);
    }
    rx = v[0];
    ry = v[1];
    rz = v[2];
}

// Velocity at (x, y, z) by trilinear interpolation of the node velocities (the
// reference's vel_interpolate), a team of 4 consecutive lanes per particle, the corner
// record held in registers.
template <typename R, int L>
RBC_D void vel_interp_team(const TracerArgs& A, const double* zb, int q, double x, double y, double z,
                           double& rx, double& ry, double& rz, R (&rec)[NodeRecLen<L>::value], int& cached)
{
    const Corner c = find_corner(A, q, x, y, z);
    // RK stages rarely leave the cell: reload this corner's record only when it changed
    if (c.node != cached) {
        load_record<R, L>(reinterpret_cast<const R*>(A.nv), (size_t)c.node, rec);
        cached = c.node;
    }
    team_velocity<R, L>(c, rec, zb, rx, ry, rz);
}

// RK4 on the frozen field (step_particle_on_GPU, particle_tracer.cu:610-687): vel(x, y, z,
// vx, vy, vz) returns the team's interpolated velocity.
template <typename V>
RBC_D void rk4_team(double& x, double& y, double& z, double dt, V&& vel)
{
    double vx, vy, vz;
    vel(x, y, z, vx, vy, vz);
    const double dx1 = dt * vx, dy1 = dt * vy, dz1 = dt * vz;
    vel(x + 0.5 * dx1, y + 0.5 * dy1, z + 0.5 * dz1, vx, vy, vz);
    const double dx2 = dt * vx, dy2 = dt * vy, dz2 = dt * vz;
    vel(x + 0.5 * dx2, y + 0.5 * dy2, z + 0.5 * dz2, vx, vy, vz);
    const double dx3 = dt * vx, dy3 = dt * vy, dz3 = dt * vz;
    vel(x + dx3, y + dy3, z + dz3, vx, vy, vz);
    const double dx4 = dt * vx, dy4 = dt * vy, dz4 = dt * vz;
    constexpr double sixth = 1.0 / 6.0;
    x += (dx1 + 2 * (dx2 + dx3) + dx4) * sixth;
    y += (dy1 + 2 * (dy2 + dy3) + dy4) * sixth;
    z += (dz1 + 2 * (dz2 + dz3) + dz4) * sixth;
}

// Diffusion step, lid reflection and store (with the track frame) of particle t's new
// position; called by one lane per particle.
RBC_D void finish_tracer(const TracerArgs& A, int t, double x, double y, double z)
{
    const long long m = *A.step_counter;
    const double sg = A.set_sigma[t / A.per_set];
    if (sg > 0.0) {
        // diffuse_particles (particle_tracer.cu:690-716) before the lid reflection
        x += sg * rbcrng::diffusion_normal(A.noise_seed, m, A.n, t, 0);
        y += sg * rbcrng::diffusion_normal(A.noise_seed, m, A.n, t, 1);
        z += sg * rbcrng::diffusion_normal(A.noise_seed, m, A.n, t, 2);
    }
    const double zm = A.zmax;
    if (!(z <= zm)) z = (z < 2 * zm) ? 2 * zm - z : zm;  // also sends NaN to the lid
    else if (z < -zm) z = (z > -2 * zm) ? -2 * zm - z : -zm;
    A.pos[t] = x;
    A.pos[A.n + t] = y;
    A.pos[2 * A.n + t] = z;
    if (A.track && m % A.track_period == 0) {
        float* fr = A.track + (size_t)((m / A.track_period) % A.track_cap) * 3 * A.n;
        fr[t] = (float)x;
        fr[A.n + t] = (float)y;
        fr[2 * A.n + t] = (float)z;
    }
}

// Corner records gathered by the lanes' own loads into registers (any record size).
template <typename R, int L>
__global__ void __launch_bounds__(128) k_tracers(TracerArgs A)
{
    __shared__ double zb[kZNum * 3 * L];
    for (int e = threadIdx.x; e < kZNum * 3 * L; e += blockDim.x) zb[e] = A.zbasis[e];
    __syncthreads();
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = gt >> 2, q = gt & 3;               // particle, corner lane
    const bool live = t < A.n;                       // whole teams are live or not
    const int tt = live ? t : 0;
    double x = A.pos[tt], y = A.pos[A.n + tt], z = A.pos[2 * A.n + tt];
    R rec[NodeRecLen<L>::value];
    int cached = -1;
    rk4_team(x, y, z, A.dt, [&](double px, double py, double pz, double& vx, double& vy, double& vz) {
        vel_interp_team<R, L>(A, zb, q, px, py, pz, vx, vy, vz, rec, cached);
    });
    if (live && q == 0) finish_tracer(A, t, x, y, z);
}

// Copies positions into one FP32 track frame (the frame of freshly set positions).
__global__ void k_track_frame(const double* __restrict__ pos, float* __restrict__ frame, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < 3 * n; i += gridDim.x * blockDim.x)
        frame[i] = (float)pos[i];
}

// Sums for the tracer moments in FP64, one CTA of 1024 threads: thread i sums particles
// i, i + 1024, ... (and pairs likewise), then a fixed shared-memory tree; deterministic.
// out[0..3] = sum x, sum y, sum x^2 + y^2, sum over pairs of the squared periodic separation.
// n positions of one set starting at pos: x at pos[i], y at pos[stride + i].
__global__ void __launch_bounds__(1024) k_tracer_sums(const double* __restrict__ pos, int n, int stride, double lx,
                                                      double ly, double* __restrict__ out)
{
    __shared__ double red[4][1024];
    double sx = 0, sy = 0, s2 = 0, sp = 0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double x = pos[i], y = pos[stride + i];
        sx += x;
        sy += y;
        s2 += x * x + y * y;
    }
    for (int i = 2 * threadIdx.x; i < n - 1; i += 2 * blockDim.x) {
        double dx = fabs(pos[i + 1] - pos[i]), dy = fabs(pos[stride + i + 1] - pos[stride + i]);
        if (dx > 0.5 * lx) dx = lx - dx;
        if (dy > 0.5 * ly) dy = ly - dy;
        sp += dx * dx + dy * dy;
    }
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = sy;
    red[2][threadIdx.x] = s2;
    red[3][threadIdx.x] = sp;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s)
            for (int c = 0; c < 4; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x < 4) out[threadIdx.x] = red[threadIdx.x][0];
}

} // namespace rbck
