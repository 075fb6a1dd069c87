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

// Loads half `hf` of the node record of grid point xy into registers (NodeRec layout:
// modes i in [hf LH, hf LH + LH), five values per mode). Records are written by the
// contraction of the same step, which has completed before the tracer kernel starts.
template <typename R, int L>
RBC_D void load_half_record(const R* __restrict__ nv, size_t xy, int hf, R (&rec)[NodeRec<L>::HALF])
{
    constexpr int HALF = NodeRec<L>::HALF;
    typedef typename cplx_t<R>::type R2;
    const R2* src = reinterpret_cast<const R2*>(nv + xy * NodeRec<L>::value + (size_t)hf * HALF);
#pragma unroll
    for (int q = 0; q < HALF / 2; ++q) {
        const R2 v = __ldg(src + q);
        rec[2 * q] = v.x;
        rec[2 * q + 1] = v.y;
    }
}

// This half's share of the velocity (u, v, w) of a node on the levels zb0 and zb1 (rows of
// the [128][3][L] basis table: C_i, S_i, C'_i) from its half record.
template <typename R, int L>
RBC_D void half_node_velocity(const R (&rec)[NodeRec<L>::HALF], int hf, const double* __restrict__ zb0,
                              const double* __restrict__ zb1, double (&u0)[3], double (&u1)[3])
{
    constexpr int LH = NodeRec<L>::LH;
    double a0 = 0, b0 = 0, c0 = 0, a1 = 0, b1 = 0, c1 = 0;
#pragma unroll
    for (int ii = 0; ii < LH; ++ii) {
        const int i = hf * LH + ii;
        if (i < L) { // the second half of an odd L has one mode less
            const double v11 = rec[5 * ii], v21 = rec[5 * ii + 1], v31 = rec[5 * ii + 2];
            const double v12 = rec[5 * ii + 3], v22 = rec[5 * ii + 4];
            const double C0 = __ldg(zb0 + i), S0 = __ldg(zb0 + L + i), D0 = __ldg(zb0 + 2 * L + i);
            const double C1 = __ldg(zb1 + i), S1 = __ldg(zb1 + L + i), D1 = __ldg(zb1 + 2 * L + i);
            a0 += D0 * v11 + S0 * v12;
            b0 += D0 * v21 + S0 * v22;
            c0 += C0 * v31;
            a1 += D1 * v11 + S1 * v12;
            b1 += D1 * v21 + S1 * v22;
            c1 += C1 * v31;
        }
    }
    u0[0] = a0; u0[1] = b0; u0[2] = c0;
    u1[0] = a1; u1[1] = b1; u1[2] = c1;
}

// Cell of (x, y, z) as the reference's vel_interpolate finds it, for the xy corner
// (q & 1, q >> 1): the corner's node, the two bracketing levels and the corner's trilinear
// weights.
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

// One team of 8 consecutive lanes per particle. The team's four corner records (the xy
// corners of the particle's cell) are copied into the team's slot of shared memory by all
// eight lanes together, 16 contiguous bytes per lane and copy (the two x-neighbours are
// adjacent records), so each copy instruction of a warp touches a few lines instead of one
// sector per lane. Lane (q, hf), q = lane & 3 the corner (q & 1, q >> 1) and hf = (lane >> 2)
// & 1 the record half, then evaluates its half of corner q's node velocity on the cell's
// two levels and keeps that share in registers: an RK stage that stays in the cell (the
// common case) only reweights the shares, and one that stays in the column re-evaluates
// them from shared memory. The 8 shares are summed with three shuffle rounds.
constexpr int kTracerThreads = 256;
template <typename R, int L> constexpr size_t tracer_smem()
{
    return (size_t)(kTracerThreads / 8) * 4 * NodeRec<L>::value * sizeof(R);
}

template <typename R, int L>
__global__ void __launch_bounds__(kTracerThreads) k_tracers(TracerArgs A)
{
    constexpr int NR = NodeRec<L>::value, HALF = NodeRec<L>::HALF;
    constexpr int CH = NR * (int)sizeof(R) / 16; // 16-byte chunks per record
    extern __shared__ __align__(16) unsigned char tr_smem[];
    const int gt = blockIdx.x * blockDim.x + threadIdx.x;
    const int t = gt >> 3, l8 = gt & 7, q = gt & 3, hf = (gt >> 2) & 1; // particle, team lane, corner, half
    R* slot = reinterpret_cast<R*>(tr_smem) + (size_t)(threadIdx.x >> 3) * 4 * NR; // the team's 4 records
    const bool live = t < A.n;                              // whole teams are live or not
    const int tt = live ? t : 0;
    double x = A.pos[tt], y = A.pos[A.n + tt], z = A.pos[2 * A.n + tt];
    int cell = -1, ev_iz = -1;
    double u0[3] = {0, 0, 0}, u1[3] = {0, 0, 0};
    const R* nv = reinterpret_cast<const R*>(A.nv);
    rk4_team(x, y, z, A.dt, [&](double px, double py, double pz, double& vx, double& vy, double& vz) {
        const Corner c = find_corner(A, q, px, py, pz);
        // the four corner nodes, gathered by the whole warp (the shuffles are outside the
        // branch below, which teams of one warp take differently); corner 0's node
        // identifies the cell (uniform over the team)
        const int n0 = __shfl_sync(0xffffffffu, c.node, 0, 4), n1 = __shfl_sync(0xffffffffu, c.node, 1, 4),
                  n2 = __shfl_sync(0xffffffffu, c.node, 2, 4), n3 = __shfl_sync(0xffffffffu, c.node, 3, 4);
        const bool load = n0 != cell;
        if (load) {
#pragma unroll
            for (int m = 0; m < (4 * CH + 7) / 8; ++m) {
                const int g = l8 + 8 * m;       // chunk g of the four records
                if (g < 4 * CH) {
                    const int cq = g / CH, part = g - cq * CH;
                    const int node = cq == 0 ? n0 : cq == 1 ? n1 : cq == 2 ? n2 : n3;
                    cp_async<16>(slot + cq * NR + part * (16 / (int)sizeof(R)),
                                 nv + (size_t)node * NR + part * (16 / (int)sizeof(R)));
                }
            }
            cell = n0;
        }
        cp_async_wait_all();
        __syncwarp();
        if (load || c.iz0 != ev_iz) {
            R rec[HALF];
            const R* src = slot + q * NR + hf * HALF;
#pragma unroll
            for (int e = 0; e < HALF; ++e) rec[e] = src[e];
            half_node_velocity<R, L>(rec, hf, A.zbasis + (size_t)c.iz0 * 3 * L, A.zbasis + (size_t)c.iz1 * 3 * L,
                                     u0, u1);
            ev_iz = c.iz0;
        }
        __syncwarp(); // the slot is rewritten by the next stage's copies only after every lane read it
        double v[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            v[d] = c.w * (c.wz0 * u0[d] + c.wz1 * u1[d]);
            v[d] += __shfl_xor_sync(0xffffffffu, v[d], 1, 8);
            v[d] += __shfl_xor_sync(0xffffffffu, v[d], 2, 8);
            v[d] += __shfl_xor_sync(0xffffffffu, v[d], 4, 8);
        }
        vx = v[0];
        vy = v[1];
        vz = v[2];
    });
    if (live && l8 == 0) finish_tracer(A, t, x, y, z);
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
