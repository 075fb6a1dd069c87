// colloc_kernels.cuh -- the Galerkin state <-> collocation fields maps of the surrogate.
//
// Encode: theta, u, v, w at nq levels z_q from the synthesised fields of a step
//   (phys [8][L][Ny][Nx]: u11 = d_x f, u21 = d_y f, u31 = q^2 f, u12 = d_y g + F,
//   u22 = -d_x g + G, theta, theta_x, theta_y), with the velocity composition of
//   calculate_velocity_operator::compose_u_from_derivs
//   (gpu_flow/code/operator/calculate_velocity_operator.cu:426-455):
//     theta = sum S_m theta_m,  u = sum C'_m u11_m + S_m u12_m,
//     v = sum C'_m u21_m + S_m u22_m,  w = sum C_m u31_m.
// Decode (an increment d of the collocation fields onto the state): per point the
//   least-squares mode amplitudes Theta_m = Ps d_theta, W_m = Pc d_w, U_m = Ps d_u,
//   V_m = Ps d_v; a direct FP64 DFT of those planes; then per wavenumber
//     theta_m += Theta^_m / P,  f_m += W^_m / (q^2 P),
//     g_m += (i qx V^_m - i qy U^_m) / (q^2 P)   (vertical vorticity: the C' parts cancel),
//     F_m += U^_m(q=0) / P,  G_m += V^_m(q=0) / P,
//   on the kept (2/3) band only, the kx = 0 column mirrored as make_real does
//   (gpu_flow/code/util/util.cu:184-209). For fields in the span of the basis the
//   round trip state -> fields -> state is exact up to rounding.
#pragma once
#include "common.cuh"
#include "step_kernels.cuh"

namespace rbck {

// One thread per point; the block's [points][4 nq] output tile goes through shared memory
// (row stride 4 nq + 1) so that the channel-last rows are written with coalesced stores.
template <typename R, int L>
__global__ void __launch_bounds__(256) k_colloc_encode(const R* __restrict__ phys, int P, int nq,
                                                       const double* __restrict__ basis, float* __restrict__ out)
{
    extern __shared__ float tile[]; // [blockDim.x][4 nq + 1]
    const int C = 4 * nq, ld = C + 1;
    const int p0 = blockIdx.x * blockDim.x, p = p0 + threadIdx.x;
    if (p < P) {
        double u11[L], u21[L], u31[L], u12[L], u22[L], th[L];
#pragma unroll
        for (int m = 0; m < L; ++m) {
            u11[m] = phys[(size_t)(0 * L + m) * P + p];
            u21[m] = phys[(size_t)(1 * L + m) * P + p];
            u31[m] = phys[(size_t)(2 * L + m) * P + p];
            u12[m] = phys[(size_t)(3 * L + m) * P + p];
            u22[m] = phys[(size_t)(4 * L + m) * P + p];
            th[m] = phys[(size_t)(5 * L + m) * P + p];
        }
        float* o = tile + threadIdx.x * ld;
        for (int q = 0; q < nq; ++q) {
            const double* b = basis + (size_t)q * 3 * L; // C, C', S
            double t = 0, u = 0, v = 0, w = 0;
#pragma unroll
            for (int m = 0; m < L; ++m) {
                const double Cb = b[m], Cp = b[L + m], S = b[2 * L + m];
                t += S * th[m];
                u += Cp * u11[m] + S * u12[m];
                v += Cp * u21[m] + S * u22[m];
                w += Cb * u31[m];
            }
            o[q] = (float)t;
            o[nq + q] = (float)u;
            o[2 * nq + q] = (float)v;
            o[3 * nq + q] = (float)w;
        }
    }
    __syncthreads();
    const int np = min((int)blockDim.x, P - p0);
    for (int e = threadIdx.x; e < np * C; e += blockDim.x) {
        const int r = e / C, c = e - r * C;
        out[(size_t)p0 * C + e] = tile[r * ld + c];
    }
}

// planes [4][L][P]: Theta, W, U, V mode amplitudes of the increment at every point. The
// block's [points][4 nq] input tile is read with coalesced loads into shared memory first.
template <int L>
__global__ void __launch_bounds__(256) k_colloc_project(const float* __restrict__ delta, int P, int nq,
                                                        const double* __restrict__ proj, double* __restrict__ planes)
{
    extern __shared__ float tile[]; // [blockDim.x][4 nq + 1]
    const int C = 4 * nq, ld = C + 1;
    const int p0 = blockIdx.x * blockDim.x, p = p0 + threadIdx.x;
    const int np = min((int)blockDim.x, P - p0);
    for (int e = threadIdx.x; e < np * C; e += blockDim.x) {
        const int r = e / C, c = e - r * C;
        tile[r * ld + c] = delta[(size_t)p0 * C + e];
    }
    __syncthreads();
    if (p >= P) return;
    const float* d = tile + threadIdx.x * ld;
    const double *Ps = proj, *Pc = proj + (size_t)L * nq;
    double a[4][L];
#pragma unroll
    for (int m = 0; m < L; ++m) a[0][m] = a[1][m] = a[2][m] = a[3][m] = 0.0;
    for (int q = 0; q < nq; ++q) {
        const double t = d[q], u = d[nq + q], v = d[2 * nq + q], w = d[3 * nq + q];
#pragma unroll
        for (int m = 0; m < L; ++m) {
            const double sv = Ps[m * nq + q], cv = Pc[m * nq + q];
            a[0][m] += sv * t;
            a[1][m] += cv * w;
            a[2][m] += sv * u;
            a[3][m] += sv * v;
        }
    }
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int m = 0; m < L; ++m) planes[(size_t)(f * L + m) * P + p] = a[f][m];
}

// Direct DFT of each real row (plane, y) for the kept columns c < ckeep:
// out[(plane ckeep + c) Ny + y] = sum_x row[x] e^{-2 pi i c x / Nx}. Grid nplanes * Ny.
// Each thread owns one c and walks x in blocks of 8: the phase of the block start comes
// from the exact table, the 7 steps inside by multiplication with e^{-2 pi i c / Nx}, so the
// table is read once per 8 terms (rounding growth ~8 ulp) and the row is a broadcast.
__global__ void __launch_bounds__(128) k_colloc_row_dft(const double* __restrict__ planes, int nx, int ny, int ckeep,
                                                        const double2* __restrict__ twx, double2* __restrict__ out)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double* row = reinterpret_cast<double*>(tw + nx);
    const int rowid = blockIdx.x, plane = rowid / ny, y = rowid - plane * ny;
    const double* src = planes + (size_t)rowid * nx;
    for (int t = threadIdx.x; t < nx; t += blockDim.x) {
        tw[t] = twx[t];
        row[t] = src[t];
    }
    __syncthreads();
    for (int c = threadIdx.x; c < ckeep; c += blockDim.x) {
        const double2 st = tw[c];
        double re = 0, im = 0;
        for (int x0 = 0; x0 < nx; x0 += 8) {
            double2 w = tw[(int)(((long long)c * x0) % nx)];
            for (int x = x0; x < x0 + 8 && x < nx; ++x) {
                re += row[x] * w.x;
                im += row[x] * w.y;
                w = make_double2(w.x * st.x - w.y * st.y, w.x * st.y + w.y * st.x);
            }
        }
        out[((size_t)plane * ckeep + c) * ny + y] = make_double2(re, im);
    }
}

// Column DFT of the four increment planes of mode m and column c, then the update of
// the state. Grid (ckeep, L).
template <int L>
__global__ void __launch_bounds__(256) k_colloc_assemble(const double2* __restrict__ rows, Geom G,
                                                         const double2* __restrict__ twy, double2* __restrict__ th,
                                                         double2* __restrict__ f, double2* __restrict__ g,
                                                         double2* __restrict__ FG)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ny = G.ny, c = blockIdx.x, m = blockIdx.y;
    double2* tw = reinterpret_cast<double2*>(smem_raw);
    double2* col = tw + ny; // [4][ny]
    for (int t = threadIdx.x; t < ny; t += blockDim.x) {
        tw[t] = twy[t];
#pragma unroll
        for (int a = 0; a < 4; ++a) col[a * ny + t] = rows[((size_t)(a * L + m) * G.ckeep + c) * ny + t];
    }
    __syncthreads();
    const double inv = 1.0 / G.P;
    for (int r = threadIdx.x; r < ny; r += blockDim.x) {
        if (!row_kept(r, ny)) continue;
        // the kx = 0 column: rows 0 < r < Ny/2 mirror row Ny - r
        const bool mirror = c == 0 && r > 0 && r < ny / 2;
        const int rs = mirror ? ny - r : r;
        double2 s[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) s[a] = make_double2(0, 0);
        // phase of each block of 8 terms from the exact table, 7 rotations inside
        const double2 st = tw[rs];
        for (int y0 = 0; y0 < ny; y0 += 8) {
            double2 w = tw[(int)(((long long)rs * y0) % ny)];
            for (int y = y0; y < y0 + 8 && y < ny; ++y) {
#pragma unroll
                for (int a = 0; a < 4; ++a) {
                    const double2 v = col[a * ny + y];
                    s[a].x += v.x * w.x - v.y * w.y;
                    s[a].y += v.x * w.y + v.y * w.x;
                }
                w = make_double2(w.x * st.x - w.y * st.y, w.x * st.y + w.y * st.x);
            }
        }
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            s[a] = s[a] * inv;
            if (mirror) s[a].y = -s[a].y;
            if (c == 0 && r == 0) s[a].y = 0.0;
        }
        const size_t e = ((size_t)m * G.ckp + c) * ny + r;
        th[e] = th[e] + s[0];
        const Mult M(c, r, G);
        const double q2 = -M.lap;
        if (q2 > 0) {
            f[e] = f[e] + s[1] * (1.0 / q2);
            // i qx V - i qy U
            const double2 z = cmul_is<double2, double>(s[3], M.fx) - cmul_is<double2, double>(s[2], M.fy);
            g[e] = g[e] + z * (1.0 / q2);
        } else {
            FG[m] = FG[m] + make_double2(s[2].x, 0.0);
            FG[L + m] = FG[L + m] + make_double2(s[3].x, 0.0);
        }
    }
}

} // namespace rbck
