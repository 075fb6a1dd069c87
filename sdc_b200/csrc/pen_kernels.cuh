// pen_kernels.cuh -- penalized parts of the nonlinear operator (the reference's PENALIZED
// builds: make rectangle / circle / diskarray, nonlinear_operator_rayleigh_noslip.cu:1097-1335).
//
// For every vertical mode j the reference transforms mask * u_j / P for the six per-mode
// synthesis fields u11, u21, u31, u12, u22, theta and adds derivatives of those spectra to
// f, F, G and theta of the output modes k with Galerkin weights (Iac, Ia2) and the factor
// Pr / eta. All of it is linear in mask * u, so here it is added in physical space to the
// contracted groups before their forward transforms, with the group's own multiplier doing
// the derivative (scaling -1/(P Pr) for f, -1/P for theta, as for the products):
//   group 3 (d_x) of k  += mask sum_j [Iac(j,k) u11_j + Ia2(k,j) u12_j + Ia2(j,k) u21_j] Pr/eta
//   group 4 (d_y) of k  += mask sum_j [Iac(j,k) u21_j + Ia2(k,j) u22_j - Ia2(j,k) u11_j] Pr/eta
//                          + mask (u12_k - u22_k) Pr / (2 eta)
//   group 7 (lap) of k  -= mask u31_k Pr/eta
//   group 12 (theta) of k += mask theta_k / (2 eta)
// Group 4 carries the reference's four "g" summands, which it adds to f (with d_y in the
// fourth). F and G receive the means (q = 0 entries) of mask * u:
//   F_k += [sum_j Ia2(j,k) <mask u11_j> - <mask u12_k> / 2] / eta, G alike with u21, u22,
// through per-CTA partial sums (k_penalize) reduced in a fixed order (k_penalize_fg).
#pragma once
#include "common.cuh"

namespace rbck {

constexpr int kPenThreads = 256;

// Coefficients: cf[(g * L + k) * 4 L + f * L + j] for g = 0 (group 3), 1 (group 4) and the
// fields f = 0 u11, 1 u21, 2 u12, 3 u22 (synthesis fields 0, 1, 3, 4).
// partial[b * 4 L + f * L + j] = sum over CTA b's points of mask * u_f,j.
template <typename R, int L>
__global__ void __launch_bounds__(kPenThreads) k_penalize(const R* __restrict__ phys, R* __restrict__ grp,
                                                          const double* __restrict__ mask,
                                                          const double* __restrict__ cf, int P, double pe,
                                                          double theta_fac, double* __restrict__ partial)
{
    __shared__ double scf[2 * L * 4 * L];
    __shared__ double red[kPenThreads / 32][4 * L];
    pdl_trigger();
    for (int i = threadIdx.x; i < 2 * L * 4 * L; i += blockDim.x) scf[i] = cf[i];
    pdl_wait(); // the contraction is complete
    __syncthreads();
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const double m = p < P ? mask[p] : 0.0;
    double v[4][L];
    const size_t sP = (size_t)P;
    const int fidx[4] = {0, 1, 3, 4};
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int j = 0; j < L; ++j) v[f][j] = m != 0.0 ? (double)ld_cg(phys + ((size_t)fidx[f] * L + j) * sP + p) : 0.0;
    if (m != 0.0) {
        // modes in pairs: every load of a pair is issued before its stores
        constexpr int KB = L < 2 ? L : 2;
#pragma unroll
        for (int k0 = 0; k0 < L; k0 += KB) {
            double u31[KB], th[KB], g[4][KB];
            const int gid[4] = {3, 4, 7, 12};
#pragma unroll
            for (int kk = 0; kk < KB; ++kk) {
                const int k = k0 + kk;
                if (k < L) {
                    u31[kk] = (double)ld_cg(phys + ((size_t)2 * L + k) * sP + p);
                    th[kk] = (double)ld_cg(phys + ((size_t)5 * L + k) * sP + p);
#pragma unroll
                    for (int q = 0; q < 4; ++q) g[q][kk] = (double)ld_cg(grp + ((size_t)gid[q] * L + k) * sP + p);
                }
            }
#pragma unroll
            for (int kk = 0; kk < KB; ++kk) {
                const int k = k0 + kk;
                if (k < L) {
                    double a3 = 0.0, a4 = 0.0;
#pragma unroll
                    for (int f = 0; f < 4; ++f)
#pragma unroll
                        for (int j = 0; j < L; ++j) {
                            a3 += scf[(0 * L + k) * 4 * L + f * L + j] * v[f][j];
                            a4 += scf[(1 * L + k) * 4 * L + f * L + j] * v[f][j];
                        }
                    grp[((size_t)3 * L + k) * sP + p] = (R)(g[0][kk] + m * a3);
                    grp[((size_t)4 * L + k) * sP + p] = (R)(g[1][kk] + m * a4);
                    grp[((size_t)7 * L + k) * sP + p] = (R)(g[2][kk] - m * pe * u31[kk]);
                    grp[((size_t)12 * L + k) * sP + p] = (R)(g[3][kk] + m * theta_fac * th[kk]);
                }
            }
        }
    }
    // fixed-order block sums of mask * u for the means of F and G
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int f = 0; f < 4; ++f)
#pragma unroll
        for (int j = 0; j < L; ++j) {
            double x = m * v[f][j];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) red[warp][f * L + j] = x;
        }
    __syncthreads();
    for (int t = threadIdx.x; t < 4 * L; t += blockDim.x) {
        double s = 0.0;
        for (int w = 0; w < kPenThreads / 32; ++w) s += red[w][t];
        partial[(size_t)blockIdx.x * 4 * L + t] = s;
    }
}

// After the column pass has written NFG (F of mode k at k, G at L + k): adds the
// penalized means. One CTA of kPenFgThreads; warp w sums the partials of values
// w, w + 32, ... (lane l takes blocks l, l + 32, ..., then a fixed shuffle tree);
// ia2[j + k L] = Ia2(j, k); inv = 1 / (eta P).
constexpr int kPenFgThreads = 1024;
template <int L>
__global__ void __launch_bounds__(kPenFgThreads) k_penalize_fg(const double* __restrict__ partial, int nblocks,
                                                               const double* __restrict__ ia2, double inv,
                                                               double* __restrict__ NFG)
{
    __shared__ double S[4 * L];
    pdl_trigger();
    pdl_wait(); // the column pass has written NFG
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    for (int t = warp; t < 4 * L; t += nwarp) {
        double s = 0.0;
#pragma unroll 8
        for (int b = lane; b < nblocks; b += 32) s += ld_cg(partial + (size_t)b * 4 * L + t);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) S[t] = s;
    }
    __syncthreads();
    if (threadIdx.x < L) {
        const int k = threadIdx.x;
        double f = -0.5 * S[2 * L + k], g = -0.5 * S[3 * L + k];
        for (int j = 0; j < L; ++j) {
            f += ia2[j + k * L] * S[0 * L + j];
            g += ia2[j + k * L] * S[1 * L + j];
        }
        NFG[k] = ld_cg(NFG + k) + f * inv;
        NFG[L + k] = ld_cg(NFG + L + k) + g * inv;
    }
}

} // namespace rbck
