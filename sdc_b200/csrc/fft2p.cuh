// fft2p.cuh -- register-resident two-pass FFTs of length N = R * R (R = 8 or 16).
//
// One transform is done by R consecutive lanes of a warp (a quarter or half warp).
// With x[n], n = t + R a, the lane t holds v[a] = x[t + R a] on entry and
//   pass 1: v[k1] = sum_a x[t + R a] W_R^(a k1), times W_N^(t k1)  (registers)
//   transpose through the transform's own padded shared tile S[k1 (R + 1) + t]
//   pass 2: v[k2] = sum_t' S[t (R + 1) + t'] W_R^(t' k2)             (registers)
// so that on exit lane t holds X[t + R k2] in v[k2] (X[k] = sum_n x[n] W_N^(n k),
// W_N = exp(sign 2 pi i / N)). The tile is private to the transform, so the lanes only
// synchronise among themselves (__syncwarp on their own lane mask). Compared with the
// shared-memory Stockham passes of fft.cuh this drops two shared-memory round trips and
// every CTA-wide barrier of the transform itself.
#pragma once
#include "common.cuh"
#include "fft.cuh"

namespace rbcfft {

// Shared tile of one transform: R * (R + 1) elements. Odd row pitch R + 1 keeps the
// column reads of pass 2 free of bank conflicts.
template <int R> RBC_HD constexpr int tile_len() { return R * (R + 1); }

// Lane mask of the R lanes that share a transform with this lane.
template <int R> RBC_D unsigned team_mask()
{
    const unsigned lane = threadIdx.x & 31;
    const unsigned base = R == 32 ? 0xffffffffu : ((1u << R) - 1u);
    return base << (lane & ~(unsigned)(R - 1));
}

template <int R, typename Rt>
RBC_D void two_pass(typename cplx_t<Rt>::type (&v)[R], int t, typename cplx_t<Rt>::type* S,
                    const typename cplx_t<Rt>::type* tw, int sign)
{
    typedef typename cplx_t<Rt>::type C;
    dft_small<R, Rt>(v, sign);
#pragma unroll
    for (int k1 = 1; k1 < R; ++k1) {
        C w = tw[t * k1];                 // W_N^(t k1), t k1 < N
        if (sign > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    const unsigned m = team_mask<R>();
#pragma unroll
    for (int k1 = 0; k1 < R; ++k1) S[k1 * (R + 1) + t] = v[k1];
    __syncwarp(m);
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = S[t * (R + 1) + j];
    dft_small<R, Rt>(v, sign);
    __syncwarp(m); // the tile may be reused by the caller after this
}

// R for a length handled by two_pass (0: use the Stockham passes).
RBC_HD constexpr int two_pass_radix(int n) { return n == 256 ? 16 : n == 64 ? 8 : 0; }

} // namespace rbcfft
