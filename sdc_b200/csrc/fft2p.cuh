// fft2p.cuh -- register-resident FFTs: two passes for N = R * R (R = 8 or 16), for
// N = 128 = 8 x 16 (two_pass_wide) and for N = 192 = 12 x 16 (fft192), three for N = 512
// (16 x 16 x 2, one warp per transform; three_pass_512 below).
//
// One transform is done by R consecutive lanes of a warp (a quarter or half warp).
// With x[n], n = t + R a, the lane t holds v[a] = x[t + R a] on entry and
//   pass 1: v[k1] = sum_a x[t + R a] W_R^(a k1), times W_N^(t k1)  (registers)
//   transpose through the transform's own padded shared tile S[k1 (R + 1) + t] (R (R + 1)
//   elements; the odd row pitch keeps the column reads of pass 2 free of bank conflicts)
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

// Length 512 = 16 x 32 on a full warp. Lane t (< 32) holds v[a] = x[t + 32 a] (a < 16) on
// entry and v[m] = X[t + 32 m] on exit, the layout two_pass gives with R = 16 values per lane
// and 32 lanes. With t = t1 + 16 t0 (t1 < 16) and k = k1 + 16 (j2 + 2 m):
//   pass 1: Y[k1] = sum_a x[t + 32 a] W_16^(a k1), times W_512^(t k1)       (registers)
//   pass 2: the 2-point DFT over t0 between lanes t and t ^ 16; lane t0 = j2 keeps
//           P[k1] = (Y_t1[k1] + (-1)^j2 Y_(t1+16)[k1]) W_32^(t1 j2)        (shuffles)
//   pass 3: transpose through S[j2 272 + k1 17 + t1], so that lane k1 + 16 j2 holds P over
//           t1, and the 16-point DFT over t1 gives X[k1 + 16 j2 + 32 m] in v[m].
// S has 544 elements (tile_len_512); odd row pitch 17 keeps the transposed reads free of
// bank conflicts.
RBC_HD constexpr int tile_len_512() { return 2 * 16 * 17; }

template <typename Rt>
RBC_D void three_pass_512(typename cplx_t<Rt>::type (&v)[16], int t, typename cplx_t<Rt>::type* S,
                          const typename cplx_t<Rt>::type* tw, int sign)
{
    typedef typename cplx_t<Rt>::type C;
    dft_small<16, Rt>(v, sign);
#pragma unroll
    for (int k1 = 1; k1 < 16; ++k1) {
        C w = tw[t * k1];                 // W_512^(t k1), t k1 <= 465
        if (sign > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    const int t1 = t & 15, j2 = t >> 4;
    C w = tw[16 * t1];                    // W_32^t1, applied by the j2 = 1 lanes
    if (sign > 0) w.y = -w.y;
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
        C o;
        o.x = __shfl_xor_sync(0xffffffffu, v[k1].x, 16);
        o.y = __shfl_xor_sync(0xffffffffu, v[k1].y, 16);
        const C p = j2 ? cmul(o - v[k1], w) : v[k1] + o;
        S[j2 * 272 + k1 * 17 + t1] = p;
    }
    __syncwarp();
    const int k1 = t & 15;
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = S[j2 * 272 + k1 * 17 + i];
    dft_small<16, Rt>(v, sign);
    __syncwarp(); // the tile may be reused by the caller after this
}

// N = TL * VL with VL = 2 TL (128 = 8 x 16) on TL lanes: lane t holds v[a] = x[t + TL a]
// (a < VL) on entry and v[m] = X[t + TL m] on exit.
//   pass 1: v[k1] = sum_a x[t + TL a] W_VL^(a k1), times W_N^(t k1)          (registers)
//   transpose through S[k1 (TL + 1) + t]
//   pass 2: lane t does the TL-point DFTs of k1 = t and t + TL over t':
//           X[k1 + VL k2] = sum_t' S[k1 (TL + 1) + t'] W_TL^(t' k2), i.e. v[j + 2 k2] for
//           k1 = t + TL j.
template <int TL, typename Rt>
RBC_D void two_pass_wide(typename cplx_t<Rt>::type (&v)[2 * TL], int t, typename cplx_t<Rt>::type* S,
                         const typename cplx_t<Rt>::type* tw, int sign)
{
    typedef typename cplx_t<Rt>::type C;
    constexpr int VL = 2 * TL;
    dft_small<VL, Rt>(v, sign);
#pragma unroll
    for (int k1 = 1; k1 < VL; ++k1) {
        C w = tw[t * k1];                 // W_N^(t k1), t k1 < N
        if (sign > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    const unsigned m = team_mask<TL>();
#pragma unroll
    for (int k1 = 0; k1 < VL; ++k1) S[k1 * (TL + 1) + t] = v[k1];
    __syncwarp(m);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        C u[TL];
#pragma unroll
        for (int i = 0; i < TL; ++i) u[i] = S[(t + TL * j) * (TL + 1) + i];
        dft_small<TL, Rt>(u, sign);
#pragma unroll
        for (int k2 = 0; k2 < TL; ++k2) v[j + 2 * k2] = u[k2];
    }
    __syncwarp(m); // the tile may be reused by the caller after this
}

// Length 192 = 12 x 16 on 16 lanes: lane t holds v[a] = x[t + 16 a] (a < 12) on entry and
// v[m] = X[t + 16 m] on exit.
//   pass 1: v[k1] = sum_a x[t + 16 a] W_12^(a k1), times W_192^(t k1)        (registers)
//   transpose through S[k1 17 + t]
//   pass 2: lanes t < 12 do the 16-point DFT of column k1 = t over t':
//           X[k1 + 12 k2] = sum_t' S[k1 17 + t'] W_16^(t' k2)
//   the results go back through the tile in natural order (S[pad(k)]), from which every
//   lane reads its X[t + 16 m].
// S has 204 elements (12 x 17; pad(191) = 202).
template <typename Rt>
RBC_D void fft192(typename cplx_t<Rt>::type (&v)[12], int t, typename cplx_t<Rt>::type* S,
                  const typename cplx_t<Rt>::type* tw, int sign)
{
    typedef typename cplx_t<Rt>::type C;
    dft_small<12, Rt>(v, sign);
#pragma unroll
    for (int k1 = 1; k1 < 12; ++k1) {
        C w = tw[t * k1];                 // W_192^(t k1), t k1 <= 165
        if (sign > 0) w.y = -w.y;
        v[k1] = cmul(v[k1], w);
    }
    const unsigned m = team_mask<16>();
#pragma unroll
    for (int k1 = 0; k1 < 12; ++k1) S[k1 * 17 + t] = v[k1];
    __syncwarp(m);
    C u[16];
    if (t < 12) {
#pragma unroll
        for (int i = 0; i < 16; ++i) u[i] = S[t * 17 + i];
        dft_small<16, Rt>(u, sign);
    }
    __syncwarp(m); // every column is read before the tile takes the results
    if (t < 12) {
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) S[pad(t + 12 * k2)] = u[k2];
    }
    __syncwarp(m);
#pragma unroll
    for (int i = 0; i < 12; ++i) v[i] = S[pad(t + 16 * i)];
    __syncwarp(m); // the tile may be reused by the caller after this
}

// Lanes per transform of the register FFT for length n (0: use the Stockham passes),
// and the shared tile one transform needs.
RBC_HD constexpr int reg_fft_lanes(int n)
{
    return n == 512 ? 32 : n == 256 ? 16 : n == 192 ? 16 : n == 128 ? 8 : n == 64 ? 8 : 0;
}
RBC_HD constexpr int reg_tile_len(int n)
{
    return n == 512 ? tile_len_512() : n == 192 ? 12 * 17 : (n / reg_fft_lanes(n)) * (reg_fft_lanes(n) + 1);
}

// The register FFT of length N done by TL = reg_fft_lanes(N) lanes, each holding
// VL = N / TL values: v[a] = x[t + TL a] on entry, v[k] = X[t + TL k] on exit.
template <int N, typename Rt>
RBC_D void reg_fft(typename cplx_t<Rt>::type (&v)[N / reg_fft_lanes(N)], int t, typename cplx_t<Rt>::type* S,
                   const typename cplx_t<Rt>::type* tw, int sign)
{
    constexpr int TL = reg_fft_lanes(N);
    if constexpr (N == 512) three_pass_512<Rt>(v, t, S, tw, sign);
    else if constexpr (N == 192) fft192<Rt>(v, t, S, tw, sign);
    else if constexpr (N == 2 * TL * TL) two_pass_wide<TL, Rt>(v, t, S, tw, sign);
    else two_pass<TL, Rt>(v, t, S, tw, sign);
}

} // namespace rbcfft
