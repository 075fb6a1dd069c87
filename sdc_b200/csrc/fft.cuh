// fft.cuh -- batched complex FFTs staged in shared memory (sm_100a, FP64 or FP32).
//
// Lengths N = 2^a 3^b (8 <= N <= 1024) run as Stockham autosort passes whose first
// radix is 16 (or 8) and whose later radices are 16, 8, 4, 2 or 3, e.g. 256 = 16 x 16,
// 512 = 16 x 16 x 2, 192 = 16 x 4 x 3. Each thread does one radix-R butterfly per pass
// in registers (the 8- and 16-point DFTs are split into radix-2/4 steps with constant
// twiddles). All threads of the CTA cooperate on `nb` transforms held in ONE shared
// buffer: a pass reads its inputs to registers, synchronises, then writes the outputs
// to their autosorted positions in the same buffer. Element i of transform t lives at
// t * stride + i + i/16 (one pad slot per 16): the first pass writes with stride R,
// which the padding turns into an odd stride, so no pass has shared-memory bank
// conflicts. Twiddles tw[t] = exp(-2 pi i t / N) come from a shared table (conjugated
// for the inverse). Conventions match the reference's cuFFT use: forward e^{-i},
// inverse e^{+i}, both unnormalised.
#pragma once
#include "common.cuh"

namespace rbcfft {

struct Plan {
    int n;
    int stride; // padded length of one transform in the buffer
    int chunk;  // transforms per CTA-wide call (all passes fit kPlanThreads threads)
    int npass;
    int radix[12];
};

constexpr int kPlanThreads = 256;

RBC_HD int pad(int i) { return i + (i >> 4); }
RBC_HD int padded_len(int n) { return n + (n >> 4) + 1; }

inline Plan make_plan(int n)
{
    Plan p;
    p.n = n;
    p.stride = padded_len(n);
    p.npass = 0;
    int m = n;
    if (m % 16 == 0) { p.radix[p.npass++] = 16; m /= 16; }
    else if (m % 8 == 0) { p.radix[p.npass++] = 8; m /= 8; }
    while (m % 16 == 0) { p.radix[p.npass++] = 16; m /= 16; }
    while (m % 8 == 0) { p.radix[p.npass++] = 8; m /= 8; }
    while (m % 4 == 0) { p.radix[p.npass++] = 4; m /= 4; }
    while (m % 2 == 0) { p.radix[p.npass++] = 2; m /= 2; }
    while (m % 3 == 0) { p.radix[p.npass++] = 3; m /= 3; }
    if (m != 1 || n < 8) p.npass = -1; // unsupported length
    // every pass must fit the CTA: radix >= 4 one butterfly per thread, radix 2 and 3
    // up to two (MAXB in run()); the smallest such "butterfly width" sets the chunk
    int eff = 1 << 30;
    for (int s = 0; s < p.npass; ++s) {
        const int r = p.radix[s];
        const int e = r >= 4 ? r : 2 * r;
        eff = e < eff ? e : eff;
    }
    p.chunk = p.npass > 0 ? (kPlanThreads * eff) / n : 0;
    if (p.npass > 0 && p.chunk < 1) p.npass = -1;
    return p;
}

template <typename C, typename R> RBC_D C rot(C a, R c, R s) // a * (c + i s)
{
    C r;
    r.x = a.x * c - a.y * s;
    r.y = a.x * s + a.y * c;
    return r;
}

template <typename R> RBC_D void dft2(typename cplx_t<R>::type& a, typename cplx_t<R>::type& b)
{
    typename cplx_t<R>::type t = a;
    a = t + b;
    b = t - b;
}

template <typename R>
RBC_D void dft4(typename cplx_t<R>::type& v0, typename cplx_t<R>::type& v1, typename cplx_t<R>::type& v2,
                typename cplx_t<R>::type& v3, int sign)
{
    typedef typename cplx_t<R>::type C;
    C a0 = v0 + v2, a1 = v0 - v2, b0 = v1 + v3, b1 = v1 - v3;
    C jb1 = cmul_is<C, R>(b1, (R)sign);
    v0 = a0 + b0;
    v2 = a0 - b0;
    v1 = a1 + jb1;
    v3 = a1 - jb1;
}

template <int RAD, typename R>
RBC_D void dft_small(typename cplx_t<R>::type* v, int sign)
{
    typedef typename cplx_t<R>::type C;
    const R s = (R)sign;
    if constexpr (RAD == 2) {
        dft2<R>(v[0], v[1]);
    } else if constexpr (RAD == 3) {
        const R c1 = (R)-0.5;
        const R s1 = (R)(sign * 0.86602540378443864676372317075294);
        C t = v[1] + v[2], d = v[1] - v[2];
        C m = v[0] + t * c1;
        C jd = cmul_is<C, R>(d, s1);
        v[0] = v[0] + t;
        v[1] = m + jd;
        v[2] = m - jd;
    } else if constexpr (RAD == 4) {
        dft4<R>(v[0], v[1], v[2], v[3], sign);
    } else if constexpr (RAD == 8) {
        // even/odd split: X[k] = E[k] + W8^k O[k], X[k+4] = E[k] - W8^k O[k]
        C e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        C o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<R>(e0, e1, e2, e3, sign);
        dft4<R>(o0, o1, o2, o3, sign);
        const R h = (R)0.70710678118654752440084436210485;
        o1 = rot<C, R>(o1, h, s * h);
        o2 = cmul_is<C, R>(o2, s);
        o3 = rot<C, R>(o3, -h, s * h);
        v[0] = e0 + o0; v[4] = e0 - o0;
        v[1] = e1 + o1; v[5] = e1 - o1;
        v[2] = e2 + o2; v[6] = e2 - o2;
        v[3] = e3 + o3; v[7] = e3 - o3;
    } else if constexpr (RAD == 16) {
        // n = 4 m + q: four 4-point DFTs over m, twiddles W16^(q k1), then 4-point DFTs over q
        C y[4][4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            y[q][0] = v[q]; y[q][1] = v[q + 4]; y[q][2] = v[q + 8]; y[q][3] = v[q + 12];
            dft4<R>(y[q][0], y[q][1], y[q][2], y[q][3], sign);
        }
        const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;
        const R h = (R)0.70710678118654752440;
        // q = 1: W16^k1, k1 = 1..3
        y[1][1] = rot<C, R>(y[1][1], c1, s * s1);
        y[1][2] = rot<C, R>(y[1][2], h, s * h);
        y[1][3] = rot<C, R>(y[1][3], s1, s * c1);
        // q = 2: W16^(2 k1) = W8^k1
        y[2][1] = rot<C, R>(y[2][1], h, s * h);
        y[2][2] = cmul_is<C, R>(y[2][2], s);
        y[2][3] = rot<C, R>(y[2][3], -h, s * h);
        // q = 3: W16^(3 k1): e = 3, 6, 9
        y[3][1] = rot<C, R>(y[3][1], s1, s * c1);
        y[3][2] = rot<C, R>(y[3][2], -h, s * h);
        y[3][3] = rot<C, R>(y[3][3], -c1, -s * s1);
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            C a = y[0][k1], b = y[1][k1], c = y[2][k1], d = y[3][k1];
            dft4<R>(a, b, c, d, sign);
            v[k1] = a; v[k1 + 4] = b; v[k1 + 8] = c; v[k1 + 12] = d;
        }
    }
}

// One Stockham pass over nb transforms (in place, see header); each thread handles up
// to MAXB butterflies.
template <int RAD, int MAXB, typename R>
RBC_D void pass(typename cplx_t<R>::type* buf, const Plan& p, int ns, int nb,
                const typename cplx_t<R>::type* tw, int sign)
{
    typedef typename cplx_t<R>::type C;
    const int n = p.n;
    const int nbf = n / RAD;
    const int total = nb * nbf;
    const int twstep = n / (ns * RAD);
    C v[MAXB][RAD];
    int tt[MAXB], i0[MAXB];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int w = threadIdx.x + b * blockDim.x;
        if (w < total) {
            const int t = w / nbf, j = w - t * nbf;
            const int k = j % ns;
            const C* src = buf + t * p.stride;
#pragma unroll
            for (int r = 0; r < RAD; ++r) v[b][r] = src[pad(j + r * nbf)];
            if (ns > 1) {
#pragma unroll
                for (int r = 1; r < RAD; ++r) {
                    C w_ = tw[k * r * twstep];
                    if (sign > 0) w_.y = -w_.y;
                    v[b][r] = cmul(v[b][r], w_);
                }
            }
            dft_small<RAD, R>(v[b], sign);
            tt[b] = t;
            i0[b] = (j - k) * RAD + k;
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int w = threadIdx.x + b * blockDim.x;
        if (w < total) {
            C* out = buf + tt[b] * p.stride;
#pragma unroll
            for (int r = 0; r < RAD; ++r) out[pad(i0[b] + r * ns)] = v[b][r];
        }
    }
    __syncthreads();
}

// Runs all passes of plan p on nb transforms in buf (caller has synchronised).
template <typename R>
RBC_D void run(typename cplx_t<R>::type* buf, const Plan& p, int nb, const typename cplx_t<R>::type* tw, int sign)
{
    int ns = 1;
    for (int s = 0; s < p.npass; ++s) {
        const int r = p.radix[s];
        if (r == 16) pass<16, 1, R>(buf, p, ns, nb, tw, sign);
        else if (r == 8) pass<8, 1, R>(buf, p, ns, nb, tw, sign);
        else if (r == 4) pass<4, 1, R>(buf, p, ns, nb, tw, sign);
        else if (r == 2) pass<2, 2, R>(buf, p, ns, nb, tw, sign);
        else pass<3, 2, R>(buf, p, ns, nb, tw, sign);
        ns *= r;
    }
}

} // namespace rbcfft
