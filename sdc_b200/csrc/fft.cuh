// fft.cuh -- batched complex FFTs staged in shared memory (sm_100a, FP64 or FP32).
//
// Lengths N = 2^a 3^b (8 <= N <= 1024) run as Stockham autosort passes with radices
// 16, 8 and one leftover 4 or 2, then 3s, largest first: e.g. 256 = 16 x 16,
// 512 = 8 x 8 x 8, 192 = 8 x 8 x 3. Each thread does one radix-R butterfly per pass
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

// Factorisation with few passes and large radices: 16s, then 8s, and a single leftover
// radix (4, 2, 3, 6 -> 3 x 2, 12 -> 4 x 3 ...). Prefers 8 x 8 x 8 over 16 x 16 x 2 so
// that the smallest radix, which limits how many transforms a CTA can batch, stays big.
inline Plan make_plan(int n)
{
    Plan p;
    p.n = n;
    p.stride = padded_len(n);
    p.npass = 0;
    int m = n;
    int twos = 0, threes = 0;
    while (m % 2 == 0) { m /= 2; ++twos; }
    while (m % 3 == 0) { m /= 3; ++threes; }
    if (m != 1 || n < 8) { p.npass = -1; p.chunk = 0; return p; }
    // powers of two as 16s and 8s (4 or 2 only when twos < 3)
    int n16 = 0, n8 = 0, rest2 = 0;
    if (twos >= 3) {
        switch (twos % 4) {
        case 0: n16 = twos / 4; break;
        case 1: n16 = (twos - 9) / 4; n8 = 3; if (twos < 9) { n16 = 0; n8 = 1; rest2 = twos - 3; } break; // 2^5 = 8 x 4
        case 2: n16 = (twos - 6) / 4; n8 = 2; if (twos < 6) { n16 = 0; n8 = 1; rest2 = twos - 3; } break;
        case 3: n16 = (twos - 3) / 4; n8 = 1; break;
        }
    } else {
        rest2 = twos;
    }
    for (int i = 0; i < n16; ++i) p.radix[p.npass++] = 16;
    for (int i = 0; i < n8; ++i) p.radix[p.npass++] = 8;
    if (rest2 == 2) p.radix[p.npass++] = 4;
    else if (rest2 == 1) p.radix[p.npass++] = 2;
    for (int i = 0; i < threes; ++i) p.radix[p.npass++] = 3;
    // put the largest radix first (stride-R writes of the first pass are padded)
    for (int a = 0; a < p.npass; ++a)
        for (int b = a + 1; b < p.npass; ++b)
            if (p.radix[b] > p.radix[a]) { int t = p.radix[a]; p.radix[a] = p.radix[b]; p.radix[b] = t; }
    int rmin = 1 << 30;
    for (int s2 = 0; s2 < p.npass; ++s2) rmin = p.radix[s2] < rmin ? p.radix[s2] : rmin;
    p.chunk = (kPlanThreads * rmin) / n;
    if (p.chunk < 1) p.npass = -1;
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
    } else if constexpr (RAD == 12) {
        // n = 3 n1 + n2: 4-point DFTs over n1 for each n2, twiddles W12^(n2 k1), 3-point
        // DFTs over n2; X[k1 + 4 k2] is the k2-th output of the k1-th 3-point DFT
        C y[3][4];
#pragma unroll
        for (int n2 = 0; n2 < 3; ++n2) {
            y[n2][0] = v[n2]; y[n2][1] = v[3 + n2]; y[n2][2] = v[6 + n2]; y[n2][3] = v[9 + n2];
            dft4<R>(y[n2][0], y[n2][1], y[n2][2], y[n2][3], sign);
        }
        const R c1 = (R)0.86602540378443864676, h = (R)0.5;
        y[1][1] = rot<C, R>(y[1][1], c1, s * h);    // W12^1
        y[1][2] = rot<C, R>(y[1][2], h, s * c1);    // W12^2
        y[1][3] = cmul_is<C, R>(y[1][3], s);        // W12^3
        y[2][1] = rot<C, R>(y[2][1], h, s * c1);    // W12^2
        y[2][2] = rot<C, R>(y[2][2], -h, s * c1);   // W12^4
        y[2][3] = y[2][3] * (R)-1;                  // W12^6
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) {
            C t3[3] = {y[0][k1], y[1][k1], y[2][k1]};
            dft_small<3, R>(t3, sign);
            v[k1] = t3[0];
            v[k1 + 4] = t3[1];
            v[k1 + 8] = t3[2];
        }
    } else if constexpr (RAD == 16) {
        // n = 4 m + q: 4-point DFTs over m in place (v[q], v[q+4], v[q+8], v[q+12] then
        // hold Y_q[k1 = 0..3]), twiddles W16^(q k1), 4-point DFTs over q for each k1;
        // X[k1 + 4 k2] ends up in v[4 k2 + k1] after the final register transpose.
#pragma unroll
        for (int q = 0; q < 4; ++q) dft4<R>(v[q], v[q + 4], v[q + 8], v[q + 12], sign);
        const R c1 = (R)0.92387953251128675613, s1 = (R)0.38268343236508977173;
        const R h = (R)0.70710678118654752440;
        v[5] = rot<C, R>(v[5], c1, s * s1);     // q=1 k1=1: W16^1
        v[9] = rot<C, R>(v[9], h, s * h);       // q=1 k1=2: W16^2
        v[13] = rot<C, R>(v[13], s1, s * c1);   // q=1 k1=3: W16^3
        v[6] = rot<C, R>(v[6], h, s * h);       // q=2 k1=1: W16^2
        v[10] = cmul_is<C, R>(v[10], s);        // q=2 k1=2: W16^4
        v[14] = rot<C, R>(v[14], -h, s * h);    // q=2 k1=3: W16^6
        v[7] = rot<C, R>(v[7], s1, s * c1);     // q=3 k1=1: W16^3
        v[11] = rot<C, R>(v[11], -h, s * h);    // q=3 k1=2: W16^6
        v[15] = rot<C, R>(v[15], -c1, -s * s1); // q=3 k1=3: W16^9
#pragma unroll
        for (int k1 = 0; k1 < 4; ++k1) dft4<R>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3], sign);
        // v[4 k1 + k2] holds X[k1 + 4 k2]: transpose the 4 x 4 block
        C t;
        t = v[1]; v[1] = v[4]; v[4] = t;
        t = v[2]; v[2] = v[8]; v[8] = t;
        t = v[3]; v[3] = v[12]; v[12] = t;
        t = v[6]; v[6] = v[9]; v[9] = t;
        t = v[7]; v[7] = v[13]; v[13] = t;
        t = v[11]; v[11] = v[14]; v[14] = t;
    }
}

// One Stockham pass over nb transforms (in place, see header); each thread handles up
// to MAXB butterflies.
// Not inlined: each radix gets its own register allocation instead of sharing the
// union of all radices' live ranges inside run().
template <int RAD, int MAXB, typename R>
__device__ __noinline__ void pass(typename cplx_t<R>::type* buf, const Plan& p, int ns, int nb,
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
        else if (r == 2) pass<2, 1, R>(buf, p, ns, nb, tw, sign);
        else pass<3, 1, R>(buf, p, ns, nb, tw, sign);
        ns *= r;
    }
}

} // namespace rbcfft
