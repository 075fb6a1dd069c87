// fft.cuh -- batched complex FFTs staged in shared memory (sm_100a, FP64 or FP32).
//
// Lengths N = 2^a 3^b (N <= 1024) are done as a sequence of Stockham autosort passes
// with radix 4, 2 or 3. All threads of the CTA cooperate on `nb` transforms stored
// contiguously in ONE shared buffer [nb][N]: each pass reads its radix-R inputs into
// registers, synchronises, and writes the butterflies' outputs to their autosorted
// positions in the same buffer, so no ping-pong buffer is needed. Twiddles come from
// a per-length table tw[t] = exp(-2 pi i t / N) held in shared memory (conjugated for
// the inverse). Conventions match the reference's cuFFT use: forward e^{-i},
// inverse e^{+i}, both unnormalised.
#pragma once
#include "common.cuh"

namespace rbcfft {

struct Plan {
    int n;
    int npass;
    int radix[12];
};

inline Plan make_plan(int n)
{
    Plan p;
    p.n = n;
    p.npass = 0;
    int m = n;
    while (m % 4 == 0) { p.radix[p.npass++] = 4; m /= 4; }
    while (m % 2 == 0) { p.radix[p.npass++] = 2; m /= 2; }
    while (m % 3 == 0) { p.radix[p.npass++] = 3; m /= 3; }
    if (m != 1 || n < 2) p.npass = -1; // unsupported length
    return p;
}

template <int RAD, typename R>
RBC_D void dft_small(typename cplx_t<R>::type* v, int sign)
{
    typedef typename cplx_t<R>::type C;
    if (RAD == 2) {
        C a = v[0], b = v[1];
        v[0] = a + b;
        v[1] = a - b;
    } else if (RAD == 4) {
        C a0 = v[0] + v[2], a1 = v[0] - v[2];
        C b0 = v[1] + v[3], b1 = v[1] - v[3];
        C jb1 = cmul_is<C, R>(b1, (R)sign); // b1 * (sign i)
        v[0] = a0 + b0;
        v[2] = a0 - b0;
        v[1] = a1 + jb1;
        v[3] = a1 - jb1;
    } else if (RAD == 3) {
        const R c1 = (R)-0.5;
        const R s1 = (R)(sign * 0.86602540378443864676372317075294);
        C t = v[1] + v[2];
        C d = v[1] - v[2];
        C m = v[0] + t * c1;
        C jd = cmul_is<C, R>(d, s1);
        v[0] = v[0] + t;
        v[1] = m + jd;
        v[2] = m - jd;
    }
}

// One Stockham pass over nb transforms of length n in buf (in place, see header).
// Every thread handles at most MAXB butterflies (the caller guarantees
// nb * n / RAD <= MAXB * blockDim.x).
template <int RAD, int MAXB, typename R>
RBC_D void pass(typename cplx_t<R>::type* buf, int n, int ns, int nb,
                const typename cplx_t<R>::type* tw, int sign)
{
    typedef typename cplx_t<R>::type C;
    const int nbf = n / RAD;
    const int total = nb * nbf;
    const int twstep = n / (ns * RAD);
    C v[MAXB][RAD];
    int dst[MAXB];
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int w = threadIdx.x + b * blockDim.x;
        if (w < total) {
            const int t = w / nbf, j = w - t * nbf;
            const int k = j % ns;
            const C* src = buf + t * n;
#pragma unroll
            for (int r = 0; r < RAD; ++r) v[b][r] = src[j + r * nbf];
#pragma unroll
            for (int r = 1; r < RAD; ++r) {
                C w_ = tw[k * r * twstep];
                if (sign > 0) w_.y = -w_.y;
                v[b][r] = cmul(v[b][r], w_);
            }
            dft_small<RAD, R>(v[b], sign);
            dst[b] = t * n + (j - k) * RAD + k;
        }
    }
    __syncthreads();
#pragma unroll
    for (int b = 0; b < MAXB; ++b) {
        const int w = threadIdx.x + b * blockDim.x;
        if (w < total) {
#pragma unroll
            for (int r = 0; r < RAD; ++r) buf[dst[b] + r * ns] = v[b][r];
        }
    }
    __syncthreads();
}

// Run all passes of plan p on nb transforms in buf (shared memory). The caller must
// make buf and tw visible (a __syncthreads() before the call) and size the launch so
// that nb * n / 2 <= MAXB * blockDim.x.
template <int MAXB, typename R>
RBC_D void run(typename cplx_t<R>::type* buf, const Plan& p, int nb, const typename cplx_t<R>::type* tw, int sign)
{
    int ns = 1;
    for (int s = 0; s < p.npass; ++s) {
        const int r = p.radix[s];
        if (r == 4) pass<4, MAXB, R>(buf, p.n, ns, nb, tw, sign);
        else if (r == 2) pass<2, MAXB, R>(buf, p.n, ns, nb, tw, sign);
        else pass<3, MAXB, R>(buf, p.n, ns, nb, tw, sign);
        ns *= r;
    }
}

} // namespace rbcfft
