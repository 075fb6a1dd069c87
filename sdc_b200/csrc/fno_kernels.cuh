// fno_kernels.cuh -- kernels of the Fourier neural operator surrogate (no reference
// counterpart): BF16 tensor-core GEMMs with FP32 accumulation and fused epilogues, the
// complex per-mode channel mixing of the spectral layers (forward and backward), and the
// reductions, loss and Adam update of training.
//
// Every contraction of the network is a GEMM: the pointwise channel maps, and the
// truncated real DFTs of the spectral layers written as products with fixed DFT
// matrices. Their K and N are small (32..256) and their operands stream from HBM, so
// the GEMMs are bandwidth-bound; mma.sync m16n8k16 BF16 tiles fed from shared memory
// reach that bound.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "splitmix.h"

namespace rbcfno {

typedef __nv_bfloat16 bf16;

enum { ACT_NONE = 0, ACT_GELU = 1, ACT_GELU_BWD = 2 };

// C[z](m, n) = epilogue(alpha * sum_k A[z](m, k) B[z](k, n)), z < batch.
// Element (m, k) of A[z] at A[z a_bs + m a_rs + k a_cs]; (k, n) of B[z] at
// B[z b_bs + k b_rs + n b_cs]; (m, n) of every output/addend at z c_bs + m c_rs + n c_cs.
// ktot > 0: split-K form, batch z covers k in [z K, min((z+1) K, ktot)) of ONE product
// (the A/B batch strides step along k), each z writing its own output slice.
struct GemmOp {
    const bf16* A = nullptr;
    long long a_rs = 0, a_cs = 0, a_bs = 0;
    const bf16* B = nullptr;
    long long b_rs = 0, b_cs = 0, b_bs = 0;
    int M = 0, N = 0, K = 0, batch = 1;
    long long ktot = 0;
    long long c_rs = 0, c_cs = 1, c_bs = 0;
    float alpha = 1.0f;
    const float* bias = nullptr; // [N]
    const float* add = nullptr;  // FP32 addend
    const float* aux = nullptr;  // FP32 pre-activation for ACT_GELU_BWD
    float* pre = nullptr;        // FP32 value before the activation
    float* outf = nullptr;       // FP32 output
    bf16* outb = nullptr;        // BF16 output (round to nearest even)
    int act = ACT_NONE;
    int amode = 0, bmode = 0;    // tile load modes (set by the host, see load_tile)
    int vec2 = 0;                // 1: outputs/addends of columns n, n+1 are adjacent and 8-byte
                                 //    aligned (c_cs == 1, c_rs and c_bs even, N even)
};

constexpr int kBK = 32, kSK = kBK + 8; // k tile and padded shared row (80 bytes)

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Load modes: 0 scalar, k fastest; 1 scalar, row fastest; 2 eight contiguous k per
// 16-byte load (cs == 1, rs % 8 == 0, K % 8 == 0, aligned base); 3 eight contiguous rows
// per 16-byte load (rs == 1, cs % 8 == 0, R % 8 == 0, aligned base).
// Fills S[r][k] (row stride kSK) for rows r0.. r0+ROWS, k0.. k0+kBK; zeros outside R x K.
template <int ROWS, int NT>
__device__ __forceinline__ void load_tile(bf16* S, const bf16* __restrict__ X, long long rs, long long cs, int r0,
                                          int k0, int R, int K, int mode)
{
    const bf16 zero = __float2bfloat16_rn(0.0f);
    if (mode == 2) {
        for (int i = threadIdx.x; i < ROWS * (kBK / 8); i += NT) {
            const int r = i / (kBK / 8), kc = (i - r * (kBK / 8)) * 8;
            const int gr = r0 + r, gk = k0 + kc;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gr < R && gk < K) v = *reinterpret_cast<const uint4*>(X + gr * rs + gk);
            *reinterpret_cast<uint4*>(S + r * kSK + kc) = v;
        }
    } else if (mode == 3) {
        for (int i = threadIdx.x; i < (ROWS / 8) * kBK; i += NT) {
            const int k = i / (ROWS / 8), rc = (i - k * (ROWS / 8)) * 8;
            const int gr = r0 + rc, gk = k0 + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gr < R && gk < K) v = *reinterpret_cast<const uint4*>(X + gk * cs + gr);
            const bf16* e = reinterpret_cast<const bf16*>(&v);
#pragma unroll
            for (int j = 0; j < 8; ++j) S[(rc + j) * kSK + k] = e[j];
        }
    } else if (mode == 1) {
        for (int i = threadIdx.x; i < ROWS * kBK; i += NT) {
            const int k = i / ROWS, r = i - k * ROWS;
            const int gr = r0 + r, gk = k0 + k;
            S[r * kSK + k] = (gr < R && gk < K) ? X[gr * rs + gk * cs] : zero;
        }
    } else {
        for (int i = threadIdx.x; i < ROWS * kBK; i += NT) {
            const int r = i / kBK, k = i - r * kBK;
            const int gr = r0 + r, gk = k0 + k;
            S[r * kSK + k] = (gr < R && gk < K) ? X[gr * rs + gk * cs] : zero;
        }
    }
}

__device__ __forceinline__ void mma_bf16(float* c, const uint32_t* a, const uint32_t* b)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};\n"
                 : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// BM x BN tile per CTA of 4 warps (2 x 2), each warp (BM/2) x (BN/2) = MT x NT mma tiles.
template <int BM, int BN>
__global__ void __launch_bounds__(128) k_gemm(GemmOp op)
{
    constexpr int MT = BM / 32, NT = BN / 16;
    __shared__ __align__(16) bf16 As[BM * kSK];
    __shared__ __align__(16) bf16 Bs[BN * kSK];
    const int z = blockIdx.z;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    int K = op.K;
    if (op.ktot > 0) {
        const long long rem = op.ktot - (long long)z * op.K;
        K = rem < op.K ? (int)rem : op.K;
    }
    const bf16* A = op.A + z * op.a_bs;
    const bf16* B = op.B + z * op.b_bs;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp >> 1, wn = warp & 1, gq = lane >> 2, tq = lane & 3;
    float acc[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.0f;
    for (int k0 = 0; k0 < K; k0 += kBK) {
        load_tile<BM, 128>(As, A, op.a_rs, op.a_cs, m0, k0, op.M, K, op.amode);
        // B tile stored n-major: Bs[n][k]; element (n, k) of B^T at B[n b_cs + k b_rs]
        load_tile<BN, 128>(Bs, B, op.b_cs, op.b_rs, n0, k0, op.N, K, op.bmode);
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 16) {
            uint32_t af[MT][4], bfr[NT][2];
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const bf16* p = As + (wm * (BM / 2) + i * 16 + gq) * kSK + kk + 2 * tq;
                af[i][0] = *reinterpret_cast<const uint32_t*>(p);
                af[i][1] = *reinterpret_cast<const uint32_t*>(p + 8 * kSK);
                af[i][2] = *reinterpret_cast<const uint32_t*>(p + 8);
                af[i][3] = *reinterpret_cast<const uint32_t*>(p + 8 * kSK + 8);
            }
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const bf16* p = Bs + (wn * (BN / 2) + j * 8 + gq) * kSK + kk + 2 * tq;
                bfr[j][0] = *reinterpret_cast<const uint32_t*>(p);
                bfr[j][1] = *reinterpret_cast<const uint32_t*>(p + 8);
            }
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j) mma_bf16(acc[i][j], af[i], bfr[j]);
        }
        __syncthreads();
    }
    const long long cz = (long long)z * op.c_bs;
    auto epi = [&](float v, long long o, int n) -> float {
        v *= op.alpha;
        if (op.bias) v += op.bias[n];
        if (op.add) v += op.add[o];
        if (op.pre) op.pre[o] = v;
        if (op.act == ACT_GELU) v = gelu(v);
        else if (op.act == ACT_GELU_BWD) v *= gelu_grad(op.aux[o]);
        return v;
    };
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j)
#pragma unroll
            for (int h2 = 0; h2 < 2; ++h2) {
                const int m = m0 + wm * (BM / 2) + i * 16 + gq + h2 * 8;
                const int n = n0 + wn * (BN / 2) + j * 8 + 2 * tq;
                if (m >= op.M || n >= op.N) continue;
                const long long o = cz + m * op.c_rs + n * op.c_cs;
                if (op.vec2) {
                    // columns n, n + 1 together: 8-byte FP32 and 4-byte BF16 accesses
                    float2 v = make_float2(acc[i][j][2 * h2] * op.alpha, acc[i][j][2 * h2 + 1] * op.alpha);
                    if (op.bias) { v.x += op.bias[n]; v.y += op.bias[n + 1]; }
                    if (op.add) { const float2 a = *reinterpret_cast<const float2*>(op.add + o); v.x += a.x; v.y += a.y; }
                    if (op.pre) *reinterpret_cast<float2*>(op.pre + o) = v;
                    if (op.act == ACT_GELU) { v.x = gelu(v.x); v.y = gelu(v.y); }
                    else if (op.act == ACT_GELU_BWD) {
                        const float2 a = *reinterpret_cast<const float2*>(op.aux + o);
                        v.x *= gelu_grad(a.x);
                        v.y *= gelu_grad(a.y);
                    }
                    if (op.outf) *reinterpret_cast<float2*>(op.outf + o) = v;
                    if (op.outb) *reinterpret_cast<__nv_bfloat162*>(op.outb + o) = __floats2bfloat162_rn(v.x, v.y);
                } else {
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        if (n + e >= op.N) continue;
                        const long long oe = o + e * op.c_cs;
                        const float v = epi(acc[i][j][2 * h2 + e], oe, n + e);
                        if (op.outf) op.outf[oe] = v;
                        if (op.outb) op.outb[oe] = __float2bfloat16_rn(v);
                    }
                }
            }
}

// Split-K finish: out(m, n) = sum of the nsplit FP32 slices [s][M][N] (in order), stored
// as FP32 and/or BF16 at z c_bs + m c_rs + n c_cs of a one-batch GEMM.
__global__ void k_splitk_finish(const float* __restrict__ part, int nsplit, int M, int N, long long c_rs,
                                long long c_cs, float* __restrict__ outf, bf16* __restrict__ outb)
{
    const long long mn = (long long)M * N;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < mn; i += (long long)gridDim.x * blockDim.x) {
        float v = 0.0f;
        for (int s = 0; s < nsplit; ++s) v += part[s * mn + i];
        const int m = (int)(i / N), n = (int)(i - (long long)m * N);
        const long long o = m * c_rs + n * c_cs;
        if (outf) outf[o] = v;
        if (outb) outb[o] = __float2bfloat16_rn(v);
    }
}

// Spectral channel mixing, one CTA per retained mode (ky index, kx):
// Y[b][ky][ri][kx][o] = sum_i X[b][ky][.][kx][i] (x) R[ky][kx][.][i][o]  (complex),
// X, Y BF16 with the (re, im) planes of a mode W apart and 2 m W apart in the row;
// R BF16 [nmode][2][W][W]. FP32 accumulation.
__global__ void __launch_bounds__(128) k_modemix_fwd(const bf16* __restrict__ X, const bf16* __restrict__ R,
                                                     bf16* __restrict__ Y, int nb, int mx, int width)
{
    extern __shared__ __align__(16) float sh[];
    const int W = width, W2 = W * W;
    float* rr = sh;        // [W][W] real
    float* ri = rr + W2;   // [W][W] imaginary
    float* xv = ri + W2;   // [nj][2][W]
    const int mode = blockIdx.x, ky = mode / mx, kx = mode - ky * mx;
    const int nrow = 2 * (gridDim.x / mx);   // (ky, ri) rows per batch entry
    const long long row = (long long)mx * W; // length of one row
    const bf16* Rm = R + (size_t)mode * 2 * W2;
    for (int t = threadIdx.x; t < W2; t += blockDim.x) {
        rr[t] = __bfloat162float(Rm[t]);
        ri[t] = __bfloat162float(Rm[W2 + t]);
    }
    const int nj = blockDim.x / W, o = threadIdx.x % W, j = threadIdx.x / W;
    for (int b0 = 0; b0 < nb; b0 += nj) {
        __syncthreads();
        for (int t = threadIdx.x; t < nj * 2 * W; t += blockDim.x) {
            const int jj = t / (2 * W), rem = t - jj * 2 * W, part = rem / W, i = rem - part * W;
            const int b = b0 + jj;
            xv[t] = b < nb ? __bfloat162float(X[((long long)b * nrow + 2 * ky + part) * row + kx * W + i]) : 0.0f;
        }
        __syncthreads();
        const int b = b0 + j;
        if (j < nj && b < nb) {
            const float* xr = xv + j * 2 * W;
            const float* xi = xr + W;
            float yr = 0.0f, yi = 0.0f;
            for (int i = 0; i < W; ++i) {
                const float a = xr[i], c = xi[i], p = rr[i * W + o], q = ri[i * W + o];
                yr += a * p - c * q;
                yi += a * q + c * p;
            }
            const long long base = ((long long)b * nrow + 2 * ky) * row + kx * W + o;
            Y[base] = __float2bfloat16_rn(yr);
            Y[base + row] = __float2bfloat16_rn(yi);
        }
    }
}

// Backward of k_modemix_fwd for one mode: dX (BF16) and dR (FP32, summed over the batch
// in order). dY, X in the layout of Y, X above.
__global__ void __launch_bounds__(256) k_modemix_bwd(const bf16* __restrict__ X, const bf16* __restrict__ R,
                                                     const bf16* __restrict__ dY, bf16* __restrict__ dX,
                                                     float* __restrict__ dR, int nb, int mx, int width)
{
    extern __shared__ __align__(16) float sh[];
    const int W = width, W2 = W * W;
    float* rtr = sh;          // R^T real [o][i]
    float* rti = rtr + W2;    // R^T imag
    float* xv = rti + W2;     // [2][W] X of batch b
    float* gv = xv + 2 * W;   // [2][W] dY of batch b
    const int mode = blockIdx.x, ky = mode / mx, kx = mode - ky * mx;
    const int nky2 = gridDim.x / mx * 2; // rows (ky, ri) per batch entry
    const bf16* Rm = R + (size_t)mode * 2 * W2;
    for (int t = threadIdx.x; t < W2; t += blockDim.x) {
        const int i = t / W, o = t - i * W;
        rtr[o * W + i] = __bfloat162float(Rm[t]);
        rti[o * W + i] = __bfloat162float(Rm[W2 + t]);
    }
    const long long row = (long long)mx * W;
    // dR accumulators: this thread's (i, o) pairs t = threadIdx.x + 256 s
    constexpr int kMaxPairs = 16; // W <= 64
    float accr[kMaxPairs], acci[kMaxPairs];
#pragma unroll
    for (int s = 0; s < kMaxPairs; ++s) accr[s] = acci[s] = 0.0f;
    for (int b = 0; b < nb; ++b) {
        __syncthreads();
        const long long base = ((long long)b * nky2 + 2 * ky) * row + kx * W;
        for (int t = threadIdx.x; t < 2 * W; t += blockDim.x) {
            const int part = t / W, i = t - part * W;
            xv[t] = __bfloat162float(X[base + part * row + i]);
            gv[t] = __bfloat162float(dY[base + part * row + i]);
        }
        __syncthreads();
#pragma unroll
        for (int s = 0; s < kMaxPairs; ++s) {
            const int t = threadIdx.x + 256 * s;
            if (t < W2) {
                const int i = t / W, o = t - i * W;
                const float ar = xv[i], ai = xv[W + i], gr = gv[o], gi = gv[W + o];
                accr[s] += gr * ar + gi * ai;
                acci[s] += -gr * ai + gi * ar;
            }
        }
        if (threadIdx.x < W) {
            const int i = threadIdx.x;
            float dr = 0.0f, di = 0.0f;
            for (int o = 0; o < W; ++o) {
                const float p = rtr[o * W + i], q = rti[o * W + i], gr = gv[o], gi = gv[W + o];
                dr += gr * p + gi * q;
                di += -gr * q + gi * p;
            }
            dX[base + i] = __float2bfloat16_rn(dr);
            dX[base + row + i] = __float2bfloat16_rn(di);
        }
    }
    float* dRm = dR + (size_t)mode * 2 * W2;
#pragma unroll
    for (int s = 0; s < kMaxPairs; ++s) {
        const int t = threadIdx.x + 256 * s;
        if (t < W2) {
            dRm[t] = accr[s];
            dRm[W2 + t] = acci[s];
        }
    }
}

__global__ void k_cast_bf16(const float* __restrict__ src, bf16* __restrict__ dst, long long n)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = __float2bfloat16_rn(src[i]);
}

// Partial column sums of a BF16 [M][N] matrix: part[blockIdx.x][n] over the block's rows.
__global__ void __launch_bounds__(256) k_colsum_part(const bf16* __restrict__ X, long long M, int N,
                                                     long long rows_per_block, float* __restrict__ part)
{
    __shared__ float red[256];
    const int per = blockDim.x / N; // rows handled side by side
    const int c = threadIdx.x % N, j = threadIdx.x / N;
    const long long r0 = blockIdx.x * rows_per_block;
    long long r1 = r0 + rows_per_block;
    if (r1 > M) r1 = M;
    float s = 0.0f;
    if (j < per)
        for (long long r = r0 + j; r < r1; r += per) s += __bfloat162float(X[r * N + c]);
    red[threadIdx.x] = s;
    __syncthreads();
    if (threadIdx.x < N) {
        float t = 0.0f;
        for (int q = 0; q < per; ++q) t += red[q * N + threadIdx.x];
        part[(size_t)blockIdx.x * N + threadIdx.x] = t;
    }
}

// out[j] (+)= sum_s in[s n + j]. Block (32, 32): lane x owns column j of its 32-column
// chunk, row y sums slices y, y + 32, ... in order, then the 32 row sums are added in a
// fixed tree: the result does not depend on scheduling.
__global__ void __launch_bounds__(1024) k_sum_slices(const float* __restrict__ in, int nslices, long long n,
                                                     float* __restrict__ out, int accumulate)
{
    __shared__ float red[32][33];
    const long long j = (long long)blockIdx.x * 32 + threadIdx.x;
    float s = 0.0f;
    if (j < n)
        for (int q = threadIdx.y; q < nslices; q += 32) s += in[q * n + j];
    red[threadIdx.y][threadIdx.x] = s;
    __syncthreads();
    for (int w = 16; w > 0; w >>= 1) {
        if (threadIdx.y < w) red[threadIdx.y][threadIdx.x] += red[threadIdx.y + w][threadIdx.x];
        __syncthreads();
    }
    if (threadIdx.y == 0 && j < n) out[j] = accumulate ? out[j] + red[0][threadIdx.x] : red[0][threadIdx.x];
}

// Mean-squared-error loss: per-block partial sums of (y - t)^2 (part[blockIdx.x]) and the
// BF16 gradient 2 (y - t) / n.
__global__ void __launch_bounds__(256) k_mse(const float* __restrict__ y, const float* __restrict__ t, long long n,
                                             bf16* __restrict__ g, float* __restrict__ part)
{
    __shared__ float red[256];
    float s = 0.0f;
    const float sc = 2.0f / (float)n;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float d = y[i] - t[i];
        s += d * d;
        g[i] = __float2bfloat16_rn(sc * d);
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = red[0];
}

// loss[idx] = sum(part[0..np)) / n in FP64, in order.
__global__ void k_loss_final(const float* __restrict__ part, int np, long long n, double* __restrict__ loss, int idx)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < np; ++i) s += part[i];
        loss[idx] = s / (double)n;
    }
}

// Adam (Kingma & Ba 2015) with bias correction; lr given per launch.
__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       long long n, float lr, float b1, float b2, float eps, float c1, float c2)
{
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// x (FP32 [M][C]) -> BF16 (x - mean[c]) * inv_std[c].
__global__ void k_normalize(const float* __restrict__ x, long long M, int C, const float* __restrict__ mean,
                            const float* __restrict__ inv_std, bf16* __restrict__ out)
{
    const long long n = M * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        out[i] = __float2bfloat16_rn((x[i] - mean[c]) * inv_std[c]);
    }
}

// delta = y std[c] + mean[c] (FP32 [M][C]).
__global__ void k_denormalize(const float* __restrict__ y, long long M, int C, const float* __restrict__ mean,
                              const float* __restrict__ stdv, float* __restrict__ out)
{
    const long long n = M * C;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(i % C);
        out[i] = y[i] * stdv[c] + mean[c];
    }
}

// Training batch from the snapshot store. Snapshots are FP32 [nslot][ny][nx][C] with
// channel field * nq + level, fields theta, u, v, w. Batch entry b reads snapshots
// a_slot[b] and z_slot[b] through the horizontal symmetry sym[b] of the periodic box
// (bit 0: transpose x <-> y, square boxes only; bit 1: x -> -x; bit 2: y -> -y);
// velocities transform as vectors: with M the point map, u_out(p) = M^T u_in(M p), i.e.
// (fx v, fy u) under the transpose and (fx u, fy v) otherwise, fx, fy = -1 for a flipped
// direction. The input state is s = a (+ the network's denormalized prediction pred[i]
// when use_pred[b]: the pushforward input), plus e = noise_rel * std of the channel's
// increment * N(0,1) (SplitMix64 + Box-Muller on element index i with seed nseed;
// noise_rel = 0: no noise). x = normalized s (BF16); target = normalized increment z - s
// (not written when target is null).
__global__ void k_gather_slots(const float* __restrict__ store, int nx, int ny, int nq,
                               const int* __restrict__ a_slot, const int* __restrict__ z_slot,
                               const int* __restrict__ sym, const int* __restrict__ use_pred,
                               const float* __restrict__ pred, int nb, const float* __restrict__ xm,
                               const float* __restrict__ xis, const float* __restrict__ dm,
                               const float* __restrict__ ds, const float* __restrict__ dis, float noise_rel,
                               unsigned long long nseed, bf16* __restrict__ x, float* __restrict__ target)
{
    const int C = 4 * nq;
    const long long snap = (long long)nx * ny * C;
    const long long n = (long long)nb * snap;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(i / snap);
        const long long e = i - (long long)b * snap;
        const int c = (int)(e % C);
        const long long p = e / C;
        const int y = (int)(p / nx), xx = (int)(p - (long long)y * nx);
        const int sy = sym ? sym[b] : 0;
        const int y1 = (sy & 4) ? (ny - y) % ny : y, x1 = (sy & 2) ? (nx - xx) % nx : xx;
        const int ys = (sy & 1) ? x1 : y1, xs = (sy & 1) ? y1 : x1;
        const int fo = c / nq, q = c - fo * nq;
        int fi = fo;
        float sgn = 1.0f;
        if (fo == 1) { fi = (sy & 1) ? 2 : 1; sgn = (sy & 2) ? -1.0f : 1.0f; }
        else if (fo == 2) { fi = (sy & 1) ? 1 : 2; sgn = (sy & 4) ? -1.0f : 1.0f; }
        const long long es = ((long long)ys * nx + xs) * C + fi * nq + q;
        float a = sgn * store[(long long)a_slot[b] * snap + es];
        if (pred && use_pred[b]) a += pred[i] * ds[c] + dm[c];
        float a_in = a;
        if (noise_rel > 0.0f) {
            const double u1 = rbcrng::unit_open(rbcrng::stream_at(nseed, 2 * (uint64_t)i));
            const double u2 = rbcrng::unit_open(rbcrng::stream_at(nseed, 2 * (uint64_t)i + 1));
            const double g = cos(6.283185307179586 * u2) * sqrt(-2.0 * log(u1));
            a_in = a + (float)(noise_rel * ds[c] * g);
        }
        x[i] = __float2bfloat16_rn((a_in - xm[c]) * xis[c]);
        if (target) {
            const float z = sgn * store[(long long)z_slot[b] * snap + es];
            target[i] = ((z - a_in) - dm[c]) * dis[c];
        }
    }
}

// Per-channel sums over the pairs for the normalization: part[blockIdx.x][4][C] =
// (sum x, sum x^2, sum d, sum d^2) over the block's rows (rows of [npairs * P][C]).
__global__ void __launch_bounds__(256) k_pair_stats(const float* __restrict__ store, long long P, int C,
                                                    const int* __restrict__ src, const int* __restrict__ dst,
                                                    int npairs, long long rows_per_block, double* __restrict__ part)
{
    __shared__ double red[4][256];
    const int per = blockDim.x / C;
    const int c = threadIdx.x % C, j = threadIdx.x / C;
    const long long total = (long long)npairs * P;
    const long long r0 = blockIdx.x * rows_per_block;
    long long r1 = r0 + rows_per_block;
    if (r1 > total) r1 = total;
    double s0 = 0, s1 = 0, s2 = 0, s3 = 0;
    if (j < per)
        for (long long r = r0 + j; r < r1; r += per) {
            const int pr = (int)(r / P);
            const long long p = r - (long long)pr * P;
            const double a = store[((long long)src[pr] * P + p) * C + c];
            const double d = store[((long long)dst[pr] * P + p) * C + c] - (float)a;
            s0 += a;
            s1 += a * a;
            s2 += d;
            s3 += d * d;
        }
    red[0][threadIdx.x] = s0;
    red[1][threadIdx.x] = s1;
    red[2][threadIdx.x] = s2;
    red[3][threadIdx.x] = s3;
    __syncthreads();
    if (threadIdx.x < C)
        for (int k = 0; k < 4; ++k) {
            double t = 0;
            for (int q = 0; q < per; ++q) t += red[k][q * C + threadIdx.x];
            part[((size_t)blockIdx.x * 4 + k) * C + threadIdx.x] = t;
        }
}

} // namespace rbcfno
