// gemm_tc.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// surrogate network's products (no reference counterpart).
//
// C[z](m, n) = epilogue(alpha * sum_k A[z](m, k) B[z](k, n)) with the operand and output
// conventions of GemmOp (fno_kernels.cuh), for A whose rows are K-contiguous (load mode 2).
// One CTA of 128 threads computes a 128-row tile of C for all N <= 256 columns:
//   - per K chunk of 64, the threads copy the A tile (128 x 64) and the B^T tile (N x 64)
//     into shared memory in the canonical no-swizzle K-major layout of the MMA (core
//     matrices of 8 rows x 16 bytes; the next core matrix along K 128 bytes on, the next
//     8-row group KC/8 * 128 bytes on), zero-filled past M, N and K;
//   - one elected thread issues 4 tcgen05.mma kind::f16 (M = 128, N, K = 16; BF16 inputs,
//     FP32 accumulate) into a TMEM accumulator of 128 lanes x N columns and commits them to
//     an mbarrier, which the CTA waits on before the chunk's shared memory is reused;
//   - per 32 output columns, each warp reads its 32 rows of the accumulator with tcgen05.ld
//     (warp w owns TMEM lanes 32 w .. 32 w + 31) into a shared [128][33] tile, and the CTA
//     applies the epilogue of GemmOp walking the tile row by row, so that consecutive threads
//     read and write consecutive outputs.
// Every wait is bounded (kMbarSpins polls); a wait that gives up sets *err and the kernel
// still frees its TMEM. TMEM is allocated by warp 0 (power-of-two columns >= 32) and freed
// by warp 0 on every path.
#pragma once
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"
#include "fno_kernels.cuh"

namespace rbcfno {

constexpr int kTcM = 128, kTcKC = 64, kTcNmax = 256;

// Shared memory of k_gemm_tc for an N-column tile (N rounded up to 16).
RBC_HD constexpr size_t gemm_tc_smem(int n16)
{
    return (size_t)kTcM * kTcKC * 2 + (size_t)n16 * kTcKC * 2 + 16 /* mbarrier + TMEM address */ + 128 /* align */;
}

// tcgen05 shared-memory matrix descriptor, no swizzle: start address, leading (K-direction)
// and stride (8-row-group) byte offsets, descriptor version 1 (bits 46-48 = 0b001).
RBC_D uint64_t umma_desc(unsigned smem_addr, unsigned lbo, unsigned sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr & 0x3FFFF) >> 4);
    d |= (uint64_t)((lbo & 0x3FFFF) >> 4) << 16;
    d |= (uint64_t)((sbo & 0x3FFFF) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d; // base offset 0, relative LBO, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
RBC_HD constexpr uint32_t umma_idesc_bf16(int M, int N)
{
    return (1u << 4)                       // D format F32
           | (1u << 7)                     // A format BF16
           | (1u << 10)                    // B format BF16
           | ((uint32_t)(N >> 3) << 17)    // N
           | ((uint32_t)(M >> 4) << 24);   // M
}

RBC_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
RBC_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Element (r, k) of a row-major [rows][KC] tile in the canonical no-swizzle K-major layout:
// core matrix (r / 8, k / 8) at ((r / 8) (KC / 8) + k / 8) * 64 elements, row r % 8 of it at
// (r % 8) * 8, element k % 8.
RBC_HD int tc_off(int r, int k) { return ((r >> 3) * (kTcKC / 8) + (k >> 3)) * 64 + (r & 7) * 8 + (k & 7); }

template <int NCOLS>
__global__ void __launch_bounds__(128) k_gemm_tc(GemmOp op, int* err)
{
    static_assert(NCOLS >= 32 && NCOLS <= 256 && (NCOLS & (NCOLS - 1)) == 0, "TMEM columns: power of two >= 32");
    extern __shared__ __align__(128) unsigned char tc_smem[];
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)tc_smem + 127) & ~(uintptr_t)127);
    const int N16 = (op.N + 15) & ~15;
    bf16* As = reinterpret_cast<bf16*>(base);
    bf16* Bs = As + kTcM * kTcKC;
    unsigned long long* mbar = reinterpret_cast<unsigned long long*>(Bs + (size_t)N16 * kTcKC);
    unsigned* taddr_slot = reinterpret_cast<unsigned*>(mbar + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int z = blockIdx.z;
    const int m0 = blockIdx.x * kTcM;
    int K = op.K;
    if (op.ktot > 0) {
        const long long rem = op.ktot - (long long)z * op.K;
        K = rem < op.K ? (int)rem : op.K;
    }
    const bf16* A = op.A + z * op.a_bs;
    const bf16* B = op.B + z * op.b_bs;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(taddr_slot)),
                     "r"(NCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 0) {
        mbar_init(mbar, 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *taddr_slot;
    const uint32_t idesc = umma_idesc_bf16(kTcM, N16);
    const bf16 zero = __float2bfloat16_rn(0.0f);
    unsigned phase = 0;
    bool ok = true;
    for (int k0 = 0; k0 < K; k0 += kTcKC) {
        // K = 16 steps of this chunk that carry data (the rest of the chunk is not read)
        const int nk = min(kTcKC / 16, (K - k0 + 15) / 16), kw = 16 * nk;
        // A tile: row-major K-contiguous rows, 16-byte loads of 8 elements
        for (int i = threadIdx.x; i < kTcM * (kw / 8); i += blockDim.x) {
            const int r = i / (kw / 8), kc = (i - r * (kw / 8)) * 8;
            const int gr = m0 + r, gk = k0 + kc;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (gr < op.M && gk < K) {
                if (gk + 8 <= K) {
                    v = *reinterpret_cast<const uint4*>(A + gr * op.a_rs + gk);
                } else {
                    bf16* e = reinterpret_cast<bf16*>(&v);
                    for (int j = 0; j < 8; ++j) e[j] = gk + j < K ? A[gr * op.a_rs + gk + j] : zero;
                }
            }
            *reinterpret_cast<uint4*>(As + tc_off(r, kc)) = v;
        }
        // B^T tile: element (n, k) = B[k b_rs + n b_cs]; consecutive threads take
        // consecutive n (the weights' rows are n-contiguous)
        for (int i = threadIdx.x; i < N16 * kw; i += blockDim.x) {
            const int k = i / N16, n = i - k * N16;
            const int gk = k0 + k;
            Bs[tc_off(n, k)] = (n < op.N && gk < K) ? B[gk * op.b_rs + n * op.b_cs] : zero;
        }
        fence_proxy_async_smem(); // the generic stores above come before the MMAs read them
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (threadIdx.x == 0) {
            const unsigned a0 = smem_u32(As), b0 = smem_u32(Bs);
            for (int kk = 0; kk < nk; ++kk) {
                // K = 16 covers two core matrices along K (128 bytes apart): +256 bytes per step
                const uint64_t ad = umma_desc(a0 + kk * 256, 128, (kTcKC / 8) * 128);
                const uint64_t bd = umma_desc(b0 + kk * 256, 128, (kTcKC / 8) * 128);
                const unsigned acc = (k0 > 0 || kk > 0) ? 1u : 0u;
                asm volatile(
                    "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(mbar))
                         : "memory");
        }
        // the MMAs of this chunk are done (their shared memory may be rewritten)
        if (!mbar_wait_parity(mbar, phase)) ok = false;
        phase ^= 1;
        tc_fence_after();
        ok = __syncthreads_and(ok) != 0;
        if (!ok) break;
    }
    if (!ok) {
        // the commit of the last chunk did not arrive: flag it and give the MMAs one more
        // bounded wait before the accumulator is freed
        if (threadIdx.x == 0) atomicOr(err, RBC_DEVERR_TIMEOUT);
        mbar_wait_parity(mbar, phase ^ 1);
    }
    // epilogue, 32 columns at a time: each warp moves its 32 accumulator rows from TMEM into
    // a shared [128][33] tile (the A/B staging area, free now), then the CTA walks the tile in
    // row-major order so that consecutive threads touch consecutive outputs (and addends)
    float* T = reinterpret_cast<float*>(base);
    const long long cz = (long long)z * op.c_bs;
    const unsigned lane_base = (unsigned)(warp * 32) << 16;
    for (int c0 = 0; c0 < N16; c0 += 32) {
        const int cw = min(32, N16 - c0);
        if (ok && K > 0) {
            for (int h = 0; h < cw; h += 16) {
                uint32_t r[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15])
                    : "r"(tmem + lane_base + (unsigned)(c0 + h))
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
                for (int j = 0; j < 16; ++j) T[threadIdx.x * 33 + h + j] = __uint_as_float(r[j]);
            }
        } else {
            for (int j = 0; j < cw; ++j) T[threadIdx.x * 33 + j] = 0.0f; // an empty split-K slice
        }
        __syncthreads();
        for (int e = threadIdx.x; e < kTcM * cw; e += blockDim.x) {
            const int rr = e / cw, j = e - rr * cw;
            const int mm = m0 + rr, n = c0 + j;
            if (mm >= op.M || n >= op.N) continue;
            const long long o = cz + mm * op.c_rs + n * op.c_cs;
            float v = T[rr * 33 + j] * op.alpha;
            if (op.bias) v += op.bias[n];
            if (op.add) v += op.add[o];
            if (op.pre) op.pre[o] = v;
            if (op.act == ACT_GELU) v = gelu(v);
            else if (op.act == ACT_GELU_BWD) v *= gelu_grad(op.aux[o]);
            if (op.outf) op.outf[o] = v;
            if (op.outb) op.outb[o] = __float2bfloat16_rn(v);
        }
        __syncthreads();
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(NCOLS) : "memory");
    }
}

} // namespace rbcfno
