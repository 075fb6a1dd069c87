// gemm_tc.cuh -- BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a) for the
// surrogate network's products (no reference counterpart).
//
// C[z](m, n) = epilogue(alpha * sum_k A[z](m, k) B(k, n)) with the operand and output
// conventions of GemmOp (fno_kernels.cuh), for A whose rows are K-contiguous (load mode 2),
// one B for every z, N <= 256 and K <= 256. Persistent CTAs (two per SM where the TMEM and
// shared memory allow, else one) walk 128-row tiles with three roles:
//   - warp 0, one lane: the TMA producer. Each 128 x 64 chunk of A is one
//     cp.async.bulk.tensor load (128-byte swizzle, zero fill past M and K) into a ring of
//     kTcStages shared-memory stages, completing on the stage's "full" mbarrier;
//   - warp 1, one lane: the MMA issuer. Per chunk it waits for "full", issues up to four
//     tcgen05.mma kind::f16 (M = 128, N, K = 16; BF16 operands, FP32 accumulator in TMEM) and
//     commits them to the stage's "empty" mbarrier (the stage is reloaded when they are done);
//     per tile it accumulates into one of two TMEM accumulators (128 lanes x N columns each)
//     and commits the tile to that accumulator's "full" mbarrier;
//   - warps 2..9: the epilogue. Warp w reads the TMEM lanes 32 (w % 4) .. + 31 (its rows) of
//     half of the 16-column blocks with tcgen05.ld, applies the GemmOp epilogue, stores, and
//     releases the accumulator on its "empty" mbarrier, so that the MMAs of the next tile
//     overlap this epilogue.
// B^T is staged once per CTA by all threads in the same 128-byte-swizzled K-major layout.
// Every mbarrier wait is bounded (kMbarSpins polls); a wait that gives up sets an abort flag
// that ends every role's loop, RBC_DEVERR_TIMEOUT in *err, and the TMEM is freed on every path.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "common.cuh"
#include "fno_kernels.cuh"

namespace rbcfno {

constexpr int kTcM = 128, kTcKC = 64, kTcNmax = 256, kTcKmax = 256, kTcStages = 3;
constexpr int kTcEpiWarps = 8, kTcThreads = 32 * (2 + kTcEpiWarps);
constexpr unsigned kTcStageBytes = kTcM * kTcKC * 2; // one 128 x 64 BF16 chunk of A

struct TcArgs {
    GemmOp op;
    int* err;
    int mtiles, ntiles, nchunk, n16;
    int vec4; // 1: outputs and addends of a row contiguous, 16-byte aligned groups of 4
};

// Dynamic shared memory: alignment slack, the A stages, B^T (nchunk blocks of n16 x 128
// bytes), 4 + 2 kTcStages mbarriers, the TMEM address and the abort flag.
RBC_HD constexpr size_t gemm_tc_smem(int nchunk, int n16)
{
    return 1024 + (size_t)kTcStages * kTcStageBytes + (size_t)nchunk * n16 * 128 + (2 * kTcStages + 4) * 8 + 16;
}

// tcgen05 shared-memory matrix descriptor of a K-major operand in the 128-byte swizzle
// layout (8-row atoms of 128-byte rows, 1024 bytes apart): start address, leading offset
// (unused for this layout, 16 bytes), stride offset 1024, version 1 (bits 46-48 = 0b001),
// layout type 2 (128-byte swizzle) in bits 61-63.
RBC_D uint64_t umma_desc_sw128(unsigned smem_addr)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr & 0x3FFFF) >> 4);
    d |= (uint64_t)(16 >> 4) << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// Instruction descriptor of kind::f16: FP32 accumulator, BF16 A and B, both K-major,
// N >> 3 in bits 17-22, M >> 4 in bits 24-28.
RBC_HD constexpr uint32_t umma_idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

RBC_D void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
RBC_D void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Byte offset of element (r, k), k < 64, in a block of 8-row atoms with the 128-byte swizzle:
// 16-byte chunk k / 8 of row r sits at chunk (k / 8) ^ (r % 8).
RBC_HD unsigned sw128_off(int r, int k)
{
    return (unsigned)((r >> 3) * 1024 + (r & 7) * 128 + ((((k >> 3) ^ (r & 7)) & 7) << 4) + (k & 7) * 2);
}

RBC_D void tma_load_3d(void* smem_dst, const CUtensorMap* map, int c0, int c1, int c2, unsigned long long* mbar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
                 "[%5];\n" ::"r"(smem_u32(smem_dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(mbar))
                 : "memory");
}

RBC_D void tc_commit(unsigned long long* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

// Bounded wait that also gives up once another role has aborted.
RBC_D bool tc_wait(unsigned long long* mbar, unsigned parity, volatile int* abort_flag)
{
    const unsigned a = smem_u32(mbar);
    for (unsigned i = 0; i < kMbarSpins; ++i) {
        unsigned ok;
        asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
        if ((i & 1023) == 1023 && *abort_flag) return false;
    }
    *abort_flag = 1;
    return false;
}

// Epilogue of one accumulator value at (m, n), flat output offset o.
RBC_D void tc_epi1(const GemmOp& op, float v, long long o, int n)
{
    v *= op.alpha;
    if (op.bias) v += op.bias[n];
    if (op.add) v += op.add[o];
    if (op.pre) op.pre[o] = v;
    if (op.act == ACT_GELU) v = gelu(v);
    else if (op.act == ACT_GELU_BWD) v *= gelu_grad(op.aux[o]);
    if (op.outf) op.outf[o] = v;
    if (op.outb) op.outb[o] = __float2bfloat16_rn(v);
}

template <int NCOLS>
__global__ void __launch_bounds__(kTcThreads, 2) k_gemm_tc(const __grid_constant__ CUtensorMap tmA, TcArgs a)
{
    static_assert(NCOLS >= 32 && NCOLS <= 256 && (NCOLS & (NCOLS - 1)) == 0, "TMEM columns: power of two >= 32");
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    unsigned char* base = reinterpret_cast<unsigned char*>(((uintptr_t)tc_smem + 1023) & ~(uintptr_t)1023);
    const GemmOp& op = a.op;
    unsigned char* As = base;
    unsigned char* Bs = As + (size_t)kTcStages * kTcStageBytes;
    unsigned long long* full = reinterpret_cast<unsigned long long*>(Bs + (size_t)a.nchunk * a.n16 * 128);
    unsigned long long* empty = full + kTcStages;
    unsigned long long* accf = empty + kTcStages;
    unsigned long long* acce = accf + 2;
    unsigned* tslot = reinterpret_cast<unsigned*>(acce + 2);
    volatile int* abort_flag = reinterpret_cast<volatile int*>(tslot + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(2 * NCOLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 32) {
        for (int s = 0; s < kTcStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&accf[b], 1);
            mbar_init(&acce[b], kTcEpiWarps);
        }
        *abort_flag = 0;
        mbar_fence_init();
    }
    // B^T, once: element (n, k) = B[k b_rs + n b_cs] (consecutive threads, consecutive n)
    const int n16 = a.n16, K = op.K;
    const bf16 zero = __float2bfloat16_rn(0.0f);
    for (int i = threadIdx.x; i < a.nchunk * kTcKC * n16; i += blockDim.x) {
        const int k = i / n16, n = i - k * n16;
        const bf16 v = (n < op.N && k < K) ? op.B[(long long)k * op.b_rs + (long long)n * op.b_cs] : zero;
        *reinterpret_cast<bf16*>(Bs + (size_t)(k / kTcKC) * n16 * 128 + sw128_off(n, k % kTcKC)) = v;
    }
    fence_proxy_async_smem(); // the generic stores of B^T come before the MMAs read them
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const unsigned tmem = *tslot;

    if (warp == 0) {
        // ---- TMA producer
        if (lane == 0) {
            unsigned g = 0;
            for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x) {
                const int mt = t % a.mtiles, z = t / a.mtiles;
                for (int c = 0; c < a.nchunk; ++c, ++g) {
                    const int s = (int)(g % kTcStages);
                    if (!tc_wait(&empty[s], ((g / kTcStages) & 1) ^ 1, abort_flag)) goto roles_done;
                    mbar_arrive_expect_tx(&full[s], kTcStageBytes);
                    tma_load_3d(As + (size_t)s * kTcStageBytes, &tmA, c * kTcKC, mt * kTcM, z, &full[s]);
                }
            }
        }
    } else if (warp == 1) {
        // ---- MMA issuer
        if (lane == 0) {
            const uint32_t idesc = umma_idesc_bf16(kTcM, n16);
            unsigned g = 0, tl = 0;
            for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++tl) {
                const unsigned b = tl & 1;
                if (!tc_wait(&acce[b], ((tl >> 1) & 1) ^ 1, abort_flag)) goto roles_done;
                tc_fence_after();
                const unsigned dcol = tmem + b * NCOLS;
                for (int c = 0; c < a.nchunk; ++c, ++g) {
                    const int s = (int)(g % kTcStages);
                    if (!tc_wait(&full[s], (g / kTcStages) & 1, abort_flag)) goto roles_done;
                    tc_fence_after();
                    const int nk = min(kTcKC / 16, (K - c * kTcKC + 15) / 16);
                    const unsigned a0 = smem_u32(As + (size_t)s * kTcStageBytes);
                    const unsigned b0 = smem_u32(Bs + (size_t)c * n16 * 128);
                    for (int kk = 0; kk < nk; ++kk) {
                        // K = 16 is 32 bytes of the 128-byte swizzled rows
                        const uint64_t ad = umma_desc_sw128(a0 + kk * 32);
                        const uint64_t bd = umma_desc_sw128(b0 + kk * 32);
                        const unsigned acc = (c > 0 || kk > 0) ? 1u : 0u;
                        asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                                     "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(dcol),
                                     "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                                     : "memory");
                    }
                    tc_commit(&empty[s]); // the stage is free once these MMAs are done
                }
                tc_commit(&accf[b]); // the tile's accumulator is complete
            }
        }
    } else {
        // ---- epilogue: quadrant q of the TMEM lanes, every other 16-column block
        const int q = warp & 3, h = (warp - 2) >> 2;
        unsigned tl = 0;
        for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++tl) {
            const unsigned b = tl & 1;
            if (!tc_wait(&accf[b], (tl >> 1) & 1, abort_flag)) break;
            tc_fence_after();
            const int mt = t % a.mtiles, z = t / a.mtiles;
            const int m = mt * kTcM + q * 32 + lane;
            const long long rowo = (long long)z * op.c_bs + (long long)m * op.c_rs;
            for (int c0 = 16 * h; c0 < n16; c0 += 32) {
                uint32_t r[16];
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];\n"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                      "=r"(r[15])
                    : "r"(tmem + b * NCOLS + ((unsigned)(q * 32) << 16) + (unsigned)c0)
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
                if (m >= op.M) continue;
                if (a.vec4) {
                    // groups of 4 contiguous outputs (16-byte FP32 and 8-byte BF16 accesses); a
                    // group that crosses N falls back to single values
#pragma unroll
                    for (int g4 = 0; g4 < 4; ++g4) {
                        const int n = c0 + 4 * g4;
                        const long long o = rowo + n;
                        if (n + 4 > op.N) {
                            for (int e = 0; e < 4 && n + e < op.N; ++e) tc_epi1(op, __uint_as_float(r[4 * g4 + e]), o + e, n + e);
                            continue;
                        }
                        float v[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) v[e] = __uint_as_float(r[4 * g4 + e]) * op.alpha;
                        if (op.bias) {
                            const float4 bb = *reinterpret_cast<const float4*>(op.bias + n);
                            v[0] += bb.x; v[1] += bb.y; v[2] += bb.z; v[3] += bb.w;
                        }
                        if (op.add) {
                            const float4 ad = *reinterpret_cast<const float4*>(op.add + o);
                            v[0] += ad.x; v[1] += ad.y; v[2] += ad.z; v[3] += ad.w;
                        }
                        if (op.pre) *reinterpret_cast<float4*>(op.pre + o) = make_float4(v[0], v[1], v[2], v[3]);
                        if (op.act == ACT_GELU) {
#pragma unroll
                            for (int e = 0; e < 4; ++e) v[e] = gelu(v[e]);
                        } else if (op.act == ACT_GELU_BWD) {
                            const float4 ax = *reinterpret_cast<const float4*>(op.aux + o);
                            v[0] *= gelu_grad(ax.x); v[1] *= gelu_grad(ax.y); v[2] *= gelu_grad(ax.z); v[3] *= gelu_grad(ax.w);
                        }
                        if (op.outf) *reinterpret_cast<float4*>(op.outf + o) = make_float4(v[0], v[1], v[2], v[3]);
                        if (op.outb) {
                            __nv_bfloat162 lo = __floats2bfloat162_rn(v[0], v[1]), hi = __floats2bfloat162_rn(v[2], v[3]);
                            uint2 pk;
                            pk.x = *reinterpret_cast<unsigned*>(&lo);
                            pk.y = *reinterpret_cast<unsigned*>(&hi);
                            *reinterpret_cast<uint2*>(op.outb + o) = pk;
                        }
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 16; ++j) {
                        const int n = c0 + j;
                        if (n < op.N) tc_epi1(op, __uint_as_float(r[j]), rowo + (long long)n * op.c_cs, n);
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce[b]);
        }
    }
roles_done:
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && *abort_flag) atomicOr(a.err, RBC_DEVERR_TIMEOUT);
    if (warp == 0) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(2 * NCOLS) : "memory");
    }
}

} // namespace rbcfno
