// colloc_tc.cuh -- the collocation form's nonlinear contraction (sm_100a; tcgen05 + bulk copy).
//
// For every physical point x the 8 L synthesised mode values (FP32, the mixed form's
// phys [8][L][P]) are taken to the Q collocation levels z_q, multiplied there and projected
// back onto the L output modes of the 13 groups (colloc_prog.h):
//   1. mode -> level, on the tensor cores: per field f, S_f[x][(j, q)] = sum_i X_f[x][i]
//      phi_{kind j, i}(z_q) as one tcgen05.mma kind::tf32 product per field and K-step of 8
//      modes (M = 128 points, N = the field's kinds x Q levels padded to 16, FP32 accumulator
//      in TMEM). TF32 keeps 10 mantissa bits, so both operands are split, X = Xh + Xl with
//      Xh = X truncated to TF32 and Xl = X - Xh exact in FP32 (likewise the basis), and
//      three products Xh Bh + Xh Bl + Xl Bh recover FP32 accuracy (3xTF32). The basis
//      operands are built on the host in the tensor cores' shared-memory layout and brought
//      in once per CTA by one bulk asynchronous copy (cp.async.bulk, mbarrier completion);
//      the point operands are written by the threads that split them.
//   2. the 41 products of a level, on the CUDA cores, from the TMEM rows (tcgen05.ld; lane =
//      point), into the 16 projected pairs of the level;
//   3. level -> mode, on the CUDA cores: out[g][k] += w_q chi_{c,k}(z_q) G_{(g,c)}, FP32 FMAs
//      with the weighted basis read from shared memory. The rule is symmetric and every basis
//      function has a definite parity in z, so each level is taken with its mirror: the
//      products of both are folded into even and odd parts and each output mode takes the
//      part of its own parity (half the multiplies, and the part the exact integrals cancel
//      is never formed by cancelling large terms in FP32).
// A CTA of 256 threads takes 128-point tiles (persistent over tiles); warps w and w + 4 read
// the TMEM lanes of quadrant w % 4 (their points) and split the output modes in two halves.
// Thread 0 issues the tensor-core products and commits them to an mbarrier; every wait is
// bounded (kMbarSpins polls) and a wait that gives up ends the kernel with RBC_DEVERR_TIMEOUT
// in *err after freeing the TMEM.
#pragma once
#include <stdint.h>

#include "colloc_prog.h"
#include "common.cuh"
#include "contract_kernel.cuh"

namespace rbck {

constexpr int kColThreads = 256, kColM = 128, kColChunk = 4; // threads, points per tile, levels per TMEM read
// (levels are read as two neighbours and their two mirrors; Q is a multiple of 8)

// Shared-memory image and TMEM columns of the collocation contraction for L modes and Q
// levels (host and device).
struct CollocGeom {
    int L, Q, Kp, LH;       // modes, levels, K padded to 8 (tf32 MMA K), output modes per half
    int Lp;                 // modes padded to 4 (rows of the level -> mode table)
    int ncol[8], col0[8];   // TMEM columns of each field's product (N padded to 16) and its first
    int tcols;              // TMEM columns allocated (power of two >= 32)
    unsigned a_bytes;       // one point operand (128 x Kp TF32)
    unsigned b_off[8];      // offset of field f's basis operand (hi; lo follows at + b_half)
    unsigned b_half, b_bytes; // bytes of the hi (= lo) basis images; both
    unsigned proj_off;      // level -> mode table [NKIND][Q][Lp] FP32
    unsigned bar_off;       // mbarriers (2) + TMEM slot + abort word
    unsigned smem;          // total dynamic shared memory (before alignment slack)
};

RBC_HD CollocGeom colloc_geom(int L, int Q)
{
    CollocGeom g{};
    g.L = L;
    g.Q = Q;
    g.Kp = (L + 7) / 8 * 8;
    g.LH = (L + 1) / 2;
    g.Lp = (L + 3) / 4 * 4;
    g.a_bytes = (unsigned)(kColM * g.Kp * 4);
    int c = 0;
    unsigned bo = 0;
    for (int f = 0; f < 8; ++f) {
        g.ncol[f] = (rbccol::field_pairs(f) * Q + 15) / 16 * 16;
        g.col0[f] = c;
        c += g.ncol[f];
        g.b_off[f] = bo;
        bo += (unsigned)(g.ncol[f] * g.Kp * 4);
    }
    g.tcols = 32;
    while (g.tcols < c) g.tcols *= 2;
    g.b_half = bo;
    g.b_bytes = 2 * bo;
    const unsigned a_all = 16u * g.a_bytes; // 8 fields x (hi, lo)
    g.proj_off = a_all + g.b_bytes;
    g.bar_off = g.proj_off + (unsigned)(rbccol::NKIND * Q * g.Lp * 4);
    g.bar_off = (g.bar_off + 15) & ~15u;
    g.smem = g.bar_off + 32;
    return g;
}

// Byte offset of element (r, k) of a K-major operand in the tensor cores' no-swizzle
// layout: 8-row x 16-byte core matrices, the K neighbours 128 bytes apart (leading offset),
// the 8-row groups 128 Kp / 4 bytes apart (stride offset).
RBC_HD unsigned colloc_kmajor_off(int r, int k, int Kp)
{
    return (unsigned)((r >> 3) * (128 * (Kp / 4)) + (k >> 2) * 128 + (r & 7) * 16 + (k & 3) * 4);
}

// tcgen05 shared-memory descriptor of such an operand: start, leading offset 128, stride
// offset 128 Kp / 4, version 1 (bit 46), no swizzle (layout type 0).
RBC_D uint64_t colloc_desc(unsigned smem_addr, int Kp)
{
    uint64_t d = 0;
    d |= (uint64_t)((smem_addr & 0x3FFFF) >> 4);
    d |= (uint64_t)(128 >> 4) << 16;
    d |= (uint64_t)((128 * (Kp / 4)) >> 4) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor of kind::tf32: FP32 accumulator (bits 4-5 = 1), TF32 A and B
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 in bits 17-22, M >> 4 in bits 24-28.
RBC_HD constexpr uint32_t colloc_idesc_tf32(int M, int N)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

RBC_D float tf32_hi(float x) { return __uint_as_float(__float_as_uint(x) & 0xFFFFE000u); }

RBC_D void col_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
RBC_D void col_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// Bounded wait for the phase of an mbarrier; false once kMbarSpins polls have passed.
RBC_D bool col_wait(unsigned long long* mbar, unsigned parity)
{
    const unsigned a = smem_u32(mbar);
    for (unsigned i = 0; i < kMbarSpins; ++i) {
        unsigned ok;
        asm volatile("{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
                     : "=r"(ok)
                     : "r"(a), "r"(parity)
                     : "memory");
        if (ok) return true;
    }
    return false;
}

// TMEM -> registers: 2 consecutive 32-bit columns of this warp's 32 lanes at each of eight
// column addresses, and the wait for them in the same statement, so that the values are
// complete before the compiler may move or spill them.
RBC_D void col_ld2x8(const unsigned (&t)[8], float (&v)[8][2])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%16];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%2,%3}, [%17];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%4,%5}, [%18];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%6,%7}, [%19];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%8,%9}, [%20];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%10,%11}, [%21];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%12,%13}, [%22];\n"
                 "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%14,%15}, [%23];\n"
                 "tcgen05.wait::ld.sync.aligned;\n"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15])
                 : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7])
                 : "memory");
#pragma unroll
    for (int e = 0; e < 8; ++e) {
        v[e][0] = __uint_as_float(r[2 * e]);
        v[e][1] = __uint_as_float(r[2 * e + 1]);
    }
}

struct CollocArgs {
    const float* phys;      // [8][L][P] synthesised fields (FP32)
    float* grp;             // [13][L][P] contracted groups (FP32)
    float* nv;              // node records of the tracers, or null
    const long long* step_counter; // copied to step_copy when nv is not null (the tracer
    long long* step_copy;          // advance reads the copy; the update increments the counter)
    const float* bimg;      // basis operands, hi then lo, in the shared-memory image layout
    const float* proj;      // [NKIND][Q][Lp] w_q chi_{c,k}(z_q)
    int P, ntiles;
    int* err;
};

// Column of level 0 of synthesised pair P (pair (f, j) level q is column col0[f] + j Q + q).
template <int P> RBC_D unsigned colloc_pair_col(const int (&col0)[8], int Q)
{
    constexpr rbccol::SPair sp = rbccol::spair_at(P);
    constexpr int j = P - rbccol::field_first_pair(sp.field);
    return (unsigned)(col0[sp.field] + j * Q);
}
// TMEM reads of the levels q, q + 1 and their mirrors Q - 2 - q, Q - 1 - q of every
// synthesised pair: s[p] = {S(q), S(q + 1), S(Q - 2 - q), S(Q - 1 - q)}; four pairs per read.
template <int P>
RBC_D void colloc_load_pairs(unsigned trow, const int (&col0)[8], int Q, int q, float (&s)[rbccol::NSPAIR][kColChunk])
{
    static_assert(rbccol::NSPAIR % 4 == 0, "pairs are read four at a time");
    if constexpr (P < rbccol::NSPAIR) {
        const unsigned c0 = colloc_pair_col<P>(col0, Q), c1 = colloc_pair_col<P + 1>(col0, Q),
                       c2 = colloc_pair_col<P + 2>(col0, Q), c3 = colloc_pair_col<P + 3>(col0, Q);
        const unsigned lo = trow + (unsigned)q, hi = trow + (unsigned)(Q - 2 - q);
        const unsigned t[8] = {lo + c0, hi + c0, lo + c1, hi + c1, lo + c2, hi + c2, lo + c3, hi + c3};
        float v[8][2];
        col_ld2x8(t, v);
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            s[P + e][0] = v[2 * e][0];
            s[P + e][1] = v[2 * e][1];
            s[P + e][2] = v[2 * e + 1][0];
            s[P + e][3] = v[2 * e + 1][1];
        }
        colloc_load_pairs<P + 4>(trow, col0, Q, q, s);
    }
}

// The 41 products of one level (column `c` of s), into its 16 projected pairs.
template <int N>
RBC_D void colloc_products(const float (&s)[rbccol::NSPAIR][kColChunk], int c, float (&G)[rbccol::NPPAIR])
{
    if constexpr (N < rbccol::NPROD) {
        constexpr rbccol::Prod pr = rbccol::prod_at(N);
        constexpr float w = (float)pr.weight;
        G[pr.to] = fmaf(w * s[pr.a][c], s[pr.b][c], G[pr.to]);
        colloc_products<N + 1>(s, c, G);
    }
}

// Parity in z of basis function k of a kind (C, S even for even k; each derivative flips).
RBC_HD constexpr int kind_derivs(int kind) { return kind == rbccol::KCP || kind == rbccol::KSP ? 1 : kind == rbccol::KCPP ? 2 : 0; }

// A level z_a and its mirror z_b = -z_a (the Gauss-Legendre rule is symmetric): the products of
// both, folded into their even and odd parts, and this thread's share of the level -> mode sums.
// Basis function k of a kind has the parity of k plus its number of z-derivatives, so its
// weighted values at z_a and -z_a are +-w_a chi(z_a) and only the matching part of the products
// enters: the mismatched part, which the exact integrals cancel, is formed as a difference of
// nearby values instead of a cancellation of large terms. Output modes k0 .. k0 + KH - 1
// (those < L) of the 13 groups; pq = row a of the weighted-basis table for kind 0 (kind c is
// kind_stride floats further).
template <int L, int KH>
RBC_D void colloc_level_pair(const float (&s)[rbccol::NSPAIR][kColChunk], int ca, int cb, const float* __restrict__ pq,
                             int kind_stride, int k0, float (&acc)[rbcprog::NGROUP][KH])
{
    float Ga[rbccol::NPPAIR], Gb[rbccol::NPPAIR];
#pragma unroll
    for (int p = 0; p < rbccol::NPPAIR; ++p) Ga[p] = Gb[p] = 0.0f;
    colloc_products<0>(s, ca, Ga);
    colloc_products<0>(s, cb, Gb);
    float cv[rbccol::NKIND][KH];
#pragma unroll
    for (int c = 0; c < rbccol::NKIND; ++c)
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) cv[c][kk] = (k0 + kk < L) ? pq[c * kind_stride + k0 + kk] : 0.0f;
#pragma unroll
    for (int p = 0; p < rbccol::NPPAIR; ++p) {
        const rbccol::PPair pp = rbccol::ppair_at(p); // constant after unrolling
        const float ge = Ga[p] + Gb[p], go = Ga[p] - Gb[p];
#pragma unroll
        for (int kk = 0; kk < KH; ++kk) {
            // z-parity of basis function k0 + kk of the pair's kind
            const bool odd = ((k0 + kk) + kind_derivs(pp.kind)) & 1;
            acc[pp.group][kk] = fmaf(cv[pp.kind][kk], odd ? go : ge, acc[pp.group][kk]);
        }
    }
}

// The collocation contraction of 128-point tiles (see the top of this file). Dynamic shared
// memory: colloc_geom(L, Q).smem + 1024 bytes of alignment slack.
template <int L>
__global__ void __launch_bounds__(kColThreads, 1) k_colloc_contract(CollocArgs A, int Q)
{
    constexpr int KH = (L + 1) / 2;
    const CollocGeom cg = colloc_geom(L, Q);
    extern __shared__ __align__(1024) unsigned char col_smem_raw[];
    unsigned char* sm = reinterpret_cast<unsigned char*>(((uintptr_t)col_smem_raw + 1023) & ~(uintptr_t)1023);
    unsigned char* a_ops = sm;                       // [8 fields][hi, lo] point operands
    unsigned char* b_ops = sm + 16u * cg.a_bytes;    // basis operands (hi image, then lo image)
    const float* projs = reinterpret_cast<const float*>(sm + cg.proj_off);
    unsigned long long* bar_b = reinterpret_cast<unsigned long long*>(sm + cg.bar_off);
    unsigned long long* bar_mma = bar_b + 1;
    unsigned* tslot = reinterpret_cast<unsigned*>(bar_b + 2);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int quad = warp & 3, half = warp >> 2;
    const int r = quad * 32 + lane;                  // this thread's point in the tile (TMEM lane)
    const int k0 = half * KH;                        // this thread's first output mode

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tslot)),
                     "r"(cg.tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    if (threadIdx.x == 32) {
        mbar_init(bar_b, 1);
        mbar_init(bar_mma, 1);
        mbar_fence_init();
    }
    // the level -> mode table (constant data, read before the programmatic wait)
    pdl_trigger();
    {
        const float* src = A.proj;
        float* dst = reinterpret_cast<float*>(sm + cg.proj_off);
        for (int e = threadIdx.x; e < rbccol::NKIND * Q * cg.Lp; e += blockDim.x) dst[e] = src[e];
        // the K padding of the point operands stays zero for the whole kernel
        if (cg.Kp > L) {
            for (int e = threadIdx.x; e < 16 * kColM; e += blockDim.x) {
                const int op = e / kColM, rr = e - op * kColM;
                for (int k = L; k < cg.Kp; ++k)
                    *reinterpret_cast<float*>(a_ops + (size_t)op * cg.a_bytes + colloc_kmajor_off(rr, k, cg.Kp)) = 0.0f;
            }
        }
    }
    col_fence_before();
    __syncthreads();
    col_fence_after();
    const unsigned tmem = *tslot;
    bool ok = true;
    if (threadIdx.x == 0) {
        // the basis operands: one bulk copy of the prebuilt image
        mbar_arrive_expect_tx(bar_b, cg.b_bytes);
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                         smem_u32(b_ops)),
                     "l"(reinterpret_cast<uint64_t>(A.bimg)), "r"(cg.b_bytes), "r"(smem_u32(bar_b))
                     : "memory");
    }
    ok = !__syncthreads_or(!col_wait(bar_b, 0)); // every thread takes the same branch
    pdl_wait(); // the synthesis is complete (and with it the previous step's update)
    if (A.nv && blockIdx.x == 0 && threadIdx.x == 0) *A.step_copy = ld_cg(A.step_counter);
    unsigned tile_no = 0;
    for (int t = blockIdx.x; t < A.ntiles && ok; t += gridDim.x, ++tile_no) {
        const long long x = (long long)t * kColM + r;
        const bool live = x < A.P;
        // ---- 1. point operands: half 0 splits fields 0-4 (and writes the tracer record),
        //         half 1 fields 5-7
        {
            float v[5][L];
            const int f0 = half == 0 ? 0 : 5, nf = half == 0 ? 5 : 3;
#pragma unroll
            for (int ff = 0; ff < 5; ++ff) {
                if (ff < nf) {
                    const int f = f0 + ff;
#pragma unroll
                    for (int i = 0; i < L; ++i) v[ff][i] = live ? ld_cg(A.phys + ((size_t)f * L + i) * A.P + x) : 0.0f;
                    unsigned char* oh = a_ops + (size_t)(2 * f) * cg.a_bytes;
                    unsigned char* ol = oh + cg.a_bytes;
#pragma unroll
                    for (int i4 = 0; i4 < (L + 3) / 4; ++i4) {
                        float h4[4], l4[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const float xv = (4 * i4 + e < L) ? v[ff][4 * i4 + e] : 0.0f;
                            h4[e] = tf32_hi(xv);
                            l4[e] = xv - h4[e];
                        }
                        const unsigned o = colloc_kmajor_off(r, 4 * i4, cg.Kp);
                        *reinterpret_cast<float4*>(oh + o) = make_float4(h4[0], h4[1], h4[2], h4[3]);
                        *reinterpret_cast<float4*>(ol + o) = make_float4(l4[0], l4[1], l4[2], l4[3]);
                    }
                }
            }
            if (A.nv && live && half == 0) store_node_record<float, L>(v, A.nv, (size_t)x);
        }
        fence_proxy_async_smem(); // the generic stores come before the tensor cores read them
        col_fence_before();
        __syncthreads();
        col_fence_after();
        // ---- 2. mode -> level products on the tensor cores (one thread issues)
        if (threadIdx.x == 0) {
#pragma unroll
            for (int f = 0; f < 8; ++f) {
                const uint32_t idesc = colloc_idesc_tf32(kColM, cg.ncol[f]);
                const unsigned d = tmem + (unsigned)cg.col0[f];
                const unsigned ah = smem_u32(a_ops + (size_t)(2 * f) * cg.a_bytes), al = ah + cg.a_bytes;
                const unsigned bh = smem_u32(b_ops + cg.b_off[f]), bl = bh + cg.b_half;
                for (int ks = 0; ks < cg.Kp / 8; ++ks) {
                    const unsigned ko = (unsigned)ks * 256; // 8 TF32 = two 16-byte core columns
                    const uint64_t dah = colloc_desc(ah + ko, cg.Kp), dal = colloc_desc(al + ko, cg.Kp);
                    const uint64_t dbh = colloc_desc(bh + ko, cg.Kp), dbl = colloc_desc(bl + ko, cg.Kp);
                    const unsigned first = ks > 0 ? 1u : 0u;
                    asm volatile("{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
                                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                                 "l"(dah), "l"(dbh), "r"(idesc), "r"(first)
                                 : "memory");
                    asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;\n" ::"r"(d), "l"(dah),
                                 "l"(dbl), "r"(idesc)
                                 : "memory");
                    asm volatile("tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, 1;\n" ::"r"(d), "l"(dal),
                                 "l"(dbh), "r"(idesc)
                                 : "memory");
                }
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                             smem_u32(bar_mma))
                         : "memory");
        }
        const bool done = col_wait(bar_mma, tile_no & 1);
        if (__syncthreads_or(!done)) {
            ok = false;
            break;
        }
        col_fence_after();
        // ---- 3. products and level -> mode sums, 4 levels per TMEM read
        float acc[rbcprog::NGROUP][KH];
#pragma unroll
        for (int g = 0; g < rbcprog::NGROUP; ++g)
#pragma unroll
            for (int kk = 0; kk < KH; ++kk) acc[g][kk] = 0.0f;
        const unsigned trow = tmem + ((unsigned)(quad * 32) << 16);
        // levels q, q + 1 with their mirrors Q - 1 - q, Q - 2 - q: Q / 4 reads cover all levels
        for (int q = 0; q < Q / 2; q += 2) {
            float s[rbccol::NSPAIR][kColChunk];
            colloc_load_pairs<0>(trow, cg.col0, Q, q, s);
            colloc_level_pair<L, KH>(s, 0, 3, projs + (size_t)q * cg.Lp, Q * cg.Lp, k0, acc);
            colloc_level_pair<L, KH>(s, 1, 2, projs + (size_t)(q + 1) * cg.Lp, Q * cg.Lp, k0, acc);
        }
        // ---- 4. this thread's output modes of the 13 groups
        if (live) {
#pragma unroll
            for (int g = 0; g < rbcprog::NGROUP; ++g)
#pragma unroll
                for (int kk = 0; kk < KH; ++kk)
                    if (k0 + kk < L) A.grp[((size_t)g * L + k0 + kk) * A.P + x] = acc[g][kk];
        }
        col_fence_before();
        __syncthreads(); // TMEM and the point operands are rewritten by the next tile
        col_fence_after();
    }
    if (threadIdx.x == 0 && !ok) atomicOr(A.err, RBC_DEVERR_TIMEOUT);
    col_fence_before();
    __syncthreads();
    if (warp == 0) {
        col_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(cg.tcols) : "memory");
    }
}

} // namespace rbck
