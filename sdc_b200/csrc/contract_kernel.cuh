// contract_kernel.cuh -- pointwise products + exact Galerkin contraction (sm_100a).
//
// For every physical point x: read the 8 L synthesised values a_f,i(x), and for every
// output mode k produce the 13 group values Q_{D,k}(x) of contract_prog.h. The unit and
// edge structure is compile-time (template recursion over the units), the coefficient
// values T'(o,s) live in shared memory, parity-compressed: for output k and row o only
// s = s0, s0+2, ... with s0 = (o + k + parity) & 1 are stored and multiplied, so every
// stored coefficient is a nonzero of the reference's tensors. k runs in pairs so its
// parity is a template parameter. Inputs stay in registers (8 L values per point).
#pragma once
#include "common.cuh"
#include "contract_prog.h"

namespace rbck {

template <typename R, int L, int KP, int U>
RBC_D void contract_units(const R (&in)[rbcprog::NFIELD][L], R (&acc)[rbcprog::NGROUP], const R* __restrict__ cbase)
{
    if constexpr (U < rbcprog::NUNIT) {
        constexpr rbcprog::Unit u = rbcprog::unit_at(U);
        constexpr int par = rbcprog::family_parity(u.family);
        constexpr int H = rbcprog::half_len(L);
        const R* cb = cbase + (size_t)U * L * L * H; // caller offsets by k
        R w[L];
#pragma unroll
        for (int o = 0; o < L; ++o) {
            const int s0 = (o + KP + par) & 1;
            R a = 0;
#pragma unroll
            for (int h = 0; h < H; ++h) {
                const int s = s0 + 2 * h;
                if (s < L) a = fma(cb[o * H + h], in[u.fixed][s], a);
            }
            w[o] = a;
        }
#pragma unroll
        for (int ed = 0; ed < u.nedge; ++ed) {
            // two interleaved partial sums halve the FMA dependency chain
            R d0 = 0, d1 = 0;
#pragma unroll
            for (int o = 0; o < L; o += 2) {
                d0 = fma(w[o], in[u.e[ed].other][o], d0);
                if (o + 1 < L) d1 = fma(w[o + 1], in[u.e[ed].other][o + 1], d1);
            }
            acc[u.e[ed].group] = fma((R)u.e[ed].weight, d0 + d1, acc[u.e[ed].group]);
        }
        contract_units<R, L, KP, U + 1>(in, acc, cbase);
    }
}

template <typename R, int L, int KP>
RBC_D void contract_mode(const R (&in)[rbcprog::NFIELD][L], const R* __restrict__ coef, int k,
                         R* __restrict__ grp, size_t P, size_t x)
{
    R acc[rbcprog::NGROUP];
#pragma unroll
    for (int gi = 0; gi < rbcprog::NGROUP; ++gi) acc[gi] = 0;
    constexpr int H = rbcprog::half_len(L);
    contract_units<R, L, KP, 0>(in, acc, coef + (size_t)k * L * H);
#pragma unroll
    for (int gi = 0; gi < rbcprog::NGROUP; ++gi) grp[((size_t)gi * L + k) * P + x] = acc[gi];
}

// Writes point x's node record (fields 0..4 of `in`, pads zero) with 8- or 16-byte stores.
template <typename R, int L, typename In>
RBC_D void store_node_record(const In& in, R* __restrict__ nv, size_t x)
{
    constexpr int NR = NodeRec<L>::value;
    typedef typename cplx_t<R>::type R2;
    R rec[NR];
#pragma unroll
    for (int e = 0; e < NR; ++e) rec[e] = 0;
#pragma unroll
    for (int f = 0; f < 5; ++f)
#pragma unroll
        for (int i = 0; i < L; ++i) rec[NodeRec<L>::at(f, i)] = in[f][i];
    R2* dst = reinterpret_cast<R2*>(nv + x * NR);
#pragma unroll
    for (int q = 0; q < NR / 2; ++q) {
        R2 v;
        v.x = rec[2 * q];
        v.y = rec[2 * q + 1];
        dst[q] = v;
    }
}

// The node records alone (no contraction): the tracer advance that runs on a state no
// step will start from (a state about to be changed between steps) needs only these.
template <typename R, int L>
__global__ void __launch_bounds__(256) k_node_records(const R* __restrict__ phys, int P, R* __restrict__ nv)
{
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < P; x += gridDim.x * blockDim.x) {
        R in[5][L];
#pragma unroll
        for (int f = 0; f < 5; ++f)
#pragma unroll
            for (int i = 0; i < L; ++i) in[f][i] = phys[((size_t)f * L + i) * P + x];
        store_node_record<R, L>(in, nv, (size_t)x);
    }
}

// Grid-stride over points; coef (global) is the packed array of pack_contraction,
// copied once per CTA into shared memory. When nv is not null the kernel also writes
// every point's node record nv[x * NodeRec] (the tracers gather those records), and
// copies the step counter to step_copy: the tracer advance that reads the records runs
// beside the update that increments the counter, and reads the copy.
template <typename R, int L>
__global__ void __launch_bounds__(128) k_contract(const R* __restrict__ phys, R* __restrict__ grp,
                                                  const R* __restrict__ coef_g, int P, R* __restrict__ nv,
                                                  const long long* __restrict__ step_counter, long long* step_copy)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* coef = reinterpret_cast<R*>(smem_raw);
    constexpr int NC = rbcprog::NUNIT * L * L * rbcprog::half_len(L);
    pdl_trigger();
    for (int e = threadIdx.x; e < NC; e += blockDim.x) coef[e] = coef_g[e];
    pdl_wait(); // the synthesis is complete (and with it the previous step's update)
    if (nv && blockIdx.x == 0 && threadIdx.x == 0) *step_copy = ld_cg(step_counter);
    __syncthreads();
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < P; x += gridDim.x * blockDim.x) {
        R in[rbcprog::NFIELD][L];
#pragma unroll
        for (int f = 0; f < rbcprog::NFIELD; ++f)
#pragma unroll
            for (int i = 0; i < L; ++i) in[f][i] = ld_cg(phys + ((size_t)f * L + i) * P + x);
        if (nv) store_node_record<R, L>(in, nv, (size_t)x);
        for (int k = 0; k < L; k += 2) {
            contract_mode<R, L, 0>(in, coef, k, grp, P, x);
            if (k + 1 < L) contract_mode<R, L, 1>(in, coef, k + 1, grp, P, x);
        }
    }
}

} // namespace rbck
