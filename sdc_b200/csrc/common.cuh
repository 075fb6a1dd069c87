// common.cuh -- small device helpers shared by the sm_100a kernels of the RBC step.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define RBC_HD __host__ __device__ __forceinline__
#define RBC_D __device__ __forceinline__

// Complex helpers on CUDA vector types (double2 / float2): .x real, .y imaginary.
template <typename R> struct cplx_t;
template <> struct cplx_t<double> { typedef double2 type; };
template <> struct cplx_t<float> { typedef float2 type; };

template <typename C> RBC_HD C cmk(double re, double im) { C c; c.x = re; c.y = im; return c; }
RBC_HD double2 operator+(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
RBC_HD double2 operator-(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
RBC_HD double2 operator*(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
RBC_HD float2 operator+(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
RBC_HD float2 operator-(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
RBC_HD float2 operator*(float2 a, float s) { return make_float2(a.x * s, a.y * s); }
template <typename C> RBC_HD C cmul(C a, C b) { C r; r.x = a.x * b.x - a.y * b.y; r.y = a.x * b.y + a.y * b.x; return r; }
template <typename C> RBC_HD C cconj(C a) { a.y = -a.y; return a; }
// multiply by i*s
template <typename C, typename R> RBC_HD C cmul_is(C a, R s) { C r; r.x = -s * a.y; r.y = s * a.x; return r; }

// One node record of the tracer velocity array: the 5 L velocity-field values u11, u21,
// u31, u12, u22 of a grid point in two halves, modes i < LH and i >= LH (LH = ceil(L/2)).
// Each half lists its modes' five values mode by mode and is padded to an even count, so
// that in FP64 every half starts on a 16-byte boundary: one tracer lane reads one half.
template <int L> struct NodeRec {
    static constexpr int LH = (L + 1) / 2;
    static constexpr int HALF = (5 * LH + 1) & ~1;
    static constexpr int value = 2 * HALF;
    static RBC_HD constexpr int at(int f, int i) { return (i / LH) * HALF + (i % LH) * 5 + f; }
};
RBC_HD constexpr int node_rec_len(int L) { return 2 * ((5 * ((L + 1) / 2) + 1) & ~1); }

// Error word written by kernels that detect a violated precondition (never traps).
enum rbc_dev_error { RBC_DEVERR_NONE = 0, RBC_DEVERR_BOUNDS = 1, RBC_DEVERR_NAN = 2, RBC_DEVERR_TIMEOUT = 4 };

// Asynchronous global -> shared copies (cp.async, sm_80+): every copy of a load phase
// is in flight at once and no registers stage the data. Element sizes 4, 8 or 16 bytes;
// both addresses aligned to the size. cp_async_wait_all() + __syncthreads() publishes
// the data to the CTA.
template <int BYTES> RBC_D void cp_async(void* smem_dst, const void* gmem_src)
{
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "cp.async copies 4, 8 or 16 bytes");
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], %2;\n" ::"r"(s), "l"(gmem_src), "n"(BYTES) : "memory");
}
RBC_D void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Reads of step data: data that an earlier kernel of the step wrote. The step's kernels
// are launched with programmatic stream serialization (below), so a kernel can be resident
// on an SM while its predecessor still runs there. Measured on B200: when the predecessor
// also READ the data it then rewrote (the penalization kernel's read-modify-write of the
// contracted groups), the dependent's non-coherent loads issued after griddepcontrol.wait
// returned the pre-write values for a few rows; no such failure was seen with loads that
// skip the L1. So step data is read with ld.global.cg / cp.async.cg, which go to L2, the
// point of coherence; the data is streamed once per kernel, so nothing is lost.
template <typename T> RBC_D T ld_cg(const T* p) { return __ldcg(p); }
// Global -> shared copy of step data of 4, 8 or 16 bytes through L2: cp.async.cg for 16
// bytes (asynchronous, completes at cp_async_wait_all), a register copy for 4 and 8
// (cp.async has no L2-only form for them). Either is published by the __syncthreads that
// follows cp_async_wait_all.
template <int BYTES> RBC_D void copy_cg(void* smem_dst, const void* gmem_src)
{
    static_assert(BYTES == 4 || BYTES == 8 || BYTES == 16, "copies of 4, 8 or 16 bytes");
    if constexpr (BYTES == 16) {
        cp_async<16>(smem_dst, gmem_src);
    } else if constexpr (BYTES == 8) {
        *static_cast<uint2*>(smem_dst) = __ldcg(static_cast<const uint2*>(gmem_src));
    } else {
        *static_cast<unsigned*>(smem_dst) = __ldcg(static_cast<const unsigned*>(gmem_src));
    }
}

// Programmatic dependent launch (sm_90+). A kernel launched with the programmatic
// stream-serialization attribute may start once every CTA of its predecessor in the stream
// has called pdl_trigger (or exited), i.e. while the predecessor drains. Before pdl_wait
// such a kernel may read only data no kernel of the step writes (twiddles, coefficient
// tables, class indices) and write nothing; pdl_wait returns when the predecessor has
// completed and its writes are visible. Both are no-ops for an ordinary launch.
RBC_D void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
RBC_D void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }

// ---------------------------------------------------------------------------------
// mbarriers (sm_90+) for the asynchronous copy engine and the tensor cores: initialisation,
// arrivals (with an expected transaction byte count), and the poll budget of every bounded
// wait on one (kMbarSpins).
RBC_D unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }
RBC_D void mbar_init(unsigned long long* mbar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(mbar)), "r"(count) : "memory");
}
// Makes initialised mbarriers visible to the copy engine (before the CTA barrier that
// publishes them).
RBC_D void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory"); }
// Orders this thread's earlier generic accesses of shared memory before later accesses by
// the async proxy (copies into it, tensor-core reads of it).
RBC_D void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
RBC_D void mbar_arrive(unsigned long long* mbar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(mbar)) : "memory");
}
RBC_D void mbar_arrive_expect_tx(unsigned long long* mbar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(mbar)), "r"(bytes)
                 : "memory");
}
constexpr unsigned kMbarSpins = 1u << 22;
