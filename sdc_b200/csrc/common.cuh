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

// Programmatic dependent launch (sm_90+). A kernel launched with the programmatic
// stream-serialization attribute may start once every CTA of its predecessor in the stream
// has called pdl_trigger (or exited), i.e. while the predecessor drains. Before pdl_wait
// such a kernel may read only data no kernel of the step writes (twiddles, coefficient
// tables, class indices) and write nothing; pdl_wait returns when the predecessor has
// completed and its writes are visible. Both are no-ops for an ordinary launch.
RBC_D void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }
RBC_D void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
