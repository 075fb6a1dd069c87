// splitmix.h -- SplitMix64 (Steele, Lea & Flood, OOPSLA 2014) read as a random-access
// stream, and the normal draw of the tracer diffusion step; host and device code.
#pragma once
#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define RBCS_HD __host__ __device__ __forceinline__
#else
#define RBCS_HD inline
#endif

namespace rbcrng {

constexpr uint64_t kGamma = 0x9E3779B97F4A7C15ULL;

RBCS_HD uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// Element i (0-based) of the stream of seed s: the generator adds kGamma before mixing.
RBCS_HD uint64_t stream_at(uint64_t s, uint64_t i) { return mix64(s + (i + 1) * kGamma); }

// Uniform in (0, 1) from the top 53 bits.
RBCS_HD double unit_open(uint64_t u) { return ((double)(u >> 11) + 0.5) * 0x1.0p-53; }

// Normal of the diffusion step for the positions of step m, particle t of n, coordinate d:
// Box-Muller on stream elements 2j and 2j + 1, j = 3 (m n + t) + d.
RBCS_HD double diffusion_normal(uint64_t seed, long long m, long long n, long long t, int d)
{
    const uint64_t j = 3ULL * ((uint64_t)m * (uint64_t)n + (uint64_t)t) + (uint64_t)d;
    const double u1 = unit_open(stream_at(seed, 2 * j)), u2 = unit_open(stream_at(seed, 2 * j + 1));
    return cos(6.283185307179586476925286766559 * u2) * sqrt(-2.0 * log(u1));
}

} // namespace rbcrng
