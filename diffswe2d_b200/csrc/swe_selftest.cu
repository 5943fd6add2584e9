// swe_selftest.cu -- device self-test of the step's arithmetic building
// blocks against CUDA's IEEE operations.
//
// The step shares reciprocals between quotients (rcp_cr / div_by in
// swe_math.cuh).  This entry point checks, on the GPU it will run on:
//   which = 0: rcp_cr(b) == __frcp_rn(b) for every float b in [2^-100, 2^100)
//              (both signs), i.e. exhaustively over the range the step uses;
//   which = 1: div_by(a, b, rcp_cr(b)) == __fdiv_rn(a, b) for `count` random
//              operand pairs (a, b) drawn from a counter-based hash;
//   which = 2: the same for quotients constructed next to rounding midpoints
//              (a = b * m for m half-way between two floats, then its
//              float neighbours), the cases a one-step correction can miss;
//   which = 3: sqrt_cr(x) == __fsqrt_rn(x) for every float x in
//              [2^-100, 2^100);
//   which = 4: pow_pos(x, t) == (float)pow((double)x, (double)t) for every
//              float x in [2^-40, 2^14), t the float whose bit pattern is
//              the low 32 bits of `seed`;
//   which = 5: div_by(a, b, rcp_cr(b)) == __fdiv_rn(a, b) for n draws of b
//              in [2^-20, 2^20) and six tiny numerators each: one random
//              below 2^-62 (subnormals included) and five next to a
//              quotient midpoint, scaled by 2^-90.
// It returns the number of mismatches and the first mismatching input.
#include <cuda_runtime.h>
#include <stdint.h>

#include "swe_common.cuh"

namespace swe {
namespace {

__device__ __forceinline__ uint32_t hash32(uint64_t x) {
    x ^= x >> 33;
    x *= 0xff51afd7ed558ccdull;
    x ^= x >> 33;
    x *= 0xc4ceb9fe1a85ec53ull;
    x ^= x >> 33;
    return (uint32_t)x;
}

// A float with a uniformly random significand and an exponent in [emin, emax].
__device__ __forceinline__ float rand_float(uint64_t key, int emin, int emax) {
    const uint32_t h = hash32(key);
    const uint32_t e = (uint32_t)(emin + (int)(hash32(key ^ 0x9e3779b97f4a7c15ull) % (uint32_t)(emax - emin + 1)));
    const uint32_t bits = ((e + 127u) << 23) | (h & 0x7fffffu);
    return u2f(bits | ((h >> 31) << 31));
}

__device__ void record(unsigned long long* count, uint32_t* first, uint32_t a, uint32_t b) {
    const unsigned long long old = atomicAdd(count, 1ull);
    if (old == 0) {
        first[0] = a;
        first[1] = b;
    }
}

__global__ void rcp_exhaustive(unsigned long long* count, uint32_t* first) {
    // all significands of all exponents -100..99 (2^23 * 200 values), both signs
    const uint64_t n = (uint64_t)200 << 24;
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t sig = (uint32_t)(t & 0x7fffffu);
        const uint32_t sign = (uint32_t)((t >> 23) & 1u);
        const uint32_t e = (uint32_t)(t >> 24) + 27u;  // biased exponent 27..226 = -100..99
        const float b = u2f((sign << 31) | (e << 23) | sig);
        const float y = rcp_cr(b);
        const float ref = __frcp_rn(b);
        if (f2u(y) != f2u(ref)) record(count, first, f2u(b), f2u(y));
    }
}

__global__ void sqrt_exhaustive(unsigned long long* count, uint32_t* first) {
    const uint64_t n = (uint64_t)200 << 23;  // exponents -100..99, all significands
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t bits = (uint32_t)t + (27u << 23);
        const float x = u2f(bits);
        const float s = sqrt_cr(x);
        if (f2u(s) != f2u(__fsqrt_rn(x))) record(count, first, bits, f2u(s));
    }
}

__global__ void pow_exhaustive(unsigned long long* count, uint32_t* first, float t) {
    const uint64_t n = (uint64_t)54 << 23;  // exponents -40..13, all significands
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t bits = (uint32_t)i + (87u << 23);
        const float x = u2f(bits);
        const float p = pow_pos(x, t);
        if (f2u(p) != f2u((float)pow((double)x, (double)t))) record(count, first, bits, f2u(p));
    }
}

__global__ void div_tiny(unsigned long long* count, uint32_t* first, uint64_t n, uint64_t seed) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const float b = rand_float(seed ^ (t * 3 + 0x2468aceull), -20, 19);
        float as[6];
        // random: exponent field 0..64 (subnormals and [2^-126, 2^-62))
        const uint32_t h = hash32(seed ^ (t * 3 + 1 + 0x1f2e3dull));
        const uint32_t ef = hash32(seed ^ (t * 3 + 2 + 0x5a5a5aull)) % 65u;
        as[0] = u2f((ef << 23) | (h & 0x7fffffu) | ((h >> 31) << 31));
        // next to a midpoint of the quotient, scaled down by 2^-90
        const float m0 = rand_float(seed ^ (t * 3 + 0xabcdefull), -10, 10);
        const double mid = 0.5 * ((double)m0 + (double)u2f(f2u(m0) + 1u));
        const float a0 = (float)((double)b * mid * 0x1p-90);
        for (int d = -2; d <= 2; ++d) as[3 + d] = u2f(f2u(a0) + (uint32_t)d);
        for (int k = 0; k < 6; ++k) {
            const float q = div_by(as[k], b, rcp_cr(b));
            if (f2u(q) != f2u(__fdiv_rn(as[k], b))) record(count, first, f2u(as[k]), f2u(b));
        }
    }
}

__global__ void div_random(unsigned long long* count, uint32_t* first, uint64_t n, uint64_t seed) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const float a = rand_float(seed ^ (t * 2 + 0x1234567ull), -60, 60);
        const float b = rand_float(seed ^ (t * 2 + 1 + 0x7654321ull), -30, 30);
        const float q = div_by(a, b, rcp_cr(b));
        if (f2u(q) != f2u(__fdiv_rn(a, b))) record(count, first, f2u(a), f2u(b));
    }
}

__global__ void div_midpoints(unsigned long long* count, uint32_t* first, uint64_t n, uint64_t seed) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < n;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const float b = rand_float(seed ^ (t * 3 + 0xabcdefull), -20, 20);
        const float m0 = rand_float(seed ^ (t * 3 + 1 + 0x13579bull), -20, 20);
        // midpoint between m0 and its successor, in double; a = RN(b * mid)
        const double mid = 0.5 * ((double)m0 + (double)u2f(f2u(m0) + 1u));
        const float a0 = (float)((double)b * mid);
        for (int d = -2; d <= 2; ++d) {
            const float a = u2f(f2u(a0) + (uint32_t)d);
            const float q = div_by(a, b, rcp_cr(b));
            if (f2u(q) != f2u(__fdiv_rn(a, b))) record(count, first, f2u(a), f2u(b));
        }
    }
}

}  // namespace
}  // namespace swe

using namespace swe;

// count: device unsigned long long; first: device uint32_t[2] (first
// mismatching inputs); both are written by the call.
extern "C" int swe_selftest_arith_f32(int which, long long n, unsigned long long seed,
                                      unsigned long long* count, uint32_t* first, void* stream) {
    if (!count || !first || which < 0 || which > 5 || n < 0) return SWE_EARG;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(count, 0, sizeof(unsigned long long), s) != cudaSuccess) return SWE_ECUDA;
    if (cudaMemsetAsync(first, 0, 2 * sizeof(uint32_t), s) != cudaSuccess) return SWE_ECUDA;
    const int blocks = 148 * 8, threads = 256;
    if (which == 0) rcp_exhaustive<<<blocks, threads, 0, s>>>(count, first);
    else if (which == 3) sqrt_exhaustive<<<blocks, threads, 0, s>>>(count, first);
    else if (which == 4) pow_exhaustive<<<blocks, threads, 0, s>>>(count, first, u2f((uint32_t)seed));
    else if (which == 5) div_tiny<<<blocks, threads, 0, s>>>(count, first, (uint64_t)n, seed);
    else if (which == 1) div_random<<<blocks, threads, 0, s>>>(count, first, (uint64_t)n, seed);
    else div_midpoints<<<blocks, threads, 0, s>>>(count, first, (uint64_t)n, seed);
    return cudaGetLastError() == cudaSuccess ? SWE_OK : SWE_ECUDA;
}
