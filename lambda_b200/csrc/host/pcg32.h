// PCG-XSH-RR 64/32 generator with the reference's seeding and float mapping
// (src/math/random.h:7-30): stream s uses increment 2s+1; seeding steps once,
// adds the seed, steps again; next() maps the 32-bit output x to float(x)/2^32
// (which rounds to 1.0f for x close to 2^32, as the reference does).
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define LAMBDA_HD __host__ __device__ __forceinline__
#else
#define LAMBDA_HD inline
#endif

namespace lambda_rng {

constexpr uint64_t kMultiplier = 6364136223846793005ULL;

LAMBDA_HD uint32_t pcg_output(uint64_t old) {
    const uint32_t xorshifted = uint32_t(((old >> 18u) ^ old) >> 27u);
    const uint32_t rot = uint32_t(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((0u - rot) & 31u));
}

LAMBDA_HD uint64_t pcg_increment(uint64_t stream) { return (stream << 1) | 1u; }

// State after Random(seed, stream)'s constructor.
LAMBDA_HD uint64_t pcg_seed(uint64_t seed, uint64_t stream) {
    const uint64_t inc = pcg_increment(stream);
    uint64_t state = inc;              // 0 * a + inc
    state += seed;
    state = state * kMultiplier + inc;
    return state;
}

LAMBDA_HD float pcg_next_float(uint64_t &state, uint64_t inc) {
    const uint64_t old = state;
    state = old * kMultiplier + inc;
    return float(pcg_output(old)) / 4294967296.0f;
}

}  // namespace lambda_rng
