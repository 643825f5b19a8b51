// orc_noise.h -- seeded initial-condition noise shared by the two checkers
// (glsm_oracle.cpp and ref_harness.cu).  TEST INFRASTRUCTURE ONLY.
//
// splitmix64 (Steele, Lea, Flood 2014; the published mixing constants), keyed by
// (seed, gel id, element slot, field) and mapped to a uniform double in [-1, 1).
// The product implements the same definition independently.
#pragma once
#include <cstdint>

static inline uint64_t orc_splitmix64(uint64_t x) {
    uint64_t z = x + 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

static inline double orc_noise_pm1(uint64_t seed, uint64_t gel_id, uint64_t slot, uint64_t field) {
    uint64_t h = orc_splitmix64(orc_splitmix64(orc_splitmix64(seed) ^ gel_id) ^ (slot * 2ull + field));
    double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
    return 2.0 * u - 1.0;
}
