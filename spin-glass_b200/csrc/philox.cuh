// philox.cuh — Philox4x32-10 counter-based generator (device + host).
//
// Algorithm: Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as
// 1, 2, 3", SC'11.  Ten rounds; each round multiplies counter words 0 and 2 by
// two odd constants (full 64-bit products), mixes the high halves into words
// 1 and 3 with the key, and the key is bumped by two Weyl increments between
// rounds.  On sm_100a a round is two 32x32 multiply pairs and two LOP3.
#pragma once
#include <cstdint>

#if defined(__CUDACC__)
#define CSG_HD __host__ __device__ __forceinline__
#else
#define CSG_HD inline
#endif

namespace csg {

struct u32x4 {
    uint32_t v0, v1, v2, v3;
};

CSG_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#if defined(__CUDA_ARCH__)
    lo = a * b;
    hi = __umulhi(a, b);
#else
    const uint64_t p = (uint64_t)a * b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

CSG_HD u32x4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                           uint32_t k1) {
    constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
    constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 0; r < 10; ++r) {
        uint32_t hi0, lo0, hi1, lo1;
        mulhilo32(kM0, c0, hi0, lo0);
        mulhilo32(kM1, c2, hi1, lo1);
        const uint32_t n0 = hi1 ^ c1 ^ k0;
        const uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0;
        c1 = lo1;
        c2 = n2;
        c3 = lo0;
        k0 += kW0;
        k1 += kW1;
    }
    return u32x4{c0, c1, c2, c3};
}

// Philox4x32-10 for many counters that differ only in word 0.  The parts of
// the first two rounds that do not depend on word 0 are computed once
// (philox_fix); philox_c0 then does one multiply in each of rounds 1 and 2
// instead of two.  philox_c0(c0, philox_fix(c1, c2, c3, k0, k1)) equals
// philox4x32_10(c0, c1, c2, c3, k0, k1) for every input.
struct PhiloxFixed {
    uint32_t x3;  // round 1: c3 ^ key 1, mixed into word 2
    uint32_t y;   // round 2: (word 1 after round 1) ^ key 0 of round 2
    uint32_t z;   // round 2: high half of M0 * (word 0 after round 1) ^ key 1 of round 2
    uint32_t w3;  // round 2: low half of that product (word 3 after round 2)
    uint32_t k0, k1;
};

CSG_HD PhiloxFixed philox_fix(uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1) {
    constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
    constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
    PhiloxFixed f;
    uint32_t hi1, lo1;
    mulhilo32(kM1, c2, hi1, lo1);
    const uint32_t a0 = hi1 ^ c1 ^ k0;  // word 0 after round 1
    const uint32_t a1 = lo1;            // word 1 after round 1
    f.x3 = c3 ^ k1;
    uint32_t bh, bl;
    mulhilo32(kM0, a0, bh, bl);
    f.y = a1 ^ (k0 + kW0);
    f.z = bh ^ (k1 + kW1);
    f.w3 = bl;
    f.k0 = k0;
    f.k1 = k1;
    return f;
}

CSG_HD u32x4 philox_c0(uint32_t c0, const PhiloxFixed& f) {
    constexpr uint32_t kM0 = 0xD2511F53u, kM1 = 0xCD9E8D57u;
    constexpr uint32_t kW0 = 0x9E3779B9u, kW1 = 0xBB67AE85u;
    // round 1
    uint32_t hi0, lo0;
    mulhilo32(kM0, c0, hi0, lo0);
    const uint32_t b2 = hi0 ^ f.x3;
    // round 2
    uint32_t hi1, lo1;
    mulhilo32(kM1, b2, hi1, lo1);
    uint32_t v0 = hi1 ^ f.y, v1 = lo1, v2 = lo0 ^ f.z, v3 = f.w3;
    uint32_t k0 = f.k0 + 2u * kW0, k1 = f.k1 + 2u * kW1;
#if defined(__CUDA_ARCH__)
#pragma unroll
#endif
    for (int r = 2; r < 10; ++r) {
        uint32_t h0, l0, h1, l1;
        mulhilo32(kM0, v0, h0, l0);
        mulhilo32(kM1, v2, h1, l1);
        const uint32_t n0 = h1 ^ v1 ^ k0;
        const uint32_t n2 = h0 ^ v3 ^ k1;
        v0 = n0;
        v1 = l1;
        v2 = n2;
        v3 = l0;
        k0 += kW0;
        k1 += kW1;
    }
    return u32x4{v0, v1, v2, v3};
}

// Counter layout shared by every generator call of the engine:
//   word 0: site index (or sample-pair index for exchanges)
//   word 1: global sweep index
//   word 2: sample word index
//   word 3: tag << 24 | copy << 8 | temperature quad (or plane)
constexpr uint32_t kTagBond = 1u << 24;
constexpr uint32_t kTagInit = 2u << 24;
constexpr uint32_t kTagSweep = 3u << 24;
constexpr uint32_t kTagSwap = 4u << 24;

}  // namespace csg
