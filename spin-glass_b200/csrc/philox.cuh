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
