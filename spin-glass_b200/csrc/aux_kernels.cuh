// aux_kernels.cuh — set-up and section-end kernels (not on the sweep path).
//
// init_kernel     : bonds and initial spins from the seed (replaces the host
//                   cuRAND generation of eamsim.cu:562-652).
// measure_kernel  : per-sample bond energy, magnetisation and overlap
//                   integers of the current state, including the overlap
//                   summed per coordinate plane, from which the Fourier
//                   overlaps of compute_q (eamsim.cu:451-511) are formed.
// records_kernel  : the reference's obs_s records from those integers.
// The kernels have internal linkage: each translation unit that launches
// them (the engine, the no-allocation records entry point) has its own copy
// of the same code.
#pragma once
#include <cstdint>

#include "philox.cuh"

namespace csg {

static __global__ void init_kernel(uint32_t* spins, uint32_t* bonds, int L, int W, int C, int Q,
                            uint32_t k0, uint32_t k1, uint32_t word0) {
    const long N = (long)L * L * L;
    const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long)W * N) return;
    const int w = (int)(idx / N);
    const int i = (int)(idx - (long)w * N);
    const int x = i % L, y = (i / L) % L, z = i / (L * L);
    const long slot = (long)((x + y + z) & 1) * (N / 2) + (long)(z * L + y) * (L / 2) + (x >> 1);
    const uint32_t wg = (uint32_t)w + word0;
    const u32x4 rb = philox4x32_10((uint32_t)i, 0u, wg, kTagBond, k0, k1);
    bonds[((long)w * 3 + 0) * N + slot] = rb.v0;
    bonds[((long)w * 3 + 1) * N + slot] = rb.v1;
    bonds[((long)w * 3 + 2) * N + slot] = rb.v2;
    uint4* sp = reinterpret_cast<uint4*>(spins);
    for (int c = 0; c < C; ++c)
        for (int q = 0; q < Q; ++q) {
            const u32x4 r = philox4x32_10((uint32_t)i, 0u, wg,
                                          kTagInit | ((uint32_t)c << 8) | (uint32_t)q, k0, k1);
            sp[(((long)w * C + c) * Q + q) * N + slot] = make_uint4(r.v0, r.v1, r.v2, r.v3);
        }
}

// One warp per (word, temperature); lane b = sample 32w+b.  Outputs
//   e[w][c][t][b] = -(sum of J s s) (bond energy), m[w][c][t][b] = 2 n_up - N,
//   d[w][t][b] = #sites where the copies differ,
//   dpl[w][t][b][dir][a] = same restricted to coordinate dir == a.
// Requires two copies. Shared memory: 32 * 3L ints per warp.
static __global__ void measure_kernel(const uint32_t* __restrict__ spins, const uint32_t* __restrict__ bonds,
                               int L, int W, int T, int* e, int* m, int* d, int* dpl) {
    extern __shared__ int sh[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair = blockIdx.x * (blockDim.x >> 5) + warp;
    const int Q = T / 4;
    const long N = (long)L * L * L, NH = N / 2;
    int* cnt = sh + warp * 3 * L * 32;  // [3L][32]
    for (int k = lane; k < 3 * L * 32; k += 32) cnt[k] = 0;
    __syncwarp();
    if (pair >= W * T) return;
    const int w = pair / T, t = pair - w * T;
    auto spin = [&](int c, long slot) {
        return spins[((((long)w * 2 + c) * Q + (t >> 2)) * N + slot) * 4 + (t & 3)];
    };
    int unsat[2] = {0, 0}, up[2] = {0, 0}, diff = 0;
    for (int z = 0; z < L; ++z)
        for (int y = 0; y < L; ++y)
            for (int x = 0; x < L; ++x) {
                const long si = (long)((x + y + z) & 1) * NH + (long)(z * L + y) * (L / 2) + (x >> 1);
                const int xp = x + 1 == L ? 0 : x + 1, yp = y + 1 == L ? 0 : y + 1,
                          zp = z + 1 == L ? 0 : z + 1;
                const long nb[3] = {(long)((xp + y + z) & 1) * NH + (long)(z * L + y) * (L / 2) + (xp >> 1),
                                    (long)((x + yp + z) & 1) * NH + (long)(z * L + yp) * (L / 2) + (x >> 1),
                                    (long)((x + y + zp) & 1) * NH + (long)(zp * L + y) * (L / 2) + (x >> 1)};
                const uint32_t f[3] = {bonds[((long)w * 3 + 0) * N + si],
                                       bonds[((long)w * 3 + 1) * N + si],
                                       bonds[((long)w * 3 + 2) * N + si]};
                uint32_t s[2];
                for (int c = 0; c < 2; ++c) {
                    s[c] = spin(c, si);
                    up[c] += (s[c] >> lane) & 1u;
                    for (int k = 0; k < 3; ++k) unsat[c] += ((s[c] ^ spin(c, nb[k]) ^ f[k]) >> lane) & 1u;
                }
                if (((s[0] ^ s[1]) >> lane) & 1u) {
                    ++diff;
                    cnt[(0 * L + x) * 32 + lane] += 1;
                    cnt[(1 * L + y) * 32 + lane] += 1;
                    cnt[(2 * L + z) * 32 + lane] += 1;
                }
            }
    for (int c = 0; c < 2; ++c) {
        const long o = (((long)w * 2 + c) * T + t) * 32 + lane;
        e[o] = 2 * unsat[c] - 3 * (int)N;
        m[o] = 2 * up[c] - (int)N;
    }
    const long o = ((long)w * T + t) * 32 + lane;
    d[o] = diff;
    for (int k = 0; k < 3 * L; ++k) dpl[(o * 3 * L) + k] = cnt[k * 32 + lane];
}

// The reference records (obs_s: e[2], m[2], q_0, q_1_r[3], q_1_i[3]) of one
// (sample, temperature) from the integers of measure_kernel, with the float
// and double operations of the host formulas (eamsim.cu:320-325, 477-509) in
// the same order; cosv/sinv hold cos(k a), sin(k a), k = 2 pi / L, computed on
// the host.  Built without contraction (-fmad=false), the records equal the
// host's bit for bit.
static __global__ void records_kernel(const int* __restrict__ e, const int* __restrict__ m,
                               const int* __restrict__ d, const int* __restrict__ dpl,
                               const double* __restrict__ cosv, const double* __restrict__ sinv,
                               int L, int W, int T, float H, float* __restrict__ rec) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;  // (w, b, t), t fastest
    if (i >= (long)W * 32 * T) return;
    const int t = (int)(i % T);
    const long sb = i / T;  // sample 32 w + b
    const int w = (int)(sb >> 5), b = (int)(sb & 31);
    const long long N = (long long)L * L * L;
    float* o = rec + i * 11;
    for (int c = 0; c < 2; ++c) {
        const size_t k = (((size_t)w * 2 + c) * T + t) * 32 + b;
        const float es = (float)(-e[k]);
        const float ms = (float)m[k];
        o[c] = -(es + H * ms) / (float)N;
        o[2 + c] = ms / (float)N;
    }
    const size_t k = ((size_t)w * T + t) * 32 + b;
    o[4] = (float)(N - 2 * (long long)d[k]) / (float)N;
    for (int dir = 0; dir < 3; ++dir) {
        double re = 0.0, im = 0.0;
        for (int a = 0; a < L; ++a) {
            const long long P = (long long)L * L - 2 * (long long)dpl[(k * 3 + dir) * L + a];
            re += (double)P * cosv[a];
            im += (double)P * sinv[a];
        }
        o[5 + dir] = (float)(re / (double)N);
        o[8 + dir] = (float)(im / (double)N);
    }
}

}  // namespace csg
