// stream_kernels.cuh — parallel tempering for lattices whose temperature quads
// do not fit in shared memory (L > 24), streamed through L2/HBM.
//
// One sweep = one fused launch that updates both colours in a single pass
// over the state (stream_sweep.cu, while its ring of z-planes fits in shared
// memory: L <= 58) or two colour launches (stream_colour_kernel), then, when
// the schedule asks for it, the exchange decisions (stream_decide_kernel), the
// masked exchange and the overlap counts in one pass
// (stream_exchange_overlap_kernel; stream_exchange_kernel or
// stream_overlap_kernel when only one of them is due) and the measurement
// (stream_measure_kernel).  The arithmetic of a site update, of the energies
// and of the exchange rule is the same as the cluster-resident kernel's
// (pt_kernel.cuh), so results are bit-identical to it and to the CPU oracle.
// Blocks add their counts to per-plane totals with integer atomics (any order
// gives the same sums); the kernel that reads a total clears it.  The kernels
// are launched with programmatic dependent launch (pdl_enter).
#pragma once
#include <cstdint>
#include <type_traits>

#include "stream_params.cuh"

namespace csg {

// One colour of one sweep.  blockIdx.x = quad (w, c, q), blockIdx.y = block
// of colour_spt * blockDim.x sites of that colour; each thread updates
// colour_spt sites in the 4 planes of the quad.  Consecutive blocks take the
// quads of one word at the same sites, so the word's bonds are read once from
// DRAM and then from L2.
template <bool GEN_H, bool ACC_E, bool ACC_M>
__global__ void __launch_bounds__(colour_threads<ACC_E || ACC_M>()) stream_colour_kernel(
    const __grid_constant__ StreamParams P, int p, long long s) {
    pdl_enter();
    const int L = P.L, LH = L / 2;
    const int N = L * L * L, NH = N / 2;
    const int gq = blockIdx.x;
    const int w = gq / (P.C * P.Q), c = (gq / P.Q) % P.C, q = gq % P.Q;
    uint4* Sq = reinterpret_cast<uint4*>(P.spins) + (size_t)gq * N;
    uint4* Sc = Sq + p * NH;
    const uint4* So = Sq + (1 - p) * NH;
    const uint32_t* Fw = P.bonds + (size_t)w * 3 * N;
    const uint32_t* Fc = Fw + p * NH;
    const uint32_t* Fo = Fw + (1 - p) * NH;
    const uint32_t ctr3 = kTagSweep | ((uint32_t)c << 8) | (uint32_t)q;
    const uint32_t wg = (uint32_t)w + P.word0;
    // the Philox rounds that do not depend on the site, once per launch
    const PhiloxFixed pf = philox_fix((uint32_t)s, wg, ctr3, P.k0, P.k1);
    const int lane = threadIdx.x & 31;
    uint32_t th0[4], th1[4], th2[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int t = 4 * q + k;
        th0[k] = P.tab.thr[t][0][0];
        th1[k] = P.tab.thr[t][0][1];
        th2[k] = P.tab.thr[t][0][2];
    }
    constexpr int NLV = kStreamNLV;
    constexpr int NLM = kStreamNLM;
    // Bit-sliced counters of the counting launches, one column per thread in
    // shared memory (conflict-free): held in registers they cost ~30 registers
    // per thread and with them resident blocks (measured 5 % slower at L=48).
    constexpr int BTS = colour_threads<ACC_E || ACC_M>();
    __shared__ uint32_t s_cnt[(ACC_E ? 4 * NLV : 0) + (ACC_M ? 4 * NLM : 0) + 1][BTS];
    uint32_t* ecb = &s_cnt[0][threadIdx.x];                        // [4][NLV], stride BTS
    uint32_t* mcb = &s_cnt[ACC_E ? 4 * NLV : 0][threadIdx.x];      // [4][NLM], stride BTS
    if constexpr (ACC_E || ACC_M) {
        for (int i = 0; i < (ACC_E ? 4 * NLV : 0) + (ACC_M ? 4 * NLM : 0); ++i) ecb[i * BTS] = 0;
    }
    const int PL = L * LH;  // sites of one colour in one z plane
    constexpr int BT = colour_threads<ACC_E || ACC_M>(), SPT = colour_spt<ACC_E || ACC_M>();
    const int n_base = blockIdx.y * (BT * SPT) + threadIdx.x;
    auto update_site = [&](const int n, uint32_t (&wd)[4][4]) {
        if (n >= (int)NH) return;
        // n = (z L + y) L/2 + h; divisions by multiply-high
        const int z = div_magic(n, PL, P.mag_plane);
        const int rem = n - z * PL;
        const int y = div_magic(rem, LH, P.mag_row);
        const int h = rem - y * LH;
        const int o = (y + z + p) & 1;
        const int x = 2 * h + o;
        const int nxm = o ? n : (h == 0 ? n + LH - 1 : n - 1);
        const int nxp = o ? (h == LH - 1 ? n - h : n + 1) : n;
        const int nym = y == 0 ? n + PL - LH : n - LH;
        const int nyp = y == L - 1 ? n - PL + LH : n + LH;
        const int nzm = z == 0 ? n + (int)NH - PL : n - PL;
        const int nzp = z == L - 1 ? n - (int)NH + PL : n + PL;
        const uint4 cv = Sc[n];
        const uint4 a0 = __ldg(So + nxm), a1 = __ldg(So + nxp), a2 = __ldg(So + nym),
                    a3 = __ldg(So + nyp), a4 = __ldg(So + nzm), a5 = __ldg(So + nzp);
        const uint32_t f0 = __ldg(Fo + nxm), f1 = __ldg(Fc + n);
        const uint32_t f2 = __ldg(Fo + N + nym), f3 = __ldg(Fc + N + n);
        const uint32_t f4 = __ldg(Fo + 2 * N + nzm), f5 = __ldg(Fc + 2 * N + n);
        const u32x4 r = philox_c0((uint32_t)((z * L + y) * L + x), pf);
        const uint32_t rr[4] = {r.v0, r.v1, r.v2, r.v3};
        uint32_t cw[4] = {cv.x, cv.y, cv.z, cv.w};
        const uint32_t n0w[4] = {a0.x, a0.y, a0.z, a0.w}, n1w[4] = {a1.x, a1.y, a1.z, a1.w};
        const uint32_t n2w[4] = {a2.x, a2.y, a2.z, a2.w}, n3w[4] = {a3.x, a3.y, a3.z, a3.w};
        const uint32_t n4w[4] = {a4.x, a4.y, a4.z, a4.w}, n5w[4] = {a5.x, a5.y, a5.z, a5.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t s0 = cw[k];
            const uint32_t u0 = s0 ^ n0w[k] ^ f0, u1 = s0 ^ n1w[k] ^ f1;
            const uint32_t u2 = s0 ^ n2w[k] ^ f2, u3 = s0 ^ n3w[k] ^ f3;
            const uint32_t u4 = s0 ^ n4w[k] ^ f4, u5 = s0 ^ n5w[k] ^ f5;
            const uint32_t sa = u0 ^ u1 ^ u2, ca = maj3(u0, u1, u2);
            const uint32_t sb = u3 ^ u4 ^ u5, cb = maj3(u3, u4, u5);
            uint32_t fl;
            if constexpr (GEN_H) {
                uint4 ta, tb;
                gen_thresholds(P.tab, 4 * q + k, ta, tb);
                fl = flip_gen(s0, sa, ca, sb, cb, rr[k], ta, tb, P.tab.ucut[4 * q + k][0],
                              P.tab.ucut[4 * q + k][1]);
            } else {
                fl = flip_h0(sa, ca, sb, cb, rr[k], th0[k], th1[k], th2[k]);
            }
            cw[k] = s0 ^ fl;
            // post-flip unsatisfied bonds (energy) and spins up, counted at once
            if constexpr (ACC_E) {
                wd[k][0] = sa ^ fl;
                wd[k][1] = sb ^ fl;
                wd[k][2] = ca ^ fl;
                wd[k][3] = cb ^ fl;
            }
            if constexpr (ACC_M) {
                uint32_t carry = cw[k];
#pragma unroll
                for (int l = 0; l < NLM; ++l) {
                    const uint32_t m = mcb[(k * NLM + l) * BTS];
                    mcb[(k * NLM + l) * BTS] = m ^ carry;
                    carry &= m;
                }
            }
        }
        Sc[n] = make_uint4(cw[0], cw[1], cw[2], cw[3]);
    };
    // sites in pairs: the energy counters take both at once (fewer counter
    // updates); the two updates themselves run one after the other
    static_assert(SPT % 2 == 0, "sites are counted in pairs");
#pragma unroll 1
    for (int m = 0; m < SPT; m += 2) {
        uint32_t wa[4][4] = {}, wb[4][4] = {};
        update_site(n_base + m * BT, wa);
        update_site(n_base + (m + 1) * BT, wb);
        if constexpr (ACC_E) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t v[NLV];
#pragma unroll
                for (int l = 0; l < NLV; ++l) v[l] = ecb[(k * NLV + l) * BTS];
                vc_add_2sites<NLV>(v, wa[k][0], wa[k][1], wa[k][2], wa[k][3], wb[k][0], wb[k][1],
                                   wb[k][2], wb[k][3]);
#pragma unroll
                for (int l = 0; l < NLV; ++l) ecb[(k * NLV + l) * BTS] = v[l];
            }
        }
    }
    __shared__ int sred[2][4][32];
    if (ACC_E || ACC_M) {
        uint32_t ecnt[4][NLV], mcnt[4][NLM];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
#pragma unroll
            for (int l = 0; l < NLV; ++l) ecnt[k][l] = ACC_E ? ecb[(k * NLV + l) * BTS] : 0u;
#pragma unroll
            for (int l = 0; l < NLM; ++l) mcnt[k][l] = ACC_M ? mcb[(k * NLM + l) * BTS] : 0u;
        }
        for (int i = threadIdx.x; i < 2 * 4 * 32; i += BT) (&sred[0][0][0])[i] = 0;
        __syncthreads();
        // all lanes of a block hold counters of its one quad: the 4 planes of a
        // warp in one 32x32 transpose per counter level
        if constexpr (ACC_E) {
            int cnt[4];
            packed_column_counts<NLV>(ecnt, lane, cnt);
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicAdd(&sred[0][k][lane], cnt[k]);
        }
        if constexpr (ACC_M) {
            int cnt[4];
            packed_column_counts<NLM>(mcnt, lane, cnt);
#pragma unroll
            for (int k = 0; k < 4; ++k) atomicAdd(&sred[1][k][lane], cnt[k]);
        }
        __syncthreads();
        if (threadIdx.x < 128) {
            const int k = threadIdx.x >> 5;
            const size_t o = (((size_t)w * P.C + c) * P.T + 4 * q + k) * 32 + lane;
            if constexpr (ACC_E) atomicAdd(&P.u_acc[o], sred[0][k][lane]);
            if constexpr (ACC_M) atomicAdd(&P.up_acc[o], sred[1][k][lane]);
        }
    }
}

// Exchange decisions of one round: block = (w, c), one warp per pair.  Also
// totals the energies (and magnetisations) of every plane and swaps them for
// the accepted samples.
__global__ void stream_decide_kernel(const __grid_constant__ StreamParams P, long long s, int par,
                                     bool need_M, bool do_swap, unsigned long long* boundary,
                                     unsigned long long* swap_acc, unsigned int* swap_log,
                                     long long log_row, long long log_rows) {
    pdl_enter();
    const int wc = blockIdx.x, w = wc / P.C, c = wc % P.C;
    const int T = P.T, N = P.L * P.L * P.L;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    int* E = P.energy + (size_t)wc * T * 32;
    int* M = P.magn + (size_t)wc * T * 32;
    // totals of every plane of this (word, copy), cleared for the next sweep
    int* ua = P.u_acc + (size_t)wc * T * 32;
    int* pa = P.up_acc + (size_t)wc * T * 32;
    for (int i = threadIdx.x; i < T * 32; i += blockDim.x) {
        const int u = ua[i];
        ua[i] = 0;
        int up = 0;
        if (need_M) {
            up = pa[i];
            pa[i] = 0;
        }
        E[i] = 2 * u - 3 * N;
        M[i] = need_M ? 2 * up - N : 0;
    }
    __syncthreads();
    if (!do_swap) return;
    const uint32_t wg = (uint32_t)w + P.word0;
    for (int t = par + 2 * warp; t + 1 < T; t += 2 * nwarps) {
        const int e0 = E[t * 32 + lane], e1 = E[(t + 1) * 32 + lane];
        const int m0 = M[t * 32 + lane], m1 = M[(t + 1) * 32 + lane];
        const u32x4 r = philox4x32_10((uint32_t)(lane >> 1), (uint32_t)s, wg,
                                      kTagSwap | ((uint32_t)c << 8) | (uint32_t)t, P.k0, P.k1);
        const uint32_t lo = (lane & 1) ? r.v2 : r.v0;
        const uint32_t hi = (lane & 1) ? r.v3 : r.v1;
        const double uu = (double)((((unsigned long long)hi << 32) | lo) >> 11) * 0x1p-53;
        const double dE = __dsub_rn((double)(e0 - e1), __dmul_rn(P.H, (double)(m0 - m1)));
        const double delta = __dmul_rn(__dsub_rn(P.tab.beta[t], P.tab.beta[t + 1]), dE);
        bool acc = true;
        if (delta < 0.0) {
            const double pr = exp(delta);
            if (boundary && fabs(uu - pr) <= pr * 0x1p-40) atomicAdd(boundary, 1ull);
            acc = uu < pr;
        }
        const uint32_t mask = __ballot_sync(0xFFFFFFFFu, acc);
        if (acc) {
            E[t * 32 + lane] = e1;
            E[(t + 1) * 32 + lane] = e0;
            M[t * 32 + lane] = m1;
            M[(t + 1) * 32 + lane] = m0;
        }
        if (lane == 0) {
            P.masks[(size_t)wc * T + t] = mask;
            if (swap_acc) atomicAdd(&swap_acc[(size_t)c * T + t], (unsigned long long)__popc(mask));
            if (swap_log && log_row >= 0 && log_row < log_rows)
                swap_log[(((size_t)log_row * P.W + w) * P.C + c) * T + t] = mask;
        }
    }
    // pairs that do not take part in this round keep a zero mask
    for (int t = threadIdx.x; t < T; t += blockDim.x)
        if (((t - par) & 1) || t + 1 >= T) P.masks[(size_t)wc * T + t] = 0;
}

// Masked exchange: a thread takes one site of one (w, c) and every quad of it,
// so both words of every pair (also across quads) are its own.
__global__ void stream_exchange_kernel(const __grid_constant__ StreamParams P, int par) {
    pdl_enter();
    const long N = (long)P.L * P.L * P.L;
    const int wc = blockIdx.x;
    const long n = (long)blockIdx.y * blockDim.x + threadIdx.x;
    if (n >= N) return;
    uint4* base = reinterpret_cast<uint4*>(P.spins) + (size_t)wc * P.Q * N + n;
    const uint32_t* mk = P.masks + (size_t)wc * P.T;
    if (par == 0) {  // pairs (0,1), (2,3) inside every quad
        for (int q = 0; q < P.Q; ++q) {
            uint4 v = base[(size_t)q * N];
            const uint32_t d0 = (v.x ^ v.y) & mk[4 * q], d1 = (v.z ^ v.w) & mk[4 * q + 2];
            v.x ^= d0; v.y ^= d0; v.z ^= d1; v.w ^= d1;
            base[(size_t)q * N] = v;
        }
        return;
    }
    // odd rounds: (1,2) inside a quad, (3 of quad q, 0 of quad q+1) across quads
    uint4 cur = base[0];
    for (int q = 0; q < P.Q; ++q) {
        const uint32_t d = (cur.y ^ cur.z) & mk[4 * q + 1];
        cur.y ^= d;
        cur.z ^= d;
        if (q + 1 < P.Q) {
            uint4 nxt = base[(size_t)(q + 1) * N];
            const uint32_t e = (cur.w ^ nxt.x) & mk[4 * q + 3];
            cur.w ^= e;
            nxt.x ^= e;
            base[(size_t)q * N] = cur;
            cur = nxt;
        } else {
            base[(size_t)q * N] = cur;
        }
    }
}

// Exchange and overlap in one pass (sweeps that both exchange and measure, two
// copies): blockIdx.x = word, blockIdx.y = block of 2048 sites.  A thread takes
// 4 sites of both copies and walks the quads in order; on odd rounds quad q is
// final only after its pair (3 of q, 0 of q+1) is exchanged, so each quad is
// written (and its overlap counted) one step after it is loaded.  Every word
// is read and written by exactly one thread.  The block's overlap counts are
// added to d_acc, as in stream_overlap_kernel.
__global__ void __launch_bounds__(kStreamThreads) stream_exchange_overlap_kernel(
    const __grid_constant__ StreamParams P, int par) {
    pdl_enter();
    constexpr int kSites = 4, kGroups = kOverlapSitesPerBlock / (kStreamThreads * kSites);
    static_assert(kGroups >= 1 && kGroups * kStreamThreads * kSites == kOverlapSitesPerBlock,
                  "a block covers whole groups of 4 sites per thread");
    const int N = P.L * P.L * P.L, T = P.T, Q = P.Q;
    const int w = blockIdx.x, blk = blockIdx.y, lane = threadIdx.x & 31;
    __shared__ int sD[kMaxT][32];
    for (int i = threadIdx.x; i < T * 32; i += kStreamThreads) (&sD[0][0])[i] = 0;
    __syncthreads();
    uint4* base0 = reinterpret_cast<uint4*>(P.spins) + (size_t)(w * 2 + 0) * Q * N;
    uint4* base1 = reinterpret_cast<uint4*>(P.spins) + (size_t)(w * 2 + 1) * Q * N;
    const uint32_t* mk0 = P.masks + (size_t)(w * 2 + 0) * T;
    const uint32_t* mk1 = P.masks + (size_t)(w * 2 + 1) * T;
    for (int grp = 0; grp < kGroups; ++grp) {
        int site[kSites];
#pragma unroll
        for (int i = 0; i < kSites; ++i)
            site[i] = blk * kOverlapSitesPerBlock + (grp * kSites + i) * kStreamThreads + threadIdx.x;
        uint4 prv[2][kSites], cur[2][kSites];
        // store quad qq and add its overlap counts
        auto finish = [&](int qq, uint4 (&v)[2][kSites]) {
            uint32_t x[4][kSites];
#pragma unroll
            for (int i = 0; i < kSites; ++i) {
                if (site[i] < N) {
                    base0[(size_t)qq * N + site[i]] = v[0][i];
                    base1[(size_t)qq * N + site[i]] = v[1][i];
                }
                x[0][i] = v[0][i].x ^ v[1][i].x;
                x[1][i] = v[0][i].y ^ v[1][i].y;
                x[2][i] = v[0][i].z ^ v[1][i].z;
                x[3][i] = v[0][i].w ^ v[1][i].w;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t cnt[3] = {0, 0, 0};
                vc_add4<3>(cnt, x[k][0], x[k][1], x[k][2], x[k][3]);
                atomicAdd(&sD[4 * qq + k][lane], column_count<3>(cnt, lane));
            }
        };
        for (int q = 0; q < Q; ++q) {
            const uint32_t a0 = mk0[4 * q], a1 = mk0[4 * q + 1], a2 = mk0[4 * q + 2];
            const uint32_t b0 = mk1[4 * q], b1 = mk1[4 * q + 1], b2 = mk1[4 * q + 2];
#pragma unroll
            for (int i = 0; i < kSites; ++i) {
                const bool ok = site[i] < N;
                uint4 u = ok ? base0[(size_t)q * N + site[i]] : make_uint4(0, 0, 0, 0);
                uint4 v = ok ? base1[(size_t)q * N + site[i]] : make_uint4(0, 0, 0, 0);
                if (par == 0) {  // (0,1) and (2,3) inside the quad
                    uint32_t d = (u.x ^ u.y) & a0; u.x ^= d; u.y ^= d;
                    d = (u.z ^ u.w) & a2; u.z ^= d; u.w ^= d;
                    d = (v.x ^ v.y) & b0; v.x ^= d; v.y ^= d;
                    d = (v.z ^ v.w) & b2; v.z ^= d; v.w ^= d;
                } else {  // (1,2) inside; (3 of q-1, 0 of q) across
                    uint32_t d = (u.y ^ u.z) & a1; u.y ^= d; u.z ^= d;
                    d = (v.y ^ v.z) & b1; v.y ^= d; v.z ^= d;
                    if (q > 0) {
                        d = (prv[0][i].w ^ u.x) & mk0[4 * q - 1]; prv[0][i].w ^= d; u.x ^= d;
                        d = (prv[1][i].w ^ v.x) & mk1[4 * q - 1]; prv[1][i].w ^= d; v.x ^= d;
                    }
                }
                cur[0][i] = u;
                cur[1][i] = v;
            }
            if (q > 0) finish(q - 1, prv);
#pragma unroll
            for (int i = 0; i < kSites; ++i) {
                prv[0][i] = cur[0][i];
                prv[1][i] = cur[1][i];
            }
        }
        finish(Q - 1, prv);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < T * 32; i += kStreamThreads) {
        const int t = i >> 5, b = i & 31;
        atomicAdd(&P.d_acc[((size_t)w * T + t) * 32 + b], sD[t][b]);
    }
}

// Overlap counts: blockIdx.x = (w, q), blockIdx.y = block of sites; each
// thread kOverlapSPT sites; the block's counts are added to d_acc.
__global__ void __launch_bounds__(kStreamThreads) stream_overlap_kernel(const __grid_constant__ StreamParams P) {
    pdl_enter();
    const long N = (long)P.L * P.L * P.L;
    const int wq = blockIdx.x, w = wq / P.Q, q = wq % P.Q;
    const int lane = threadIdx.x & 31;
    const uint4* A = reinterpret_cast<const uint4*>(P.spins) + ((size_t)(w * P.C + 0) * P.Q + q) * N;
    const uint4* B = reinterpret_cast<const uint4*>(P.spins) + ((size_t)(w * P.C + 1) * P.Q + q) * N;
    constexpr int NL = kOverlapNL;
    uint32_t dc[4][NL];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int l = 0; l < NL; ++l) dc[k][l] = 0;
    const long n_base = (long)blockIdx.y * kOverlapSitesPerBlock + threadIdx.x;
    for (int m = 0; m < kOverlapSPT; ++m) {
        const long n = n_base + (long)m * kStreamThreads;
        uint4 x = make_uint4(0, 0, 0, 0);
        if (n < N) {
            const uint4 a = __ldg(A + n), b = __ldg(B + n);
            x = make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
        }
        const uint32_t xs[4] = {x.x, x.y, x.z, x.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uint32_t carry = xs[k];
#pragma unroll
            for (int l = 0; l < NL; ++l) {
                const uint32_t t = dc[k][l] & carry;
                dc[k][l] ^= carry;
                carry = t;
            }
        }
    }
    __shared__ int sred[4][32];
    for (int i = threadIdx.x; i < 128; i += kStreamThreads) (&sred[0][0])[i] = 0;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) atomicAdd(&sred[k][lane], column_count<NL>(dc[k], lane));
    __syncthreads();
    if (threadIdx.x < 128) {
        const int k = threadIdx.x >> 5;
        atomicAdd(&P.d_acc[((size_t)w * P.T + 4 * q + k) * 32 + lane], sred[k][lane]);
    }
}

// Measurement accumulators from the energies and the overlap totals:
// blockIdx.x = (word, temperature), thread = (copy, sample); the first 32
// threads also take (and clear) the plane's overlap totals.
__global__ void stream_measure_kernel(const __grid_constant__ StreamParams P, bool need_M,
                                      StreamObs O) {
    pdl_enter();
    const int w = blockIdx.x / P.T, t = blockIdx.x % P.T, T = P.T, N = P.L * P.L * P.L;
    const int c = threadIdx.x >> 5, b = threadIdx.x & 31;
    if (c < P.C) {
        const size_t o = (((size_t)w * P.C + c) * T + t) * 32 + b;
        const int e = P.energy[o], m = P.magn[o];
        if (O.e_sum) atomicAdd(reinterpret_cast<unsigned long long*>(O.e_sum + o), (unsigned long long)(long long)e);
        if (O.e_last) O.e_last[o] = e;
        if (need_M) {
            if (O.m_sum) atomicAdd(reinterpret_cast<unsigned long long*>(O.m_sum + o), (unsigned long long)(long long)m);
            if (O.m_last) O.m_last[o] = m;
        }
    }
    if (P.C != 2 || c != 0) return;
    int* dp = P.d_acc + ((size_t)w * T + t) * 32 + b;
    const int D = *dp;
    *dp = 0;
    const long long Qv = (long long)N - 2LL * D;
    const unsigned long long q2 = (unsigned long long)(Qv * Qv);
    const size_t o = ((size_t)w * T + t) * 32 + b;
    if (O.q_sum) atomicAdd(reinterpret_cast<unsigned long long*>(O.q_sum + o), (unsigned long long)Qv);
    if (O.q2_sum) atomicAdd(reinterpret_cast<unsigned long long*>(O.q2_sum + o), q2);
    if (O.q4_sum) {
        const unsigned long long lo = q2 * q2, hi = __umul64hi(q2, q2);
        atomicAdd(O.q4_sum + 2 * o, lo & 0xFFFFFFFFull);
        atomicAdd(O.q4_sum + 2 * o + 1, (lo >> 32) | (hi << 32));
    }
    if (O.hist) atomicAdd(&O.hist[(size_t)t * (N + 1) + D], 1u);
    if (O.d_last) O.d_last[o] = D;
}

}  // namespace csg
