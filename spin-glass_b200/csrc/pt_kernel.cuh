// pt_kernel.cuh — cluster-resident parallel-tempering kernel for sm_100a.
//
// Work decomposition.  A thread-block cluster owns one sample word w (32
// disorder samples) with all its copies and temperatures.  The word's
// C*T/4 temperature quads (4 planes of N uint32 each, stored as one uint4 per
// site) are split over the K CTAs of the cluster, Qc quads per CTA, and stay
// in shared memory for the whole launch (a section of sweeps).  Nothing but
// the bonds (read-only, through L1) touches global memory between the load at
// the start and the store at the end.
//
// Per sweep (reference: perform_MC_steps, eamsim.cu:112-208):
//   phase 0 / phase 1 — every team of TPQ threads updates the sites of one
//     colour of its quad; a thread handles one site for the 4 temperatures of
//     the quad with one Philox block, counts unsatisfied bonds with two full
//     adders per triple and takes the flip mask from the threshold table.
//   energies — while phase 1 runs, the post-flip unsatisfied-bond counts are
//     added into bit-sliced per-thread counters (each bond has exactly one
//     colour-1 end); warps reduce them with a 32x32 bit transpose + popc.
//   exchange (perform_PT_shuffle/shuffle, eamsim.cu:43-90, 211-330) — the CTA
//     owning plane t decides pair (t,t+1) for the 32 samples (FP64 exp on the
//     device) and swaps the accepted samples' configurations, reaching into
//     the neighbouring CTA's shared memory when t+1 lives there.
//   measurement (compute_q, eamsim.cu:451-511) — popcount overlaps of the two
//     copies, integer moments and a histogram.
#pragma once
#include <cooperative_groups.h>

#include <cstdint>
#include <type_traits>

#include "philox.cuh"

namespace csg {
namespace cgx = cooperative_groups;

constexpr int kMaxT = 64;
constexpr int kMaxThreads = 512;  // CTA size cap: keeps 128 registers per thread available

struct PtTables {
    double beta[kMaxT];
    uint32_t thr[kMaxT][2][7];  // acceptance thresholds, valid for U < ucut
    uint8_t ucut[kMaxT][2];     // first U that is always accepted
};

struct PtParams {
    uint32_t* spins;
    const uint32_t* bonds;
    long long* e_sum;
    long long* m_sum;
    long long* q_sum;
    long long* q2_sum;
    unsigned long long* q4_sum;
    unsigned int* hist;
    int* e_last;
    int* m_last;
    int* d_last;
    unsigned long long* swap_acc;
    unsigned int* swap_log;
    long long swap_log_rounds;
    long long swap_round0;
    unsigned long long* boundary;
    double H;
    uint32_t k0, k1;
    uint32_t word0;  // global index of word 0 (Philox counter word 2)
    int W, C, T, Q;
    int K, Qc;
    long long sweep0;
    const long long* sweep_dev;  // if set, added to sweep0 (lets a captured graph advance)
    int n_sweeps;
    int sps, spm;
    long long meas_start;
    int flags;
    PtTables tab;
};

constexpr int kFlagMeasureM = 1;

constexpr int bit_length(int v) {
    int b = 0;
    while (v > 0) {
        ++b;
        v >>= 1;
    }
    return b;
}

// Threads per quad for each lattice side: about 16 sites of each colour per
// thread, a multiple of the warp size.
constexpr int tpq_for(int L) {
    return L <= 6 ? 32 : L <= 10 ? 64 : L == 12 ? 96 : L <= 16 ? 128 : L == 18 ? 192
           : L == 20 ? 256 : L == 22 ? 352 : 448;
}

template <int L>
struct LCfg {
    static constexpr int LH = L / 2;
    static constexpr int N = L * L * L;
    static constexpr int NH = N / 2;
    static constexpr int TPQ = tpq_for(L);
    static constexpr int SPT = (NH + TPQ - 1) / TPQ;          // sites per thread per colour
    static constexpr int NLV = bit_length(6 * SPT);           // energy counter levels
    static constexpr int MPT = (N + 4 * TPQ - 1) / (4 * TPQ); // 4-site groups per thread
    static constexpr int NLD = bit_length(4 * MPT);           // magnetisation counter levels
    static constexpr int MPH = (NH + 4 * TPQ - 1) / (4 * TPQ); // 4-site groups per half lattice
    static constexpr int NLH = bit_length(4 * MPH);           // overlap counter levels
};

__device__ __forceinline__ uint32_t maj3(uint32_t a, uint32_t b, uint32_t c) {
    return (a & b) | (a & c) | (b & c);
}

#define CSG_FA(s, cy, a, b, c)                             \
    do {                                                   \
        const uint32_t fa_a = (a), fa_b = (b), fa_c = (c); \
        (s) = fa_a ^ fa_b ^ fa_c;                          \
        (cy) = maj3(fa_a, fa_b, fa_c);                     \
    } while (0)

// Bit-sliced counter update: value += a1 + a2 + 2*(a3 + a4).
template <int NLV>
__device__ __forceinline__ void vc_add_site(uint32_t (&v)[NLV], uint32_t a1, uint32_t a2,
                                            uint32_t a3, uint32_t a4) {
    uint32_t k1, k2a, k2b, k3;
    CSG_FA(v[0], k1, v[0], a1, a2);
    CSG_FA(v[1], k2a, v[1], a3, a4);
    k2b = v[1] & k1;
    v[1] ^= k1;
    if constexpr (NLV > 2) {
        CSG_FA(v[2], k3, v[2], k2a, k2b);
#pragma unroll
        for (int l = 3; l < NLV; ++l) {
            const uint32_t t = v[l] & k3;
            v[l] ^= k3;
            k3 = t;
        }
    }
}

// Two sites at once: value += a1+a2+b1+b2 + 2*(a3+a4+b3+b4).
template <int NLV>
__device__ __forceinline__ void vc_add_2sites(uint32_t (&v)[NLV], uint32_t a1, uint32_t a2,
                                              uint32_t a3, uint32_t a4, uint32_t b1, uint32_t b2,
                                              uint32_t b3, uint32_t b4) {
    uint32_t k1a, k1b, k2a, k2b, k2c, k3a, k3b;
    CSG_FA(v[0], k1a, v[0], a1, a2);
    CSG_FA(v[0], k1b, v[0], b1, b2);
    CSG_FA(v[1], k2a, v[1], a3, a4);
    CSG_FA(v[1], k2b, v[1], b3, b4);
    CSG_FA(v[1], k2c, v[1], k1a, k1b);
    CSG_FA(v[2], k3a, v[2], k2a, k2b);
    k3b = v[2] & k2c;
    v[2] ^= k2c;
    if constexpr (NLV > 3) {
        uint32_t k4;
        CSG_FA(v[3], k4, v[3], k3a, k3b);
#pragma unroll
        for (int l = 4; l < NLV; ++l) {
            const uint32_t t = v[l] & k4;
            v[l] ^= k4;
            k4 = t;
        }
    }
}

// Four single-weight words at once: value += x1 + x2 + x3 + x4.
template <int NLV>
__device__ __forceinline__ void vc_add4(uint32_t (&v)[NLV], uint32_t x1, uint32_t x2, uint32_t x3,
                                        uint32_t x4) {
    uint32_t k1a, k1b, k2;
    CSG_FA(v[0], k1a, v[0], x1, x2);
    CSG_FA(v[0], k1b, v[0], x3, x4);
    CSG_FA(v[1], k2, v[1], k1a, k1b);
#pragma unroll
    for (int l = 2; l < NLV; ++l) {
        const uint32_t t = v[l] & k2;
        v[l] ^= k2;
        k2 = t;
    }
}

// Column popcount of a 32x32 bit matrix held one row per lane: returns, in
// lane j, the number of lanes whose bit j is set.  Five butterfly stages of a
// bit transpose (shuffle, funnel rotate, bit select), then popc.
__device__ __forceinline__ int column_popc(uint32_t v, int lane) {
#pragma unroll
    for (int d = 16; d >= 1; d >>= 1) {
        const uint32_t m = d == 16 ? 0x0000FFFFu
                         : d == 8  ? 0x00FF00FFu
                         : d == 4  ? 0x0F0F0F0Fu
                         : d == 2  ? 0x33333333u
                                   : 0x55555555u;
        const bool upper = (lane & d) != 0;
        const uint32_t t = __shfl_xor_sync(0xFFFFFFFFu, v, d);
        const uint32_t rot = __funnelshift_r(t, t, upper ? d : 32 - d);
        const uint32_t keep = upper ? ~m : m;
        v = (v & keep) | (rot & ~keep);
    }
    return __popc(v);
}

template <int NLV>
__device__ __forceinline__ int column_count(const uint32_t (&v)[NLV], int lane) {
    int s = 0;
#pragma unroll
    for (int l = 0; l < NLV; ++l) s += column_popc(v[l], lane) << l;
    return s;
}

// Flip mask at H = 0: U >= 3 always accepted; U = 2, 1, 0 accepted when the
// draw is below thr[U] (t2, t1, t0; t0 <= t1 <= t2).
__device__ __forceinline__ uint32_t flip_h0(uint32_t sa, uint32_t ca, uint32_t sb, uint32_t cb,
                                            uint32_t r, uint32_t t0, uint32_t t1, uint32_t t2) {
    const uint32_t v = sa | sb;
    const uint32_t ge1 = ca | cb | v;
    const uint32_t ge2 = ca | cb | (sa & sb);
    const uint32_t ge3 = maj3(ca, cb, v);
    uint32_t f = ge3;
    f = (r < t2) ? ge2 : f;
    f = (r < t1) ? ge1 : f;
    f = (r < t0) ? 0xFFFFFFFFu : f;
    return f;
}

// General field, 0 <= H <= 4.  A flip of centre spin s with U unsatisfied
// bonds is accepted iff U >= ucut_s (dE <= 0) or the draw r < thr[s][U].
// thr[s][U] does not decrease with U and is 0xFFFFFFFF from ucut_s on, and
// ucut_0 <= 3, ucut_1 <= 5, so walking U down from there the accepted set is
// {U >= the smallest U with r < thr[s][U]} - a select chain like the H = 0
// rule.  Only the draw r = 0xFFFFFFFF, below none of the thresholds, needs the
// cut itself.  ta = {thr0[0], thr0[1], thr0[2], thr1[0]},
// tb = {thr1[1], thr1[2], thr1[3], thr1[4]}.
__device__ __forceinline__ uint32_t flip_gen(uint32_t s0, uint32_t sa, uint32_t ca, uint32_t sb,
                                             uint32_t cb, uint32_t r, const uint4 ta, const uint4 tb,
                                             int uc0, int uc1) {
    // U = sa + sb + 2(ca + cb): U >= 4 needs both carries, or one carry and
    // both sum bits; U >= 5 and U >= 6 need both carries.
    const uint32_t v = sa | sb, cx = ca | cb, cc = ca & cb;
    const uint32_t ge1 = cx | v, ge2 = cx | (sa & sb), ge3 = maj3(ca, cb, v);
    const uint32_t ge4 = cc | (cx & sa & sb), ge5 = cc & v;
    uint32_t g0 = ge3;
    g0 = (r < ta.z) ? ge2 : g0;
    g0 = (r < ta.y) ? ge1 : g0;
    g0 = (r < ta.x) ? 0xFFFFFFFFu : g0;
    uint32_t g1 = ge5;
    g1 = (r < tb.w) ? ge4 : g1;
    g1 = (r < tb.z) ? ge3 : g1;
    g1 = (r < tb.y) ? ge2 : g1;
    g1 = (r < tb.x) ? ge1 : g1;
    g1 = (r < ta.w) ? 0xFFFFFFFFu : g1;
    if (r == 0xFFFFFFFFu) {  // accepted: exactly U >= ucut
        const uint32_t ge[8] = {0xFFFFFFFFu, ge1, ge2, ge3, ge4, ge5, cc & sa & sb, 0u};
        g0 = ge[uc0 & 7];
        g1 = ge[uc1 & 7];
    }
    return (s0 & g1) | (~s0 & g0);
}

// The thresholds of plane t in the layout flip_gen takes.
__host__ __device__ inline void gen_thresholds(const PtTables& tab, int t, uint4& ta, uint4& tb) {
    ta = make_uint4(tab.thr[t][0][0], tab.thr[t][0][1], tab.thr[t][0][2], tab.thr[t][1][0]);
    tb = make_uint4(tab.thr[t][1][1], tab.thr[t][1][2], tab.thr[t][1][3], tab.thr[t][1][4]);
}

// Shared-memory layout of one CTA (dynamic):
//   uint32 planes[Qc][4][N] (the 4 temperature planes of each quad as separate
//   arrays, so that every access of one plane by a warp is conflict-free);
//   int sE[Qc*4][32]; int sD[Qc*4][32];
//   int sM[Qc*4][32]                      (only with magnetisations)
//   uint4 sThr[Qc*4][2]; uint8 sUcut[Qc*4][2]   (only for H != 0)
// The exchange masks of a round live in the first 2*Qc words of sD, which is
// cleared again before the overlap counts are added.  At L=16 with 3 quads the
// H=0 layout is 195 KB, under the 196 KB carve-out, so the 48 KB of bonds of
// the word stay in L1.
template <int L>
struct SmemMap {
    static __host__ __device__ size_t bytes(int Qc, bool has_m, bool gen) {
        return (size_t)Qc * LCfg<L>::N * 16 + (size_t)Qc * 4 * 32 * 4 * (has_m ? 3 : 2) +
               (gen ? (size_t)Qc * 4 * 32 + (size_t)Qc * 4 * 2 : 0);
    }
};

template <int L, bool GEN_H>
__global__ void __launch_bounds__(kMaxThreads) pt_resident_kernel(const __grid_constant__ PtParams P) {
    using CF = LCfg<L>;
    constexpr int N = CF::N, NH = CF::NH, LH = CF::LH, TPQ = CF::TPQ;
    constexpr int NLV = CF::NLV, NLD = CF::NLD, NLH = CF::NLH;

    cgx::cluster_group cluster = cgx::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int Qc = P.Qc, Q = P.Q, T = P.T, C = P.C;
    const int w = blockIdx.x / P.K;
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    const int j = tid / TPQ;
    const int lt = tid - j * TPQ;
    // Quad g of the word holds copy g % C and temperatures 4(g / C)..4(g / C)+3:
    // the copies of one temperature quad sit side by side, so that with two
    // copies most overlaps are counted from the CTA's own shared memory.
    const int g = rank * Qc + j;
    const int c = g % C;
    const int q = g / C;
    const int warp = tid >> 5, lane = tid & 31, nwarps = nthreads >> 5;

    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* S = reinterpret_cast<uint32_t*>(smem_raw);  // planes[Qc][4][N]
    // the 4 planes of a quad at one site
    auto ld4 = [](const uint32_t* b, int i) {
        return make_uint4(b[i], b[N + i], b[2 * N + i], b[3 * N + i]);
    };
    auto st4 = [](uint32_t* b, int i, uint4 v) {
        b[i] = v.x;
        b[N + i] = v.y;
        b[2 * N + i] = v.z;
        b[3 * N + i] = v.w;
    };
    const bool has_M = GEN_H || (P.flags & kFlagMeasureM);
    int* sE = reinterpret_cast<int*>(smem_raw + (size_t)Qc * N * 16);
    int* sD = sE + Qc * 4 * 32;
    int* sM = sD + Qc * 4 * 32;  // valid only when has_M
    uint32_t* sMask = reinterpret_cast<uint32_t*>(sD);
    uint4* sThr = reinterpret_cast<uint4*>(sM + (has_M ? Qc * 4 * 32 : 0));  // 16-byte aligned
    uint8_t* sUcut = reinterpret_cast<uint8_t*>(sThr + Qc * 4 * 2);

    // global offset of local quad jj (layout [W][C][T/4][N])
    auto quad_base = [&](int jj) {
        const int gg = rank * Qc + jj;
        return ((size_t)(w * C + gg % C) * Q + gg / C) * N;
    };
    // ---- load this CTA's quads ----
    {
        const uint4* src = reinterpret_cast<const uint4*>(P.spins);
        for (int i = tid; i < Qc * N; i += nthreads) {
            const int jj = i / N, n = i - jj * N;
            st4(S + (size_t)jj * 4 * N, n, src[quad_base(jj) + n]);
        }
    }
    if constexpr (GEN_H) {
        for (int pl = tid; pl < Qc * 4; pl += nthreads) {
            const int gg = rank * Qc + pl / 4;
            const int t = 4 * (gg / C) + (pl & 3);
            gen_thresholds(P.tab, t, sThr[2 * pl], sThr[2 * pl + 1]);
        }
        for (int i = tid; i < Qc * 4 * 2; i += nthreads) {
            const int pl = i / 2;
            const int gg = rank * Qc + pl / 4;
            const int t = 4 * (gg / C) + (pl & 3);
            sUcut[i] = P.tab.ucut[t][i & 1];
        }
    }
    uint32_t th0[4], th1[4], th2[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int t = 4 * q + k;
        th0[k] = P.tab.thr[t][0][0];
        th1[k] = P.tab.thr[t][0][1];
        th2[k] = P.tab.thr[t][0][2];
    }
    __syncthreads();

    uint32_t* Sq = S + (size_t)j * 4 * N;
    const uint32_t* Fw = P.bonds + (size_t)w * 3 * N;
    const uint32_t ctr3 = kTagSweep | ((uint32_t)c << 8) | (uint32_t)q;
    const uint32_t wg = (uint32_t)w + P.word0;  // global sample word
    const uint4* thrq = sThr + (size_t)j * 4 * 2;
    // the cuts of this quad's 4 planes, one byte each (used only for r = 0xFFFFFFFF)
    uint32_t uc0 = 0, uc1 = 0;
    if constexpr (GEN_H) {
        const uint8_t* ucq = sUcut + (size_t)j * 4 * 2;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            uc0 |= (uint32_t)ucq[2 * k] << (8 * k);
            uc1 |= (uint32_t)ucq[2 * k + 1] << (8 * k);
        }
    }

    const long long sweep_base = P.sweep0 + (P.sweep_dev ? *P.sweep_dev : 0ll);
    for (int it = 0; it < P.n_sweeps; ++it) {
        const long long s = sweep_base + it;
        const bool do_swap = P.sps > 0 && ((s + 1) % P.sps) == 0;
        const bool do_meas = P.spm > 0 && ((s + 1) % P.spm) == 0 && s >= P.meas_start;
        const bool need_E = do_swap || do_meas;
        const bool need_M = need_E && (GEN_H || (do_meas && (P.flags & kFlagMeasureM)));
        const uint32_t s32 = (uint32_t)s;

        if (need_E)  // sE, sD and (if present) sM are contiguous
            for (int i = tid; i < Qc * 4 * 32 * (has_M ? 3 : 2); i += nthreads) sE[i] = 0;

        uint32_t ecnt[4][NLV];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int l = 0; l < NLV; ++l) ecnt[k][l] = 0;

        // one colour of the checkerboard; ACC: also add the post-flip
        // unsatisfied-bond counts into the energy counters
        auto colour_pass = [&](const int p, auto acc_tag) {
            constexpr bool ACC = decltype(acc_tag)::value;
            uint32_t* Sc = Sq + p * NH;
            const uint32_t* So = Sq + (1 - p) * NH;
            const uint32_t* Fc = Fw + p * NH;
            const uint32_t* Fo = Fw + (1 - p) * NH;
#pragma unroll 1
                for (int n0 = lt; n0 < NH; n0 += 2 * TPQ) {
                    uint32_t wA[4][4], wB[4][4];
                    bool hasB = false;
    #pragma unroll
                    for (int sidx = 0; sidx < 2; ++sidx) {
                        const int n = n0 + sidx * TPQ;
                        if (sidx == 1 && n >= NH) break;
                        if (sidx == 1) hasB = true;
                        const int z = n / (L * LH);
                        const int rem = n - z * (L * LH);
                        const int y = rem / LH;
                        const int h = rem - y * LH;
                        const int o = (y + z + p) & 1;
                        const int x = 2 * h + o;
                        const int hxm = o ? h : (h == 0 ? LH - 1 : h - 1);
                        const int hxp = o ? (h == LH - 1 ? 0 : h + 1) : h;
                        const int ym = y == 0 ? L - 1 : y - 1, yp = y == L - 1 ? 0 : y + 1;
                        const int zm = z == 0 ? L - 1 : z - 1, zp = z == L - 1 ? 0 : z + 1;
                        const int row = (z * L + y) * LH;
                        const int nxm = row + hxm, nxp = row + hxp;
                        const int nym = (z * L + ym) * LH + h, nyp = (z * L + yp) * LH + h;
                        const int nzm = (zm * L + y) * LH + h, nzp = (zp * L + y) * LH + h;

                        uint4 cv = ld4(Sc, n);
                        const uint4 a0 = ld4(So, nxm), a1 = ld4(So, nxp), a2 = ld4(So, nym),
                                    a3 = ld4(So, nyp), a4 = ld4(So, nzm), a5 = ld4(So, nzp);
                        const uint32_t f0 = __ldg(Fo + nxm), f1 = __ldg(Fc + n);
                        const uint32_t f2 = __ldg(Fo + N + nym), f3 = __ldg(Fc + N + n);
                        const uint32_t f4 = __ldg(Fo + 2 * N + nzm), f5 = __ldg(Fc + 2 * N + n);
                        const u32x4 r = philox4x32_10((uint32_t)((z * L + y) * L + x), s32, wg,
                                                      ctr3, P.k0, P.k1);
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
                            if constexpr (GEN_H)
                                fl = flip_gen(s0, sa, ca, sb, cb, rr[k], thrq[2 * k], thrq[2 * k + 1],
                                              (int)((uc0 >> (8 * k)) & 0xFF),
                                              (int)((uc1 >> (8 * k)) & 0xFF));
                            else
                                fl = flip_h0(sa, ca, sb, cb, rr[k], th0[k], th1[k], th2[k]);
                            cw[k] = s0 ^ fl;
                            if constexpr (ACC) {
                                uint32_t(&wd)[4] = sidx == 0 ? wA[k] : wB[k];
                                wd[0] = sa ^ fl;
                                wd[1] = sb ^ fl;
                                wd[2] = ca ^ fl;
                                wd[3] = cb ^ fl;
                            }
                        }
                        st4(Sc, n, make_uint4(cw[0], cw[1], cw[2], cw[3]));
                    }
                    if constexpr (ACC) {
    #pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            if (hasB)
                                vc_add_2sites<NLV>(ecnt[k], wA[k][0], wA[k][1], wA[k][2], wA[k][3],
                                                   wB[k][0], wB[k][1], wB[k][2], wB[k][3]);
                            else
                                vc_add_site<NLV>(ecnt[k], wA[k][0], wA[k][1], wA[k][2], wA[k][3]);
                        }
                    }
                }
        };
        colour_pass(0, std::false_type{});
        __syncthreads();
        if (need_E)
            colour_pass(1, std::true_type{});
        else
            colour_pass(1, std::false_type{});
        __syncthreads();

        if (!need_E) continue;

        // ---- per-sample unsatisfied-bond totals of this CTA's planes ----
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int cnt = column_count<NLV>(ecnt[k], lane);
            atomicAdd(&sE[(j * 4 + k) * 32 + lane], cnt);
        }
        if (need_M) {
            uint32_t mc[4][NLD];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int l = 0; l < NLD; ++l) mc[k][l] = 0;
#pragma unroll 1
            for (int n = lt; n < N; n += 4 * TPQ) {
                uint4 v[4];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int nn = n + u * TPQ;
                    v[u] = nn < N ? ld4(Sq, nn) : make_uint4(0, 0, 0, 0);
                }
                vc_add4<NLD>(mc[0], v[0].x, v[1].x, v[2].x, v[3].x);
                vc_add4<NLD>(mc[1], v[0].y, v[1].y, v[2].y, v[3].y);
                vc_add4<NLD>(mc[2], v[0].z, v[1].z, v[2].z, v[3].z);
                vc_add4<NLD>(mc[3], v[0].w, v[1].w, v[2].w, v[3].w);
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int cnt = column_count<NLD>(mc[k], lane);
                atomicAdd(&sM[(j * 4 + k) * 32 + lane], cnt);
            }
        }
        __syncthreads();
        // convert to E_b = 2U - 3N and M = 2 n_up - N
        for (int i = tid; i < Qc * 4 * 32; i += nthreads) {
            sE[i] = 2 * sE[i] - 3 * N;
            if (need_M) sM[i] = 2 * sM[i] - N;
        }

        uint32_t mask_keep = 0;  // exchange mask word this thread later finds in sD
        if (do_swap) {
            const long long round = (s + 1) / P.sps - 1;
            const int par = (int)(round & 1);
            // the uniform of this lane for the warp's first pair does not depend
            // on the energies: draw it while the cluster barrier is pending
            auto uniform_for = [&](int pi) {
                const int gg = rank * Qc + (pi >> 1);
                const int cc = gg % C, t = 4 * (gg / C) + par + 2 * (pi & 1);
                const u32x4 r = philox4x32_10((uint32_t)(lane >> 1), s32, wg,
                                              kTagSwap | ((uint32_t)cc << 8) | (uint32_t)t,
                                              P.k0, P.k1);
                const uint32_t lo = (lane & 1) ? r.v2 : r.v0;
                const uint32_t hi = (lane & 1) ? r.v3 : r.v1;
                return (double)((((unsigned long long)hi << 32) | lo) >> 11) * 0x1p-53;
            };
            const double u_first = warp < 2 * Qc ? uniform_for(warp) : 0.0;
            // Odd rounds pair plane 3 of a quad with plane 0 of the next, whose
            // energies may live in another CTA; even rounds pair planes of one
            // quad, so a CTA barrier suffices (the choice is the same in every
            // CTA of the cluster).
            if (par) cluster.sync();
            else __syncthreads();
            for (int pi = warp; pi < 2 * Qc; pi += nwarps) {
                const int jj = pi >> 1;
                const int tq = par + 2 * (pi & 1);
                const int gg = rank * Qc + jj;
                const int cc = gg % C, qq = gg / C;
                const int t = 4 * qq + tq;
                uint32_t mask = 0;
                if (t + 1 < T) {
                    int* E0 = sE + (jj * 4 + tq) * 32;
                    int* M0 = sM + (jj * 4 + tq) * 32;
                    int *E1, *M1;
                    if (tq < 3) {
                        E1 = E0 + 32;
                        M1 = M0 + 32;
                    } else {
                        const int g2 = gg + C, r2 = g2 / Qc, j2 = g2 - r2 * Qc;  // next quad, same copy
                        E1 = cluster.map_shared_rank(sE + j2 * 4 * 32, r2);
                        M1 = cluster.map_shared_rank(sM + j2 * 4 * 32, r2);
                    }
                    const int e0 = E0[lane], e1 = E1[lane];
                    const int m0 = need_M ? M0[lane] : 0, m1 = need_M ? M1[lane] : 0;
                    const double u = pi == warp ? u_first : uniform_for(pi);
                    const double dE = __dsub_rn((double)(e0 - e1), __dmul_rn(P.H, (double)(m0 - m1)));
                    const double delta = __dmul_rn(__dsub_rn(P.tab.beta[t], P.tab.beta[t + 1]), dE);
                    bool acc = true;
                    if (delta < 0.0) {
                        const double pr = exp(delta);
                        if (P.boundary && fabs(u - pr) <= pr * 0x1p-40) atomicAdd(P.boundary, 1ull);
                        acc = u < pr;
                    }
                    mask = __ballot_sync(0xFFFFFFFFu, acc);
                    if (acc) {
                        E0[lane] = e1;
                        E1[lane] = e0;
                        if (need_M) {
                            M0[lane] = m1;
                            M1[lane] = m0;
                        }
                    }
                    if (lane == 0) {
                        if (P.swap_acc)
                            atomicAdd(&P.swap_acc[(size_t)cc * T + t],
                                      (unsigned long long)__popc(mask));
                        // log row = global round index - round of row 0
                        const long long k = round - P.swap_round0;
                        if (P.swap_log && k >= 0 && k < P.swap_log_rounds)
                            P.swap_log[(((size_t)k * P.W + w) * C + cc) * T + t] = mask;
                    }
                }
                if (lane == 0) sMask[pi] = mask;
            }
            __syncthreads();
            // masked exchange of the accepted samples' configurations; on odd
            // rounds the pair (3 of quad g, 0 of quad g+1) crosses quads (and
            // CTAs when g+1 lives in another CTA of the cluster)
            const uint32_t mA = sMask[2 * j], mB = sMask[2 * j + 1];
            // the mask words stay in sD: the thread that later reads word tid
            // of the overlap counts subtracts them again
            if (tid < 2 * Qc) mask_keep = sMask[tid];
            // exchange the masked bits of two planes, chunks of 8 sites: all
            // loads (some perhaps from a peer CTA) are in flight before the
            // first store
            auto exchange = [&](uint32_t* pa, uint32_t* pb, const uint32_t m) {
                constexpr int CH = 8;
                for (int n0 = lt; n0 < N; n0 += CH * TPQ) {
                    uint32_t a[CH], b[CH];
#pragma unroll
                    for (int u = 0; u < CH; ++u) {
                        const int n = n0 + u * TPQ;
                        a[u] = n < N ? pa[n] : 0u;
                        b[u] = n < N ? pb[n] : 0u;
                    }
#pragma unroll
                    for (int u = 0; u < CH; ++u) {
                        const int n = n0 + u * TPQ;
                        if (n < N) {
                            const uint32_t d = (a[u] ^ b[u]) & m;
                            pa[n] = a[u] ^ d;
                            pb[n] = b[u] ^ d;
                        }
                    }
                }
            };
            if (par == 0) {
                if (mA) exchange(Sq, Sq + N, mA);
                if (mB) exchange(Sq + 2 * N, Sq + 3 * N, mB);
            } else {
                if (mA) exchange(Sq + N, Sq + 2 * N, mA);
                if (mB) {
                    const int g2 = g + C, r2 = g2 / Qc, j2 = g2 - r2 * Qc;  // next quad, same copy
                    uint32_t* nb = r2 == rank ? S + (size_t)j2 * 4 * N
                                              : cluster.map_shared_rank(S + (size_t)j2 * 4 * N, r2);
                    exchange(Sq + 3 * N, nb, mB);
                }
            }
            // exchanges (local and, on odd rounds, remote) complete; a
            // measurement then reads the other copy's planes, perhaps remote
            if (par || do_meas) cluster.sync();
            else __syncthreads();
        } else {
            __syncthreads();
        }

        if (do_meas) {
            for (int i = tid; i < Qc * 4 * 32; i += nthreads) {
                const int pl = i >> 5, b = i & 31;
                const int gg = rank * Qc + (pl >> 2);
                const int cc = gg % C, t = 4 * (gg / C) + (pl & 3);
                const size_t o = (((size_t)w * C + cc) * T + t) * 32 + b;
                if (P.e_sum) atomicAdd(reinterpret_cast<unsigned long long*>(P.e_sum + o),
                                       (unsigned long long)(long long)sE[i]);
                if (P.e_last) P.e_last[o] = sE[i];
                if (need_M) {
                    if (P.m_sum) atomicAdd(reinterpret_cast<unsigned long long*>(P.m_sum + o),
                                           (unsigned long long)(long long)sM[i]);
                    if (P.m_last) P.m_last[o] = sM[i];
                }
            }
            if (C == 2) {
                if (!do_swap) cluster.sync();  // partner copies finished the sweep
                // Overlap of quad q: the copy-0 team counts the colour-0 sites,
                // the copy-1 team the colour-1 sites; both add into the counts of
                // the copy-0 quad's CTA.
                const int gp = g ^ 1;  // the other copy's quad
                const int rp = gp / Qc, jp = gp - rp * Qc;
                const uint32_t* Sp = rp == rank ? S + (size_t)jp * 4 * N
                                                : cluster.map_shared_rank(S + (size_t)jp * 4 * N, rp);
                const uint32_t* Sh = Sq + c * NH;
                Sp += c * NH;
                uint32_t dc[4][NLH];
#pragma unroll
                for (int k = 0; k < 4; ++k)
#pragma unroll
                    for (int l = 0; l < NLH; ++l) dc[k][l] = 0;
#pragma unroll 2
                for (int n = lt; n < NH; n += 4 * TPQ) {
                    uint4 v[4];
#pragma unroll
                    for (int u = 0; u < 4; ++u) {
                        const int nn = n + u * TPQ;
                        if (nn < NH) {
                            const uint4 a = ld4(Sh, nn), b = ld4(Sp, nn);
                            v[u] = make_uint4(a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
                        } else {
                            v[u] = make_uint4(0, 0, 0, 0);
                        }
                    }
                    vc_add4<NLH>(dc[0], v[0].x, v[1].x, v[2].x, v[3].x);
                    vc_add4<NLH>(dc[1], v[0].y, v[1].y, v[2].y, v[3].y);
                    vc_add4<NLH>(dc[2], v[0].z, v[1].z, v[2].z, v[3].z);
                    vc_add4<NLH>(dc[3], v[0].w, v[1].w, v[2].w, v[3].w);
                }
                int* dst = c == 0 ? sD + j * 4 * 32
                         : rp == rank ? sD + jp * 4 * 32 : cluster.map_shared_rank(sD + jp * 4 * 32, rp);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    const int cnt = column_count<NLH>(dc[k], lane);
                    atomicAdd(&dst[k * 32 + lane], cnt);
                }
                cluster.sync();  // all counts in; partner planes may be modified again
                for (int i = tid; i < Qc * 4 * 32; i += nthreads) {
                    const int pl = i >> 5, b = i & 31;
                    const int gg = rank * Qc + (pl >> 2);
                    if (gg & 1) continue;  // copy-1 quads: counted in the copy-0 owner
                    const int t = 4 * (gg >> 1) + (pl & 3);
                    const int D = (int)((uint32_t)sD[i] - (i == tid ? mask_keep : 0u));
                    const long long Qv = (long long)N - 2LL * D;
                    const unsigned long long q2 = (unsigned long long)(Qv * Qv);
                    const size_t o = ((size_t)w * T + t) * 32 + b;
                    if (P.q_sum)
                        atomicAdd(reinterpret_cast<unsigned long long*>(P.q_sum + o),
                                  (unsigned long long)Qv);
                    if (P.q2_sum)
                        atomicAdd(reinterpret_cast<unsigned long long*>(P.q2_sum + o), q2);
                    if (P.q4_sum) {  // Q^4 as sum of low 32 bits and sum of the rest
                        const unsigned long long lo = q2 * q2, hi = __umul64hi(q2, q2);
                        atomicAdd(P.q4_sum + 2 * o, lo & 0xFFFFFFFFull);
                        atomicAdd(P.q4_sum + 2 * o + 1, (lo >> 32) | (hi << 32));
                    }
                    if (P.hist) atomicAdd(&P.hist[(size_t)t * (N + 1) + D], 1u);
                    if (P.d_last) P.d_last[o] = D;
                }
            }
            __syncthreads();  // sE / sD are cleared at the start of the next sweep
        }
    }

    // ---- store this CTA's quads ----
    {
        uint4* dst = reinterpret_cast<uint4*>(P.spins);
        for (int i = tid; i < Qc * N; i += nthreads) {
            const int jj = i / N, n = i - jj * N;
            dst[quad_base(jj) + n] = ld4(S + (size_t)jj * 4 * N, n);
        }
    }
    cluster.sync();  // no CTA leaves while a peer may still read its shared memory
}

// Advances a device-resident sweep counter after a launch of a captured graph.
__global__ void advance_counter(long long* counter, long long n) { *counter += n; }

}  // namespace csg
