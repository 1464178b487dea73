// pt_kernel.cuh — what the parallel-tempering kernels share: launch
// parameters, acceptance tables, the bit-sliced counting helpers and the flip
// rules, and the thread layout of the cluster-resident kernel
// (pt_resident.cuh, instantiated per lattice side in pt_instances.cu).
//
// Work decomposition of the resident kernel.  A thread-block cluster owns one
// sample word w (32 disorder samples) with all its copies and temperatures.
// The word's C*T/4 temperature quads (4 planes of N uint32 each) are split
// over the K CTAs of the cluster, Qc quads per CTA, and stay in shared memory
// for the whole launch (a section of sweeps).  Nothing but the bonds
// (read-only, through L1) touches global memory between the load at the
// start and the store at the end.
#pragma once
#include <cooperative_groups.h>

#include <cstdint>
#include <type_traits>

#include "philox.cuh"

namespace csg {
namespace cgx = cooperative_groups;

constexpr int kMaxT = 64;
constexpr int kMaxThreads = 512;  // CTA size cap: keeps 128 registers per thread available
// The general-field kernels whose threads each walk a whole column (one
// segment) keep more state live per site than 128 registers hold (they spilled
// up to 316 bytes at L = 24); their CTAs are capped at 384 threads, which
// leaves 168 registers per thread.
constexpr int kMaxThreadsGenWalk = 384;
__host__ __device__ constexpr int max_cta_threads(bool gen, int nseg) {
    return gen && nseg == 1 ? kMaxThreadsGenWalk : kMaxThreads;
}

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

// Thread layout of the resident kernel for lattice side L: every thread of a
// quad's team owns one column (y, x/2) of a checkerboard colour and a segment
// of ZS = L / NSEG consecutive z; the team has TPQ = L * L/2 * NSEG threads.
// Walking its column along z, a thread finds all six neighbours and bonds of
// each site at offsets fixed for the whole launch (only the first and last
// site of a segment may wrap around in z).
template <int L, int NSEG>
struct Walk {
    static_assert(L % 2 == 0 && L % NSEG == 0, "segments must tile the column");
    static constexpr int LH = L / 2;
    static constexpr int N = L * L * L;
    static constexpr int NH = N / 2;
    static constexpr int PL = L * LH;                          // sites of a colour per z-plane
    static constexpr int NC = PL;                              // columns per colour
    static constexpr int ZS = L / NSEG;                        // sites per thread per colour
    static constexpr int TPQ = NC * NSEG;                      // threads per quad
    static constexpr int NLV = bit_length(6 * ZS);             // energy counter levels
    static constexpr int MPT = (N + 4 * TPQ - 1) / (4 * TPQ);  // 4-site groups per thread
    static constexpr int NLD = bit_length(4 * MPT);            // magnetisation counter levels
    static constexpr int MPH = (NH + 4 * TPQ - 1) / (4 * TPQ); // 4-site groups per half lattice
    static constexpr int NLH = bit_length(4 * MPH);            // overlap counter levels
    static_assert(TPQ >= 32, "a warp spans at most two quads");
};

// Column segments per thread the resident kernel is built with, for each L:
// the first entry is the default, the second (if any) a team twice as large
// with half as many sites per thread.
__host__ __device__ constexpr int nseg_option(int L, int i) {
    return L == 4 ? (i == 0 ? 4 : 0)
         : L == 6 ? (i == 0 ? 2 : 0)
         : L <= 16 ? (i == 0 ? (L <= 10 ? 2 : 1) : i == 1 ? (L <= 10 ? 1 : 2) : 0)
         : (i == 0 ? 1 : 0);
}
__host__ __device__ constexpr int threads_per_quad(int L, int nseg) { return L * (L / 2) * nseg; }

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

// Column sums of the 4 planes of a warp whose 32 lanes all hold counters of
// one quad: two rounds of lane exchange (lanes i, i^16, then i, i^8) leave
// each lane with one plane, k = lane >> 3, summed over 4 lanes (two more
// counter levels); one 32x32 transpose per level then gives every lane j the
// bits of sample j of all lanes, plane k in bits 8k..8k+7.  Returns, in lane
// j, the totals of sample j for planes 0..3.
template <int NLV>
__device__ __forceinline__ void packed_column_counts(const uint32_t (&v)[4][NLV], int lane,
                                                     int (&cnt)[4]) {
    const bool hi16 = (lane & 16) != 0, hi8 = (lane & 8) != 0;
    uint32_t a[2][NLV + 1];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        uint32_t cy = 0;
#pragma unroll
        for (int l = 0; l < NLV; ++l) {
            const uint32_t mine = hi16 ? v[k + 2][l] : v[k][l];
            const uint32_t other = __shfl_xor_sync(0xFFFFFFFFu, hi16 ? v[k][l] : v[k + 2][l], 16);
            a[k][l] = mine ^ other ^ cy;
            cy = maj3(mine, other, cy);
        }
        a[k][NLV] = cy;
    }
    uint32_t b[NLV + 2];
    uint32_t cy = 0;
#pragma unroll
    for (int l = 0; l <= NLV; ++l) {
        const uint32_t mine = hi8 ? a[1][l] : a[0][l];
        const uint32_t other = __shfl_xor_sync(0xFFFFFFFFu, hi8 ? a[0][l] : a[1][l], 8);
        b[l] = mine ^ other ^ cy;
        cy = maj3(mine, other, cy);
    }
    b[NLV + 1] = cy;
#pragma unroll
    for (int k = 0; k < 4; ++k) cnt[k] = 0;
#pragma unroll
    for (int l = 0; l < NLV + 2; ++l) {
        uint32_t x = b[l];
#pragma unroll
        for (int d = 16; d >= 1; d >>= 1) {  // 32x32 bit transpose (as in column_popc)
            const uint32_t m = d == 16 ? 0x0000FFFFu
                             : d == 8  ? 0x00FF00FFu
                             : d == 4  ? 0x0F0F0F0Fu
                             : d == 2  ? 0x33333333u
                                       : 0x55555555u;
            const bool upper = (lane & d) != 0;
            const uint32_t t = __shfl_xor_sync(0xFFFFFFFFu, x, d);
            const uint32_t rot = __funnelshift_r(t, t, upper ? d : 32 - d);
            const uint32_t keep = upper ? ~m : m;
            x = (x & keep) | (rot & ~keep);
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) cnt[k] += __popc((x >> (8 * k)) & 0xFFu) << l;
    }
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
        return (size_t)Qc * L * L * L * 16 + (size_t)Qc * 4 * 32 * 4 * (has_m ? 3 : 2) +
               (gen ? (size_t)Qc * 4 * 32 + (size_t)Qc * 4 * 2 : 0);
    }
};

using ResidentFn = void (*)(PtParams);

// The resident kernel for lattice side L (each defined in its own translation
// unit, pt_instances.cu built with CSG_PT_L = L): the general-field variant
// when gen, with nseg column segments per thread; nullptr if not built.
#define CSG_DECLARE_RESIDENT(LL) ResidentFn resident_kernel_L##LL(bool gen, int nseg);
CSG_DECLARE_RESIDENT(4)
CSG_DECLARE_RESIDENT(6)
CSG_DECLARE_RESIDENT(8)
CSG_DECLARE_RESIDENT(10)
CSG_DECLARE_RESIDENT(12)
CSG_DECLARE_RESIDENT(14)
CSG_DECLARE_RESIDENT(16)
CSG_DECLARE_RESIDENT(18)
CSG_DECLARE_RESIDENT(20)
CSG_DECLARE_RESIDENT(22)
CSG_DECLARE_RESIDENT(24)
#undef CSG_DECLARE_RESIDENT

}  // namespace csg
