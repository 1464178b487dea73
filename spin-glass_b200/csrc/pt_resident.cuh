// pt_resident.cuh — the cluster-resident parallel-tempering kernel (sm_100a).
//
// Per sweep (reference: perform_MC_steps, eamsim.cu:112-208):
//   colour 0 / colour 1 — each thread walks its column of the colour along z
//     (Walk<L, NSEG>): for every site it loads the 4 temperature planes of the
//     site and its six neighbours from shared memory at offsets fixed for the
//     launch, draws one Philox block for the 4 planes, counts unsatisfied
//     bonds with two full adders per triple and takes the flip mask from the
//     threshold table.
//   energies — while colour 1 runs, the post-flip unsatisfied-bond counts are
//     added into bit-sliced per-thread counters (each bond has exactly one
//     colour-1 end); warps reduce them with a 32x32 bit transpose + popc.
//   exchange (perform_PT_shuffle/shuffle, eamsim.cu:43-90, 211-330) — the CTA
//     owning plane t decides pair (t,t+1) for the 32 samples (FP64 exp on the
//     device) and swaps the accepted samples' configurations, reaching into
//     the neighbouring CTA's shared memory when t+1 lives there.
//   measurement (compute_q, eamsim.cu:451-511) — popcount overlaps of the two
//     copies, integer moments and a histogram.
#pragma once
#include "pt_kernel.cuh"

namespace csg {

// Adds, for each of the 4 planes k of the lane's quad jj, the per-sample
// column counts of the warp's bit-sliced counters v[k] to dst_of(jj)[32k + b].
// A warp of one quad reduces all 4 planes in one transpose per level
// (packed_column_counts); a warp holding lanes of two quads (a team size that
// is not a multiple of 32) does so once per quad, the other quad's lanes
// counting zeros.
// Lanes with jj >= Qc (the CTA's padding threads) hold zeros and count nothing.
template <int NLV, class DstOf>
__device__ __forceinline__ void add_plane_counts(const uint32_t (&v)[4][NLV], int jj, int Qc,
                                                 int lane, DstOf&& dst_of) {
    const int jlo = __shfl_sync(0xFFFFFFFFu, jj, 0);
    const int jhi = __shfl_sync(0xFFFFFFFFu, jj, 31);
    if (jlo == jhi) {
        if (jlo >= Qc) return;  // a warp of padding threads
        int cnt[4];
        packed_column_counts<NLV>(v, lane, cnt);
        int* d = dst_of(jlo);
#pragma unroll
        for (int k = 0; k < 4; ++k) atomicAdd(d + k * 32 + lane, cnt[k]);
        return;
    }
    for (int part = 0; part < 2; ++part) {
        const int jp = part ? jhi : jlo;
        if (jp >= Qc) continue;  // uniform over the warp
        const bool mine = jj == jp;
        // the other quad's lanes count as zeros
        uint32_t x[4][NLV];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int l = 0; l < NLV; ++l) x[k][l] = mine ? v[k][l] : 0u;
        int cnt[4];
        packed_column_counts<NLV>(x, lane, cnt);
        int* d = dst_of(jp);
#pragma unroll
        for (int k = 0; k < 4; ++k) atomicAdd(d + k * 32 + lane, cnt[k]);
    }
}

// Sites per thread up to which a colour pass is unrolled completely; longer
// columns run as a loop over pairs of sites.
#ifndef CSG_UNROLL_ALL_ZS
#define CSG_UNROLL_ALL_ZS 8
#endif
constexpr int kUnrollAllZS = CSG_UNROLL_ALL_ZS;
// Longer columns run as a loop over groups of sites: the largest even divisor
// of the column length up to this many.
#ifndef CSG_SITE_GROUP
#define CSG_SITE_GROUP 4
#endif
// 1: one copy of the colour pass serves both colours, the energy counting
// guarded by a flag (half the code); 0: a copy with and one without counting.
#ifndef CSG_RUNTIME_ACC
#define CSG_RUNTIME_ACC 0
#endif
constexpr bool kRuntimeAcc = CSG_RUNTIME_ACC != 0;

__host__ __device__ constexpr int site_group(int zs, int cap) {
    int u = 2;
    for (int d = 2; d <= cap && d <= zs; d += 2)
        if (zs % d == 0) u = d;
    return u;
}

template <int L, bool GEN_H, int NSEG>
__global__ void __launch_bounds__(max_cta_threads(GEN_H, NSEG)) pt_resident_kernel(const __grid_constant__ PtParams P) {
    using CF = Walk<L, NSEG>;
    constexpr int N = CF::N, NH = CF::NH, LH = CF::LH, PL = CF::PL, NC = CF::NC, ZS = CF::ZS;
    constexpr int TPQ = CF::TPQ;
    constexpr int NLV = CF::NLV, NLD = CF::NLD, NLH = CF::NLH;

    cgx::cluster_group cluster = cgx::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int Qc = P.Qc, Q = P.Q, T = P.T, C = P.C;
    const int w = blockIdx.x / P.K;
    const int tid = threadIdx.x;
    const int nthreads = blockDim.x;
    // team jt of TPQ threads per quad; the threads past Qc*TPQ (padding of
    // the CTA to whole warps) take part in barriers and warp reductions only
    const int jt = tid / TPQ;
    const bool active = jt < Qc;
    const int j = active ? jt : Qc - 1;
    const int lt = tid - jt * TPQ;
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

    // ---- this thread's column: (y, x/2) = (cy, ch), z in [z0, z0 + ZS) ----
    const int seg = lt / NC;
    const int col = lt - seg * NC;
    const int cy = col / LH, ch = col - cy * LH;
    const int z0 = seg * ZS;
    // neighbour offsets in a colour's half array (site (z, y, h) at (z*L + y)*LH + h)
    const int dxA = ch == 0 ? LH - 1 : -1;            // x-1 neighbour of a site with x = 2h
    const int dxB = ch == LH - 1 ? -(LH - 1) : 1;     // x+1 neighbour of a site with x = 2h+1
    const int dyM = (cy == 0 ? L - 1 : -1) * LH;
    const int dyP = (cy == L - 1 ? -(L - 1) : 1) * LH;
    const int dzF = (z0 == 0 ? L - 1 : -1) * PL;       // z-1 of the segment's first site
    const int dzL = (z0 + ZS == L ? -(L - 1) : 1) * PL; // z+1 of its last site
    const int colbase = z0 * PL + cy * LH + ch;
    const uint32_t site0 = (uint32_t)((z0 * L + cy) * L + 2 * ch);  // Philox word 0 without x & 1

    const long long sweep_base = P.sweep0 + (P.sweep_dev ? *P.sweep_dev : 0ll);
    for (int it = 0; it < P.n_sweeps; ++it) {
        const long long s = sweep_base + it;
        const bool do_swap = P.sps > 0 && ((s + 1) % P.sps) == 0;
        const bool do_meas = P.spm > 0 && ((s + 1) % P.spm) == 0 && s >= P.meas_start;
        const bool need_E = do_swap || do_meas;
        const bool need_M = need_E && (GEN_H || (do_meas && (P.flags & kFlagMeasureM)));
        const uint32_t s32 = (uint32_t)s;
        const PhiloxFixed pf = philox_fix(s32, wg, ctr3, P.k0, P.k1);

        if (need_E)  // sE, sD and (if present) sM are contiguous
            for (int i = tid; i < Qc * 4 * 32 * (has_M ? 3 : 2); i += nthreads) sE[i] = 0;

        uint32_t ecnt[4][NLV];
#pragma unroll
        for (int k = 0; k < 4; ++k)
#pragma unroll
            for (int l = 0; l < NLV; ++l) ecnt[k][l] = 0;

        // one colour of the checkerboard; ACC (and, with runtime counting,
        // accum): also add the post-flip unsatisfied-bond counts into the
        // energy counters
        auto colour_pass = [&](const int p, auto acc_tag, const bool accum) {
            constexpr bool ACC = decltype(acc_tag)::value;
            // x parity of the column's sites alternates along z: sites k = 0, 2, ...
            // have x = 2h + o0, sites k = 1, 3, ... x = 2h + 1 - o0
            const int o0 = (cy + z0 + p) & 1;
            const int xmE = o0 ? 0 : dxA, xpE = o0 ? dxB : 0;
            const int xmO = o0 ? dxA : 0, xpO = o0 ? 0 : dxB;
            uint32_t* const Sc = Sq + p * NH + colbase;
            const uint32_t* const So = Sq + (1 - p) * NH + colbase;
            const uint32_t* const SoXmE = So + xmE;
            const uint32_t* const SoXpE = So + xpE;
            const uint32_t* const SoXmO = So + xmO;
            const uint32_t* const SoXpO = So + xpO;
            const uint32_t* const SoYm = So + dyM;
            const uint32_t* const SoYp = So + dyP;
            const uint32_t* const Fc = Fw + p * NH + colbase;
            const uint32_t* const Fo = Fw + (1 - p) * NH + colbase;
            const uint32_t* const FoXmE = Fo + xmE;
            const uint32_t* const FoXmO = Fo + xmO;
            const uint32_t* const FoYm = Fo + N + dyM;
            const uint32_t* const FoZ = Fo + 2 * N;
            const uint32_t iE = site0 + (uint32_t)o0, iO = site0 + (uint32_t)(1 - o0);

            // site k of the column (odd: k & 1; dzm, dzp: z-neighbour offsets);
            // wd receives the post-flip full-adder words for the energy counters
            auto site = [&](const int k, const bool odd, const int dzm, const int dzp,
                            uint32_t (&wd)[4][4]) {
                const int off = k * PL;
                const uint4 cv = ld4(Sc, off);
                const uint4 a0 = ld4(odd ? SoXmO : SoXmE, off);
                const uint4 a1 = ld4(odd ? SoXpO : SoXpE, off);
                const uint4 a2 = ld4(SoYm, off), a3 = ld4(SoYp, off);
                const uint4 a4 = ld4(So, off + dzm), a5 = ld4(So, off + dzp);
                const uint32_t f0 = __ldg((odd ? FoXmO : FoXmE) + off), f1 = __ldg(Fc + off);
                const uint32_t f2 = __ldg(FoYm + off), f3 = __ldg(Fc + N + off);
                const uint32_t f4 = __ldg(FoZ + off + dzm), f5 = __ldg(Fc + 2 * N + off);
                const u32x4 r = philox_c0((odd ? iO : iE) + (uint32_t)(k * L * L), pf);
                const uint32_t rr[4] = {r.v0, r.v1, r.v2, r.v3};
                uint32_t cw[4] = {cv.x, cv.y, cv.z, cv.w};
                const uint32_t n0w[4] = {a0.x, a0.y, a0.z, a0.w}, n1w[4] = {a1.x, a1.y, a1.z, a1.w};
                const uint32_t n2w[4] = {a2.x, a2.y, a2.z, a2.w}, n3w[4] = {a3.x, a3.y, a3.z, a3.w};
                const uint32_t n4w[4] = {a4.x, a4.y, a4.z, a4.w}, n5w[4] = {a5.x, a5.y, a5.z, a5.w};
#pragma unroll
                for (int kq = 0; kq < 4; ++kq) {
                    const uint32_t s0 = cw[kq];
                    const uint32_t u0 = s0 ^ n0w[kq] ^ f0, u1 = s0 ^ n1w[kq] ^ f1;
                    const uint32_t u2 = s0 ^ n2w[kq] ^ f2, u3 = s0 ^ n3w[kq] ^ f3;
                    const uint32_t u4 = s0 ^ n4w[kq] ^ f4, u5 = s0 ^ n5w[kq] ^ f5;
                    const uint32_t sa = u0 ^ u1 ^ u2, ca = maj3(u0, u1, u2);
                    const uint32_t sb = u3 ^ u4 ^ u5, cb = maj3(u3, u4, u5);
                    uint32_t fl;
                    if constexpr (GEN_H)
                        fl = flip_gen(s0, sa, ca, sb, cb, rr[kq], thrq[2 * kq], thrq[2 * kq + 1],
                                      (int)((uc0 >> (8 * kq)) & 0xFF), (int)((uc1 >> (8 * kq)) & 0xFF));
                    else
                        fl = flip_h0(sa, ca, sb, cb, rr[kq], th0[kq], th1[kq], th2[kq]);
                    cw[kq] = s0 ^ fl;
                    if constexpr (ACC) {
                        if (accum) {
                            wd[kq][0] = sa ^ fl;
                            wd[kq][1] = sb ^ fl;
                            wd[kq][2] = ca ^ fl;
                            wd[kq][3] = cb ^ fl;
                        }
                    }
                }
                st4(Sc, off, make_uint4(cw[0], cw[1], cw[2], cw[3]));
            };
            auto acc2 = [&](const uint32_t (&wa)[4][4], const uint32_t (&wb)[4][4]) {
                if constexpr (ACC) {
                    if (accum) {
#pragma unroll
                        for (int kq = 0; kq < 4; ++kq)
                            vc_add_2sites<NLV>(ecnt[kq], wa[kq][0], wa[kq][1], wa[kq][2], wa[kq][3],
                                               wb[kq][0], wb[kq][1], wb[kq][2], wb[kq][3]);
                    }
                }
            };
            if constexpr (ZS <= kUnrollAllZS) {
#pragma unroll
                for (int k = 0; k < ZS; k += 2) {
                    uint32_t wa[4][4], wb[4][4];
                    site(k, false, k == 0 ? dzF : -PL, k == ZS - 1 ? dzL : PL, wa);
                    if (k + 1 < ZS) {
                        site(k + 1, true, -PL, k + 1 == ZS - 1 ? dzL : PL, wb);
                        acc2(wa, wb);
                    } else if constexpr (ACC) {
                        if (accum) {
#pragma unroll
                            for (int kq = 0; kq < 4; ++kq)
                                vc_add_site<NLV>(ecnt[kq], wa[kq][0], wa[kq][1], wa[kq][2], wa[kq][3]);
                        }
                    }
                }
            } else {
                // groups of U sites: a group's sites sit at fixed offsets from
                // its first one; only the first group's first site and the last
                // group's last site wrap around in z
                constexpr int U = site_group(ZS, CSG_SITE_GROUP);
                static_assert(ZS % U == 0 && U % 2 == 0, "groups must tile the column");
#pragma unroll 1
                for (int k0 = 0; k0 < ZS; k0 += U) {
                    const int dzm0 = k0 == 0 ? dzF : -PL;
                    const int dzpL = k0 + U == ZS ? dzL : PL;
#pragma unroll
                    for (int u = 0; u < U; u += 2) {
                        uint32_t wa[4][4], wb[4][4];
                        site(k0 + u, false, u == 0 ? dzm0 : -PL, PL, wa);
                        site(k0 + u + 1, true, -PL, u + 2 == U ? dzpL : PL, wb);
                        acc2(wa, wb);
                    }
                }
            }
        };
        if constexpr (kRuntimeAcc) {
            if (active) colour_pass(0, std::true_type{}, false);
            __syncthreads();
            if (active) colour_pass(1, std::true_type{}, need_E);
        } else {
            if (active) colour_pass(0, std::false_type{}, false);
            __syncthreads();
            if (active) {
                if (need_E)
                    colour_pass(1, std::true_type{}, true);
                else
                    colour_pass(1, std::false_type{}, false);
            }
        }
        __syncthreads();

        if (!need_E) continue;

        // ---- per-sample unsatisfied-bond totals of this CTA's planes ----
        add_plane_counts<NLV>(ecnt, jt, Qc, lane, [&](int jj) { return sE + jj * 4 * 32; });
        if (need_M) {
            uint32_t mc[4][NLD];
#pragma unroll
            for (int k = 0; k < 4; ++k)
#pragma unroll
                for (int l = 0; l < NLD; ++l) mc[k][l] = 0;
            if (active) {
                // four consecutive sites of a plane per 128-bit load
#pragma unroll 1
                for (int i = lt; i < N / 4; i += TPQ) {
#pragma unroll
                    for (int k = 0; k < 4; ++k) {
                        const uint4 v = reinterpret_cast<const uint4*>(Sq + k * N)[i];
                        vc_add4<NLD>(mc[k], v.x, v.y, v.z, v.w);
                    }
                }
            }
            add_plane_counts<NLD>(mc, jt, Qc, lane, [&](int jj) { return sM + jj * 4 * 32; });
        }
        // sE / sM hold per-sample counts: U unsatisfied bonds (E_b = 2U - 3N)
        // and n_up up spins (M = 2 n_up - N); the barriers before their
        // readers below complete them
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
                    const int u0 = E0[lane], u1 = E1[lane];
                    const int n0 = need_M ? M0[lane] : 0, n1 = need_M ? M1[lane] : 0;
                    const int e0 = 2 * u0 - 3 * N, e1 = 2 * u1 - 3 * N;
                    const int m0 = 2 * n0 - N, m1 = 2 * n1 - N;
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
                        E0[lane] = u1;
                        E1[lane] = u0;
                        if (need_M) {
                            M0[lane] = n1;
                            M1[lane] = n0;
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
            // four consecutive sites of a plane per 128-bit access (N is a
            // multiple of 8, the plane arrays 16-byte aligned)
            auto exchange = [&](uint32_t* pa, uint32_t* pb, const uint32_t m) {
                constexpr int N4 = N / 4, CH = 2;
                uint4* const a4 = reinterpret_cast<uint4*>(pa);
                uint4* const b4 = reinterpret_cast<uint4*>(pb);
                auto mix = [m](uint32_t& x, uint32_t& y) {
                    const uint32_t d = (x ^ y) & m;
                    x ^= d;
                    y ^= d;
                };
                for (int i0 = lt; i0 < N4; i0 += CH * TPQ) {
                    uint4 a[CH], b[CH];
#pragma unroll
                    for (int u = 0; u < CH; ++u) {
                        const int i = i0 + u * TPQ;
                        a[u] = i < N4 ? a4[i] : make_uint4(0, 0, 0, 0);
                        b[u] = i < N4 ? b4[i] : make_uint4(0, 0, 0, 0);
                    }
#pragma unroll
                    for (int u = 0; u < CH; ++u) {
                        const int i = i0 + u * TPQ;
                        if (i < N4) {
                            mix(a[u].x, b[u].x);
                            mix(a[u].y, b[u].y);
                            mix(a[u].z, b[u].z);
                            mix(a[u].w, b[u].w);
                            a4[i] = a[u];
                            b4[i] = b[u];
                        }
                    }
                }
            };
            if (active) {
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
                const int ev = 2 * sE[i] - 3 * N;
                if (P.e_sum) atomicAdd(reinterpret_cast<unsigned long long*>(P.e_sum + o),
                                       (unsigned long long)(long long)ev);
                if (P.e_last) P.e_last[o] = ev;
                if (need_M) {
                    const int mv = 2 * sM[i] - N;
                    if (P.m_sum) atomicAdd(reinterpret_cast<unsigned long long*>(P.m_sum + o),
                                           (unsigned long long)(long long)mv);
                    if (P.m_last) P.m_last[o] = mv;
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
                if (active) {
                    // four consecutive sites of a plane per 128-bit load
#pragma unroll 2
                    for (int i = lt; i < NH / 4; i += TPQ) {
#pragma unroll
                        for (int k = 0; k < 4; ++k) {
                            const uint4 a = reinterpret_cast<const uint4*>(Sh + k * N)[i];
                            const uint4 b = reinterpret_cast<const uint4*>(Sp + k * N)[i];
                            vc_add4<NLH>(dc[k], a.x ^ b.x, a.y ^ b.y, a.z ^ b.z, a.w ^ b.w);
                        }
                    }
                }
                // counts of quad jj go to the copy-0 quad of its temperature quad
                add_plane_counts<NLH>(dc, jt, Qc, lane, [&](int jj) {
                    const int gg = rank * Qc + jj;
                    if (gg % C == 0) return sD + jj * 4 * 32;
                    const int g0 = gg ^ 1, r0 = g0 / Qc, j0 = g0 - r0 * Qc;
                    return r0 == rank ? sD + j0 * 4 * 32 : cluster.map_shared_rank(sD + j0 * 4 * 32, r0);
                });
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

}  // namespace csg
