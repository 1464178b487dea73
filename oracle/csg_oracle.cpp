// csg_oracle.cpp — CPU oracle (test infrastructure only; see csg_oracle.h).
//
// Scalar restatement of the reference update rule, one sample at a time.
// It deliberately shares no code with the CUDA engine: its Philox, its
// indexing and its acceptance test are written out here on their own so that
// a bit-exact match between the two is evidence, not a tautology.
// orc_run_multispin, the CPU timing baseline, replaces only the per-sample
// acceptance loop by one evaluated for the 32 samples of a word at once; the
// tests check that the two give the same bits.
#include "csg_oracle.h"

#include <cmath>
#include <cstring>
#include <utility>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// Counter tags (top byte of the fourth Philox counter word).
constexpr uint32_t kTagBond = 1u << 24;
constexpr uint32_t kTagInit = 2u << 24;
constexpr uint32_t kTagSweep = 3u << 24;
constexpr uint32_t kTagSwap = 4u << 24;

// Philox4x32-10, Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11: ten rounds of two 32x32->64 products, key bumped by the
// Weyl constants between rounds.
void philox(const uint32_t in[4], uint32_t k0, uint32_t k1, uint32_t out[4]) {
    uint32_t c0 = in[0], c1 = in[1], c2 = in[2], c3 = in[3];
    for (int round = 0; round < 10; ++round) {
        if (round > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

void philox_ctr(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint64_t seed, uint32_t out[4]) {
    const uint32_t in[4] = {a, b, c, d};
    philox(in, (uint32_t)seed, (uint32_t)(seed >> 32), out);
}

struct Geo {
    int L, LH;
    int64_t N, NH;
    explicit Geo(int l) : L(l), LH(l / 2), N((int64_t)l * l * l), NH((int64_t)l * l * l / 2) {}
    int wrap(int a) const { return (a % L + L) % L; }
    int64_t slot(int x, int y, int z) const {
        return (int64_t)((x + y + z) & 1) * NH + ((int64_t)(z * L + y) * LH + (x >> 1));
    }
    int64_t site(int x, int y, int z) const { return ((int64_t)z * L + y) * L + x; }
};

struct Dims {
    int L, W, C, T, Q;
    Geo g;
    Dims(int l, int w, int c, int t) : L(l), W(w), C(c), T(t), Q(t / 4), g(l) {}
    size_t spin(int w, int c, int t, int64_t slot) const {
        return ((((size_t)w * C + c) * Q + (t >> 2)) * (size_t)g.N + (size_t)slot) * 4 + (t & 3);
    }
    size_t bond(int w, int d, int64_t slot) const {
        return ((size_t)w * 3 + d) * (size_t)g.N + (size_t)slot;
    }
};

bool dims_ok(int L, int W, int C, int T) {
    return L >= 4 && L <= 64 && (L % 2) == 0 && W >= 1 && (C == 1 || C == 2) &&
           T >= 4 && T <= 64 && (T % 4) == 0;
}

// Per-sample bit counter: byte-wise accumulation, flushed before overflow.
struct BitCounter {
    uint32_t acc[8] = {0};
    int pending = 0;
    int64_t cnt[32] = {0};
    void add(uint32_t w) {
        for (int g = 0; g < 8; ++g) acc[g] += (w >> g) & 0x01010101u;
        if (++pending == 255) flush();
    }
    void flush() {
        for (int g = 0; g < 8; ++g) {
            for (int k = 0; k < 4; ++k) cnt[8 * k + g] += (acc[g] >> (8 * k)) & 0xFFu;
            acc[g] = 0;
        }
        pending = 0;
    }
};

int threads_for(const orc_params* p) {
#ifdef _OPENMP
    return p->n_threads > 0 ? p->n_threads : omp_get_max_threads();
#else
    (void)p;
    return 1;
#endif
}

// Bond energy (eamsim.cu:246-282, 320-324: E = -(2 S - 3N), S = satisfied
// bonds) and magnetisation (eamsim.cu:296-323: M = 2 n_up - N) of one plane.
void plane_energy(const Dims& D, const uint32_t* spins, const uint32_t* bonds, int w, int c,
                  int t, int32_t e[32], int32_t m[32]) {
    const Geo& g = D.g;
    BitCounter unsat, up;
    for (int z = 0; z < g.L; ++z)
        for (int y = 0; y < g.L; ++y)
            for (int x = 0; x < g.L; ++x) {
                const int64_t si = g.slot(x, y, z);
                const uint32_t s0 = spins[D.spin(w, c, t, si)];
                up.add(s0);
                const int64_t nb[3] = {g.slot(g.wrap(x + 1), y, z), g.slot(x, g.wrap(y + 1), z),
                                       g.slot(x, y, g.wrap(z + 1))};
                for (int d = 0; d < 3; ++d)
                    unsat.add(s0 ^ spins[D.spin(w, c, t, nb[d])] ^ bonds[D.bond(w, d, si)]);
            }
    unsat.flush();
    up.flush();
    for (int b = 0; b < 32; ++b) {
        e[b] = (int32_t)(2 * unsat.cnt[b] - 3 * g.N);
        m[b] = (int32_t)(2 * up.cnt[b] - g.N);
    }
}

// Overlap integers of one temperature: d[b] = #sites where the copies differ,
// dpl[b][dir][a] = same restricted to coordinate dir == a.
void plane_overlap(const Dims& D, const uint32_t* spins, int w, int t, int32_t d[32],
                   int32_t* dpl /* [32][3][L] or null */) {
    const Geo& g = D.g;
    BitCounter tot;
    std::vector<int64_t> pl;
    if (dpl) pl.assign((size_t)32 * 3 * g.L, 0);
    for (int z = 0; z < g.L; ++z)
        for (int y = 0; y < g.L; ++y)
            for (int x = 0; x < g.L; ++x) {
                const int64_t si = g.slot(x, y, z);
                const uint32_t diff = spins[D.spin(w, 0, t, si)] ^ spins[D.spin(w, 1, t, si)];
                tot.add(diff);
                if (dpl && diff) {
                    const int co[3] = {x, y, z};
                    for (int b = 0; b < 32; ++b)
                        if ((diff >> b) & 1u)
                            for (int k = 0; k < 3; ++k) pl[((size_t)b * 3 + k) * g.L + co[k]] += 1;
                }
            }
    tot.flush();
    for (int b = 0; b < 32; ++b) d[b] = (int32_t)tot.cnt[b];
    if (dpl)
        for (size_t i = 0; i < pl.size(); ++i) dpl[i] = (int32_t)pl[i];
}

void add_u128(uint64_t* acc, uint64_t lo, uint64_t hi) {
    const uint64_t old = acc[0];
    acc[0] += lo;
    acc[1] += hi + (acc[0] < old ? 1u : 0u);
}

// ---------------------------------------------------------------------------
// The multispin restatement (timing baseline, checked equal to the
// per-sample loop of run_impl by the tests).  It evaluates the same rule for
// all 32 samples of a word at once, as the reference's own kernel does for its
// 24 temperatures (SWAR counts, eamsim.cu:173-180): the unsatisfied-bond count
// U of every sample as three bit-slices, then, per class (centre bit s, U),
// the samples of that class when the draw is below thr[s][U].
// ---------------------------------------------------------------------------

// The four temperature planes of a quad side by side, one per lane.
typedef uint32_t v4u __attribute__((vector_size(16)));

inline v4u load4(const uint32_t* a) {
    v4u v;
    std::memcpy(&v, a, sizeof v);
    return v;
}
inline void store4(uint32_t* a, v4u v) { std::memcpy(a, &v, sizeof v); }
inline v4u splat(uint32_t x) { return v4u{x, x, x, x}; }

// Thresholds thr[t][s][U] of a quad's 4 planes (lane k = plane 4q+k) as
// 32-bit lanes: r < thr  <=>  r < lo || always, where always marks thr = 2^32.
struct QuadThresholds {
    v4u lo[2][7], always[2][7];
    explicit QuadThresholds(const uint64_t* thr /* [4][2][7] */) {
        for (int sb = 0; sb < 2; ++sb)
            for (int U = 0; U < 7; ++U)
                for (int k = 0; k < 4; ++k) {
                    const uint64_t t = thr[(size_t)k * 14 + sb * 7 + U];
                    lo[sb][U][k] = t >> 32 ? 0u : (uint32_t)t;
                    always[sb][U][k] = t >> 32 ? 0xFFFFFFFFu : 0u;
                }
    }
};

// Accepted flips of the 32 samples of the 4 planes of a site: U of every
// sample as three bit-slices from full adders, then the samples of every
// class (centre bit, U) whose threshold the plane's draw is below.
inline v4u accept_quad(const v4u u[6], v4u s0, v4u r, const QuadThresholds& th) {
    const v4u sa = u[0] ^ u[1] ^ u[2], ca = (u[0] & u[1]) | (u[2] & (u[0] ^ u[1]));
    const v4u sb = u[3] ^ u[4] ^ u[5], cb = (u[3] & u[4]) | (u[5] & (u[3] ^ u[4]));
    // U = sa + sb + 2 (ca + cb) = b0 + 2 (c0 + ca + cb) = b0 + 2 b1 + 4 b2
    const v4u b0 = sa ^ sb, c0 = sa & sb;
    const v4u b1 = ca ^ cb ^ c0, b2 = (ca & cb) | (c0 & (ca ^ cb));
    v4u acc = splat(0);
    for (int U = 0; U <= 6; ++U) {
        const v4u eq = ((U & 1) ? b0 : ~b0) & ((U & 2) ? b1 : ~b1) & ((U & 4) ? b2 : ~b2);
        const v4u lt0 = (v4u)(r < th.lo[0][U]) | th.always[0][U];
        const v4u lt1 = (v4u)(r < th.lo[1][U]) | th.always[1][U];
        acc |= eq & ((lt0 & ~s0) | (lt1 & s0));
    }
    return acc;
}

// Neighbour slots (-x, +x, -y, +y, -z, +z) and the site index of every slot.
struct Neighbours {
    std::vector<int32_t> nb, site;
    explicit Neighbours(const Geo& g) : nb((size_t)g.N * 6), site((size_t)g.N) {
        for (int z = 0; z < g.L; ++z)
            for (int y = 0; y < g.L; ++y)
                for (int x = 0; x < g.L; ++x) {
                    const int64_t si = g.slot(x, y, z);
                    site[si] = (int32_t)g.site(x, y, z);
                    const int64_t n[6] = {g.slot(g.wrap(x - 1), y, z), g.slot(g.wrap(x + 1), y, z),
                                          g.slot(x, g.wrap(y - 1), z), g.slot(x, g.wrap(y + 1), z),
                                          g.slot(x, y, g.wrap(z - 1)), g.slot(x, y, g.wrap(z + 1))};
                    for (int k = 0; k < 6; ++k) nb[(size_t)si * 6 + k] = (int32_t)n[k];
                }
    }
};

// Sweep s of every (word, copy, quad), colour 0 then colour 1: the sites,
// draws and thresholds of the per-sample loop; sites of one colour are
// independent, so their order does not matter.
void sweep_multispin(const orc_params* p, const Dims& D, const Neighbours& G, uint32_t* spins,
                     const uint32_t* bonds, int64_t s, int nthr) {
    const int64_t NH = D.g.NH;
    const int W = D.W, C = D.C, Q = D.Q;
    for (int phase = 0; phase < 2; ++phase) {
#pragma omp parallel for collapse(3) schedule(static) num_threads(nthr)
        for (int w = 0; w < W; ++w)
            for (int c = 0; c < C; ++c)
                for (int q = 0; q < Q; ++q) {
                    const uint32_t ctr3 = kTagSweep | ((uint32_t)c << 8) | (uint32_t)q;
                    const uint32_t* Jx = bonds + D.bond(w, 0, 0);
                    const uint32_t* Jy = bonds + D.bond(w, 1, 0);
                    const uint32_t* Jz = bonds + D.bond(w, 2, 0);
                    uint32_t* S = spins + D.spin(w, c, 4 * q, 0);  // S[slot * 4 + k]
                    const QuadThresholds th(p->thr + (size_t)(4 * q) * 14);
                    for (int64_t si = phase * NH; si < (phase + 1) * NH; ++si) {
                        const int32_t* nb = &G.nb[(size_t)si * 6];
                        const uint32_t J[6] = {Jx[nb[0]], Jx[si], Jy[nb[2]], Jy[si], Jz[nb[4]], Jz[si]};
                        uint32_t r[4];
                        philox_ctr((uint32_t)G.site[si], (uint32_t)s, (uint32_t)(w + p->word0), ctr3,
                                   p->seed, r);
                        const v4u s0 = load4(S + si * 4);
                        v4u u[6];
                        for (int n = 0; n < 6; ++n) u[n] = s0 ^ load4(S + (size_t)nb[n] * 4) ^ splat(J[n]);
                        store4(S + si * 4, s0 ^ accept_quad(u, s0, v4u{r[0], r[1], r[2], r[3]}, th));
                    }
                }
    }
}

int run_impl(const orc_params* p, uint32_t* spins, const uint32_t* bonds, int64_t sweep0,
             int64_t n_sweeps, orc_obs* obs, bool multispin);

}  // namespace

extern "C" {

void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    philox(ctr, key[0], key[1], out);
}

// Acceptance thresholds.  The reference builds s_prob[r][2c+b] =
// expf(2 beta E)*UINT_MAX with E = (6-2c) + H(1-2b) (eamsim.cu:33-37) and
// accepts when a 32-bit draw is below it (eamsim.cu:187-194).  Here U = 6-c
// counts unsatisfied bonds and the centre bit s selects the field term, so
// dE = 12 - 4U + 2H(2s-1); the table holds floor(exp(-beta dE) 2^32) for
// dE > 0 and 2^32 ("always") otherwise, computed once in double precision.
int orc_thresholds(int32_t T, const double* betas, double H, uint64_t* thr) {
    if (T <= 0 || !betas || !thr || !(H >= 0.0)) return 1;
    for (int t = 0; t < T; ++t)
        for (int s = 0; s < 2; ++s)
            for (int U = 0; U <= 6; ++U) {
                const double dE = 12.0 - 4.0 * U + 2.0 * H * (s ? 1.0 : -1.0);
                uint64_t v = (uint64_t)1 << 32;
                if (dE > 0.0) v = (uint64_t)(std::exp(-betas[t] * dE) * 4294967296.0);
                thr[((size_t)t * 2 + s) * 7 + U] = v;
            }
    return 0;
}

// Bonds: one Philox block per (word, site) gives the x, y, z bonds of 32
// samples (eamsim.cu:589-595 draws three bits per site per sample).  Spins:
// one block per (word, copy, site, temperature quad), uniform random
// (eamsim.cu:570-574).
int orc_init(int32_t L, int32_t W, int32_t C, int32_t T, uint64_t seed, int32_t word0,
             uint32_t* spins, uint32_t* bonds) {
    if (!dims_ok(L, W, C, T) || !spins || !bonds) return 1;
    const Dims D(L, W, C, T);
    const Geo& g = D.g;
    for (int w = 0; w < W; ++w)
        for (int z = 0; z < L; ++z)
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const int64_t i = g.site(x, y, z), si = g.slot(x, y, z);
                    uint32_t r[4];
                    const uint32_t wg = (uint32_t)(w + word0);
                    philox_ctr((uint32_t)i, 0u, wg, kTagBond, seed, r);
                    for (int d = 0; d < 3; ++d) bonds[D.bond(w, d, si)] = r[d];
                    for (int c = 0; c < C; ++c)
                        for (int q = 0; q < D.Q; ++q) {
                            philox_ctr((uint32_t)i, 0u, wg,
                                       kTagInit | ((uint32_t)c << 8) | (uint32_t)q, seed, r);
                            for (int k = 0; k < 4; ++k) spins[D.spin(w, c, 4 * q + k, si)] = r[k];
                        }
                }
    return 0;
}

int orc_energies(int32_t L, int32_t W, int32_t C, int32_t T, const uint32_t* spins,
                 const uint32_t* bonds, int32_t* e, int32_t* m) {
    if (!dims_ok(L, W, C, T)) return 1;
    const Dims D(L, W, C, T);
#pragma omp parallel for collapse(3) schedule(static)
    for (int w = 0; w < W; ++w)
        for (int c = 0; c < C; ++c)
            for (int t = 0; t < T; ++t) {
                const size_t o = (((size_t)w * C + c) * T + t) * 32;
                plane_energy(D, spins, bonds, w, c, t, e + o, m + o);
            }
    return 0;
}

int orc_overlaps(int32_t L, int32_t W, int32_t T, const uint32_t* spins, int32_t* d,
                 int32_t* dpl) {
    if (!dims_ok(L, W, 2, T)) return 1;
    const Dims D(L, W, 2, T);
#pragma omp parallel for collapse(2) schedule(static)
    for (int w = 0; w < W; ++w)
        for (int t = 0; t < T; ++t) {
            const size_t o = ((size_t)w * T + t) * 32;
            plane_overlap(D, spins, w, t, d + o, dpl ? dpl + o * 3 * L : nullptr);
        }
    return 0;
}

// One sweep = the two checkerboard phases of eamsim.cu:138-205 (parity
// (x+y+z)&1 == 0 first, eamsim.cu:141).  Each site sees its six neighbours
// through the bond words (eamsim.cu:155-167; here bit 1 = unsatisfied when the
// spins are equal), counts unsatisfied bonds per sample (the SWAR count of
// eamsim.cu:173-180) and accepts with the table entry of that count
// (eamsim.cu:184-195).  One 32-bit draw serves the 32 samples of a word.
int orc_run(const orc_params* p, uint32_t* spins, const uint32_t* bonds, int64_t sweep0,
            int64_t n_sweeps, orc_obs* obs) {
    return run_impl(p, spins, bonds, sweep0, n_sweeps, obs, false);
}

int orc_run_multispin(const orc_params* p, uint32_t* spins, const uint32_t* bonds, int64_t sweep0,
                      int64_t n_sweeps, orc_obs* obs) {
    return run_impl(p, spins, bonds, sweep0, n_sweeps, obs, true);
}

}  // extern "C"

namespace {

int run_impl(const orc_params* p, uint32_t* spins, const uint32_t* bonds, int64_t sweep0,
             int64_t n_sweeps, orc_obs* obs, bool multispin) {
    if (!p || !spins || !bonds || !p->betas || !p->thr || n_sweeps < 0) return 1;
    if (!dims_ok(p->L, p->W, p->C, p->T)) return 1;
    const Dims D(p->L, p->W, p->C, p->T);
    const Geo& g = D.g;
    const int L = p->L, W = p->W, C = p->C, T = p->T, Q = D.Q;
    const int nthr = threads_for(p);
    std::vector<int32_t> E((size_t)W * C * T * 32), M((size_t)W * C * T * 32);
    std::vector<int32_t> Dq((size_t)W * T * 32);
    std::vector<Neighbours> G;
    if (multispin) G.emplace_back(g);

    for (int64_t s = sweep0; s < sweep0 + n_sweeps; ++s) {
        if (multispin) sweep_multispin(p, D, G[0], spins, bonds, s, nthr);
        for (int phase = 0; phase < 2 && !multispin; ++phase) {
#pragma omp parallel for collapse(3) schedule(static) num_threads(nthr)
            for (int w = 0; w < W; ++w)
                for (int c = 0; c < C; ++c)
                    for (int q = 0; q < Q; ++q)
                        for (int z = 0; z < L; ++z)
                            for (int y = 0; y < L; ++y)
                                for (int x = (y + z + phase) & 1; x < L; x += 2) {
                                    const int64_t si = g.slot(x, y, z);
                                    const int64_t nb[6] = {
                                        g.slot(g.wrap(x - 1), y, z), g.slot(g.wrap(x + 1), y, z),
                                        g.slot(x, g.wrap(y - 1), z), g.slot(x, g.wrap(y + 1), z),
                                        g.slot(x, y, g.wrap(z - 1)), g.slot(x, y, g.wrap(z + 1))};
                                    const uint32_t J[6] = {
                                        bonds[D.bond(w, 0, nb[0])], bonds[D.bond(w, 0, si)],
                                        bonds[D.bond(w, 1, nb[2])], bonds[D.bond(w, 1, si)],
                                        bonds[D.bond(w, 2, nb[4])], bonds[D.bond(w, 2, si)]};
                                    uint32_t r[4];
                                    philox_ctr((uint32_t)g.site(x, y, z), (uint32_t)s,
                                               (uint32_t)(w + p->word0),
                                               kTagSweep | ((uint32_t)c << 8) | (uint32_t)q, p->seed,
                                               r);
                                    for (int k = 0; k < 4; ++k) {
                                        const int t = 4 * q + k;
                                        const size_t at = D.spin(w, c, t, si);
                                        const uint32_t s0 = spins[at];
                                        uint32_t u[6];
                                        for (int n = 0; n < 6; ++n)
                                            u[n] = s0 ^ spins[D.spin(w, c, t, nb[n])] ^ J[n];
                                        uint32_t flip = 0;
                                        for (int b = 0; b < 32; ++b) {
                                            int U = 0;
                                            for (int n = 0; n < 6; ++n) U += (u[n] >> b) & 1u;
                                            const int sb = (s0 >> b) & 1u;
                                            if ((uint64_t)r[k] < p->thr[((size_t)t * 2 + sb) * 7 + U])
                                                flip |= 1u << b;
                                        }
                                        spins[at] = s0 ^ flip;
                                    }
                                }
        }

        const bool do_swap = p->sweeps_per_swap > 0 && (s + 1) % p->sweeps_per_swap == 0;
        const bool do_meas = p->sweeps_per_meas > 0 && (s + 1) % p->sweeps_per_meas == 0 &&
                             s >= p->meas_start;
        if (!do_swap && !do_meas) continue;
        orc_energies(L, W, C, T, spins, bonds, E.data(), M.data());

        if (do_swap) {
            // Replica exchange of eamsim.cu:43-90: pairs (t,t+1) with t even
            // on even rounds and odd on odd rounds; accept when a uniform in
            // [0,1) is below exp((b_t - b_t+1)(E_t - E_t+1)).  Exchanging the
            // configurations of the two planes replaces the reference's
            // exchange of (idx, beta) (eamsim.cu:83-86), because all 32
            // samples of a word share one temperature per plane.
            const int64_t round = (s + 1) / p->sweeps_per_swap - 1;
            const int parity = (int)(round & 1);
            uint64_t boundary = 0;
#pragma omp parallel for collapse(2) schedule(static) num_threads(nthr) reduction(+ : boundary)
            for (int w = 0; w < W; ++w)
                for (int c = 0; c < C; ++c)
                    for (int t = parity; t + 1 < T; t += 2) {
                        int32_t* E0 = &E[(((size_t)w * C + c) * T + t) * 32];
                        int32_t* E1 = E0 + 32;
                        int32_t* M0 = &M[(((size_t)w * C + c) * T + t) * 32];
                        int32_t* M1 = M0 + 32;
                        uint32_t mask = 0;
                        for (int j = 0; j < 16; ++j) {
                            uint32_t r[4];
                            philox_ctr((uint32_t)j, (uint32_t)s, (uint32_t)(w + p->word0),
                                       kTagSwap | ((uint32_t)c << 8) | (uint32_t)t, p->seed, r);
                            for (int h = 0; h < 2; ++h) {
                                const int b = 2 * j + h;
                                const uint64_t bits = ((uint64_t)r[2 * h + 1] << 32) | r[2 * h];
                                const double u = (double)(bits >> 11) * 0x1p-53;
                                const double dE = (double)(E0[b] - E1[b]) - p->H * (double)(M0[b] - M1[b]);
                                const double delta = (p->betas[t] - p->betas[t + 1]) * dE;
                                bool acc = true;
                                if (delta < 0.0) {
                                    const double pr = std::exp(delta);
                                    if (std::fabs(u - pr) <= pr * 0x1p-40) ++boundary;
                                    acc = u < pr;
                                }
                                if (acc) mask |= 1u << b;
                            }
                        }
                        if (mask) {
                            for (int64_t si = 0; si < g.N; ++si) {
                                uint32_t& a = spins[D.spin(w, c, t, si)];
                                uint32_t& bb = spins[D.spin(w, c, t + 1, si)];
                                const uint32_t dd = (a ^ bb) & mask;
                                a ^= dd;
                                bb ^= dd;
                            }
                            for (int b = 0; b < 32; ++b)
                                if ((mask >> b) & 1u) {
                                    std::swap(E0[b], E1[b]);
                                    std::swap(M0[b], M1[b]);
                                }
                        }
                        if (obs && obs->swap_acc) {
#pragma omp atomic
                            obs->swap_acc[(size_t)c * T + t] += (uint64_t)__builtin_popcount(mask);
                        }
                        if (obs && obs->swap_log) {
                            const int64_t k = obs->swap_rounds;
                            if (k < obs->swap_log_rounds)
                                obs->swap_log[((((size_t)k * W + w) * C + c) * T) + t] = mask;
                        }
                    }
            if (obs) {
                obs->boundary += boundary;
                obs->swap_rounds += 1;
            }
        }

        if (do_meas && obs) {
            // Measurement: energies, magnetisations and the overlap
            // q = (1/N) sum_i s1_i s2_i of the two copies (eamsim.cu:477-504),
            // kept as integers: Q = N - 2D with D the number of differing sites.
            const size_t nE = (size_t)W * C * T * 32;
            for (size_t i = 0; i < nE; ++i) {
                if (obs->e_sum) obs->e_sum[i] += E[i];
                if (obs->m_sum) obs->m_sum[i] += M[i];
                if (obs->e_last) obs->e_last[i] = E[i];
                if (obs->m_last) obs->m_last[i] = M[i];
            }
            if (C == 2) {
                orc_overlaps(L, W, T, spins, Dq.data(), nullptr);
                for (int w = 0; w < W; ++w)
                    for (int t = 0; t < T; ++t)
                        for (int b = 0; b < 32; ++b) {
                            const size_t i = ((size_t)w * T + t) * 32 + b;
                            const int64_t Qv = g.N - 2 * (int64_t)Dq[i];
                            const uint64_t q2 = (uint64_t)(Qv * Qv);
                            const unsigned __int128 q4 = (unsigned __int128)q2 * q2;
                            if (obs->q_sum) obs->q_sum[i] += Qv;
                            if (obs->q2_sum) obs->q2_sum[i] += (int64_t)q2;
                            if (obs->q4_sum)
                                add_u128(obs->q4_sum + 2 * i, (uint64_t)q4, (uint64_t)(q4 >> 64));
                            if (obs->hist) obs->hist[(size_t)t * (g.N + 1) + Dq[i]] += 1;
                            if (obs->d_last) obs->d_last[i] = Dq[i];
                        }
            }
            obs->n_meas += 1;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

// Observable records of eamsim.cuh:55-62 for the current state.  e and m
// follow the float arithmetic of eamsim.cu:320-325 and :413-414; q_0 and
// q_1 follow eamsim.cu:477-509 with k = 2 pi / L, summed per coordinate
// plane in integers and combined in double.
int orc_obs_records(int32_t L, int32_t W, int32_t T, float H, const uint32_t* spins,
                    const uint32_t* bonds, float* rec) {
    if (!dims_ok(L, W, 2, T) || !rec) return 1;
    const int64_t N = (int64_t)L * L * L;
    std::vector<int32_t> e((size_t)W * 2 * T * 32), m(e.size()), d((size_t)W * T * 32),
        dpl((size_t)W * T * 32 * 3 * L);
    orc_energies(L, W, 2, T, spins, bonds, e.data(), m.data());
    orc_overlaps(L, W, T, spins, d.data(), dpl.data());
    const double k = 2.0 * M_PI / L;
    for (int w = 0; w < W; ++w)
        for (int b = 0; b < 32; ++b)
            for (int t = 0; t < T; ++t) {
                float* o = rec + (((size_t)(32 * w + b)) * T + t) * 11;
                for (int c = 0; c < 2; ++c) {
                    const size_t i = (((size_t)w * 2 + c) * T + t) * 32 + b;
                    const float es = (float)(-e[i]);  // 2 S - 3N
                    const float ms = (float)m[i];
                    o[c] = -(es + H * ms) / (float)N;
                    o[2 + c] = ms / (float)N;
                }
                const size_t i = ((size_t)w * T + t) * 32 + b;
                o[4] = (float)(N - 2 * (int64_t)d[i]) / (float)N;
                for (int dir = 0; dir < 3; ++dir) {
                    double re = 0.0, im = 0.0;
                    for (int a = 0; a < L; ++a) {
                        const int64_t P = (int64_t)L * L - 2 * (int64_t)dpl[(i * 3 + dir) * L + a];
                        re += (double)P * std::cos(k * a);
                        im += (double)P * std::sin(k * a);
                    }
                    o[5 + dir] = (float)(re / (double)N);
                    o[8 + dir] = (float)(im / (double)N);
                }
            }
    return 0;
}

// Reference lattice word (eamsim.cuh:27-35, eamsim.cu:598-616): bits 0..23
// spins by temperature index, bits 26..31 the bonds -x,+x,-y,+y,-z,+z with
// bit 1 = ferromagnetic; lattice index 2*sample + copy (eamsim.cu:632-640).
int orc_to_ref_lattice(int32_t L, int32_t W, int32_t T, const uint32_t* spins,
                       const uint32_t* bonds, uint32_t* ref) {
    if (!dims_ok(L, W, 2, T) || T > 24 || !ref) return 1;
    const Dims D(L, W, 2, T);
    const Geo& g = D.g;
    for (int w = 0; w < W; ++w)
        for (int z = 0; z < L; ++z)
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const int64_t si = g.slot(x, y, z), i = g.site(x, y, z);
                    const uint32_t f[6] = {bonds[D.bond(w, 0, g.slot(g.wrap(x - 1), y, z))],
                                           bonds[D.bond(w, 0, si)],
                                           bonds[D.bond(w, 1, g.slot(x, g.wrap(y - 1), z))],
                                           bonds[D.bond(w, 1, si)],
                                           bonds[D.bond(w, 2, g.slot(x, y, g.wrap(z - 1)))],
                                           bonds[D.bond(w, 2, si)]};
                    for (int b = 0; b < 32; ++b) {
                        uint32_t jbits = 0;
                        for (int k = 0; k < 6; ++k) jbits |= ((~f[k] >> b) & 1u) << (26 + k);
                        for (int c = 0; c < 2; ++c) {
                            uint32_t v = jbits;
                            for (int t = 0; t < T; ++t) v |= ((spins[D.spin(w, c, t, si)] >> b) & 1u) << t;
                            ref[((size_t)(2 * (32 * w + b) + c)) * g.N + i] = v;
                        }
                    }
                }
    return 0;
}

int orc_from_ref_lattice(int32_t L, int32_t W, int32_t T, const uint32_t* ref, uint32_t* spins,
                         uint32_t* bonds) {
    if (!dims_ok(L, W, 2, T) || T > 24 || !ref) return 1;
    const Dims D(L, W, 2, T);
    const Geo& g = D.g;
    int bad = 0;
    for (int w = 0; w < W; ++w)
        for (int z = 0; z < L; ++z)
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const int64_t si = g.slot(x, y, z), i = g.site(x, y, z);
                    uint32_t f[3] = {0, 0, 0};
                    for (int c = 0; c < 2; ++c)
                        for (int t = 0; t < T; ++t) spins[D.spin(w, c, t, si)] = 0;
                    for (int b = 0; b < 32; ++b) {
                        const uint32_t v0 = ref[((size_t)(2 * (32 * w + b))) * g.N + i];
                        const uint32_t v1 = ref[((size_t)(2 * (32 * w + b) + 1)) * g.N + i];
                        if ((v0 >> 26) != (v1 >> 26)) bad = 1;
                        for (int d = 0; d < 3; ++d) f[d] |= ((~v0 >> (27 + 2 * d)) & 1u) << b;
                        for (int t = 0; t < T; ++t) {
                            spins[D.spin(w, 0, t, si)] |= ((v0 >> t) & 1u) << b;
                            spins[D.spin(w, 1, t, si)] |= ((v1 >> t) & 1u) << b;
                        }
                    }
                    for (int d = 0; d < 3; ++d) bonds[D.bond(w, d, si)] = f[d];
                }
    // Each bond is stored at both of its ends; the "-" copy must agree.
    for (int w = 0; w < W && !bad; ++w)
        for (int z = 0; z < L; ++z)
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const int64_t i = g.site(x, y, z);
                    const int64_t nbs[3] = {g.site(g.wrap(x - 1), y, z), g.site(x, g.wrap(y - 1), z),
                                            g.site(x, y, g.wrap(z - 1))};
                    for (int b = 0; b < 32; ++b) {
                        const uint32_t v = ref[((size_t)(2 * (32 * w + b))) * g.N + i];
                        for (int d = 0; d < 3; ++d) {
                            const uint32_t vn = ref[((size_t)(2 * (32 * w + b))) * g.N + nbs[d]];
                            if (((v >> (26 + 2 * d)) & 1u) != ((vn >> (27 + 2 * d)) & 1u)) bad = 1;
                        }
                    }
                }
    return bad ? 2 : 0;
}

}  // extern "C"
