// csg_engine.cu — host side of libcsg.so: configuration checks, acceptance
// tables, launch planning, the sweep launches of both engines and the C ABI of
// one engine (include/csg.h).  The batched engine is batch.cpp, the request
// server server.cpp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "csg.h"
#include "engine_internal.h"
#include "philox.cuh"
#include "pt_kernel.cuh"
#include "aux_kernels.cuh"
#include "stream_kernels.cuh"

namespace csg {
// Advances a device-resident sweep counter after a launch of a captured graph.
__global__ void advance_counter(long long* counter, long long n) { *counter += n; }
}  // namespace csg

namespace csg_detail {

namespace {
thread_local std::string g_err;
}  // namespace

int fail(int code, const std::string& msg) {
    g_err = msg;
    return code;
}

void set_last_error(const std::string& msg) { g_err = msg; }

const std::string& last_error() { return g_err; }

}  // namespace csg_detail

using namespace csg_detail;

namespace {

constexpr int kMaxResidentL = 24;  // largest L of the cluster-resident kernel
constexpr int kMaxL = 128;         // largest L of the streaming engine

bool lattice_supported(int L) { return L >= 4 && L <= kMaxL && L % 2 == 0; }

}  // namespace

// Lattices whose quads do not fit in a cluster's shared memory run on the
// streaming engine; CSG_ENGINE_STREAM selects it for any L.
bool csg_detail::use_stream(const csg_config& c) {
    return c.dims.L > kMaxResidentL || (c.flags & CSG_ENGINE_STREAM);
}

int csg_detail::validate(const csg_config* cfg) {
    if (!cfg) return fail(CSG_ERR_ARG, "null configuration");
    const csg_dims& d = cfg->dims;
    if (d.L < 4 || d.L % 2 != 0) return fail(CSG_ERR_ARG, "L must be even and >= 4");
    if (!lattice_supported(d.L))
        return fail(CSG_ERR_UNSUPPORTED, "L=" + std::to_string(d.L) + " outside 4..128");
    if (d.n_words < 1) return fail(CSG_ERR_ARG, "n_words must be >= 1");
    if (d.n_copies != 1 && d.n_copies != 2) return fail(CSG_ERR_ARG, "n_copies must be 1 or 2");
    if (d.n_temps < 4 || d.n_temps > csg::kMaxT || d.n_temps % 4 != 0)
        return fail(CSG_ERR_ARG, "n_temps must be a multiple of 4 in 4..64");
    if (!(cfg->H >= 0.0 && cfg->H <= 4.0)) return fail(CSG_ERR_ARG, "H out of range");
    if (!cfg->betas) return fail(CSG_ERR_ARG, "null betas");
    for (int t = 0; t < d.n_temps; ++t)
        if (!(cfg->betas[t] >= 0.0) || !std::isfinite(cfg->betas[t]))
            return fail(CSG_ERR_ARG, "betas must be finite and >= 0");
    if (cfg->sched.sweeps_per_swap < 0 || cfg->sched.sweeps_per_meas < 0 ||
        cfg->sched.meas_start < 0)
        return fail(CSG_ERR_ARG, "negative schedule entry");
    if (cfg->swap_log_rounds < 0) return fail(CSG_ERR_ARG, "negative swap_log_rounds");
    if (cfg->word0 < 0) return fail(CSG_ERR_ARG, "negative word0");
    return CSG_OK;
}

namespace {

// Acceptance table: for centre spin bit s and U unsatisfied bonds the energy
// change of a flip is dE = 12 - 4U + 2H(2s-1); the flip is accepted when a
// 32-bit draw r satisfies r < floor(exp(-beta dE) 2^32), and always when
// that value reaches 2^32 (dE <= 0).  ucut[t][s] is the first such U.
// Returns whether the H=0 kernel (3 thresholds, U >= 3 always) describes the
// table exactly.
bool build_tables(const csg_config& cfg, csg::PtTables& tab) {
    std::memset(&tab, 0, sizeof(tab));
    bool h0_exact = true;
    for (int t = 0; t < cfg.dims.n_temps; ++t) {
        tab.beta[t] = cfg.betas[t];
        for (int s = 0; s < 2; ++s) {
            int cut = 7;
            for (int U = 0; U <= 6; ++U) {
                const double dE = 12.0 - 4.0 * U + 2.0 * cfg.H * (s ? 1.0 : -1.0);
                uint64_t v = (uint64_t)1 << 32;
                if (dE > 0.0) v = (uint64_t)(std::exp(-cfg.betas[t] * dE) * 4294967296.0);
                if (v >= ((uint64_t)1 << 32)) {
                    if (cut == 7) cut = U;
                    tab.thr[t][s][U] = 0xFFFFFFFFu;
                } else {
                    if (cut != 7) h0_exact = false;  // non-monotone (cannot happen for beta >= 0)
                    tab.thr[t][s][U] = (uint32_t)v;
                }
            }
            tab.ucut[t][s] = (uint8_t)cut;
            if (cut != 3) h0_exact = false;
            // cut <= 3 (s = 0) and cut <= 5 (s = 1) for 0 <= H <= 4 (validate()),
            // as the general-field rule (flip_gen) requires
        }
        for (int U = 0; U < 3; ++U)
            if (tab.thr[t][0][U] != tab.thr[t][1][U]) h0_exact = false;
    }
    return h0_exact && cfg.H == 0.0;
}

using KernelFn = csg::ResidentFn;

// The resident kernel for L (general-field variant when gen) with nseg column
// segments per thread; nullptr if that variant is not built.
KernelFn select_kernel(int L, bool gen, int nseg) {
    switch (L) {
        case 4: return csg::resident_kernel_L4(gen, nseg);
        case 6: return csg::resident_kernel_L6(gen, nseg);
        case 8: return csg::resident_kernel_L8(gen, nseg);
        case 10: return csg::resident_kernel_L10(gen, nseg);
        case 12: return csg::resident_kernel_L12(gen, nseg);
        case 14: return csg::resident_kernel_L14(gen, nseg);
        case 16: return csg::resident_kernel_L16(gen, nseg);
        case 18: return csg::resident_kernel_L18(gen, nseg);
        case 20: return csg::resident_kernel_L20(gen, nseg);
        case 22: return csg::resident_kernel_L22(gen, nseg);
        case 24: return csg::resident_kernel_L24(gen, nseg);
        default: return nullptr;
    }
}

size_t smem_for(int L, int Qc, bool has_m, bool gen) {
    switch (L) {
        case 4: return csg::SmemMap<4>::bytes(Qc, has_m, gen);
        case 6: return csg::SmemMap<6>::bytes(Qc, has_m, gen);
        case 8: return csg::SmemMap<8>::bytes(Qc, has_m, gen);
        case 10: return csg::SmemMap<10>::bytes(Qc, has_m, gen);
        case 12: return csg::SmemMap<12>::bytes(Qc, has_m, gen);
        case 14: return csg::SmemMap<14>::bytes(Qc, has_m, gen);
        case 16: return csg::SmemMap<16>::bytes(Qc, has_m, gen);
        case 18: return csg::SmemMap<18>::bytes(Qc, has_m, gen);
        case 20: return csg::SmemMap<20>::bytes(Qc, has_m, gen);
        case 22: return csg::SmemMap<22>::bytes(Qc, has_m, gen);
        case 24: return csg::SmemMap<24>::bytes(Qc, has_m, gen);
        default: return 0;
    }
}

constexpr size_t kMaxSmem = 227 * 1024;

// Shared-memory carve-out (percent) that holds a CTA of smem bytes (plus the
// 1 KB the system reserves per CTA): the rest of the SM's 256 KB stays L1 for
// the bonds.
int carveout_pct(size_t smem) {
    const int pct = (int)((smem + 1024) * 100 / (228 * 1024));
    return pct < 100 ? pct : 100;
}

std::mutex g_plan_mu;
csg_plan g_override = {0, 0, 0, 0};

int prepare_kernel(KernelFn fn, size_t smem, int K) {
    // the limit covers every plan of this kernel (several engines may share it)
    CSG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kMaxSmem));
    // the smallest carve-out that holds the CTA (also given per launch)
    CSG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  carveout_pct(smem)));
    if (K > 8) CSG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    return CSG_OK;
}

// attr must hold 2 entries.  The carve-out travels with the launch (and with
// a graph's kernel node), so plans of other engines that set the kernel's
// own carve-out attribute do not change it.
void fill_launch(cudaLaunchConfig_t& lc, cudaLaunchAttribute* attr, int W, const Plan& pl,
                 cudaStream_t st) {
    lc = cudaLaunchConfig_t{};
    lc.gridDim = dim3((unsigned)(W * pl.K), 1, 1);
    lc.blockDim = dim3((unsigned)pl.threads, 1, 1);
    lc.dynamicSmemBytes = pl.smem;
    lc.stream = st;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = (unsigned)pl.K;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    attr[1].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
    attr[1].val.sharedMemCarveout = (unsigned)carveout_pct(pl.smem);
    lc.attrs = attr;
    lc.numAttrs = 2;
}

// Launch plan: split the G = C*T/4 quads of a word over K = G/Qc CTAs of a
// cluster, each quad's team of TPQ = L * L/2 * NSEG threads.  The score is the
// number of quads the busiest SM must sweep (waves of co-resident clusters
// times the quads per SM in a wave); ties go to the smaller cluster (fewer
// cross-CTA exchanges), then to the default column split.  Fields of `forced`
// (and of the process-wide override) that are non-zero fix that part.
int make_plan(const csg_config& cfg, bool gen, Plan& out, PlanChoice forced = PlanChoice{}) {
    const int L = cfg.dims.L, W = cfg.dims.n_words;
    const int G = cfg.dims.n_copies * cfg.dims.n_temps / 4;
    if (use_stream(cfg)) {  // fixed launch shapes, nothing to plan
        out = Plan{};
        int nt = 0, smem = 0;
        if (cfg.flags & CSG_STREAM_FUSED) csg::stream_sweep_shape(L, &nt, &smem);
        if (nt > 0) {  // fused sweep launch: one CTA per quad, no clusters
            out.Qc = 1;
            out.K = G;
            out.TPQ = nt;
            out.threads = nt;
            out.smem = (size_t)smem;
        } else {  // colour launches
            out.TPQ = csg::kStreamThreads;
        }
        return CSG_OK;
    }
    const bool has_m = gen || (cfg.flags & CSG_MEASURE_M);
    {
        std::lock_guard<std::mutex> lk(g_plan_mu);
        if (forced.qc == 0) forced.qc = g_override.quads_per_cta;
        if (forced.nseg == 0 && g_override.threads_per_quad > 0)
            forced.nseg = g_override.threads_per_quad / (L * (L / 2));
    }
    if (forced.qc < 0 || forced.nseg < 0) return fail(CSG_ERR_ARG, "negative plan entry");
    if (forced.qc > 0 && G % forced.qc != 0)
        return fail(CSG_ERR_ARG, "plan override does not divide the quads");
    int dev = 0, nsm = 0;
    CSG_CUDA(cudaGetDevice(&dev));
    CSG_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    long best = -1;
    for (int oi = 0; csg::nseg_option(L, oi) > 0; ++oi) {
        const int nseg = csg::nseg_option(L, oi);
        if (forced.nseg > 0 && nseg != forced.nseg) continue;
        KernelFn fn = select_kernel(L, gen, nseg);
        if (!fn) continue;
        for (int Qc = 1; Qc <= G; ++Qc) {
            if (G % Qc || (forced.qc > 0 && Qc != forced.qc)) continue;
            Plan pl;
            pl.Qc = Qc;
            pl.K = G / Qc;
            pl.NSEG = nseg;
            pl.TPQ = csg::threads_per_quad(L, nseg);
            pl.threads = (Qc * pl.TPQ + 31) / 32 * 32;
            pl.smem = smem_for(L, Qc, has_m, gen);
            if (pl.K > 16 || pl.smem > kMaxSmem || pl.threads > csg::max_cta_threads(gen, nseg))
                continue;
            if (prepare_kernel(fn, pl.smem, pl.K) != CSG_OK) continue;
            cudaLaunchConfig_t lc;
            cudaLaunchAttribute attr[2];
            fill_launch(lc, attr, W, pl, nullptr);
            int nclusters = 0;
            if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &lc) != cudaSuccess || nclusters < 1) {
                cudaGetLastError();
                continue;
            }
            const long waves = (W + nclusters - 1) / nclusters;
            const long per_wave = (long)std::min(W, nclusters) * pl.K;
            const long load = waves * ((per_wave + nsm - 1) / nsm) * Qc;
            const long score = (load * 64 + pl.K) * 8 + oi;
            if (best < 0 || score < best) {
                best = score;
                out = pl;
            }
        }
    }
    if (best < 0)
        return fail(CSG_ERR_UNSUPPORTED, forced.qc > 0 || forced.nseg > 0
                                             ? "plan override exceeds device limits"
                                             : "no launch plan fits this configuration");
    return prepare_kernel(select_kernel(L, gen, out.NSEG), out.smem, out.K);
}

int64_t count_events(int64_t s0, int64_t n, int64_t k, int64_t first_sweep) {
    // number of s in [max(s0, first_sweep), s0+n) with (s+1) % k == 0
    if (k <= 0 || n <= 0) return 0;
    const int64_t lo = std::max(s0, first_sweep) + 1, hi = s0 + n;
    if (hi < lo) return 0;
    return hi / k - (lo - 1) / k;
}

int fill_params(const csg_config& cfg, csg::PtParams& P, bool& gen) {
    std::memset(&P, 0, sizeof(P));
    gen = !build_tables(cfg, P.tab);
    P.H = cfg.H;
    P.k0 = (uint32_t)cfg.seed;
    P.k1 = (uint32_t)(cfg.seed >> 32);
    P.word0 = (uint32_t)cfg.word0;
    P.W = cfg.dims.n_words;
    P.C = cfg.dims.n_copies;
    P.T = cfg.dims.n_temps;
    P.Q = cfg.dims.n_temps / 4;
    P.sps = cfg.sched.sweeps_per_swap;
    P.spm = cfg.sched.sweeps_per_meas;
    P.meas_start = cfg.sched.meas_start;
    P.flags = (cfg.flags & CSG_MEASURE_M) ? csg::kFlagMeasureM : 0;
    return CSG_OK;
}

constexpr int64_t kSweepsPerLaunch = 1024;

// ---------------------------------------------------------------------------
// Streaming engine (stream_kernels.cuh): scratch layout and the launch
// sequence of one sweep.
// ---------------------------------------------------------------------------
struct StreamLayout {
    int nblk = 0, nblk_plain = 0, nblk2 = 0;
    size_t u_acc = 0, up_acc = 0, d_acc = 0, energy = 0, magn = 0, masks = 0, err = 0, bytes = 0;
};

StreamLayout stream_layout(const csg_config& c) {
    const csg_dims& d = c.dims;
    const size_t N = (size_t)d.L * d.L * d.L;
    const size_t spb = (size_t)csg::kStreamThreads * csg::kStreamSPT;
    const size_t spa = csg::kStreamAccSitesPerBlock, spo = csg::kOverlapSitesPerBlock;
    StreamLayout s;
    s.nblk = (int)((N / 2 + spa - 1) / spa);  // blocks of the counting colour launches
    s.nblk_plain = (int)((N / 2 + spb - 1) / spb);
    s.nblk2 = (int)((N + spo - 1) / spo);
    const size_t planes = (size_t)d.n_words * d.n_copies * d.n_temps;
    auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t off = 0;
    s.u_acc = off, off += up(planes * 32 * 4);
    s.up_acc = off, off += up(planes * 32 * 4);
    s.d_acc = off, off += up((size_t)d.n_words * d.n_temps * 32 * 4);
    s.energy = off, off += up(planes * 32 * 4);
    s.magn = off, off += up(planes * 32 * 4);
    s.masks = off, off += up(planes * 4);
    s.err = off, off += 256;
    s.bytes = off;
    return s;
}

// A launch of the streaming engine's sweep sequence, with programmatic
// dependent launch (the kernels wait for their predecessor in pdl_enter()).
template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, cudaStream_t st,
                       Args&&... args) {
    cudaLaunchConfig_t lc = {};
    lc.gridDim = grid;
    lc.blockDim = block;
    lc.dynamicSmemBytes = 0;
    lc.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    lc.attrs = attr;
    lc.numAttrs = 1;
    return cudaLaunchKernelEx(&lc, kernel, std::forward<Args>(args)...);
}

using ColourLaunch = void (*)(const csg::StreamParams&, const StreamLayout&, int, long long,
                              cudaStream_t);

template <bool G, bool E, bool M>
void launch_colour(const csg::StreamParams& S, const StreamLayout& lay, int p, long long s,
                   cudaStream_t st) {
    const dim3 grid((unsigned)(S.W * S.C * S.Q), (unsigned)(E || M ? lay.nblk : lay.nblk_plain));
    launch_pdl(csg::stream_colour_kernel<G, E, M>, grid, dim3(csg::colour_threads<E || M>()), st, S, p, s);
}

ColourLaunch colour_launch(bool gen, bool acc_e, bool acc_m) {
    static const ColourLaunch fns[8] = {
        launch_colour<false, false, false>, launch_colour<false, false, true>,
        launch_colour<false, true, false>,  launch_colour<false, true, true>,
        launch_colour<true, false, false>,  launch_colour<true, false, true>,
        launch_colour<true, true, false>,   launch_colour<true, true, true>};
    return fns[(gen ? 4 : 0) + (acc_e ? 2 : 0) + (acc_m ? 1 : 0)];
}

// Same schedule, Philox counters and arithmetic as the resident kernel's sweep
// loop; per sweep: colour 0, colour 1 (energies, magnetisations when needed),
// then the exchange decisions, the masked exchange and the measurement.
int run_stream(const csg_config& cfg, uint32_t* spins, const uint32_t* bonds,
               const csg_device_obs* obs, int64_t sweep0, int64_t n_sweeps, cudaStream_t st) {
    csg::PtParams tp;
    bool gen = false;
    fill_params(cfg, tp, gen);
    const csg_dims& d = cfg.dims;
    const StreamLayout lay = stream_layout(cfg);
    csg::StreamParams S;
    std::memset(&S, 0, sizeof(S));
    S.spins = spins;
    S.bonds = bonds;
    S.L = d.L;
    S.W = d.n_words;
    S.C = d.n_copies;
    S.T = d.n_temps;
    S.Q = d.n_temps / 4;
    S.nblk = lay.nblk;
    S.nblk2 = lay.nblk2;
    S.k0 = tp.k0;
    S.k1 = tp.k1;
    S.word0 = tp.word0;
    S.H = tp.H;
    auto magic = [](uint64_t d) { return (uint32_t)(((uint64_t)1 << 32) / d + ((((uint64_t)1 << 32) % d) ? 1 : 0)); };
    S.mag_plane = magic((uint64_t)d.L * (d.L / 2));
    S.mag_row = magic((uint64_t)(d.L / 2));
    S.tab = tp.tab;
    csg::StreamObs O{};
    unsigned long long *boundary = nullptr, *swap_acc = nullptr;
    unsigned int* swap_log = nullptr;
    long long log_rounds = 0, round0 = 0;
    if (obs) {
        O.e_sum = reinterpret_cast<long long*>(obs->e_sum);
        O.m_sum = reinterpret_cast<long long*>(obs->m_sum);
        O.q_sum = reinterpret_cast<long long*>(obs->q_sum);
        O.q2_sum = reinterpret_cast<long long*>(obs->q2_sum);
        O.q4_sum = reinterpret_cast<unsigned long long*>(obs->q4_sum);
        O.hist = obs->hist;
        O.e_last = obs->e_last;
        O.m_last = obs->m_last;
        O.d_last = obs->d_last;
        boundary = reinterpret_cast<unsigned long long*>(obs->boundary);
        swap_acc = reinterpret_cast<unsigned long long*>(obs->swap_acc);
        swap_log = obs->swap_log;
        log_rounds = obs->swap_log_rounds;
        round0 = obs->swap_round0;
    }
    char* base = nullptr;
    CSG_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&base), lay.bytes, st));
    S.u_acc = reinterpret_cast<int*>(base + lay.u_acc);
    S.up_acc = reinterpret_cast<int*>(base + lay.up_acc);
    S.d_acc = reinterpret_cast<int*>(base + lay.d_acc);
    // the totals start at zero; each consumer clears what it read
    CSG_CUDA(cudaMemsetAsync(base + lay.u_acc, 0, lay.energy - lay.u_acc, st));
    S.energy = reinterpret_cast<int*>(base + lay.energy);
    S.magn = reinterpret_cast<int*>(base + lay.magn);
    S.masks = reinterpret_cast<uint32_t*>(base + lay.masks);
    S.err = reinterpret_cast<int*>(base + lay.err);
    CSG_CUDA(cudaMemsetAsync(S.err, 0, sizeof(int), st));
    // one fused launch per sweep where asked for and its ring of z-planes fits
    const bool fused = (cfg.flags & CSG_STREAM_FUSED) && csg::stream_sweep_fits(d.L);

    const long N = (long)d.L * d.L * d.L;
    const unsigned W = (unsigned)d.n_words, C = (unsigned)d.n_copies, Q = (unsigned)S.Q;
    const dim3 g_exchange(W * C, (unsigned)((N + 255) / 256));
    const dim3 g_overlap(W * Q, (unsigned)lay.nblk2);
    const int64_t sps = cfg.sched.sweeps_per_swap, spm = cfg.sched.sweeps_per_meas;
    cudaError_t ce = cudaSuccess;
    for (int64_t i = 0; i < n_sweeps && ce == cudaSuccess; ++i) {
        const long long s = sweep0 + i;
        const bool do_swap = sps > 0 && (s + 1) % sps == 0;
        const bool do_meas = spm > 0 && (s + 1) % spm == 0 && s >= cfg.sched.meas_start;
        const bool need_E = do_swap || do_meas;
        const bool need_M = need_E && (gen || (do_meas && (cfg.flags & CSG_MEASURE_M)));
        if (fused) {
            ce = csg::launch_stream_sweep(S, s, gen, need_E, need_M, st);
            if (ce != cudaSuccess) break;
        } else {
            colour_launch(gen, false, need_M)(S, lay, 0, s, st);
            colour_launch(gen, need_E, need_M)(S, lay, 1, s, st);
        }
        if (need_E) {
            const long long round = do_swap ? (s + 1) / sps - 1 : 0;
            const int par = (int)(round & 1);
            launch_pdl(csg::stream_decide_kernel, dim3(W * C), dim3(std::min(1024, 32 * d.n_temps)), st,
                       S, s, par, need_M, do_swap, boundary, swap_acc, swap_log, round - round0,
                       log_rounds);
            const bool overlap = do_meas && obs && C == 2;
            if (do_swap && overlap)  // one pass: exchange, then count the overlaps
                launch_pdl(csg::stream_exchange_overlap_kernel, dim3(W, (unsigned)lay.nblk2),
                           dim3(csg::kStreamThreads), st, S, par);
            else if (do_swap)
                launch_pdl(csg::stream_exchange_kernel, g_exchange, dim3(256), st, S, par);
            else if (overlap)
                launch_pdl(csg::stream_overlap_kernel, g_overlap, dim3(csg::kStreamThreads), st, S);
            if (do_meas && obs)
                launch_pdl(csg::stream_measure_kernel, dim3(W * (unsigned)d.n_temps), dim3(64), st, S,
                           need_M, O);
        }
        ce = cudaGetLastError();
    }
    // the fused launches report a staging wait that gave up
    int err = 0;
    if (ce == cudaSuccess && fused) {
        ce = cudaMemcpyAsync(&err, S.err, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    }
    const cudaError_t ce2 = cudaFreeAsync(base, st);
    if (ce != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("stream launch: ") + cudaGetErrorString(ce));
    if (ce2 != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("cudaFreeAsync: ") + cudaGetErrorString(ce2));
    if (err) return fail(CSG_ERR_CUDA, "streaming engine: a shared-memory staging wait gave up");
    return CSG_OK;
}

}  // namespace

int csg_detail::run_device(const csg_config& cfg, uint32_t* spins, const uint32_t* bonds,
                           const csg_device_obs* obs, int64_t sweep0, int64_t n_sweeps,
                           cudaStream_t st, PlanChoice forced, long long* sweep_dev,
                           const Plan* plan_in) {
    if (use_stream(cfg)) {
        if (sweep_dev)
            return fail(CSG_ERR_UNSUPPORTED, "the streaming engine takes no device sweep counter");
        return run_stream(cfg, spins, bonds, obs, sweep0, n_sweeps, st);
    }
    csg::PtParams P;
    bool gen = false;
    fill_params(cfg, P, gen);
    Plan pl;
    if (plan_in)
        pl = *plan_in;  // planned before a stream capture
    else if (int rc = make_plan(cfg, gen, pl, forced))
        return rc;
    P.sweep_dev = sweep_dev;
    KernelFn fn = select_kernel(cfg.dims.L, gen, pl.NSEG);
    if (!fn) return fail(CSG_ERR_UNSUPPORTED, "no resident kernel for this plan");
    P.spins = spins;
    P.bonds = bonds;
    if (obs) {
        P.e_sum = reinterpret_cast<long long*>(obs->e_sum);
        P.m_sum = reinterpret_cast<long long*>(obs->m_sum);
        P.q_sum = reinterpret_cast<long long*>(obs->q_sum);
        P.q2_sum = reinterpret_cast<long long*>(obs->q2_sum);
        P.q4_sum = reinterpret_cast<unsigned long long*>(obs->q4_sum);
        P.hist = obs->hist;
        P.e_last = obs->e_last;
        P.m_last = obs->m_last;
        P.d_last = obs->d_last;
        P.swap_acc = reinterpret_cast<unsigned long long*>(obs->swap_acc);
        P.swap_log = obs->swap_log;
        P.swap_log_rounds = obs->swap_log_rounds;
        P.swap_round0 = obs->swap_round0;
        P.boundary = reinterpret_cast<unsigned long long*>(obs->boundary);
    }
    P.K = pl.K;
    P.Qc = pl.Qc;
    for (int64_t done = 0; done < n_sweeps; done += kSweepsPerLaunch) {
        // with a device counter the launches of a section read their start
        // from it (advanced after each launch); otherwise from the offset
        P.sweep0 = sweep_dev ? sweep0 : sweep0 + done;
        P.n_sweeps = (int)std::min<int64_t>(kSweepsPerLaunch, n_sweeps - done);
        cudaLaunchConfig_t lc;
        cudaLaunchAttribute attr[2];
        fill_launch(lc, attr, cfg.dims.n_words, pl, st);
        CSG_CUDA(cudaLaunchKernelEx(&lc, fn, P));
        if (sweep_dev) {
            csg::advance_counter<<<1, 1, 0, st>>>(sweep_dev, (long long)P.n_sweeps);
            CSG_CUDA(cudaGetLastError());
        }
    }
    return CSG_OK;
}


int csg_detail::chain_launch_starts(cudaGraph_t g, const std::vector<const csg_engine*>& members,
                                    const std::vector<int>& nseg) {
    // each member's resident kernel: a node is one of its launches when it
    // runs that kernel on the member's state buffer
    std::vector<const void*> fns(members.size());
    for (size_t i = 0; i < members.size(); ++i) {
        csg::PtParams P;
        bool gen = false;
        fill_params(members[i]->cfg, P, gen);
        fns[i] = reinterpret_cast<const void*>(select_kernel(members[i]->cfg.dims.L, gen, nseg[i]));
    }
    size_t n = 0;
    CSG_CUDA(cudaGraphGetNodes(g, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    CSG_CUDA(cudaGraphGetNodes(g, nodes.data(), &n));
    std::vector<cudaGraphNode_t> first(members.size(), nullptr);
    for (cudaGraphNode_t node : nodes) {
        cudaGraphNodeType type;
        CSG_CUDA(cudaGraphNodeGetType(node, &type));
        if (type != cudaGraphNodeTypeKernel) continue;
        // a section's first launch is its branch's root; later launches of a
        // section longer than one launch follow the sweep counter's kernel
        size_t n_deps = 0;
        CSG_CUDA(cudaGraphNodeGetDependencies(node, nullptr, &n_deps));
        if (n_deps != 0) continue;
        cudaKernelNodeParams kp = {};
        CSG_CUDA(cudaGraphKernelNodeGetParams(node, &kp));
        for (size_t i = 0; i < members.size(); ++i) {
            if (kp.func != fns[i] || !kp.kernelParams) continue;
            const csg::PtParams* P = static_cast<const csg::PtParams*>(kp.kernelParams[0]);
            if (P->spins == members[i]->spins) first[i] = node;
        }
    }
    for (size_t i = 1; i < first.size(); ++i) {
        if (!first[i - 1] || !first[i]) return fail(CSG_ERR_STATE, "captured launch not found");
        cudaGraphEdgeData ed = {};
        ed.from_port = cudaGraphKernelNodePortLaunchCompletion;
        ed.to_port = 0;
        ed.type = cudaGraphDependencyTypeProgrammatic;
        CSG_CUDA(cudaGraphAddDependencies_v2(g, &first[i - 1], &first[i], &ed, 1));
    }
    return CSG_OK;
}

std::vector<PlanChoice> csg_detail::plan_options(const csg_config& c) {
    std::vector<PlanChoice> out;
    if (use_stream(c)) return out;
    csg::PtParams P;
    bool gen = false;
    fill_params(c, P, gen);
    const int L = c.dims.L, G = c.dims.n_copies * c.dims.n_temps / 4;
    const bool has_m = gen || (c.flags & CSG_MEASURE_M);
    for (int oi = 0; csg::nseg_option(L, oi) > 0; ++oi) {
        const int nseg = csg::nseg_option(L, oi);
        const int tpq = csg::threads_per_quad(L, nseg);
        for (int qc = 1; qc <= G; ++qc)
            if (G % qc == 0 && G / qc <= 16 && smem_for(L, qc, has_m, gen) <= kMaxSmem &&
                (qc * tpq + 31) / 32 * 32 <= csg::max_cta_threads(gen, nseg))
                out.push_back(PlanChoice{qc, nseg});
    }
    return out;
}

int csg_detail::plan_engine(csg_engine* e, Plan& pl, size_t min_smem) {
    csg::PtParams P;
    bool gen = false;
    fill_params(e->cfg, P, gen);
    if (int rc = make_plan(e->cfg, gen, pl, PlanChoice{e->qc, e->nseg})) return rc;
    if (pl.smem < min_smem && !use_stream(e->cfg)) {
        pl.smem = min_smem;
        return prepare_kernel(select_kernel(e->cfg.dims.L, gen, pl.NSEG), pl.smem, pl.K);
    }
    return CSG_OK;
}

size_t csg_detail::footprint_bytes(const csg_config& c) {
    const csg_dims& d = c.dims;
    const size_t N = (size_t)d.L * d.L * d.L;
    const size_t ne = (size_t)d.n_words * d.n_copies * d.n_temps * 32;
    const size_t nq = d.n_copies == 2 ? (size_t)d.n_words * d.n_temps * 32 : 0;
    const size_t nh = d.n_copies == 2 ? (size_t)d.n_temps * (N + 1) : 0;
    return (size_t)d.n_words * d.n_copies * d.n_temps * N * 4 + (size_t)d.n_words * 3 * N * 4 +
           ne * (8 + 8 + 4 + 4) + nq * (8 + 8 + 16 + 4) + nh * 4 +
           (size_t)d.n_copies * d.n_temps * 8 + (size_t)c.swap_log_rounds * ne / 32 * 4 + 8 +
           (use_stream(c) ? stream_layout(c).bytes : 0);
}

void csg_detail::account(csg_engine* e, int64_t n) {
    const csg_schedule& sc = e->cfg.sched;
    e->swap_rounds += count_events(e->sweep, n, sc.sweeps_per_swap, 0);
    e->n_meas += count_events(e->sweep, n, sc.sweeps_per_meas, sc.meas_start);
    e->sweep += n;
}

csg_device_obs csg_detail::device_obs(const csg_engine* e) {
    csg_device_obs o{};
    o.e_sum = e->e_sum;
    o.m_sum = e->m_sum;
    o.q_sum = e->q_sum;
    o.q2_sum = e->q2_sum;
    o.q4_sum = e->q4_sum;
    o.hist = e->hist;
    o.e_last = e->e_last;
    o.m_last = e->m_last;
    o.d_last = e->d_last;
    o.swap_acc = e->swap_acc;
    o.swap_log = e->swap_log;
    o.swap_log_rounds = e->cfg.swap_log_rounds;
    o.swap_round0 = e->swap_round0;
    o.boundary = e->boundary;
    return o;
}

// ---------------------------------------------------------------------------
// Engine object
// ---------------------------------------------------------------------------
namespace {

void free_engine(csg_engine* e) {
    void* ptrs[] = {e->spins, e->bonds, e->e_sum, e->m_sum, e->q_sum, e->q2_sum, e->q4_sum,
                    e->hist, e->e_last, e->m_last, e->d_last, e->swap_acc, e->swap_log,
                    e->boundary, e->rec_scratch};
    for (void* p : ptrs) {
        if (!p) continue;
        if (e->pool)
            cudaFreeAsync(p, e->stream);  // back to the pool after the stream's work
        else
            cudaFree(p);
    }
    if (e->stream && e->own_stream) cudaStreamDestroy(e->stream);
}

int reset_obs(csg_engine* e) {
    struct Z {
        void* p;
        size_t bytes;
    } z[] = {{e->e_sum, e->n_e * 8}, {e->m_sum, e->n_e * 8}, {e->q_sum, e->n_q * 8},
             {e->q2_sum, e->n_q * 8}, {e->q4_sum, e->n_q * 16}, {e->hist, e->n_hist * 4},
             {e->e_last, e->n_e * 4}, {e->m_last, e->n_e * 4}, {e->d_last, e->n_q * 4},
             {e->swap_acc, (size_t)e->cfg.dims.n_copies * e->cfg.dims.n_temps * 8},
             {e->swap_log, (size_t)e->cfg.swap_log_rounds * e->n_e / 32 * 4},
             {e->boundary, 8}};
    for (auto& zz : z)
        if (zz.p && zz.bytes) CSG_CUDA(cudaMemsetAsync(zz.p, 0, zz.bytes, e->stream));
    e->n_meas = 0;
    e->swap_rounds = 0;
    const int64_t k = e->cfg.sched.sweeps_per_swap;
    e->swap_round0 = k > 0 ? (e->sweep + k) / k - 1 : 0;
    return CSG_OK;
}

}  // namespace

int csg_detail::engine_alloc(csg_engine* e, void** p, size_t bytes) {
    *p = nullptr;
    if (bytes == 0) return CSG_OK;
    const cudaError_t ce = e->pool ? cudaMallocFromPoolAsync(p, bytes, e->pool, e->stream)
                                   : cudaMalloc(p, bytes);
    if (ce != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(CSG_ERR_NOMEM, std::string(e->pool ? "cudaMallocFromPoolAsync: " : "cudaMalloc: ") +
                                       cudaGetErrorString(ce));
    }
    return CSG_OK;
}

int csg_detail::engine_create_pooled(const csg_config* cfg, cudaMemPool_t pool, cudaStream_t stream,
                                     csg_engine** out) {
    if (!out) return fail(CSG_ERR_ARG, "null output pointer");
    *out = nullptr;
    if (int rc = validate(cfg)) return rc;
    csg_engine* e = new (std::nothrow) csg_engine();
    if (!e) return fail(CSG_ERR_NOMEM, "host allocation failed");
    e->cfg = *cfg;
    e->betas.assign(cfg->betas, cfg->betas + cfg->dims.n_temps);
    e->cfg.betas = e->betas.data();
    const csg_dims& d = cfg->dims;
    const size_t N = (size_t)d.L * d.L * d.L;
    e->n_spins = (size_t)d.n_words * d.n_copies * d.n_temps * N;
    e->n_bonds = (size_t)d.n_words * 3 * N;
    e->n_e = (size_t)d.n_words * d.n_copies * d.n_temps * 32;
    e->n_q = d.n_copies == 2 ? (size_t)d.n_words * d.n_temps * 32 : 0;
    e->n_hist = d.n_copies == 2 ? (size_t)d.n_temps * (N + 1) : 0;
    if (pool) {
        e->pool = pool;
        e->stream = stream;
        e->own_stream = false;
    } else if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        e->stream = nullptr;
        delete e;
        return fail(CSG_ERR_CUDA, "cudaStreamCreate failed");
    }
    int rc = CSG_OK;
    // stops at the first failure (nothing more is allocated)
    auto alloc = [&](auto** p, size_t n) {
        if (rc == CSG_OK) rc = engine_alloc(e, reinterpret_cast<void**>(p), n * sizeof(**p));
    };
    alloc(&e->spins, e->n_spins);
    alloc(&e->bonds, e->n_bonds);
    alloc(&e->e_sum, e->n_e);
    alloc(&e->m_sum, e->n_e);
    alloc(&e->e_last, e->n_e);
    alloc(&e->m_last, e->n_e);
    alloc(&e->q_sum, e->n_q);
    alloc(&e->q2_sum, e->n_q);
    alloc(&e->q4_sum, 2 * e->n_q);
    alloc(&e->d_last, e->n_q);
    alloc(&e->hist, e->n_hist);
    alloc(&e->swap_acc, (size_t)d.n_copies * d.n_temps);
    alloc(&e->swap_log, (size_t)cfg->swap_log_rounds * e->n_e / 32);
    alloc(&e->boundary, 1);
    if (rc == CSG_OK) rc = reset_obs(e);
    if (rc == CSG_OK) {
        // A launch plan must exist before the engine is handed out.
        csg::PtParams P;
        bool gen = false;
        fill_params(e->cfg, P, gen);
        Plan pl;
        rc = make_plan(e->cfg, gen, pl);
    }
    if (rc != CSG_OK) {
        const std::string msg = last_error();
        free_engine(e);
        delete e;
        set_last_error(msg);
        return rc;
    }
    *out = e;
    return CSG_OK;
}

void csg_detail::engine_release(csg_engine* e) {
    if (!e) return;
    free_engine(e);
    delete e;
}

extern "C" {

const char* csg_last_error(void) { return last_error().c_str(); }

int csg_engine_footprint(const csg_config* cfg, size_t* bytes) {
    if (int rc = validate(cfg)) return rc;
    if (!bytes) return fail(CSG_ERR_ARG, "null output");
    *bytes = footprint_bytes(*cfg);
    return CSG_OK;
}

int csg_engine_create(const csg_config* cfg, csg_engine** out) {
    return engine_create_pooled(cfg, nullptr, nullptr, out);
}

int csg_engine_destroy(csg_engine* e) {
    if (!e) return CSG_OK;
    if (e->stream) cudaStreamSynchronize(e->stream);
    free_engine(e);
    delete e;
    return CSG_OK;
}

int csg_init_device(const csg_config* cfg, uint32_t* spins, uint32_t* bonds, void* stream) {
    if (int rc = validate(cfg)) return rc;
    if (!spins || !bonds) return fail(CSG_ERR_ARG, "null device buffer");
    const csg_dims& d = cfg->dims;
    const long N = (long)d.L * d.L * d.L;
    const long total = (long)d.n_words * N;
    const int block = 256;
    csg::init_kernel<<<(unsigned)((total + block - 1) / block), block, 0, (cudaStream_t)stream>>>(
        spins, bonds, d.L, d.n_words, d.n_copies, d.n_temps / 4, (uint32_t)cfg->seed,
        (uint32_t)(cfg->seed >> 32), (uint32_t)cfg->word0);
    CSG_CUDA(cudaGetLastError());
    return CSG_OK;
}

int csg_init_lattice(csg_engine* e) {
    if (!e) return fail(CSG_ERR_ARG, "null engine");
    if (int rc = csg_init_device(&e->cfg, e->spins, e->bonds, e->stream)) return rc;
    e->sweep = 0;
    return reset_obs(e);
}

int csg_set_state(csg_engine* e, const uint32_t* spins, size_t n_spins, const uint32_t* bonds,
                  size_t n_bonds, int64_t sweep) {
    if (!e) return fail(CSG_ERR_ARG, "null engine");
    if (!spins || n_spins != e->n_spins) return fail(CSG_ERR_ARG, "spins size mismatch");
    if (!bonds || n_bonds != e->n_bonds) return fail(CSG_ERR_ARG, "bonds size mismatch");
    if (sweep < 0) return fail(CSG_ERR_ARG, "negative sweep index");
    CSG_CUDA(cudaMemcpyAsync(e->spins, spins, n_spins * 4, cudaMemcpyHostToDevice, e->stream));
    CSG_CUDA(cudaMemcpyAsync(e->bonds, bonds, n_bonds * 4, cudaMemcpyHostToDevice, e->stream));
    e->sweep = sweep;
    return reset_obs(e);
}

int csg_get_state(csg_engine* e, uint32_t* spins, size_t n_spins, uint32_t* bonds,
                  size_t n_bonds, int64_t* sweep) {
    if (!e) return fail(CSG_ERR_ARG, "null engine");
    if (spins) {
        if (n_spins != e->n_spins) return fail(CSG_ERR_ARG, "spins size mismatch");
        CSG_CUDA(cudaMemcpyAsync(spins, e->spins, n_spins * 4, cudaMemcpyDeviceToHost, e->stream));
    }
    if (bonds) {
        if (n_bonds != e->n_bonds) return fail(CSG_ERR_ARG, "bonds size mismatch");
        CSG_CUDA(cudaMemcpyAsync(bonds, e->bonds, n_bonds * 4, cudaMemcpyDeviceToHost, e->stream));
    }
    CSG_CUDA(cudaStreamSynchronize(e->stream));
    if (sweep) *sweep = e->sweep;
    return CSG_OK;
}

int csg_run(csg_engine* e, int64_t n_sweeps) {
    if (!e) return fail(CSG_ERR_ARG, "null engine");
    if (n_sweeps < 0) return fail(CSG_ERR_ARG, "negative sweep count");
    if (n_sweeps == 0) return CSG_OK;
    const csg_device_obs o = device_obs(e);
    if (int rc = run_device(e->cfg, e->spins, e->bonds, &o, e->sweep, n_sweeps, e->stream,
                            PlanChoice{e->qc, e->nseg}))
        return rc;
    account(e, n_sweeps);
    return CSG_OK;
}

int csg_reset_observables(csg_engine* e) {
    if (!e) return fail(CSG_ERR_ARG, "null engine");
    return reset_obs(e);
}

int csg_get_observables(csg_engine* e, csg_observables* out) {
    if (!e || !out) return fail(CSG_ERR_ARG, "null argument");
    struct C {
        void* dst;
        const void* src;
        size_t bytes;
    } cp[] = {{out->e_sum, e->e_sum, e->n_e * 8},   {out->m_sum, e->m_sum, e->n_e * 8},
              {out->q_sum, e->q_sum, e->n_q * 8},   {out->q2_sum, e->q2_sum, e->n_q * 8},
              {out->q4_sum, e->q4_sum, e->n_q * 16}, {out->hist, e->hist, e->n_hist * 4},
              {out->e_last, e->e_last, e->n_e * 4}, {out->m_last, e->m_last, e->n_e * 4},
              {out->d_last, e->d_last, e->n_q * 4},
              {out->swap_acc, e->swap_acc, (size_t)e->cfg.dims.n_copies * e->cfg.dims.n_temps * 8}};
    for (auto& c : cp)
        if (c.dst && c.src && c.bytes)
            CSG_CUDA(cudaMemcpyAsync(c.dst, c.src, c.bytes, cudaMemcpyDeviceToHost, e->stream));
    if (out->swap_log && e->swap_log) {
        const int64_t rows = std::min<int64_t>(out->swap_log_rounds, e->cfg.swap_log_rounds);
        if (rows > 0)
            CSG_CUDA(cudaMemcpyAsync(out->swap_log, e->swap_log, (size_t)rows * e->n_e / 32 * 4,
                                     cudaMemcpyDeviceToHost, e->stream));
    }
    uint64_t b = 0;
    CSG_CUDA(cudaMemcpyAsync(&b, e->boundary, 8, cudaMemcpyDeviceToHost, e->stream));
    CSG_CUDA(cudaStreamSynchronize(e->stream));
    if (out->q4_sum)  // device split {sum of low 32 bits, sum of the rest} -> 128-bit
        for (size_t i = 0; i < e->n_q; ++i) {
            const uint64_t low = out->q4_sum[2 * i], high = out->q4_sum[2 * i + 1];
            const uint64_t shifted = high << 32;  // total = high * 2^32 + low
            const uint64_t lo = shifted + low;
            out->q4_sum[2 * i] = lo;
            out->q4_sum[2 * i + 1] = (high >> 32) + (lo < shifted ? 1u : 0u);
        }
    out->boundary = b;
    out->n_meas = e->n_meas;
    out->swap_rounds = e->swap_rounds;
    return CSG_OK;
}

int csg_pt_run_device(const csg_config* cfg, uint32_t* spins, const uint32_t* bonds,
                      const csg_device_obs* obs, int64_t sweep0, int64_t n_sweeps, void* stream) {
    if (int rc = validate(cfg)) return rc;
    if (!spins || !bonds) return fail(CSG_ERR_ARG, "null device buffer");
    if (sweep0 < 0 || n_sweeps < 0) return fail(CSG_ERR_ARG, "negative sweep index or count");
    if (n_sweeps == 0) return CSG_OK;
    return run_device(*cfg, spins, bonds, obs, sweep0, n_sweeps, (cudaStream_t)stream);
}

int csg_query_plan(const csg_config* cfg, csg_plan* out) {
    if (int rc = validate(cfg)) return rc;
    if (!out) return fail(CSG_ERR_ARG, "null output");
    csg::PtParams P;
    bool gen = false;
    fill_params(*cfg, P, gen);
    Plan pl;
    if (int rc = make_plan(*cfg, gen, pl)) return rc;
    out->quads_per_cta = pl.Qc;
    out->ctas_per_word = pl.K;
    out->threads_per_quad = pl.TPQ;
    out->smem_bytes = (int32_t)pl.smem;
    return CSG_OK;
}

int csg_set_plan_override(const csg_plan* plan) {
    std::lock_guard<std::mutex> lk(g_plan_mu);
    if (!plan) {
        g_override = csg_plan{0, 0, 0, 0};
        return CSG_OK;
    }
    if (plan->quads_per_cta < 0) return fail(CSG_ERR_ARG, "negative quads_per_cta");
    g_override = *plan;
    return CSG_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Reference-format outputs: observable records and checkpoints
// ---------------------------------------------------------------------------
namespace {

size_t slot_of(int L, int x, int y, int z) {
    const size_t N = (size_t)L * L * L;
    return (size_t)((x + y + z) & 1) * (N / 2) + (size_t)(z * L + y) * (L / 2) + (size_t)(x >> 1);
}

size_t spin_at(const csg_dims& d, int w, int c, int t, size_t slot) {
    const size_t N = (size_t)d.L * d.L * d.L;
    return ((((size_t)w * d.n_copies + c) * (d.n_temps / 4) + (size_t)(t >> 2)) * N + slot) * 4 +
           (size_t)(t & 3);
}

}  // namespace

extern "C" {

// Records follow eamsim.cu:320-325 (e = -(2S-3N + H M)/N, m = M/N, float
// arithmetic as in the reference) and eamsim.cu:477-509 (q_0 = sum s1 s2 / N,
// q_1 = sum s1 s2 exp(i k x) / N with k = 2 pi / L), the latter formed from
// exact per-plane integer sums combined in double precision.
int csg_obs_records(csg_engine* e, float* rec, size_t n_floats) {
    if (!e || !rec) return fail(CSG_ERR_ARG, "null argument");
    const csg_dims& d = e->cfg.dims;
    if (d.n_copies != 2) return fail(CSG_ERR_UNSUPPORTED, "observable records need two copies");
    const int L = d.L, W = d.n_words, T = d.n_temps;
    const size_t need = (size_t)32 * W * T * 11;
    if (n_floats != need) return fail(CSG_ERR_ARG, "record buffer size mismatch");
    const size_t nE = (size_t)W * 2 * T * 32, nD = (size_t)W * T * 32, nP = nD * 3 * L;
    // scratch: integers, the phase tables, the records
    const size_t o_m = nE * 4, o_d = o_m + nE * 4, o_p = o_d + nD * 4, o_cs = (o_p + nP * 4 + 15) & ~(size_t)15;
    const size_t o_rec = o_cs + (size_t)2 * L * 8, bytes = o_rec + need * 4;
    if (!e->rec_scratch)
        if (int rc = engine_alloc(e, reinterpret_cast<void**>(&e->rec_scratch), bytes)) return rc;
    char* sc = e->rec_scratch;
    int* de = reinterpret_cast<int*>(sc);
    int* dm = reinterpret_cast<int*>(sc + o_m);
    int* dd = reinterpret_cast<int*>(sc + o_d);
    int* dp = reinterpret_cast<int*>(sc + o_p);
    double* dcs = reinterpret_cast<double*>(sc + o_cs);
    float* drec = reinterpret_cast<float*>(sc + o_rec);
    // the L phases exp(i k a), k = 2 pi / L, computed on the host
    const double k = 2.0 * M_PI / L;
    std::vector<double> cs(2 * (size_t)L);
    for (int a = 0; a < L; ++a) {
        cs[a] = std::cos(k * a);
        cs[L + a] = std::sin(k * a);
    }
    // 3L counters per lane; as many warps as fit in 48 KB (4 up to L = 32)
    const size_t per_warp = (size_t)32 * 3 * L * sizeof(int);
    const int warps = (int)std::max<size_t>(1, std::min<size_t>(4, 49152 / per_warp));
    const unsigned blocks = (unsigned)((W * T + warps - 1) / warps);
    const size_t sh = (size_t)warps * per_warp;
    cudaError_t ce = cudaMemcpyAsync(dcs, cs.data(), cs.size() * 8, cudaMemcpyHostToDevice, e->stream);
    if (ce == cudaSuccess) {
        csg::measure_kernel<<<blocks, warps * 32, sh, e->stream>>>(e->spins, e->bonds, L, W, T, de, dm,
                                                                   dd, dp);
        const long total = (long)W * 32 * T;
        csg::records_kernel<<<(unsigned)((total + 127) / 128), 128, 0, e->stream>>>(
            de, dm, dd, dp, dcs, dcs + L, L, W, T, (float)e->cfg.H, drec);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(rec, drec, need * 4, cudaMemcpyDeviceToHost, e->stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(e->stream);
    if (ce != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("records: ") + cudaGetErrorString(ce));
    return CSG_OK;
}

// Reference checkpoint (eamsim.cu:655-676): uint32 [2*32W][N], lattice
// 2*sample+copy, site (z*L+y)*L+x; bits 0..T-1 spins by temperature, bits
// 26..31 bonds -x,+x,-y,+y,-z,+z with bit 1 = ferromagnetic (eamsim.cu:598-616).
int csg_save_checkpoint(csg_engine* e, uint32_t* ref, size_t n_words) {
    if (!e || !ref) return fail(CSG_ERR_ARG, "null argument");
    const csg_dims& d = e->cfg.dims;
    if (d.n_copies != 2 || d.n_temps > 24)
        return fail(CSG_ERR_UNSUPPORTED, "checkpoint layout needs 2 copies and <= 24 temperatures");
    const int L = d.L, W = d.n_words, T = d.n_temps;
    const size_t N = (size_t)L * L * L;
    if (n_words != (size_t)64 * W * N) return fail(CSG_ERR_ARG, "checkpoint size mismatch");
    std::vector<uint32_t> sp(e->n_spins), bd(e->n_bonds);
    if (int rc = csg_get_state(e, sp.data(), sp.size(), bd.data(), bd.size(), nullptr)) return rc;
    for (int w = 0; w < W; ++w)
        for (int z = 0; z < L; ++z)
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const size_t si = slot_of(L, x, y, z), i = ((size_t)z * L + y) * L + x;
                    const int xm = (x + L - 1) % L, ym = (y + L - 1) % L, zm = (z + L - 1) % L;
                    const uint32_t f[6] = {bd[((size_t)w * 3 + 0) * N + slot_of(L, xm, y, z)],
                                           bd[((size_t)w * 3 + 0) * N + si],
                                           bd[((size_t)w * 3 + 1) * N + slot_of(L, x, ym, z)],
                                           bd[((size_t)w * 3 + 1) * N + si],
                                           bd[((size_t)w * 3 + 2) * N + slot_of(L, x, y, zm)],
                                           bd[((size_t)w * 3 + 2) * N + si]};
                    uint32_t sv[2][24];
                    for (int c = 0; c < 2; ++c)
                        for (int t = 0; t < T; ++t) sv[c][t] = sp[spin_at(d, w, c, t, si)];
                    for (int b = 0; b < 32; ++b) {
                        uint32_t jb = 0;
                        for (int k = 0; k < 6; ++k) jb |= ((~f[k] >> b) & 1u) << (26 + k);
                        for (int c = 0; c < 2; ++c) {
                            uint32_t v = jb;
                            for (int t = 0; t < T; ++t) v |= ((sv[c][t] >> b) & 1u) << t;
                            ref[((size_t)2 * (32 * w + b) + c) * N + i] = v;
                        }
                    }
                }
    return CSG_OK;
}

int csg_load_checkpoint(csg_engine* e, const uint32_t* ref, size_t n_words, int64_t sweep) {
    if (!e || !ref) return fail(CSG_ERR_ARG, "null argument");
    const csg_dims& d = e->cfg.dims;
    if (d.n_copies != 2 || d.n_temps > 24)
        return fail(CSG_ERR_UNSUPPORTED, "checkpoint layout needs 2 copies and <= 24 temperatures");
    const int L = d.L, W = d.n_words, T = d.n_temps;
    const size_t N = (size_t)L * L * L;
    if (n_words != (size_t)64 * W * N) return fail(CSG_ERR_ARG, "checkpoint size mismatch");
    std::vector<uint32_t> sp(e->n_spins, 0u), bd(e->n_bonds, 0u);
    for (int w = 0; w < W; ++w)
        for (int z = 0; z < L; ++z)
            for (int y = 0; y < L; ++y)
                for (int x = 0; x < L; ++x) {
                    const size_t si = slot_of(L, x, y, z), i = ((size_t)z * L + y) * L + x;
                    const size_t nbi[3] = {((size_t)z * L + y) * L + (x + 1) % L,
                                           ((size_t)z * L + (y + 1) % L) * L + x,
                                           ((size_t)((z + 1) % L) * L + y) * L + x};
                    uint32_t f[3] = {0, 0, 0};
                    uint32_t sv[2][24] = {};
                    for (int b = 0; b < 32; ++b) {
                        const uint32_t v0 = ref[((size_t)2 * (32 * w + b)) * N + i];
                        const uint32_t v1 = ref[((size_t)2 * (32 * w + b) + 1) * N + i];
                        if ((v0 >> 26) != (v1 >> 26))
                            return fail(CSG_ERR_STATE, "copies of a sample disagree on its bonds");
                        for (int k = 0; k < 3; ++k) {
                            const uint32_t vn = ref[((size_t)2 * (32 * w + b)) * N + nbi[k]];
                            if (((v0 >> (27 + 2 * k)) & 1u) != ((vn >> (26 + 2 * k)) & 1u))
                                return fail(CSG_ERR_STATE, "the two ends of a bond disagree");
                            f[k] |= ((~v0 >> (27 + 2 * k)) & 1u) << b;
                        }
                        for (int t = 0; t < T; ++t) {
                            sv[0][t] |= ((v0 >> t) & 1u) << b;
                            sv[1][t] |= ((v1 >> t) & 1u) << b;
                        }
                    }
                    for (int k = 0; k < 3; ++k) bd[((size_t)w * 3 + k) * N + si] = f[k];
                    for (int c = 0; c < 2; ++c)
                        for (int t = 0; t < T; ++t) sp[spin_at(d, w, c, t, si)] = sv[c][t];
                }
    return csg_set_state(e, sp.data(), sp.size(), bd.data(), bd.size(), sweep);
}

}  // extern "C"

