// batch.cpp — the batched engine: several simulations (any mix of L, samples,
// ladders) run as parallel branches of one captured CUDA graph, so that their
// clusters share the SMs that any single one leaves idle.  Each member keeps
// its own Philox counters, so its results do not depend on the batch it runs
// in.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "csg.h"
#include "engine_internal.h"

using namespace csg_detail;

struct csg_batch {
    std::vector<csg_engine*> eng;
    cudaStream_t main = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    // ordering of launches on a caller's stream against the members' streams
    std::vector<cudaEvent_t> ready;
    cudaEvent_t done = nullptr;
    long long* counters = nullptr;  // device sweep counter per member
    std::vector<std::pair<int64_t, cudaGraphExec_t>> graphs;
    // per member: pad its CTAs' shared memory past half an SM, so that none
    // of them shares an SM (chosen by the tuner)
    std::vector<char> spread;
};

namespace {

void drop_graphs(csg_batch* b) {
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.second);
    b->graphs.clear();
}

// more than half of an SM's 228 KB (with the 1 KB per-CTA reserve)
constexpr size_t kSpreadSmem = 116 * 1024;

int capture(csg_batch* b, int64_t n_sweeps, bool with_obs, cudaGraphExec_t* out) {
    std::vector<Plan> plans(b->eng.size());
    for (size_t i = 0; i < b->eng.size(); ++i)
        if (int rc = plan_engine(b->eng[i], plans[i], b->spread[i] ? kSpreadSmem : 0)) return rc;
    // Branches in order of decreasing cluster size (then shared memory per CTA):
    // the GPU places the clusters of the first branches first, and putting the
    // largest first packs the GPCs best (best-fit decreasing).  On the mixed
    // L=12/14/16 workload this order measured up to 36 % faster than member
    // order.
    std::vector<size_t> order(b->eng.size());
    for (size_t i = 0; i < order.size(); ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        if (plans[x].K != plans[y].K) return plans[x].K > plans[y].K;
        return plans[x].smem > plans[y].smem;
    });
    CSG_CUDA(cudaStreamBeginCapture(b->main, cudaStreamCaptureModeThreadLocal));
    int rc = CSG_OK;
    cudaError_t ce = cudaEventRecord(b->fork, b->main);
    for (size_t oi = 0; oi < order.size() && rc == CSG_OK && ce == cudaSuccess; ++oi) {
        const size_t i = order[oi];
        csg_engine* e = b->eng[i];
        ce = cudaStreamWaitEvent(e->stream, b->fork, 0);
        if (ce != cudaSuccess) break;
        const csg_device_obs o = device_obs(e);
        rc = run_device(e->cfg, e->spins, e->bonds, with_obs ? &o : nullptr, 0, n_sweeps, e->stream,
                        PlanChoice{}, b->counters + i, &plans[i]);
        if (rc == CSG_OK) ce = cudaEventRecord(b->join[i], e->stream);
        if (ce == cudaSuccess) ce = cudaStreamWaitEvent(b->main, b->join[i], 0);
    }
    cudaGraph_t g = nullptr;
    const cudaError_t ce2 = cudaStreamEndCapture(b->main, &g);
    if (rc != CSG_OK) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess || ce2 != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return fail(CSG_ERR_CUDA, std::string("graph capture: ") +
                                      cudaGetErrorString(ce != cudaSuccess ? ce : ce2));
    }
    // the capture order (largest clusters first) becomes the placement order
    // even when the graph's launch waits on other streams and every branch
    // becomes ready at once
    std::vector<const csg_engine*> starts;
    std::vector<int> nsegs;
    for (size_t i : order) {
        starts.push_back(b->eng[i]);
        nsegs.push_back(plans[i].NSEG);
    }
    if (int rc2 = chain_launch_starts(g, starts, nsegs)) {
        cudaGraphDestroy(g);
        return rc2;
    }
    const cudaError_t ce3 = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ce3 != cudaSuccess)
        return fail(CSG_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(ce3));
    return CSG_OK;
}

// Queue n sweeps of every member on stream st: after the work already queued
// on the members' own streams, and before anything queued on them later.
// plain = false: one launch of the batch graph (captured on first use for this
// n_sweeps and replayed afterwards) from the members' host sweep counters;
// plain = true: the plain engine, member after member, each with its own
// automatic plan.  The members' host counters advance at once.
int launch_batch(csg_batch* b, int64_t n_sweeps, bool plain, cudaStream_t st) {
    for (size_t i = 0; i < b->eng.size(); ++i) {
        CSG_CUDA(cudaEventRecord(b->ready[i], b->eng[i]->stream));
        CSG_CUDA(cudaStreamWaitEvent(st, b->ready[i], 0));
    }
    if (plain) {
        for (csg_engine* e : b->eng) {
            const csg_device_obs o = device_obs(e);
            if (int rc = run_device(e->cfg, e->spins, e->bonds, &o, e->sweep, n_sweeps, st)) return rc;
        }
    } else {
        cudaGraphExec_t exec = nullptr;
        for (auto& g : b->graphs)
            if (g.first == n_sweeps) exec = g.second;
        if (!exec) {
            if (int rc = capture(b, n_sweeps, true, &exec)) return rc;
            b->graphs.push_back({n_sweeps, exec});
        }
        std::vector<long long> start(b->eng.size());
        for (size_t i = 0; i < b->eng.size(); ++i) start[i] = b->eng[i]->sweep;
        // pageable source: staged before the call returns
        CSG_CUDA(cudaMemcpyAsync(b->counters, start.data(), start.size() * sizeof(long long),
                                 cudaMemcpyHostToDevice, st));
        CSG_CUDA(cudaGraphLaunch(exec, st));
    }
    CSG_CUDA(cudaEventRecord(b->done, st));
    for (csg_engine* e : b->eng) CSG_CUDA(cudaStreamWaitEvent(e->stream, b->done, 0));
    for (csg_engine* e : b->eng) account(e, n_sweeps);
    return CSG_OK;
}

}  // namespace

extern "C" {

int csg_batch_create(const csg_config* cfgs, int32_t n, csg_batch** out) {
    if (!out || !cfgs || n < 1) return fail(CSG_ERR_ARG, "bad batch arguments");
    *out = nullptr;
    csg_batch* b = new (std::nothrow) csg_batch();
    if (!b) return fail(CSG_ERR_NOMEM, "host allocation failed");
    int rc = CSG_OK;
    for (int i = 0; i < n && rc == CSG_OK; ++i) {
        csg_engine* e = nullptr;
        rc = csg_engine_create(&cfgs[i], &e);
        if (rc == CSG_OK && use_stream(cfgs[i])) {
            csg_engine_destroy(e);
            rc = fail(CSG_ERR_UNSUPPORTED,
                      "batch members need the cluster-resident kernel (L <= 24, no CSG_ENGINE_STREAM)");
        }
        if (rc == CSG_OK) {
            b->eng.push_back(e);
            b->spread.push_back(0);
        }
    }
    if (rc == CSG_OK && cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking) != cudaSuccess)
        rc = fail(CSG_ERR_CUDA, "cudaStreamCreate failed");
    if (rc == CSG_OK && cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(CSG_ERR_CUDA, "cudaEventCreate failed");
    for (int i = 0; i < n && rc == CSG_OK; ++i) {
        cudaEvent_t ev, ev2;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess)
            rc = fail(CSG_ERR_CUDA, "cudaEventCreate failed");
        else
            b->join.push_back(ev);
        if (rc == CSG_OK) {
            if (cudaEventCreateWithFlags(&ev2, cudaEventDisableTiming) != cudaSuccess)
                rc = fail(CSG_ERR_CUDA, "cudaEventCreate failed");
            else
                b->ready.push_back(ev2);
        }
    }
    if (rc == CSG_OK && cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming) != cudaSuccess)
        rc = fail(CSG_ERR_CUDA, "cudaEventCreate failed");
    if (rc == CSG_OK) rc = dalloc(&b->counters, (size_t)n);
    if (rc != CSG_OK) {
        const std::string msg = last_error();
        csg_batch_destroy(b);
        set_last_error(msg);
        return rc;
    }
    *out = b;
    return CSG_OK;
}

int csg_batch_destroy(csg_batch* b) {
    if (!b) return CSG_OK;
    if (b->main) cudaStreamSynchronize(b->main);
    // a launch on a caller's stream is waited for through the members' streams,
    // which csg_engine_destroy synchronises
    for (csg_engine* e : b->eng) csg_engine_destroy(e);
    drop_graphs(b);
    for (cudaEvent_t ev : b->join) cudaEventDestroy(ev);
    for (cudaEvent_t ev : b->ready) cudaEventDestroy(ev);
    if (b->done) cudaEventDestroy(b->done);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->main) cudaStreamDestroy(b->main);
    if (b->counters) cudaFree(b->counters);
    delete b;
    return CSG_OK;
}

int csg_batch_engine(csg_batch* b, int32_t i, csg_engine** out) {
    if (!b || !out || i < 0 || i >= (int32_t)b->eng.size()) return fail(CSG_ERR_ARG, "bad member index");
    *out = b->eng[i];
    return CSG_OK;
}

int csg_batch_run(csg_batch* b, int64_t n_sweeps) {
    if (!b || n_sweeps < 0) return fail(CSG_ERR_ARG, "bad batch run arguments");
    if (n_sweeps == 0) return CSG_OK;
    if (int rc = launch_batch(b, n_sweeps, false, b->main)) return rc;
    CSG_CUDA(cudaStreamSynchronize(b->main));
    return CSG_OK;
}

int csg_batch_run_sequential(csg_batch* b, int64_t n_sweeps) {
    if (!b || n_sweeps < 0) return fail(CSG_ERR_ARG, "bad batch run arguments");
    if (n_sweeps == 0) return CSG_OK;
    if (int rc = launch_batch(b, n_sweeps, true, b->main)) return rc;
    CSG_CUDA(cudaStreamSynchronize(b->main));
    return CSG_OK;
}

int csg_batch_launch(csg_batch* b, int64_t n_sweeps, int32_t plain, void* stream) {
    if (!b || n_sweeps < 0 || (plain != 0 && plain != 1))
        return fail(CSG_ERR_ARG, "bad batch launch arguments");
    if (n_sweeps == 0) return CSG_OK;
    return launch_batch(b, n_sweeps, plain != 0, (cudaStream_t)stream);
}

int csg_batch_set_plan(csg_batch* b, const int32_t* quads_per_cta) {
    if (!b || !quads_per_cta) return fail(CSG_ERR_ARG, "null argument");
    for (size_t i = 0; i < b->eng.size(); ++i) {
        const csg_dims& d = b->eng[i]->cfg.dims;
        const int G = d.n_copies * d.n_temps / 4;
        if (quads_per_cta[i] < 0 || (quads_per_cta[i] > 0 && G % quads_per_cta[i]))
            return fail(CSG_ERR_ARG, "quads_per_cta must divide n_copies*n_temps/4");
    }
    for (size_t i = 0; i < b->eng.size(); ++i) {
        b->eng[i]->qc = quads_per_cta[i];
        b->eng[i]->nseg = 0;
    }
    drop_graphs(b);
    return CSG_OK;
}

int csg_batch_set_member_plan(csg_batch* b, int32_t i, const csg_plan* plan) {
    if (!b || !plan || i < 0 || i >= (int32_t)b->eng.size()) return fail(CSG_ERR_ARG, "bad member index");
    csg_engine* e = b->eng[i];
    const int qc = plan->quads_per_cta, tpq = plan->threads_per_quad;
    if (qc < 0 || tpq < 0) return fail(CSG_ERR_ARG, "negative plan entry");
    const int L = e->cfg.dims.L;
    const int nseg = tpq > 0 ? tpq / (L * (L / 2)) : 0;
    if (tpq > 0 && nseg * L * (L / 2) != tpq) return fail(CSG_ERR_ARG, "threads_per_quad is not L*L/2*s");
    bool ok = qc == 0 && nseg == 0;
    for (const PlanChoice& o : plan_options(e->cfg))
        if ((qc == 0 || o.qc == qc) && (nseg == 0 || o.nseg == nseg)) ok = true;
    if (!ok) return fail(CSG_ERR_UNSUPPORTED, "no built tile with these quads per CTA and threads per quad");
    e->qc = qc;
    e->nseg = nseg;
    drop_graphs(b);
    return CSG_OK;
}

int csg_batch_member_plan(csg_batch* b, int32_t i, csg_plan* out) {
    if (!b || !out || i < 0 || i >= (int32_t)b->eng.size()) return fail(CSG_ERR_ARG, "bad member index");
    Plan pl;
    if (int rc = plan_engine(b->eng[i], pl, b->spread[i] ? kSpreadSmem : 0)) return rc;
    out->quads_per_cta = pl.Qc;
    out->ctas_per_word = pl.K;
    out->threads_per_quad = pl.TPQ;
    out->smem_bytes = (int32_t)pl.smem;
    return CSG_OK;
}

// Autotuner: times the whole batch graph for probe_sweeps sweeps (best of two)
// for every combination of the members' tiles (quads per CTA, threads per
// quad), each member with and without an SM per CTA, when there are at most
// 1024 such combinations; otherwise coordinate descent over one member at a
// time with the others fixed (two passes).  The members' spins are saved before and restored
// after, and the probes accumulate no observables, so tuning leaves the
// simulations exactly as they were.
int csg_batch_tune(csg_batch* b, int64_t probe_sweeps, int32_t* chosen) {
    if (!b || probe_sweeps < 1) return fail(CSG_ERR_ARG, "bad tune arguments");
    const size_t n = b->eng.size();
    std::vector<uint32_t*> saved(n, nullptr);
    int rc = CSG_OK;
    for (size_t i = 0; i < n && rc == CSG_OK; ++i) {
        rc = dalloc(&saved[i], b->eng[i]->n_spins);
        if (rc == CSG_OK)
            if (cudaMemcpyAsync(saved[i], b->eng[i]->spins, b->eng[i]->n_spins * 4,
                                cudaMemcpyDeviceToDevice, b->eng[i]->stream) != cudaSuccess)
                rc = fail(CSG_ERR_CUDA, "snapshot copy failed");
    }
    // the probes run on the batch's own stream: the snapshots must be complete
    for (size_t i = 0; i < n && rc == CSG_OK; ++i)
        if (cudaStreamSynchronize(b->eng[i]->stream) != cudaSuccess)
            rc = fail(CSG_ERR_CUDA, "snapshot copy failed");
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    if (rc == CSG_OK && (cudaEventCreate(&t0) != cudaSuccess || cudaEventCreate(&t1) != cudaSuccess))
        rc = fail(CSG_ERR_CUDA, "cudaEventCreate failed");
    auto time_batch = [&](float& ms_out) -> int {
        cudaGraphExec_t exec = nullptr;
        if (int r = capture(b, probe_sweeps, false, &exec)) return r;
        float best = 1e30f;
        for (int rep = 0; rep < 3; ++rep) {  // first launch warms up
            std::vector<long long> start(n, 0);
            CSG_CUDA(cudaMemcpyAsync(b->counters, start.data(), n * sizeof(long long),
                                     cudaMemcpyHostToDevice, b->main));
            CSG_CUDA(cudaEventRecord(t0, b->main));
            CSG_CUDA(cudaGraphLaunch(exec, b->main));
            CSG_CUDA(cudaEventRecord(t1, b->main));
            CSG_CUDA(cudaEventSynchronize(t1));
            float ms = 0.f;
            CSG_CUDA(cudaEventElapsedTime(&ms, t0, t1));
            if (rep > 0 && ms < best) best = ms;
        }
        cudaGraphExecDestroy(exec);
        ms_out = best;
        return CSG_OK;
    };
    for (size_t i = 0; i < n && rc == CSG_OK; ++i) {
        Plan pl;
        rc = plan_engine(b->eng[i], pl);  // start from the per-member plan
        if (rc == CSG_OK) {
            b->eng[i]->qc = pl.Qc;
            b->eng[i]->nseg = pl.NSEG;
        }
    }
    // the (quads per CTA, column segments per thread) plans each member can take
    std::vector<std::vector<PlanChoice>> options(n);
    size_t combos = 1;
    for (size_t i = 0; i < n; ++i) {
        options[i] = plan_options(b->eng[i]->cfg);
        combos *= std::max<size_t>(1, options[i].size());
    }
    auto set_choice = [&](size_t i, const PlanChoice& pc) {
        b->eng[i]->qc = pc.qc;
        b->eng[i]->nseg = pc.nseg;
    };
    auto choice_of = [&](size_t i) { return PlanChoice{b->eng[i]->qc, b->eng[i]->nseg}; };
    // every (plan, spread) combination of every member when there are at most
    // kMaxProbes of them: members share the GPU, so the best plan of one
    // member depends on the others'
    constexpr size_t kMaxProbes = 1024;
    const size_t masks = n < 16 ? (size_t)1 << n : kMaxProbes + 1;
    if (combos * masks <= kMaxProbes) {
        float best_ms = 1e30f;
        std::vector<PlanChoice> best(n);
        std::vector<char> best_spread(b->spread);
        for (size_t i = 0; i < n; ++i) best[i] = choice_of(i);
        for (size_t k = 0; k < combos * masks && rc == CSG_OK; ++k) {
            const size_t mask = k / combos;
            size_t r = k % combos;
            for (size_t i = 0; i < n; ++i) {
                const size_t m = options[i].size();
                if (m) set_choice(i, options[i][r % m]);
                r /= std::max<size_t>(1, m);
                b->spread[i] = (char)((mask >> i) & 1);
            }
            float ms = 0.f;
            if (time_batch(ms) != CSG_OK) {  // e.g. a cluster shape the device cannot place
                cudaGetLastError();
                continue;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best_spread = b->spread;
                for (size_t i = 0; i < n; ++i) best[i] = choice_of(i);
            }
        }
        for (size_t i = 0; i < n; ++i) set_choice(i, best[i]);
        b->spread = best_spread;
    }
    // otherwise coordinate descent: each member's (plan, spread) in turn with
    // the others fixed, two passes
    for (int pass = 0; pass < 2 && rc == CSG_OK && combos * masks > kMaxProbes; ++pass)
        for (size_t i = 0; i < n && rc == CSG_OK; ++i) {
            PlanChoice best_pc = choice_of(i);
            char best_sp = b->spread[i];
            float best_ms = 1e30f;
            for (const PlanChoice& pc : options[i])
                for (char sp = 0; sp < 2; ++sp) {
                    set_choice(i, pc);
                    b->spread[i] = sp;
                    float ms = 0.f;
                    const int r = time_batch(ms);
                    if (r != CSG_OK) {  // e.g. a cluster shape the device cannot place
                        cudaGetLastError();
                        continue;
                    }
                    if (ms < best_ms) {
                        best_ms = ms;
                        best_pc = pc;
                        best_sp = sp;
                    }
                }
            set_choice(i, best_pc);
            b->spread[i] = best_sp;
        }
    for (size_t i = 0; i < n; ++i) {
        if (saved[i]) {
            if (rc == CSG_OK &&
                cudaMemcpy(b->eng[i]->spins, saved[i], b->eng[i]->n_spins * 4,
                           cudaMemcpyDeviceToDevice) != cudaSuccess)
                rc = fail(CSG_ERR_CUDA, "restore copy failed");
            cudaFree(saved[i]);
        }
        if (chosen) chosen[i] = b->eng[i]->qc;
    }
    if (t0) cudaEventDestroy(t0);
    if (t1) cudaEventDestroy(t1);
    drop_graphs(b);
    return rc;
}

}  // extern "C"
