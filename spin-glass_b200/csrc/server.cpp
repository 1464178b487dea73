// server.cpp — serving: continuous batching of simulation requests.  Requests
// queue FIFO, are admitted while a device-memory budget and a slot count
// allow, and run as plain engines on their own streams in sections of a fixed
// number of sweeps, so that new requests join between sections.
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <string>
#include <utility>
#include <vector>

#include "csg.h"
#include "engine_internal.h"

using namespace csg_detail;

namespace {

// Plan for a request that shares the GPU with others: the largest split of
// quads that fits one CTA with the default column split (fewest CTAs and
// cluster barriers per unit of work); automatic (the single-request plan) for
// the streaming engine.
PlanChoice shared_gpu_plan(const csg_config& c) {
    const std::vector<PlanChoice> opts = plan_options(c);
    PlanChoice best{};
    for (const PlanChoice& o : opts)
        if (o.nseg == opts.front().nseg && o.qc > best.qc) best = o;
    return best;
}

}  // namespace

struct csg_server {
    struct Req {
        int64_t id;
        csg_config cfg;
        std::vector<double> betas;
        int64_t total = 0, launched = 0;
        size_t bytes = 0;
        csg_engine* e = nullptr;
        bool done = false;
        // a request whose engine could not be created or launched completes
        // with this error, which csg_server_result returns
        int status = CSG_OK;
        std::string error;
    };
    size_t budget = 0, in_use = 0;
    int max_active = 0;
    int64_t chunk = 1024, next_id = 1;
    std::vector<Req> queue;   // waiting, FIFO
    std::vector<Req> active;  // admitted (running or finished, result not fetched)
};

extern "C" {

int csg_server_create(size_t memory_budget_bytes, int32_t max_active, int32_t sweeps_per_launch,
                      csg_server** out) {
    if (!out || memory_budget_bytes == 0 || max_active < 1 || sweeps_per_launch < 1)
        return fail(CSG_ERR_ARG, "bad server arguments");
    csg_server* s = new (std::nothrow) csg_server();
    if (!s) return fail(CSG_ERR_NOMEM, "host allocation failed");
    s->budget = memory_budget_bytes;
    s->max_active = max_active;
    s->chunk = sweeps_per_launch;
    *out = s;
    return CSG_OK;
}

int csg_server_destroy(csg_server* s) {
    if (!s) return CSG_OK;
    for (auto& r : s->active)
        if (r.e) csg_engine_destroy(r.e);
    delete s;
    return CSG_OK;
}

int csg_server_submit(csg_server* s, const csg_config* cfg, int64_t n_sweeps, int64_t* id) {
    if (!s || !id || n_sweeps < 1) return fail(CSG_ERR_ARG, "bad request");
    if (int rc = validate(cfg)) return rc;
    csg_server::Req r;
    r.id = s->next_id++;
    r.cfg = *cfg;
    r.betas.assign(cfg->betas, cfg->betas + cfg->dims.n_temps);
    r.total = n_sweeps;
    r.bytes = footprint_bytes(*cfg);
    if (r.bytes > s->budget) return fail(CSG_ERR_NOMEM, "request larger than the memory budget");
    s->queue.push_back(std::move(r));
    s->queue.back().cfg.betas = s->queue.back().betas.data();
    *id = s->queue.back().id;
    return CSG_OK;
}

// One non-blocking scheduling pass: completes requests whose device work has
// drained, admits waiting requests (FIFO, while the budget and the active-slot
// count allow), and launches the next section of every request whose stream
// is idle.  Completed ids are reported once.
int csg_server_poll(csg_server* s, int64_t* completed, int32_t max_completed,
                    int32_t* n_completed, int32_t* n_active, int32_t* n_queued) {
    if (!s) return fail(CSG_ERR_ARG, "null server");
    int32_t nc = 0;
    auto report = [&](csg_server::Req& r) {
        r.done = true;
        if (completed && nc < max_completed) completed[nc] = r.id;
        ++nc;
    };
    // a failed request gives its memory back at once; its id is reported done
    auto failed = [&](csg_server::Req& r, int rc) {
        r.status = rc;
        r.error = last_error();
        if (r.e) {
            csg_engine_destroy(r.e);
            r.e = nullptr;
            s->in_use -= r.bytes;
        }
        report(r);
    };
    for (auto& r : s->active) {
        if (r.done) continue;
        const cudaError_t q = cudaStreamQuery(r.e->stream);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("request stream: ") + cudaGetErrorString(q));
        if (r.launched >= r.total) report(r);
    }
    while (!s->queue.empty() && (int)s->active.size() < s->max_active &&
           s->in_use + s->queue.front().bytes <= s->budget) {
        s->active.push_back(std::move(s->queue.front()));
        s->queue.erase(s->queue.begin());
        csg_server::Req& r = s->active.back();
        r.cfg.betas = r.betas.data();
        int rc = csg_engine_create(&r.cfg, &r.e);
        if (rc == CSG_OK) {
            s->in_use += r.bytes;
            rc = csg_init_lattice(r.e);
        }
        if (rc != CSG_OK) failed(r, rc);
    }
    int running = 0;
    for (auto& r : s->active) running += (!r.done && r.launched < r.total) ? 1 : 0;
    for (auto& r : s->active) {
        if (r.done || r.launched >= r.total) continue;
        if (cudaStreamQuery(r.e->stream) != cudaSuccess) continue;
        const int64_t n = std::min<int64_t>(s->chunk, r.total - r.launched);
        // alone, a request takes the plan that spreads it widest; sharing the
        // GPU, the one with the fewest CTAs (every plan gives the same bits)
        const PlanChoice pc = running > 1 ? shared_gpu_plan(r.cfg) : PlanChoice{};
        r.e->qc = pc.qc;
        r.e->nseg = pc.nseg;
        if (int rc = csg_run(r.e, n)) {
            failed(r, rc);
            continue;
        }
        r.launched += n;
    }
    if (n_completed) *n_completed = nc;
    int32_t na = 0;
    for (auto& r : s->active) na += r.done ? 0 : 1;
    if (n_active) *n_active = na;
    if (n_queued) *n_queued = (int32_t)s->queue.size();
    return CSG_OK;
}

// Results of a completed request (observables, optionally the final state in
// the canonical layout); releases its device memory.
int csg_server_result(csg_server* s, int64_t id, csg_observables* obs, uint32_t* spins,
                      size_t n_spins) {
    if (!s) return fail(CSG_ERR_ARG, "null server");
    for (size_t i = 0; i < s->active.size(); ++i) {
        csg_server::Req& r = s->active[i];
        if (r.id != id) continue;
        if (!r.done) return fail(CSG_ERR_STATE, "request not completed");
        if (r.status != CSG_OK) {
            const int st = r.status;
            const std::string msg = "request " + std::to_string(id) + ": " + r.error;
            s->active.erase(s->active.begin() + (long)i);
            return fail(st, msg);
        }
        int rc = CSG_OK;
        if (obs) rc = csg_get_observables(r.e, obs);
        if (rc == CSG_OK && spins) rc = csg_get_state(r.e, spins, n_spins, nullptr, 0, nullptr);
        if (rc != CSG_OK) return rc;
        csg_engine_destroy(r.e);
        s->in_use -= r.bytes;
        s->active.erase(s->active.begin() + (long)i);
        return CSG_OK;
    }
    return fail(CSG_ERR_ARG, "unknown request id");
}

}  // extern "C"
