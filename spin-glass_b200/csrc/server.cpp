// server.cpp — serving: continuous batching of simulation requests.  Requests
// queue FIFO, are admitted while a device-memory budget and a slot count
// allow, and run as plain engines on their own streams in sections of a fixed
// number of sweeps, so that new requests join between sections.
//
// Nothing on the serving path waits for the whole device: every request's
// device memory comes from the server's own memory pool in the order of the
// request's stream (cudaMallocFromPoolAsync at admission, cudaFreeAsync when
// its result is fetched or it fails), and the pool and the streams are made
// once, at the first admission.  A completed request keeps its memory (its results live there)
// until csg_server_result, but no longer takes an active slot.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
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
        cudaStream_t stream = nullptr;  // borrowed from the server while admitted
        bool done = false;
        // a request whose engine could not be created or launched, or whose
        // stream reported an error, completes with this error, which
        // csg_server_result returns
        int status = CSG_OK;
        std::string error;
    };
    size_t budget = 0, in_use = 0;
    int max_active = 0;
    int64_t chunk = 1024, next_id = 1;
    cudaMemPool_t pool = nullptr;
    std::vector<cudaStream_t> streams;  // all the server's streams
    std::vector<cudaStream_t> idle;     // streams no admitted request holds
    std::vector<Req> queue;             // waiting, FIFO
    std::vector<Req> active;            // admitted: running, or completed and not fetched
    bool device_ready = false;
};

namespace {

void release_request(csg_server* s, csg_server::Req& r) {
    if (r.e) {
        engine_release(r.e);  // memory back to the pool in the stream's order
        r.e = nullptr;
        s->in_use -= r.bytes;
    }
    if (r.stream) {
        s->idle.push_back(r.stream);
        r.stream = nullptr;
    }
}

// The pool and the streams, on the current device, at the first admission.
int ensure_device(csg_server* s) {
    if (s->device_ready) return CSG_OK;
    int dev = 0;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    cudaError_t ce = cudaGetDevice(&dev);
    props.location.id = dev;
    if (ce == cudaSuccess && !s->pool) ce = cudaMemPoolCreate(&s->pool, &props);
    if (ce == cudaSuccess) {
        // keep freed memory in the pool (up to the budget, which admission
        // enforces) instead of returning it to the driver at each sync point
        uint64_t keep = s->budget;
        ce = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    while (ce == cudaSuccess && (int)s->streams.size() < s->max_active) {
        cudaStream_t st = nullptr;
        ce = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (ce == cudaSuccess) {
            s->streams.push_back(st);
            s->idle.push_back(st);
        }
    }
    if (ce != cudaSuccess) {
        cudaGetLastError();
        return fail(CSG_ERR_CUDA, std::string("server device setup: ") + cudaGetErrorString(ce));
    }
    s->device_ready = true;
    return CSG_OK;
}

void destroy_server(csg_server* s) {
    for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
    for (auto& r : s->active) release_request(s, r);
    for (cudaStream_t st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
}

}  // namespace

extern "C" {

int csg_server_create(size_t memory_budget_bytes, int32_t max_active, int32_t sweeps_per_launch,
                      csg_server** out) {
    if (!out || memory_budget_bytes == 0 || max_active < 1 || sweeps_per_launch < 1)
        return fail(CSG_ERR_ARG, "bad server arguments");
    *out = nullptr;
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
    destroy_server(s);
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
    // a failed request gives its memory and stream back at once; its id is
    // reported done and the other requests carry on
    auto failed = [&](csg_server::Req& r, int rc, const std::string& msg) {
        r.status = rc;
        r.error = msg;
        release_request(s, r);
        report(r);
    };
    for (auto& r : s->active) {
        if (r.done) continue;
        const cudaError_t q = cudaStreamQuery(r.stream);
        if (q == cudaErrorNotReady) continue;
        if (q != cudaSuccess) {
            cudaGetLastError();
            failed(r, CSG_ERR_CUDA, std::string("request stream: ") + cudaGetErrorString(q));
            continue;
        }
        if (r.launched >= r.total) report(r);
    }
    auto running_count = [&] {
        int n = 0;
        for (auto& r : s->active) n += r.done ? 0 : 1;
        return n;
    };
    int running = running_count();
    while (!s->queue.empty() && running < s->max_active &&
           s->in_use + s->queue.front().bytes <= s->budget) {
        const int dev_rc = ensure_device(s);
        if (dev_rc == CSG_OK && s->idle.empty()) break;
        s->active.push_back(std::move(s->queue.front()));
        s->queue.erase(s->queue.begin());
        csg_server::Req& r = s->active.back();
        r.cfg.betas = r.betas.data();
        ++running;
        if (dev_rc != CSG_OK) {  // e.g. no device: the request completes with the error
            failed(r, dev_rc, last_error());
            --running;
            continue;
        }
        r.stream = s->idle.back();
        s->idle.pop_back();
        int rc = engine_create_pooled(&r.cfg, s->pool, r.stream, &r.e);
        if (rc == CSG_OK) {
            s->in_use += r.bytes;
            rc = csg_init_lattice(r.e);
        }
        if (rc != CSG_OK) {
            failed(r, rc, last_error());
            --running;
        }
    }
    for (auto& r : s->active) {
        if (r.done || r.launched >= r.total) continue;
        if (cudaStreamQuery(r.stream) != cudaSuccess) continue;
        const int64_t n = std::min<int64_t>(s->chunk, r.total - r.launched);
        // alone, a request takes the plan that spreads it widest; sharing the
        // GPU, the one with the fewest CTAs (every plan gives the same bits)
        const PlanChoice pc = running > 1 ? shared_gpu_plan(r.cfg) : PlanChoice{};
        r.e->qc = pc.qc;
        r.e->nseg = pc.nseg;
        if (int rc = csg_run(r.e, n)) {
            failed(r, rc, last_error());
            continue;
        }
        r.launched += n;
    }
    if (n_completed) *n_completed = nc;
    if (n_active) *n_active = running_count();
    if (n_queued) *n_queued = (int32_t)s->queue.size();
    return CSG_OK;
}

// Results of a completed request (observables, optionally the final state in
// the canonical layout); gives its memory back to the server's pool.
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
            release_request(s, r);
            s->active.erase(s->active.begin() + (long)i);
            return fail(st, msg);
        }
        // copies on the request's own stream: waits for nothing else
        int rc = CSG_OK;
        if (obs) rc = csg_get_observables(r.e, obs);
        if (rc == CSG_OK && spins) rc = csg_get_state(r.e, spins, n_spins, nullptr, 0, nullptr);
        if (rc != CSG_OK) return rc;
        release_request(s, r);
        s->active.erase(s->active.begin() + (long)i);
        return CSG_OK;
    }
    return fail(CSG_ERR_ARG, "unknown request id");
}

}  // extern "C"
