// engine_internal.h — what the host translation units of libcsg.so share: the
// engine object, error reporting, and the planning and launch entry points
// defined in csg_engine.cu.  Nothing here is exported; the library's ABI is
// include/csg.h.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include "csg.h"

// One simulation: its configuration, device state, accumulators and stream.
struct csg_engine {
    csg_config cfg{};
    std::vector<double> betas;
    cudaStream_t stream = nullptr;
    size_t n_spins = 0, n_bonds = 0, n_e = 0, n_q = 0, n_hist = 0;
    uint32_t* spins = nullptr;
    uint32_t* bonds = nullptr;
    // device accumulators
    int64_t *e_sum = nullptr, *m_sum = nullptr, *q_sum = nullptr, *q2_sum = nullptr;
    uint64_t* q4_sum = nullptr;
    uint32_t* hist = nullptr;
    int32_t *e_last = nullptr, *m_last = nullptr, *d_last = nullptr;
    uint64_t* swap_acc = nullptr;
    uint32_t* swap_log = nullptr;
    uint64_t* boundary = nullptr;
    int64_t sweep = 0, n_meas = 0, swap_rounds = 0, swap_round0 = 0;
    // resident-kernel plan chosen by a batch's tuner or a server (0: automatic)
    int qc = 0;    // quads per CTA
    int nseg = 0;  // column segments per thread (threads per quad = L * L/2 * nseg)
    // device scratch of csg_obs_records, allocated at its first call
    char* rec_scratch = nullptr;
    // Set for a server's engines: device memory comes from this pool in the
    // order of the engine's stream (cudaMallocFromPoolAsync / cudaFreeAsync),
    // so creating and releasing the engine never waits for the device; the
    // stream then belongs to the server.
    cudaMemPool_t pool = nullptr;
    bool own_stream = true;
};

#define CSG_INTERNAL __attribute__((visibility("hidden")))

namespace csg_detail {

// Launch shape of the cluster-resident kernel: Qc quads per CTA, K CTAs per
// cluster (one cluster per sample word), TPQ threads per quad (NSEG column
// segments per thread), CTA of `threads` (Qc*TPQ rounded up to whole warps).
struct Plan {
    int Qc = 0, K = 0, TPQ = 0, NSEG = 0, threads = 0;
    size_t smem = 0;
};

// A resident-kernel plan to force (0 in a field: choose it automatically).
struct PlanChoice {
    int qc = 0, nseg = 0;
};

// Error reporting: the message is what csg_last_error() returns on this thread.
CSG_INTERNAL int fail(int code, const std::string& msg);
CSG_INTERNAL void set_last_error(const std::string& msg);
CSG_INTERNAL const std::string& last_error();

// An engine whose device memory comes from `pool` in the order of `stream`
// (borrowed, not destroyed with the engine), and its release: the memory goes
// back to the pool in stream order and nothing waits for the device.
CSG_INTERNAL int engine_create_pooled(const csg_config* cfg, cudaMemPool_t pool,
                                      cudaStream_t stream, csg_engine** out);
CSG_INTERNAL void engine_release(csg_engine* e);

// Device memory for an engine: from its pool (stream-ordered) or cudaMalloc.
CSG_INTERNAL int engine_alloc(csg_engine* e, void** p, size_t bytes);

// Configuration checks.
CSG_INTERNAL int validate(const csg_config* cfg);
CSG_INTERNAL bool use_stream(const csg_config& c);  // streaming engine, not the resident kernel
CSG_INTERNAL size_t footprint_bytes(const csg_config& c);

// The (quads per CTA, column segments) pairs that fit one CTA and one
// cluster of the resident kernel (empty for the streaming engine).
CSG_INTERNAL std::vector<PlanChoice> plan_options(const csg_config& c);

// Plan of an engine's resident kernel (its tuner choice e->qc / e->nseg, if
// any), with the CTA's shared memory raised to at least min_smem.
CSG_INTERNAL int plan_engine(csg_engine* e, Plan& pl, size_t min_smem = 0);

// n_sweeps sweeps from sweep0 on caller buffers, launched on st.  forced
// fixes parts of the plan; sweep_dev (resident kernel only) makes the kernel
// read its starting sweep from device memory and advance it, for replayed
// graphs; plan_in skips planning (required inside a stream capture).
CSG_INTERNAL int run_device(const csg_config& cfg, uint32_t* spins, const uint32_t* bonds,
                            const csg_device_obs* obs, int64_t sweep0, int64_t n_sweeps,
                            cudaStream_t st, PlanChoice forced = PlanChoice{},
                            long long* sweep_dev = nullptr, const Plan* plan_in = nullptr);

CSG_INTERNAL csg_device_obs device_obs(const csg_engine* e);

// In a graph captured from run_device calls of several engines (in the order
// given, each with the column split nseg of its plan), makes the first
// resident-kernel launch of each engine after the first depend on every block
// of the previous one's first launch having begun (a programmatic edge from
// its launch-completion port): the GPU then places the launches' clusters in
// this order however the graph's launch is gated, and nothing waits for a
// launch to finish.
CSG_INTERNAL int chain_launch_starts(cudaGraph_t g, const std::vector<const csg_engine*>& members,
                                     const std::vector<int>& nseg);

// Host counters after n sweeps ran: sweep index, exchange rounds, measurements.
CSG_INTERNAL void account(csg_engine* e, int64_t n);

// n elements of device memory (nullptr for n == 0); CSG_ERR_NOMEM on failure.
template <typename T>
int dalloc(T** p, size_t n) {
    *p = nullptr;
    if (n == 0) return CSG_OK;
    const cudaError_t e = cudaMalloc(reinterpret_cast<void**>(p), n * sizeof(T));
    if (e != cudaSuccess) {
        cudaGetLastError();
        *p = nullptr;
        return fail(CSG_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return CSG_OK;
}

}  // namespace csg_detail

#define CSG_CUDA(call)                                                                     \
    do {                                                                                   \
        const cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess)                                                             \
            return ::csg_detail::fail(CSG_ERR_CUDA,                                        \
                                      std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)
