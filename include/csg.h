/*
 * csg.h — C ABI of the B200 parallel-tempering engine for the 3D +-J
 * Edwards-Anderson spin glass (libcsg.so).
 *
 * The reference program (Marco-Mendivil-Carboni/Spin-Glass) has no library
 * interface; its boundary is the `csg <sim_dir> <H>` command and the host
 * class `eamsim` (Program/src/eamsim.cuh:66-110).  Each entry point below
 * names the member or kernel of that class it replaces.  Conventions:
 *   - every function returns CSG_OK (0) or a CSG_ERR_* code; the message of
 *     the last failure on the calling thread is csg_last_error();
 *   - no exception, exit() or abort() crosses this boundary;
 *   - an engine owns its device memory; callers own every host buffer;
 *   - an engine is driven by one host thread and runs on one CUDA stream.
 *
 * Layouts (host and device, "canonical"):
 *   spins  uint32 [W][C][T/4][N][4]  — W words of 32 disorder samples (bit b
 *          of a word is sample 32w+b), C copies, T temperatures grouped in
 *          quads, N = L^3 sites in checkerboard order
 *          slot(x,y,z) = ((x+y+z)&1)*N/2 + ((z*L+y)*(L/2) + x/2),
 *          innermost axis t%4.  Bit 1 = spin up.
 *   bonds  uint32 [W][3][N] — bond between slot(i) and i+e_d, d = x,y,z;
 *          bit 1 = antiferromagnetic (J = -1).  Copies share bonds.
 */
#ifndef CSG_H
#define CSG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    CSG_OK = 0,
    CSG_ERR_ARG = 1,         /* invalid argument or configuration */
    CSG_ERR_CUDA = 2,        /* CUDA runtime failure */
    CSG_ERR_UNSUPPORTED = 3, /* configuration outside what the kernels cover */
    CSG_ERR_STATE = 4,       /* inconsistent input state (e.g. checkpoint) */
    CSG_ERR_NOMEM = 5        /* device or host allocation failed */
};

typedef struct csg_dims {
    int32_t L;        /* lattice side: even, 4..128 (L > 24: streaming engine) */
    int32_t n_words;  /* disorder samples / 32 */
    int32_t n_copies; /* independent copies per sample: 1 or 2 */
    int32_t n_temps;  /* temperatures: multiple of 4, 4..64 */
} csg_dims;

typedef struct csg_schedule {
    int32_t sweeps_per_swap; /* exchange after sweep s when (s+1)%k == 0; 0 = never */
    int32_t sweeps_per_meas; /* measure after sweep s when (s+1)%k == 0 ... */
    int64_t meas_start;      /* ... and s >= meas_start; k == 0: never */
} csg_schedule;

enum {
    CSG_MEASURE_M = 1,   /* also accumulate magnetisations at measurements */
    CSG_ENGINE_STREAM = 2, /* run the streaming engine (state in global memory, one
                              launch per colour) even where the cluster-resident
                              kernel fits; it always runs for L > 24 */
    CSG_STREAM_FUSED = 4   /* streaming engine, L <= 58: one launch per sweep that
                              updates both colours in a single pass over the state
                              (z-planes staged in shared memory by bulk copies): a
                              third of the DRAM traffic of the colour launches, but
                              slower on an otherwise idle B200 (one CTA per quad) */
};

typedef struct csg_config {
    csg_dims dims;
    csg_schedule sched;
    double H;                /* external field, 0 <= H <= 4 (eamsim.cu:520) */
    uint64_t seed;           /* Philox key of the whole simulation */
    const double* betas;     /* n_temps inverse temperatures (host); exchanges pair t, t+1 */
    int32_t flags;           /* CSG_MEASURE_M | CSG_ENGINE_STREAM | CSG_STREAM_FUSED */
    int32_t swap_log_rounds; /* keep accepted-exchange masks of this many rounds (tests) */
    int32_t word0;           /* global index of the first sample word (Philox counter word
                                2): a simulation split into shards of words with matching
                                word0 reproduces the unsplit run bit for bit */
} csg_config;

/* Accumulated observables (host arrays; any pointer may be NULL).
 * Shapes: e/m: [W][C][T][32]; q: [W][T][32]; q4: [W][T][32][2] (128-bit
 * little-endian halves); hist: [T][N+1] counts of D = #sites where the two
 * copies differ; swap_acc: [C][T] accepted exchanges of pair (t,t+1);
 * swap_log: [rounds][W][C][T] accepted-sample masks. */
typedef struct csg_observables {
    int64_t* e_sum;
    int64_t* m_sum;
    int64_t* q_sum;
    int64_t* q2_sum;
    uint64_t* q4_sum;
    uint32_t* hist;
    int32_t* e_last;
    int32_t* m_last;
    int32_t* d_last;
    uint64_t* swap_acc;
    uint32_t* swap_log;
    int64_t swap_log_rounds; /* capacity of swap_log (in) */
    int64_t swap_rounds;     /* exchange rounds done (out) */
    int64_t n_meas;          /* measurements done (out) */
    uint64_t boundary;       /* exchange decisions within 2^-40 (relative) of
                                their acceptance probability (out; must be 0) */
} csg_observables;

/* Device-side accumulators for csg_pt_run_device (device pointers, any may be
 * NULL).  swap_log row k holds global exchange round swap_round0 + k.  On the
 * device q4_sum[..][0] accumulates Q^4 mod 2^32 and q4_sum[..][1] accumulates
 * floor(Q^4 / 2^32); the total is q4_sum[1]*2^32 + q4_sum[0]
 * (csg_get_observables returns it as a 128-bit value). */
typedef struct csg_device_obs {
    int64_t* e_sum;
    int64_t* m_sum;
    int64_t* q_sum;
    int64_t* q2_sum;
    uint64_t* q4_sum;
    uint32_t* hist;
    int32_t* e_last;
    int32_t* m_last;
    int32_t* d_last;
    uint64_t* swap_acc;
    uint32_t* swap_log;
    int64_t swap_log_rounds;
    int64_t swap_round0;
    uint64_t* boundary;
} csg_device_obs;

/* Launch plan: quads per CTA, CTAs per sample word (cluster size), threads
 * per quad, dynamic shared memory bytes. */
typedef struct csg_plan {
    int32_t quads_per_cta;
    int32_t ctas_per_word;
    int32_t threads_per_quad;
    int32_t smem_bytes;
} csg_plan;

typedef struct csg_engine csg_engine;

/* Message of the last failure on this thread ("" if none). */
const char* csg_last_error(void);

/* eamsim::eamsim (eamsim.cu:516-543): validate the configuration, allocate
 * device state on the current CUDA device. */
int csg_engine_create(const csg_config* cfg, csg_engine** out);

/* eamsim::~eamsim (eamsim.cu:546-559). NULL is accepted. */
int csg_engine_destroy(csg_engine* e);

/* eamsim::init_lattice (eamsim.cu:622-652): +-J bonds and uniform random
 * spins from the seed, generated on the device.  Resets the sweep counter
 * and the observables. */
int csg_init_lattice(csg_engine* e);

/* Host <-> device state in the canonical layout (counts in uint32 words:
 * spins W*C*T*N, bonds W*3*N).  set_state resets observables and sets the
 * sweep counter to `sweep`. */
int csg_set_state(csg_engine* e, const uint32_t* spins, size_t n_spins, const uint32_t* bonds,
                  size_t n_bonds, int64_t sweep);
int csg_get_state(csg_engine* e, uint32_t* spins, size_t n_spins, uint32_t* bonds,
                  size_t n_bonds, int64_t* sweep);

/* run_simulation_section (eamsim.cu:347-416) looped as in
 * eamsim::run_simulation (eamsim.cu:689-709): n_sweeps Metropolis sweeps
 * with the exchange and measurement schedule of the configuration,
 * continuing from the engine's sweep counter.  Asynchronous on the engine's
 * stream; csg_get_observables / csg_get_state synchronise. */
int csg_run(csg_engine* e, int64_t n_sweeps);

/* Copy the accumulated observables to host arrays. */
int csg_get_observables(csg_engine* e, csg_observables* out);

/* Reset all accumulators to zero. */
int csg_reset_observables(csg_engine* e);

/* rearrange + compute_q (eamsim.cu:419-511) and the e/m output of
 * eamsim.cu:407-415: observable records obs_s (eamsim.cuh:55-62), 11 floats
 * {e[2], m[2], q_0, q_1_r[3], q_1_i[3]} per (sample, temperature), shape
 * [32W][T][11].  Requires n_copies == 2.  All fields are of the current
 * state; the reference's e/m are those of its last exchange round (taken
 * before that round's swap, 16 sweeps before the section ends), its q fields
 * are of the current state as here. */
int csg_obs_records(csg_engine* e, float* rec, size_t n_floats);

/* eamsim::save_checkpoint / load_checkpoint (eamsim.cu:655-676): the
 * reference's checkpoint layout uint32 [2*32W][N] — lattice 2*sample+copy,
 * site (z*L+y)*L+x, bits 0..T-1 spins by temperature, bits 26..31 the six
 * bonds (-x,+x,-y,+y,-z,+z; bit 1 = ferromagnetic).  Requires
 * n_copies == 2 and n_temps <= 24.  load_checkpoint checks that the bond
 * bits agree between the ends of every bond and between the two copies. */
int csg_save_checkpoint(csg_engine* e, uint32_t* ref, size_t n_words);
int csg_load_checkpoint(csg_engine* e, const uint32_t* ref, size_t n_words, int64_t sweep);

/* run_simulation_section (eamsim.cu:347-416) on caller-owned device buffers:
 * n_sweeps sweeps of `spins` (canonical layout, device memory) starting at
 * global sweep index sweep0, adding to the device accumulators of `obs`
 * (may be NULL).  stream: a cudaStream_t (NULL = legacy default stream).
 * Queued on the stream; the cluster-resident kernel (L <= 24) allocates
 * nothing, the streaming engine (L > 24 or CSG_ENGINE_STREAM) takes a few MB
 * of stream-ordered scratch (cudaMallocAsync / cudaFreeAsync on the stream). */
int csg_pt_run_device(const csg_config* cfg, uint32_t* spins, const uint32_t* bonds,
                      const csg_device_obs* obs, int64_t sweep0, int64_t n_sweeps, void* stream);

/* init_multispins + init_coupling_constants (eamsim.cu:562-619) into
 * caller-owned device buffers, from the seed. */
int csg_init_device(const csg_config* cfg, uint32_t* spins, uint32_t* bonds, void* stream);

/* Launch plan the engine picks for a configuration (no counterpart in the
 * reference, whose launch shape is fixed at eamsim.cu:695). */
int csg_query_plan(const csg_config* cfg, csg_plan* out);

/* Force quads_per_cta (must divide n_copies*n_temps/4) and/or
 * threads_per_quad (L * L/2 * s for a built column split s) for later launches
 * of the resident kernel; a zero field keeps that part automatic, NULL
 * restores the automatic plan.  A CTA takes at most 512 threads, and at most
 * 384 when H != 0 with threads_per_quad = L * L/2 (the general-field kernel
 * walking whole columns, built for 168 registers per thread); a forced tile
 * beyond that is refused with CSG_ERR_UNSUPPORTED by engine creation, plan
 * queries and runs. */
int csg_set_plan_override(const csg_plan* plan);

/* No counterpart in the reference.  The observable records of
 * csg_obs_records for a state held in the caller's device memory, without
 * allocating anything: for callers whose device memory all belongs to their
 * own pool or budget (a framework's caching allocator, a server admitting
 * work against a fixed budget), where a library's cudaMalloc could fail and
 * its cudaFree would synchronise the device.  spins/bonds (canonical layout)
 * and rec ([32W][T][11] floats) are device pointers; the kernels are queued
 * on `stream` and the caller synchronises.  The intermediate integers live in
 * one fixed 16 MiB device array per GPU, held until the process exits; a call
 * needs W*T*32*(5+3L) ints of it and larger states are rejected with
 * CSG_ERR_UNSUPPORTED.  The first call on a device looks up that array's
 * device address (make it before any stream capture).  All calls share the
 * array: calls that overlap on the GPU (other streams, other threads) race.
 * Every element a call reads is written by that call first. */
int csg_obs_records_noalloc(const csg_config* cfg, const uint32_t* spins, const uint32_t* bonds,
                            float* rec, size_t n_floats, void* stream);

/* analyze-all.py:38-71 (the reference's analysis script): the result table of
 * a record series on the GPU.  rec: device pointer to n_meas * ndis * nrep
 * records (obs_s, 11 floats, the layout of <H>-obs.bin) - pass the part after
 * the thermalisation, as the script drops the first half.  table: host array
 * [nrep][8] receiving chi_0, its error, xi_L/L, its error, e, its error, m, its
 * error (the script's estimators; the error is the standard error over
 * disorder samples).  Runs on stream (NULL: the default stream) and returns
 * when the table is ready; takes ndis * nrep * 72 bytes of stream-ordered
 * scratch. */
int csg_analyze_records(const float* rec, int64_t n_meas, int32_t ndis, int32_t nrep, int32_t L,
                        double* table, void* stream);

/* ---- Batched engine -------------------------------------------------------
 * No counterpart in the reference, which compiles one lattice size into its
 * binary (eamsim.cuh:13) and runs one simulation per process.  A batch holds
 * several simulations (any mix of L, sample counts, ladders, schedules), each
 * a full engine, and advances all of them with one launch of a captured CUDA
 * graph whose parallel branches are the members' cluster-resident kernels.
 * Every member keeps its own Philox counters: its results are bit-identical
 * to running it alone. */
typedef struct csg_batch csg_batch;

int csg_batch_create(const csg_config* cfgs, int32_t n, csg_batch** out);
int csg_batch_destroy(csg_batch* b);

/* Borrowed handle of member i (init / set / get state, observables, ...). */
int csg_batch_engine(csg_batch* b, int32_t i, csg_engine** out);

/* n_sweeps sweeps of every member, one graph launch (the graph is captured on
 * first use for this n_sweeps and replayed afterwards). */
int csg_batch_run(csg_batch* b, int64_t n_sweeps);

/* The same work as the plain engine would do it: member after member, each
 * with the plan it would take alone. */
int csg_batch_run_sequential(csg_batch* b, int64_t n_sweeps);

/* Queue n_sweeps sweeps of every member on `stream` (a cudaStream_t; NULL =
 * legacy default stream) without waiting: plain == 0 launches the batch graph
 * (as csg_batch_run), plain == 1 the plain engine member after member (as
 * csg_batch_run_sequential).  The launch is ordered after the work already
 * queued on the members' streams and before work queued on them later (state
 * and observable calls on a member wait for it).  For timing on the caller's
 * stream. */
int csg_batch_launch(csg_batch* b, int64_t n_sweeps, int32_t plain, void* stream);

/* Autotuner: chooses each member's tile — quads per CTA (hence its cluster
 * size) and threads per quad (how many z-segments a column of the checkerboard
 * is split into) — and, per member, whether each of its CTAs gets an SM of
 * its own (its shared memory padded past half an SM), by timing the whole
 * batch graph for probe_sweeps sweeps; states are restored after.  chosen
 * (may be NULL) receives the quads per CTA per member; csg_batch_member_plan
 * reports the whole plan (smem_bytes includes the padding). */
int csg_batch_tune(csg_batch* b, int64_t probe_sweeps, int32_t* chosen);

/* Set each member's quads per CTA (0 = automatic; threads per quad automatic). */
int csg_batch_set_plan(csg_batch* b, const int32_t* quads_per_cta);

/* The launch plan member i runs with (after csg_batch_tune: the tuned one). */
int csg_batch_member_plan(csg_batch* b, int32_t i, csg_plan* out);

/* Fix member i's tile: quads_per_cta and threads_per_quad (0 in either:
 * automatic; the other fields are ignored), e.g. a plan an earlier
 * csg_batch_tune chose. */
int csg_batch_set_member_plan(csg_batch* b, int32_t i, const csg_plan* plan);

/* ---- Serving: continuous batching -------------------------------------------
 * No counterpart in the reference.  Requests (full simulation configurations
 * plus a sweep count) are queued, admitted FIFO while a device-memory budget
 * and an active-slot limit allow, initialised from their seeds on the GPU,
 * and advanced section by section on their own streams, so that the kernels
 * of different requests overlap on the device.  Each request keeps its own
 * Philox counters: its result equals running it alone. */
typedef struct csg_server csg_server;

/* Device bytes an engine for this configuration allocates. */
int csg_engine_footprint(const csg_config* cfg, size_t* bytes);

int csg_server_create(size_t memory_budget_bytes, int32_t max_active, int32_t sweeps_per_launch,
                      csg_server** out);
int csg_server_destroy(csg_server* s);

/* Queue a request; fails with CSG_ERR_NOMEM if it can never fit the budget. */
int csg_server_submit(csg_server* s, const csg_config* cfg, int64_t n_sweeps, int64_t* id);

/* Non-blocking scheduling pass (call it often): reports requests completed
 * since the last pass (up to max_completed ids), active and queued counts. */
int csg_server_poll(csg_server* s, int64_t* completed, int32_t max_completed,
                    int32_t* n_completed, int32_t* n_active, int32_t* n_queued);

/* Observables (and optionally the final spins) of a completed request;
 * releases its memory.  Any output pointer may be NULL.  A request whose
 * engine could not be created at admission (e.g. device memory exhausted) or
 * whose launch failed is reported completed by csg_server_poll; this call
 * then returns that error code (message in csg_last_error) and releases it. */
int csg_server_result(csg_server* s, int64_t id, csg_observables* obs, uint32_t* spins,
                      size_t n_spins);

#ifdef __cplusplus
}
#endif
#endif /* CSG_H */
