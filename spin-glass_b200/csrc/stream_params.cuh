// stream_params.cuh — what the streaming engine's kernels (stream_kernels.cuh,
// stream_sweep.cu) and its host code share: launch shapes, the parameter
// block, the measurement accumulators and programmatic dependent launch.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "philox.cuh"
#include "pt_kernel.cuh"

namespace csg {


// Launch shapes (measured at L=32 and L=48).  Plain colour launches: blocks of
// kStreamThreads threads, kStreamSPT sites of the colour per thread.
constexpr int kStreamThreads = 256;
constexpr int kStreamSPT = 8;
// Colour launches that count (energies, magnetisations) run smaller blocks of
// kStreamAccSitesPerBlock sites (their counters live in shared memory, one
// column per thread).
constexpr int kStreamAccThreads = 128;
#ifndef CSG_STREAM_ACC_SPT
#define CSG_STREAM_ACC_SPT 8
#endif
constexpr int kStreamAccSPT = CSG_STREAM_ACC_SPT;
constexpr int kStreamAccSitesPerBlock = kStreamAccThreads * kStreamAccSPT;
template <bool ACC>
__host__ __device__ constexpr int colour_threads() { return ACC ? kStreamAccThreads : kStreamThreads; }
template <bool ACC>
__host__ __device__ constexpr int colour_spt() { return ACC ? kStreamAccSPT : kStreamSPT; }
constexpr int kStreamNLV = bit_length(6 * kStreamAccSPT);  // bits of a per-thread bond count
constexpr int kStreamNLM = bit_length(kStreamAccSPT);      // bits of a per-thread site count
// Overlap passes (both copies of every quad): blocks of kStreamThreads threads
// over kOverlapSitesPerBlock sites (all N sites of a lattice).
constexpr int kOverlapSPT = 8;
constexpr int kOverlapSitesPerBlock = kStreamThreads * kOverlapSPT;
constexpr int kOverlapNL = bit_length(kOverlapSPT);

struct StreamParams {
    uint32_t* spins;
    const uint32_t* bonds;
    // per-plane totals, added to by the blocks (integer atomics: any order gives
    // the same sums) and cleared by the kernel that consumes them
    int* u_acc;   // [W][C][T][32] unsatisfied bonds after the sweep
    int* up_acc;  // [W][C][T][32] spins up after the sweep
    int* d_acc;   // [W][T][32] sites where the copies differ
    int* energy;  // [W][C][T][32] bond energies after the exchange
    int* magn;    // [W][C][T][32]
    uint32_t* masks;  // [W][C][T] accepted-sample masks of the current round
    int* err;         // set to 1 by a sweep launch whose staging wait gave up
    int L, W, C, T, Q;
    int nblk;   // blocks per quad of a counting colour launch
    int nblk2;  // blocks per quad of an overlap pass (over all N sites)
    uint32_t k0, k1, word0;
    uint32_t mag_plane;  // ceil(2^32 / (L*L/2)): division by multiply-high
    uint32_t mag_row;    // ceil(2^32 / (L/2))
    double H;
    PtTables tab;
};

// n / d for 0 <= n < L^3/2, d in {L/2, L*L/2}, with mag = ceil(2^32 / d): the
// multiply-high estimate is never below n / d and at most one above it for
// every even L <= 128 (checked exhaustively), so one correction makes it exact.
__device__ __forceinline__ int div_magic(int n, int d, uint32_t mag) {
    const int q = (int)__umulhi((uint32_t)n, mag);
    return q - (q * d > n ? 1 : 0);
}

// The fused sweep launch (stream_sweep.cu): both colours of one sweep in one
// pass over the state, for lattices whose ring of z-planes fits in shared
// memory (stream_sweep_fits).  Energies (acc_e) and magnetisations (acc_m) go
// to the same per-plane totals as the colour launches' counts.
bool stream_sweep_fits(int L);
// Threads per CTA (one CTA per quad) and dynamic shared memory of the fused
// sweep launch for lattice side L (zeros where it does not fit).
void stream_sweep_shape(int L, int* threads, int* smem_bytes);
cudaError_t launch_stream_sweep(const StreamParams& P, long long s, bool gen, bool acc_e, bool acc_m,
                                cudaStream_t st);

// Measurement accumulators (layouts as in PtParams / csg_device_obs).
struct StreamObs {
    long long* e_sum;
    long long* m_sum;
    long long* q_sum;
    long long* q2_sum;
    unsigned long long* q4_sum;
    unsigned int* hist;
    int* e_last;
    int* m_last;
    int* d_last;
};

// Programmatic dependent launch (the sweep's kernels are launched with it): a
// kernel waits here until the previous kernel on the stream has finished and
// its writes are visible, then lets the next kernel's blocks be scheduled as
// soon as all of its own blocks run, so launch latency overlaps the tail.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace csg
