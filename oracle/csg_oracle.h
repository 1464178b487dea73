/*
 * csg_oracle.h — CPU oracle for the parallel-tempering Metropolis path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the CUDA engine
 * is compared against, bit for bit.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline / --impl reference legs may load it.  Nothing in
 * the product (spin-glass_b200/) links, loads or calls it.
 *
 * It restates, one site and one sample at a time, the update rule of the
 * reference program (Program/src/eamsim.cu of Marco-Mendivil-Carboni/
 * Spin-Glass) in the sample-packed layout used by the engine:
 *   - checkerboard Metropolis sweep          eamsim.cu:112-208
 *   - acceptance-table construction          eamsim.cu:24-40
 *   - energy / magnetisation definitions     eamsim.cu:237-325
 *   - even/odd replica-exchange rule         eamsim.cu:43-90
 *   - overlap q and its Fourier components   eamsim.cu:451-511
 *   - bond generation / per-site bond bits   eamsim.cu:578-619
 *   - beta ladder                            eamsim.cu:725-744
 * The random numbers come from its own Philox4x32-10 (Salmon et al., SC'11),
 * written independently of the engine's copy.  orc_run_multispin (the CPU
 * timing baseline) evaluates the acceptance of the 32 samples of a word at
 * once and is checked against the per-sample orc_run.
 *
 * Layout (identical to the engine's canonical host layout):
 *   spins  uint32 [W][C][T/4][N][4]   site index = checkerboard slot, last
 *                                     axis = temperature t%4 of quad t/4
 *   bonds  uint32 [W][3][N]           bond i -> i+e_d at slot(i), bit=1: J=-1
 *   slot(x,y,z) = ((x+y+z)&1)*N/2 + ((z*L+y)*(L/2) + x/2)
 * Bit b of every word is disorder sample 32*w+b.
 */
#ifndef CSG_ORACLE_H
#define CSG_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    int32_t L, W, C, T;
    int32_t sweeps_per_swap;   /* 0 = never */
    int32_t sweeps_per_meas;   /* 0 = never */
    int64_t meas_start;        /* first sweep that may be measured */
    double H;
    uint64_t seed;
    const double* betas;       /* [T] */
    const uint64_t* thr;       /* [T][2][7] from orc_thresholds */
    int32_t n_threads;         /* OpenMP threads, 0 = runtime default */
    int32_t word0;             /* global index of word 0 (Philox counter word 2) */
} orc_params;

typedef struct orc_obs {
    int64_t* e_sum;            /* [W][C][T][32]  sum of bond energies */
    int64_t* m_sum;            /* [W][C][T][32]  sum of magnetisations */
    int64_t* q_sum;            /* [W][T][32]     sum of Q = N - 2D */
    int64_t* q2_sum;           /* [W][T][32]     sum of Q^2 */
    uint64_t* q4_sum;          /* [W][T][32][2]  sum of Q^4, 128-bit lo,hi */
    uint32_t* hist;            /* [T][N+1]       histogram of D */
    int32_t* e_last;           /* [W][C][T][32] */
    int32_t* m_last;           /* [W][C][T][32] */
    int32_t* d_last;           /* [W][T][32] */
    uint64_t* swap_acc;        /* [C][T]  accepted exchanges of pair (t,t+1) */
    uint32_t* swap_log;        /* [rounds][W][C][T] masks, or NULL */
    int64_t swap_log_rounds;   /* capacity of swap_log in rounds */
    int64_t swap_rounds;       /* rounds performed (out) */
    int64_t n_meas;            /* measurements performed (out) */
    uint64_t boundary;         /* swap decisions within the ulp window (out) */
} orc_obs;

/* Philox4x32-10 block function. */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* Metropolis acceptance thresholds thr[t][s][U] (s = centre spin bit, U =
 * unsatisfied bonds 0..6); 2^32 means "always accept". Returns 0 on success. */
int orc_thresholds(int32_t T, const double* betas, double H, uint64_t* thr);

/* Bonds and initial spins from the seed. */
int orc_init(int32_t L, int32_t W, int32_t C, int32_t T, uint64_t seed, int32_t word0,
             uint32_t* spins, uint32_t* bonds);

/* n_sweeps sweeps starting at global sweep index sweep0, with the exchange
 * and measurement schedule of p.  obs accumulators are added to. */
int orc_run(const orc_params* p, uint32_t* spins, const uint32_t* bonds,
            int64_t sweep0, int64_t n_sweeps, orc_obs* obs);

/* orc_run with the Metropolis step evaluated for all 32 samples of a word at
 * once (bit-sliced bond counts, a mask per acceptance class) instead of one
 * sample at a time: the CPU timing baseline.  Same arguments, same results
 * bit for bit (checked by the tests); exchange and measurement are shared. */
int orc_run_multispin(const orc_params* p, uint32_t* spins, const uint32_t* bonds,
                      int64_t sweep0, int64_t n_sweeps, orc_obs* obs);

/* Bond energy E_b = -(sum of J s s) and magnetisation per sample, per plane:
 * e[W][C][T][32], m[W][C][T][32]. */
int orc_energies(int32_t L, int32_t W, int32_t C, int32_t T,
                 const uint32_t* spins, const uint32_t* bonds,
                 int32_t* e, int32_t* m);

/* Overlap integers of the current state: d[W][T][32] = sum_i [s1 != s2] and
 * per-coordinate partial sums dpl[W][T][32][3][L] (direction x,y,z, value
 * of that coordinate). Requires C == 2. */
int orc_overlaps(int32_t L, int32_t W, int32_t T, const uint32_t* spins,
                 int32_t* d, int32_t* dpl);

/* Reference obs_s records (eamsim.cuh:55-62) for the current state, samples
 * in order, temperatures in order: 11 floats per record
 * {e[2], m[2], q_0, q_1_r[3], q_1_i[3]}, shape [32W][T][11]. */
int orc_obs_records(int32_t L, int32_t W, int32_t T, float H,
                    const uint32_t* spins, const uint32_t* bonds, float* rec);

/* Conversions between the sample-packed layout and the reference's
 * checkpoint layout uint32 [32W*2][N] (eamsim.cu:598-616, 655-676).
 * Requires C == 2 and T <= 24. */
int orc_to_ref_lattice(int32_t L, int32_t W, int32_t T, const uint32_t* spins,
                       const uint32_t* bonds, uint32_t* ref);
int orc_from_ref_lattice(int32_t L, int32_t W, int32_t T, const uint32_t* ref,
                         uint32_t* spins, uint32_t* bonds);

#ifdef __cplusplus
}
#endif
#endif
