// stream_sweep.cu — one launch per sweep of the streaming engine: both
// checkerboard colours in a single pass over the state (reference:
// perform_MC_steps, eamsim.cu:112-208, for lattices too large to stay on chip).
//
// One CTA per temperature quad (w, c, q) walks the lattice along z.  Shared
// memory holds a ring of kSweepSlots z-planes of each colour (L*L/2 uint4:
// the quad's 4 planes per site), filled by 1-D bulk async copies one step
// ahead (cp.async.bulk, completion on an mbarrier, bounded waits).  Step z
// updates colour 0 in plane z, then (after a barrier) colour 1 in plane z-1:
//   colour 0 at z   reads colour 1 at z-1, z, z+1 as they were before the sweep;
//   colour 1 at z-1 reads colour 0 at z-2, z-1, z, all updated by then.
// A plane's bonds are read in two consecutive steps (the ring leaves ~90 KB
// of L1 at L = 48 for them).  Colour 1 of plane 0 waits until the end (it
// needs colour 0 of plane L-1), and the planes past L-1 (colour 1 of plane 0
// before its update, colour 0 of planes 0 and 1 after theirs) are read back
// from global memory, where each update is written as soon as it is made.
// New colour-0 words also go to their ring slot (colour 1 reads them there);
// new colour-1 words only to global memory.
// Every word of the state is read once and written once per sweep.
//
// The arithmetic of a site update, the Philox counters and the energy and
// magnetisation counts are those of the colour launches (stream_kernels.cuh)
// and of the resident kernel, so results are bit-identical to them and to the
// CPU oracle.
#include <cuda_runtime.h>

#include <algorithm>

#include "pt_resident.cuh"
#include "stream_params.cuh"

namespace csg {

namespace {

constexpr int kSweepSlots = 4;  // ring slots per colour: 3 in use, 1 being filled
constexpr int kSweepMaxThreads = 512;
constexpr int kSweepWaitTries = 1 << 22;  // bound on every mbarrier wait

__host__ __device__ inline size_t sweep_smem_bytes(int L) {
    return (size_t)2 * kSweepSlots * L * (L / 2) * 16;
}
constexpr size_t kSweepMaxSmem = 216 * 1024;  // the ring at L = 58 (215,296 B) fits under this

// Sites of a colour per thread and step: the fewest that keep a CTA within
// kSweepMaxThreads threads (0: the plane is too large).
__host__ __device__ inline int sweep_spt(int L) {
    const int PL = L * (L / 2);
    for (int spt = 1; spt <= 4; ++spt)
        if ((PL + spt - 1) / spt <= kSweepMaxThreads) return spt;
    return 0;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}
// global -> this CTA's shared memory; 16-byte aligned addresses, size a multiple of 16
__device__ __forceinline__ void bulk_copy(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < kSweepWaitTries; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}
// order this thread's generic-proxy stores before later bulk copies that read
// or overwrite the same memory: shared and global, or shared memory only
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Counter sizes: the counts of KF steps fit in NLV (energy: 6 bonds per
// colour-1 site) and NLM (spins up: one colour-0 and one colour-1 site per
// step) bits per thread before they are added to the CTA's totals.
template <int SPT>
struct SweepCounts {
    static constexpr int KF = 127 / (6 * SPT);
    static constexpr int NLV = bit_length(6 * SPT * KF);
    static constexpr int NLM = bit_length(2 * SPT * KF);
    static_assert(KF >= 1 && NLV <= 7, "counters of one flush period");
};

template <bool GEN_H, bool ACC_E, bool ACC_M, int SPT>
__global__ void __launch_bounds__(kSweepMaxThreads) stream_sweep_kernel(const __grid_constant__ StreamParams P,
                                                                        long long s) {
    pdl_enter();
    using CN = SweepCounts<SPT>;
    constexpr int NLV = CN::NLV, NLM = CN::NLM, KF = CN::KF;
    const int L = P.L, LH = L / 2, PL = L * LH, LL = L * L;
    const int N = LL * L, NH = N / 2;
    const int gq = blockIdx.x;
    const int w = gq / (P.C * P.Q), c = (gq / P.Q) % P.C, q = gq % P.Q;
    const int tid = threadIdx.x, NT = blockDim.x, lane = tid & 31;
    uint4* const Sq = reinterpret_cast<uint4*>(P.spins) + (size_t)gq * N;  // [colour][NH]
    const uint32_t* const Fw = P.bonds + (size_t)w * 3 * N;             // [dir][colour][NH]

    extern __shared__ __align__(128) uint4 ring[];  // [colour][kSweepSlots][PL]
    __shared__ __align__(8) uint64_t bar[2];
    __shared__ int sE[4][32], sM[4][32];
    __shared__ uint4 sThr[4][2];
    // ring slot of plane index u >= -1 of colour p (u may pass L - 1: the
    // planes of the wrap-around are read again from global memory)
    auto slot = [&](int p, int u) {
        return ring + (size_t)(p * kSweepSlots + (u + kSweepSlots) % kSweepSlots) * PL;
    };
    auto plane = [&](int p, int u) { return Sq + (size_t)p * NH + (size_t)((u + L) % L) * PL; };
    const uint32_t bytes = (uint32_t)PL * 16;

    if (tid == 0) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int i = tid; i < 4 * 32; i += NT) {
        (&sE[0][0])[i] = 0;
        (&sM[0][0])[i] = 0;
    }
    if constexpr (GEN_H)
        if (tid < 4) gen_thresholds(P.tab, 4 * q + tid, sThr[tid][0], sThr[tid][1]);
    __syncthreads();
    if (tid == 0) {  // the planes of step 0: colour 0 at 0, colour 1 at -1, 0, 1
        mbar_arrive_expect(&bar[0], 4 * bytes);
        bulk_copy(slot(0, 0), plane(0, 0), bytes, &bar[0]);
        bulk_copy(slot(1, -1), plane(1, -1), bytes, &bar[0]);
        bulk_copy(slot(1, 0), plane(1, 0), bytes, &bar[0]);
        bulk_copy(slot(1, 1), plane(1, 1), bytes, &bar[0]);
    }

    // this thread's sites of a z-plane: in-plane index i = y * L/2 + h
    int si[SPT], dxA[SPT], dxB[SPT], dyM[SPT], dyP[SPT], ybit[SPT];
    uint32_t sbase[SPT];  // Philox word 0 of the site in plane 0, without x & 1
#pragma unroll
    for (int k = 0; k < SPT; ++k) {
        const int i = tid + k * NT;
        const int y = i / LH, h = i - y * LH;
        si[k] = i < PL ? i : -1;
        dxA[k] = h == 0 ? LH - 1 : -1;           // x-1 of a site with x = 2h
        dxB[k] = h == LH - 1 ? -(LH - 1) : 1;    // x+1 of a site with x = 2h+1
        dyM[k] = y == 0 ? (L - 1) * LH : -LH;
        dyP[k] = y == L - 1 ? -(L - 1) * LH : LH;
        ybit[k] = y & 1;
        sbase[k] = (uint32_t)(y * L + 2 * h);
    }
    uint32_t th0[4], th1[4], th2[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int t = 4 * q + k;
        th0[k] = P.tab.thr[t][0][0];
        th1[k] = P.tab.thr[t][0][1];
        th2[k] = P.tab.thr[t][0][2];
    }
    const uint32_t ctr3 = kTagSweep | ((uint32_t)c << 8) | (uint32_t)q;
    const PhiloxFixed pf = philox_fix((uint32_t)s, (uint32_t)w + P.word0, ctr3, P.k0, P.k1);

    uint32_t ecnt[4][NLV], mcnt[4][NLM];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int l = 0; l < NLV; ++l) ecnt[k][l] = 0;
#pragma unroll
        for (int l = 0; l < NLM; ++l) mcnt[k][l] = 0;
    }
    // the counts of the last period into the CTA's per-plane totals (every
    // thread of every warp takes part)
    auto flush = [&]() {
        if constexpr (ACC_E) {
            int cnt[4];
            packed_column_counts<NLV>(ecnt, lane, cnt);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                atomicAdd(&sE[k][lane], cnt[k]);
#pragma unroll
                for (int l = 0; l < NLV; ++l) ecnt[k][l] = 0;
            }
        }
        if constexpr (ACC_M) {
            int cnt[4];
            packed_column_counts<NLM>(mcnt, lane, cnt);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                atomicAdd(&sM[k][lane], cnt[k]);
#pragma unroll
                for (int l = 0; l < NLM; ++l) mcnt[k][l] = 0;
            }
        }
    };
    auto count_up = [&](const uint4 v) {
        if constexpr (ACC_M) {
            const uint32_t x[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                uint32_t carry = x[k];
#pragma unroll
                for (int l = 0; l < NLM; ++l) {
                    const uint32_t t = mcnt[k][l] & carry;
                    mcnt[k][l] ^= carry;
                    carry = t;
                }
            }
        }
    };

    // One site of colour p in plane zp: own word cv, the other colour's
    // planes below (om), at (oc) and above (op) in the ring; bonds of the
    // site's colour (Fc) and of the other (Fo).  Returns the new word;
    // wd receives the post-flip full-adder words (energy counters).
    auto update = [&](const int k, const int p, const int zp, const uint4 cv, const uint4* oc,
                      const uint4* om, const uint4* op, uint32_t (&wd)[4][4]) {
        const int i = si[k];
        const int o = ybit[k] ^ (zp & 1) ^ p;  // x & 1 of the site
        const int xm = o ? 0 : dxA[k], xp = o ? dxB[k] : 0;
        const uint32_t* Fc = Fw + p * NH + zp * PL + i;
        const uint32_t* Fo = Fw + (1 - p) * NH + zp * PL + i;
        const int zmo = (zp == 0 ? L - 1 : -1) * PL;  // z-1 of the site, relative
        const uint4 a0 = oc[i + xm], a1 = oc[i + xp], a2 = oc[i + dyM[k]], a3 = oc[i + dyP[k]];
        const uint4 a4 = om[i], a5 = op[i];
        const uint32_t f0 = __ldg(Fo + xm), f1 = __ldg(Fc);
        const uint32_t f2 = __ldg(Fo + N + dyM[k]), f3 = __ldg(Fc + N);
        const uint32_t f4 = __ldg(Fo + 2 * N + zmo), f5 = __ldg(Fc + 2 * N);
        const u32x4 r = philox_c0((uint32_t)(zp * LL) + sbase[k] + (uint32_t)o, pf);
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
                fl = flip_gen(s0, sa, ca, sb, cb, rr[kq], sThr[kq][0], sThr[kq][1],
                              P.tab.ucut[4 * q + kq][0], P.tab.ucut[4 * q + kq][1]);
            else
                fl = flip_h0(sa, ca, sb, cb, rr[kq], th0[kq], th1[kq], th2[kq]);
            cw[kq] = s0 ^ fl;
            wd[kq][0] = sa ^ fl;
            wd[kq][1] = sb ^ fl;
            wd[kq][2] = ca ^ fl;
            wd[kq][3] = cb ^ fl;
        }
        return make_uint4(cw[0], cw[1], cw[2], cw[3]);
    };

    bool ok = true;
    int z = 0;
    for (; z <= L + 1; ++z) {
        // the planes of step z + 1: colour 0 at z + 1 (up to L + 1) and colour 1
        // at z + 2 (up to L), into slots whose planes were last read in step z - 1
        if (tid == 0) {
            const bool l0 = z + 1 <= L + 1, l1 = z + 2 <= L;
            if (l0 || l1) {
                uint64_t* b = &bar[(z + 1) & 1];
                mbar_arrive_expect(b, (uint32_t)(l0 + l1) * bytes);
                if (l0) bulk_copy(slot(0, z + 1), plane(0, z + 1), bytes, b);
                if (l1) bulk_copy(slot(1, z + 2), plane(1, z + 2), bytes, b);
            }
        }
        // this step's planes (issued in step z - 1, or before the loop)
        if (z <= L + 1 && ok) ok = mbar_wait_bounded(&bar[z & 1], (uint32_t)(z >> 1) & 1);

        if (z < L) {  // colour 0 in plane z
            uint4* const own = slot(0, z);
            const uint4* const om = slot(1, z - 1);
            const uint4* const oc = slot(1, z);
            const uint4* const op = slot(1, z + 1);
            uint4* const g = Sq + (size_t)z * PL;
#pragma unroll
            for (int k = 0; k < SPT; ++k) {
                if (si[k] < 0) continue;
                uint32_t wd[4][4];
                const uint4 nv = update(k, 0, z, own[si[k]], oc, om, op, wd);
                own[si[k]] = nv;
                g[si[k]] = nv;
                count_up(nv);
            }
        }
        __syncthreads();  // colour 0 of plane z is in its ring slot
        if (z >= 2) {  // colour 1 in plane v = z - 1 (v = L: plane 0)
            const int v = z - 1, zv = v == L ? 0 : v;
            const uint4* const own = slot(1, v);
            const uint4* const om = slot(0, v - 1);
            const uint4* const oc = slot(0, v);
            const uint4* const op = slot(0, v + 1);
            uint4* const g = Sq + (size_t)NH + (size_t)zv * PL;
            uint32_t wa[4][4], wb[4][4];
#pragma unroll
            for (int k = 0; k < SPT; ++k) {
                uint32_t(&wd)[4][4] = (k & 1) ? wb : wa;
                if (si[k] >= 0) {
                    const uint4 nv = update(k, 1, zv, own[si[k]], oc, om, op, wd);
                    g[si[k]] = nv;
                    count_up(nv);
                } else {  // padding site: counts nothing
#pragma unroll
                    for (int kq = 0; kq < 4; ++kq)
#pragma unroll
                        for (int b = 0; b < 4; ++b) wd[kq][b] = 0;
                }
                if constexpr (ACC_E) {
                    if (k & 1) {  // sites k - 1 and k
#pragma unroll
                        for (int kq = 0; kq < 4; ++kq)
                            vc_add_2sites<NLV>(ecnt[kq], wa[kq][0], wa[kq][1], wa[kq][2], wa[kq][3],
                                               wb[kq][0], wb[kq][1], wb[kq][2], wb[kq][3]);
                    } else if (k == SPT - 1) {  // the last of an odd number
#pragma unroll
                        for (int kq = 0; kq < 4; ++kq)
                            vc_add_site<NLV>(ecnt[kq], wa[kq][0], wa[kq][1], wa[kq][2], wa[kq][3]);
                    }
                }
            }
        }
        if ((z + 1) % KF == 0) flush();
        // stores of this step before the bulk copies that later overwrite its
        // ring slots or (colour 0 of planes 0 and 1) read them back from global
        // memory; all reads of this step before the next step's copies land
        if (z < 2)
            fence_proxy_async();
        else
            fence_proxy_async_smem();
        if (__syncthreads_or(!ok)) break;
    }
    if (__syncthreads_or(!ok)) {
        // a wait gave up: report it, let the copies still in flight land
        // (bounded), and leave the totals alone
        if (tid == 0) {  // the step that gave up, and the copies it issued for the next
            atomicExch(P.err, 1);
            mbar_wait_bounded(&bar[z & 1], (uint32_t)(z >> 1) & 1);
            if (z + 1 <= L + 1) mbar_wait_bounded(&bar[(z + 1) & 1], (uint32_t)((z + 1) >> 1) & 1);
        }
        __syncthreads();
        return;
    }
    flush();
    __syncthreads();
    for (int i = tid; i < 4 * 32; i += NT) {  // a CTA may be a single warp
        const int k = i >> 5, b = i & 31;
        const size_t o = (((size_t)w * P.C + c) * P.T + 4 * q + k) * 32 + b;
        if constexpr (ACC_E) atomicAdd(&P.u_acc[o], sE[k][b]);
        if constexpr (ACC_M) atomicAdd(&P.up_acc[o], sM[k][b]);
    }
}

template <bool G, bool E, bool M, int SPT>
cudaError_t launch_one(const StreamParams& P, long long s, cudaStream_t st) {
    auto* kernel = stream_sweep_kernel<G, E, M, SPT>;
    // set on every launch: the attribute belongs to the current device
    const cudaError_t attr = cudaFuncSetAttribute(
        kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSweepMaxSmem);
    if (attr != cudaSuccess) return attr;
    int nt = 0, smem = 0;
    stream_sweep_shape(P.L, &nt, &smem);
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3((unsigned)(P.W * P.C * P.Q));
    lc.blockDim = dim3((unsigned)nt);
    lc.dynamicSmemBytes = (size_t)smem;
    lc.stream = st;
    // the smallest shared-memory carve-out that holds the ring (plus the
    // static part and the 1 KB per-CTA reserve): the rest of the SM's 256 KB
    // stays L1 for the bonds, each of which is read in two consecutive steps
    cudaLaunchAttribute a[2];
    a[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    a[0].val.programmaticStreamSerializationAllowed = 1;
    a[1].id = cudaLaunchAttributePreferredSharedMemoryCarveout;
    a[1].val.sharedMemCarveout =
        (unsigned)std::min<size_t>(100, ((size_t)smem + 4096) * 100 / (228 * 1024) + 1);
    lc.attrs = a;
    lc.numAttrs = 2;
    return cudaLaunchKernelEx(&lc, kernel, P, s);
}

template <bool G, bool E, bool M>
cudaError_t launch_spt(const StreamParams& P, long long s, cudaStream_t st) {
    switch (sweep_spt(P.L)) {
        case 1: return launch_one<G, E, M, 1>(P, s, st);
        case 2: return launch_one<G, E, M, 2>(P, s, st);
        case 3: return launch_one<G, E, M, 3>(P, s, st);
        case 4: return launch_one<G, E, M, 4>(P, s, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

bool stream_sweep_fits(int L) {
    return L >= 4 && L % 2 == 0 && sweep_spt(L) > 0 && sweep_smem_bytes(L) <= kSweepMaxSmem;
}

void stream_sweep_shape(int L, int* threads, int* smem_bytes) {
    const bool fits = stream_sweep_fits(L);
    const int spt = fits ? sweep_spt(L) : 1, PL = L * (L / 2);
    if (threads) *threads = fits ? ((PL + spt - 1) / spt + 31) / 32 * 32 : 0;
    if (smem_bytes) *smem_bytes = fits ? (int)sweep_smem_bytes(L) : 0;
}

cudaError_t launch_stream_sweep(const StreamParams& P, long long s, bool gen, bool acc_e, bool acc_m,
                                cudaStream_t st) {
    using Fn = cudaError_t (*)(const StreamParams&, long long, cudaStream_t);
    static const Fn fns[8] = {launch_spt<false, false, false>, launch_spt<false, false, true>,
                              launch_spt<false, true, false>,  launch_spt<false, true, true>,
                              launch_spt<true, false, false>,  launch_spt<true, false, true>,
                              launch_spt<true, true, false>,   launch_spt<true, true, true>};
    if (!stream_sweep_fits(P.L)) return cudaErrorInvalidValue;
    return fns[(gen ? 4 : 0) + (acc_e ? 2 : 0) + (acc_m ? 1 : 0)](P, s, st);
}

}  // namespace csg
