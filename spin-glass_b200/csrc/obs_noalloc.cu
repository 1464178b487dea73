// obs_noalloc.cu — observable records without any device allocation.
//
// csg_obs_records() allocates temporary device buffers for the per-sample
// integers it reduces the lattice to.  Some callers cannot let a library do
// that: a process that hands all device memory to its own pool (a framework's
// caching allocator, a server that admits work against a fixed memory budget)
// must not see cudaMalloc fail or cudaFree synchronise the device behind its
// back.  csg_obs_records_noalloc() is for them: the caller passes the state and
// the output in its own device memory, and the intermediate integers live in
// one fixed, file-scope device array that every GPU loading libcsg.so keeps
// until the process exits.  The kernels are those of csg_obs_records
// (aux_kernels.cuh), so both entry points give the same records bit for bit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "csg.h"
#include "engine_internal.h"
#include "aux_kernels.cuh"

using csg_detail::fail;  // reported by csg_last_error()

namespace {

// 16 MiB of int32: the integers of a call, W*T*32*(5 + 3L), and the 2L
// doubles of the cos/sin table must fit.
constexpr size_t kScratchInts = (size_t)4 << 20;
static __device__ __align__(256) int g_obs_scratch[kScratchInts];

// Device address of the scratch array on the current device (the symbol name
// is only a host-side handle).  Looked up at every call, so that it stays
// right after the device's context was torn down and made again.
int scratch_for_current_device(int** out) {
    int* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_obs_scratch);
    if (e != cudaSuccess || !p)
        return fail(CSG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = p;
    return CSG_OK;
}

}  // namespace

extern "C" {

int csg_obs_records_noalloc(const csg_config* cfg, const uint32_t* spins, const uint32_t* bonds,
                            float* rec, size_t n_floats, void* stream) {
    if (!cfg || !spins || !bonds || !rec) return fail(CSG_ERR_ARG, "null argument");
    if (int rc = csg_detail::validate(cfg)) return rc;
    const csg_dims& d = cfg->dims;
    if (d.n_copies != 2) return fail(CSG_ERR_UNSUPPORTED, "observable records need two copies");
    const int L = d.L, W = d.n_words, T = d.n_temps;
    if (n_floats != (size_t)32 * W * T * 11) return fail(CSG_ERR_ARG, "record buffer size mismatch");
    // scratch layout (ints): e [W][2][T][32], m (same), d [W][T][32],
    // per-plane d [W][T][32][3L], then the cos/sin table (2L doubles)
    const size_t nE = (size_t)W * 2 * T * 32, nD = (size_t)W * T * 32, nP = nD * 3 * L;
    const size_t o_m = nE, o_d = 2 * nE, o_p = o_d + nD, o_cs = (o_p + nP + 1) & ~(size_t)1;
    const size_t need = o_cs + 4 * (size_t)L;
    if (need > kScratchInts)
        return fail(CSG_ERR_UNSUPPORTED,
                    "state too large for the fixed 16 MiB scratch: W*T*32*(5+3L) + 4L = " +
                        std::to_string(need) + " ints > " + std::to_string(kScratchInts));
    int* scratch = nullptr;
    if (int rc = scratch_for_current_device(&scratch)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    // the L phases exp(i k a), k = 2 pi / L, computed on the host as
    // csg_obs_records does
    const double k = 2.0 * M_PI / L;
    std::vector<double> cs(2 * (size_t)L);
    for (int a = 0; a < L; ++a) {
        cs[a] = std::cos(k * a);
        cs[L + a] = std::sin(k * a);
    }
    double* dcs = reinterpret_cast<double*>(scratch + o_cs);
    cudaError_t e = cudaMemcpyAsync(dcs, cs.data(), cs.size() * sizeof(double),
                                    cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("table copy: ") + cudaGetErrorString(e));
    // 3L counters per lane; as many warps as fit in 48 KB (4 up to L = 32)
    const size_t per_warp = (size_t)32 * 3 * L * sizeof(int);
    const int warps = (int)std::max<size_t>(1, std::min<size_t>(4, 49152 / per_warp));
    int* de = scratch;
    int* dm = scratch + o_m;
    int* dd = scratch + o_d;
    int* dp = scratch + o_p;
    // each launch is checked on its own (an error left by the caller's earlier
    // work stays theirs)
    {
        void* args[] = {&spins, &bonds, (void*)&L, (void*)&W, (void*)&T, &de, &dm, &dd, &dp};
        e = cudaLaunchKernel(reinterpret_cast<const void*>(csg::measure_kernel),
                             dim3((unsigned)((W * T + warps - 1) / warps)), dim3(warps * 32), args,
                             (size_t)warps * per_warp, st);
    }
    if (e != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    {
        const long total = (long)W * 32 * T;
        const double* dc = dcs;
        const double* dsn = dcs + L;
        const float H = (float)cfg->H;
        void* args[] = {&de, &dm, &dd, &dp, &dc, &dsn, (void*)&L, (void*)&W, (void*)&T,
                        (void*)&H, &rec};
        e = cudaLaunchKernel(reinterpret_cast<const void*>(csg::records_kernel),
                             dim3((unsigned)((total + 127) / 128)), dim3(128), args, 0, st);
    }
    if (e != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return CSG_OK;
}

}  // extern "C"
