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
// until the process exits.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "csg.h"
#include "engine_internal.h"

using csg_detail::fail;  // reported by csg_last_error()

namespace {

// 16 MiB of int32: W*T*32*(5 + 3L) integers per call must fit.
constexpr size_t kScratchInts = (size_t)4 << 20;
static __device__ __align__(256) int g_obs_scratch[kScratchInts];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
int* g_scratch_ptr[kMaxDevices] = {};

// The integers of one (word, temperature) pair, lane b = sample 32w+b:
// bond energy and magnetisation of both copies, number of sites where the
// copies differ, and that number per coordinate plane (3L values).  One warp
// per pair; every output element is written, so nothing needs clearing.
__global__ void obs_integers_kernel(const uint32_t* __restrict__ spins,
                                    const uint32_t* __restrict__ bonds, int L, int W, int T,
                                    int* __restrict__ out) {
    extern __shared__ int sh[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair = blockIdx.x * (blockDim.x >> 5) + warp;
    const int Q = T / 4, stride = 5 + 3 * L;
    const long N = (long)L * L * L, NH = N / 2;
    int* cnt = sh + warp * 3 * L * 32;
    for (int k = lane; k < 3 * L * 32; k += 32) cnt[k] = 0;
    __syncwarp();
    if (pair >= W * T) return;
    const int w = pair / T, t = pair - w * T;
    auto spin = [&](int c, long slot) {
        return spins[((((long)w * 2 + c) * Q + (t >> 2)) * N + slot) * 4 + (t & 3)];
    };
    auto slot = [&](int x, int y, int z) {
        return (long)((x + y + z) & 1) * NH + (long)(z * L + y) * (L / 2) + (x >> 1);
    };
    int unsat[2] = {0, 0}, up[2] = {0, 0}, diff = 0;
    for (int z = 0; z < L; ++z)
        for (int y = 0; y < L; ++y)
            for (int x = 0; x < L; ++x) {
                const long si = slot(x, y, z);
                const long nb[3] = {slot(x + 1 == L ? 0 : x + 1, y, z),
                                    slot(x, y + 1 == L ? 0 : y + 1, z),
                                    slot(x, y, z + 1 == L ? 0 : z + 1)};
                uint32_t s[2];
                for (int c = 0; c < 2; ++c) {
                    s[c] = spin(c, si);
                    up[c] += (s[c] >> lane) & 1u;
                    for (int k = 0; k < 3; ++k)
                        unsat[c] += ((s[c] ^ spin(c, nb[k]) ^ bonds[((long)w * 3 + k) * N + si]) >>
                                     lane) & 1u;
                }
                if (((s[0] ^ s[1]) >> lane) & 1u) {
                    ++diff;
                    cnt[(0 * L + x) * 32 + lane] += 1;
                    cnt[(1 * L + y) * 32 + lane] += 1;
                    cnt[(2 * L + z) * 32 + lane] += 1;
                }
            }
    int* o = out + ((long)pair * 32 + lane) * stride;
    o[0] = 2 * unsat[0] - 3 * (int)N;
    o[1] = 2 * unsat[1] - 3 * (int)N;
    o[2] = 2 * up[0] - (int)N;
    o[3] = 2 * up[1] - (int)N;
    o[4] = diff;
    for (int k = 0; k < 3 * L; ++k) o[5 + k] = cnt[k * 32 + lane];
}

// Records {e[2], m[2], q_0, q_1_r[3], q_1_i[3]} from the integers, with the
// float arithmetic of csg_obs_records (eamsim.cu:320-325, 477-509).
__global__ void obs_records_kernel(const int* __restrict__ in, int L, int W, int T, float H,
                                   float* __restrict__ rec) {
    const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long)W * T * 32) return;
    const int b = (int)(i & 31);
    const long pair = i >> 5;
    const int w = (int)(pair / T), t = (int)(pair - (long)w * T);
    const int stride = 5 + 3 * L;
    const int* v = in + i * stride;
    const long N = (long)L * L * L;
    float* o = rec + (((long)(32 * w + b)) * T + t) * 11;
    for (int c = 0; c < 2; ++c) {
        const float es = (float)(-v[c]);
        const float ms = (float)v[2 + c];
        o[c] = -(es + H * ms) / (float)N;
        o[2 + c] = ms / (float)N;
    }
    o[4] = (float)(N - 2 * (long)v[4]) / (float)N;
    const double k = 2.0 * M_PI / L;
    for (int dir = 0; dir < 3; ++dir) {
        double re = 0.0, im = 0.0;
        for (int a = 0; a < L; ++a) {
            const long P = (long)L * L - 2 * (long)v[5 + dir * L + a];
            re += (double)P * cos(k * a);
            im += (double)P * sin(k * a);
        }
        o[5 + dir] = (float)(re / (double)N);
        o[8 + dir] = (float)(im / (double)N);
    }
}

// Device address of the scratch array on the current device, looked up once
// per device (the symbol name is only a host-side handle).
int scratch_for_current_device(int** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(CSG_ERR_UNSUPPORTED, "device index too large");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_ptr[dev]) {
        int* p = nullptr;
        e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_obs_scratch);
        if (e != cudaSuccess || !p)
            return fail(CSG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_ptr[dev] = p;
    }
    *out = g_scratch_ptr[dev];
    return CSG_OK;
}

}  // namespace

extern "C" {

int csg_obs_records_noalloc(const csg_config* cfg, const uint32_t* spins, const uint32_t* bonds,
                            float* rec, size_t n_floats, void* stream) {
    if (!cfg || !spins || !bonds || !rec) return fail(CSG_ERR_ARG, "null argument");
    const csg_dims& d = cfg->dims;
    if (d.L < 4 || d.L > 24 || d.L % 2 || d.n_words < 1 || d.n_temps < 4 || d.n_temps > 64 ||
        d.n_temps % 4)
        return fail(CSG_ERR_ARG, "invalid dimensions");
    if (d.n_copies != 2) return fail(CSG_ERR_UNSUPPORTED, "observable records need two copies");
    const int L = d.L, W = d.n_words, T = d.n_temps;
    if (n_floats != (size_t)32 * W * T * 11) return fail(CSG_ERR_ARG, "record buffer size mismatch");
    const size_t need = (size_t)W * T * 32 * (5 + 3 * (size_t)L);
    if (need > kScratchInts)
        return fail(CSG_ERR_UNSUPPORTED,
                    "state too large for the fixed 16 MiB scratch: W*T*32*(5+3L) = " +
                        std::to_string(need) + " ints > " + std::to_string(kScratchInts));
    int* scratch = nullptr;
    if (int rc = scratch_for_current_device(&scratch)) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int warps = 4;
    const unsigned blocks = (unsigned)((W * T + warps - 1) / warps);
    obs_integers_kernel<<<blocks, warps * 32, (size_t)warps * 32 * 3 * L * sizeof(int), st>>>(
        spins, bonds, L, W, T, scratch);
    const long total = (long)W * T * 32;
    obs_records_kernel<<<(unsigned)((total + 127) / 128), 128, 0, st>>>(scratch, L, W, T,
                                                                        (float)cfg->H, rec);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return CSG_OK;
}

}  // extern "C"
