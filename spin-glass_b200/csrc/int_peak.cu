// int_peak.cu — microbenchmark of the SM integer logic pipe (libcsg_peak.so).
//
// The sweep kernel is bound by 32-bit logic instructions; the driver-measured
// peaks cover HBM copies and bf16 tensor GEMMs only.  This kernel issues
// independent LOP3 instructions (8 chains per thread, no memory traffic) over
// every SM and reports the sustained LOP3 rate, the denominator of the
// integer-pipe roofline.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

__global__ void lop3_chains(uint32_t* out, int iters) {
    uint32_t a[8], b[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        a[k] = threadIdx.x * 2654435761u + k * 40503u + blockIdx.x;
        b[k] = (a[k] << 7) ^ 0x9E3779B9u;
    }
    const uint32_t c = blockIdx.x * 977u;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 16; ++r)
#pragma unroll
            for (int k = 0; k < 8; ++k)
                asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[k]) : "r"(b[k]), "r"(c));
    }
    uint32_t x = 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) x ^= a[k];
    if (x == 0x12345678u) out[blockIdx.x * blockDim.x + threadIdx.x] = x;
}

}  // namespace

// LOP3 instructions per second summed over all SMs (best of `reps` runs).
extern "C" int csg_int_peak(double* ops_per_s, int reps) {
    int dev = 0, nsm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 1;
    const int threads = 512, blocks = nsm * 4, iters = 4096;
    uint32_t* out = nullptr;
    if (cudaMalloc(&out, (size_t)threads * blocks * 4) != cudaSuccess) return 1;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    lop3_chains<<<blocks, threads>>>(out, 64);  // warm-up
    double best = 0.0;
    for (int r = 0; r < reps; ++r) {
        cudaEventRecord(e0);
        lop3_chains<<<blocks, threads>>>(out, iters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double ops = (double)blocks * threads * iters * 16.0 * 8.0;
        if (ms > 0.f && ops / (ms * 1e-3) > best) best = ops / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *ops_per_s = best;
    return cudaGetLastError() == cudaSuccess ? 0 : 1;
}
