// analysis_kernels.cu — the result table of a record series on the GPU.
//
// Restates the estimators of the reference's analyze-all.py (lines 38-71) as a
// two-kernel reduction over records already in device memory: per (sample,
// temperature) thermal sums over the measurements, then per temperature the
// disorder mean and variance of every sum (two passes, double precision).  The
// host forms chi_0, xi_L/L, e, m and their errors from those moments with the
// script's formulas.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "csg.h"
#include "engine_internal.h"

using csg_detail::fail;  // reported by csg_last_error()

namespace {

constexpr int kRecFloats = 11;  // obs_s: e[2], m[2], q_0, q_1_r[3], q_1_i[3]
constexpr int kSums = 9;        // q_0^2, q_1_r[a]^2 (3), q_1_i[a]^2 (3), e (both copies), m

// Thermal sums of one (sample, temperature) over the measurements.
__global__ void thermal_sums_kernel(const float* __restrict__ rec, long long n_meas, int n_pairs,
                                    double* __restrict__ sums) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_pairs) return;
    double acc[kSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (long long m = 0; m < n_meas; ++m) {
        const float* v = rec + ((size_t)m * n_pairs + i) * kRecFloats;
        const double q0 = v[4];
        acc[0] += q0 * q0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const double qr = v[5 + a], qi = v[8 + a];
            acc[1 + a] += qr * qr;
            acc[4 + a] += qi * qi;
        }
        acc[7] += (double)v[0] + (double)v[1];
        acc[8] += (double)v[2] + (double)v[3];
    }
#pragma unroll
    for (int k = 0; k < kSums; ++k) sums[(size_t)i * kSums + k] = acc[k];
}

// Disorder mean and variance (population, like numpy's var) of each thermal
// mean, per temperature: blockIdx.x = temperature.
__global__ void disorder_moments_kernel(const double* __restrict__ sums, int ndis, int nrep,
                                        double n_meas, double* __restrict__ moments) {
    const int r = blockIdx.x;
    __shared__ double red[kSums][256];
    __shared__ double mean[kSums];
    // the thermal mean of e and m is over measurements and both copies
    auto value = [&](int d, int k) {
        const double v = sums[((size_t)d * nrep + r) * kSums + k] / n_meas;
        return k >= 7 ? v / 2.0 : v;
    };
    double s[kSums] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int d = threadIdx.x; d < ndis; d += blockDim.x)
#pragma unroll
        for (int k = 0; k < kSums; ++k) s[k] += value(d, k);
#pragma unroll
    for (int k = 0; k < kSums; ++k) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
#pragma unroll
            for (int k = 0; k < kSums; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < kSums) mean[threadIdx.x] = red[threadIdx.x][0] / ndis;
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSums; ++k) s[k] = 0.0;
    for (int d = threadIdx.x; d < ndis; d += blockDim.x)
#pragma unroll
        for (int k = 0; k < kSums; ++k) {
            const double x = value(d, k) - mean[k];
            s[k] += x * x;
        }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < kSums; ++k) red[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int h = blockDim.x / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
#pragma unroll
            for (int k = 0; k < kSums; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < kSums) {
        moments[((size_t)r * 2 + 0) * kSums + threadIdx.x] = mean[threadIdx.x];
        moments[((size_t)r * 2 + 1) * kSums + threadIdx.x] = red[threadIdx.x][0] / ndis;
    }
}

}  // namespace

extern "C" {

int csg_analyze_records(const float* rec, int64_t n_meas, int32_t ndis, int32_t nrep, int32_t L,
                        double* table, void* stream) {
    if (!rec || !table) return fail(CSG_ERR_ARG, "null argument");
    if (n_meas < 1 || ndis < 1 || nrep < 1 || L < 4) return fail(CSG_ERR_ARG, "invalid dimensions");
    cudaStream_t st = (cudaStream_t)stream;
    const int n_pairs = ndis * nrep;
    double* dev = nullptr;
    const size_t n_sums = (size_t)n_pairs * kSums, n_mom = (size_t)nrep * 2 * kSums;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&dev), (n_sums + n_mom) * sizeof(double), st);
    if (e != cudaSuccess) return fail(CSG_ERR_NOMEM, std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
    thermal_sums_kernel<<<(n_pairs + 255) / 256, 256, 0, st>>>(rec, n_meas, n_pairs, dev);
    disorder_moments_kernel<<<nrep, 256, 0, st>>>(dev, ndis, nrep, (double)n_meas, dev + n_sums);
    std::vector<double> mom(n_mom);
    e = cudaGetLastError();
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(mom.data(), dev + n_sums, n_mom * sizeof(double), cudaMemcpyDeviceToHost, st);
    const cudaError_t e2 = cudaFreeAsync(dev, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("analysis: ") + cudaGetErrorString(e));
    if (e2 != cudaSuccess) return fail(CSG_ERR_CUDA, std::string("cudaFreeAsync: ") + cudaGetErrorString(e2));
    // analyze-all.py:52-71, from the disorder moments
    const double pi = 3.14159265358979323846;
    for (int r = 0; r < nrep; ++r) {
        const double* mu = &mom[((size_t)r * 2 + 0) * kSums];
        const double* va = &mom[((size_t)r * 2 + 1) * kSums];
        const double chi0 = mu[0], chi0_v = va[0];
        double chi1 = 0.0, chi1_v = 0.0;
        for (int a = 0; a < 3; ++a) {
            chi1 += mu[1 + a] + mu[4 + a];
            chi1_v += va[1 + a] + va[4 + a];
        }
        chi1 /= 3.0;
        chi1_v /= 3.0;
        const double chif = chi0 / chi1;
        const double chif_v = chif * chif * (chi0_v / (chi0 * chi0) + chi1_v / (chi1 * chi1));
        const double xi = std::sqrt(chif - 1.0) / (2.0 * std::sin(pi / L)) / L;
        const double xi_f = xi / (2.0 * (chif - 1.0));
        const double xi_v = xi_f * xi_f * chif_v;
        double* o = table + (size_t)r * 8;
        o[0] = chi0;
        o[1] = std::sqrt(chi0_v / ndis);
        o[2] = xi;
        o[3] = std::sqrt(xi_v / ndis);
        o[4] = mu[7];
        o[5] = std::sqrt(va[7] / ndis);
        o[6] = mu[8];
        o[7] = std::sqrt(va[8] / ndis);
    }
    return CSG_OK;
}

}  // extern "C"
