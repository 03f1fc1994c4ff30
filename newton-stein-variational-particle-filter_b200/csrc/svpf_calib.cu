// svpf_calib.cu -- measured issue rates of the two pipes the pair sweeps run
// on: the MUFU unit (ex2.approx and rcp.approx, one of each per
// pair-iteration) and the FP32 pipe (packed FFMA2).  One CTA of 1024 threads
// per SM (a shared-memory request above half an SM keeps a second CTA off),
// eight independent dependency chains per thread, cycles counted per CTA with
// clock64, so the rates are per SM clock whatever the clock is.
#include <algorithm>
#include <vector>

#include "svpf_device.cuh"
#include "svpf_internal.h"

namespace svpf {
namespace {

constexpr int kCalThreads = 1024;
constexpr int kCalIters = 4096;
constexpr int kCalChains = 8;
constexpr int kCalSmem = 120 * 1024;   // > half of an SM's shared memory: one CTA per SM

__device__ __forceinline__ unsigned int sm_id() {
    unsigned int r;
    asm volatile("mov.u32 %0, %%smid;" : "=r"(r));
    return r;
}

// MUFU: chains alternate ex2(-a) (values in (0.36, 1]) and rcp(1 + a)
// (values in (0.5, 1)); 8 MUFU results per thread and iteration.
__global__ void __launch_bounds__(kCalThreads, 1) mufu_rate_kernel(float* sink, long long* cycles,
                                                                   unsigned int* smid) {
    float a[kCalChains];
#pragma unroll
    for (int k = 0; k < kCalChains; ++k) a[k] = 0.5f + 0.01f * (float)(threadIdx.x & 7) + 0.001f * (float)k;
    __syncthreads();
    const long long t0 = clock64();
    for (int it = 0; it < kCalIters; ++it) {
#pragma unroll
        for (int k = 0; k < kCalChains; k += 2) {
            a[k] = ex2_approx(-a[k]);
            a[k + 1] = rcp_approx(1.0f + a[k + 1]);
        }
    }
    __syncthreads();
    const long long t1 = clock64();
    if (threadIdx.x == 0) {
        cycles[blockIdx.x] = t1 - t0;
        smid[blockIdx.x] = sm_id();
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kCalChains; ++k) s += a[k];
    if (s == -1.0f) sink[threadIdx.x] = s;   // never true: keeps the chains live
}

// FP32: packed FFMA2 chains a = a * 0.999 + 0.001 (bounded); 16 FP32 results
// per thread and iteration.
__global__ void __launch_bounds__(kCalThreads, 1) fp32_rate_kernel(float* sink, long long* cycles,
                                                                   unsigned int* smid) {
    float2 a[kCalChains];
#pragma unroll
    for (int k = 0; k < kCalChains; ++k) a[k] = f2(0.5f + 0.01f * (float)(threadIdx.x & 7) + 0.001f * (float)k);
    const float2 m = f2(0.999f), c = f2(0.001f);
    __syncthreads();
    const long long t0 = clock64();
    for (int it = 0; it < kCalIters; ++it) {
#pragma unroll
        for (int k = 0; k < kCalChains; ++k) a[k] = fma2(a[k], m, c);
    }
    __syncthreads();
    const long long t1 = clock64();
    if (threadIdx.x == 0) {
        cycles[blockIdx.x] = t1 - t0;
        smid[blockIdx.x] = sm_id();
    }
    float s = 0.0f;
#pragma unroll
    for (int k = 0; k < kCalChains; ++k) s += a[k].x + a[k].y;
    if (s == -1.0f) sink[threadIdx.x] = s;
}

// Runs one of the kernels on every SM; the median over SMs of results per
// SM clock.  Returns a negative rate when the placement was not one CTA per SM.
template <class K>
cudaError_t pipe_rate(K kernel, double results_per_cta, double* rate) {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kCalSmem);
    if (e != cudaSuccess) return e;
    float* sink = nullptr;
    long long* cyc = nullptr;
    unsigned int* sid = nullptr;
    if ((e = cudaMalloc(&sink, kCalThreads * sizeof(float))) != cudaSuccess) return e;
    if ((e = cudaMalloc(&cyc, sms * sizeof(long long))) != cudaSuccess) {
        cudaFree(sink);
        return e;
    }
    if ((e = cudaMalloc(&sid, sms * sizeof(unsigned int))) != cudaSuccess) {
        cudaFree(sink);
        cudaFree(cyc);
        return e;
    }
    std::vector<long long> hc(sms);
    std::vector<unsigned int> hs(sms);
    for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {   // the first launch warms up
        kernel<<<sms, kCalThreads, kCalSmem>>>(sink, cyc, sid);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    if (e == cudaSuccess) e = cudaMemcpy(hc.data(), cyc, sms * sizeof(long long), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(hs.data(), sid, sms * sizeof(unsigned int), cudaMemcpyDeviceToHost);
    cudaFree(sink);
    cudaFree(cyc);
    cudaFree(sid);
    if (e != cudaSuccess) return e;
    std::vector<unsigned int> sorted_ids = hs;
    std::sort(sorted_ids.begin(), sorted_ids.end());
    const bool one_per_sm = std::adjacent_find(sorted_ids.begin(), sorted_ids.end()) == sorted_ids.end();
    std::sort(hc.begin(), hc.end());
    const double med = (double)hc[sms / 2];
    *rate = (one_per_sm && med > 0.0) ? results_per_cta / med : -1.0;
    return cudaSuccess;
}

}  // namespace
}  // namespace svpf

extern "C" int svpf_measure_pipe_rates(double* mufu_per_clk_sm, double* fp32_per_clk_sm) {
    using namespace svpf;
    if (!mufu_per_clk_sm || !fp32_per_clk_sm) return SVPF_ERR_INVALID_ARG;
    const double per_thread = (double)kCalIters * kCalChains;
    cudaError_t e = pipe_rate(mufu_rate_kernel, per_thread * kCalThreads, mufu_per_clk_sm);
    if (e == cudaSuccess) e = pipe_rate(fp32_rate_kernel, 2.0 * per_thread * kCalThreads, fp32_per_clk_sm);
    if (e != cudaSuccess) return SVPF_ERR_CUDA;
    return (*mufu_per_clk_sm > 0.0 && *fp32_per_clk_sm > 0.0) ? SVPF_OK : SVPF_ERR_UNSUPPORTED;
}
