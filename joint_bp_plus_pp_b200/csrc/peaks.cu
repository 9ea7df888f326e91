// Measured throughput of the special-function unit (MUFU) for the operations the BP kernels
// use -- ex2, lg2 and rcp in FP32 (approx, flush-to-zero), the roofline of the trial-resident
// and table-driven kernels, which are bound by these and by instruction issue, not by HBM.
// Every thread runs 8 independent chains of one operation, so the unit, not the latency of a
// chain, sets the pace; the grid fills every SM.
#include <cuda_runtime.h>

#include <string>

#include "../../include/jbp_b200.h"
#include "ctx.hpp"

namespace {

constexpr int kChains = 8;

template <int OP>
__device__ __forceinline__ float sfu_step(float x) {
    float y;
    if (OP == 0) {
        asm volatile("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(-x));        // x -> 2^-x, stays in (0, 1]
    } else if (OP == 1) {
        asm volatile("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x + 3.0f));  // stays in [1.58, 2.3]
    } else {
        asm volatile("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x + 1.5f));  // stays in (0.3, 0.67)
    }
    return y;
}

template <int OP>
__global__ void k_sfu_peak(float *sink, int iters) {
    float x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = 0.5f + 0.01f * (threadIdx.x & 31) + 0.001f * c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = sfu_step<OP>(x[c]);
    }
    float s = 0.0f;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (s == 12345.0f) sink[blockIdx.x] = s;   // keeps the chains live; never true in practice
}

template <int OP>
std::string time_op(int sms, float *sink, double *gops) {
    const int threads = 256, blocks = sms * 8, iters = 2048;
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return "cudaEventCreate";
    k_sfu_peak<OP><<<blocks, threads>>>(sink, iters);   // warm-up
    float best = 1e30f;
    for (int r = 0; r < 3; ++r) {
        cudaEventRecord(a);
        k_sfu_peak<OP><<<blocks, threads>>>(sink, iters);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, a, b);
        if (ms < best) best = ms;
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cudaGetErrorString(e);
    *gops = static_cast<double>(blocks) * threads * iters * kChains / (best * 1e-3) / 1e9;
    return "";
}

}  // namespace

extern "C" int jbp_measure_sfu(int device, double *ex2_gops, double *lg2_gops, double *rcp_gops) {
    if (cudaSetDevice(device) != cudaSuccess) return jbp::set_last_error(JBP_ERR_CUDA, "cudaSetDevice failed");
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return jbp::set_last_error(JBP_ERR_CUDA, "device attributes");
    float *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(float) * sms * 8) != cudaSuccess)
        return jbp::set_last_error(JBP_ERR_CUDA, "cudaMalloc(sink)");
    double r[3] = {0.0, 0.0, 0.0};
    std::string e = time_op<0>(sms, sink, &r[0]);
    if (e.empty()) e = time_op<1>(sms, sink, &r[1]);
    if (e.empty()) e = time_op<2>(sms, sink, &r[2]);
    cudaFree(sink);
    if (!e.empty()) return jbp::set_last_error(JBP_ERR_CUDA, "SFU measurement: " + e);
    if (ex2_gops) *ex2_gops = r[0];
    if (lg2_gops) *lg2_gops = r[1];
    if (rcp_gops) *rcp_gops = r[2];
    return JBP_OK;
}
