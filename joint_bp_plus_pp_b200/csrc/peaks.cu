// Measured throughput of the special-function unit (MUFU) for the operations the BP kernels
// use -- ex2, lg2 and rcp in FP32 (approx, flush-to-zero), the roofline of the trial-resident
// and table-driven kernels, which are bound by these and by instruction issue, not by HBM.
// Every thread runs 8 independent chains of one operation, so the unit, not the latency of a
// chain, sets the pace; the grid fills every SM.  Also the device self-check of the FP64
// kernels' branch-free reciprocal against the division intrinsic, and of the two forms of the
// us-signal oscillation test against the rule as the reference states it.
#include <cuda_runtime.h>

#include <string>

#include "../../include/jbp_b200.h"
#include "ctx.hpp"
#include "kernels_bp.cuh"
#include "kernels_slots.cuh"

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

// Divisor k of the reciprocal self-check: exponent uniform in [-900, 899]; significand random,
// all ones, zero (a power of two), one ulp above it, or just below all ones, by k mod 8.
__device__ double check_divisor(unsigned long long seed, unsigned long long k) {
    unsigned long long h = seed ^ (k * 0x9E3779B97F4A7C15ull);
    auto mix = [&h]() {
        h += 0x9E3779B97F4A7C15ull;
        unsigned long long z = h;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    const unsigned long long e = static_cast<unsigned long long>(-900 + static_cast<int>(mix() % 1800) + 1023) << 52;
    const unsigned long long ones = (1ull << 52) - 1;
    unsigned long long frac;
    switch (k & 7) {
    case 0: frac = ones; break;
    case 1: frac = 0; break;
    case 2: frac = 1; break;
    case 3: frac = ones - (mix() & 0xFFFF); break;
    default: frac = mix() & ones; break;
    }
    return __longlong_as_double(static_cast<long long>(e | frac));
}

__global__ void k_check_reciprocal(unsigned long long seed, unsigned long long n, unsigned long long *bad,
                                   unsigned long long *first_bad) {
    unsigned long long local = 0;
    for (unsigned long long k = blockIdx.x * static_cast<unsigned long long>(blockDim.x) + threadIdx.x; k < n;
         k += static_cast<unsigned long long>(gridDim.x) * blockDim.x) {
        const double s = check_divisor(seed, k);
        const double got = jbp::recip_rn_fast(s), want = __ddiv_rn(1.0, s);
        if (__double_as_longlong(got) != __double_as_longlong(want)) {
            ++local;
            atomicMin(first_bad, k);
        }
    }
    if (local) atomicAdd(bad, local);
}

// detect_us_oscillation as the reference states it (jointbp_ets.cpp:2021-2053), the checker of
// the two forms the decoders use (us_oscillation, us_oscillation_warp in kernels_slots.cuh).
__device__ bool us_oscillation_plain(const unsigned short *h, int k1) {
    if (k1 < 100) return false;
    int mn = h[(k1 - 99) % 100], mx = mn;
    long long sum = 0;
    for (int j = k1 - 99; j <= k1; ++j) {
        const int v = h[j % 100];
        mn = v < mn ? v : mn;
        mx = v > mx ? v : mx;
        sum += v;
    }
    const double mean = static_cast<double>(sum) / 100.0;
    if (mean <= 0.0) return false;
    int min_range = static_cast<int>(mean * 0.2);
    if (min_range < 10) min_range = 10;
    if (mx - mn < min_range) return false;
    int prev_sign = 0, turns = 0;
    for (int j = k1 - 98; j <= k1; ++j) {
        const int d = static_cast<int>(h[j % 100]) - static_cast<int>(h[(j - 1) % 100]);
        const int sg = d > 0 ? 1 : (d < 0 ? -1 : 0);
        if (sg) {
            if (prev_sign && sg != prev_sign) turns++;
            prev_sign = sg;
        }
    }
    return turns >= 2;
}

__device__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// One history per warp and case: 100 samples of a pattern chosen by the case number (constant,
// small noise, large noise, alternating, a ramp up then down, rare spikes, a few steps), and a
// window end k1 in [100, 1100).
__global__ void k_check_us_oscillation(unsigned long long seed, long long n, unsigned long long *bad,
                                       unsigned long long *fired) {
    __shared__ unsigned short hist[8][100];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (long long c = blockIdx.x * 8ll + w; c < n; c += gridDim.x * 8ll) {
        const unsigned long long hc = mix64(seed ^ (c * 0x9E3779B97F4A7C15ull));
        const int pat = static_cast<int>(hc % 7), k1 = 100 + static_cast<int>((hc >> 8) % 1000);
        const int level = static_cast<int>((hc >> 20) % 200), amp = 1 + static_cast<int>((hc >> 28) % 60);
        for (int i = lane; i < 100; i += 32) {
            const unsigned long long r = mix64(hc + static_cast<unsigned long long>(i) * 0xD1B54A32D192ED03ull);
            int v = level;
            switch (pat) {
            case 0: break;
            case 1: v += static_cast<int>(r % 3); break;
            case 2: v += static_cast<int>(r % (2 * amp + 1)); break;
            case 3: v += (i & 1) ? amp : 0; break;
            case 4: v += (i < 50 ? i : 100 - i) * amp / 10; break;
            case 5: v += (r % 17 == 0) ? amp * 3 : 0; break;
            default: v += static_cast<int>((i / 25) % 2) * amp + static_cast<int>(r % 2); break;
            }
            hist[w][i] = static_cast<unsigned short>(v < 0 ? 0 : (v > 65535 ? 65535 : v));
        }
        __syncwarp();
        const bool a = us_oscillation_plain(hist[w], k1);
        const bool b = jbp::us_oscillation(hist[w], k1);
        const bool d = jbp::us_oscillation_warp(hist[w], k1);
        if (lane == 0) {
            if (a != b || a != d) atomicAdd(bad, 1ull);
            if (a) atomicAdd(fired, 1ull);
        }
        __syncwarp();
    }
}

}  // namespace

extern "C" int jbp_check_us_oscillation(int device, unsigned long long seed, long long n, long long *mismatches,
                                        long long *fired) {
    if (n < 0 || !mismatches) return jbp::set_last_error(JBP_ERR_ARG, "n >= 0 and mismatches required");
    if (cudaSetDevice(device) != cudaSuccess) return jbp::set_last_error(JBP_ERR_CUDA, "cudaSetDevice failed");
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess)
        return jbp::set_last_error(JBP_ERR_CUDA, "cudaMalloc(counts)");
    cudaError_t e = cudaMemset(d, 0, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) {
        k_check_us_oscillation<<<148 * 4, 256>>>(seed, n, d, d + 1);
        e = cudaGetLastError();
    }
    unsigned long long h[2] = {0ull, 0ull};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess)
        return jbp::set_last_error(JBP_ERR_CUDA, std::string("us-oscillation check: ") + cudaGetErrorString(e));
    *mismatches = static_cast<long long>(h[0]);
    if (fired) *fired = static_cast<long long>(h[1]);
    return JBP_OK;
}

extern "C" int jbp_check_reciprocal(int device, unsigned long long seed, long long n, long long *mismatches,
                                    long long *first_mismatch) {
    if (n < 0 || !mismatches) return jbp::set_last_error(JBP_ERR_ARG, "n >= 0 and mismatches required");
    if (cudaSetDevice(device) != cudaSuccess) return jbp::set_last_error(JBP_ERR_CUDA, "cudaSetDevice failed");
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
        return jbp::set_last_error(JBP_ERR_CUDA, "device attributes");
    unsigned long long *d = nullptr;
    if (cudaMalloc(&d, 2 * sizeof(unsigned long long)) != cudaSuccess)
        return jbp::set_last_error(JBP_ERR_CUDA, "cudaMalloc(counts)");
    const unsigned long long init[2] = {0ull, ~0ull};
    cudaError_t e = cudaMemcpy(d, init, sizeof(init), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_check_reciprocal<<<sms * 8, 256>>>(seed, static_cast<unsigned long long>(n), d, d + 1);
        e = cudaGetLastError();
    }
    unsigned long long h[2] = {0ull, ~0ull};
    if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return jbp::set_last_error(JBP_ERR_CUDA, std::string("reciprocal check: ") + cudaGetErrorString(e));
    *mismatches = static_cast<long long>(h[0]);
    if (first_mismatch) *first_mismatch = h[0] ? static_cast<long long>(h[1]) : -1;
    return JBP_OK;
}

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
