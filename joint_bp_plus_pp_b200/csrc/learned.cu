// Training and standalone inference of the learned flip proposal (mlp.cuh): hand-written
// FP32 forward/backward kernels with Adam, the BF16 tensor-core inference kernel the decoder
// fuses after a stall, and their C entry points (include/jbp_b200.h).  No counterpart in the
// reference.
//
// Loss: per sample, the sum over the two outputs (x-flip, z-flip) of the binary cross-entropy
// with logits, positives weighted by pos_weight; the batch loss is the mean over samples.
#include <algorithm>
#include <cmath>
#include <numeric>
#include <random>
#include <string>
#include <vector>

#include "../../include/jbp_b200.h"
#include "ctx.hpp"
#include "engine.hpp"
#include "mlp.cuh"

namespace jbp {
namespace {

constexpr int kTile = 32;          // samples per tile
constexpr int kGradThreads = 64;   // one thread per hidden unit

__device__ __forceinline__ float softplus(float x) { return x > 0.0f ? x + log1pf(expf(-x)) : log1pf(expf(x)); }
__device__ __forceinline__ float sigmoid(float x) { return 1.0f / (1.0f + expf(-x)); }

// Gradient of the mean loss over samples [0, nsamples) of X/Y (rows idx[i] when idx is
// given), accumulated into grad (zeroed by the caller); loss sum into *loss.
// Block: 64 threads, thread j owns hidden unit j; tiles of 32 samples.
__global__ void __launch_bounds__(kGradThreads) k_mlp_grad(const float *__restrict__ prm, const float *__restrict__ X,
                                                           const float *__restrict__ Y, const int *__restrict__ idx,
                                                           int nsamples, int per_block, float pos_weight, float scale,
                                                           float *grad, double *loss) {
    __shared__ float W2[kMlpH][kMlpH + 1];    // W2[j][i]; the padding keeps rows and columns conflict-free
    __shared__ float xs[kTile][kMlpIn], ys[kTile][kMlpOut];
    __shared__ float h1[kTile][kMlpH + 1], h2[kTile][kMlpH + 1], dh2[kTile][kMlpH + 1];
    __shared__ float dz[kTile][kMlpOut];
    __shared__ float lsum[kTile];
    const int j = threadIdx.x;
    for (int i = 0; i < kMlpH; ++i) {
        W2[j][i] = prm[kMlpW2 + j * kMlpH + i];
    }
    float w1[kMlpIn], dw1[kMlpIn], dw2[kMlpH];
    for (int k = 0; k < kMlpIn; ++k) { w1[k] = prm[kMlpW1 + j * kMlpIn + k]; dw1[k] = 0.0f; }
    for (int i = 0; i < kMlpH; ++i) dw2[i] = 0.0f;
    const float b1 = prm[kMlpB1 + j], b2 = prm[kMlpB2 + j];
    const float w30 = prm[kMlpW3 + j], w31 = prm[kMlpW3 + kMlpH + j];
    const float b30 = prm[kMlpB3], b31 = prm[kMlpB3 + 1];
    float db1 = 0.0f, db2 = 0.0f, dw30 = 0.0f, dw31 = 0.0f, db30 = 0.0f, db31 = 0.0f;
    double lacc = 0.0;
    const int s0 = blockIdx.x * per_block, s1 = min(nsamples, s0 + per_block);
    __syncthreads();
    for (int t0 = s0; t0 < s1; t0 += kTile) {
        const int cnt = min(kTile, s1 - t0);
        for (int e = j; e < kTile * kMlpIn; e += kGradThreads) {
            const int s = e / kMlpIn, k = e % kMlpIn;
            xs[s][k] = s < cnt ? X[static_cast<size_t>(idx ? idx[t0 + s] : t0 + s) * kMlpIn + k] : 0.0f;
        }
        for (int e = j; e < kTile * kMlpOut; e += kGradThreads) {
            const int s = e / kMlpOut, o = e % kMlpOut;
            ys[s][o] = s < cnt ? Y[static_cast<size_t>(idx ? idx[t0 + s] : t0 + s) * kMlpOut + o] : 0.0f;
        }
        __syncthreads();
        for (int s = 0; s < kTile; ++s) {
            float a = b1;
            for (int k = 0; k < kMlpIn; ++k) a = fmaf(w1[k], xs[s][k], a);
            h1[s][j] = fmaxf(a, 0.0f);
        }
        __syncthreads();
        for (int s = 0; s < kTile; ++s) {
            float a = b2;
            for (int i = 0; i < kMlpH; ++i) a = fmaf(W2[j][i], h1[s][i], a);
            h2[s][j] = fmaxf(a, 0.0f);
        }
        __syncthreads();
        if (j < kTile) {
            const int s = j;
            float z0 = b30, z1 = b31;
            for (int i = 0; i < kMlpH; ++i) {
                z0 = fmaf(prm[kMlpW3 + i], h2[s][i], z0);
                z1 = fmaf(prm[kMlpW3 + kMlpH + i], h2[s][i], z1);
            }
            float l = 0.0f, g0 = 0.0f, g1 = 0.0f;
            if (s < cnt) {
                const float y0 = ys[s][0], y1 = ys[s][1];
                l = pos_weight * y0 * softplus(-z0) + (1.0f - y0) * softplus(z0) + pos_weight * y1 * softplus(-z1) +
                    (1.0f - y1) * softplus(z1);
                g0 = (pos_weight * y0 * (sigmoid(z0) - 1.0f) + (1.0f - y0) * sigmoid(z0)) * scale;
                g1 = (pos_weight * y1 * (sigmoid(z1) - 1.0f) + (1.0f - y1) * sigmoid(z1)) * scale;
            }
            dz[s][0] = g0;
            dz[s][1] = g1;
            lsum[s] = l;
        }
        __syncthreads();
        if (j == 0)
            for (int s = 0; s < cnt; ++s) lacc += lsum[s];
        for (int s = 0; s < kTile; ++s) {
            const float d0 = dz[s][0], d1 = dz[s][1], hv = h2[s][j];
            dw30 = fmaf(d0, hv, dw30);
            dw31 = fmaf(d1, hv, dw31);
            const float d = hv > 0.0f ? w30 * d0 + w31 * d1 : 0.0f;
            dh2[s][j] = d;
            db2 += d;
            if (j == 0) { db30 += d0; db31 += d1; }
            for (int i = 0; i < kMlpH; ++i) dw2[i] = fmaf(d, h1[s][i], dw2[i]);
        }
        __syncthreads();
        for (int s = 0; s < kTile; ++s) {
            float a = 0.0f;
            for (int jj = 0; jj < kMlpH; ++jj) a = fmaf(W2[jj][j], dh2[s][jj], a);
            const float d = h1[s][j] > 0.0f ? a : 0.0f;
            db1 += d;
            for (int k = 0; k < kMlpIn; ++k) dw1[k] = fmaf(d, xs[s][k], dw1[k]);
        }
        __syncthreads();
    }
    for (int k = 0; k < kMlpIn; ++k) atomicAdd(&grad[kMlpW1 + j * kMlpIn + k], dw1[k]);
    atomicAdd(&grad[kMlpB1 + j], db1);
    for (int i = 0; i < kMlpH; ++i) atomicAdd(&grad[kMlpW2 + j * kMlpH + i], dw2[i]);
    atomicAdd(&grad[kMlpB2 + j], db2);
    atomicAdd(&grad[kMlpW3 + j], dw30);
    atomicAdd(&grad[kMlpW3 + kMlpH + j], dw31);
    if (j == 0) {
        atomicAdd(&grad[kMlpB3], db30);
        atomicAdd(&grad[kMlpB3 + 1], db31);
        atomicAdd(loss, lacc);
    }
}

__global__ void k_adam(float *prm, const float *grad, float *m, float *v, int n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float g = grad[i];
    const float mi = b1 * m[i] + (1.0f - b1) * g, vi = b2 * v[i] + (1.0f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    prm[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// Standalone BF16 tensor-core inference (the device code the decoder runs after a stall).
__global__ void k_mlp_infer(MlpDev w, const float *X, long long n, float *logits) {
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
    const long long tiles = (n + 15) / 16;
    for (long long t = wid; t < tiles; t += nw) {
        auto feat = [&](int row, int k) -> float {
            const long long r = t * 16 + row;
            return r < n ? X[r * kMlpIn + k] : 0.0f;
        };
        float o[4];
        mlp_tile(w, feat, o);
        const int lane = threadIdx.x & 31;
        if ((lane & 3) == 0) {
            const long long r0 = t * 16 + (lane >> 2), r1 = r0 + 8;
            if (r0 < n) { logits[r0 * 2] = o[0]; logits[r0 * 2 + 1] = o[1]; }
            if (r1 < n) { logits[r1 * 2] = o[2]; logits[r1 * 2 + 1] = o[3]; }
        }
    }
}

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() { cudaFree(p); }
    template <typename T>
    T *as() { return static_cast<T *>(p); }
};

std::string alloc(DevBuf &b, size_t bytes) {
    cudaError_t e = jbp::dev_malloc(&b.p, std::max<size_t>(bytes, 16));
    return e == cudaSuccess ? "" : cuda_err(e, "cudaMalloc(mlp)");
}

#define MLP_TRY(expr, what)                                                  \
    do {                                                                     \
        cudaError_t e_ = (expr);                                             \
        if (e_ != cudaSuccess) return set_last_error(JBP_ERR_CUDA, cuda_err(e_, what)); \
    } while (0)

int grad_launch(const float *d_prm, const float *d_x, const float *d_y, const int *d_idx, int n, float pos_weight,
                float *d_grad, double *d_loss) {
    const int per_block = std::max(kTile, (n + 4 * 148 - 1) / (4 * 148) / kTile * kTile);
    const int blocks = (n + per_block - 1) / per_block;
    k_mlp_grad<<<blocks, kGradThreads>>>(d_prm, d_x, d_y, d_idx, n, per_block, pos_weight, 1.0f / n, d_grad, d_loss);
    return cudaGetLastError() == cudaSuccess ? JBP_OK : JBP_ERR_CUDA;
}

}  // namespace
}  // namespace jbp

using namespace jbp;

int jbp_mlp_param_count(void) { return kMlpParams; }

int jbp_mlp_grad(jbp_ctx *ctx, const float *params, long long nsamples, const float *x, const float *y,
                 float pos_weight, float *grad_out, double *loss_out) {
    if (!ctx || !params || !x || !y || !grad_out || nsamples <= 0 || nsamples > (1LL << 30))
        return set_last_error(JBP_ERR_ARG, "invalid argument");
    MLP_TRY(cudaSetDevice(ctx->engine.device()), "cudaSetDevice");
    DevBuf p, dx, dy, g, l;
    std::string e = alloc(p, sizeof(float) * kMlpParams);
    if (e.empty()) e = alloc(dx, sizeof(float) * kMlpIn * nsamples);
    if (e.empty()) e = alloc(dy, sizeof(float) * kMlpOut * nsamples);
    if (e.empty()) e = alloc(g, sizeof(float) * kMlpParams);
    if (e.empty()) e = alloc(l, sizeof(double));
    if (!e.empty()) return set_last_error(JBP_ERR_CUDA, e);
    MLP_TRY(cudaMemcpy(p.p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemcpy(dx.p, x, sizeof(float) * kMlpIn * nsamples, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemcpy(dy.p, y, sizeof(float) * kMlpOut * nsamples, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemset(g.p, 0, sizeof(float) * kMlpParams), "memset");
    MLP_TRY(cudaMemset(l.p, 0, sizeof(double)), "memset");
    if (grad_launch(p.as<float>(), dx.as<float>(), dy.as<float>(), nullptr, static_cast<int>(nsamples), pos_weight,
                    g.as<float>(), l.as<double>()) != JBP_OK)
        return set_last_error(JBP_ERR_CUDA, "mlp gradient launch failed");
    MLP_TRY(cudaMemcpy(grad_out, g.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost), "download");
    double ls = 0.0;
    MLP_TRY(cudaMemcpy(&ls, l.p, sizeof(double), cudaMemcpyDeviceToHost), "download");
    if (loss_out) *loss_out = ls / static_cast<double>(nsamples);
    return JBP_OK;
}

int jbp_mlp_train(jbp_ctx *ctx, float *params, long long nsamples, const float *x, const float *y, int epochs,
                  int batch, float lr, float pos_weight, uint64_t seed, double *epoch_loss) {
    if (!ctx || !params || !x || !y || nsamples <= 0 || nsamples > (1LL << 30) || epochs < 0 || batch <= 0 ||
        !(lr > 0.0f))
        return set_last_error(JBP_ERR_ARG, "invalid argument");
    MLP_TRY(cudaSetDevice(ctx->engine.device()), "cudaSetDevice");
    const int n = static_cast<int>(nsamples);
    DevBuf p, dx, dy, g, m, v, l, ix;
    std::string e = alloc(p, sizeof(float) * kMlpParams);
    if (e.empty()) e = alloc(dx, sizeof(float) * kMlpIn * nsamples);
    if (e.empty()) e = alloc(dy, sizeof(float) * kMlpOut * nsamples);
    if (e.empty()) e = alloc(g, sizeof(float) * kMlpParams);
    if (e.empty()) e = alloc(m, sizeof(float) * kMlpParams);
    if (e.empty()) e = alloc(v, sizeof(float) * kMlpParams);
    if (e.empty()) e = alloc(l, sizeof(double));
    if (e.empty()) e = alloc(ix, sizeof(int) * nsamples);
    if (!e.empty()) return set_last_error(JBP_ERR_CUDA, e);
    MLP_TRY(cudaMemcpy(p.p, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemcpy(dx.p, x, sizeof(float) * kMlpIn * nsamples, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemcpy(dy.p, y, sizeof(float) * kMlpOut * nsamples, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemset(m.p, 0, sizeof(float) * kMlpParams), "memset");
    MLP_TRY(cudaMemset(v.p, 0, sizeof(float) * kMlpParams), "memset");
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::mt19937_64 rng(seed);
    long long step = 0;
    const float b1 = 0.9f, b2 = 0.999f;
    for (int ep = 0; ep < epochs; ++ep) {
        std::shuffle(perm.begin(), perm.end(), rng);
        MLP_TRY(cudaMemcpy(ix.p, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice), "upload");
        MLP_TRY(cudaMemset(l.p, 0, sizeof(double)), "memset");
        for (int s0 = 0; s0 < n; s0 += batch) {
            const int cnt = std::min(batch, n - s0);
            MLP_TRY(cudaMemset(g.p, 0, sizeof(float) * kMlpParams), "memset");
            if (grad_launch(p.as<float>(), dx.as<float>(), dy.as<float>(), ix.as<int>() + s0, cnt, pos_weight,
                            g.as<float>(), l.as<double>()) != JBP_OK)
                return set_last_error(JBP_ERR_CUDA, "mlp gradient launch failed");
            ++step;
            const float c1 = 1.0f - std::pow(b1, static_cast<float>(step));
            const float c2 = 1.0f - std::pow(b2, static_cast<float>(step));
            k_adam<<<(kMlpParams + 255) / 256, 256>>>(p.as<float>(), g.as<float>(), m.as<float>(), v.as<float>(),
                                                      kMlpParams, lr, b1, b2, 1e-8f, c1, c2);
        }
        double ls = 0.0;
        MLP_TRY(cudaMemcpy(&ls, l.p, sizeof(double), cudaMemcpyDeviceToHost), "download");
        if (epoch_loss) epoch_loss[ep] = ls / n;
    }
    MLP_TRY(cudaGetLastError(), "training");
    MLP_TRY(cudaMemcpy(params, p.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost), "download");
    return JBP_OK;
}

int jbp_mlp_infer(jbp_ctx *ctx, const float *params, long long nsamples, const float *x, float *logits) {
    if (!ctx || !params || !x || !logits || nsamples <= 0) return set_last_error(JBP_ERR_ARG, "invalid argument");
    MLP_TRY(cudaSetDevice(ctx->engine.device()), "cudaSetDevice");
    std::vector<uint32_t> packed(kMlpDevWords);
    mlp_pack(params, packed.data());
    DevBuf w, dx, dl;
    std::string e = alloc(w, sizeof(uint32_t) * kMlpDevWords);
    if (e.empty()) e = alloc(dx, sizeof(float) * kMlpIn * nsamples);
    if (e.empty()) e = alloc(dl, sizeof(float) * kMlpOut * nsamples);
    if (!e.empty()) return set_last_error(JBP_ERR_CUDA, e);
    MLP_TRY(cudaMemcpy(w.p, packed.data(), sizeof(uint32_t) * kMlpDevWords, cudaMemcpyHostToDevice), "upload");
    MLP_TRY(cudaMemcpy(dx.p, x, sizeof(float) * kMlpIn * nsamples, cudaMemcpyHostToDevice), "upload");
    MlpDev md{w.as<uint32_t>()};
    k_mlp_infer<<<ctx->engine.sm_count() * 4, 256>>>(md, dx.as<float>(), nsamples, dl.as<float>());
    MLP_TRY(cudaGetLastError(), "inference launch");
    MLP_TRY(cudaMemcpy(logits, dl.p, sizeof(float) * kMlpOut * nsamples, cudaMemcpyDeviceToHost), "download");
    return JBP_OK;
}

int jbp_set_flip_model(jbp_ctx *ctx, const float *params) {
    if (!ctx) return set_last_error(JBP_ERR_ARG, "invalid argument");
    std::string e = ctx->engine.set_flip_model(params);
    return e.empty() ? JBP_OK : set_last_error(JBP_ERR_CUDA, e);
}
