// Learned flip proposal: a 3-layer MLP over per-qubit features of a stalled BP state
// (8 -> 64 -> 64 -> 2, ReLU) whose two logits score the qubit's x-bit and z-bit as wrong.  The
// decoder orders the qubits by these scores (most likely wrong first), takes the flips from
// the shortest ordered prefix whose columns span the syndrome difference (the OSD stage's
// incremental GF(2) elimination, unique solution of weight <= 30), and keeps the result only
// if both syndromes then match exactly; otherwise the plain post-processing stages run as
// before.
// The reference has no counterpart: this is an addition of the B200 build.
//
// Parameters (FP32, this order, 4,866 values): W1 [64][8], b1 [64], W2 [64][64], b2 [64],
// W3 [2][64], b3 [2]; layer l computes h = W h_prev + b (W row-major, out x in).
//
// Inference runs on the tensor cores with mma.sync m16n8k16 (BF16 operands, FP32
// accumulate) inside one warp per 16 qubits: the 8 features are the first 8 of 16 K columns
// of layer 1, layer outputs stay in registers (the FP32 accumulator fragment of two n8 tiles
// is the BF16 A fragment of the next layer's k16 tile), and the weights are read from global
// memory in fragment order (one coalesced 8-byte load per lane per tile).  Per stalled trial
// this is 576 tiles x 44 MMAs; at that size the tensor-core issue path of mma.sync is not the
// limit, so the fused form keeps the shared memory of the resident trial untouched.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>
#include <cstring>

namespace jbp {

constexpr int kMlpIn = 8, kMlpH = 64, kMlpOut = 2;
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpH * kMlpIn, kMlpW2 = kMlpB1 + kMlpH, kMlpB2 = kMlpW2 + kMlpH * kMlpH,
              kMlpW3 = kMlpB2 + kMlpH, kMlpB3 = kMlpW3 + kMlpOut * kMlpH, kMlpParams = kMlpB3 + kMlpOut;
static_assert(kMlpParams == 4866, "parameter layout");

// Fragment-ordered BF16 weights and FP32 biases on the device.
constexpr int kMlpW1Frag = 8 * 32 * 2;          // 8 n-tiles (K = 16, features padded)
constexpr int kMlpW2Frag = 4 * 8 * 32 * 2;      // 4 k-tiles x 8 n-tiles
constexpr int kMlpW3Frag = 4 * 32 * 2;          // 4 k-tiles x 1 n-tile (columns 0, 1 used)
constexpr int kMlpDevWords = kMlpW1Frag + kMlpW2Frag + kMlpW3Frag + kMlpH + kMlpH + 8;

struct MlpDev {
    const uint32_t *w;   // kMlpDevWords: w1 frags | w2 frags | w3 frags | b1 (f32) | b2 | b3 (8)
};

__host__ __device__ inline uint16_t mlp_bf16_bits(float f) {
    // round to nearest even (finite inputs)
    uint32_t u;
    memcpy(&u, &f, 4);
    const uint32_t r = u + 0x7FFFu + ((u >> 16) & 1u);
    return static_cast<uint16_t>(r >> 16);
}

__host__ __device__ inline float mlp_bf16_to_float(uint16_t b) {
    const uint32_t u = static_cast<uint32_t>(b) << 16;
    float f;
    memcpy(&f, &u, 4);
    return f;
}

// Packs FP32 parameters into the device layout (host side).  B fragment of an m16n8k16 MMA
// for lane L: k = (L % 4) * 2 + {0, 1} (register 0) and + 8 (register 1), n = L / 4; the B
// matrix of a layer is W^T (K = in, N = out).
inline void mlp_pack(const float *p, uint32_t *out) {
    auto wb = [&](int base, int nout, int nin, int k, int n) -> uint16_t {
        return (k < nin && n < nout) ? mlp_bf16_bits(p[base + n * nin + k]) : 0;
    };
    auto frag = [&](uint32_t *dst, int base, int nout, int nin, int kt, int nt) {
        for (int L = 0; L < 32; ++L) {
            const int n = nt * 8 + L / 4, k0 = kt * 16 + (L % 4) * 2;
            dst[L * 2 + 0] = wb(base, nout, nin, k0, n) | (static_cast<uint32_t>(wb(base, nout, nin, k0 + 1, n)) << 16);
            dst[L * 2 + 1] =
                wb(base, nout, nin, k0 + 8, n) | (static_cast<uint32_t>(wb(base, nout, nin, k0 + 9, n)) << 16);
        }
    };
    uint32_t *w1 = out, *w2 = w1 + kMlpW1Frag, *w3 = w2 + kMlpW2Frag;
    for (int nt = 0; nt < 8; ++nt) frag(w1 + nt * 64, kMlpW1, kMlpH, kMlpIn, 0, nt);
    for (int kt = 0; kt < 4; ++kt)
        for (int nt = 0; nt < 8; ++nt) frag(w2 + (kt * 8 + nt) * 64, kMlpW2, kMlpH, kMlpH, kt, nt);
    for (int kt = 0; kt < 4; ++kt) frag(w3 + kt * 64, kMlpW3, kMlpOut, kMlpH, kt, 0);
    float *b = reinterpret_cast<float *>(w3 + kMlpW3Frag);
    for (int i = 0; i < kMlpH; ++i) b[i] = p[kMlpB1 + i];
    for (int i = 0; i < kMlpH; ++i) b[kMlpH + i] = p[kMlpB2 + i];
    for (int i = 0; i < 8; ++i) b[2 * kMlpH + i] = i < kMlpOut ? p[kMlpB3 + i] : 0.0f;
}

#ifdef __CUDACC__

__device__ __forceinline__ void mma_bf16_16816(float c[4], const uint32_t a[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

__device__ __forceinline__ uint32_t pack_bf16x2(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t *>(&v);
}

// Logits of 16 qubits (rows g = lane/4 and g + 8 of the tile) from their features.
// feat(row, k) gives feature k (0..7) of tile row `row`.  Returns the x-flip and z-flip
// logits of rows g (out[0], out[1]) and g + 8 (out[2], out[3]) in lanes with lane % 4 == 0.
template <class Feat>
__device__ __forceinline__ void mlp_tile(const MlpDev &w, const Feat &feat, float out[4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const uint32_t *w1 = w.w, *w2 = w1 + kMlpW1Frag, *w3 = w2 + kMlpW2Frag;
    const float *b = reinterpret_cast<const float *>(w3 + kMlpW3Frag);
    uint32_t a[4];
    a[0] = pack_bf16x2(feat(g, 2 * q), feat(g, 2 * q + 1));
    a[1] = pack_bf16x2(feat(g + 8, 2 * q), feat(g + 8, 2 * q + 1));
    a[2] = 0u;
    a[3] = 0u;
    // layer 1 -> A fragments of layer 2 (bias + ReLU on the accumulators)
    uint32_t h[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const uint2 bf = __ldg(reinterpret_cast<const uint2 *>(w1 + nt * 64) + lane);
        const float b0 = __ldg(b + nt * 8 + 2 * q), b1 = __ldg(b + nt * 8 + 2 * q + 1);
        float c[4] = {b0, b1, b0, b1};
        mma_bf16_16816(c, a, bf.x, bf.y);
        const int kt = nt >> 1, hi = nt & 1;
        h[kt][2 * hi + 0] = pack_bf16x2(fmaxf(c[0], 0.0f), fmaxf(c[1], 0.0f));
        h[kt][2 * hi + 1] = pack_bf16x2(fmaxf(c[2], 0.0f), fmaxf(c[3], 0.0f));
    }
    // A fragment register order: (row g, k lo), (row g+8, k lo), (row g, k hi), (row g+8, k hi)
    uint32_t a2[4][4];
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        a2[kt][0] = h[kt][0];
        a2[kt][1] = h[kt][1];
        a2[kt][2] = h[kt][2];
        a2[kt][3] = h[kt][3];
    }
    uint32_t h2[4][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        const float b0 = __ldg(b + kMlpH + nt * 8 + 2 * q), b1 = __ldg(b + kMlpH + nt * 8 + 2 * q + 1);
        float c[4] = {b0, b1, b0, b1};
#pragma unroll
        for (int kt = 0; kt < 4; ++kt) {
            const uint2 bf = __ldg(reinterpret_cast<const uint2 *>(w2 + (kt * 8 + nt) * 64) + lane);
            mma_bf16_16816(c, a2[kt], bf.x, bf.y);
        }
        const int kt2 = nt >> 1, hi = nt & 1;
        h2[kt2][2 * hi + 0] = pack_bf16x2(fmaxf(c[0], 0.0f), fmaxf(c[1], 0.0f));
        h2[kt2][2 * hi + 1] = pack_bf16x2(fmaxf(c[2], 0.0f), fmaxf(c[3], 0.0f));
    }
    const float b0 = __ldg(b + 2 * kMlpH + 2 * q), b1 = __ldg(b + 2 * kMlpH + 2 * q + 1);
    float c[4] = {b0, b1, b0, b1};
#pragma unroll
    for (int kt = 0; kt < 4; ++kt) {
        const uint2 bf = __ldg(reinterpret_cast<const uint2 *>(w3 + kt * 64) + lane);
        mma_bf16_16816(c, h2[kt], bf.x, bf.y);
    }
    out[0] = c[0];
    out[1] = c[1];
    out[2] = c[2];
    out[3] = c[3];
}

#endif

}  // namespace jbp
