// Trial-resident BP: one persistent thread block per SM owns one trial at a time and keeps
// its BP state in shared memory, from sampling to classification.  No message ever travels to
// HBM; the only global traffic per trial is its error (or syndrome), its result record and,
// when asked for, its estimate.  With FP32 message storage (the GC instantiation) the Z side's
// messages live in a per-block global scratch that stays in L2; everything else as below.
//
// Code structure.  The kernel is built for quasi-cyclic codes whose blocks are affine
// permutations (the APM construction of the reference params file, jointbp_ets.cpp:98-160):
// check j*P + x of a side meets, in block column l, variable l*P + ((fa*x + fb) mod P), and
// variable l*P + y meets, in block row j, check j*P + ((ia*y + ib) mod P).  Neighbours are
// computed, not read from tables, so the only shared-memory traffic is the messages.
//
// State of the trial in shared memory (shipped code: P = 768, J = 3, L = 12):
//   c2v[side][l][c]  16-bit LLR (base 2), check-to-variable message of the edge of check c in
//                    block column l                                    2*12*2304*2 = 110,592 B
//                    (FP32 storage: the X side here, 12*2304*4 = 110,592 B)
//   A[side][v]       FP32 "all but one" total of variable v on that side: the variable-to-check
//                    message of edge (c, v) is A[side][v] - c2v[side][l][c], clamped.  The
//                    lowest mantissa bit of A carries the hard decision bit of that side.
//                                                                        2*9216*4 = 73,728 B
//   err[v]           true error (0..3)                                            9,216 B
//   syn[side][c/32]  target syndrome bits                                           576 B
// A warp's lanes take consecutive checks (check phase) or consecutive variables (variable
// phase); with the affine maps and P a multiple of 64 every 32-lane access of c2v and A hits
// 32 distinct banks (odd multipliers permute residues mod 64).
//
// Arithmetic (FP32, base-2 LLRs, the same model as the slot engine's LLR kernels):
//   check node, tanh rule in ratio form: u_i = 2^-|y_i|, t_i = (1 - u_i) / (1 + u_i), so the
//     product of the other edges' t is PN/PD with PN = prod (1 - u_j), PD = prod (1 + u_j), and
//     the output magnitude log2((1 + T) / (1 - T)) = log2((PD + PN) / (PD - PN)), carried in the
//     cancellation-free form of res_row_rule: one ex2 per input, one rcp and one lg2 per
//     output; prefix/suffix products exclude the edge itself.
//   variable node: Lam = sum of the X c2v, Mu = sum of the Z c2v; log2 weights of I, X, Z, Y
//     are lp0, lp1 - Lam, lp2 - Mu, lp3 - Lam - Mu (first maximum = hard decision); the x-bit
//     coupling through the Z side Gx = lse2(lp0, lp2 - Mu) - lse2(lp1, lp3 - Mu) and the z-bit
//     coupling Hz = lse2(lp0, lp1 - Lam) - lse2(lp2, lp3 - Lam) give A_x = Lam + Gx and
//     A_z = Mu + Hz (jointbp_ets.cpp:2451-2519 in the LLR domain).
// The flooding schedule and the per-iteration syndrome test with early exit follow
// jointbp_ets.cpp:1943-2535; the syndrome test of iteration k is fused into the check phase
// of iteration k + 1, which reads the decision bits from A's low bits anyway.
#pragma once

#include <cuda_fp16.h>

#include "engine.cuh"
#include "kernels_slots.cuh"
#include "kernels_pp.cuh"
#include "mlp.cuh"

namespace jbp {

constexpr int kResMaxJ = 4;
constexpr int kResMaxL = 16;
constexpr int kResThreads = 768;

struct ResCode {
    int P, J, L, n, m;             // n = L*P, m = J*P checks per side
    // affine maps in fixed point: y = (a x + b) mod P is __umulhi(x F + G, P) with
    // F = ceil(a 2^32 / P), G = ceil(b 2^32 / P) (exact for x < P, checked at start-up)
    unsigned fF[2][kResMaxJ][kResMaxL], fG[2][kResMaxJ][kResMaxL];   // check -> variable
    unsigned iF[2][kResMaxJ][kResMaxL], iG[2][kResMaxJ][kResMaxL];   // variable -> check
    int words;
    const uint64_t *basis_rows[2];
    const int *pivot_row[2];
};

// Per-run parameters of the resident kernel.
struct ResRun {
    int max_iter, check_warmup, check_interval;
    int source;
    double p, p_max;               // p_max > p: per-trial p uniform in [p, p_max) (trial_p)
    int use_prior;
    double prior4[4];
    unsigned long long seed;
    long long first_trial, ntrials;
    const long long *trial_list;   // optional: trial k is trial_list[k] instead of first_trial + k
    const uint8_t *src_err;        // [ntrials][n]
    const uint8_t *src_sx, *src_sz;
    uint8_t *est_out;
    float *llr_out;                // [ntrials][n][2] final LLRs (x, z), natural units, or null
    jbp_trial_result *res_out;
    unsigned long long *hist;
    DevCounters *cnt;
    // post-processing (PP instantiations only)
    int flip_hist;
    DevCode dc;                    // table form of the code for the post-processing stages
    DevEts ets;
    unsigned char *pp_scratch;     // per block: PpScratch | decision ring [R][n] | |LLR| [2][n] doubles |
                                   // features [n][kMlpIn]
    size_t pp_scratch_stride;
    size_t pp_smem_base;           // offset of the post-processing arrays in shared memory
    // FP32 messages (the instantiation with GC): the Z side's c2v of each block in global memory,
    // L2-resident (the X side's stay in shared memory)
    unsigned char *c2v_scratch;
    size_t c2v_stride;
    // learned flip proposal (mlp.cuh): tried at stalls from iteration learned_from (0 = off)
    int learned_from;
    int learned_order;             // 0: the model's scores; 1: |LLR| order (no network)
    int learned_cols;              // columns the proposal's elimination may use
    MlpDev mlp;
    int collect;                   // 1: record stall-state samples instead of proposing
    unsigned collect_every;        // ... 1 in this many of the quiet, correctly decided qubits
    float *col_x, *col_y;          // [col_cap][8], [col_cap][2]
    unsigned long long *col_count;
    long long col_cap;
    // run budget (jbp_options.watchdog_ms): > 0, a block that has run this long (global timer,
    // from its start) claims no further trial and abandons the one it decodes at its next check
    // (every kResBudgetEvery iterations); cnt->watchdog counts the blocks that stopped so
    unsigned long long budget_ns;
    // jbp_request_abort's flag (pinned host memory): a block that sees it set claims no further
    // trial; it looks at every kResAbortEvery-th claim and, in a trial past iteration
    // kResAbortFrom, every kResBudgetEvery iterations; cnt->aborted counts the blocks that stopped
    const volatile int *abort_flag;
};

constexpr int kResBudgetEvery = 16;   // iterations between two run-budget checks of a block
constexpr unsigned long long kResAbortEvery = 8;   // trial claims between two reads of the abort flag
constexpr int kResAbortFrom = 64;      // iteration from which a long trial also reads it

// Nanoseconds of the GPU's global timer (the run budget of the persistent kernels).
__device__ __forceinline__ unsigned long long dev_globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr int kLearnedTries = 3;   // learned proposals per trial at most
constexpr int kLearnedMaxUnsat = 30;   // ... and only while max(us_x, us_z) is at most this
constexpr int kLearnedMaxCols = 512;   // ... solved from at most this many of the best-scored qubits (default)

// Per-block global scratch of a post-processing run: the GF(2) work areas, the ring of the
// last R iterations' decisions and the |LLR| keys of the OSD order.
__host__ __device__ inline size_t res_pp_scratch_bytes(int n, int mmax, int R) {
    return pp_align(pp_scratch_bytes(n, mmax)) + pp_align(static_cast<size_t>(R) * n) + pp_align(16ull * n) +
           pp_align(4ull * kMlpIn * n);
}

// (a x + b) mod P from the fixed-point constants of the map: one multiply-add and one
// high-half multiply.
template <int P>
__device__ __forceinline__ unsigned res_map(unsigned F, unsigned G, unsigned x) {
    return __umulhi(x * F + G, static_cast<unsigned>(P));
}


// 16-bit message storage: IEEE half.
struct StoreHalf {
    using T = __half;
    static __device__ __forceinline__ float ld(const T *p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(T *p, float v) { *p = __float2half_rn(v); }
};

// 32-bit message storage.
struct StoreFloat {
    using T = float;
    static __device__ __forceinline__ float ld(const T *p) { return *p; }
    static __device__ __forceinline__ void st(T *p, float v) { *p = v; }
};

__device__ __forceinline__ float res_ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float res_lg2(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float res_rcp(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float res_lse2(float a, float b) {
    return fmaxf(a, b) + res_lg2(1.0f + res_ex2(-fabsf(a - b)));
}

constexpr float kResCmax = 110.0f;     // check-to-variable magnitude clamp (exact in FP16 storage)
constexpr int kResSepTest = 24;        // test on its own when at most this many threads failed the last test

__device__ __forceinline__ float with_bit(float a, unsigned b) {
    return __uint_as_float((__float_as_uint(a) & ~1u) | b);
}

// Shared-memory bytes of the resident kernel for a code: the trial state (the c2v of the sides
// kept in shared memory, A, err, syn, 16 ints), then the post-processing arrays at pp_align(base).
__host__ __device__ inline size_t res_base_bytes(int n, int m, int L, size_t store_bytes, int c2v_sides_in_smem) {
    const size_t c2v = (static_cast<size_t>(c2v_sides_in_smem) * L * m * store_bytes + 15) / 16 * 16;
    const size_t A = 2ull * n * 4;
    const size_t err = (static_cast<size_t>(n) + 15) / 16 * 16;
    const size_t syn = (2ull * ((m + 31) / 32) + 3) / 4 * 4 * 4;
    return c2v + A + err + syn + 64;
}
// The slow path's decision planes (post-processing instantiations): the x and z decisions of
// the last three iterations, 32 qubits per word, after the post-processing arrays.
__host__ __device__ inline size_t res_plane_bytes(int n) { return 3ull * 2 * ((n + 31) / 32) * 4; }
__host__ __device__ inline size_t res_plane_offset(size_t pp_smem_base, int n, int m) {
    return pp_smem_base + pp_smem_bytes(n, 2 * m, m) + 256;
}
__host__ __device__ inline size_t res_smem_bytes(int n, int m, int L, size_t store_bytes, bool pp,
                                                 int c2v_sides_in_smem = 2) {
    const size_t base = res_base_bytes(n, m, L, store_bytes, c2v_sides_in_smem);
    return pp ? res_plane_offset(pp_align(base), n, m) + res_plane_bytes(n) : base;
}


// The check rule on one check of L edges: from the edges' variable-to-check inputs in(l) and
// the check's syndrome bit, out(l, c2v of edge l) for l = 0 .. L-1.
//
// Stable tanh rule.  Per edge u = 2^-|y|, N = 1 - u, D = 1 + u, t = N / D, so the product of a
// set's t is T = PN / PD with PN = prod N, PD = prod D.  A set is carried as (H, G) with
// H = (PD - PN) / 2 and G = (PD + PN) / 2: the empty set is (0, 1), a single edge (u, 1), and
// joining a set with one edge gives H' = H + u G, G' = G + u H -- sums of positive terms with
// one rounding each, which keep full relative precision however close T is to 1.  Joining two
// sets a, b: H = G_a H_b + H_a G_b, G = G_a G_b + H_a H_b.  The output magnitude
// log2((1 + T) / (1 - T)) over the other edges of a check is log2(G / H) of the set they form: it
// grows like min |y| instead of saturating where 1 - T rounds to zero.  H is zero only when every
// other edge has u = 0 (|y| above 126); the output is then +inf before the clamp to kResCmax, as
// it is whenever all other edges are that reliable, so no input clamp is needed.  (G >= H, so the
// magnitude is >= 0; its absolute value removes a rounding of G / H to just below 1.)
template <int L, class In, class Out>
__device__ __forceinline__ void res_row_rule(In in, unsigned sbit, Out out) {
    float u[L];
    unsigned sgn = 0u;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const float v = in(l);
        const unsigned sv = __float_as_uint(v) & 0x80000000u;
        sgn ^= sv;
        // sign of the edge kept in u's sign bit, |u| = 2^-|v| (flushed to zero above |v| = 126)
        u[l] = __uint_as_float(__float_as_uint(res_ex2(-fabsf(v))) | sv);
    }
    // suffix sets {l, .., L-1}
    float sH[L + 1], sG[L + 1];
    sH[L] = 0.0f;
    sG[L] = 1.0f;
#pragma unroll
    for (int l = L - 1; l >= 0; --l) {
        const float au = fabsf(u[l]);
        sH[l] = fmaf(au, sG[l + 1], sH[l + 1]);
        sG[l] = fmaf(au, sH[l + 1], sG[l + 1]);
    }
    sgn ^= sbit << 31;
    // prefix set {0, .., l-1} joined with the suffix {l+1, .., L-1}
    float pH = 0.0f, pG = 1.0f;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const float eG = fmaf(pG, sG[l + 1], pH * sH[l + 1]);
        const float eH = fmaf(pG, sH[l + 1], pH * sG[l + 1]);
        const float mag = fminf(fabsf(res_lg2(eG * res_rcp(eH))), kResCmax);
        out(l, __uint_as_float(__float_as_uint(mag) ^ ((sgn ^ __float_as_uint(u[l])) & 0x80000000u)));
        const float au = fabsf(u[l]);
        const float nH = fmaf(au, pG, pH);
        pG = fmaf(au, pH, pG);
        pH = nH;
    }
}

// The first iteration in closed form: every variable starts at the prior and every c2v at 0,
// so every edge of a side has the same input v0 and a check's outputs depend only on the
// position l and the check's syndrome bit (bit 1 negates them).  out[l] = the output for
// syndrome bit 0, by the same rule (and so the same bits) as res_row_rule on such a row; out of
// line, as it runs once per trial on two threads.
template <int L>
__device__ __noinline__ void res_first_row(float v0, float *out) {
    res_row_rule<L>([&](int) { return v0; }, 0u, [&](int l, float x) { out[l] = x; });
}

// Check phase, one block row JJ of side SIDE, check offset x: new c2v of the row's L edges
// from A and the old c2v; with `test`, also the parity of the decision bits against the
// target.  Returns whether the tested check failed.
template <int P, int J, int L, class ST, int SIDE, int JJ>
__device__ __forceinline__ bool res_check_row(const ResCode &code, typename ST::T *c2v_side, const float *A_all,
                                              const unsigned *syn_all, int x, bool test) {
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    typename ST::T *c2v = c2v_side + JJ * P + x;
    const float *A = A_all + SIDE * n;
    const int c = JJ * P + x;
    const unsigned sbit = (syn_all[SIDE * mw + (c >> 5)] >> (c & 31)) & 1u;
    unsigned par = 0u;
    res_row_rule<L>(
        [&](int l) {
            const unsigned y = res_map<P>(code.fF[SIDE][JJ][l], code.fG[SIDE][JJ][l], static_cast<unsigned>(x));
            const float a = A[l * P + y];
            par ^= __float_as_uint(a);
            return a - ST::ld(c2v + l * m);
        },
        sbit, [&](int l, float y) { ST::st(c2v + l * m, y); });
    return test && ((par & 1u) != sbit);
}

// Returns this thread's number of tested checks that failed (c2v: the side's [l][c] messages).
template <int P, int J, int L, class ST, int SIDE>
__device__ __forceinline__ int res_check_side(const ResCode &code, typename ST::T *c2v, const float *A,
                                              const unsigned *syn, bool test) {
    int bad = 0;
    for (int x = threadIdx.x; x < P; x += blockDim.x) {
        bad += res_check_row<P, J, L, ST, SIDE, 0>(code, c2v, A, syn, x, test);
        if (J > 1) bad += res_check_row<P, J, L, ST, SIDE, (J > 1 ? 1 : 0)>(code, c2v, A, syn, x, test);
        if (J > 2) bad += res_check_row<P, J, L, ST, SIDE, (J > 2 ? 2 : 0)>(code, c2v, A, syn, x, test);
        if (J > 3) bad += res_check_row<P, J, L, ST, SIDE, (J > 3 ? 3 : 0)>(code, c2v, A, syn, x, test);
    }
    return bad;
}

// Syndrome test of the decisions in A's low bits: this thread's failing checks of one side.
template <int P, int J, int L>
__device__ __forceinline__ int res_test_side(const ResCode &code, const float *A_all, const unsigned *syn_all,
                                             int side) {
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    int bad = 0;
    for (int c = threadIdx.x; c < m; c += blockDim.x) {
        const int j = c / P, x = c - j * P;
        unsigned par = 0;
#pragma unroll
        for (int l = 0; l < L; ++l) {
            const unsigned y = res_map<P>(code.fF[side][j][l], code.fG[side][j][l], static_cast<unsigned>(x));
            par ^= __float_as_uint(A_all[side * n + l * P + y]);
        }
        bad += (par & 1u) != ((syn_all[side * mw + (c >> 5)] >> (c & 31)) & 1u);
    }
    return bad;
}

// Block sums of two per-thread counts through cnt[0..1] (zero on entry; left zero on return).
__device__ __forceinline__ int2 res_block_sum2(int a, int b, int *cnt) {
    a = __reduce_add_sync(0xffffffffu, a);
    b = __reduce_add_sync(0xffffffffu, b);
    if ((threadIdx.x & 31) == 0) {
        if (a) atomicAdd(&cnt[0], a);
        if (b) atomicAdd(&cnt[1], b);
    }
    __syncthreads();
    const int2 r = make_int2(cnt[0], cnt[1]);
    __syncthreads();
    if (threadIdx.x == 0) { cnt[0] = 0; cnt[1] = 0; }
    return r;
}

// log2((c0 + c1 2^-s) / (c2 + c3 2^-s)) for any sign of s, with one ex2 and two lg2:
// the x-bit coupling Gx (s = Mu; c = P0, P2, P1, P3) and the z-bit coupling Hz (s = Lam;
// c = P0, P1, P2, P3), where P = the prior probabilities.
__device__ __forceinline__ float res_couple(float s, float c0, float c1, float c2, float c3) {
    const float e = res_ex2(-fabsf(s));
    const bool pos = s >= 0.0f;
    const float num = pos ? fmaf(c1, e, c0) : fmaf(c0, e, c1);
    const float den = pos ? fmaf(c3, e, c2) : fmaf(c2, e, c3);
    return res_lg2(num) - res_lg2(den);
}

// Variable phase for block column LL, variable offset y: sums, hard decision, new A.
// With HIST the low 6 mantissa bits of A keep the side's decision bits of the last 6
// iterations (bit 0 = this one), and ch1 / ch2 collect whether any decision differs from the
// previous iteration / the one before (the stall and oscillation tests of the learned
// proposal).  The perturbation is below 2^-17 of |A|, far under the FP16 message precision.
template <int P, int J, int L, class ST, int LL, bool HIST>
__device__ __forceinline__ void res_var_col(const ResCode &code, const typename ST::T *c2v,
                                            const typename ST::T *c2vz, float *A, int y,
                                            const float4 *lps, const float4 *prs, unsigned &ch1, unsigned &ch2) {
    const float4 lp = *lps, pr = *prs;   // block constants, re-read from shared memory
    constexpr int m = J * P, n = L * P;
    float Lam = 0.0f, Mu = 0.0f;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const unsigned xx = res_map<P>(code.iF[0][j][LL], code.iG[0][j][LL], static_cast<unsigned>(y));
        const unsigned xz = res_map<P>(code.iF[1][j][LL], code.iG[1][j][LL], static_cast<unsigned>(y));
        Lam += ST::ld(c2v + LL * m + j * P + xx);
        Mu += ST::ld(c2vz + LL * m + j * P + xz);
    }
    const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
    unsigned best = 0;
    float bv = w0;
    if (w1 > bv) { best = 1; bv = w1; }
    if (w2 > bv) { best = 2; bv = w2; }
    if (w3 > bv) { best = 3; }
    const float Gx = res_couple(Mu, pr.x, pr.z, pr.y, pr.w);
    const float Hz = res_couple(Lam, pr.x, pr.y, pr.z, pr.w);
    const int v = LL * P + y;
    if (HIST) {
        const unsigned hx = ((__float_as_uint(A[v]) << 1) | (best & 1u)) & 0x3Fu;
        const unsigned hz = ((__float_as_uint(A[n + v]) << 1) | (best >> 1)) & 0x3Fu;
        // both sides' histories in one word (x in bits 0-5, z in bits 8-13): bit 0 and bit 8 of
        // ch1 / ch2 say whether a decision differs from the previous iteration / the one before
        const unsigned h = hx | (hz << 8);
        ch1 |= h ^ (h >> 1);
        ch2 |= h ^ (h >> 2);
        A[v] = __uint_as_float((__float_as_uint(Lam + Gx) & ~0x3Fu) | hx);
        A[n + v] = __uint_as_float((__float_as_uint(Mu + Hz) & ~0x3Fu) | hz);
    } else {
        A[v] = with_bit(Lam + Gx, best & 1u);
        A[n + v] = with_bit(Mu + Hz, best >> 1);
    }
}

template <int P, int J, int L, class ST, int LL, bool HIST>
__device__ __forceinline__ void res_var_cols(const ResCode &code, const typename ST::T *c2v,
                                             const typename ST::T *c2vz, float *A, int y,
                                             const float4 *lps, const float4 *prs, unsigned &ch1, unsigned &ch2) {
    res_var_col<P, J, L, ST, LL, HIST>(code, c2v, c2vz, A, y, lps, prs, ch1, ch2);
    if constexpr (LL + 1 < L) res_var_cols<P, J, L, ST, LL + 1, HIST>(code, c2v, c2vz, A, y, lps, prs, ch1, ch2);
}

// Block-wide membership test of vec (shared memory, `words` 64-bit words) in a row space
// (in_row_space, jointbp_ets.cpp:904-920), run by warp 0 with the same reduction as the slot
// engine's classifier.
__device__ __forceinline__ bool res_in_row_space(uint64_t *vec, int words, const uint64_t *rows, const int *pivot_row,
                                                 int *flag) {
    if (threadIdx.x < 32) {
        const bool r = warp_in_row_space(vec, words, rows, pivot_row);
        if (threadIdx.x == 0) *flag = r ? 1 : 0;
    }
    __syncthreads();
    const bool r = *flag != 0;
    __syncthreads();
    return r;
}

// |LLR| of the x and z bits of every variable from the current c2v (the slot engine's FP32
// keys, base 2), as doubles for the OSD column order.
template <int P, int J, int L, class ST>
__device__ void res_abs_llr(const ResCode &code, const typename ST::T *c2v, const typename ST::T *c2vz, const float4 lp,
                            double *llr) {
    constexpr int m = J * P, n = L * P;
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        const int l = v / P, y = v - l * P;
        float Lam = 0.0f, Mu = 0.0f;
        for (int j = 0; j < J; ++j) {
            const unsigned xx = res_map<P>(code.iF[0][j][l], code.iG[0][j][l], static_cast<unsigned>(y));
            const unsigned xz = res_map<P>(code.iF[1][j][l], code.iG[1][j][l], static_cast<unsigned>(y));
            Lam += ST::ld(c2v + l * m + j * P + xx);
            Mu += ST::ld(c2vz + l * m + j * P + xz);
        }
        const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
        llr[v] = fabsf(res_lse2(w1, w3) - res_lse2(w0, w2));
        llr[n + v] = fabsf(res_lse2(w2, w3) - res_lse2(w0, w1));
    }
}

// Per-qubit features of the stalled state at iteration `it` (mlp.cuh, include/jbp_b200.h):
// the normalized log2 weights of I, X, Z, Y from the current c2v (w - max w, / 16, >= -4), the
// x-bit and z-bit flips over the last 5 iterations (decision history in A's low bits, / 5),
// and the unsatisfied X and Z checks at the qubit (/ 3, from psh.est against psh.tgt).
template <int P, int J, int L, class ST>
__device__ void res_features(const ResCode &code, const DevCode &dc, const typename ST::T *c2v,
                             const typename ST::T *c2vz, const float *A,
                             const float4 lp, int it, const PpShared &psh, float *feat) {
    constexpr int m = J * P, n = L * P;
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        const int l = v / P, y = v - l * P;
        float Lam = 0.0f, Mu = 0.0f;
        for (int j = 0; j < J; ++j) {
            const unsigned xx = res_map<P>(code.iF[0][j][l], code.iG[0][j][l], static_cast<unsigned>(y));
            const unsigned xz = res_map<P>(code.iF[1][j][l], code.iG[1][j][l], static_cast<unsigned>(y));
            Lam += ST::ld(c2v + l * m + j * P + xx);
            Mu += ST::ld(c2vz + l * m + j * P + xz);
        }
        const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
        const float mx = fmaxf(fmaxf(w0, w1), fmaxf(w2, w3));
        float *f = feat + static_cast<size_t>(v) * kMlpIn;
        f[0] = fmaxf((w0 - mx) * 0.0625f, -4.0f);
        f[1] = fmaxf((w1 - mx) * 0.0625f, -4.0f);
        f[2] = fmaxf((w2 - mx) * 0.0625f, -4.0f);
        f[3] = fmaxf((w3 - mx) * 0.0625f, -4.0f);
        // flips over the last 5 iterations, from the decision history in A's low bits
        const unsigned hx = __float_as_uint(A[v]) & 0x3Fu, hz = __float_as_uint(A[n + v]) & 0x3Fu;
        const int span = min(5, it - 1);
        const unsigned msk = (1u << max(span, 0)) - 1u;
        f[4] = __popc((hx ^ (hx >> 1)) & msk) * 0.2f;
        f[5] = __popc((hz ^ (hz >> 1)) & msk) * 0.2f;
    }
    for (int side = 0; side < 2; ++side) {
        blk_side_diff(dc, psh, side);
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            int u = 0;
            for (int k = 0; k < dc.s[side].dv; ++k) {
                const int c = var_check(dc, side, v, k);
                if (c >= 0) u += psh.diff[c];
            }
            feat[static_cast<size_t>(v) * kMlpIn + 6 + side] = u * (1.0f / 3.0f);
        }
        __syncthreads();
    }
}

// Post-processing working areas of this block: shared arrays after the trial state, and the
// per-block global scratch (recomputed where needed so that the BP loop keeps no pointers).
struct ResPpPtrs {
    PpShared psh;
    PpScratch psc;
    uint8_t *ring;
    double *llr;
    float *feat;
    int R;
};

template <int P, int J, int L, class ST>
__device__ __forceinline__ ResPpPtrs res_pp_ptrs(const ResRun &run, unsigned char *smem) {
    constexpr int m = J * P, n = L * P;
    ResPpPtrs q;
    q.R = max(run.flip_hist + 1, run.learned_from > 0 ? 6 : 3);
    q.psh = pp_shared_carve(smem + run.pp_smem_base, n, 2 * m, m);
    unsigned char *g = run.pp_scratch + run.pp_scratch_stride * blockIdx.x;
    q.psc = pp_scratch_carve(g, n, m);
    q.ring = g + pp_align(pp_scratch_bytes(n, m));
    q.llr = reinterpret_cast<double *>(q.ring + pp_align(static_cast<size_t>(q.R) * n));
    q.feat = reinterpret_cast<float *>(reinterpret_cast<unsigned char *>(q.llr) + pp_align(16ull * n));
    return q;
}

// The proposal's solve: per side, the columns in ascending key order (key[side * n + v]) enter
// the incremental GF(2) elimination of the OSD stage over at most run.learned_cols of them; the
// correction is kept only if unique, of weight <= 30 (the reference's OSD acceptance,
// jointbp_ets.cpp:3056-3073) and both syndromes then match, with the corrected decisions
// written into A's low bits.  Returns whether it was accepted.
__device__ __forceinline__ bool res_learned_solve(const ResRun &run, const PpShared &psh, const PpScratch &psc,
                                                  const double *key, float *A, int n) {
    int left = 0;
    for (int side = 0; side < 2; ++side) {
        if (blk_side_diff(run.dc, psh, side) == 0) continue;
        if (!blk_osd_side(run.dc, key + static_cast<size_t>(side) * n, psh, psc, side, run.learned_cols)) ++left;
    }
    const bool accepted = left == 0;
    if (accepted)
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            A[v] = with_bit(A[v], psh.est[v] & 1u);
            A[n + v] = with_bit(A[n + v], (psh.est[v] >> 1) & 1u);
        }
    // a rejected proposal leaves nothing behind: later stages reload the estimate from the ring
    __syncthreads();
    return accepted;
}

// The learned flip proposal on the stalled state of iteration `it` (rare path, kept out of
// line so that the BP loop's registers are not shaped by it).  In collection mode it records
// the samples and returns false; otherwise it solves the proposed flip sets and returns true,
// with the corrected decisions in A's low bits, only if both syndromes then match exactly.
template <int P, int J, int L, class ST>
__device__ __noinline__ bool res_learned_attempt(const ResCode &code, const ResRun &run, unsigned char *smem,
                                                 typename ST::T *c2v, typename ST::T *c2vz, float *A, const unsigned *syn,
                                                 const uint8_t *err,
                                                 bool have_err, int it, long long t, const float4 lp) {
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    const ResPpPtrs q = res_pp_ptrs<P, J, L, ST>(run, smem);
    const PpShared &psh = q.psh;
    const PpScratch &psc = q.psc;
    float *feat = q.feat;
    double *llr_scratch = q.llr;
    for (int v = threadIdx.x; v < n; v += blockDim.x)
        psh.est[v] = static_cast<uint8_t>((__float_as_uint(A[v]) & 1u) | ((__float_as_uint(A[n + v]) & 1u) << 1));
    for (int r = threadIdx.x; r < 2 * m; r += blockDim.x) {
        const int side = r >= m, c = r - side * m;
        psh.tgt[r] = static_cast<uint8_t>((syn[side * mw + (c >> 5)] >> (c & 31)) & 1u);
    }
    __syncthreads();
    if (run.learned_order == 1 && !run.collect) {
        // the ablation baseline: the same trigger, elimination and acceptance, with the columns
        // in the decoder's own reliability order (ascending |LLR| of the current totals)
        if (threadIdx.x == 0) atomicAdd(&run.cnt->learned_attempts, 1ull);
        double *key = reinterpret_cast<double *>(feat);
        res_abs_llr<P, J, L, ST>(code, c2v, c2vz, lp, key);
        __syncthreads();
        return res_learned_solve(run, psh, psc, key, A, n);
    }
    res_features<P, J, L, ST>(code, run.dc, c2v, c2vz, A, lp, it, psh, feat);
    if (run.collect) {
        if (threadIdx.x == 0) atomicAdd(&run.cnt->learned_attempts, 1ull);   // stalls recorded
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            const float *f = feat + static_cast<size_t>(v) * kMlpIn;
            const unsigned lab = have_err ? (err[v] ^ psh.est[v]) : 0u;
            const unsigned h = static_cast<unsigned>(splitmix64(static_cast<unsigned long long>(t) * 1315423911ull +
                                                                static_cast<unsigned long long>(it) * 9216ull + v));
            if (!(lab || f[6] + f[7] > 0.0f || h % run.collect_every == 0u)) continue;
            const unsigned long long q = atomicAdd(run.col_count, 1ull);
            if (q >= static_cast<unsigned long long>(run.col_cap)) continue;
            for (int kk = 0; kk < kMlpIn; ++kk) run.col_x[q * kMlpIn + kk] = f[kk];
            run.col_y[q * 2] = static_cast<float>(lab & 1u);
            run.col_y[q * 2 + 1] = static_cast<float>((lab >> 1) & 1u);
        }
        __syncthreads();
        return false;
    }
    if (threadIdx.x == 0) atomicAdd(&run.cnt->learned_attempts, 1ull);
    // logits of every qubit (x-flip, z-flip) into the |LLR| scratch, which is free here
    float *logit = reinterpret_cast<float *>(llr_scratch);
    const int wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int tile = wid; tile * 16 < n; tile += nwarps) {
        auto fget = [&](int row, int kk) -> float {
            const int v = tile * 16 + row;
            return v < n ? feat[static_cast<size_t>(v) * kMlpIn + kk] : 0.0f;
        };
        float o[4];
        mlp_tile(run.mlp, fget, o);
        if ((lane & 3) == 0) {
            const int v0 = tile * 16 + (lane >> 2), v1 = v0 + 8;
            if (v0 < n) { logit[2 * v0] = o[0]; logit[2 * v0 + 1] = o[1]; }
            if (v1 < n) { logit[2 * v1] = o[2]; logit[2 * v1 + 1] = o[3]; }
        }
    }
    __syncthreads();
    // The proposal per side: the qubits in the order of their learned score (most likely wrong
    // first) enter the incremental GF(2) elimination of the OSD stage (blk_osd_side); the first
    // prefix whose span holds the side's syndrome difference gives the flips, kept only if the
    // solution is unique and of weight <= 30 (the reference's OSD acceptance), so that the side's
    // syndrome then matches.  Keys: 1 - sigmoid(logit) > 0, ascending = most likely wrong first.
    double *key = reinterpret_cast<double *>(feat);   // the features are no longer needed
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        key[v] = 1.0 / (1.0 + exp(static_cast<double>(logit[2 * v])));
        key[n + v] = 1.0 / (1.0 + exp(static_cast<double>(logit[2 * v + 1])));
    }
    __syncthreads();
    return res_learned_solve(run, psh, psc, key, A, n);
}

// One post-processing pass (in-loop attempt or post-BP) on the decisions of iteration `it`
// (rare path, out of line).  Returns the trial's result flags when the pass ends the trial
// (in-loop success, or the post-BP pass), with the corrected decisions in A's low bits;
// 0 when BP continues.
template <int P, int J, int L, class ST>
__device__ __forceinline__ int res_pp_attempt(const ResCode &code, const ResRun &run, const ResPpPtrs &q,
                                              const typename ST::T *c2v, const typename ST::T *c2vz, float *A,
                                              const unsigned *syn,
                                              const uint8_t *cur, int it, int mode, int act_k, const float4 lp) {
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    const PpShared &psh = q.psh;
    const PpScratch &psc = q.psc;
    const uint8_t *ring = q.ring;
    const int R = q.R;
    double *llr = q.llr;
    for (int v = threadIdx.x; v < n; v += blockDim.x) psh.est[v] = cur[v];
    for (int r = threadIdx.x; r < 2 * m; r += blockDim.x) {
        const int side = r >= m, c = r - side * m;
        psh.tgt[r] = static_cast<uint8_t>((syn[side * mw + (c >> 5)] >> (c & 31)) & 1u);
    }
    res_abs_llr<P, J, L, ST>(code, c2v, c2vz, lp, llr);
    __syncthreads();
    const RingHistory hist{ring, R};
    const PpOutcome o = blk_pp_stages(run.dc, run.ets, hist, run.flip_hist, act_k, it, llr, llr + n, psh, psc);
    const bool in_loop_success = mode == kPpInLoop && o.ok;
    const bool post = !in_loop_success && (mode == kPpPost || it >= run.max_iter);
    int rf = 0;
    if (in_loop_success || post) {
        for (int v = threadIdx.x; v < n; v += blockDim.x) {
            A[v] = with_bit(A[v], psh.est[v] & 1u);
            A[n + v] = with_bit(A[n + v], (psh.est[v] >> 1) & 1u);
        }
        rf = pp_result_flags(o, in_loop_success);
    }
    __syncthreads();
    return rf;
}

// One iteration from `slow_from` on (post-processing instantiations; rare path, out of line):
// syndrome test after the variable phase, the decision ring, the stall / oscillation /
// us-signal triggers (jointbp_ets.cpp:2521-2633), the learned proposal and the
// post-processing pass.  Returns 0 to continue BP, else the trial's result flags (-1 for
// a finished trial without any flag: not converged, no stage succeeded).
template <int P, int J, int L, class ST>
__device__ __noinline__ int res_slow_step(const ResCode &code, const ResRun &run, unsigned char *smem,
                                          typename ST::T *c2v, typename ST::T *c2vz, float *A, const unsigned *syn,
                                          const uint8_t *err,
                                          bool have_err, int it, long long t, const float4 lp,
                                          unsigned short *us_hist, int *pp_sh, int *ints, bool slow) {
    constexpr int n = L * P;
    const ResPpPtrs q = res_pp_ptrs<P, J, L, ST>(run, smem);
    const int R = q.R;
    const int2 us = res_block_sum2(res_test_side<P, J, L>(code, A, syn, 0), res_test_side<P, J, L>(code, A, syn, 1),
                                   ints);
    if (us.x + us.y == 0) return kResSyndromeOk | kResBpOk;
    if (!slow) {
        // a stall before slow_from: only the learned proposal (the fused test of the next check
        // phase records this iteration's us signal)
        if (max(us.x, us.y) > kLearnedMaxUnsat) return 0;
        __syncthreads();
        if (threadIdx.x == 0) pp_sh[3] += 1;
        return res_learned_attempt<P, J, L, ST>(code, run, smem, c2v, c2vz, A, syn, err, have_err, it, t, lp)
                   ? (kResSyndromeOk | kResLearned) : 0;
    }
    // this iteration's decisions: a byte per qubit in the global ring (the flip window reads it)
    // and x / z bit planes in shared memory, 32 qubits per word, for the stall tests
    constexpr int W = (n + 31) / 32;
    uint32_t *planes = reinterpret_cast<uint32_t *>(smem + res_plane_offset(run.pp_smem_base, n, J * P));
    uint32_t *pc = planes + (it % 3) * 2 * W;
    const uint32_t *pl1 = planes + ((it + 2) % 3) * 2 * W, *pl2 = planes + ((it + 1) % 3) * 2 * W;
    uint8_t *cur = q.ring + static_cast<size_t>(it % R) * n;
    for (int base = (threadIdx.x >> 5) * 32; base < n; base += blockDim.x) {
        const int v = base + (threadIdx.x & 31);
        const unsigned xb = v < n ? __float_as_uint(A[v]) & 1u : 0u, zb = v < n ? __float_as_uint(A[n + v]) & 1u : 0u;
        if (v < n) cur[v] = static_cast<uint8_t>(xb | (zb << 1));
        const unsigned xw = __ballot_sync(0xffffffffu, xb), zw = __ballot_sync(0xffffffffu, zb);
        if ((threadIdx.x & 31) == 0) {
            pc[base >> 5] = xw;
            pc[W + (base >> 5)] = zw;
        }
    }
    __syncthreads();
    // est == prev_est / prev_prev_est (jointbp_ets.cpp:2555-2556), word by word
    bool s1 = it >= 2, s2 = it >= 3;
    for (int w = threadIdx.x; w < 2 * W; w += blockDim.x) {
        if (s1) s1 = pc[w] == pl1[w];
        if (s2) s2 = pc[w] == pl2[w];
    }
    const bool same = __syncthreads_and(s1) != 0;
    const bool pp2 = __syncthreads_and(s2) != 0;
    if (threadIdx.x < 32) {
        // the triggers, in warp 0 (the us-signal test over its 100 samples by the whole warp)
        const int sig = max(us.x, us.y);
        if (threadIdx.x == 0) us_hist[it % 100] = static_cast<unsigned short>(min(sig, 65535));
        __syncwarp();
        const bool allow = it >= 100 || it == run.max_iter;
        int st = pp_sh[2];
        const bool us_osc = !(st & 4) && allow && us_oscillation_warp(us_hist, it);   // warp-uniform
        if (threadIdx.x == 0) {
            const bool osc = pp2 && !same;
            bool act = false;
            if (!(st & 1) && (same || it == run.max_iter) && allow) { st |= 1; act = true; }
            if (!(st & 2) && osc && allow) { st |= 2; act = true; }
            if (us_osc) { st |= 4; act = true; }
            pp_sh[2] = st;
            if (act && pp_sh[1] == 0 && run.flip_hist > 0) pp_sh[1] = it;
            pp_sh[0] = (st && sig <= 20) ? kPpInLoop : (it >= run.max_iter ? kPpPost : 0);
        }
    }
    __syncthreads();
    // learned flip proposal at a stall (decisions unchanged or oscillating)
    if (run.learned_from > 0 && it >= run.learned_from && (same || (pp2 && !same)) && pp_sh[3] < kLearnedTries &&
        max(us.x, us.y) <= kLearnedMaxUnsat) {
        __syncthreads();
        if (threadIdx.x == 0) pp_sh[3] += 1;
        if (res_learned_attempt<P, J, L, ST>(code, run, smem, c2v, c2vz, A, syn, err, have_err, it, t, lp))
            return kResSyndromeOk | kResLearned;
    }
    const int mode = pp_sh[0];
    if (mode) {
        const int r2 = res_pp_attempt<P, J, L, ST>(code, run, q, c2v, c2vz, A, syn, cur, it, mode, pp_sh[1], lp);
        if (r2) return r2;
    }
    return it >= run.max_iter ? -1 : 0;
}

// Final LLRs of a trial (diagnostics of the precision report; out of line): natural log of
// P(bit = 1) / P(bit = 0) of the x and z bits from the c2v in shared memory when the trial
// ends (those of its last variable update when the syndrome is tested only at max_iter).
template <int P, int J, int L, class ST>
__device__ __noinline__ void res_write_llr(const ResCode &code, const typename ST::T *c2v, const typename ST::T *c2vz,
                                           const float4 lp,
                                           float *out) {
    constexpr int m = J * P, n = L * P;
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        const int l = v / P, y = v - l * P;
        float Lam = 0.0f, Mu = 0.0f;
        for (int j = 0; j < J; ++j) {
            Lam += ST::ld(c2v + l * m + j * P + res_map<P>(code.iF[0][j][l], code.iG[0][j][l], y));
            Mu += ST::ld(c2vz + l * m + j * P + res_map<P>(code.iF[1][j][l], code.iG[1][j][l], y));
        }
        const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
        out[2 * v] = (res_lse2(w1, w3) - res_lse2(w0, w2)) * 0.69314718f;
        out[2 * v + 1] = (res_lse2(w2, w3) - res_lse2(w0, w1)) * 0.69314718f;
    }
}

// Prior of a trial (error rate pt; thread 0, once per run or per trial; out of line): FP64 as
// the slot engine's refill, then its log2 weights and probabilities in FP32.
__device__ __noinline__ void res_set_prior(int use_prior, const double *prior4, double pt, float4 *lp, float4 *pr,
                                           float *lpx, float *lpz) {
    double q[4];
    if (use_prior) {
        for (int i = 0; i < 4; ++i) q[i] = prior4[i];
    } else {
        q[0] = 1.0 - pt; q[1] = pt / 3.0; q[2] = q[1]; q[3] = q[1];
        const double s = ((q[0] + q[1]) + q[2]) + q[3];
        for (int i = 0; i < 4; ++i) q[i] = s > 0.0 ? q[i] / s : 0.25;
    }
    for (int i = 0; i < 4; ++i) q[i] = fmax(q[i], 1e-30);
    *lp = make_float4(static_cast<float>(log2(q[0])), static_cast<float>(log2(q[1])), static_cast<float>(log2(q[2])),
                      static_cast<float>(log2(q[3])));
    *pr = make_float4(static_cast<float>(q[0]), static_cast<float>(q[1]), static_cast<float>(q[2]),
                      static_cast<float>(q[3]));
    *lpx = static_cast<float>(log2((q[0] + q[2]) / (q[1] + q[3])));
    *lpz = static_cast<float>(log2((q[0] + q[1]) / (q[2] + q[3])));
}

// GC: the Z side's c2v live in a per-block global scratch (L2-resident) instead of shared
// memory -- the FP32-message instantiation, whose 221 KB of c2v per trial do not all fit beside
// the rest (the X side's 110.6 KB do).
template <int P, int J, int L, class ST, bool PP, bool LEARNED, bool GC = false>
__global__ void __launch_bounds__(kResThreads, 1)
    k_resident(const __grid_constant__ ResCode code, const __grid_constant__ ResRun run) {
    extern __shared__ __align__(16) unsigned char res_smem[];
    using T = typename ST::T;
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    T *const c2v = reinterpret_cast<T *>(res_smem);   // side X, [l][c]
    T *const c2vz = GC ? reinterpret_cast<T *>(run.c2v_scratch + run.c2v_stride * blockIdx.x)
                       : c2v + L * m;                   // side Z
    constexpr size_t c2v_bytes = ((GC ? 1ull : 2ull) * L * m * sizeof(T) + 15) / 16 * 16;
    float *const A = reinterpret_cast<float *>(res_smem + c2v_bytes);
    uint8_t *const err = res_smem + c2v_bytes + 2ull * n * 4;
    unsigned *const syn = reinterpret_cast<unsigned *>(err + (n + 15) / 16 * 16);
    int *const ints = reinterpret_cast<int *>(syn + (2 * mw + 3) / 4 * 4);   // 16 ints
    __shared__ long long trial_sh;
    __shared__ float4 lp_sh, pr_sh;
    __shared__ float lpx_sh, lpz_sh;
    __shared__ float first_sh[2][L];   // first-iteration c2v of each position (syndrome bit 0)
    __shared__ unsigned short us_hist[100];
    __shared__ int us_cnt[2][2];   // unsatisfied checks per side of the tested iteration, by its parity
    __shared__ int pp_sh[4];   // mode, act_k, pstate
    const bool have_err = run.source != kSrcSyndromes;

    // post-processing state (PP instantiations)
    constexpr bool learned = LEARNED && PP;   // the host launches this instantiation only with a model
    const int llr_from = min(100, run.max_iter);
    const int slow_from = PP ? max(1, llr_from - 2) : 0x7fffffff;

    __shared__ double pt_sh;
    __shared__ int abort_sh;          // 1: the run budget ran out during this trial; 2: abort requested
    // global-timer end of the run budget (0 = none), in shared memory so that the BP loop keeps
    // no register for it
    __shared__ unsigned long long deadline_sh;
    unsigned long long claimed = 0;   // thread 0: the next trial index this block has claimed
    if (threadIdx.x == 0) {
        deadline_sh = run.budget_ns ? dev_globaltimer() + run.budget_ns : 0ull;
        claimed = atomicAdd(&run.cnt->next_trial, 1ull);
        res_set_prior(run.use_prior, run.prior4, run.p, &lp_sh, &pr_sh, &lpx_sh, &lpz_sh);
        for (int i = 0; i < 16; ++i) ints[i] = 0;
    }
    __syncthreads();

    for (;;) {
        if (threadIdx.x == 0) {
            // the index claimed at the previous trial's start; the next claim's latency overlaps
            // this trial
            const unsigned long long k = claimed;
            claimed = atomicAdd(&run.cnt->next_trial, 1ull);
            trial_sh = k < static_cast<unsigned long long>(run.ntrials) ? static_cast<long long>(k) : -1;
            if (trial_sh >= 0 && deadline_sh && dev_globaltimer() > deadline_sh) {
                trial_sh = -1;   // the run budget is spent: no further trial
                atomicAdd(&run.cnt->watchdog, 1ull);
            } else if (trial_sh >= 0 && k % kResAbortEvery == 0 && *run.abort_flag) {
                trial_sh = -1;   // abort requested: no further trial
                atomicAdd(&run.cnt->aborted, 1ull);
            }
            abort_sh = 0;
            pp_sh[1] = 0;   // act_k
            pp_sh[2] = 0;   // pstate
            pp_sh[3] = 0;   // learned proposals tried
            us_cnt[0][0] = us_cnt[0][1] = us_cnt[1][0] = us_cnt[1][1] = 0;
        }
        __syncthreads();
        const long long k = trial_sh;
        if (k < 0) break;
        const long long t = run.trial_list ? run.trial_list[k] : run.first_trial + k;
        const long long local = t - run.first_trial;
        if (run.p_max > run.p) {
            if (threadIdx.x == 0) {
                pt_sh = trial_p(run.p, run.p_max, run.seed, t);
                res_set_prior(run.use_prior, run.prior4, pt_sh, &lp_sh, &pr_sh, &lpx_sh, &lpz_sh);
            }
            __syncthreads();
        } else if (threadIdx.x == 0) {
            pt_sh = run.p;
        }
        const double pt = run.p_max > run.p ? pt_sh : run.p;

        // ---- error and target syndrome
        if (!have_err)
            for (int w = threadIdx.x; w < 2 * mw; w += blockDim.x) syn[w] = 0u;
        if (run.source == kSrcPhilox) {
            for (int v2 = threadIdx.x; 2 * v2 < n; v2 += blockDim.x) {
                uint8_t e0, e1;
                sample_philox_pair(run.seed, t, v2, pt, e0, e1);
                err[2 * v2] = e0;
                if (2 * v2 + 1 < n) err[2 * v2 + 1] = e1;
            }
        } else if (run.source == kSrcErrors) {
            const uint8_t *src = run.src_err + local * n;
            if ((n & 15) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
                // 16-byte loads; a byte above 3 is reported and masked
                const uint4 *s16 = reinterpret_cast<const uint4 *>(src);
                uint4 *d16 = reinterpret_cast<uint4 *>(err);
                unsigned badw = 0u;
                for (int i = threadIdx.x; i < n / 16; i += blockDim.x) {
                    uint4 w = s16[i];
                    badw |= (w.x | w.y | w.z | w.w) & 0xFCFCFCFCu;
                    w.x &= 0x03030303u; w.y &= 0x03030303u; w.z &= 0x03030303u; w.w &= 0x03030303u;
                    d16[i] = w;
                }
                if (badw) atomicAdd(&run.cnt->bad_input, 1ull);
            } else {
                for (int v = threadIdx.x; v < n; v += blockDim.x) {
                    const uint8_t e = src[v];
                    if (e > 3) atomicAdd(&run.cnt->bad_input, 1ull);
                    err[v] = e & 3;
                }
            }
        } else if (run.source == kSrcMt19937) {
            if (threadIdx.x < 32) warp_mt_trial(reinterpret_cast<unsigned long long *>(A), run.seed, t, pt, n, err);
        }
        __syncthreads();
        if (run.source == kSrcSyndromes) {
            for (int c = threadIdx.x; c < m; c += blockDim.x) {
                if (run.src_sx[local * m + c] & 1) atomicOr(&syn[c >> 5], 1u << (c & 31));
                if (run.src_sz[local * m + c] & 1) atomicOr(&syn[mw + (c >> 5)], 1u << (c & 31));
            }
        } else {
            // one syndrome word per warp and step: the 32 lanes take 32 consecutive checks of
            // one side (m is a multiple of 32), so row r0 / 32 is word side * mw + c / 32
            static_assert(m % 32 == 0 && kResThreads % 32 == 0, "warp-aligned syndrome words");
            for (int r0 = threadIdx.x & ~31; r0 < 2 * m; r0 += blockDim.x) {
                const int r = r0 + (threadIdx.x & 31);
                const int side = r >= m, c = r - side * m, j = c / P, x = c - j * P;
                unsigned par = 0;
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    const unsigned y = res_map<P>(code.fF[side][j][l], code.fG[side][j][l], static_cast<unsigned>(x));
                    par ^= err[l * P + y];
                }
                const unsigned word = __ballot_sync(0xffffffffu, (par >> side) & 1u);
                if ((threadIdx.x & 31) == 0) syn[r0 >> 5] = word;
            }
        }
        // ---- BP state: A = prior LLR of each side's bit, and the c2v of the first iteration in
        // closed form (res_first_row): every edge of a side starts from the same input
        {
            const float ax = with_bit(lpx_sh, 0u), az = with_bit(lpz_sh, 0u);
            for (int v = threadIdx.x; v < n; v += blockDim.x) { A[v] = ax; A[n + v] = az; }
            if (threadIdx.x < 2) res_first_row<L>(threadIdx.x ? az : ax, first_sh[threadIdx.x]);
        }
        __syncthreads();
        for (int r = threadIdx.x; r < 2 * m; r += blockDim.x) {
            const int side = r >= m, c = r - side * m;
            const bool neg = (syn[side * mw + (c >> 5)] >> (c & 31)) & 1u;
#pragma unroll
            for (int l = 0; l < L; ++l)
                ST::st((side ? c2vz : c2v) + l * m + c, neg ? -first_sh[side][l] : first_sh[side][l]);
        }
        __syncthreads();

        // ---- BP iterations (it = completed iterations).  Until slow_from the check phase of
        // iteration it+1 also tests the decisions of iteration it; from slow_from on (only with
        // post-processing) each iteration is tested after its variable phase and feeds the stall
        // triggers, the flip window and the post-processing attempts (jointbp_ets.cpp:2521-2633).
        int it = 0, rf = 0, iters = run.max_iter;
        bool stall = false;   // (learned) decisions of iteration `it` equal those of it-1, or of it-2
        int near = 0x7fffffff;   // threads with a failing check at the last test
        for (;;) {
            const bool fused = it >= 1 && it < slow_from &&
                               (it >= run.max_iter ||
                                (it > run.check_warmup && (it - run.check_warmup) % run.check_interval == 0));
            // Close to convergence the test runs on its own first: when it passes, the check
            // phase it would have been fused into is not computed (the same decisions and
            // iteration counts either way; only the c2v left behind differ).
            const bool sep = fused && it < run.max_iter && near <= kResSepTest;
            int bx = 0, bz = 0;
            if (it < run.max_iter && !sep && it > 0) {   // iteration 1's check phase is the closed form above
                bx = res_check_side<P, J, L, ST, 0>(code, c2v, A, syn, fused);
                bz = res_check_side<P, J, L, ST, 1>(code, c2vz, A, syn, fused);
            } else if (fused) {
                bx = res_test_side<P, J, L>(code, A, syn, 0);
                bz = res_test_side<P, J, L>(code, A, syn, 1);
            }
            if (PP && fused) {
                // per-side counts of the tested iteration (the us signal): one atomic per warp
                const int wx = __reduce_add_sync(0xffffffffu, bx), wz = __reduce_add_sync(0xffffffffu, bz);
                if ((threadIdx.x & 31) == 0) {
                    if (wx) atomicAdd(&us_cnt[it & 1][0], wx);
                    if (wz) atomicAdd(&us_cnt[it & 1][1], wz);
                }
            }
            // run budget: thread 0 looks at the timer every kResBudgetEvery iterations; the flag
            // is read by every thread after the barrier below (at the iteration-limit exit, which
            // keeps the loop's register use as it was) and written again only after the next
            // variable phase's barrier
            if (threadIdx.x == 0 && it % kResBudgetEvery == kResBudgetEvery - 1) {
                if (deadline_sh && dev_globaltimer() > deadline_sh) abort_sh = 1;
                else if (it >= kResAbortFrom && *run.abort_flag) abort_sh = 2;
            }
            const int nbad = __syncthreads_count(bx + bz != 0);
            if (fused) {
                if (nbad == 0) { rf = kResSyndromeOk | kResBpOk; iters = it; break; }
                near = nbad;
                if (PP && threadIdx.x == 0)
                    us_hist[it % 100] =
                        static_cast<unsigned short>(min(max(us_cnt[it & 1][0], us_cnt[it & 1][1]), 65535));
            }
            if (it >= run.max_iter || abort_sh) break;
            if (sep) {
                res_check_side<P, J, L, ST, 0>(code, c2v, A, syn, false);
                res_check_side<P, J, L, ST, 1>(code, c2vz, A, syn, false);
                __syncthreads();
            }
            if (PP && threadIdx.x == 0) us_cnt[(it + 1) & 1][0] = us_cnt[(it + 1) & 1][1] = 0;   // next test's slot
            if constexpr (learned) {
                unsigned ch1 = 0u, ch2 = 0u;
                for (int y = threadIdx.x; y < P; y += blockDim.x)
                    res_var_cols<P, J, L, ST, 0, true>(code, c2v, c2vz, A, y, &lp_sh, &pr_sh, ch1, ch2);
                const bool d1 = __syncthreads_or(ch1 & 0x101u) != 0;
                const bool d2 = __syncthreads_or(ch2 & 0x101u) != 0;
                stall = it + 1 >= 3 && (!d1 || !d2);
            } else {
                unsigned ch1 = 0u, ch2 = 0u;
                for (int y = threadIdx.x; y < P; y += blockDim.x)
                    res_var_cols<P, J, L, ST, 0, false>(code, c2v, c2vz, A, y, &lp_sh, &pr_sh, ch1, ch2);
                __syncthreads();
            }
            ++it;
            // rare paths, one out-of-line call site: iterations from slow_from on, and (learned)
            // a stall of this iteration, whose c2v are still those its decisions came from
            const bool slow = PP && it >= slow_from;
            if (slow || (learned && stall && it >= run.learned_from && pp_sh[3] < kLearnedTries)) {
                const int r3 = res_slow_step<P, J, L, ST>(code, run, res_smem, c2v, c2vz, A, syn, err, have_err, it, t,
                                                         lp_sh,
                                                         us_hist, pp_sh, ints, slow);
                if (r3 != 0) {
                    rf = r3 < 0 ? 0 : r3;
                    iters = it;
                    break;
                }
            }
        }
        if (abort_sh && rf == 0 && it < run.max_iter) {
            // abandoned for the run budget: not classified, not counted; the block stops
            if (threadIdx.x == 0) atomicAdd(abort_sh == 2 ? &run.cnt->aborted : &run.cnt->watchdog, 1ull);
            break;
        }
        const bool ok = (rf & kResSyndromeOk) != 0;
        if (run.llr_out) res_write_llr<P, J, L, ST>(code, c2v, c2vz, lp_sh, run.llr_out + local * n * 2);

        // ---- classification (jointbp_ets.cpp:6199-6245): exact, stabilizer-equivalent residual
        const int words = (n + 63) / 64, w32 = 2 * words;
        unsigned *rx = reinterpret_cast<unsigned *>(c2v);     // BP state is no longer needed
        unsigned *rz = rx + w32;
        for (int w = threadIdx.x; w < 2 * w32; w += blockDim.x) rx[w] = 0u;
        __syncthreads();
        bool exact = true;
        for (int base = (threadIdx.x >> 5) * 32; base < n; base += blockDim.x) {
            const int v = base + (threadIdx.x & 31);
            const bool in = v < n;
            const unsigned e = in ? ((__float_as_uint(A[v]) & 1u) | ((__float_as_uint(A[n + v]) & 1u) << 1)) : 0u;
            const unsigned tv = in && have_err ? err[v] : e;
            if (in && run.est_out) run.est_out[local * n + v] = static_cast<uint8_t>(e);
            exact &= tv == e;
            const unsigned bxm = __ballot_sync(0xffffffffu, ((tv ^ e) & 1u) != 0);
            const unsigned bzm = __ballot_sync(0xffffffffu, ((tv ^ e) & 2u) != 0);
            if ((threadIdx.x & 31) == 0) { rx[base >> 5] = bxm; rz[base >> 5] = bzm; }
        }
        exact = __syncthreads_and(exact) && have_err;
        bool stab = false;
        if (have_err && ok && !exact) {
            stab = res_in_row_space(reinterpret_cast<uint64_t *>(rx), words, code.basis_rows[1], code.pivot_row[1],
                                    ints + 8);
            if (stab)
                stab = res_in_row_space(reinterpret_cast<uint64_t *>(rz), words, code.basis_rows[0], code.pivot_row[0],
                                        ints + 8);
        } else if (have_err && ok) {
            stab = true;   // exact: the residual is zero
        }
        const bool success = have_err ? (ok && stab) : ok;
        if (threadIdx.x == 0)
            account_trial(run.cnt, run.hist, run.res_out, run.max_iter, local, iters, rf, ok, success, exact, stab);
        __syncthreads();
    }
}

}  // namespace jbp
