// Trial-resident BP: one persistent thread block per SM owns one trial at a time and keeps
// all of its BP state in shared memory, from sampling to classification.  No message ever
// travels to HBM; the only global traffic per trial is its error (or syndrome), its result
// record and, when asked for, its estimate.
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
//     the output magnitude log2((1 + T) / (1 - T)) = log2((PD + PN) / (PD - PN)): one ex2 per
//     input, one rcp and one lg2 per output; prefix/suffix products exclude the edge itself.
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

namespace jbp {

constexpr int kResMaxJ = 4;
constexpr int kResMaxL = 16;
constexpr int kResThreads = 768;

struct ResCode {
    int P, J, L, n, m;             // n = L*P, m = J*P checks per side
    unsigned magic;                // ceil(2^32 / P): x mod P for x < 2^32
    unsigned short fa[2][kResMaxJ][kResMaxL], fb[2][kResMaxJ][kResMaxL];  // check -> variable
    unsigned short ia[2][kResMaxJ][kResMaxL], ib[2][kResMaxJ][kResMaxL];  // variable -> check
    int words;
    const uint64_t *basis_rows[2];
    const int *pivot_row[2];
};

// Per-run parameters of the resident kernel.
struct ResRun {
    int max_iter, check_warmup, check_interval;
    int source;
    double p;
    int use_prior;
    double prior4[4];
    unsigned long long seed;
    long long first_trial, ntrials;
    const long long *trial_list;   // optional: trial k is trial_list[k] instead of first_trial + k
    const uint8_t *src_err;        // [ntrials][n]
    const uint8_t *src_sx, *src_sz;
    uint8_t *est_out;
    jbp_trial_result *res_out;
    unsigned long long *hist;
    DevCounters *cnt;
};

__device__ __forceinline__ unsigned res_mod(unsigned x, unsigned P, unsigned magic) {
    const unsigned q = __umulhi(x, magic);
    int r = static_cast<int>(x - q * P);
    return static_cast<unsigned>(r < 0 ? r + static_cast<int>(P) : r);
}

// 16-bit message storage: IEEE half.
struct StoreHalf {
    using T = __half;
    static __device__ __forceinline__ float ld(const T *p) { return __half2float(*p); }
    static __device__ __forceinline__ void st(T *p, float v) { *p = __float2half_rn(v); }
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

constexpr float kResVinMax = 120.0f;   // variable-to-check magnitude clamp (2^-120 is a normal float)
constexpr float kResCmax = 110.0f;     // check-to-variable magnitude clamp (exact in FP16 storage)

__device__ __forceinline__ float with_bit(float a, unsigned b) {
    return __uint_as_float((__float_as_uint(a) & ~1u) | b);
}

// Shared-memory bytes of the resident kernel for a code.
__host__ __device__ inline size_t res_smem_bytes(int n, int m, int L, size_t store_bytes) {
    const size_t c2v = (2ull * L * m * store_bytes + 15) / 16 * 16;
    const size_t A = 2ull * n * 4;
    const size_t err = (static_cast<size_t>(n) + 15) / 16 * 16;
    const size_t syn = (2ull * ((m + 31) / 32) + 3) / 4 * 4 * 4;
    return c2v + A + err + syn + 64;
}


// Check phase, one block row JJ of side SIDE, check offset x: new c2v of the row's L edges
// from A and the old c2v; with `test`, also the parity of the decision bits against the
// target.  Returns whether the tested check failed.
//
// Stable tanh rule.  Per edge u = 2^-|y|, N = 1 - u, D = 1 + u, t = N / D.  A set of edges is
// carried as (PN, Q) with PN = prod N and Q = prod D - prod N, so prod D = PN + Q and
// 1 - T = Q / prod D; joining two sets, Q = PD_a * Q_b + PN_b * Q_a, is a sum of positive terms
// and keeps full relative precision however close T is to 1.  A single edge has Q = 2u exactly.
// The output magnitude log2((1 + T) / (1 - T)) = log2((2 PN + Q) / Q) over the other edges
// therefore grows like min |y| instead of saturating where 1 - T rounds to zero.
template <int P, int J, int L, class ST, int SIDE, int JJ>
__device__ __forceinline__ bool res_check_row(const ResCode &code, typename ST::T *c2v_all, const float *A_all,
                                              const unsigned *syn_all, int x, bool test) {
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    typename ST::T *c2v = c2v_all + SIDE * L * m + JJ * P + x;
    const float *A = A_all + SIDE * n;
    const int c = JJ * P + x;
    const unsigned sbit = (syn_all[SIDE * mw + (c >> 5)] >> (c & 31)) & 1u;
    float u[L];
    unsigned sgn = 0u, par = 0u;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const unsigned y = (static_cast<unsigned>(code.fa[SIDE][JJ][l]) * static_cast<unsigned>(x) +
                            code.fb[SIDE][JJ][l]) % static_cast<unsigned>(P);
        const float a = A[l * P + y];
        par ^= __float_as_uint(a);
        const float v = a - ST::ld(c2v + l * m);
        const unsigned sv = __float_as_uint(v) & 0x80000000u;
        sgn ^= sv;
        // sign of the edge kept in u's sign bit, |u| = 2^-min(|v|, kResVinMax)
        u[l] = __uint_as_float(__float_as_uint(res_ex2(-fminf(fabsf(v), kResVinMax))) | sv);
    }
    const bool bad = test && ((par & 1u) != sbit);
    float sPN[L + 1], sQ[L + 1];
    sPN[L] = 1.0f;
    sQ[L] = 0.0f;
#pragma unroll
    for (int l = L - 1; l >= 0; --l) {
        const float au = fabsf(u[l]);
        const float N = 1.0f - au, D = 1.0f + au, Q = au + au;
        sQ[l] = fmaf(D, sQ[l + 1], sPN[l + 1] * Q);
        sPN[l] = N * sPN[l + 1];
    }
    sgn ^= sbit << 31;
    float pPN = 1.0f, pQ = 0.0f;
#pragma unroll
    for (int l = 0; l < L; ++l) {
        const float ePN = pPN * sPN[l + 1];
        const float eQ = fmaf(pPN + pQ, sQ[l + 1], sPN[l + 1] * pQ);
        const float mag = fminf(res_lg2(fmaf(2.0f, ePN, eQ) * res_rcp(eQ)), kResCmax);
        ST::st(c2v + l * m, __uint_as_float(__float_as_uint(mag) ^ ((sgn ^ __float_as_uint(u[l])) & 0x80000000u)));
        const float au = fabsf(u[l]);
        const float N = 1.0f - au, Q = au + au;
        pQ = fmaf(pPN + pQ, Q, N * pQ);
        pPN *= N;
    }
    return bad;
}

template <int P, int J, int L, class ST, int SIDE>
__device__ __forceinline__ bool res_check_side(const ResCode &code, typename ST::T *c2v, const float *A,
                                               const unsigned *syn, bool test) {
    bool bad = false;
    for (int x = threadIdx.x; x < P; x += blockDim.x) {
        bad |= res_check_row<P, J, L, ST, SIDE, 0>(code, c2v, A, syn, x, test);
        if (J > 1) bad |= res_check_row<P, J, L, ST, SIDE, (J > 1 ? 1 : 0)>(code, c2v, A, syn, x, test);
        if (J > 2) bad |= res_check_row<P, J, L, ST, SIDE, (J > 2 ? 2 : 0)>(code, c2v, A, syn, x, test);
        if (J > 3) bad |= res_check_row<P, J, L, ST, SIDE, (J > 3 ? 3 : 0)>(code, c2v, A, syn, x, test);
    }
    return bad;
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
template <int P, int J, int L, class ST, int LL>
__device__ __forceinline__ void res_var_col(const ResCode &code, const typename ST::T *c2v, float *A, int y,
                                            const float4 lp, const float4 pr) {
    constexpr int m = J * P, n = L * P;
    float Lam = 0.0f, Mu = 0.0f;
#pragma unroll
    for (int j = 0; j < J; ++j) {
        const unsigned xx = (static_cast<unsigned>(code.ia[0][j][LL]) * static_cast<unsigned>(y) + code.ib[0][j][LL]) %
                            static_cast<unsigned>(P);
        const unsigned xz = (static_cast<unsigned>(code.ia[1][j][LL]) * static_cast<unsigned>(y) + code.ib[1][j][LL]) %
                            static_cast<unsigned>(P);
        Lam += ST::ld(c2v + LL * m + j * P + xx);
        Mu += ST::ld(c2v + (L + LL) * m + j * P + xz);
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
    A[v] = with_bit(Lam + Gx, best & 1u);
    A[n + v] = with_bit(Mu + Hz, best >> 1);
}

template <int P, int J, int L, class ST, int LL>
__device__ __forceinline__ void res_var_cols(const ResCode &code, const typename ST::T *c2v, float *A, int y,
                                             const float4 lp, const float4 pr) {
    res_var_col<P, J, L, ST, LL>(code, c2v, A, y, lp, pr);
    if constexpr (LL + 1 < L) res_var_cols<P, J, L, ST, LL + 1>(code, c2v, A, y, lp, pr);
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

template <int P, int J, int L, class ST>
__global__ void __launch_bounds__(kResThreads, 1) k_resident(ResCode code, ResRun run) {
    extern __shared__ __align__(16) unsigned char res_smem[];
    using T = typename ST::T;
    constexpr int m = J * P, n = L * P, mw = (m + 31) / 32;
    T *const c2v = reinterpret_cast<T *>(res_smem);
    constexpr size_t c2v_bytes = (2ull * L * m * sizeof(T) + 15) / 16 * 16;
    float *const A = reinterpret_cast<float *>(res_smem + c2v_bytes);
    uint8_t *const err = res_smem + c2v_bytes + 2ull * n * 4;
    unsigned *const syn = reinterpret_cast<unsigned *>(err + (n + 15) / 16 * 16);
    int *const ints = reinterpret_cast<int *>(syn + (2 * mw + 3) / 4 * 4);
    __shared__ long long trial_sh;
    __shared__ float4 lp_sh, pr_sh;
    __shared__ float lpx_sh, lpz_sh;
    const bool have_err = run.source != kSrcSyndromes;

    // prior: FP64 as the slot engine's refill, then its log2 weights and probabilities in FP32
    if (threadIdx.x == 0) {
        double q[4];
        if (run.use_prior) {
            for (int i = 0; i < 4; ++i) q[i] = run.prior4[i];
        } else {
            q[0] = 1.0 - run.p; q[1] = run.p / 3.0; q[2] = q[1]; q[3] = q[1];
            const double s = ((q[0] + q[1]) + q[2]) + q[3];
            for (int i = 0; i < 4; ++i) q[i] = s > 0.0 ? q[i] / s : 0.25;
        }
        for (int i = 0; i < 4; ++i) q[i] = fmax(q[i], 1e-30);
        lp_sh = make_float4(static_cast<float>(log2(q[0])), static_cast<float>(log2(q[1])),
                            static_cast<float>(log2(q[2])), static_cast<float>(log2(q[3])));
        pr_sh = make_float4(static_cast<float>(q[0]), static_cast<float>(q[1]), static_cast<float>(q[2]),
                            static_cast<float>(q[3]));
        lpx_sh = static_cast<float>(log2((q[0] + q[2]) / (q[1] + q[3])));
        lpz_sh = static_cast<float>(log2((q[0] + q[1]) / (q[2] + q[3])));
    }
    __syncthreads();
    const float4 lp = lp_sh, pr = pr_sh;
    const float lpx = lpx_sh, lpz = lpz_sh;

    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long k = atomicAdd(&run.cnt->next_trial, 1ull);
            trial_sh = k < static_cast<unsigned long long>(run.ntrials) ? static_cast<long long>(k) : -1;
        }
        __syncthreads();
        const long long k = trial_sh;
        if (k < 0) break;
        const long long t = run.trial_list ? run.trial_list[k] : run.first_trial + k;
        const long long local = t - run.first_trial;

        // ---- error and target syndrome
        for (int w = threadIdx.x; w < 2 * mw; w += blockDim.x) syn[w] = 0u;
        if (run.source == kSrcPhilox) {
            for (int v2 = threadIdx.x; 2 * v2 < n; v2 += blockDim.x) {
                uint8_t e0, e1;
                sample_philox_pair(run.seed, t, v2, run.p, e0, e1);
                err[2 * v2] = e0;
                if (2 * v2 + 1 < n) err[2 * v2 + 1] = e1;
            }
        } else if (run.source == kSrcErrors) {
            const uint8_t *src = run.src_err + local * n;
            for (int v = threadIdx.x; v < n; v += blockDim.x) err[v] = src[v];
        } else if (run.source == kSrcMt19937) {
            if (threadIdx.x < 32) warp_mt_trial(reinterpret_cast<unsigned long long *>(A), run.seed, t, run.p, n, err);
        }
        __syncthreads();
        if (run.source == kSrcSyndromes) {
            for (int c = threadIdx.x; c < m; c += blockDim.x) {
                if (run.src_sx[local * m + c] & 1) atomicOr(&syn[c >> 5], 1u << (c & 31));
                if (run.src_sz[local * m + c] & 1) atomicOr(&syn[mw + (c >> 5)], 1u << (c & 31));
            }
        } else {
            for (int r = threadIdx.x; r < 2 * m; r += blockDim.x) {
                const int side = r >= m, c = r - side * m, j = c / P, x = c - j * P;
                unsigned par = 0;
#pragma unroll
                for (int l = 0; l < L; ++l) {
                    const unsigned y = (static_cast<unsigned>(code.fa[side][j][l]) * static_cast<unsigned>(x) +
                                        code.fb[side][j][l]) % static_cast<unsigned>(P);
                    par ^= (err[l * P + y] >> side) & 1u;
                }
                if (par) atomicOr(&syn[side * mw + (c >> 5)], 1u << (c & 31));
            }
        }
        // ---- BP state: c2v = 0, A = prior LLR of each side's bit
        {
            uint4 *z = reinterpret_cast<uint4 *>(c2v);
            constexpr int nz = static_cast<int>(c2v_bytes / 16);
            for (int i = threadIdx.x; i < nz; i += blockDim.x) z[i] = make_uint4(0u, 0u, 0u, 0u);
            const float ax = with_bit(lpx, 0u), az = with_bit(lpz, 0u);
            for (int v = threadIdx.x; v < n; v += blockDim.x) { A[v] = ax; A[n + v] = az; }
        }
        __syncthreads();

        // ---- BP iterations (it = completed iterations); the check phase of iteration it+1
        // also tests the decisions of iteration it
        int it = 0;
        bool ok = false;
        for (;;) {
            const bool test = it >= 1 && (it >= run.max_iter ||
                                          (it > run.check_warmup && (it - run.check_warmup) % run.check_interval == 0));
            bool bad = false;
            if (it < run.max_iter) {
                bad = res_check_side<P, J, L, ST, 0>(code, c2v, A, syn, test);
                bad |= res_check_side<P, J, L, ST, 1>(code, c2v, A, syn, test);
            } else {
                for (int r = threadIdx.x; r < 2 * m; r += blockDim.x) {
                    const int side = r >= m, c = r - side * m, j = c / P, x = c - j * P;
                    unsigned par = 0;
#pragma unroll
                    for (int l = 0; l < L; ++l) {
                        const unsigned y = (static_cast<unsigned>(code.fa[side][j][l]) * static_cast<unsigned>(x) +
                                            code.fb[side][j][l]) % static_cast<unsigned>(P);
                        par ^= __float_as_uint(A[side * n + l * P + y]);
                    }
                    bad |= (par & 1u) != ((syn[side * mw + (c >> 5)] >> (c & 31)) & 1u);
                }
            }
            bad = __syncthreads_or(bad);
            if (test && !bad) { ok = true; break; }
            if (it >= run.max_iter) break;
            for (int y = threadIdx.x; y < P; y += blockDim.x) res_var_cols<P, J, L, ST, 0>(code, c2v, A, y, lp, pr);
            __syncthreads();
            ++it;
        }
        const int iters = ok ? it : run.max_iter;

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
            const unsigned bx = __ballot_sync(0xffffffffu, ((tv ^ e) & 1u) != 0);
            const unsigned bz = __ballot_sync(0xffffffffu, ((tv ^ e) & 2u) != 0);
            if ((threadIdx.x & 31) == 0) { rx[base >> 5] = bx; rz[base >> 5] = bz; }
        }
        exact = __syncthreads_and(exact) && have_err;
        bool stab = false;
        if (have_err && ok && !exact) {
            stab = res_in_row_space(reinterpret_cast<uint64_t *>(rx), words, code.basis_rows[1], code.pivot_row[1], ints);
            if (stab)
                stab = res_in_row_space(reinterpret_cast<uint64_t *>(rz), words, code.basis_rows[0], code.pivot_row[0],
                                        ints);
        } else if (have_err && ok) {
            stab = true;   // exact: the residual is zero
        }
        const bool success = have_err ? (ok && stab) : ok;
        if (threadIdx.x == 0) {
            DevCounters *cn = run.cnt;
            atomicAdd(&cn->done, 1ull);
            atomicAdd(&cn->total_iters, static_cast<unsigned long long>(iters));
            atomicAdd(&cn->bp_trial_iterations, static_cast<unsigned long long>(iters));
            if (!success) atomicAdd(&cn->failures, 1ull);
            if (!ok) atomicAdd(&cn->bp_fail, 1ull);
            if (exact) atomicAdd(&cn->exact, 1ull);
            if (ok) atomicAdd(&cn->syndrome_ok, 1ull);
            if (success && !exact && stab) atomicAdd(&cn->stab_success, 1ull);
            if (run.hist && iters >= 1 && iters <= run.max_iter) atomicAdd(&run.hist[iters], 1ull);
            if (run.res_out) {
                jbp_trial_result rec{};
                rec.iterations = iters;
                rec.syndrome_ok = ok;
                rec.bp_ok = ok;
                rec.success = success;
                rec.exact = exact;
                rec.stab_equiv = stab;
                run.res_out[local] = rec;
            }
        }
        __syncthreads();
    }
}

}  // namespace jbp
