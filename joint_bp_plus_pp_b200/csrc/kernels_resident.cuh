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

constexpr float kResLlrMax = 43.0f;   // same clamp as the slot engine's LLR kernels

__device__ __forceinline__ float with_bit(float a, unsigned b) {
    return __uint_as_float((__float_as_uint(a) & ~1u) | b);
}

// Shared-memory bytes of the resident kernel for a code.
__host__ __device__ inline size_t res_smem_bytes(int n, int m, int L, size_t store_bytes) {
    const size_t c2v = (2ull * L * m * store_bytes + 15) / 16 * 16;
    const size_t A = 2ull * n * 4;
    const size_t err = (static_cast<size_t>(n) + 15) / 16 * 16;
    const size_t syn = (2ull * ((m + 31) / 32) * 4 + 15) / 16 * 16;
    return c2v + A + err + syn + 64;
}

struct ResShared {
    void *c2v;
    float *A;        // [2][n]
    uint8_t *err;    // [n]
    unsigned *syn;   // [2][mw]
    int *ints;       // [16]
};

// Check phase of one side: new c2v from A and the old c2v; with `test`, also the parity of
// the decision bits of every check against its target.  Returns whether a tested check of
// this thread failed.
template <int J, int L, class ST>
__device__ __forceinline__ bool res_check_side(const ResCode &code, const ResShared &sh, int side, bool test) {
    using T = typename ST::T;
    const int P = code.P, m = code.m, n = code.n;
    const int mw = (m + 31) >> 5;
    T *c2v = static_cast<T *>(sh.c2v) + static_cast<size_t>(side) * L * m;
    const float *A = sh.A + static_cast<size_t>(side) * n;
    const unsigned *syn = sh.syn + side * mw;
    bool bad = false;
#pragma unroll 1
    for (int j = 0; j < J; ++j) {
#pragma unroll 1
        for (int x = threadIdx.x; x < P; x += blockDim.x) {
            const int c = j * P + x;
            const unsigned sbit = (syn[c >> 5] >> (c & 31)) & 1u;
            float u[L];
            unsigned neg = 0, par = 0;
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const unsigned y = res_mod(static_cast<unsigned>(code.fa[side][j][l]) * x + code.fb[side][j][l], P,
                                           code.magic);
                const float a = A[l * P + y];
                par ^= __float_as_uint(a) & 1u;
                const float v = fminf(fmaxf(a - ST::ld(c2v + l * m + c), -kResLlrMax), kResLlrMax);
                neg |= (__float_as_uint(v) >> 31) << l;
                u[l] = res_ex2(-fabsf(v));
            }
            if (test) bad |= (par & 1u) != sbit;
            // suffix products of N = 1 - u and D = 1 + u
            float sN[L + 1], sD[L + 1];
            sN[L] = 1.0f;
            sD[L] = 1.0f;
#pragma unroll
            for (int l = L - 1; l >= 0; --l) {
                sN[l] = sN[l + 1] * (1.0f - u[l]);
                sD[l] = sD[l + 1] * (1.0f + u[l]);
            }
            const unsigned sg = (__popc(neg) & 1u) ^ sbit;
            float pN = 1.0f, pD = 1.0f;
#pragma unroll
            for (int l = 0; l < L; ++l) {
                const float eN = pN * sN[l + 1], eD = pD * sD[l + 1];
                const float mag = fminf(res_lg2((eD + eN) * res_rcp(eD - eN)), kResLlrMax);
                const unsigned s = sg ^ ((neg >> l) & 1u);
                ST::st(c2v + l * m + c, s ? -mag : mag);
                pN *= 1.0f - u[l];
                pD *= 1.0f + u[l];
            }
        }
    }
    return bad;
}

// Variable phase: sums, hard decision, and the new A of both sides.
template <int J, int L, class ST>
__device__ __forceinline__ void res_var(const ResCode &code, const ResShared &sh, const float4 lp) {
    using T = typename ST::T;
    const int P = code.P, m = code.m, n = code.n;
    const T *c2vx = static_cast<const T *>(sh.c2v);
    const T *c2vz = c2vx + static_cast<size_t>(L) * m;
    float *Ax = sh.A, *Az = sh.A + n;
#pragma unroll 1
    for (int l = 0; l < L; ++l) {
#pragma unroll 1
        for (int y = threadIdx.x; y < P; y += blockDim.x) {
            float Lam = 0.0f, Mu = 0.0f;
#pragma unroll
            for (int j = 0; j < J; ++j) {
                const unsigned xx = res_mod(static_cast<unsigned>(code.ia[0][j][l]) * y + code.ib[0][j][l], P, code.magic);
                const unsigned xz = res_mod(static_cast<unsigned>(code.ia[1][j][l]) * y + code.ib[1][j][l], P, code.magic);
                Lam += ST::ld(c2vx + l * m + j * P + xx);
                Mu += ST::ld(c2vz + l * m + j * P + xz);
            }
            const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
            unsigned best = 0;
            float bv = w0;
            if (w1 > bv) { best = 1; bv = w1; }
            if (w2 > bv) { best = 2; bv = w2; }
            if (w3 > bv) { best = 3; }
            const float Gx = res_lse2(lp.x, lp.z - Mu) - res_lse2(lp.y, lp.w - Mu);
            const float Hz = res_lse2(lp.x, lp.y - Lam) - res_lse2(lp.z, lp.w - Lam);
            const int v = l * P + y;
            Ax[v] = with_bit(Lam + Gx, best & 1u);
            Az[v] = with_bit(Mu + Hz, best >> 1);
        }
    }
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

template <int J, int L, class ST>
__global__ void __launch_bounds__(kResThreads, 1) k_resident(ResCode code, ResRun run) {
    extern __shared__ __align__(16) unsigned char res_smem[];
    using T = typename ST::T;
    const int P = code.P, m = code.m, n = code.n;
    const int mw = (m + 31) >> 5;
    ResShared sh;
    {
        size_t o = 0;
        sh.c2v = res_smem + o; o += (2ull * L * m * sizeof(T) + 15) / 16 * 16;
        sh.A = reinterpret_cast<float *>(res_smem + o); o += 2ull * n * 4;
        sh.err = res_smem + o; o += (static_cast<size_t>(n) + 15) / 16 * 16;
        sh.syn = reinterpret_cast<unsigned *>(res_smem + o); o += (2ull * mw * 4 + 15) / 16 * 16;
        sh.ints = reinterpret_cast<int *>(res_smem + o);
    }
    __shared__ long long trial_sh;
    __shared__ float4 lp_sh;
    __shared__ float lpx_sh, lpz_sh;
    const bool have_err = run.source != kSrcSyndromes;

    // log2 prior weights (FP64 prior as the slot engine's refill, then rounded to FP32)
    if (threadIdx.x == 0) {
        double p0, p1, p2, p3;
        if (run.use_prior) {
            p0 = run.prior4[0]; p1 = run.prior4[1]; p2 = run.prior4[2]; p3 = run.prior4[3];
        } else {
            p0 = 1.0 - run.p; p1 = run.p / 3.0; p2 = p1; p3 = p1;
            const double s = ((p0 + p1) + p2) + p3;
            if (s <= 0.0) { p0 = p1 = p2 = p3 = 0.25; }
            else { p0 /= s; p1 /= s; p2 /= s; p3 /= s; }
        }
        lp_sh = make_float4(static_cast<float>(log2(p0)), static_cast<float>(log2(p1)), static_cast<float>(log2(p2)),
                            static_cast<float>(log2(p3)));
        lpx_sh = static_cast<float>(log2((p0 + p2) / (p1 + p3)));
        lpz_sh = static_cast<float>(log2((p0 + p1) / (p2 + p3)));
    }
    __syncthreads();
    const float4 lp = lp_sh;
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
        for (int w = threadIdx.x; w < 2 * mw; w += blockDim.x) sh.syn[w] = 0u;
        if (run.source == kSrcPhilox) {
            for (int v2 = threadIdx.x; 2 * v2 < n; v2 += blockDim.x) {
                uint8_t e0, e1;
                sample_philox_pair(run.seed, t, v2, run.p, e0, e1);
                sh.err[2 * v2] = e0;
                if (2 * v2 + 1 < n) sh.err[2 * v2 + 1] = e1;
            }
        } else if (run.source == kSrcErrors) {
            const uint8_t *src = run.src_err + local * n;
            for (int v = threadIdx.x; v < n; v += blockDim.x) sh.err[v] = src[v];
        } else if (run.source == kSrcMt19937) {
            if (threadIdx.x < 32) warp_mt_trial(reinterpret_cast<unsigned long long *>(sh.A), run.seed, t, run.p, n, sh.err);
        }
        __syncthreads();
        if (run.source == kSrcSyndromes) {
            for (int c = threadIdx.x; c < m; c += blockDim.x) {
                if (run.src_sx[local * m + c] & 1) atomicOr(&sh.syn[c >> 5], 1u << (c & 31));
                if (run.src_sz[local * m + c] & 1) atomicOr(&sh.syn[mw + (c >> 5)], 1u << (c & 31));
            }
        } else {
            for (int side = 0; side < 2; ++side)
                for (int j = 0; j < code.J; ++j)
                    for (int x = threadIdx.x; x < P; x += blockDim.x) {
                        unsigned par = 0;
#pragma unroll
                        for (int l = 0; l < L; ++l) {
                            const unsigned y = res_mod(static_cast<unsigned>(code.fa[side][j][l]) * x + code.fb[side][j][l],
                                                       P, code.magic);
                            par ^= (sh.err[l * P + y] >> side) & 1u;
                        }
                        const int c = j * P + x;
                        if (par) atomicOr(&sh.syn[side * mw + (c >> 5)], 1u << (c & 31));
                    }
        }
        // ---- BP state: c2v = 0, A = prior LLR of each side's bit
        {
            uint4 *z = static_cast<uint4 *>(sh.c2v);
            const int nz = static_cast<int>((2ull * L * m * sizeof(T)) / 16);
            for (int i = threadIdx.x; i < nz; i += blockDim.x) z[i] = make_uint4(0u, 0u, 0u, 0u);
            const float ax = with_bit(lpx, 0u), az = with_bit(lpz, 0u);
            for (int v = threadIdx.x; v < n; v += blockDim.x) { sh.A[v] = ax; sh.A[n + v] = az; }
        }
        __syncthreads();

        // ---- BP iterations (it = completed iterations)
        int it = 0;
        bool ok = false;
        for (;;) {
            const bool test = it >= 1 && (it >= run.max_iter ||
                                          (it > run.check_warmup && (it - run.check_warmup) % run.check_interval == 0));
            bool bad = false;
            if (it < run.max_iter) {
                bad = res_check_side<J, L, ST>(code, sh, 0, test);
                bad |= res_check_side<J, L, ST>(code, sh, 1, test);
            } else {
                // final test only
                for (int side = 0; side < 2; ++side)
                    for (int j = 0; j < code.J; ++j)
                        for (int x = threadIdx.x; x < P; x += blockDim.x) {
                            unsigned par = 0;
                            const float *A = sh.A + static_cast<size_t>(side) * n;
#pragma unroll
                            for (int l = 0; l < L; ++l) {
                                const unsigned y = res_mod(static_cast<unsigned>(code.fa[side][j][l]) * x +
                                                               code.fb[side][j][l], P, code.magic);
                                par ^= __float_as_uint(A[l * P + y]) & 1u;
                            }
                            const int c = j * P + x;
                            bad |= (par & 1u) != ((sh.syn[side * mw + (c >> 5)] >> (c & 31)) & 1u);
                        }
            }
            bad = __syncthreads_or(bad);
            if (test && !bad) { ok = true; break; }
            if (it >= run.max_iter) break;
            res_var<J, L, ST>(code, sh, lp);
            __syncthreads();
            ++it;
        }
        const int iters = ok ? it : run.max_iter;

        // ---- classification (jointbp_ets.cpp:6199-6245): exact, stabilizer-equivalent residual
        unsigned *rx = reinterpret_cast<unsigned *>(sh.c2v);     // BP state is no longer needed
        const int w32 = 2 * code.words;
        unsigned *rz = rx + w32;
        for (int w = threadIdx.x; w < 2 * w32; w += blockDim.x) rx[w] = 0u;
        __syncthreads();
        bool exact = true;
        for (int base = (threadIdx.x >> 5) * 32; base < n; base += blockDim.x) {
            const int v = base + (threadIdx.x & 31);
            const bool in = v < n;
            const unsigned e = in ? ((__float_as_uint(sh.A[v]) & 1u) | ((__float_as_uint(sh.A[n + v]) & 1u) << 1)) : 0u;
            const unsigned tv = in && have_err ? sh.err[v] : e;
            if (in && run.est_out) run.est_out[local * n + v] = static_cast<uint8_t>(e);
            exact &= tv == e;
            const unsigned bx = __ballot_sync(0xffffffffu, ((tv ^ e) & 1u) != 0);
            const unsigned bz = __ballot_sync(0xffffffffu, ((tv ^ e) & 2u) != 0);
            if ((threadIdx.x & 31) == 0) { rx[base >> 5] = bx; rz[base >> 5] = bz; }
        }
        exact = __syncthreads_and(exact) && have_err;
        bool stab = false;
        if (have_err && ok && !exact) {
            stab = res_in_row_space(reinterpret_cast<uint64_t *>(rx), code.words, code.basis_rows[1], code.pivot_row[1],
                                    sh.ints);
            if (stab)
                stab = res_in_row_space(reinterpret_cast<uint64_t *>(rz), code.words, code.basis_rows[0],
                                        code.pivot_row[0], sh.ints);
        } else if (have_err && ok) {
            stab = true;   // exact: the residual is zero
        }
        const bool success = have_err ? (ok && stab) : ok;
        if (threadIdx.x == 0) {
            DevCounters *c = run.cnt;
            atomicAdd(&c->done, 1ull);
            atomicAdd(&c->total_iters, static_cast<unsigned long long>(iters));
            atomicAdd(&c->bp_trial_iterations, static_cast<unsigned long long>(iters));
            if (!success) atomicAdd(&c->failures, 1ull);
            if (!ok) atomicAdd(&c->bp_fail, 1ull);
            if (exact) atomicAdd(&c->exact, 1ull);
            if (ok) atomicAdd(&c->syndrome_ok, 1ull);
            if (success && !exact && stab) atomicAdd(&c->stab_success, 1ull);
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
