// Mixed-size Monte Carlo in one launch: the trials of several codes (any check-regular CSS
// codes with the same check degree DC, e.g. hypergraph products of (3,4)-regular classical
// codes, n = 1,600 ... 14,400, variable degrees 3 and 4) decoded by one persistent kernel.
// One block of 768 threads per SM takes work items -- (code, trial) pairs, the codes in the
// host's order, largest first -- from one atomic counter, so trials of all sizes share the
// SMs with no partition to tune and the tail of the launch is made of the smallest trials.
//
// Per trial, in shared memory: A [side][v] (FP32 variable totals, decision bit in the lowest
// mantissa bit, as in kernels_resident.cuh), the error [v] and the target syndrome bits; the
// check-to-variable messages c2v [side][i][c] (edge i of check c) stay in shared memory when
// the code's trial fits beside them (the launch's shared size is the largest such trial), and
// otherwise in a per-block global scratch that stays in L2.  Neighbours come from tables built
// on the host: the variable of edge i of check c, chk[i*m + c], and the c2v slot i*m + c of
// edge k of variable v, slot[k*n + v] (kMixNone for the missing edges of lower-degree
// variables), both 16-bit (codes up to 65,535 variables and message slots per side, so that
// more of the tables stay in L1).  Both are index-major so that a warp's lanes, which take
// consecutive checks or variables, read them coalesced; the check phase
// reads its c2v row by row the same way, the variable phase gathers, with all of a variable's
// slot loads issued before its message loads (variable degree at most kMixMaxDv).
//
// Arithmetic per edge and per variable is the resident engine's (the stable tanh rule in
// (PN, H) form, the exact 4-ary coupling, the flooding schedule with early exit and the
// syndrome test fused into the next check phase, jointbp_ets.cpp:1943-2535); classification
// as jointbp_ets.cpp:6199-6211.  No post-processing: the mixed workload decodes with plain BP.
#pragma once

#include "kernels_resident.cuh"

namespace jbp {

constexpr int kMixThreads = 768;
constexpr int kMixMaxCodes = 8;
constexpr int kMixMaxDv = 4;
constexpr unsigned kMixNone = 0xFFFFu;   // a missing edge in the 16-bit slot table

struct MixCode {
    DevCode dc;                    // n, per-side m / dc / dv, basis rows (classification)
    const uint16_t *chk[2];        // [DC][m] variable of edge i of check c
    const uint16_t *slot[2];       // [dv][n] c2v slot (i*m + c) of each variable's edges, kMixNone pads
    unsigned long long seed;
    long long first_trial, ntrials;
    long long item_end;            // work items of codes 0..this one
    DevCounters *cnt;
    jbp_trial_result *res_out;     // optional, [ntrials]
    unsigned long long *hist;      // optional iteration histogram [max_iter + 1]
    const uint8_t *src_err;        // optional [ntrials][n] errors (0..3) instead of Philox noise
    uint8_t *est_out;              // optional [ntrials][n] final estimates
    float *llr_out;                // optional [ntrials][n][2] final LLRs (natural log of P(1)/P(0))
    int c2v_in_smem;
};

struct MixRun {
    MixCode code[kMixMaxCodes];
    int ncodes;
    unsigned long long *next;      // work counter
    int max_iter, check_warmup, check_interval;
    double p, p_max;
    int use_prior;
    double prior4[4];
    unsigned char *scratch;        // per block, scratch_stride bytes (c2v of the codes that do not fit)
    size_t scratch_stride;
    unsigned long long budget_ns;  // run budget as ResRun::budget_ns; stops are counted in code[0].cnt
    const volatile int *abort_flag;   // as ResRun::abort_flag (the first context's), read at item claims
};

__host__ __device__ inline size_t mix_align(size_t b) { return (b + 15) / 16 * 16; }

// Shared bytes of a trial of a code without and with its c2v.
__host__ __device__ inline size_t mix_state_bytes(int n, int mx, int mz) {
    const int mw = (mx > mz ? mx : mz) / 32 + 1;
    return mix_align(8ull * n) + mix_align(static_cast<size_t>(n)) + mix_align(8ull * mw);
}
__host__ __device__ inline size_t mix_c2v_bytes(int mx, int mz, int dc, size_t store_bytes) {
    return mix_align(store_bytes * dc * (static_cast<size_t>(mx) + mz));
}

// New c2v of check c of one side (its DC edges at c2v[i*m + c]); with `test`, also whether
// the decisions in A's low bits fail the check.  The stable tanh rule of res_check_row.
template <int DC, class ST>
__device__ __forceinline__ bool mix_check_row(const uint16_t *__restrict__ chk, typename ST::T *c2v, int m,
                                              const float *A, int c, unsigned sbit, bool test) {
    // the row's variable indices, loaded together up front where the registers allow it
    constexpr bool kPre = DC <= 8;
    int vv[kPre ? DC : 1];
    if constexpr (kPre) {
#pragma unroll
        for (int i = 0; i < DC; ++i) vv[i] = __ldg(chk + static_cast<size_t>(i) * m + c);
    }
    unsigned par = 0u;
    res_row_rule<DC>(
        [&](int i) {
            int v;
            if constexpr (kPre) v = vv[i];
            else v = __ldg(chk + static_cast<size_t>(i) * m + c);
            const float a = A[v];
            par ^= __float_as_uint(a);
            return a - ST::ld(c2v + static_cast<size_t>(i) * m + c);
        },
        sbit, [&](int i, float y) { ST::st(c2v + static_cast<size_t>(i) * m + c, y); });
    return test && ((par & 1u) != sbit);
}

// Syndrome test alone (the decisions in A's low bits against the target): failing checks of
// this thread on one side.
template <int DC>
__device__ __forceinline__ int mix_test_side(const uint16_t *__restrict__ chk, int m, const float *A,
                                             const unsigned *syn) {
    int bad = 0;
    for (int c = threadIdx.x; c < m; c += blockDim.x) {
        unsigned par = 0;
#pragma unroll
        for (int i = 0; i < DC; ++i) par ^= __float_as_uint(A[__ldg(chk + static_cast<size_t>(i) * m + c)]);
        bad += (par & 1u) != ((syn[c >> 5] >> (c & 31)) & 1u);
    }
    return bad;
}

// Variable v: sums of its X and Z c2v, hard decision, new totals (res_var_col without the
// decision history).
template <class ST>
__device__ __forceinline__ void mix_var(const uint16_t *__restrict__ slot_x, int dvx, const uint16_t *__restrict__ slot_z,
                                        int dvz, const typename ST::T *c2v_x, const typename ST::T *c2v_z, float *A,
                                        int n, int v, const float4 lp, const float4 pr) {
    unsigned sx[kMixMaxDv], sz[kMixMaxDv];
#pragma unroll
    for (int k = 0; k < kMixMaxDv; ++k) {
        sx[k] = k < dvx ? __ldg(slot_x + static_cast<size_t>(k) * n + v) : kMixNone;
        sz[k] = k < dvz ? __ldg(slot_z + static_cast<size_t>(k) * n + v) : kMixNone;
    }
    float Lam = 0.0f, Mu = 0.0f;
#pragma unroll
    for (int k = 0; k < kMixMaxDv; ++k) {
        if (sx[k] != kMixNone) Lam += ST::ld(c2v_x + sx[k]);
        if (sz[k] != kMixNone) Mu += ST::ld(c2v_z + sz[k]);
    }
    const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
    unsigned best = 0;
    float bv = w0;
    if (w1 > bv) { best = 1; bv = w1; }
    if (w2 > bv) { best = 2; bv = w2; }
    if (w3 > bv) { best = 3; }
    const float Gx = res_couple(Mu, pr.x, pr.z, pr.y, pr.w);
    const float Hz = res_couple(Lam, pr.x, pr.y, pr.z, pr.w);
    A[v] = with_bit(Lam + Gx, best & 1u);
    A[n + v] = with_bit(Mu + Hz, best >> 1);
}

// Final LLRs of a trial from its c2v (res_write_llr with table neighbours; out of line).
template <class ST>
__device__ __noinline__ void mix_write_llr(const uint16_t *__restrict__ slot_x, int dvx,
                                           const uint16_t *__restrict__ slot_z,
                                           int dvz, const typename ST::T *c2v_x, const typename ST::T *c2v_z, int n,
                                           const float4 lp, float *out) {
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        float Lam = 0.0f, Mu = 0.0f;
        for (int k = 0; k < dvx; ++k) {
            const unsigned s = __ldg(slot_x + static_cast<size_t>(k) * n + v);
            if (s != kMixNone) Lam += ST::ld(c2v_x + s);
        }
        for (int k = 0; k < dvz; ++k) {
            const unsigned s = __ldg(slot_z + static_cast<size_t>(k) * n + v);
            if (s != kMixNone) Mu += ST::ld(c2v_z + s);
        }
        const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
        out[2 * v] = (res_lse2(w1, w3) - res_lse2(w0, w2)) * 0.69314718f;
        out[2 * v + 1] = (res_lse2(w2, w3) - res_lse2(w0, w1)) * 0.69314718f;
    }
}

template <int DC, class ST>
__global__ void __launch_bounds__(kMixThreads, 1) k_mixed(const __grid_constant__ MixRun run) {
    extern __shared__ __align__(16) unsigned char mix_smem[];
    using T = typename ST::T;
    __shared__ long long item_sh;
    __shared__ int code_sh;
    __shared__ float4 lp_sh, pr_sh;
    __shared__ float lpx_sh, lpz_sh;
    __shared__ float first_sh[2][DC];   // first-iteration c2v of each position (syndrome bit 0)
    __shared__ int ints[16];
    __shared__ int abort_sh;   // 1: the run budget ran out during this trial; 2: abort requested
    if (threadIdx.x < 16) ints[threadIdx.x] = 0;
    __shared__ unsigned long long deadline_sh;   // global-timer end of the run budget (0 = none)
    if (threadIdx.x == 0) deadline_sh = run.budget_ns ? dev_globaltimer() + run.budget_ns : 0ull;
    for (;;) {
        if (threadIdx.x == 0) {
            const unsigned long long k = atomicAdd(run.next, 1ull);
            const long long total = run.code[run.ncodes - 1].item_end;
            long long item = k < static_cast<unsigned long long>(total) ? static_cast<long long>(k) : -1;
            if (item >= 0 && deadline_sh && dev_globaltimer() > deadline_sh) {
                item = -1;   // the run budget is spent: no further trial
                atomicAdd(&run.code[0].cnt->watchdog, 1ull);
            } else if (item >= 0 && k % kResAbortEvery == 0 && *run.abort_flag) {
                item = -1;   // abort requested: no further trial
                atomicAdd(&run.code[0].cnt->aborted, 1ull);
            }
            abort_sh = 0;
            int ci = 0;
            if (item >= 0) {
                while (item >= run.code[ci].item_end) ++ci;
                item -= ci > 0 ? run.code[ci - 1].item_end : 0;
            }
            item_sh = item;
            code_sh = ci;
            if (item >= 0) {
                const double pt = run.p_max > run.p
                                      ? trial_p(run.p, run.p_max, run.code[ci].seed, run.code[ci].first_trial + item)
                                      : run.p;
                res_set_prior(run.use_prior, run.prior4, pt, &lp_sh, &pr_sh, &lpx_sh, &lpz_sh);
            }
        }
        __syncthreads();
        const long long local = item_sh;
        if (local < 0) break;
        const MixCode &mc = run.code[code_sh];
        const int n = mc.dc.n, mx = mc.dc.s[0].m, mz = mc.dc.s[1].m;
        const int mwx = (mx + 31) / 32, mwz = (mz + 31) / 32;
        const long long t = mc.first_trial + local;
        const double pt = run.p_max > run.p ? trial_p(run.p, run.p_max, mc.seed, t) : run.p;
        float *const A = reinterpret_cast<float *>(mix_smem);
        uint8_t *const err = mix_smem + mix_align(8ull * n);
        unsigned *const syn = reinterpret_cast<unsigned *>(err + mix_align(static_cast<size_t>(n)));
        unsigned *const synz = syn + mwx;
        T *const c2v = mc.c2v_in_smem
                           ? reinterpret_cast<T *>(mix_smem + mix_state_bytes(n, mx, mz))
                           : reinterpret_cast<T *>(run.scratch + run.scratch_stride * blockIdx.x);
        T *const c2vz = c2v + static_cast<size_t>(DC) * mx;
        const int dvx = mc.dc.s[0].dv, dvz = mc.dc.s[1].dv;

        // ---- error (Philox, the stream of the other engines), target syndrome, BP state
        for (int w = threadIdx.x; w < mwx + mwz; w += blockDim.x) syn[w] = 0u;
        if (mc.src_err) {
            // given errors (device memory or mapped pinned host memory); a byte above 3 is
            // reported and masked
            const uint8_t *src = mc.src_err + local * n;
            if ((n & 15) == 0 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
                const uint4 *s16 = reinterpret_cast<const uint4 *>(src);
                uint4 *d16 = reinterpret_cast<uint4 *>(err);
                unsigned badw = 0u;
                for (int i = threadIdx.x; i < n / 16; i += blockDim.x) {
                    uint4 w = s16[i];
                    badw |= (w.x | w.y | w.z | w.w) & 0xFCFCFCFCu;
                    w.x &= 0x03030303u; w.y &= 0x03030303u; w.z &= 0x03030303u; w.w &= 0x03030303u;
                    d16[i] = w;
                }
                if (badw) atomicAdd(&mc.cnt->bad_input, 1ull);
            } else {
                for (int v = threadIdx.x; v < n; v += blockDim.x) {
                    const uint8_t e = src[v];
                    if (e > 3) atomicAdd(&mc.cnt->bad_input, 1ull);
                    err[v] = e & 3;
                }
            }
        } else {
            for (int v2 = threadIdx.x; 2 * v2 < n; v2 += blockDim.x) {
                uint8_t e0, e1;
                sample_philox_pair(mc.seed, t, v2, pt, e0, e1);
                err[2 * v2] = e0;
                if (2 * v2 + 1 < n) err[2 * v2 + 1] = e1;
            }
        }
        __syncthreads();
        for (int r = threadIdx.x; r < mx + mz; r += blockDim.x) {
            const int side = r >= mx, c = r - side * mx;
            const uint16_t *ck = mc.chk[side];
            const int ms = side ? mz : mx;
            unsigned par = 0;
#pragma unroll
            for (int i = 0; i < DC; ++i) par ^= err[__ldg(ck + static_cast<size_t>(i) * ms + c)];
            if ((par >> side) & 1u) atomicOr(&(side ? synz : syn)[c >> 5], 1u << (c & 31));
        }
        {
            const float ax = with_bit(lpx_sh, 0u), az = with_bit(lpz_sh, 0u);
            for (int v = threadIdx.x; v < n; v += blockDim.x) { A[v] = ax; A[n + v] = az; }
            if (threadIdx.x < 2) res_first_row<DC>(threadIdx.x ? az : ax, first_sh[threadIdx.x]);
        }
        __syncthreads();
        {
            // the first iteration's c2v in closed form (res_first_row)
            for (int r = threadIdx.x; r < mx + mz; r += blockDim.x) {
                const int side = r >= mx, c = r - side * mx, ms = side ? mz : mx;
                const bool neg = ((side ? synz : syn)[c >> 5] >> (c & 31)) & 1u;
                T *row = (side ? c2vz : c2v) + c;
#pragma unroll
                for (int i = 0; i < DC; ++i)
                    ST::st(row + static_cast<size_t>(i) * ms, neg ? -first_sh[side][i] : first_sh[side][i]);
            }
        }
        __syncthreads();

        // ---- BP iterations (it = completed iterations; the test of iteration it rides in the
        // check phase of iteration it + 1)
        int it = 0, rf = 0, iters = run.max_iter;
        const float4 lp = lp_sh, pr = pr_sh;
        for (;;) {
            const bool fused = it >= 1 && (it >= run.max_iter ||
                                           (it > run.check_warmup && (it - run.check_warmup) % run.check_interval == 0));
            int bad = 0;
            if (it < run.max_iter && it > 0) {   // iteration 1's check phase is the closed form above
                for (int c = threadIdx.x; c < mx; c += blockDim.x)
                    bad += mix_check_row<DC, ST>(mc.chk[0], c2v, mx, A, c, (syn[c >> 5] >> (c & 31)) & 1u, fused);
                for (int c = threadIdx.x; c < mz; c += blockDim.x)
                    bad += mix_check_row<DC, ST>(mc.chk[1], c2vz, mz, A + n, c, (synz[c >> 5] >> (c & 31)) & 1u,
                                                 fused);
            } else if (fused) {
                bad = mix_test_side<DC>(mc.chk[0], mx, A, syn) + mix_test_side<DC>(mc.chk[1], mz, A + n, synz);
            }
            // run budget (as k_resident): thread 0 writes the flag before the barrier, every thread
            // reads it after it
            if (threadIdx.x == 0 && it % kResBudgetEvery == kResBudgetEvery - 1) {
                if (deadline_sh && dev_globaltimer() > deadline_sh) abort_sh = 1;
                else if (it >= kResAbortFrom && *run.abort_flag) abort_sh = 2;
            }
            const bool any = __syncthreads_or(bad) != 0;
            if (fused && !any) { rf = kResSyndromeOk | kResBpOk; iters = it; break; }
            if (it >= run.max_iter || abort_sh) break;
            for (int v = threadIdx.x; v < n; v += blockDim.x)
                mix_var<ST>(mc.slot[0], dvx, mc.slot[1], dvz, c2v, c2vz, A, n, v, lp, pr);
            __syncthreads();
            ++it;
        }
        if (abort_sh && rf == 0 && it < run.max_iter) {
            // abandoned for the run budget: not classified, not counted; the block stops
            if (threadIdx.x == 0)
                atomicAdd(abort_sh == 2 ? &run.code[0].cnt->aborted : &run.code[0].cnt->watchdog, 1ull);
            break;
        }
        const bool ok = (rf & kResSyndromeOk) != 0;
        if (mc.llr_out) mix_write_llr<ST>(mc.slot[0], dvx, mc.slot[1], dvz, c2v, c2vz, n, lp, mc.llr_out + local * n * 2);

        // ---- classification (jointbp_ets.cpp:6199-6211): exact, stabilizer-equivalent residual
        const int words = (n + 63) / 64, w32 = 2 * words;
        unsigned *rx = reinterpret_cast<unsigned *>(c2v);     // the messages are no longer needed
        unsigned *rz = rx + w32;
        for (int w = threadIdx.x; w < 2 * w32; w += blockDim.x) rx[w] = 0u;
        __syncthreads();
        bool exact = true;
        for (int base = (threadIdx.x >> 5) * 32; base < n; base += blockDim.x) {
            const int v = base + (threadIdx.x & 31);
            const bool in = v < n;
            const unsigned e = in ? ((__float_as_uint(A[v]) & 1u) | ((__float_as_uint(A[n + v]) & 1u) << 1)) : 0u;
            const unsigned tv = in ? err[v] : e;
            if (in && mc.est_out) mc.est_out[local * n + v] = static_cast<uint8_t>(e);
            exact &= tv == e;
            const unsigned bxm = __ballot_sync(0xffffffffu, ((tv ^ e) & 1u) != 0);
            const unsigned bzm = __ballot_sync(0xffffffffu, ((tv ^ e) & 2u) != 0);
            if ((threadIdx.x & 31) == 0) { rx[base >> 5] = bxm; rz[base >> 5] = bzm; }
        }
        exact = __syncthreads_and(exact) != 0;
        bool stab = false;
        if (ok && !exact) {
            stab = res_in_row_space(reinterpret_cast<uint64_t *>(rx), words, mc.dc.basis_rows[1], mc.dc.pivot_row[1],
                                    ints + 8);
            if (stab)
                stab = res_in_row_space(reinterpret_cast<uint64_t *>(rz), words, mc.dc.basis_rows[0],
                                        mc.dc.pivot_row[0], ints + 8);
        } else if (ok) {
            stab = true;
        }
        const bool success = ok && stab;
        if (threadIdx.x == 0)
            account_trial(mc.cnt, mc.hist, mc.res_out, run.max_iter, local, iters, rf, ok, success, exact, stab);
        __syncthreads();
    }
}

}  // namespace jbp
