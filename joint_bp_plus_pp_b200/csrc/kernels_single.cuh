// One FP64 trial per launch, for calls that decode one or a few trials -- the drop-in's
// cuda_bp_decode decodes one trial per call (jointbp_cuda.cu:681-1104).  A cooperative launch of
// a few dozen blocks runs the whole BP loop of the trial: the check phase with one thread per
// check row, the variable phase with one thread per variable and the syndrome test, separated by
// a grid barrier, instead of the slot engine's per-iteration kernels over warps of 32 slots of
// which one would be busy.  The arithmetic is the slot engine's FP64 path (check_f64_row,
// var_f64_update), so decisions and iteration counts are the same bit for bit; messages are
// indexed by edge (e = c * dc + pos, check-major as the reference numbers edges) and stay in L2.
#pragma once

#include "kernels_bp.cuh"
#include "kernels_slots.cuh"

namespace jbp {

constexpr int kSingleThreads = 256;
constexpr int kSingleBlocks = 36;
constexpr unsigned long long kGridBarrierWaitNs = 1000000000ull;   // a barrier gives up after 1 s

struct SingleRun {
    DevCode code;
    const uint8_t *sx, *sz;         // target syndrome bits, one byte per check (bit 0)
    double prior[4];                // normalized prior of the trial
    int max_iter, check_warmup, check_interval;
    double2 *c2v[2], *v2c[2];       // [side][edge]
    uint8_t *est;                   // [n] decisions (0..3): the caller's output buffer
    unsigned *bar;                  // grid barrier: [0] arrivals, [1] generation
    int *bad;                       // [2] failing checks of the last two syndrome tests
    int *err;                       // set when a barrier gave up (the launch then ends)
    DevCounters *cnt;
    unsigned long long *hist;
    jbp_trial_result *res_out;
    long long local;                // the trial's index in the run (result record, counters)
};

// Grid-wide barrier for a cooperative launch (every block resident): the last block to arrive
// resets the count and advances the generation the others wait on.  The count is reset before
// the generation moves, and no block can arrive at the next barrier before it moves, so no
// arrival is lost.  A wait that lasts kGridBarrierWaitNs sets *err; the barrier then returns
// false in every block that looks at the flag, and the caller returns.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, int *err) {
    __shared__ int ok_sh;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = bar + 1;
        const unsigned g = *gen;
        __threadfence();
        bool ok = true;
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            atomicAdd(bar + 1, 1u);
        } else {
            unsigned long long t0;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
            while (*gen == g) {
                unsigned long long t;
                asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                if (t - t0 > kGridBarrierWaitNs) {
                    atomicExch(err, 1);
                    ok = false;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_sh = ok && *reinterpret_cast<volatile int *>(err) == 0;
    }
    __syncthreads();
    return ok_sh != 0;
}

template <int DC, int DV>
__global__ void __launch_bounds__(kSingleThreads) k_single_f64(const __grid_constant__ SingleRun run) {
    const DevCode &code = run.code;
    const int mx = code.s[0].m, M = mx + code.s[1].m, n = code.n;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    // views for var_f64_update: one slot (0) with the run's prior; its first-iteration flag is
    // only read by the damped update, which this kernel does not run
    int fresh_iter = 0;
    DevRun rv{};
    rv.iter = &fresh_iter;
    rv.prior = const_cast<double *>(run.prior);
    DevMsgs mv{};
    mv.v2c[0] = run.v2c[0];
    mv.v2c[1] = run.v2c[1];
    __shared__ int bad_sh;
    // the test counters start at zero for every trial (the first test adds to them two barriers
    // later)
    if (tid == 0) {
        run.bad[0] = 0;
        run.bad[1] = 0;
    }
    int iters = run.max_iter, tests = 0;
    bool ok = false;
    // the check schedule of the slot engine's check_due (1-based iteration k1)
    auto due = [&](int k1) {
        return k1 >= run.max_iter || (k1 > run.check_warmup && (k1 - run.check_warmup) % run.check_interval == 0);
    };
    // whether the decisions in run.est fail check ch of a side (jointbp_ets.cpp:2521-2525)
    auto fails = [&](int side, int ch) -> int {
        const int dc = code.s[side].dc;
        unsigned par = 0;
        for (int i = 0; i < dc; ++i) {
            const int v = __ldg(code.s[side].chk_var + static_cast<size_t>(ch) * dc + i);
            if (v >= 0) par ^= (run.est[v] >> side) & 1u;
        }
        return par != static_cast<unsigned>((side ? run.sz : run.sx)[ch] & 1);
    };
    // adds this block's failing checks to the test's count in bad[tests & 1] and clears the
    // other entry (last read before the previous barrier) for the next test
    auto post_count = [&](int bad) {
        bad = __reduce_add_sync(0xffffffffu, bad);
        if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&bad_sh, bad);
        __syncthreads();
        if (threadIdx.x == 0 && bad_sh) atomicAdd(&run.bad[tests & 1], bad_sh);
        if (tid == 0) run.bad[(tests + 1) & 1] = 0;
    };
    for (int it = 0; it < run.max_iter; ++it) {
        // the test of iteration it's decisions (1-based) rides in this check phase, which reads
        // the same decisions; when they satisfy both syndromes, the phase's messages are unused
        const bool test_now = it >= 1 && due(it);
        if (test_now) {
            if (threadIdx.x == 0) bad_sh = 0;
            __syncthreads();
        }
        int bad = 0;
        // check phase: new c2v of every check row (jointbp_ets.cpp:2373-2449)
        for (int row = tid; row < M; row += nthreads) {
            const int side = row >= mx, ch = side ? row - mx : row;
            double q0[DC], q1[DC];
            const double2 *v2c = run.v2c[side] + static_cast<size_t>(ch) * DC;
#pragma unroll
            for (int i = 0; i < DC; ++i) {
                if (it == 0) {
                    const double m0 = run.prior[0], m1 = run.prior[1], m2 = run.prior[2], m3 = run.prior[3];
                    if (side == 0) { q0[i] = dadd(m0, m2); q1[i] = dadd(m1, m3); }
                    else { q0[i] = dadd(m0, m1); q1[i] = dadd(m2, m3); }
                } else {
                    const double2 q = v2c[i];
                    q0[i] = q.x;
                    q1[i] = q.y;
                }
            }
            const int s = (side ? run.sz : run.sx)[ch] & 1;
            double2 *out = run.c2v[side] + static_cast<size_t>(ch) * DC;
            if (!check_f64_row_fast<DC>(q0, q1, s, side, out, 1)) check_f64_row<DC>(q0, q1, s, side, out, 1);
            if (test_now) bad += fails(side, ch);
        }
        if (test_now) post_count(bad);
        if (!grid_barrier(run.bar, run.err)) return;
        if (test_now) {
            const int total_bad = *reinterpret_cast<volatile int *>(&run.bad[tests & 1]);
            ++tests;
            if (total_bad == 0) {
                ok = true;
                iters = it;
                break;
            }
        }
        // variable phase: decisions and new v2c (jointbp_ets.cpp:2451-2519)
        for (int v = tid; v < n; v += nthreads) {
            size_t ox[DV], oz[DV];
            bool vx[DV], vz[DV];
            double ax[DV], bx[DV], az[DV], bz[DV];
#pragma unroll
            for (int k = 0; k < DV; ++k) {
                const int ex = __ldg(code.s[0].var_edge + v * DV + k), ez = __ldg(code.s[1].var_edge + v * DV + k);
                vx[k] = ex >= 0;
                vz[k] = ez >= 0;
                ox[k] = vx[k] ? static_cast<size_t>(ex) : 0;
                oz[k] = vz[k] ? static_cast<size_t>(ez) : 0;
                const double2 cx = vx[k] ? run.c2v[0][ox[k]] : make_double2(1.0, 1.0);
                const double2 cz = vz[k] ? run.c2v[1][oz[k]] : make_double2(1.0, 1.0);
                ax[k] = cx.x; bx[k] = cx.y; az[k] = cz.x; bz[k] = cz.y;
            }
            bool fast_ok = true;
            int best = var_f64_update<DV, false, true>(rv, mv, 0.0, 0, 0, ox, oz, vx, vz, ax, bx, az, bz, fast_ok);
            if (!fast_ok) best = var_f64_update<DV, false, false>(rv, mv, 0.0, 0, 0, ox, oz, vx, vz, ax, bx, az, bz, fast_ok);
            run.est[v] = static_cast<uint8_t>(best);
        }
        if (!grid_barrier(run.bar, run.err)) return;
        if (it + 1 == run.max_iter) {
            // the last iteration's decisions have no check phase after them: a test of their own
            if (threadIdx.x == 0) bad_sh = 0;
            __syncthreads();
            int lbad = 0;
            for (int row = tid; row < M; row += nthreads) {
                const int side = row >= mx, ch = side ? row - mx : row;
                lbad += fails(side, ch);
            }
            post_count(lbad);
            if (!grid_barrier(run.bar, run.err)) return;
            if (*reinterpret_cast<volatile int *>(&run.bad[tests & 1]) == 0) {
                ok = true;
                iters = run.max_iter;
            }
        }
    }
    if (tid == 0)
        account_trial(run.cnt, run.hist, run.res_out, run.max_iter, run.local, iters,
                      ok ? (kResSyndromeOk | kResBpOk) : 0, ok, ok, false, false);
}

}  // namespace jbp
