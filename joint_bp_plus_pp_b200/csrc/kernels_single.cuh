// One trial per launch (FP64, and the FP32 LLR form at the end of this file), for calls that
// decode one or a few trials -- the drop-in's
// cuda_bp_decode decodes one trial per call (jointbp_cuda.cu:681-1104).  A cooperative launch of
// small blocks, about one per SM, runs the whole BP loop of the trial: the check phase with one
// thread per check row, the variable phase with one thread per variable and the syndrome test,
// separated by a grid barrier (the phases are bound by the latency of each thread's FP64 chain,
// 23 cycles per dependent operation, so spreading them over the SMs shortens nothing but the
// wait for issue slots), instead of the slot engine's per-iteration kernels over warps of 32 slots of
// which one would be busy.  The arithmetic is the slot engine's FP64 path (check_f64_row,
// var_f64_update), so decisions and iteration counts are the same bit for bit.  Messages stay in
// L2, position-major ([side][pos][check]) so that a warp's check rows read and write them
// coalesced; the variable phase gathers and scatters through the code's edge lists.  Each v2c
// message carries its variable's decision bit of that side in the sign of its first value, so
// the syndrome test of the check phase reads no memory of its own.
#pragma once

#include "kernels_bp.cuh"
#include "kernels_slots.cuh"

namespace jbp {

constexpr int kSingleThreads = 64;
constexpr int kSingleBlocks = 144;   // about one block per SM: the phases are latency-bound per thread
constexpr int kSingleMaxTrials = 3;      // trials (launches) of one run, each with its own barrier word
constexpr int kSingleErrWord = 6;        // int index of the error flag among the control words
constexpr unsigned long long kGridBarrierWaitNs = 1000000000ull;   // a barrier gives up after 1 s
constexpr unsigned long long kBarErr = 1ull << 31;

struct SingleRun {
    DevCode code;
    const uint8_t *sx, *sz;         // target syndrome bits, one byte per check (bit 0)
    double prior[4];                // normalized prior of the trial
    int max_iter, check_warmup, check_interval;
    double2 *c2v[2], *v2c[2];       // [side][pos * m_side + check] (k_single_llr: float / uint2 entries)
    uint8_t *est;                   // [n] decisions (0..3): the caller's output buffer
    // this launch's barrier word, zero at launch: arrivals in bits 0-30, the error bit 31, and in
    // bits 32-63 the number of (block, test) pairs in which the block found a failing check
    unsigned long long *bar;
    int *err;                       // set when a barrier gave up (the launch then ends)
    DevCounters *cnt;
    unsigned long long *hist;
    jbp_trial_result *res_out;
    long long local;                // the trial's index in the run (result record, counters)
};

// Grid-wide barrier of a cooperative launch (every block resident) on one 64-bit word.  Each
// block adds one arrival -- plus 2^32 when one of its threads passed a nonzero `flag` -- with
// release semantics, and waits with acquire loads until the arrivals reach the number of
// barriers it has passed times the grid size (`target`, kept by the caller).  At a `test`
// barrier *any says whether some block set its flag: the upper half grew since the last test
// barrier.  Every block reads the same answer: the word holds all of this barrier's flags once
// the arrivals are complete, and no block can add the next test's flags before every block has
// passed the barrier in between (test barriers never follow one another).  A wait that lasts
// kGridBarrierWaitNs sets the error bit, which ends the other blocks' waits too, and *err; the
// barrier then returns false and the caller returns.
__device__ __forceinline__ bool grid_sync(unsigned long long *bar, int *err, int flag, bool test, unsigned &target,
                                          unsigned &flags_seen, bool &any) {
    __shared__ int sync_sh[2];
    const int block_flag = __syncthreads_or(flag);
    target += gridDim.x;
    if (threadIdx.x == 0) {
        const unsigned long long add = 1ull | (block_flag ? (1ull << 32) : 0ull);
        asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(bar), "l"(add) : "memory");
        bool ok = true;
        unsigned long long cur, t0 = 0;
        for (bool first = true;; first = false) {
            asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(cur) : "l"(bar) : "memory");
            if (cur & kBarErr) { ok = false; break; }
            if (static_cast<int>((static_cast<unsigned>(cur) & 0x7FFFFFFFu) - target) >= 0) break;
            unsigned long long t;
            asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
            if (first) {
                t0 = t;
            } else if (t - t0 > kGridBarrierWaitNs) {
                atomicOr(bar, kBarErr);
                atomicExch(err, 1);
                ok = false;
                break;
            }
        }
        int a = 0;
        if (test) {
            const unsigned f = static_cast<unsigned>(cur >> 32);
            a = f != flags_seen;
            flags_seen = f;
        }
        sync_sh[0] = ok;
        sync_sh[1] = a;
    }
    __syncthreads();
    any = sync_sh[1] != 0;
    return sync_sh[0] != 0;
}

// Offset of edge e = c * DC + pos (the code's check-major edge numbering) in the
// position-major message arrays of a side with m checks.
template <int DC>
__device__ __forceinline__ size_t single_msg_off(int e, int m) {
    const int c = e / DC;
    return static_cast<size_t>(e - c * DC) * m + c;
}

template <int DC, int DV>
__global__ void __launch_bounds__(kSingleThreads, 1) k_single_f64(const __grid_constant__ SingleRun run) {
    const DevCode &code = run.code;
    const int mx = code.s[0].m, mz = code.s[1].m, M = mx + mz, n = code.n;
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
    // message offsets of this thread's first variable stay in registers (one variable per
    // thread on codes of up to 9,216 qubits); further variables compute theirs
    size_t var_ox[DV], var_oz[DV];
    bool var_vx[DV], var_vz[DV];
    auto edges_of = [&](int v, size_t *ox, size_t *oz, bool *vx, bool *vz) {
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            const int ex = __ldg(code.s[0].var_edge + v * DV + k), ez = __ldg(code.s[1].var_edge + v * DV + k);
            vx[k] = ex >= 0;
            vz[k] = ez >= 0;
            ox[k] = vx[k] ? single_msg_off<DC>(ex, mx) : 0;
            oz[k] = vz[k] ? single_msg_off<DC>(ez, mz) : 0;
        }
    };
    if (tid < n) edges_of(tid, var_ox, var_oz, var_vx, var_vz);
    unsigned target = 0, flags_seen = 0;
    bool any_bad = false;
    int iters = run.max_iter;
    bool ok = false;
    // the check schedule of the slot engine's check_due (1-based iteration k1)
    auto due = [&](int k1) {
        return k1 >= run.max_iter || (k1 > run.check_warmup && (k1 - run.check_warmup) % run.check_interval == 0);
    };
    for (int it = 0; it < run.max_iter; ++it) {
        // the test of iteration it's decisions (1-based) rides in this check phase, which reads
        // the messages that carry them; when they satisfy both syndromes, the phase's outputs
        // are unused
        const bool test_now = it >= 1 && due(it);
        int bad = 0;
        // check phase: new c2v of every check row (jointbp_ets.cpp:2373-2449); the parity of the
        // decision bits against the target syndrome (jointbp_ets.cpp:2521-2525)
        for (int row = tid; row < M; row += nthreads) {
            const int side = row >= mx, ch = side ? row - mx : row, ms = side ? mz : mx;
            const int s = (side ? run.sz : run.sx)[ch] & 1;
            double q0[DC], q1[DC];
            const double2 *v2c = run.v2c[side] + ch;
            unsigned long long par = 0;
#pragma unroll
            for (int i = 0; i < DC; ++i) {
                if (it == 0) {
                    const double m0 = run.prior[0], m1 = run.prior[1], m2 = run.prior[2], m3 = run.prior[3];
                    if (side == 0) { q0[i] = dadd(m0, m2); q1[i] = dadd(m1, m3); }
                    else { q0[i] = dadd(m0, m1); q1[i] = dadd(m2, m3); }
                } else {
                    const double2 q = v2c[static_cast<size_t>(i) * ms];
                    const unsigned long long bits = static_cast<unsigned long long>(__double_as_longlong(q.x));
                    par ^= bits;
                    q0[i] = __longlong_as_double(static_cast<long long>(bits & ~(1ull << 63)));
                    q1[i] = q.y;
                }
            }
            if (test_now) bad |= static_cast<int>(par >> 63) != s;
            double2 *out = run.c2v[side] + ch;
            if (!check_f64_row_fast<DC>(q0, q1, s, side, out, ms)) check_f64_row<DC>(q0, q1, s, side, out, ms);
        }
        if (!grid_sync(run.bar, run.err, bad, test_now, target, flags_seen, any_bad)) return;
        if (test_now && !any_bad) {
            ok = true;
            iters = it;
            break;
        }
        // variable phase: decisions and new v2c (jointbp_ets.cpp:2451-2519)
        for (int v = tid; v < n; v += nthreads) {
            size_t ox[DV], oz[DV];
            bool vx[DV], vz[DV];
            if (v == tid) {
#pragma unroll
                for (int k = 0; k < DV; ++k) { ox[k] = var_ox[k]; oz[k] = var_oz[k]; vx[k] = var_vx[k]; vz[k] = var_vz[k]; }
            } else {
                edges_of(v, ox, oz, vx, vz);
            }
            double ax[DV], bx[DV], az[DV], bz[DV];
#pragma unroll
            for (int k = 0; k < DV; ++k) {
                const double2 cx = vx[k] ? run.c2v[0][ox[k]] : make_double2(1.0, 1.0);
                const double2 cz = vz[k] ? run.c2v[1][oz[k]] : make_double2(1.0, 1.0);
                ax[k] = cx.x; bx[k] = cx.y; az[k] = cz.x; bz[k] = cz.y;
            }
            bool fast_ok = true;
            int best = var_f64_update<DV, false, true, true>(rv, mv, 0.0, 0, 0, ox, oz, vx, vz, ax, bx, az, bz, fast_ok);
            if (!fast_ok)
                best = var_f64_update<DV, false, false, true>(rv, mv, 0.0, 0, 0, ox, oz, vx, vz, ax, bx, az, bz, fast_ok);
            run.est[v] = static_cast<uint8_t>(best);
        }
        if (!grid_sync(run.bar, run.err, 0, false, target, flags_seen, any_bad)) return;
        if (it + 1 == run.max_iter) {
            // the last iteration's decisions have no check phase after them: a test of their own
            // from the sign bits of the messages
            int lbad = 0;
            for (int row = tid; row < M; row += nthreads) {
                const int side = row >= mx, ch = side ? row - mx : row, ms = side ? mz : mx;
                const double2 *v2c = run.v2c[side] + ch;
                unsigned long long par = 0;
#pragma unroll
                for (int i = 0; i < DC; ++i) par ^= static_cast<unsigned long long>(__double_as_longlong(v2c[static_cast<size_t>(i) * ms].x));
                lbad |= static_cast<int>(par >> 63) != ((side ? run.sz : run.sx)[ch] & 1);
            }
            if (!grid_sync(run.bar, run.err, lbad, true, target, flags_seen, any_bad)) return;
            if (!any_bad) {
                ok = true;
                iters = run.max_iter;
            }
        }
    }
    if (tid == 0)
        account_trial(run.cnt, run.hist, run.res_out, run.max_iter, run.local, iters,
                      ok ? (kResSyndromeOk | kResBpOk) : 0, ok, ok, false, false);
}

// The FP32 form: the slot engine's LLR arithmetic (llr_check_row, var_llr_core, the log prior of
// llr_prior_entry) on FP32 messages, so that decisions and iteration counts equal those of the
// slot engine's FP32 decoder.  The run's message arrays hold, position-major, FP32 c2v and v2c
// pairs (message bits, the variable's decision bit of that side): an LLR's sign is its own, so
// the decision bit travels beside it, in the same 8-byte store.
template <int DC, int DV>
__global__ void __launch_bounds__(kSingleThreads, 1) k_single_llr(const __grid_constant__ SingleRun run) {
    const DevCode &code = run.code;
    const int mx = code.s[0].m, mz = code.s[1].m, M = mx + mz, n = code.n;
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nthreads = gridDim.x * blockDim.x;
    float *const c2vx = reinterpret_cast<float *>(run.c2v[0]), *const c2vz = reinterpret_cast<float *>(run.c2v[1]);
    uint2 *const v2cx = reinterpret_cast<uint2 *>(run.v2c[0]), *const v2cz = reinterpret_cast<uint2 *>(run.v2c[1]);
    __shared__ float lp_sh[6];
    if (threadIdx.x < 6) lp_sh[threadIdx.x] = llr_prior_entry(threadIdx.x, run.prior[0], run.prior[1], run.prior[2], run.prior[3]);
    __syncthreads();
    const float4 lp = make_float4(lp_sh[0], lp_sh[1], lp_sh[2], lp_sh[3]);
    const float lpx = lp_sh[4], lpz = lp_sh[5];
    size_t var_ox[DV], var_oz[DV];
    bool var_vx[DV], var_vz[DV];
    auto edges_of = [&](int v, size_t *ox, size_t *oz, bool *vx, bool *vz) {
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            const int ex = __ldg(code.s[0].var_edge + v * DV + k), ez = __ldg(code.s[1].var_edge + v * DV + k);
            vx[k] = ex >= 0;
            vz[k] = ez >= 0;
            ox[k] = vx[k] ? single_msg_off<DC>(ex, mx) : 0;
            oz[k] = vz[k] ? single_msg_off<DC>(ez, mz) : 0;
        }
    };
    if (tid < n) edges_of(tid, var_ox, var_oz, var_vx, var_vz);
    unsigned target = 0, flags_seen = 0;
    bool any_bad = false;
    int iters = run.max_iter;
    bool ok = false;
    auto due = [&](int k1) {
        return k1 >= run.max_iter || (k1 > run.check_warmup && (k1 - run.check_warmup) % run.check_interval == 0);
    };
    for (int it = 0; it < run.max_iter; ++it) {
        const bool test_now = it >= 1 && due(it);
        int bad = 0;
        for (int row = tid; row < M; row += nthreads) {
            const int side = row >= mx, ch = side ? row - mx : row, ms = side ? mz : mx;
            const unsigned s = (side ? run.sz : run.sx)[ch] & 1;
            const uint2 *in = (side ? v2cz : v2cx) + ch;
            float *out = (side ? c2vz : c2vx) + ch;
            const float lp_in = side ? lpz : lpx;
            unsigned par = 0;
            llr_check_row<DC>(
                [&](int i) -> float {
                    if (it == 0) return lp_in;
                    const uint2 q = in[static_cast<size_t>(i) * ms];
                    par ^= q.y;
                    return __uint_as_float(q.x);
                },
                s, [&](int i, float y) { out[static_cast<size_t>(i) * ms] = y; });
            if (test_now) bad |= par != s;
        }
        if (!grid_sync(run.bar, run.err, bad, test_now, target, flags_seen, any_bad)) return;
        if (test_now && !any_bad) {
            ok = true;
            iters = it;
            break;
        }
        for (int v = tid; v < n; v += nthreads) {
            size_t ox[DV], oz[DV];
            bool vx[DV], vz[DV];
            if (v == tid) {
#pragma unroll
                for (int k = 0; k < DV; ++k) { ox[k] = var_ox[k]; oz[k] = var_oz[k]; vx[k] = var_vx[k]; vz[k] = var_vz[k]; }
            } else {
                edges_of(v, ox, oz, vx, vz);
            }
            float lx[DV], lz[DV], outx[DV], outz[DV];
#pragma unroll
            for (int k = 0; k < DV; ++k) {
                lx[k] = vx[k] ? c2vx[ox[k]] : 0.0f;
                lz[k] = vz[k] ? c2vz[oz[k]] : 0.0f;
            }
            const int best = var_llr_core<DV>(lx, lz, lp, outx, outz);
#pragma unroll
            for (int k = 0; k < DV; ++k) {
                if (vx[k]) v2cx[ox[k]] = make_uint2(__float_as_uint(outx[k]), static_cast<unsigned>(best & 1));
                if (vz[k]) v2cz[oz[k]] = make_uint2(__float_as_uint(outz[k]), static_cast<unsigned>(best >> 1));
            }
            run.est[v] = static_cast<uint8_t>(best);
        }
        if (!grid_sync(run.bar, run.err, 0, false, target, flags_seen, any_bad)) return;
        if (it + 1 == run.max_iter) {
            int lbad = 0;
            for (int row = tid; row < M; row += nthreads) {
                const int side = row >= mx, ch = side ? row - mx : row, ms = side ? mz : mx;
                unsigned par = 0;
#pragma unroll
                for (int i = 0; i < DC; ++i) par ^= (side ? v2cz : v2cx)[static_cast<size_t>(i) * ms + ch].y;
                lbad |= par != static_cast<unsigned>((side ? run.sz : run.sx)[ch] & 1);
            }
            if (!grid_sync(run.bar, run.err, lbad, true, target, flags_seen, any_bad)) return;
            if (!any_bad) {
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
