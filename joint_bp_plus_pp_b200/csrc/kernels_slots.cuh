// Slot lifecycle kernels: hard-decision syndrome test, retirement, success classification,
// refill from the trial source, error sampling and fresh-trial syndromes.
#pragma once

#include "engine.cuh"

namespace jbp {

__device__ __forceinline__ int xbit(int s) { return s & 1; }          // X or Y
__device__ __forceinline__ int zbit(int s) { return (s >> 1) & 1; }   // Z or Y

// ------------------------------------------------------------------ samplers

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11): 10 rounds of the 4x32 bijection.
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

// Depolarizing channel as the reference maps a uniform u in [0,1) (jointbp_ets.cpp:5937-5945).
__device__ __forceinline__ uint8_t pauli_from_uniform(double u, double p) {
    const double q = __dsub_rn(1.0, p);
    if (u < q) return 0;
    const double v = __ddiv_rn(__dsub_rn(u, q), p);
    return v < 1.0 / 3.0 ? 1 : (v < 2.0 / 3.0 ? 2 : 3);
}

// Philox stream: qubit v of trial t uses half of block (v/2, t); 53-bit uniform.
__device__ __forceinline__ uint8_t sample_philox(unsigned long long seed, long long t, int v, double p) {
    const uint4 r = philox4x32_10(make_uint4(static_cast<uint32_t>(v >> 1), static_cast<uint32_t>(t),
                                             static_cast<uint32_t>(static_cast<unsigned long long>(t) >> 32),
                                             0x4A425042u),
                                  make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)));
    const unsigned long long x = (v & 1) ? (static_cast<unsigned long long>(r.w) << 32 | r.z)
                                         : (static_cast<unsigned long long>(r.y) << 32 | r.x);
    const double u = static_cast<double>(x >> 11) * 0x1.0p-53;
    return pauli_from_uniform(u, p);
}

// Both qubits 2*vp and 2*vp+1 of one Philox block (the same stream as sample_philox).
__device__ __forceinline__ void sample_philox_pair(unsigned long long seed, long long t, int vp, double p, uint8_t &e0,
                                                   uint8_t &e1) {
    const uint4 r = philox4x32_10(make_uint4(static_cast<uint32_t>(vp), static_cast<uint32_t>(t),
                                             static_cast<uint32_t>(static_cast<unsigned long long>(t) >> 32),
                                             0x4A425042u),
                                  make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)));
    const unsigned long long x0 = static_cast<unsigned long long>(r.y) << 32 | r.x;
    const unsigned long long x1 = static_cast<unsigned long long>(r.w) << 32 | r.z;
    e0 = pauli_from_uniform(static_cast<double>(x0 >> 11) * 0x1.0p-53, p);
    e1 = pauli_from_uniform(static_cast<double>(x1 >> 11) * 0x1.0p-53, p);
}

// Error rate of trial t: p, or with p_max > p a uniform draw from [p, p_max) keyed by
// (seed, t) (its own Philox stream, independent of the error samples).
__device__ __forceinline__ double trial_p(double p, double p_max, unsigned long long seed, long long t) {
    if (!(p_max > p)) return p;
    const uint4 r = philox4x32_10(make_uint4(0xFFFFFFFFu, static_cast<uint32_t>(t),
                                             static_cast<uint32_t>(static_cast<unsigned long long>(t) >> 32),
                                             0x50524154u),
                                  make_uint2(static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32)));
    const double u = static_cast<double>((static_cast<unsigned long long>(r.y) << 32 | r.x) >> 11) * 0x1.0p-53;
    return p + (p_max - p) * u;
}

// ------------------------------------------------------------------ per-iteration kernels

// Whether iteration k1 (1-based) of a slot ends with a syndrome test: always at max_iter,
// else every check_interval iterations after check_warmup (jointbp_cuda.cu:971-975; the
// defaults 0 and 1 test every iteration as the CPU decoder does).
__device__ __forceinline__ bool check_due(const DevRun &run, int k1) {
    return k1 >= run.max_iter || (k1 > run.check_warmup && (k1 - run.check_warmup) % run.check_interval == 0);
}

// Hard-decision syndrome test (jointbp_ets.cpp:2521-2525) on bit planes.  A warp takes one
// group and 32 consecutive check rows: lane r XORs the decision words of its row's
// variables, which gives the row's parity for all 32 slots at once; slots whose parity
// differs from the target are OR-ed into the group's unsatisfied mask of that side.
static __global__ void __launch_bounds__(256) k_syndrome_check(DevCode code, DevRun run) {
    const int lane = threadIdx.x & 31;
    const int n = code.n, G = run.S / kGroup;
    const int mx = code.s[0].m, M = mx + code.s[1].m;
    const int blocks = (M + 31) >> 5;
    const unsigned total = static_cast<unsigned>(*run.n_groups) * blocks;
    const size_t plane = plane_offset(run, n, 0);
    for (unsigned w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / static_cast<unsigned>(blocks));
        const int rb = static_cast<int>(w - static_cast<unsigned>(gi) * blocks);
        const int group = run.groups[gi];
        const int slot = group * kGroup + lane;
        const bool due = (run.flags[slot] & kRunning) && check_due(run, run.iter[slot] + 1);
        const unsigned due_mask = __ballot_sync(0xffffffffu, due);
        if (!due_mask) continue;
        if (rb == 0 && lane == 0) atomicAdd(&run.cnt->syndrome_tests, static_cast<unsigned long long>(__popc(due_mask)));
        const int row = rb * 32 + lane;
        unsigned mm[2] = {0u, 0u};
        if (row < M) {
            const int side = row >= mx;
            const int ch = side ? row - mx : row;
            const int dc = side ? code.s[1].dc : code.s[0].dc;
            const int *chk_var = side ? code.s[1].chk_var : code.s[0].chk_var;
            const unsigned *planes = (side ? run.estz : run.estx) + plane + static_cast<size_t>(group) * n;
            unsigned par = 0;
            for (int i = 0; i < dc; ++i) par ^= planes[__ldg(chk_var + ch * dc + i)];
            mm[side] = (par ^ run.synm[static_cast<size_t>(row) * G + group]) & due_mask;
        }
        const unsigned ux = __reduce_or_sync(0xffffffffu, mm[0]);
        const unsigned uz = __reduce_or_sync(0xffffffffu, mm[1]);
        if (lane == 0 && ux) atomicOr(&run.unsat_mask[group], ux);
        if (lane == 1 && uz) atomicOr(&run.unsat_mask[G + group], uz);
        if (run.pp && (ux | uz)) {
            // per-slot unsatisfied counts (post-processing gates and the us history):
            // lane s gathers bit s of the 32 rows' mismatch masks
            for (int side = 0; side < 2; ++side) {
                const unsigned any = side ? uz : ux;
                if (!any) continue;
                int cnt = 0;
                for (int b = 0; b < 32; ++b) {
                    const unsigned col = __ballot_sync(0xffffffffu, (mm[side] >> b) & 1u);
                    if (lane == b) cnt = __popc(col);
                }
                if (cnt) atomicAdd(&run.unsat[side * run.S + slot], cnt);
            }
        }
    }
}

// Post-processing bookkeeping: slots whose decisions differ from 1 and 2 iterations back
// (the reference's est == prev_est / prev_prev_est, jointbp_ets.cpp:2555-2556), for groups
// holding a slot at or past the first iteration that can trigger post-processing.
static __global__ void __launch_bounds__(256) k_stall_compare(DevCode code, DevRun run) {
    const int lane = threadIdx.x & 31;
    const int n = code.n;
    const int chunks = (n + 31) >> 5;
    const unsigned total = static_cast<unsigned>(*run.n_groups) * chunks;
    const size_t p0 = plane_offset(run, n, 0), p1 = plane_offset(run, n, 1), p2 = plane_offset(run, n, 2);
    for (unsigned w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / static_cast<unsigned>(chunks));
        const int cb = static_cast<int>(w - static_cast<unsigned>(gi) * chunks);
        const int group = run.groups[gi];
        const int slot = group * kGroup + lane;
        const bool late = (run.flags[slot] & kRunning) && run.iter[slot] + 1 >= run.llr_from;
        if (!__any_sync(0xffffffffu, late)) continue;
        const int v = cb * 32 + lane;
        unsigned d1 = 0, d2 = 0;
        if (v < n) {
            const size_t o = static_cast<size_t>(group) * n + v;
            const unsigned cx = run.estx[p0 + o], cz = run.estz[p0 + o];
            d1 = (cx ^ run.estx[p1 + o]) | (cz ^ run.estz[p1 + o]);
            d2 = (cx ^ run.estx[p2 + o]) | (cz ^ run.estz[p2 + o]);
        }
        d1 = __reduce_or_sync(0xffffffffu, d1);
        d2 = __reduce_or_sync(0xffffffffu, d2);
        if (lane == 0 && d1) atomicOr(&run.dprev[group], d1);
        if (lane == 1 && d2) atomicOr(&run.dpprev[group], d2);
    }
}

// detect_us_oscillation (jointbp_ets.cpp:2021-2053) over the last 100 samples of
// max(us_x, us_z), kept by iteration number modulo 100 (samples k1-99 .. k1).
static __device__ bool us_oscillation(const unsigned short *h, int k1) {
    if (k1 < 100) return false;
    // one pass over the window k1-99 .. k1 (ring position advanced without a division per entry):
    // range, sum, and the sign changes of the successive differences
    int idx = (k1 - 99) % 100;
    int prev = h[idx], mn = prev, mx = prev;
    long long sum = prev;
    int prev_sign = 0, turns = 0;
    for (int i = 1; i < 100; ++i) {
        if (++idx == 100) idx = 0;
        const int v = h[idx];
        mn = v < mn ? v : mn;
        mx = v > mx ? v : mx;
        sum += v;
        const int d = v - prev;
        const int sg = d > 0 ? 1 : (d < 0 ? -1 : 0);
        if (sg) {
            if (prev_sign && sg != prev_sign) turns++;
            prev_sign = sg;
        }
        prev = v;
    }
    const double mean = static_cast<double>(sum) / 100.0;
    if (mean <= 0.0) return false;
    int min_range = static_cast<int>(mean * 0.2);
    if (min_range < 10) min_range = 10;
    if (mx - mn < min_range) return false;
    return turns >= 2;
}

// us_oscillation computed by the 32 lanes of a warp (all call it; every lane gets the result).
// Each lane takes window entries lane, lane + 32, ...; min, max and sum reduce exactly.  Two or
// more sign changes among the nonzero signs of the successive differences happen exactly when
// both signs occur and each sign occurs after some occurrence of the other (a sequence with at
// most one change is all of one sign, then all of the other): with P and N the positions of
// the rises and falls, maxP > minN and maxN > minP.
static __device__ bool us_oscillation_warp(const unsigned short *h, int k1) {
    if (k1 < 100) return false;
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, base = k1 - 99;
    int mn = 0x7fffffff, mx = -1, sum = 0;
    unsigned rise[4], fall[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const int i = c * 32 + lane;
        int d = 0;
        if (i < 100) {
            const int v = h[(base + i) % 100];
            mn = v < mn ? v : mn;
            mx = v > mx ? v : mx;
            sum += v;
            if (i > 0) d = v - static_cast<int>(h[(base + i - 1) % 100]);
        }
        rise[c] = __ballot_sync(full, d > 0);
        fall[c] = __ballot_sync(full, d < 0);
    }
    mn = __reduce_min_sync(full, mn);
    mx = __reduce_max_sync(full, mx);
    sum = __reduce_add_sync(full, sum);
    const double mean = static_cast<double>(sum) / 100.0;
    if (mean <= 0.0) return false;
    int min_range = static_cast<int>(mean * 0.2);
    if (min_range < 10) min_range = 10;
    if (mx - mn < min_range) return false;
    int minP = -1, maxP = -1, minN = -1, maxN = -1;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (rise[c]) {
            if (minP < 0) minP = c * 32 + __ffs(rise[c]) - 1;
            maxP = c * 32 + 31 - __clz(rise[c]);
        }
        if (fall[c]) {
            if (minN < 0) minN = c * 32 + __ffs(fall[c]) - 1;
            maxN = c * 32 + 31 - __clz(fall[c]);
        }
    }
    return minP >= 0 && minN >= 0 && maxP > minN && maxN > minP;
}

// Counts the finished iteration; a slot retires when its checked syndrome matches or it
// reaches max_iter (the CPU's iteration accounting, jointbp_ets.cpp:2733-2735, 3078).
static __global__ void k_retire(DevRun run) {
    const int gi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (gi >= *run.n_groups) return;
    const int lane = threadIdx.x & 31;
    const int group = run.groups[gi];
    const int slot = group * kGroup + lane;
    const int G = run.S / kGroup;
    const unsigned ux_mask = run.unsat_mask[group], uz_mask = run.unsat_mask[G + group];
    const unsigned bad = ux_mask | uz_mask;
    const unsigned dp = run.pp ? run.dprev[group] : 0u, dpp = run.pp ? run.dpprev[group] : 0u;
    __syncwarp();
    if (lane == 0) {
        run.unsat_mask[group] = 0u;
        run.unsat_mask[G + group] = 0u;
        if (run.pp) {
            run.dprev[group] = 0u;
            run.dpprev[group] = 0u;
        }
    }
    if (!(run.flags[slot] & kRunning)) return;
    const int k1 = run.iter[slot] + 1;
    run.iter[slot] = k1;
    const bool conv = check_due(run, k1) && !((bad >> lane) & 1u);
    if (run.freeze_syn) {
        // a side whose syndrome matches at this check freezes; the check kernel of the next
        // iteration writes its deterministic messages (bits 2, 3) once
        int f = run.frz[slot] & 3;
        if (check_due(run, k1)) {
            if (!((ux_mask >> lane) & 1u) && !(f & 1)) f |= 1 | 4;
            if (!((uz_mask >> lane) & 1u) && !(f & 2)) f |= 2 | 8;
        }
        run.frz[slot] = f;
    }
    if (run.pp) {
        const int S = run.S;
        const int ux = run.unsat[slot], uz = run.unsat[S + slot];
        run.unsat[slot] = 0;
        run.unsat[S + slot] = 0;
        if (!conv) {
            // stall / oscillation triggers and the flip window (jointbp_ets.cpp:2536-2633)
            const int sig = ux > uz ? ux : uz;
            unsigned short *h = run.us_hist + static_cast<size_t>(slot) * 100;
            h[k1 % 100] = static_cast<unsigned short>(sig > 65535 ? 65535 : sig);
            const bool same = k1 >= 2 && !((dp >> lane) & 1u);
            const bool osc = k1 >= 3 && !((dpp >> lane) & 1u) && !same;
            const bool allow = k1 >= 100 || k1 == run.max_iter;
            const int ss = same ? run.stall_same[slot] + 1 : 0;
            run.stall_same[slot] = ss;
            int st = run.pstate[slot];
            bool act = false;
            if (!(st & 1) && (ss >= 1 || k1 == run.max_iter) && allow) { st |= 1; act = true; }
            if (!(st & 2) && osc && allow) { st |= 2; act = true; }
            if (!(st & 4) && allow && us_oscillation(h, k1)) { st |= 4; act = true; }
            run.pstate[slot] = st;
            if (act && run.act_k[slot] == 0 && run.flip_hist > 0) run.act_k[slot] = k1;
            int mode = 0;
            if (st && sig <= 20) mode = kPpInLoop;
            else if (k1 >= run.max_iter) mode = kPpPost;
            if (mode) {
                run.pp_mode[slot] = mode;
                run.pp_list[atomicAdd(run.n_pp, 1)] = slot;
            }
        }
    }
    if (conv || k1 >= run.max_iter) {
        run.res_iters[slot] = k1;
        run.res_flags[slot] = conv ? 3 : 0;
        run.flags[slot] = kFinished;
        run.retired[atomicAdd(run.n_retired, 1)] = slot;
    }
}

// Warp-wide test of vec (smem, `words` 64-bit words) for membership in a row space given
// in echelon form by its highest bits (in_row_space, jointbp_ets.cpp:904-920): repeatedly
// clear the highest set bit with the basis row that has it as pivot; a bit with no such
// row means the vector is outside the space.  vec is destroyed.
static __device__ bool warp_in_row_space(uint64_t *vec, int words, const uint64_t *rows, const int *pivot_row) {
    const int lane = threadIdx.x & 31;
    for (int guard = 0; guard < 1 << 20; ++guard) {
        int hw = -1;
        for (int w = lane; w < words; w += 32)
            if (vec[w]) hw = w;
        hw = __reduce_max_sync(0xffffffffu, hw + 1) - 1;
        if (hw < 0) return true;
        const uint64_t top = vec[hw];
        const int bit = hw * 64 + 63 - __clzll(static_cast<long long>(top));
        const int r = pivot_row[bit];
        __syncwarp();
        if (r < 0) return false;
        const uint64_t *row = rows + static_cast<size_t>(r) * words;
        for (int w = lane; w <= hw; w += 32) vec[w] ^= row[w];
        __syncwarp();
    }
    return false;
}

// Run Summary counters exactly as the simulate loop derives them (jointbp_ets.cpp:6012-6019,
// 6070-6080, 6199-6224), the iteration histogram and the per-trial record, from a trial's
// iterations, result flags (ResultBit) and classification.  One thread per trial.
__device__ __forceinline__ void account_trial(DevCounters *c, unsigned long long *hist, jbp_trial_result *res_out,
                                              int max_iter, long long local, int iters, int rf, bool ok, bool success,
                                              bool exact, bool stab) {
    const bool in_dec = rf & kResPpInDecode;
    const bool used_any = rf & kResUsedAny, used6 = rf & kResUsed6, used12 = rf & kResUsed12;
    const bool post = rf & kResPostEntered;
    const bool ets_ok = in_dec ? (rf & kResPpInEts) : (rf & kResEtsOk);
    const bool flip_ok = in_dec ? (rf & kResPpInFlip) : (rf & kResFlipOk);
    const bool osd_ok = rf & kResOsdOk;
    const bool osd_success = osd_ok || (in_dec && !(rf & kResPpInEts) && !(rf & kResPpInFlip));
    const bool pp_this = success && (in_dec || ets_ok || flip_ok || osd_ok);
    atomicAdd(&c->done, 1ull);
    atomicAdd(&c->total_iters, static_cast<unsigned long long>(iters));
    atomicAdd(&c->bp_trial_iterations, static_cast<unsigned long long>(iters));
    if (!success) atomicAdd(&c->failures, 1ull);
    if (!(rf & kResBpOk)) atomicAdd(&c->bp_fail, 1ull);
    if (exact) atomicAdd(&c->exact, 1ull);
    if (ok) atomicAdd(&c->syndrome_ok, 1ull);
    if (success && !exact && stab) atomicAdd(&c->stab_success, 1ull);
    if (in_dec && used_any) {
        atomicAdd(&c->ets_used, 1ull);
        if (used6) atomicAdd(&c->ets6_used, 1ull);
        if (used12) atomicAdd(&c->ets12_used, 1ull);
    }
    if (post) {
        if (rf & kResEtsPost) atomicAdd(&c->ets_used, 1ull);
        if (used6) atomicAdd(&c->ets6_used, 1ull);
        if (used12) atomicAdd(&c->ets12_used, 1ull);
    }
    if (success && ets_ok) {
        atomicAdd(&c->ets_saved, 1ull);
        if (used6) atomicAdd(&c->ets6_saved, 1ull);
        if (used12) atomicAdd(&c->ets12_saved, 1ull);
    }
    if (success && flip_ok) atomicAdd(&c->flip_pp_success, 1ull);
    if (pp_this) atomicAdd(&c->pp_success, 1ull);
    if (success && osd_success) atomicAdd(&c->osd_pp_success, 1ull);
    const bool learned = rf & kResLearned;
    if (success && learned) atomicAdd(&c->learned_success, 1ull);
    if (hist && iters >= 1 && iters <= max_iter) atomicAdd(&hist[iters], 1ull);
    if (res_out) {
        jbp_trial_result rec;
        rec.iterations = iters;
        rec.syndrome_ok = ok;
        rec.bp_ok = (rf & kResBpOk) ? 1 : 0;
        rec.success = success;
        rec.exact = exact;
        rec.stab_equiv = stab;
        rec.pp_success = pp_this;
        rec.pp_ets = ets_ok;
        rec.pp_flip = flip_ok;
        rec.pp_osd = osd_success;
        rec.ets_used_flags = static_cast<uint8_t>((used_any ? 1 : 0) | (used6 ? 2 : 0) | (used12 ? 4 : 0) |
                                                  ((rf & kResEtsPost) ? 8 : 0) | (post ? 16 : 0) |
                                                  (learned ? 32 : 0));
        rec.pp_in_decode = in_dec;
        rec.reserved = osd_ok;
        res_out[local] = rec;
    }
}

// Classifies each retired trial (jointbp_ets.cpp:6199-6245): exact match, stabilizer
// equivalence of the residual (x-part in rowspace(Hz), z-part in rowspace(Hx)), success;
// writes the per-trial record and estimate and updates the run counters.
static __global__ void k_classify(DevCode code, DevRun run) {
    extern __shared__ uint64_t smem_words[];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const int words = code.words;
    uint64_t *dx = smem_words + static_cast<size_t>(wib) * 2 * words;
    uint64_t *dz = dx + words;
    const int nret = *run.n_retired;
    const int n = code.n;
    const bool have_err = run.source != kSrcSyndromes;
    const size_t plane = plane_offset(run, n, 0);
    for (int r = blockIdx.x * wpb + wib; r < nret; r += gridDim.x * wpb) {
        const int slot = run.retired[r];
        const long long local = run.trial[slot] - run.first_trial;
        const int iters = run.res_iters[slot];
        const int rf = run.res_flags[slot];
        const bool ok = rf & kResSyndromeOk;
        for (int w = lane; w < words; w += 32) { dx[w] = 0; dz[w] = 0; }
        __syncwarp();
        bool exact = true;
        const uint8_t *err = run.err + static_cast<size_t>(slot) * n;
        const unsigned *px = run.estx + plane + static_cast<size_t>(slot / kGroup) * n;
        const unsigned *pz = run.estz + plane + static_cast<size_t>(slot / kGroup) * n;
        const int bit = slot % kGroup;
        constexpr int U = 8;  // chunks of 32 variables whose loads are issued together
        for (int base0 = 0; base0 < n; base0 += 32 * U) {
            unsigned xw[U], zw[U];
            int tv[U];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int v = base0 + u * 32 + lane;
                const bool in = v < n;
                xw[u] = in ? px[v] : 0u;
                zw[u] = in ? pz[v] : 0u;
                tv[u] = (in && have_err) ? err[v] : -1;
            }
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int base = base0 + u * 32;
                const int v = base + lane;
                const bool in = v < n;
                const int e = in ? static_cast<int>(((xw[u] >> bit) & 1u) | (((zw[u] >> bit) & 1u) << 1)) : 0;
                const int t = tv[u] >= 0 ? tv[u] : e;
                if (in && run.est_out) run.est_out[local * n + v] = static_cast<uint8_t>(e);
                if (t != e) exact = false;
                const unsigned bx = __ballot_sync(0xffffffffu, xbit(t) != xbit(e));
                const unsigned bz = __ballot_sync(0xffffffffu, zbit(t) != zbit(e));
                if (lane == 0 && base < n) {
                    const int sh = base & 32;  // which half of the 64-bit word
                    dx[base >> 6] |= static_cast<uint64_t>(bx) << sh;
                    dz[base >> 6] |= static_cast<uint64_t>(bz) << sh;
                }
            }
        }
        exact = __all_sync(0xffffffffu, exact) && have_err;
        __syncwarp();
        bool stab = false;
        if (have_err && ok) {
            stab = warp_in_row_space(dx, words, code.basis_rows[1], code.pivot_row[1]);
            if (stab) stab = warp_in_row_space(dz, words, code.basis_rows[0], code.pivot_row[0]);
        }
        const bool success = have_err ? (ok && stab) : ok;
        if (lane == 0) {
            account_trial(run.cnt, run.hist, run.res_out, run.max_iter, local, iters, rf, ok, success, exact, stab);
            run.flags[slot] = 0;
        }
        __syncwarp();
    }
}

// Hands the next trials of the source to the retired (or never used) slots.
// Entry i (0..5) of the LLR prior of a normalized prior (p0..p3 of I, X, Z, Y): the base-2 log
// weights (0..3) and the base-2 prior LLRs of the x bit (4) and the z bit (5) that seed the
// fresh v2c messages of the LLR decoders.
__device__ __forceinline__ float llr_prior_entry(int i, double p0, double p1, double p2, double p3) {
    switch (i) {
    case 0: return static_cast<float>(log2(p0));
    case 1: return static_cast<float>(log2(p1));
    case 2: return static_cast<float>(log2(p2));
    case 3: return static_cast<float>(log2(p3));
    case 4: return static_cast<float>(log2((p0 + p2) / (p1 + p3)));
    default: return static_cast<float>(log2((p0 + p1) / (p2 + p3)));
    }
}

static __global__ void k_refill(DevRun run, int precision) {
    const int nret = *run.n_retired;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < nret; r += gridDim.x * blockDim.x) {
        const int slot = run.retired[r];
        const unsigned long long t = atomicAdd(&run.cnt->next_trial, 1ull);
        if (t < static_cast<unsigned long long>(run.ntrials)) {
            run.trial[slot] = run.first_trial + static_cast<long long>(t);
            run.iter[slot] = 0;
            run.flags[slot] = kRunning;
            if (run.pp) {
                run.act_k[slot] = 0;
                run.pstate[slot] = 0;
                run.stall_same[slot] = 0;
            }
            if (run.freeze_syn) run.frz[slot] = 0;
            // prior = normalize(1-p, p/3, p/3, p/3) (jointbp_ets.cpp:5484-5485), or the given one
            double p0, p1, p2, p3;
            if (run.use_prior) {
                p0 = run.prior4[0]; p1 = run.prior4[1]; p2 = run.prior4[2]; p3 = run.prior4[3];
            } else {
                const double pt = trial_p(run.p, run.p_max, run.seed, run.trial[slot]);
                run.slot_p[slot] = pt;
                p0 = __dsub_rn(1.0, pt); p1 = __ddiv_rn(pt, 3.0); p2 = p1; p3 = p1;
                const double s = __dadd_rn(__dadd_rn(__dadd_rn(p0, p1), p2), p3);
                if (s <= 0.0) { p0 = p1 = p2 = p3 = 0.25; }
                else { p0 = __ddiv_rn(p0, s); p1 = __ddiv_rn(p1, s); p2 = __ddiv_rn(p2, s); p3 = __ddiv_rn(p3, s); }
            }
            if (precision == JBP_PREC_FP64) {
                double *pr = run.prior + 4 * slot;
                pr[0] = p0; pr[1] = p1; pr[2] = p2; pr[3] = p3;
            } else {
                // base-2 log prior and the prior LLRs (base 2) that seed fresh v2c messages
                float *lp = run.lprior + 8 * slot;
                for (int i = 0; i < 6; ++i) lp[i] = llr_prior_entry(i, p0, p1, p2, p3);
                lp[6] = lp[7] = 0.0f;
            }
            run.fresh[atomicAdd(run.n_fresh, 1)] = slot;
        } else {
            run.trial[slot] = -1;
            run.flags[slot] = 0;
        }
    }
}

// Errors of fresh trials: Philox, or copied from a device buffer of known errors.
static __global__ void k_sample(DevCode code, DevRun run) {
    const int nf = *run.n_fresh;
    const int n = code.n;
    const long long total = static_cast<long long>(nf) * n;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int f = static_cast<int>(i / n);
        const int v = static_cast<int>(i - static_cast<long long>(f) * n);
        const int slot = run.fresh[f];
        const long long t = run.trial[slot];
        uint8_t e = 0;
        if (run.source == kSrcPhilox) e = sample_philox(run.seed, t, v, run.slot_p[slot]);
        else if (run.source == kSrcErrors) {
            e = run.src_err[(t - run.first_trial) * n + v];
            if (e > 3) { atomicAdd(&run.cnt->bad_input, 1ull); e &= 3; }
        }
        run.err[static_cast<size_t>(slot) * n + v] = e;
    }
}

// The reference stream on the device: splitmix64 seed, mt19937_64 and libstdc++'s
// uniform_real_distribution<double> (one draw, x * 2^-64, clamped below 1), for one trial
// per warp; s is the warp's 312-word state.  The twist runs in two dependency-free halves:
// words 0..155 read only words of the previous block, words 156..311 read words 0..155 of
// this block.
static __device__ void warp_mt_trial(unsigned long long *s, unsigned long long base_seed, long long t, double p, int n,
                              uint8_t *out) {
    const int lane = threadIdx.x & 31;
    const unsigned long long seed =
        splitmix64(base_seed ^ (static_cast<unsigned long long>(t) * 0x9e3779b97f4a7c15ull));
    if (lane == 0) {
        s[0] = seed;
        for (int i = 1; i < 312; ++i) s[i] = 6364136223846793005ull * (s[i - 1] ^ (s[i - 1] >> 62)) + i;
    }
    __syncwarp();
    const unsigned long long hi = 0xFFFFFFFF80000000ull, lo = 0x7FFFFFFFull, A = 0xB5026F5AA96619E9ull;
    for (int base = 0; base < n; base += 312) {
        unsigned long long nv[5];
        for (int j = 0; j < 5; ++j) {
            const int k = lane + 32 * j;
            if (k < 156) {
                const unsigned long long y = (s[k] & hi) | (s[k + 1] & lo);
                nv[j] = s[k + 156] ^ (y >> 1) ^ ((y & 1) ? A : 0ull);
            }
        }
        __syncwarp();
        for (int j = 0; j < 5; ++j) {
            const int k = lane + 32 * j;
            if (k < 156) s[k] = nv[j];
        }
        __syncwarp();
        for (int j = 0; j < 5; ++j) {
            const int k = 156 + lane + 32 * j;
            if (k < 312) {
                const unsigned long long y = (s[k] & hi) | (s[(k + 1) % 312] & lo);
                nv[j] = s[k - 156] ^ (y >> 1) ^ ((y & 1) ? A : 0ull);
            }
        }
        __syncwarp();
        for (int j = 0; j < 5; ++j) {
            const int k = 156 + lane + 32 * j;
            if (k < 312) s[k] = nv[j];
        }
        __syncwarp();
        for (int k = lane; k < 312 && base + k < n; k += 32) {
            unsigned long long x = s[k];
            x ^= (x >> 29) & 0x5555555555555555ull;
            x ^= (x << 17) & 0x71D67FFFEDA60000ull;
            x ^= (x << 37) & 0xFFF7EEE000000000ull;
            x ^= x >> 43;
            double u = static_cast<double>(x) * 0x1.0p-64;
            if (u >= 1.0) u = 0x1.fffffffffffffp-1;
            out[base + k] = pauli_from_uniform(u, p);
        }
        __syncwarp();
    }
}

static __global__ void k_sample_mt(DevCode code, DevRun run) {
    __shared__ unsigned long long st[8][312];
    const int wib = threadIdx.x >> 5;
    const int nf = *run.n_fresh;
    for (int f = blockIdx.x * 8 + wib; f < nf; f += gridDim.x * 8) {
        const int slot = run.fresh[f];
        warp_mt_trial(st[wib], run.seed, run.trial[slot], run.slot_p[slot], code.n,
                      run.err + static_cast<size_t>(slot) * code.n);
    }
}

// Errors of trials first..first+count-1 written trial-major (jbp_sample_errors).
static __global__ void k_sample_out(int n, unsigned long long seed, long long first, long long count, double p, int sampler,
                             uint8_t *out) {
    __shared__ unsigned long long st[8][312];
    if (sampler == kSrcMt19937) {
        const int wib = threadIdx.x >> 5;
        for (long long t = blockIdx.x * 8LL + wib; t < count; t += gridDim.x * 8LL)
            warp_mt_trial(st[wib], seed, first + t, p, n, out + t * n);
    } else {
        const long long total = count * n;
        for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
             i += static_cast<long long>(gridDim.x) * blockDim.x) {
            const long long t = i / n;
            out[i] = sample_philox(seed, first + t, static_cast<int>(i - t * n), p);
        }
    }
}

// Syndromes of fresh trials, from their errors or copied from the source.
static __global__ void k_fresh_syndrome(DevCode code, DevRun run) {
    const int nf = *run.n_fresh;
    const int mx = code.s[0].m, M = mx + code.s[1].m;
    const int n = code.n, S = run.S;
    const long long total = static_cast<long long>(nf) * M;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int f = static_cast<int>(i / M);
        const int row = static_cast<int>(i - static_cast<long long>(f) * M);
        const int slot = run.fresh[f];
        const int side = row >= mx;
        const int ch = side ? row - mx : row;
        uint8_t bit;
        if (run.source == kSrcSyndromes) {
            const long long local = run.trial[slot] - run.first_trial;
            bit = side ? run.src_sz[local * code.s[1].m + ch] : run.src_sx[local * mx + ch];
            bit &= 1;
        } else {
            const int dc = side ? code.s[1].dc : code.s[0].dc;
            const int *chk_var = side ? code.s[1].chk_var : code.s[0].chk_var;
            const uint8_t *err = run.err + static_cast<size_t>(slot) * n;
            int par = 0;
            for (int k = 0; k < dc; ++k) {
                const int s = err[chk_var[ch * dc + k]];
                par ^= side ? zbit(s) : xbit(s);
            }
            bit = static_cast<uint8_t>(par);
        }
        unsigned *word = run.synm + static_cast<size_t>(row) * (S / kGroup) + slot / kGroup;
        const unsigned m = 1u << (slot % kGroup);
        if (bit) atomicOr(word, m);
        else atomicAnd(word, ~m);
    }
}

// The condition of the slot engine's device-side iteration loop (a CUDA graph while node whose
// body is one BP iteration): go on while trials are left, the iteration bound, which every
// run reaches only by an internal error, is not, and no abort is requested (jbp_request_abort's
// flag, a pinned host word).
static __global__ void k_loop_cond(cudaGraphConditionalHandle h, const DevCounters *cnt, const int *it,
                                   unsigned long long ntrials, int it_bound, const volatile int *abort_flag) {
    if (threadIdx.x == 0)
        cudaGraphSetConditional(h, (cnt->done < ntrials && *it < it_bound && !*abort_flag) ? 1u : 0u);
}

// Compacts the groups that still hold a running slot and advances the global iteration
// counter (the last kernel of an iteration).
static __global__ void k_groups(DevRun run) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *run.it += 1;
    const int g = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (g >= run.S / kGroup) return;
    const int lane = threadIdx.x & 31;
    const bool any = __any_sync(0xffffffffu, run.flags[g * kGroup + lane] & kRunning);
    if (any && lane == 0) run.groups[atomicAdd(run.n_groups, 1)] = g;
}

static __global__ void k_init_slots(DevRun run) {
    for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < run.S; s += gridDim.x * blockDim.x) {
        run.retired[s] = s;
        run.flags[s] = 0;
        run.trial[s] = -1;
        run.iter[s] = 0;
        run.unsat[s] = 0;
        run.unsat[run.S + s] = 0;
        if (s < 2 * (run.S / kGroup)) run.unsat_mask[s] = 0u;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *run.n_retired = run.S;
}

}  // namespace jbp
