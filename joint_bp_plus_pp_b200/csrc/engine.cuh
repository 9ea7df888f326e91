// Batched joint X/Z BP engine for sm_100a: shared declarations.
//
// Trials live in "slots", grouped by 32 (one warp per group); only groups with a running
// slot are scheduled.  Message layout: see kernels_bp.cuh.  Each BP iteration is a fixed
// sequence of kernels captured in a CUDA graph; converged or exhausted trials are retired,
// post-processed, classified and replaced by fresh trials on the device, so the host only
// watches a completion counter.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "../../include/jbp_b200.h"

namespace jbp {

constexpr int kGroup = 32;          // slots per warp
constexpr int kMaxDc = 16;          // largest check degree the kernels are built for
constexpr int kMaxDv = 8;           // largest per-side variable degree

enum SlotFlag : int {
    kRunning = 1,
    kFinished = 2,                  // retired this iteration, awaiting classification
};

enum SourceKind : int {
    kSrcPhilox = 0,
    kSrcMt19937 = 1,
    kSrcErrors = 2,                 // device buffer of errors, trial-major
    kSrcSyndromes = 3,              // device buffers of syndromes, trial-major
};

struct DevSide {
    int m, edges, dc, dv;
    const int *chk_var;             // [edges], edge = c * dc + position
    const int *var_edge;            // [n * dv], ascending check; -1 pads variables of lower degree
};

struct DevCode {
    int n;
    DevSide s[2];
    int words;                      // 64-bit words of an n-bit vector
    const uint64_t *basis_rows[2];  // row space of Hx (0) / Hz (1)
    const int *pivot_row[2];        // [n] basis row with that pivot column, or -1
};

// All loaded ETS tables, flattened (group order = reference load order).
constexpr int kMaxEtsGroups = 16;
struct DevEts {
    int ngroups;
    int size[kMaxEtsGroups];                 // variables per entry
    int first[kMaxEtsGroups][2];             // first entry of (group, side)
    int count[kMaxEtsGroups][2];             // entries of (group, side), 0 when not loaded
    const unsigned long long *key;           // per entry: (c0 << 32) | c1
    const int *vars;                         // per entry: size sorted variables at var_first
    const int *var_first;
};

// Result bits of a trial (res_flags), shared by retirement, post-processing and
// classification.
enum ResultBit : int {
    kResSyndromeOk = 1 << 0,
    kResBpOk = 1 << 1,
    kResPpInDecode = 1 << 2,     // in-loop post-processing succeeded
    kResPpInEts = 1 << 3,
    kResPpInFlip = 1 << 4,
    kResUsedAny = 1 << 5,        // an ETS correction was applied (the reference's used_any)
    kResUsed6 = 1 << 6,
    kResUsed12 = 1 << 7,
    kResEtsPost = 1 << 8,        // post-BP ETS applied
    kResEtsOk = 1 << 9,          // ets_pp_ok of the simulate loop
    kResFlipOk = 1 << 10,
    kResOsdOk = 1 << 11,
    kResPostEntered = 1 << 12,   // post-BP stages ran
    kResLearned = 1 << 13,       // a learned flip proposal produced the final estimate
};

// Post-processing request kinds (pp_mode).
enum PpMode : int { kPpInLoop = 1, kPpPost = 2 };

struct DevCounters {
    unsigned long long next_trial;  // trials handed to slots
    unsigned long long done;        // trials classified
    unsigned long long failures, bp_fail, stab_success, exact, total_iters, syndrome_ok;
    unsigned long long pp_success, flip_pp_success, osd_pp_success;
    unsigned long long ets_used, ets_saved, ets6_used, ets6_saved, ets12_used, ets12_saved;
    unsigned long long bp_trial_iterations;
    unsigned long long watchdog;
    unsigned long long bad_input;   // error bytes outside 0..3 seen in a kSrcErrors source
    unsigned long long learned_attempts, learned_success;   // learned flip proposals tried / saves
    unsigned long long syndrome_tests;   // slot engine: per-trial syndrome tests run
    unsigned long long aborted;          // blocks (persistent kernels) that stopped on the abort flag
};

struct DevRun {
    // configuration
    int S;                          // slots
    int max_iter, check_warmup, check_interval;
    int source;
    double p, p_max;                // p_max > p: per-trial p uniform in [p, p_max) (trial_p)
    unsigned long long seed;
    long long first_trial, ntrials;
    const uint8_t *src_err;         // [ntrials][n]
    const uint8_t *src_sx, *src_sz; // [ntrials][m]
    uint8_t *est_out;               // [ntrials][n] or null
    float *llr_out;                 // [ntrials][n][2] final LLRs (x, z) or null
    jbp_trial_result *res_out;      // [ntrials] or null
    unsigned long long *hist;       // [max_iter + 1] or null
    // slot state
    long long *trial;               // [S]
    int *iter;                      // [S] completed iterations
    int *flags;                     // [S]
    int *unsat;                     // [2][S] unsatisfied-check counts (kept when PP needs them)
    unsigned *unsat_mask;           // [2][G] slots of a group with an unsatisfied check, per side
    double *prior;                  // [S][4] normalized prior (FP64 path)
    double *slot_p;                 // [S] error rate of the slot's trial
    float *lprior;                  // [S][8] log prior x4, prior LLR x/z (FP32 path)
    uint8_t *err;                   // [S][n] true error of the slot's trial
    // Hard decisions as bit planes: bit (slot % 32) of plane[g * n + v] is the x-bit (estx)
    // or z-bit (estz) of variable v in slot g * 32 + slot % 32.  One 32-slot word per
    // variable makes the syndrome test an XOR of words and keeps a group's decisions in one
    // contiguous row.  The planes form a ring of R iterations ([R][G][n]); the planes of the
    // current global iteration are (*it % R).  A running slot advances one iteration per
    // global iteration, so its decisions d iterations back are in plane (*it - d) % R.
    unsigned *estx, *estz;
    int R;
    int *it;                        // global BP iteration counter
    unsigned *synm;                 // [(mx+mz)][G] target syndrome bits, same slot bit order
    // freeze-syn (jointbp_ets.cpp:1884-1901, 2526-2535): once a side's syndrome matches at a
    // check, its messages become deterministic copies of the decisions and stop updating.
    int freeze_syn;
    int *frz;                       // [S] bit0/1 X/Z frozen, bit2/3 X/Z frozen at the last check
    // explicit prior (the jointbp_cuda.h interface passes it instead of p)
    int use_prior;
    double prior4[4];
    int *res_iters;                 // [S] iterations at retirement
    int *res_flags;                 // [S] ResultBit flags
    // work lists
    int *retired, *n_retired;
    int *fresh, *n_fresh;
    int *groups, *n_groups;
    DevCounters *cnt;
    // post-processing (enabled when pp != 0)
    int pp;
    int flip_hist;                  // flip-history window H (R >= H + 1)
    int llr_from;                   // first 1-based iteration of the stall triggers: min(100, max_iter)
    int *act_k;                     // [S] iteration the flip window started (0: not started)
    int *pstate;                    // [S] bit0 stall, bit1 oscillation, bit2 us-oscillation active
    int *stall_same;                // [S]
    unsigned short *us_hist;        // [S][100] max(us_x, us_z) by iteration (mod 100)
    unsigned *dprev, *dpprev;       // [G] slots whose decisions differ from 1 / 2 iterations back
    int *pp_list, *n_pp;            // slots to post-process this iteration
    int *pp_mode;                   // [S] PpMode
    DevEts ets;
    unsigned char *pp_scratch;      // per post-processing block
    size_t pp_scratch_stride;
};

__device__ __forceinline__ size_t plane_offset(const DevRun &run, int n, int back) {
    const int r = ((*run.it - back) % run.R + run.R) % run.R;
    return static_cast<size_t>(r) * (run.S / 32) * n;
}

// Messages of one run.  FP64: c2v as (a, b) pairs, v2c as (q0, q1) pairs, or the full
// 4-vector (two pairs) when damping is on.  FP32/FP16: one LLR per edge and direction.
struct DevMsgs {
    void *c2v[2];
    void *v2c[2];
    void *v2c_hi[2];                // FP64 with damping: (m2, m3) half of the v2c 4-vector
};

// splitmix64 finaliser of the reference per-trial seed (jointbp_ets.cpp:4401-4411).
__host__ __device__ __forceinline__ unsigned long long splitmix64(unsigned long long x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

}  // namespace jbp
