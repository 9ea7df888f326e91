// Batched joint X/Z BP engine for sm_100a: shared declarations.
//
// Trials live in "slots".  All per-edge state is stored edge-major and slot-minor,
// msg[edge * S + slot], so a warp that handles one check (or one variable) for 32
// consecutive slots makes one contiguous access per edge.  Slots are grouped by 32
// (one warp); only groups with a running slot are scheduled.  Each BP iteration is a
// fixed sequence of kernels captured in a CUDA graph; converged or exhausted trials are
// retired, classified and replaced by fresh trials on the device, so the host only
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
    const int *var_edge;            // [n * dv], ascending check
};

struct DevCode {
    int n;
    DevSide s[2];
    int words;                      // 64-bit words of an n-bit vector
    const uint64_t *basis_rows[2];  // row space of Hx (0) / Hz (1)
    const int *pivot_row[2];        // [n] basis row with that pivot column, or -1
};

struct DevCounters {
    unsigned long long next_trial;  // trials handed to slots
    unsigned long long done;        // trials classified
    unsigned long long failures, bp_fail, stab_success, exact, total_iters, syndrome_ok;
    unsigned long long pp_success, flip_pp_success, osd_pp_success;
    unsigned long long ets_used, ets_saved, ets6_used, ets6_saved, ets12_used, ets12_saved;
    unsigned long long bp_trial_iterations;
    unsigned long long watchdog;
};

struct DevRun {
    // configuration
    int S;                          // slots
    int max_iter, check_warmup, check_interval;
    int source;
    double p;
    unsigned long long seed;
    long long first_trial, ntrials;
    const uint8_t *src_err;         // [ntrials][n]
    const uint8_t *src_sx, *src_sz; // [ntrials][m]
    uint8_t *est_out;               // [ntrials][n] or null
    jbp_trial_result *res_out;      // [ntrials] or null
    unsigned long long *hist;       // [max_iter + 1] or null
    // slot state
    long long *trial;               // [S]
    int *iter;                      // [S] completed iterations
    int *flags;                     // [S]
    int *unsat;                     // [2][S] unsatisfied-check counts (kept when PP needs them)
    unsigned *unsat_mask;           // [2][G] slots of a group with an unsatisfied check, per side
    double *prior;                  // [S][4] normalized prior (FP64 path)
    float *lprior;                  // [S][8] log prior x4, prior LLR x/z (FP32 path)
    uint8_t *err;                   // [S][n] true error of the slot's trial
    // Hard decisions as bit planes: bit (slot % 32) of estx[g * n + v] is the x-bit of
    // variable v in slot g * 32 + slot % 32 (estz: the z-bit).  One 32-slot word per
    // variable makes the syndrome test an XOR of words and keeps a group's decisions in
    // one contiguous row.
    unsigned *estx, *estz;          // [G][n]
    unsigned *synm;                 // [(mx+mz)][G] target syndrome bits, same slot bit order
    int *res_iters;                 // [S] iterations at retirement
    int *res_flags;                 // [S] bit0 syndrome_ok, bit1 bp_ok
    // work lists
    int *retired, *n_retired;
    int *fresh, *n_fresh;
    int *groups, *n_groups;
    DevCounters *cnt;
};

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
