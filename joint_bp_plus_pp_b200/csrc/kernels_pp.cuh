// Post-processing on the GPU: ETS, flip and OSD stages for stalled or exhausted trials.
//
// One thread block takes one pending slot (a grid-stride loop over the pending list).  The
// trial's decisions, target syndromes and scratch flags live in shared memory; GF(2)
// matrices, the OSD ordering and its basis in a per-block global scratch area.  The stages
// and their acceptance rules follow the reference (jointbp_ets.cpp):
//   ETS   attempt_ets_fix_side[_multi]  3525-3668   (exactly two unsatisfied checks, table
//         entries keyed by the pair, local GF(2) solve, accept when the side syndrome matches)
//   flip  build_flip_sets / attempt_flip_pp_side  3670-3880  (candidate sets from the flip
//         window; accept only a unique solution that reproduces the syndrome)
//   OSD   attempt_osd_pp_side  4078-4386  (columns ordered by |LLR| then index; smallest
//         solvable K and largest unique K; accept weight <= 30)
// and the driver order of the in-loop and post-BP sequences (2736-3074, 6020-6197).
//
// The GF(2) answers do not depend on how the elimination is organised: the reduced echelon
// form of a system is unique, so the accepted corrections are the reference's.  Two
// reformulations make the stages cheap on a block:
//  * a candidate's acceptance "side syndrome matches after applying the solution" is
//    equivalent to "the local system is solvable and every unsatisfied check is covered",
//    because the solution satisfies each covered check and leaves the others unchanged;
//  * the OSD predicates solvable(K) and unique(K) are monotone in K (column spans only
//    grow), so the reference's two binary searches return the first K at which the syndrome
//    difference enters the span of the first K ordered columns and the last K before the
//    first dependent column.  One incremental elimination over the ordered columns
//    (reduced basis with the combination of original columns kept per basis vector)
//    yields both and the unique solution.
#pragma once

#include "engine.cuh"

namespace jbp {

constexpr int kPpThreads = 512;

struct PpShared {
    uint8_t *est;      // [n] trial estimate (0..3)
    uint8_t *tgt;      // [mx + mz] target syndrome bits
    uint8_t *diff;     // [max m] side syndrome difference
    uint8_t *mark;     // [n] candidate-set membership
    uint8_t *touch;    // [max m]
    int *ints;         // [64] block scalars
    uint64_t *wv;      // [MW] OSD vector being inserted
    uint64_t *wc;      // [CW] its column combination
};

struct PpScratch {
    uint64_t *rows;    // flip: [max m][words(n)]
    int *rhs;          // [max m]
    int *list;         // [n] candidate variables, ascending
    int *pos;          // [n] position of a variable in list, or -1
    int *tlist;        // [max m] covered checks
    unsigned long long *key;  // OSD: [npow2]
    int *idx;          // [npow2]
    uint64_t *vec;     // [max m][MW]
    uint64_t *comb;    // [max m][CW]
    int *piv;          // [max m] basis vector whose pivot is that row, or -1
    uint64_t *rvec;    // [MW]
    uint64_t *rcomb;   // [CW]
    uint64_t *delta;   // [CW]
};

__host__ __device__ inline int pp_npow2(int n) {
    int p = 1;
    while (p < n) p <<= 1;
    return p;
}

__host__ __device__ inline size_t pp_align(size_t b) { return (b + 255) / 256 * 256; }

// Bytes of per-block global scratch for a code (n variables, at most mmax checks per side).
__host__ __device__ inline size_t pp_scratch_bytes(int n, int mmax) {
    const int words = (n + 63) / 64, MW = (mmax + 63) / 64, CW = (mmax + 2 + 63) / 64, np2 = pp_npow2(n);
    return pp_align(sizeof(uint64_t) * static_cast<size_t>(mmax) * words) + pp_align(sizeof(int) * mmax) +
           2 * pp_align(sizeof(int) * n) + pp_align(sizeof(int) * mmax) + pp_align(8ull * np2) +
           pp_align(4ull * np2) + pp_align(8ull * mmax * MW) + pp_align(8ull * mmax * CW) + pp_align(4ull * mmax) +
           pp_align(8ull * MW) + 2 * pp_align(8ull * CW);
}

static __device__ inline PpScratch pp_scratch_carve(unsigned char *base, int n, int mmax) {
    const int words = (n + 63) / 64, MW = (mmax + 63) / 64, CW = (mmax + 2 + 63) / 64, np2 = pp_npow2(n);
    PpScratch s;
    size_t o = 0;
    s.rows = reinterpret_cast<uint64_t *>(base + o); o += pp_align(sizeof(uint64_t) * static_cast<size_t>(mmax) * words);
    s.rhs = reinterpret_cast<int *>(base + o); o += pp_align(sizeof(int) * mmax);
    s.list = reinterpret_cast<int *>(base + o); o += pp_align(sizeof(int) * n);
    s.pos = reinterpret_cast<int *>(base + o); o += pp_align(sizeof(int) * n);
    s.tlist = reinterpret_cast<int *>(base + o); o += pp_align(sizeof(int) * mmax);
    s.key = reinterpret_cast<unsigned long long *>(base + o); o += pp_align(8ull * np2);
    s.idx = reinterpret_cast<int *>(base + o); o += pp_align(4ull * np2);
    s.vec = reinterpret_cast<uint64_t *>(base + o); o += pp_align(8ull * mmax * MW);
    s.comb = reinterpret_cast<uint64_t *>(base + o); o += pp_align(8ull * mmax * CW);
    s.piv = reinterpret_cast<int *>(base + o); o += pp_align(4ull * mmax);
    s.rvec = reinterpret_cast<uint64_t *>(base + o); o += pp_align(8ull * MW);
    s.rcomb = reinterpret_cast<uint64_t *>(base + o); o += pp_align(8ull * CW);
    s.delta = reinterpret_cast<uint64_t *>(base + o);
    return s;
}

// Shared-memory bytes of the post-processing kernel.
__host__ __device__ inline size_t pp_smem_bytes(int n, int M, int mmax) {
    const int MW = (mmax + 63) / 64, CW = (mmax + 2 + 63) / 64;
    return pp_align(n) * 2 + pp_align(M) + pp_align(mmax) * 2 + pp_align(64 * 4) + pp_align(8ull * MW) +
           pp_align(8ull * CW);
}

// Carves the post-processing shared arrays from `base` (pp_smem_bytes(n, M, mmax) bytes).
__device__ __forceinline__ PpShared pp_shared_carve(unsigned char *base, int n, int M, int mmax) {
    const int MW = (mmax + 63) / 64;
    PpShared sh;
    size_t o = 0;
    sh.est = base + o; o += pp_align(n);
    sh.mark = base + o; o += pp_align(n);
    sh.tgt = base + o; o += pp_align(M);
    sh.diff = base + o; o += pp_align(mmax);
    sh.touch = base + o; o += pp_align(mmax);
    sh.ints = reinterpret_cast<int *>(base + o); o += pp_align(64 * 4);
    sh.wv = reinterpret_cast<uint64_t *>(base + o); o += pp_align(8ull * MW);
    sh.wc = reinterpret_cast<uint64_t *>(base + o);
    return sh;
}

__device__ __forceinline__ int side_bit(int state, int side) { return (state >> side) & 1; }

// Check (row of `side`) of a variable's k-th edge on that side, or -1 past its degree.
__device__ __forceinline__ int var_check(const DevCode &code, int side, int v, int k) {
    const DevSide &g = code.s[side];
    const int e = __ldg(g.var_edge + v * g.dv + k);
    return e >= 0 ? e / g.dc : -1;
}

// diff = side syndrome of est xor target; returns the number of unsatisfied checks and
// stores the first two of them (ascending) in ints[8], ints[9].
static __device__ int blk_side_diff(const DevCode &code, const PpShared &sh, int side) {
    const int m = code.s[side].m, dc = code.s[side].dc, mx = code.s[0].m;
    const int *chk_var = code.s[side].chk_var;
    if (threadIdx.x == 0) { sh.ints[7] = 0; sh.ints[8] = 0x7fffffff; sh.ints[9] = 0x7fffffff; }
    __syncthreads();
    int local = 0;
    for (int c = threadIdx.x; c < m; c += blockDim.x) {
        int par = 0;
        for (int i = 0; i < dc; ++i) par ^= side_bit(sh.est[__ldg(chk_var + c * dc + i)], side);
        const uint8_t d = static_cast<uint8_t>(par ^ sh.tgt[side ? mx + c : c]);
        sh.diff[c] = d;
        if (d) {
            local++;
            // keep the two smallest unsatisfied rows
            int cur = c;
            const int old = atomicMin(&sh.ints[8], cur);
            cur = old > cur ? old : cur;
            if (cur != 0x7fffffff) atomicMin(&sh.ints[9], cur);
        }
    }
    if (local) atomicAdd(&sh.ints[7], local);
    __syncthreads();
    const int cnt = sh.ints[7];
    __syncthreads();
    return cnt;
}

// ------------------------------------------------------------------ ETS

// Gauss-Jordan over <= 32 columns with free variables 0 (solve_gf2, jointbp_ets.cpp:3357).
static __device__ bool gf2_solve32(uint32_t *a, uint8_t *b, int m, int nv, uint32_t *sol) {
    int where[32];
    for (int c = 0; c < nv; ++c) where[c] = -1;
    int r = 0;
    for (int c = 0; c < nv && r < m; ++c) {
        int sel = r;
        while (sel < m && !((a[sel] >> c) & 1u)) ++sel;
        if (sel == m) continue;
        const uint32_t ta = a[sel]; a[sel] = a[r]; a[r] = ta;
        const uint8_t tb = b[sel]; b[sel] = b[r]; b[r] = tb;
        where[c] = r;
        for (int i = 0; i < m; ++i)
            if (i != r && ((a[i] >> c) & 1u)) { a[i] ^= a[r]; b[i] ^= b[r]; }
        ++r;
    }
    for (int i = r; i < m; ++i)
        if (a[i] == 0 && b[i]) return false;
    uint32_t s = 0;
    for (int c = 0; c < nv; ++c)
        if (where[c] >= 0 && b[where[c]]) s |= 1u << c;
    *sol = s;
    return true;
}

// One ETS table of one side (attempt_ets_fix_side).  diff / ints[7..9] hold the side's
// syndrome difference.  Serial in thread 0: a few dozen entries of <= 32 variables.
static __device__ bool blk_ets_table(const DevCode &code, const DevEts &ets, const PpShared &sh, int side, int g) {
    if (threadIdx.x == 0) {
        sh.ints[10] = 0;
        const int c0 = sh.ints[8], c1 = sh.ints[9];
        const unsigned long long key = (static_cast<unsigned long long>(static_cast<unsigned>(c0)) << 32) |
                                       static_cast<unsigned>(c1);
        const int nv = ets.size[g];
        const int first = ets.first[g][side], count = ets.count[g][side];
        const int dv = code.s[side].dv, dc = code.s[side].dc;
        const int *chk_var = code.s[side].chk_var;
        int checks[32 * kMaxDv];
        uint32_t rows[32 * kMaxDv];
        uint8_t rhs[32 * kMaxDv];
        for (int e = first; e < first + count && nv > 0 && nv <= 32; ++e) {
            if (ets.key[e] != key) continue;
            const int *vars = ets.vars + ets.var_first[e];
            int nch = 0;
            for (int i = 0; i < nv; ++i)
                for (int k = 0; k < dv; ++k) {
                    const int c = var_check(code, side, vars[i], k);
                    if (c < 0) continue;
                    bool seen = false;
                    for (int j = 0; j < nch; ++j) seen |= checks[j] == c;
                    if (!seen) checks[nch++] = c;
                }
            bool ok = true, has0 = false, has1 = false;
            for (int j = 0; j < nch; ++j) {
                const int c = checks[j];
                has0 |= c == c0;
                has1 |= c == c1;
                if (sh.diff[c] && c != c0 && c != c1) ok = false;
            }
            if (!ok) continue;
            int nr = 0;
            for (int j = 0; j < nch; ++j) {
                const int c = checks[j];
                uint32_t mask = 0;
                for (int t = 0; t < dc; ++t) {
                    const int v = __ldg(chk_var + c * dc + t);
                    for (int i = 0; i < nv; ++i)
                        if (vars[i] == v) { mask |= 1u << i; break; }
                }
                if (!mask) continue;
                rows[nr] = mask;
                rhs[nr++] = sh.diff[c];
            }
            uint32_t sol = 0;
            if (!gf2_solve32(rows, rhs, nr, nv, &sol)) continue;
            // the corrected side syndrome matches iff both unsatisfied checks are covered
            if (!(has0 && has1)) continue;
            for (int i = 0; i < nv; ++i)
                if ((sol >> i) & 1u) sh.est[vars[i]] ^= static_cast<uint8_t>(1 << side);
            sh.ints[10] = 1;
            break;
        }
    }
    __syncthreads();
    const bool applied = sh.ints[10];
    __syncthreads();
    return applied;
}

// attempt_ets_fix_side_multi: the first group whose table applies; returns its index or -1.
static __device__ int blk_ets_multi(const DevCode &code, const DevEts &ets, const PpShared &sh, int side) {
    bool any = false;
    for (int g = 0; g < ets.ngroups; ++g) any |= ets.count[g][side] > 0;
    if (!any) return -1;
    if (blk_side_diff(code, sh, side) != 2) return -1;
    for (int g = 0; g < ets.ngroups; ++g) {
        if (ets.count[g][side] == 0) continue;
        if (blk_ets_table(code, ets, sh, side, g)) return g;
    }
    return -1;
}

// ------------------------------------------------------------------ flip

// Block exclusive scan of per-thread counts; returns this thread's offset, total in ints[20].
static __device__ int blk_scan(const PpShared &sh, int cnt) {
    __shared__ int part[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int incl = cnt;
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += y;
    }
    if (lane == 31) part[w] = incl;
    __syncthreads();
    if (threadIdx.x == 0) {
        int s = 0;
        for (int i = 0; i < static_cast<int>(blockDim.x >> 5); ++i) { const int t = part[i]; part[i] = s; s += t; }
        sh.ints[20] = s;
    }
    __syncthreads();
    const int off = part[w] + incl - cnt;
    __syncthreads();
    return off;
}

// attempt_flip_pp_side on the variables marked in sh.mark: applies and returns true only for
// a unique solution that reproduces the side syndrome.
static __device__ bool blk_flip_attempt(const DevCode &code, const PpShared &sh, const PpScratch &sc, int side) {
    const int n = code.n, m = code.s[side].m, dc = code.s[side].dc, dv = code.s[side].dv;
    const int *chk_var = code.s[side].chk_var;
    // ascending variable list and positions
    const int per = (n + blockDim.x - 1) / blockDim.x;
    const int v0 = threadIdx.x * per, v1 = min(n, v0 + per);
    int cnt = 0;
    for (int v = v0; v < v1; ++v) cnt += sh.mark[v] != 0;
    int off = blk_scan(sh, cnt);
    const int nv = sh.ints[20];
    for (int v = v0; v < v1; ++v) {
        if (sh.mark[v]) { sc.list[off] = v; sc.pos[v] = off++; }
        else sc.pos[v] = -1;
    }
    for (int c = threadIdx.x; c < m; c += blockDim.x) sh.touch[c] = 0;
    __syncthreads();
    if (nv == 0) return false;
    for (int i = threadIdx.x; i < nv; i += blockDim.x)
        for (int k = 0; k < dv; ++k) {
            const int c = var_check(code, side, sc.list[i], k);
            if (c >= 0) sh.touch[c] = 1;
        }
    __syncthreads();
    // every unsatisfied check must be covered; covered checks become rows
    const int cper = (m + blockDim.x - 1) / blockDim.x;
    const int c0 = threadIdx.x * cper, c1 = min(m, c0 + cper);
    int tc = 0;
    bool uncovered = false;
    for (int c = c0; c < c1; ++c) {
        tc += sh.touch[c];
        uncovered |= sh.diff[c] && !sh.touch[c];
    }
    const bool bad = __syncthreads_or(uncovered);
    int toff = blk_scan(sh, tc);
    const int nr = sh.ints[20];
    if (bad || nv > nr) return false;   // unsolvable, or more columns than rows (not unique)
    const int words = (nv + 63) / 64;
    for (int c = c0; c < c1; ++c) {
        if (!sh.touch[c]) continue;
        const int r = toff++;
        sc.tlist[r] = c;
        sc.rhs[r] = sh.diff[c];
        uint64_t *row = sc.rows + static_cast<size_t>(r) * words;
        for (int w = 0; w < words; ++w) row[w] = 0;
        for (int t = 0; t < dc; ++t) {
            const int p = sc.pos[__ldg(chk_var + c * dc + t)];
            if (p >= 0) row[p >> 6] |= 1ull << (p & 63);
        }
    }
    __syncthreads();
    // Gauss-Jordan; a column without pivot means the solution is not unique
    for (int col = 0; col < nv; ++col) {
        const int w = col >> 6;
        const uint64_t bit = 1ull << (col & 63);
        if (threadIdx.x == 0) sh.ints[21] = 0x7fffffff;
        __syncthreads();
        int best = 0x7fffffff;
        for (int r = col + threadIdx.x; r < nr; r += blockDim.x)
            if (sc.rows[static_cast<size_t>(r) * words + w] & bit) { best = r; break; }
        if (best != 0x7fffffff) atomicMin(&sh.ints[21], best);
        __syncthreads();
        const int piv = sh.ints[21];
        if (piv == 0x7fffffff) return false;
        if (piv != col) {
            for (int k = w + threadIdx.x; k < words; k += blockDim.x) {
                uint64_t *a = sc.rows + static_cast<size_t>(piv) * words, *b = sc.rows + static_cast<size_t>(col) * words;
                const uint64_t t = a[k]; a[k] = b[k]; b[k] = t;
            }
            if (threadIdx.x == 0) { const int t = sc.rhs[piv]; sc.rhs[piv] = sc.rhs[col]; sc.rhs[col] = t; }
        }
        __syncthreads();
        const uint64_t *prow = sc.rows + static_cast<size_t>(col) * words;
        const int prhs = sc.rhs[col];
        for (int r = threadIdx.x; r < nr; r += blockDim.x) {
            if (r == col) continue;
            uint64_t *row = sc.rows + static_cast<size_t>(r) * words;
            if (!(row[w] & bit)) continue;
            for (int k = w; k < words; ++k) row[k] ^= prow[k];
            sc.rhs[r] ^= prhs;
        }
        __syncthreads();
    }
    // rows beyond nv are zero: a 1 on their right-hand side means no solution
    bool inconsistent = false;
    for (int r = nv + threadIdx.x; r < nr; r += blockDim.x) inconsistent |= sc.rhs[r] != 0;
    if (__syncthreads_or(inconsistent)) return false;
    for (int i = threadIdx.x; i < nv; i += blockDim.x)
        if (sc.rhs[i]) sh.est[sc.list[i]] ^= static_cast<uint8_t>(1 << side);
    __syncthreads();
    return true;
}

// Decision history of one trial for the flip window: bit `side` of the trial's decision of
// variable v flipped between iterations j - 1 and j.
// Slot engine: the ring of 32-slot bit planes (the trial's bit in each word).
struct SlotHistory {
    const DevRun *run;
    int slot, k;   // k = the trial's current iteration (planes are indexed relative to it)
    __device__ unsigned flip(int side, int j, int v, int n) const {
        const size_t pa = plane_offset(*run, n, k - j), pb = plane_offset(*run, n, k - j + 1);
        const unsigned *planes = side ? run->estz : run->estx;
        const size_t row = static_cast<size_t>(slot / kGroup) * n;
        return ((planes[pa + row + v] ^ planes[pb + row + v]) >> (slot % kGroup)) & 1u;
    }
};
// Trial-resident engine: a ring of R per-iteration decision arrays (bytes 0..3).
struct RingHistory {
    const uint8_t *ring;
    int R;
    __device__ unsigned flip(int side, int j, int v, int n) const {
        const uint8_t a = ring[static_cast<size_t>(j % R) * n + v], b = ring[static_cast<size_t>((j - 1) % R) * n + v];
        return ((a ^ b) >> side) & 1u;
    }
};

// Marks the flips of `side` between iterations j - 1 and j.
template <class Hist>
static __device__ void blk_mark_flips(const DevCode &code, const Hist &hist, const PpShared &sh, int side, int j,
                                      bool accumulate) {
    const int n = code.n;
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        const uint8_t f = static_cast<uint8_t>(hist.flip(side, j, v, n));
        sh.mark[v] = accumulate ? static_cast<uint8_t>(sh.mark[v] | f) : f;
    }
    __syncthreads();
}

static __device__ bool blk_any_mark(const DevCode &code, const PpShared &sh) {
    bool any = false;
    for (int v = threadIdx.x; v < code.n; v += blockDim.x) any |= sh.mark[v] != 0;
    return __syncthreads_or(any);
}

// build_flip_sets + the first set that applies (union, then the window newest to oldest,
// or the last flips when there is neither window nor union).  k = current iteration,
// act = iteration the flip window started (0: none).
template <class Hist>
static __device__ bool blk_flip_side(const DevCode &code, const Hist &hist, int flip_hist, int act,
                                     const PpShared &sh, const PpScratch &sc, int side, int k) {
    blk_side_diff(code, sh, side);
    const bool window = act > 0 && flip_hist > 0;
    int jlo = 0, wlen = 0;
    if (window) {
        jlo = max(max(act, 2), k - flip_hist + 1);
        wlen = k >= jlo ? k - jlo + 1 : 0;
    }
    bool have_union = false;
    if (window) {
        for (int v = threadIdx.x; v < code.n; v += blockDim.x) sh.mark[v] = 0;
        __syncthreads();
        for (int j = jlo; j <= k; ++j) blk_mark_flips(code, hist, sh, side, j, true);
        have_union = blk_any_mark(code, sh);
        if (have_union && blk_flip_attempt(code, sh, sc, side)) return true;
    }
    if (wlen > 0) {
        for (int j = k; j >= jlo; --j) {
            blk_mark_flips(code, hist, sh, side, j, false);
            if (!blk_any_mark(code, sh)) continue;
            if (blk_flip_attempt(code, sh, sc, side)) return true;
        }
    } else if (!have_union && k >= 2) {
        blk_mark_flips(code, hist, sh, side, k, false);
        if (blk_any_mark(code, sh) && blk_flip_attempt(code, sh, sc, side)) return true;
    }
    return false;
}

// ------------------------------------------------------------------ OSD

// Ascending sort of (key, index) pairs in global scratch (bitonic network, np2 entries).
static __device__ void blk_sort_pairs(unsigned long long *key, int *idx, int np2) {
    for (int size = 2; size <= np2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j <= i) continue;
                const bool asc = (i & size) == 0;
                const unsigned long long ki = key[i], kj = key[j];
                const int ii = idx[i], ij = idx[j];
                const bool gt = ki > kj || (ki == kj && ii > ij);
                if (gt == asc) {
                    key[i] = kj; key[j] = ki;
                    idx[i] = ij; idx[j] = ii;
                }
            }
            __syncthreads();
        }
    }
}

// attempt_osd_pp_side restated as one incremental elimination (see the file comment).
// The basis is kept fully reduced (no basis vector has a bit at another one's pivot), so a new
// column is reduced by the basis vectors pivoted at its own checks alone.  Per column, warp 0
// builds the reduced column and its lowest set bit; after one barrier every warp clears the
// new pivot from its share of the basis, testing 32 basis vectors per load and ballot; warp 0
// appends the column and updates the residual of the syndrome difference; a second barrier
// ends the column.  `max_cols` limits the columns taken (the whole order by default).
static __device__ bool blk_osd_side(const DevCode &code, const double *llr, const PpShared &sh, const PpScratch &sc,
                                    int side, int max_cols = 0x7fffffff) {
    const int n = code.n, m = code.s[side].m, dv = code.s[side].dv;
    const int MW = (m + 63) / 64, CW = (m + 2 + 63) / 64;
    const int np2 = pp_npow2(n);
    const int cnt = blk_side_diff(code, sh, side);
    if (cnt == 0) return false;  // "skipped (no syndrome diff)"
    for (int i = threadIdx.x; i < np2; i += blockDim.x) {
        sc.key[i] = i < n ? static_cast<unsigned long long>(__double_as_longlong(llr[i])) : ~0ull;
        sc.idx[i] = i < n ? i : 0x7fffffff;
    }
    for (int w = threadIdx.x; w < MW; w += blockDim.x) {
        uint64_t x = 0;
        for (int b = 0; b < 64 && w * 64 + b < m; ++b) x |= static_cast<uint64_t>(sh.diff[w * 64 + b] & 1) << b;
        sc.rvec[w] = x;
    }
    for (int w = threadIdx.x; w < CW; w += blockDim.x) { sc.rcomb[w] = 0; sc.delta[w] = 0; }
    for (int r = threadIdx.x; r < m; r += blockDim.x) sc.piv[r] = -1;
    if (threadIdx.x == 0) { sh.ints[30] = 0; sh.ints[31] = -1; }  // rank, K_s
    __syncthreads();
    blk_sort_pairs(sc.key, sc.idx, np2);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int ncols = min(n, max_cols);
    for (int j = 0; j < ncols; ++j) {
        const int rank = sh.ints[30];
        if (warp == 0) {
            // the column: the variable's checks, reduced by the basis vectors pivoted there.
            // Lane k fetches check k and its pivot; the basis words are gathered in registers,
            // 4 words per lane per pass, so the loads of the different checks overlap.
            const int var = sc.idx[j];
            for (int w0 = 0; w0 < MW || w0 < CW; w0 += 128) {
                uint64_t av[4] = {0ull, 0ull, 0ull, 0ull}, ac[4] = {0ull, 0ull, 0ull, 0ull};
                for (int k0 = 0; k0 < dv; k0 += 32) {
                    int ck = -1, bk = -1;
                    if (k0 + lane < dv) {
                        ck = var_check(code, side, var, k0 + lane);
                        bk = ck >= 0 ? sc.piv[ck] : -1;
                    }
                    const int kn = min(32, dv - k0);
#pragma unroll 4
                    for (int k = 0; k < kn; ++k) {
                        const int c = __shfl_sync(0xffffffffu, ck, k), b = __shfl_sync(0xffffffffu, bk, k);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const int w = w0 + q * 32 + lane;
                            if (c >= 0 && (c >> 6) == w) av[q] ^= 1ull << (c & 63);
                            if (b >= 0) {
                                if (w < MW) av[q] ^= sc.vec[static_cast<size_t>(b) * MW + w];
                                if (w < CW) ac[q] ^= sc.comb[static_cast<size_t>(b) * CW + w];
                            }
                        }
                    }
                }
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    const int w = w0 + q * 32 + lane;
                    if (w < MW) sh.wv[w] = av[q];
                    if (w < CW) sh.wc[w] = ac[q] ^ (w == (j >> 6) ? 1ull << (j & 63) : 0ull);
                }
            }
            __syncwarp();
            // lowest set bit of the reduced column, or none (first dependent column)
            unsigned lo = 0x7fffffffu;
            for (int w = lane; w < MW; w += 32) {
                const uint64_t x = sh.wv[w];
                if (x) lo = min(lo, static_cast<unsigned>(w * 64 + __ffsll(static_cast<long long>(x)) - 1));
            }
            lo = __reduce_min_sync(0xffffffffu, lo);
            if (lane == 0) sh.ints[32] = static_cast<int>(lo);
        }
        __syncthreads();
        const int p = sh.ints[32];
        if (p == 0x7fffffff) break;
        // clear the new pivot row from the basis
        const int pw = p >> 6;
        const uint64_t pb = 1ull << (p & 63);
        for (int b0 = warp * 32; b0 < rank; b0 += nwarps * 32) {
            const int b = b0 + lane;
            unsigned hits = __ballot_sync(0xffffffffu, b < rank && (sc.vec[static_cast<size_t>(b) * MW + pw] & pb));
            while (hits) {
                const int bb = b0 + __ffs(hits) - 1;
                hits &= hits - 1;
                uint64_t *bv = sc.vec + static_cast<size_t>(bb) * MW;
                uint64_t *bc = sc.comb + static_cast<size_t>(bb) * CW;
                for (int w = lane; w < MW; w += 32) bv[w] ^= sh.wv[w];
                for (int w = lane; w < CW; w += 32) bc[w] ^= sh.wc[w];
            }
        }
        if (warp == 0) {
            // append; update the residual of the syndrome difference
            uint64_t *nvp = sc.vec + static_cast<size_t>(rank) * MW, *ncp = sc.comb + static_cast<size_t>(rank) * CW;
            for (int w = lane; w < MW; w += 32) nvp[w] = sh.wv[w];
            for (int w = lane; w < CW; w += 32) ncp[w] = sh.wc[w];
            const bool hit = (sc.rvec[pw] & pb) != 0;
            __syncwarp();
            bool nz = false;
            if (hit) {
                for (int w = lane; w < MW; w += 32) nz |= (sc.rvec[w] ^= sh.wv[w]) != 0;
                for (int w = lane; w < CW; w += 32) sc.rcomb[w] ^= sh.wc[w];
            }
            const bool solved = hit && !__any_sync(0xffffffffu, nz);
            __syncwarp();
            if (solved) {
                // the unique solution for every K up to the first dependent column
                for (int w = lane; w < CW; w += 32) sc.delta[w] = sc.rcomb[w];
            }
            if (lane == 0) {
                sc.piv[p] = rank;
                sh.ints[30] = rank + 1;
                if (solved) sh.ints[31] = j + 1;
            }
        }
        __syncthreads();
        if (sh.ints[31] >= 0) break;
    }
    __syncthreads();
    if (sh.ints[31] < 0) return false;
    int wloc = 0;
    for (int w = threadIdx.x; w < CW; w += blockDim.x) wloc += __popcll(sc.delta[w]);
    if (threadIdx.x == 0) sh.ints[33] = 0;
    __syncthreads();
    if (wloc) atomicAdd(&sh.ints[33], wloc);
    __syncthreads();
    if (sh.ints[33] > 30) return false;  // osd_weight_limit
    for (int i = threadIdx.x; i < CW * 64 && i < n; i += blockDim.x)
        if ((sc.delta[i >> 6] >> (i & 63)) & 1ull) sh.est[sc.idx[i]] ^= static_cast<uint8_t>(1 << side);
    __syncthreads();
    return true;
}

// ------------------------------------------------------------------ driver

// Outcome of one post-processing pass.
struct PpOutcome {
    bool ets_used, e6, e12, ok, ets_ok, flip_ok, osd_ok;
};

// The stage sequence of an in-loop attempt or a post-BP pass on sh.est (in place): ETS on
// both sides, then (if the syndromes do not both match) flip sets, then OSD when at most
// 20 checks per side are unsatisfied (jointbp_ets.cpp:2736-3074, 6020-6197).  llr_x / llr_z
// are the |LLR| keys of the OSD column order.
template <class Hist>
static __device__ PpOutcome blk_pp_stages(const DevCode &code, const DevEts &ets, const Hist &hist, int flip_hist,
                                          int act, int k, const double *llr_x, const double *llr_z,
                                          const PpShared &sh, const PpScratch &sc) {
    PpOutcome r{};
    const int gx = blk_ets_multi(code, ets, sh, 0);
    const int gz = blk_ets_multi(code, ets, sh, 1);
    r.ets_used = gx >= 0 || gz >= 0;
    r.e6 = (gx >= 0 && ets.size[gx] == 6) || (gz >= 0 && ets.size[gz] == 6);
    r.e12 = (gx >= 0 && ets.size[gx] == 12) || (gz >= 0 && ets.size[gz] == 12);
    bool ok = false;
    if (r.ets_used) {
        ok = blk_side_diff(code, sh, 0) == 0;
        ok = (blk_side_diff(code, sh, 1) == 0) && ok;
        r.ets_ok = ok;
    }
    if (!ok) {
        const bool fx = blk_flip_side(code, hist, flip_hist, act, sh, sc, 0, k);
        const bool fz = blk_flip_side(code, hist, flip_hist, act, sh, sc, 1, k);
        if (fx || fz) {
            ok = blk_side_diff(code, sh, 0) == 0;
            ok = (blk_side_diff(code, sh, 1) == 0) && ok;
            r.flip_ok = ok;
        }
    }
    if (!ok) {
        const int ux = blk_side_diff(code, sh, 0), uz = blk_side_diff(code, sh, 1);
        if ((ux > uz ? ux : uz) <= 20) {
            const bool ox = blk_osd_side(code, llr_x, sh, sc, 0);
            const bool oz = blk_osd_side(code, llr_z, sh, sc, 1);
            if (ox || oz) {
                ok = blk_side_diff(code, sh, 0) == 0;
                ok = (blk_side_diff(code, sh, 1) == 0) && ok;
                r.osd_ok = ok;
            }
        }
    }
    r.ok = ok;
    return r;
}

// Result flags of a pass (ResultBit), for an in-loop success or a post-BP pass.
__device__ __forceinline__ int pp_result_flags(const PpOutcome &o, bool in_loop_success) {
    if (in_loop_success)
        return kResSyndromeOk | kResPpInDecode | (o.ets_ok ? kResPpInEts : 0) | (o.flip_ok ? kResPpInFlip : 0) |
               (o.ets_used ? kResUsedAny : 0) | (o.e6 ? kResUsed6 : 0) | (o.e12 ? kResUsed12 : 0);
    return kResPostEntered | (o.ok ? kResSyndromeOk : 0) | (o.ets_used ? kResEtsPost : 0) | (o.e6 ? kResUsed6 : 0) |
           (o.e12 ? kResUsed12 : 0) | (o.ets_ok ? kResEtsOk : 0) | (o.flip_ok ? kResFlipOk : 0) |
           (o.osd_ok ? kResOsdOk : 0);
}

}  // namespace jbp
