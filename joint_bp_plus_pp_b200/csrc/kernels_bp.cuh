// BP message kernels (check and variable updates) for the three precisions.
//
// Message layout.  Edge e = c * dc + pos of a side (check-major, as the reference numbers
// edges) of slot s = g * 32 + lane lives at ((c * G + g) * dc + pos) * 32 + lane, G = S / 32.
// A check-node warp therefore reads and writes one contiguous block (dc x 32 messages);
// a variable-node warp gathers dv such 32-message chunks per side.
//
// FP64 path: the reference CPU decoder's arithmetic, operation by operation
// (jointbp_ets.cpp:2373-2519), with explicit round-to-nearest intrinsics so that the
// compiler cannot contract a multiply and an add into an FMA.  Messages are kept in the
// reduced form that carries every bit the reference uses:
//   c2v X = (a, b, a, b) and c2v Z = (a, a, b, b)  -> stored as the pair (a, b)
//   v2c enters a check only through q0 = m0+m2, q1 = m1+m3 (X) or m0+m1, m2+m3 (Z)
//                                                 -> stored as (q0, q1)
// With damping the full v2c 4-vector is kept, since scaled_mix needs the old message.
//
// FP32/FP16 path: log-likelihood ratios in base 2 (y = log2(q0/q1)), so that the
// exponentials and logarithms are single ex2/lg2 operations.  Check node: the tanh rule in a
// cancellation-free form: per edge u = 2^-|y| (t = (1 - u) / (1 + u)), sets of edges carried as
// (PN, Q) = (prod (1 - u), prod (1 + u) - prod (1 - u)), joined as Q = PD_a Q_b + PN_b Q_a; the
// output over the other edges is log2((2 PN + Q) / Q), clamped at 110; the syndrome bit flips
// the sign.  Variable node: sums of the incoming LLRs and the exact joint 4-ary coupling of
// the X and Z sides; variable-to-check messages are clamped at 120 (2^-120 stays normal).
#pragma once

#include <cuda_fp16.h>

#include "engine.cuh"
#include "numerics.cuh"

namespace jbp {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Correctly rounded quotients m / s of several dividends by one divisor, with one reciprocal
// instead of one division each.  Markstein's theorem (P. Markstein, "Computation of elementary
// functions on the IBM RISC System/6000 processor", IBM J. Res. Dev. 34(1), 1990; Handbook of
// Floating-Point Arithmetic, the FMA-based division): with y = RN(1/s) and q = RN(m y) within one
// ulp of m / s, the remainder r = m - s q is exact by one FMA and RN(q + r y) is RN(m / s) --
// provided nothing underflows or overflows.  The guard keeps m >= 2^-900 and s <= 2^900 (the
// quotients of a normalization are at most 1, so r and q stay normal); outside it, and for
// NaN or infinite operands, the plain division runs.  The result is the IEEE quotient either
// way, so the reference's divisions are reproduced bit for bit (tests/test_division.py checks
// the sequence against IEEE division on the host).
__device__ __forceinline__ double recip_for_div(double s) { return s <= 0x1p900 ? __ddiv_rn(1.0, s) : 0.0; }
__device__ __forceinline__ double div_by_recip(double m, double s, double y) {
    if (m >= 0x1p-900 && s <= 0x1p900) {
        const double q = __dmul_rn(m, y);
        return __fma_rn(__fma_rn(-s, q, m), y, q);
    }
    return __ddiv_rn(m, s);
}

__device__ __forceinline__ double rcp_approx_f64(double s) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(s));
    return y;
}

// RN(1/s) for s in [2^-900, 2^900] without a branch.  Two Newton steps
// y <- y + y (1 - s y) (two FMAs each; each squares the relative error, so any start better than
// 2^-14 ends within one ulp) from the hardware approximation rcp.approx.ftz.f64 (measured on
// B200: relative error at most 2^-19.9 over 10^9 divisors of the domain), then the choice between y and its
// two neighbours: with the remainder r = 1 - s y, exact by one FMA, 1/s - y = r / s, so y is the
// nearest double when -s ulp_below(y) / 2 <= r <= s ulp(y) / 2 (1/s is never a midpoint between
// two doubles, so no tie arises).  Outside the domain the result is not used (the callers take
// the exact path there).  tests/native/reciprocal_rn_check.c runs the sequence on the host
// against IEEE division from perturbed starts; jbp_check_reciprocal compares it on the device
// with the division intrinsic.
__device__ __forceinline__ double recip_rn_fast(double s) {
    double y = rcp_approx_f64(s);
#pragma unroll
    for (int i = 0; i < 2; ++i) y = __fma_rn(y, __fma_rn(-s, y, 1.0), y);
    const double r = __fma_rn(-s, y, 1.0);
    const long long yb = __double_as_longlong(y);
    const double ulp = __longlong_as_double((yb & 0x7FF0000000000000ll) - (52ll << 52));
    const double t_up = __dmul_rn(__dmul_rn(s, ulp), 0.5);
    const double t_dn = (yb & 0x000FFFFFFFFFFFFFll) == 0 ? __dmul_rn(t_up, 0.5) : t_up;
    return r > t_up ? __longlong_as_double(yb + 1) : (r < -t_dn ? __longlong_as_double(yb - 1) : y);
}

// The domain of the branch-free normalization: a divisor in [2^-900, 2^900] and dividends that
// are 0 or at least 2^-900 (the quotients, at most 1, and the remainders stay normal).
__device__ __forceinline__ bool fast_div_ok(double m) { return m == 0.0 || m >= 0x1p-900; }

// normalize_msg (jointbp_ets.cpp:650-657) for operands in the fast domain, without branches:
// one reciprocal (recip_rn_fast) and Markstein's correction per entry (as div_by_recip), so
// the results are the IEEE quotients.  Clears ok when an operand is outside the domain; the
// caller then recomputes with norm4.
__device__ __forceinline__ void norm4_fast(double &m0, double &m1, double &m2, double &m3, bool &ok) {
    const double s = dadd(dadd(dadd(m0, m1), m2), m3);
    ok = ok && s >= 0x1p-900 && s <= 0x1p900 && fast_div_ok(m0) && fast_div_ok(m1) && fast_div_ok(m2) &&
         fast_div_ok(m3);
    const double y = recip_rn_fast(s);
    double q;
    q = __dmul_rn(m0, y); m0 = __fma_rn(__fma_rn(-s, q, m0), y, q);
    q = __dmul_rn(m1, y); m1 = __fma_rn(__fma_rn(-s, q, m1), y, q);
    q = __dmul_rn(m2, y); m2 = __fma_rn(__fma_rn(-s, q, m2), y, q);
    q = __dmul_rn(m3, y); m3 = __fma_rn(__fma_rn(-s, q, m3), y, q);
}

// normalize_msg (jointbp_ets.cpp:650-657): each entry divided by ((m0 + m1) + m2) + m3
__device__ __forceinline__ void norm4(double &m0, double &m1, double &m2, double &m3) {
    double s = dadd(dadd(dadd(m0, m1), m2), m3);
    if (s <= 0.0) {
        m0 = m1 = m2 = m3 = 0.25;
        return;
    }
    const double y = recip_for_div(s);
    m0 = div_by_recip(m0, s, y);
    m1 = div_by_recip(m1, s, y);
    m2 = div_by_recip(m2, s, y);
    m3 = div_by_recip(m3, s, y);
}

__device__ __forceinline__ int warp_global_id() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int warps_total() { return (gridDim.x * blockDim.x) >> 5; }

// Offset of message (edge e of a side with check degree DC, slot group g, lane).
template <int DC>
__device__ __forceinline__ size_t msg_off(int e, int G, int g, int lane) {
    const int c = e / DC, pos = e - c * DC;
    return ((static_cast<size_t>(c) * G + g) * DC + pos) * kGroup + lane;
}

// Hard decisions of one variable for the warp's 32 slots, as x-bit and z-bit planes of the
// current iteration (plane = plane_offset(run, n, 0)).  Called by all lanes; lanes of slots
// that are not running contribute 0 bits.
__device__ __forceinline__ void store_est_bits(const DevRun &run, size_t plane, int group, int n, int v, int best,
                                               bool active) {
    const unsigned xm = __ballot_sync(0xffffffffu, active && (best & 1));
    const unsigned zm = __ballot_sync(0xffffffffu, active && (best & 2));
    const int lane = threadIdx.x & 31;
    if (lane == 0) run.estx[plane + static_cast<size_t>(group) * n + v] = xm;
    if (lane == 1) run.estz[plane + static_cast<size_t>(group) * n + v] = zm;
}

// freeze-syn state of a slot's side in a check kernel: 0 = update normally, 1 = frozen
// (skip), 2 = frozen at the last check (write the deterministic messages, then skip).
__device__ __forceinline__ int frozen_state(const DevRun &run, int slot, int side) {
    if (!run.freeze_syn) return 0;
    const int f = run.frz[slot];
    if (!((f >> side) & 1)) return 0;
    return ((f >> (2 + side)) & 1) ? 2 : 1;
}

// Decision bit (x-bit for side 0, z-bit for side 1) of variable v of a slot in the previous
// iteration's planes, i.e. the estimate the freeze saw (freeze_side_msgs, jointbp_ets.cpp:1884).
__device__ __forceinline__ int frozen_bit(const DevRun &run, int n, int side, int group, int lane, int v) {
    const unsigned *planes = side ? run.estz : run.estx;
    return (planes[plane_offset(run, n, 1) + static_cast<size_t>(group) * n + v] >> lane) & 1u;
}

// ------------------------------------------------------------------ FP64, bit-exact

// The outputs of one check row (jointbp_ets.cpp:2373-2450) from its edges' (q0, q1): suffix
// parities (se, so), then for each edge i the even / odd parity of the other edges (prefix pe,
// po times suffix), ordered by the syndrome bit s and normalized by its side's sum;
// out[i * stride] gets edge i's (a, b).
template <int DC>
__device__ __forceinline__ void check_f64_row(const double *q0, const double *q1, int s, int side, double2 *out,
                                              size_t stride) {
    double se[DC + 1], so[DC + 1];
    se[DC] = 1.0;
    so[DC] = 0.0;
#pragma unroll
    for (int i = DC - 1; i >= 0; --i) {
        se[i] = dadd(dmul(se[i + 1], q0[i]), dmul(so[i + 1], q1[i]));
        so[i] = dadd(dmul(se[i + 1], q1[i]), dmul(so[i + 1], q0[i]));
    }
    double pe = 1.0, po = 0.0;
#pragma unroll
    for (int i = 0; i < DC; ++i) {
        const double p_even = dadd(dmul(pe, se[i + 1]), dmul(po, so[i + 1]));
        const double p_odd = dadd(dmul(pe, so[i + 1]), dmul(po, se[i + 1]));
        const double v0 = s == 0 ? p_even : p_odd;
        const double v1 = s == 0 ? p_odd : p_even;
        const double sum = side == 0 ? dadd(dadd(dadd(v0, v1), v0), v1) : dadd(dadd(dadd(v0, v0), v1), v1);
        double2 o;
        if (sum <= 0.0) {
            o.x = 0.25;
            o.y = 0.25;
        } else {
            o.x = ddiv(v0, sum);
            o.y = ddiv(v1, sum);
        }
        out[i * stride] = o;
        const double ne = dadd(dmul(pe, q0[i]), dmul(po, q1[i]));
        const double no = dadd(dmul(pe, q1[i]), dmul(po, q0[i]));
        pe = ne;
        po = no;
    }
}

// check_f64_row with the two quotients of each output by one branch-free reciprocal and
// Markstein's correction (recip_rn_fast; the IEEE quotients inside the fast domain), the row in
// one basic block.  Returns false, after writing outputs that must not be used, when an operand
// is outside the domain (a sum outside [2^-900, 2^900], a dividend below 2^-900 and not 0): the
// caller then rewrites the row with check_f64_row.
template <int DC>
__device__ __forceinline__ bool check_f64_row_fast(const double *q0, const double *q1, int s, int side,
                                                   double2 *out, size_t stride) {
    double se[DC + 1], so[DC + 1];
    se[DC] = 1.0;
    so[DC] = 0.0;
#pragma unroll
    for (int i = DC - 1; i >= 0; --i) {
        se[i] = dadd(dmul(se[i + 1], q0[i]), dmul(so[i + 1], q1[i]));
        so[i] = dadd(dmul(se[i + 1], q1[i]), dmul(so[i + 1], q0[i]));
    }
    bool ok = true;
    double pe = 1.0, po = 0.0;
#pragma unroll
    for (int i = 0; i < DC; ++i) {
        const double p_even = dadd(dmul(pe, se[i + 1]), dmul(po, so[i + 1]));
        const double p_odd = dadd(dmul(pe, so[i + 1]), dmul(po, se[i + 1]));
        const double v0 = s == 0 ? p_even : p_odd;
        const double v1 = s == 0 ? p_odd : p_even;
        const double sum = side == 0 ? dadd(dadd(dadd(v0, v1), v0), v1) : dadd(dadd(dadd(v0, v0), v1), v1);
        ok = ok && sum >= 0x1p-900 && sum <= 0x1p900 && fast_div_ok(v0) && fast_div_ok(v1);
        const double y = recip_rn_fast(sum);
        const double a = __dmul_rn(v0, y), b = __dmul_rn(v1, y);
        out[i * stride] = make_double2(__fma_rn(__fma_rn(-sum, a, v0), y, a), __fma_rn(__fma_rn(-sum, b, v1), y, b));
        const double ne = dadd(dmul(pe, q0[i]), dmul(po, q1[i]));
        const double no = dadd(dmul(pe, q1[i]), dmul(po, q0[i]));
        pe = ne;
        po = no;
    }
    return ok;
}

template <int DC, bool DAMP>
__global__ void __launch_bounds__(256, 3) k_check_f64(DevCode code, DevRun run, DevMsgs msg) {
    const int lane = threadIdx.x & 31;
    const int G = run.S / kGroup;
    const int mx = code.s[0].m, M = mx + code.s[1].m;
    const unsigned total = static_cast<unsigned>(*run.n_groups) * M;
    for (unsigned w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / static_cast<unsigned>(M));
        const int row = static_cast<int>(w - static_cast<unsigned>(gi) * M);
        const int group = run.groups[gi];
        const int slot = group * kGroup + lane;
        if (!(run.flags[slot] & kRunning)) continue;
        const int side = row >= mx;
        const int ch = side ? row - mx : row;
        const bool fresh = run.iter[slot] == 0;
        const size_t base = (static_cast<size_t>(ch) * G + group) * DC * kGroup + lane;
        const double2 *v2c = static_cast<const double2 *>(side ? msg.v2c[1] : msg.v2c[0]) + base;
        const double2 *v2c_hi = static_cast<const double2 *>(side ? msg.v2c_hi[1] : msg.v2c_hi[0]) + base;
        double2 *c2v = static_cast<double2 *>(side ? msg.c2v[1] : msg.c2v[0]) + base;
        const int fz = frozen_state(run, slot, side);
        if (fz) {
            // det_msg_xbit / det_msg_zbit: bit 0 -> (a, b) = (0.5, 0), bit 1 -> (0, 0.5)
            if (fz == 2) {
#pragma unroll
                for (int i = 0; i < DC; ++i) {
                    const int b = frozen_bit(run, code.n, side, group, lane, __ldg(code.s[side].chk_var + ch * DC + i));
                    c2v[i * kGroup] = b ? make_double2(0.0, 0.5) : make_double2(0.5, 0.0);
                }
            }
            continue;
        }
        const double *pr = run.prior + 4 * slot;
        double q0[DC], q1[DC];
#pragma unroll
        for (int i = 0; i < DC; ++i) {
            double m0, m1, m2, m3;
            if (fresh) {
                m0 = pr[0]; m1 = pr[1]; m2 = pr[2]; m3 = pr[3];
            } else if (DAMP) {
                double2 lo = v2c[i * kGroup], hi = v2c_hi[i * kGroup];
                m0 = lo.x; m1 = lo.y; m2 = hi.x; m3 = hi.y;
            } else {
                double2 q = v2c[i * kGroup];
                q0[i] = q.x;
                q1[i] = q.y;
                continue;
            }
            if (side == 0) { q0[i] = dadd(m0, m2); q1[i] = dadd(m1, m3); }
            else { q0[i] = dadd(m0, m1); q1[i] = dadd(m2, m3); }
        }
        const int s = (run.synm[static_cast<size_t>(row) * G + group] >> lane) & 1;
        check_f64_row<DC>(q0, q1, s, side, c2v, kGroup);
    }
}

// sign: OR-ed into the bits of the undamped message's first value (0, or the sign bit carrying a
// decision bit: probabilities are never negative, so the magnitude stays exact)
template <bool DAMP>
__device__ __forceinline__ void store_v2c_f64(double2 *v2c, double2 *v2c_hi, size_t idx, int side, double n0,
                                              double n1, double n2, double n3, bool fresh, const double *pr,
                                              double damping, unsigned long long sign = 0ull) {
    if (DAMP) {
        if (damping > 0.0) {
            double o0, o1, o2, o3;
            if (fresh) { o0 = pr[0]; o1 = pr[1]; o2 = pr[2]; o3 = pr[3]; }
            else {
                double2 lo = v2c[idx], hi = v2c_hi[idx];
                o0 = lo.x; o1 = lo.y; o2 = hi.x; o3 = hi.y;
            }
            const double a = dsub(1.0, damping);
            n0 = dadd(dmul(a, n0), dmul(damping, o0));
            n1 = dadd(dmul(a, n1), dmul(damping, o1));
            n2 = dadd(dmul(a, n2), dmul(damping, o2));
            n3 = dadd(dmul(a, n3), dmul(damping, o3));
            norm4(n0, n1, n2, n3);
        }
        v2c[idx] = make_double2(n0, n1);
        v2c_hi[idx] = make_double2(n2, n3);
    } else {
        double2 m = side == 0 ? make_double2(dadd(n0, n2), dadd(n1, n3)) : make_double2(dadd(n0, n1), dadd(n2, n3));
        if (sign) m.x = __longlong_as_double(static_cast<long long>(static_cast<unsigned long long>(__double_as_longlong(m.x)) | sign));
        v2c[idx] = m;
    }
}

// The variable update of one slot's variable from its incoming messages: (ax, bx) of each X
// edge and (az, bz) of each Z edge (a padded edge of a lower-degree variable is the identity
// message (1, 1), which leaves the products unchanged exactly).  Writes the new v2c at offsets
// ox / oz of the present edges (unless the side is frozen) and returns the hard decision
// (0..3, the first maximum of the normalized total).  FAST: every normalization through
// norm4_fast, one basic block for the whole update (the seven normalizations' dependency chains
// interleave); ok is cleared when an operand left the fast domain, and the caller then redoes
// the update with FAST = false (norm4), which rewrites the same outputs.  SIGN (undamped only):
// each X message carries the decision's x bit in the sign of its first value, each Z message
// the z bit, for a check phase that tests the syndrome from the messages it reads.
template <int DV, bool DAMP, bool FAST, bool SIGN = false>
__device__ __forceinline__ int var_f64_update(const DevRun &run, const DevMsgs &msg, double damping, int slot, int frz,
                                              const size_t *ox, const size_t *oz, const bool *vx, const bool *vz,
                                              const double *ax, const double *bx, const double *az,
                                              const double *bz, bool &ok) {
    const bool fresh = run.iter[slot] == 0;
    const double *pr = run.prior + 4 * slot;
    const double p0 = pr[0], p1 = pr[1], p2 = pr[2], p3 = pr[3];
    // prefix / suffix products of the X messages (a, b, a, b) and Z messages (a, a, b, b)
    double PA[DV + 1], PB[DV + 1], SA[DV + 1], SB[DV + 1];
    double QA[DV + 1], QB[DV + 1], TA[DV + 1], TB[DV + 1];
    PA[0] = PB[0] = QA[0] = QB[0] = 1.0;
    SA[DV] = SB[DV] = TA[DV] = TB[DV] = 1.0;
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        PA[k + 1] = dmul(PA[k], ax[k]); PB[k + 1] = dmul(PB[k], bx[k]);
        QA[k + 1] = dmul(QA[k], az[k]); QB[k + 1] = dmul(QB[k], bz[k]);
    }
#pragma unroll
    for (int k = DV - 1; k >= 0; --k) {
        SA[k] = dmul(SA[k + 1], ax[k]); SB[k] = dmul(SB[k + 1], bx[k]);
        TA[k] = dmul(TA[k + 1], az[k]); TB[k] = dmul(TB[k + 1], bz[k]);
    }
    const double XA = PA[DV], XB = PB[DV], ZA = QA[DV], ZB = QB[DV];
    // total = normalize(prior * (PX * PZ)); est = first argmax
    double t0 = dmul(p0, dmul(XA, ZA)), t1 = dmul(p1, dmul(XB, ZA));
    double t2 = dmul(p2, dmul(XA, ZB)), t3 = dmul(p3, dmul(XB, ZB));
    int best = 0;
    if (FAST) {
        // The total serves only its first maximum.  Normalizing divides by one positive sum: it
        // keeps the order and merges only values within a rounding of each other, so when every
        // earlier entry is below the maximum by a relative 2^-50 (two roundings of 2^-53 cannot
        // close that gap) and the maximum is normal, the first maximum of the unnormalized total
        // is that of the normalized one.  Otherwise the exact path decides.
        double bv = t0;
        if (t1 > bv) { best = 1; bv = t1; }
        if (t2 > bv) { best = 2; bv = t2; }
        if (t3 > bv) { best = 3; bv = t3; }
        const double lim = dmul(bv, 1.0 - 0x1p-50);
        ok = ok && bv >= 0x1p-1000 && (best < 1 || t0 < lim) && (best < 2 || t1 < lim) && (best < 3 || t2 < lim);
    } else {
        norm4(t0, t1, t2, t3);
        double bv = t0;
        if (t1 > bv) { best = 1; bv = t1; }
        if (t2 > bv) { best = 2; bv = t2; }
        if (t3 > bv) { best = 3; }
    }
    // (the |LLR| keys of the OSD order are computed from the same messages by the block
    // that post-processes the slot: kernels_slot_pp.cuh)
    double2 *v2cx = static_cast<double2 *>(msg.v2c[0]);
    double2 *v2cz = static_cast<double2 *>(msg.v2c[1]);
    double2 *v2cx_hi = static_cast<double2 *>(msg.v2c_hi[0]);
    double2 *v2cz_hi = static_cast<double2 *>(msg.v2c_hi[1]);
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        if (frz & 1) break;
        if (!vx[k]) continue;
        const double EA = dmul(PA[k], SA[k + 1]), EB = dmul(PB[k], SB[k + 1]);
        double n0 = dmul(dmul(p0, EA), ZA), n1 = dmul(dmul(p1, EB), ZA);
        double n2 = dmul(dmul(p2, EA), ZB), n3 = dmul(dmul(p3, EB), ZB);
        if (FAST) norm4_fast(n0, n1, n2, n3, ok);
        else norm4(n0, n1, n2, n3);
        store_v2c_f64<DAMP>(v2cx, v2cx_hi, ox[k], 0, n0, n1, n2, n3, fresh, pr, damping,
                            SIGN ? static_cast<unsigned long long>(best & 1) << 63 : 0ull);
    }
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        if (frz & 2) break;
        if (!vz[k]) continue;
        const double FA = dmul(QA[k], TA[k + 1]), FB = dmul(QB[k], TB[k + 1]);
        double n0 = dmul(dmul(p0, XA), FA), n1 = dmul(dmul(p1, XB), FA);
        double n2 = dmul(dmul(p2, XA), FB), n3 = dmul(dmul(p3, XB), FB);
        if (FAST) norm4_fast(n0, n1, n2, n3, ok);
        else norm4(n0, n1, n2, n3);
        store_v2c_f64<DAMP>(v2cz, v2cz_hi, oz[k], 1, n0, n1, n2, n3, fresh, pr, damping,
                            SIGN ? static_cast<unsigned long long>((best >> 1) & 1) << 63 : 0ull);
    }
    return best;
}

template <int DC, int DV, bool DAMP>
__global__ void __launch_bounds__(256, 2) k_var_f64(DevCode code, DevRun run, DevMsgs msg, double damping) {
    const int lane = threadIdx.x & 31;
    const int G = run.S / kGroup, n = code.n;
    const unsigned total = static_cast<unsigned>(*run.n_groups) * n;
    const size_t plane = plane_offset(run, n, 0);
    const double2 *c2vx = static_cast<const double2 *>(msg.c2v[0]);
    const double2 *c2vz = static_cast<const double2 *>(msg.c2v[1]);
    for (unsigned w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / static_cast<unsigned>(n));
        const int v = static_cast<int>(w - static_cast<unsigned>(gi) * n);
        const int group = run.groups[gi];
        const int slot = group * kGroup + lane;
        const bool active = run.flags[slot] & kRunning;
        if (!__any_sync(0xffffffffu, active)) continue;
        int best = 0;
        if (active) {
            size_t ox[DV], oz[DV];
            bool vx[DV], vz[DV];   // edge present (a variable of lower degree is padded with -1)
            double ax[DV], bx[DV], az[DV], bz[DV];
#pragma unroll
            for (int k = 0; k < DV; ++k) {
                const int ex = __ldg(code.s[0].var_edge + v * DV + k), ez = __ldg(code.s[1].var_edge + v * DV + k);
                vx[k] = ex >= 0;
                vz[k] = ez >= 0;
                ox[k] = vx[k] ? msg_off<DC>(ex, G, group, lane) : 0;
                oz[k] = vz[k] ? msg_off<DC>(ez, G, group, lane) : 0;
            }
#pragma unroll
            for (int k = 0; k < DV; ++k) {
                const double2 cx = vx[k] ? c2vx[ox[k]] : make_double2(1.0, 1.0);
                const double2 cz = vz[k] ? c2vz[oz[k]] : make_double2(1.0, 1.0);
                ax[k] = cx.x; bx[k] = cx.y; az[k] = cz.x; bz[k] = cz.y;
            }
            const int frz = run.freeze_syn ? run.frz[slot] : 0;
            // damped updates (scaled_mix renormalizes inside store_v2c_f64) take the exact path
            bool ok = !DAMP;
            if (!DAMP) best = var_f64_update<DV, DAMP, true>(run, msg, damping, slot, frz, ox, oz, vx, vz, ax, bx, az, bz, ok);
            if (!ok) best = var_f64_update<DV, DAMP, false>(run, msg, damping, slot, frz, ox, oz, vx, vz, ax, bx, az, bz, ok);
        }
        store_est_bits(run, plane, group, n, v, best, active);
    }
}

// ------------------------------------------------------------------ FP32 / FP16 LLR (base 2)

template <typename T>
__device__ __forceinline__ float ld_msg(const T *p);
template <>
__device__ __forceinline__ float ld_msg<float>(const float *p) { return *p; }
template <>
__device__ __forceinline__ float ld_msg<__half>(const __half *p) { return __half2float(*p); }
template <typename T>
__device__ __forceinline__ void st_msg(T *p, float v);
template <>
__device__ __forceinline__ void st_msg<float>(float *p, float v) { *p = v; }
template <>
__device__ __forceinline__ void st_msg<__half>(__half *p, float v) { *p = __float2half_rn(v); }

constexpr float kLlrMax = 110.0f;    // check-to-variable magnitude clamp, base 2 (exact in FP16 storage)
constexpr float kLlrInMax = 120.0f;  // variable-to-check magnitude clamp (2^-120 is a normal float)

// Single special-function-unit operations.
__device__ __forceinline__ float ex2_approx(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float lg2_approx(float x) {
    float y;
    asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// log2(2^a + 2^b)
__device__ __forceinline__ float lse2(float a, float b) {
    return fmaxf(a, b) + lg2_approx(1.0f + ex2_approx(-fabsf(a - b)));
}

__device__ __forceinline__ float clamp_llr(float x) { return fminf(fmaxf(x, -kLlrInMax), kLlrInMax); }

// The LLR check rule on one check of DC edges: from the edges' variable-to-check inputs in(i)
// (base-2 LLRs) and the check's target syndrome bit, out(i, c2v of edge i).  Stable tanh rule
// (PN, Q = prod D - prod N) over u = 2^-|y|, N = 1 - u, D = 1 + u: the output
// log2((2 PN + Q) / Q) keeps its precision when the product of the other edges' tanh is close
// to 1 (see kernels_resident.cuh).
template <int DC, class In, class Out>
__device__ __forceinline__ void llr_check_row(In in, unsigned sbit, Out out) {
    float u[DC];
    unsigned sgn = sbit << 31;
#pragma unroll
    for (int i = 0; i < DC; ++i) {
        const float y = in(i);
        const unsigned sy = __float_as_uint(y) & 0x80000000u;
        sgn ^= sy;
        u[i] = __uint_as_float(__float_as_uint(ex2_approx(-fminf(fabsf(y), kLlrInMax))) | sy);
    }
    float sPN[DC + 1], sQ[DC + 1];
    sPN[DC] = 1.0f;
    sQ[DC] = 0.0f;
#pragma unroll
    for (int i = DC - 1; i >= 0; --i) {
        const float au = fabsf(u[i]);
        sQ[i] = fmaf(1.0f + au, sQ[i + 1], sPN[i + 1] * (au + au));
        sPN[i] = (1.0f - au) * sPN[i + 1];
    }
    float pPN = 1.0f, pQ = 0.0f;
#pragma unroll
    for (int i = 0; i < DC; ++i) {
        const float ePN = pPN * sPN[i + 1];
        const float eQ = fmaf(pPN + pQ, sQ[i + 1], sPN[i + 1] * pQ);
        const float mag = fminf(lg2_approx(fmaf(2.0f, ePN, eQ) * rcp_approx(eQ)), kLlrMax);
        out(i, __uint_as_float(__float_as_uint(mag) ^ ((sgn ^ __float_as_uint(u[i])) & 0x80000000u)));
        const float au = fabsf(u[i]);
        pQ = fmaf(pPN + pQ, au + au, (1.0f - au) * pQ);
        pPN *= 1.0f - au;
    }
}

template <typename T, int DC>
__global__ void __launch_bounds__(256) k_check_llr(DevCode code, DevRun run, DevMsgs msg) {
    const int lane = threadIdx.x & 31;
    const int G = run.S / kGroup;
    const int mx = code.s[0].m, M = mx + code.s[1].m;
    const unsigned total = static_cast<unsigned>(*run.n_groups) * M;
    for (unsigned w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / static_cast<unsigned>(M));
        const int row = static_cast<int>(w - static_cast<unsigned>(gi) * M);
        const int group = run.groups[gi];
        const int slot = group * kGroup + lane;
        if (!(run.flags[slot] & kRunning)) continue;
        const int side = row >= mx;
        const int ch = side ? row - mx : row;
        const bool fresh = run.iter[slot] == 0;
        const size_t base = (static_cast<size_t>(ch) * G + group) * DC * kGroup + lane;
        const T *v2c = static_cast<const T *>(side ? msg.v2c[1] : msg.v2c[0]) + base;
        T *c2v = static_cast<T *>(side ? msg.c2v[1] : msg.c2v[0]) + base;
        const int fz = frozen_state(run, slot, side);
        if (fz) {
            // deterministic messages: bit 0 -> +max, bit 1 -> -max
            if (fz == 2) {
#pragma unroll
                for (int i = 0; i < DC; ++i) {
                    const int b = frozen_bit(run, code.n, side, group, lane, __ldg(code.s[side].chk_var + ch * DC + i));
                    st_msg<T>(c2v + i * kGroup, b ? -kLlrMax : kLlrMax);
                }
            }
            continue;
        }
        const float lp = run.lprior[8 * slot + 4 + side];
        const unsigned sbit = (run.synm[static_cast<size_t>(row) * G + group] >> lane) & 1u;
        llr_check_row<DC>([&](int i) { return fresh ? lp : ld_msg<T>(v2c + i * kGroup); }, sbit,
                          [&](int i, float y) { st_msg<T>(c2v + i * kGroup, y); });
    }
}

__device__ __forceinline__ float sigm2(float y) { return rcp_approx(1.0f + ex2_approx(-y)); }

// The LLR variable rule of one variable from its incoming c2v (lx of the X edges, lz of the Z
// edges; 0 for a padded edge) and its log prior weights lp (I, X, Z, Y): the hard decision
// (first maximum, returned) and the undamped extrinsic outputs with the 4-ary coupling of the
// two sides.
template <int DV>
__device__ __forceinline__ int var_llr_core(const float *lx, const float *lz, float4 lp, float *outx, float *outz) {
    float Lam = 0.0f, Mu = 0.0f;
#pragma unroll
    for (int k = 0; k < DV; ++k) { Lam += lx[k]; Mu += lz[k]; }
    // log2 weights of I, X, Z, Y up to a common constant; first maximum wins
    const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
    int best = 0;
    float bv = w0;
    if (w1 > bv) { best = 1; bv = w1; }
    if (w2 > bv) { best = 2; bv = w2; }
    if (w3 > bv) { best = 3; }
    const float Gx = lse2(lp.x, lp.z - Mu) - lse2(lp.y, lp.w - Mu);   // x-bit coupling through Z
    const float Hz = lse2(lp.x, lp.y - Lam) - lse2(lp.z, lp.w - Lam); // z-bit coupling through X
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        outx[k] = clamp_llr(Lam - lx[k] + Gx);
        outz[k] = clamp_llr(Mu - lz[k] + Hz);
    }
    return best;
}

// One variable of the LLR variable update: sums of the incoming X and Z messages, hard
// decision, and the extrinsic outputs with the 4-ary coupling of the two sides.
template <typename T, int DC, int DV, bool DAMP>
__device__ __forceinline__ int var_llr_one(const DevCode &code, const DevRun &run, const DevMsgs &msg, int v, int group,
                                           int lane, float damping) {
    const int G = run.S / kGroup;
    const int slot = group * kGroup + lane;
    const T *c2vx = static_cast<const T *>(msg.c2v[0]);
    const T *c2vz = static_cast<const T *>(msg.c2v[1]);
    T *v2cx = static_cast<T *>(msg.v2c[0]);
    T *v2cz = static_cast<T *>(msg.v2c[1]);
    size_t ox[DV], oz[DV];
    bool vx[DV], vz[DV];   // edge present (a variable of lower degree is padded with -1)
    float lx[DV], lz[DV];
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        const int ex = __ldg(code.s[0].var_edge + v * DV + k), ez = __ldg(code.s[1].var_edge + v * DV + k);
        vx[k] = ex >= 0;
        vz[k] = ez >= 0;
        ox[k] = vx[k] ? msg_off<DC>(ex, G, group, lane) : 0;
        oz[k] = vz[k] ? msg_off<DC>(ez, G, group, lane) : 0;
    }
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        lx[k] = vx[k] ? ld_msg<T>(c2vx + ox[k]) : 0.0f;
        lz[k] = vz[k] ? ld_msg<T>(c2vz + oz[k]) : 0.0f;
    }
    const float4 lp = *reinterpret_cast<const float4 *>(run.lprior + 8 * slot);
    float outx[DV], outz[DV];
    const int best = var_llr_core<DV>(lx, lz, lp, outx, outz);
    const int frz = run.freeze_syn ? run.frz[slot] : 0;
#pragma unroll
    for (int k = 0; k < DV; ++k) {
        float ox_v = outx[k];
        float oz_v = outz[k];
        if (DAMP) {
            // scaled_mix on the binary marginal: q0 = (1-d) q0_new + d q0_old
            const bool fresh = run.iter[slot] == 0;
            const float oldx = fresh ? run.lprior[8 * slot + 4] : ld_msg<T>(v2cx + ox[k]);
            const float oldz = fresh ? run.lprior[8 * slot + 5] : ld_msg<T>(v2cz + oz[k]);
            const float d = damping, e = 1.0f - damping;
            const float qx0 = e * sigm2(ox_v) + d * sigm2(oldx), qx1 = e * sigm2(-ox_v) + d * sigm2(-oldx);
            const float qz0 = e * sigm2(oz_v) + d * sigm2(oldz), qz1 = e * sigm2(-oz_v) + d * sigm2(-oldz);
            ox_v = clamp_llr(lg2_approx(fmaxf(qx0, 1e-30f)) - lg2_approx(fmaxf(qx1, 1e-30f)));
            oz_v = clamp_llr(lg2_approx(fmaxf(qz0, 1e-30f)) - lg2_approx(fmaxf(qz1, 1e-30f)));
        }
        if (!(frz & 1) && vx[k]) st_msg<T>(v2cx + ox[k], ox_v);
        if (!(frz & 2) && vz[k]) st_msg<T>(v2cz + oz[k], oz_v);
    }
    return best;
}

// Variable-node update over (variable pair, group) warp items: two variables per item keep
// twelve independent message loads in flight per thread.
template <typename T, int DC, int DV, bool DAMP>
__global__ void __launch_bounds__(256) k_var_llr(DevCode code, DevRun run, DevMsgs msg, float damping) {
    const int lane = threadIdx.x & 31;
    const int n = code.n;
    const int pairs = (n + 1) >> 1;
    const unsigned total = static_cast<unsigned>(*run.n_groups) * pairs;
    const size_t plane = plane_offset(run, n, 0);
    for (unsigned w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / static_cast<unsigned>(pairs));
        const int v0 = 2 * static_cast<int>(w - static_cast<unsigned>(gi) * pairs);
        const int group = run.groups[gi];
        const bool active = run.flags[group * kGroup + lane] & kRunning;
        if (!__any_sync(0xffffffffu, active)) continue;
        int b0 = 0, b1 = 0;
        const bool has1 = v0 + 1 < n;
        if (active) {
            b0 = var_llr_one<T, DC, DV, DAMP>(code, run, msg, v0, group, lane, damping);
            if (has1) b1 = var_llr_one<T, DC, DV, DAMP>(code, run, msg, v0 + 1, group, lane, damping);
        }
        store_est_bits(run, plane, group, n, v0, b0, active);
        if (has1) store_est_bits(run, plane, group, n, v0 + 1, b1, active);
    }
}

// Final LLRs of retired trials (diagnostics of the precision report): per variable, natural
// log of P(bit = 1) / P(bit = 0) of the x and z bits, from the c2v in memory when the trial
// retires (those of its last variable update when the syndrome is tested only at max_iter).
template <typename T>
__global__ void k_llr_out(DevCode code, DevRun run, DevMsgs msg) {
    const int nret = *run.n_retired;
    const int n = code.n, G = run.S / kGroup, dc = code.s[0].dc, dv = code.s[0].dv;
    const long long total = static_cast<long long>(nret) * n;
    for (long long i = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; i < total;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int r = static_cast<int>(i / n), v = static_cast<int>(i - static_cast<long long>(r) * n);
        const int slot = run.retired[r];
        const long long local = run.trial[slot] - run.first_trial;
        const int g = slot / kGroup, lane = slot % kGroup;
        float lx, lz;
        if constexpr (sizeof(T) == sizeof(double2)) {
            const double *pr = run.prior + 4 * slot;
            double XA = 1.0, XB = 1.0, ZA = 1.0, ZB = 1.0;
            for (int side = 0; side < 2; ++side)
                for (int k = 0; k < dv; ++k) {
                    const int e = __ldg(code.s[side].var_edge + v * dv + k);
                    if (e < 0) continue;
                    const int c = e / dc, pos = e - c * dc;
                    const double2 m = static_cast<const double2 *>(msg.c2v[side])
                        [((static_cast<size_t>(c) * G + g) * dc + pos) * kGroup + lane];
                    if (side == 0) { XA *= m.x; XB *= m.y; } else { ZA *= m.x; ZB *= m.y; }
                }
            const double t0 = pr[0] * XA * ZA, t1 = pr[1] * XB * ZA, t2 = pr[2] * XA * ZB, t3 = pr[3] * XB * ZB;
            lx = static_cast<float>(log(fmax(t1 + t3, 1e-300)) - log(fmax(t0 + t2, 1e-300)));
            lz = static_cast<float>(log(fmax(t2 + t3, 1e-300)) - log(fmax(t0 + t1, 1e-300)));
        } else {
            float Lam = 0.0f, Mu = 0.0f;
            for (int side = 0; side < 2; ++side)
                for (int k = 0; k < dv; ++k) {
                    const int e = __ldg(code.s[side].var_edge + v * dv + k);
                    if (e < 0) continue;
                    const int c = e / dc, pos = e - c * dc;
                    const float m = ld_msg<T>(static_cast<const T *>(msg.c2v[side]) +
                                              ((static_cast<size_t>(c) * G + g) * dc + pos) * kGroup + lane);
                    if (side == 0) Lam += m; else Mu += m;
                }
            const float *lp = run.lprior + 8 * slot;
            const float w0 = lp[0], w1 = lp[1] - Lam, w2 = lp[2] - Mu, w3 = lp[3] - Lam - Mu;
            lx = (lse2(w1, w3) - lse2(w0, w2)) * 0.69314718f;
            lz = (lse2(w2, w3) - lse2(w0, w1)) * 0.69314718f;
        }
        run.llr_out[(local * n + v) * 2] = lx;
        run.llr_out[(local * n + v) * 2 + 1] = lz;
    }
}

}  // namespace jbp
