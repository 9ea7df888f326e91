// BP message kernels (check and variable updates) for the three precisions.
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
// FP32/FP16 path: log-likelihood ratios.  Check: sign product and the phi-sum rule
// (phi(x) = -log tanh(x/2), its own inverse) over prefix/suffix sums; variable: sums of
// incoming LLRs with the exact joint 4-ary coupling of the X and Z sides.
#pragma once

#include <cuda_fp16.h>

#include "engine.cuh"

namespace jbp {

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// normalize_msg (jointbp_ets.cpp:650-657)
__device__ __forceinline__ void norm4(double &m0, double &m1, double &m2, double &m3) {
    double s = dadd(dadd(dadd(m0, m1), m2), m3);
    if (s <= 0.0) {
        m0 = m1 = m2 = m3 = 0.25;
        return;
    }
    m0 = ddiv(m0, s);
    m1 = ddiv(m1, s);
    m2 = ddiv(m2, s);
    m3 = ddiv(m3, s);
}

// Work item of a (row, group) loop: warps walk rows fastest, groups slowest.
struct WarpItem {
    int row, slot, lane;
};

__device__ __forceinline__ int warp_global_id() { return (blockIdx.x * blockDim.x + threadIdx.x) >> 5; }
__device__ __forceinline__ int warps_total() { return (gridDim.x * blockDim.x) >> 5; }

// ------------------------------------------------------------------ FP64, bit-exact

template <int DC, bool DAMP>
__global__ void __launch_bounds__(256) k_check_f64(DevCode code, DevRun run, DevMsgs msg) {
    const int lane = threadIdx.x & 31;
    const int S = run.S;
    const int mx = code.s[0].m, M = mx + code.s[1].m;
    const long long total = static_cast<long long>(*run.n_groups) * M;
    for (long long w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / M);
        const int row = static_cast<int>(w - static_cast<long long>(gi) * M);
        const int slot = run.groups[gi] * kGroup + lane;
        const int flags = run.flags[slot];
        if (!(flags & kRunning)) continue;
        const int side = row >= mx;
        const int ch = side ? row - mx : row;
        const bool fresh = run.iter[slot] == 0;
        const double2 *v2c = static_cast<const double2 *>(msg.v2c[side]);
        const double2 *v2c_hi = static_cast<const double2 *>(msg.v2c_hi[side]);
        double2 *c2v = static_cast<double2 *>(msg.c2v[side]);
        const double *pr = run.prior + 4 * slot;
        double q0[DC], q1[DC];
#pragma unroll
        for (int i = 0; i < DC; ++i) {
            const size_t idx = static_cast<size_t>(ch * DC + i) * S + slot;
            double m0, m1, m2, m3;
            if (fresh) {
                m0 = pr[0]; m1 = pr[1]; m2 = pr[2]; m3 = pr[3];
            } else if (DAMP) {
                double2 lo = v2c[idx], hi = v2c_hi[idx];
                m0 = lo.x; m1 = lo.y; m2 = hi.x; m3 = hi.y;
            } else {
                double2 q = v2c[idx];
                q0[i] = q.x;
                q1[i] = q.y;
                continue;
            }
            if (side == 0) { q0[i] = dadd(m0, m2); q1[i] = dadd(m1, m3); }
            else { q0[i] = dadd(m0, m1); q1[i] = dadd(m2, m3); }
        }
        double se[DC + 1], so[DC + 1];
        se[DC] = 1.0;
        so[DC] = 0.0;
#pragma unroll
        for (int i = DC - 1; i >= 0; --i) {
            se[i] = dadd(dmul(se[i + 1], q0[i]), dmul(so[i + 1], q1[i]));
            so[i] = dadd(dmul(se[i + 1], q1[i]), dmul(so[i + 1], q0[i]));
        }
        const int s = run.syn[static_cast<size_t>(row) * S + slot];
        double pe = 1.0, po = 0.0;
#pragma unroll
        for (int i = 0; i < DC; ++i) {
            const double p_even = dadd(dmul(pe, se[i + 1]), dmul(po, so[i + 1]));
            const double p_odd = dadd(dmul(pe, so[i + 1]), dmul(po, se[i + 1]));
            const double v0 = s == 0 ? p_even : p_odd;
            const double v1 = s == 0 ? p_odd : p_even;
            const double sum = side == 0 ? dadd(dadd(dadd(v0, v1), v0), v1) : dadd(dadd(dadd(v0, v0), v1), v1);
            double2 out;
            if (sum <= 0.0) {
                out.x = 0.25;
                out.y = 0.25;
            } else {
                out.x = ddiv(v0, sum);
                out.y = ddiv(v1, sum);
            }
            c2v[static_cast<size_t>(ch * DC + i) * S + slot] = out;
            const double ne = dadd(dmul(pe, q0[i]), dmul(po, q1[i]));
            const double no = dadd(dmul(pe, q1[i]), dmul(po, q0[i]));
            pe = ne;
            po = no;
        }
    }
}

template <bool DAMP>
__device__ __forceinline__ void store_v2c_f64(double2 *v2c, double2 *v2c_hi, size_t idx, int side, double n0,
                                              double n1, double n2, double n3, bool fresh, const double *pr,
                                              double damping) {
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
        v2c[idx] = side == 0 ? make_double2(dadd(n0, n2), dadd(n1, n3)) : make_double2(dadd(n0, n1), dadd(n2, n3));
    }
}

template <int DV, bool DAMP>
__global__ void __launch_bounds__(256) k_var_f64(DevCode code, DevRun run, DevMsgs msg, double damping) {
    const int lane = threadIdx.x & 31;
    const int S = run.S, n = code.n;
    const long long total = static_cast<long long>(*run.n_groups) * n;
    const double2 *c2vx = static_cast<const double2 *>(msg.c2v[0]);
    const double2 *c2vz = static_cast<const double2 *>(msg.c2v[1]);
    for (long long w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / n);
        const int v = static_cast<int>(w - static_cast<long long>(gi) * n);
        const int slot = run.groups[gi] * kGroup + lane;
        if (!(run.flags[slot] & kRunning)) continue;
        const bool fresh = run.iter[slot] == 0;
        const double *pr = run.prior + 4 * slot;
        const double p0 = pr[0], p1 = pr[1], p2 = pr[2], p3 = pr[3];
        int ex[DV], ez[DV];
        double ax[DV], bx[DV], az[DV], bz[DV];
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            ex[k] = code.s[0].var_edge[v * DV + k];
            ez[k] = code.s[1].var_edge[v * DV + k];
            const double2 cx = c2vx[static_cast<size_t>(ex[k]) * S + slot];
            const double2 cz = c2vz[static_cast<size_t>(ez[k]) * S + slot];
            ax[k] = cx.x; bx[k] = cx.y; az[k] = cz.x; bz[k] = cz.y;
        }
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
        norm4(t0, t1, t2, t3);
        int best = 0;
        double bv = t0;
        if (t1 > bv) { best = 1; bv = t1; }
        if (t2 > bv) { best = 2; bv = t2; }
        if (t3 > bv) { best = 3; }
        run.est[static_cast<size_t>(v) * S + slot] = static_cast<uint8_t>(best);
        double2 *v2cx = static_cast<double2 *>(msg.v2c[0]);
        double2 *v2cz = static_cast<double2 *>(msg.v2c[1]);
        double2 *v2cx_hi = static_cast<double2 *>(msg.v2c_hi[0]);
        double2 *v2cz_hi = static_cast<double2 *>(msg.v2c_hi[1]);
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            const double EA = dmul(PA[k], SA[k + 1]), EB = dmul(PB[k], SB[k + 1]);
            double n0 = dmul(dmul(p0, EA), ZA), n1 = dmul(dmul(p1, EB), ZA);
            double n2 = dmul(dmul(p2, EA), ZB), n3 = dmul(dmul(p3, EB), ZB);
            norm4(n0, n1, n2, n3);
            store_v2c_f64<DAMP>(v2cx, v2cx_hi, static_cast<size_t>(ex[k]) * S + slot, 0, n0, n1, n2, n3, fresh, pr,
                                damping);
        }
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            const double FA = dmul(QA[k], TA[k + 1]), FB = dmul(QB[k], TB[k + 1]);
            double n0 = dmul(dmul(p0, XA), FA), n1 = dmul(dmul(p1, XB), FA);
            double n2 = dmul(dmul(p2, XA), FB), n3 = dmul(dmul(p3, XB), FB);
            norm4(n0, n1, n2, n3);
            store_v2c_f64<DAMP>(v2cz, v2cz_hi, static_cast<size_t>(ez[k]) * S + slot, 1, n0, n1, n2, n3, fresh, pr,
                                damping);
        }
    }
}

// ------------------------------------------------------------------ FP32 / FP16 LLR

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

constexpr float kLlrMax = 30.0f;     // message LLR clamp
constexpr float kPhiArgMin = 1e-12f; // phi(1e-12) ~ 28.3

// phi(x) = log((1 + e^-x) / (1 - e^-x)) for x >= 0, an involution on (0, inf).
__device__ __forceinline__ float phi_f(float x) {
    x = fmaxf(x, kPhiArgMin);
    if (x > 15.0f) return 2.0f * __expf(-x);
    float t;  // 1 - e^-x without cancellation for small x
    if (x < 0.1f) t = x * (1.0f - x * (0.5f - x * (0.16666667f - x * (0.041666668f - x * 0.008333334f))));
    else t = 1.0f - __expf(-x);
    return __logf(__fdividef(2.0f - t, t));
}

__device__ __forceinline__ float lse2(float a, float b) {
    const float m = fmaxf(a, b);
    return m + __logf(1.0f + __expf(-fabsf(a - b)));
}

__device__ __forceinline__ float clamp_llr(float x) { return fminf(fmaxf(x, -kLlrMax), kLlrMax); }

template <typename T, int DC>
__global__ void __launch_bounds__(256) k_check_llr(DevCode code, DevRun run, DevMsgs msg) {
    const int lane = threadIdx.x & 31;
    const int S = run.S;
    const int mx = code.s[0].m, M = mx + code.s[1].m;
    const long long total = static_cast<long long>(*run.n_groups) * M;
    for (long long w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / M);
        const int row = static_cast<int>(w - static_cast<long long>(gi) * M);
        const int slot = run.groups[gi] * kGroup + lane;
        if (!(run.flags[slot] & kRunning)) continue;
        const int side = row >= mx;
        const int ch = side ? row - mx : row;
        const bool fresh = run.iter[slot] == 0;
        const T *v2c = static_cast<const T *>(msg.v2c[side]);
        T *c2v = static_cast<T *>(msg.c2v[side]);
        const float lp = run.lprior[8 * slot + 4 + side];
        float a[DC];
        unsigned neg = 0;
#pragma unroll
        for (int i = 0; i < DC; ++i) {
            const float L = fresh ? lp : ld_msg<T>(v2c + static_cast<size_t>(ch * DC + i) * S + slot);
            neg |= (L < 0.0f ? 1u : 0u) << i;
            a[i] = phi_f(fabsf(L));
        }
        float suf[DC + 1];
        suf[DC] = 0.0f;
#pragma unroll
        for (int i = DC - 1; i >= 0; --i) suf[i] = suf[i + 1] + a[i];
        const unsigned par = (__popc(neg) & 1u) ^ static_cast<unsigned>(run.syn[static_cast<size_t>(row) * S + slot]);
        float pre = 0.0f;
#pragma unroll
        for (int i = 0; i < DC; ++i) {
            const float mag = fminf(phi_f(pre + suf[i + 1]), kLlrMax);
            const unsigned sg = par ^ ((neg >> i) & 1u);
            st_msg<T>(c2v + static_cast<size_t>(ch * DC + i) * S + slot, sg ? -mag : mag);
            pre += a[i];
        }
    }
}

__device__ __forceinline__ float sigm(float x) { return __fdividef(1.0f, 1.0f + __expf(-x)); }

template <typename T, int DV, bool DAMP>
__global__ void __launch_bounds__(256) k_var_llr(DevCode code, DevRun run, DevMsgs msg, float damping) {
    const int lane = threadIdx.x & 31;
    const int S = run.S, n = code.n;
    const long long total = static_cast<long long>(*run.n_groups) * n;
    const T *c2vx = static_cast<const T *>(msg.c2v[0]);
    const T *c2vz = static_cast<const T *>(msg.c2v[1]);
    T *v2cx = static_cast<T *>(msg.v2c[0]);
    T *v2cz = static_cast<T *>(msg.v2c[1]);
    for (long long w = warp_global_id(); w < total; w += warps_total()) {
        const int gi = static_cast<int>(w / n);
        const int v = static_cast<int>(w - static_cast<long long>(gi) * n);
        const int slot = run.groups[gi] * kGroup + lane;
        if (!(run.flags[slot] & kRunning)) continue;
        int ex[DV], ez[DV];
        float lx[DV], lz[DV];
        float Lam = 0.0f, Mu = 0.0f;
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            ex[k] = code.s[0].var_edge[v * DV + k];
            ez[k] = code.s[1].var_edge[v * DV + k];
            lx[k] = ld_msg<T>(c2vx + static_cast<size_t>(ex[k]) * S + slot);
            lz[k] = ld_msg<T>(c2vz + static_cast<size_t>(ez[k]) * S + slot);
        }
#pragma unroll
        for (int k = 0; k < DV; ++k) { Lam += lx[k]; Mu += lz[k]; }
        const float *lp = run.lprior + 8 * slot;
        // log weights of I, X, Z, Y up to a common constant; first maximum wins
        const float w0 = lp[0], w1 = lp[1] - Lam, w2 = lp[2] - Mu, w3 = lp[3] - Lam - Mu;
        int best = 0;
        float bv = w0;
        if (w1 > bv) { best = 1; bv = w1; }
        if (w2 > bv) { best = 2; bv = w2; }
        if (w3 > bv) { best = 3; }
        run.est[static_cast<size_t>(v) * S + slot] = static_cast<uint8_t>(best);
        const float G = lse2(lp[0], lp[2] - Mu) - lse2(lp[1], lp[3] - Mu);   // x-bit coupling through Z
        const float H = lse2(lp[0], lp[1] - Lam) - lse2(lp[2], lp[3] - Lam); // z-bit coupling through X
        const bool fresh = run.iter[slot] == 0;
#pragma unroll
        for (int k = 0; k < DV; ++k) {
            float ox = clamp_llr(Lam - lx[k] + G);
            float oz = clamp_llr(Mu - lz[k] + H);
            T *px = v2cx + static_cast<size_t>(ex[k]) * S + slot;
            T *pz = v2cz + static_cast<size_t>(ez[k]) * S + slot;
            if (DAMP) {
                const float oldx = fresh ? lp[4] : ld_msg<T>(px);
                const float oldz = fresh ? lp[5] : ld_msg<T>(pz);
                const float d = damping, e = 1.0f - damping;
                const float qx0 = e * sigm(ox) + d * sigm(oldx), qx1 = e * sigm(-ox) + d * sigm(-oldx);
                const float qz0 = e * sigm(oz) + d * sigm(oldz), qz1 = e * sigm(-oz) + d * sigm(-oldz);
                ox = clamp_llr(__logf(fmaxf(qx0, 1e-30f)) - __logf(fmaxf(qx1, 1e-30f)));
                oz = clamp_llr(__logf(fmaxf(qz0, 1e-30f)) - __logf(fmaxf(qz1, 1e-30f)));
            }
            st_msg<T>(px, ox);
            st_msg<T>(pz, oz);
        }
    }
}

}  // namespace jbp
