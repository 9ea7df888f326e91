// Post-processing of the slot engine (ETS / flip / OSD on the GPU, kernels_pp.cuh stages) with
// the |LLR| keys of the OSD order computed on demand.
//
// The OSD stage orders a trial's variables by the |LLR| of the current iteration's totals
// (jointbp_ets.cpp:2484-2492).  Instead of writing those keys for every running slot in every
// variable update from iteration 100 on -- a trial stuck until max-iter pays 2n correctly
// rounded logarithms per iteration whether or not post-processing then runs -- the block that
// post-processes a slot recomputes its totals from the check-to-variable messages, which are
// still those the variable kernel of this iteration read (the next check update comes after
// post-processing), with the variable kernel's own operations in the same order: the same
// doubles (FP64) or floats (FP32 / FP16 storage) as computing them in the variable kernel.
#pragma once

#include "kernels_bp.cuh"
#include "kernels_pp.cuh"

namespace jbp {

// Offset of edge e's message of slot `lane` in group g (msg_off with a run-time check degree).
__device__ __forceinline__ size_t slot_msg_off(int e, int dc, int G, int g, int lane) {
    const int c = e / dc, pos = e - c * dc;
    return ((static_cast<size_t>(c) * G + g) * dc + pos) * kGroup + lane;
}

// |LLR| of the x and z bits of every variable of one slot (block-wide): FP64 as k_var_f64
// (prior * (PX * PZ), normalized, natural-log difference by log_dd), FP32 / FP16 storage as
// k_var_llr (base-2 weights, lse2).
template <typename T>
__device__ void slot_abs_llr_llr(const DevCode &code, const DevRun &run, const DevMsgs &msg, int slot, double *lx_out,
                                 double *lz_out) {
    const int n = code.n, G = run.S / kGroup, group = slot / kGroup, lane = slot % kGroup;
    const int dvx = code.s[0].dv, dvz = code.s[1].dv, dcx = code.s[0].dc, dcz = code.s[1].dc;
    const T *c2vx = static_cast<const T *>(msg.c2v[0]);
    const T *c2vz = static_cast<const T *>(msg.c2v[1]);
    const float4 lp = *reinterpret_cast<const float4 *>(run.lprior + 8 * slot);
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        float Lam = 0.0f, Mu = 0.0f;
        // the variable kernel adds its DV messages in edge order, 0 for a padded edge
        for (int k = 0; k < (dvx > dvz ? dvx : dvz); ++k) {
            const int ex = k < dvx ? __ldg(code.s[0].var_edge + v * dvx + k) : -1;
            const int ez = k < dvz ? __ldg(code.s[1].var_edge + v * dvz + k) : -1;
            Lam += ex >= 0 ? ld_msg<T>(c2vx + slot_msg_off(ex, dcx, G, group, lane)) : 0.0f;
            Mu += ez >= 0 ? ld_msg<T>(c2vz + slot_msg_off(ez, dcz, G, group, lane)) : 0.0f;
        }
        const float w0 = lp.x, w1 = lp.y - Lam, w2 = lp.z - Mu, w3 = lp.w - Lam - Mu;
        lx_out[v] = fabsf(lse2(w1, w3) - lse2(w0, w2));
        lz_out[v] = fabsf(lse2(w2, w3) - lse2(w0, w1));
    }
}

__device__ void slot_abs_llr_f64(const DevCode &code, const DevRun &run, const DevMsgs &msg, int slot, double *lx_out,
                                 double *lz_out) {
    const int n = code.n, G = run.S / kGroup, group = slot / kGroup, lane = slot % kGroup;
    const int dvx = code.s[0].dv, dvz = code.s[1].dv, dcx = code.s[0].dc, dcz = code.s[1].dc;
    const double2 *c2vx = static_cast<const double2 *>(msg.c2v[0]);
    const double2 *c2vz = static_cast<const double2 *>(msg.c2v[1]);
    const double *pr = run.prior + 4 * slot;
    const double p0 = pr[0], p1 = pr[1], p2 = pr[2], p3 = pr[3];
    for (int v = threadIdx.x; v < n; v += blockDim.x) {
        // PX = (XA, XB, XA, XB), PZ = (ZA, ZA, ZB, ZB): products in edge order from 1 (a padded
        // edge multiplies by 1, which changes nothing)
        double XA = 1.0, XB = 1.0, ZA = 1.0, ZB = 1.0;
        for (int k = 0; k < dvx; ++k) {
            const int ex = __ldg(code.s[0].var_edge + v * dvx + k);
            if (ex < 0) continue;
            const double2 m = c2vx[slot_msg_off(ex, dcx, G, group, lane)];
            XA = dmul(XA, m.x);
            XB = dmul(XB, m.y);
        }
        for (int k = 0; k < dvz; ++k) {
            const int ez = __ldg(code.s[1].var_edge + v * dvz + k);
            if (ez < 0) continue;
            const double2 m = c2vz[slot_msg_off(ez, dcz, G, group, lane)];
            ZA = dmul(ZA, m.x);
            ZB = dmul(ZB, m.y);
        }
        double t0 = dmul(p0, dmul(XA, ZA)), t1 = dmul(p1, dmul(XB, ZA));
        double t2 = dmul(p2, dmul(XA, ZB)), t3 = dmul(p3, dmul(XB, ZB));
        norm4(t0, t1, t2, t3);
        const double eps = 1e-300;
        const double px1 = dadd(t1, t3), px0 = dadd(t0, t2), pz1 = dadd(t2, t3), pz0 = dadd(t0, t1);
        lx_out[v] = fabs(dsub(log_dd(px1 > eps ? px1 : eps), log_dd(px0 > eps ? px0 : eps)));
        lz_out[v] = fabs(dsub(log_dd(pz1 > eps ? pz1 : eps), log_dd(pz0 > eps ? pz0 : eps)));
    }
}

// Per-block scratch of k_postprocess: the stages' GF(2) work areas, then the slot's |LLR| keys.
__host__ __device__ inline size_t slot_pp_scratch_bytes(int n, int mmax) {
    return pp_align(pp_scratch_bytes(n, mmax)) + pp_align(16ull * n);
}

// Post-processing of the pending slots (in-loop attempt at iteration k, or post-BP on the
// final estimate).  The stage sequence is the same in both; an in-loop attempt keeps the
// corrected estimate only if both syndromes match, a post-BP run keeps whatever its stages
// applied.  An in-loop attempt at max_iter that fails is followed by post-BP stages on the
// same estimate, which repeat its steps exactly; their result is taken from the same pass.
static __global__ void __launch_bounds__(kPpThreads) k_postprocess(DevCode code, DevRun run, DevMsgs msg,
                                                                    int precision) {
    extern __shared__ unsigned char pp_smem[];
    const int n = code.n, mx = code.s[0].m, mz = code.s[1].m, M = mx + mz, mmax = mx > mz ? mx : mz;
    const PpShared sh = pp_shared_carve(pp_smem, n, M, mmax);
    unsigned char *const blk = run.pp_scratch + run.pp_scratch_stride * blockIdx.x;
    const PpScratch sc = pp_scratch_carve(blk, n, mmax);
    double *const llr = reinterpret_cast<double *>(blk + pp_align(pp_scratch_bytes(n, mmax)));   // [2][n]
    const int npend = *run.n_pp;
    const int G = run.S / kGroup;
    const size_t plane = plane_offset(run, n, 0);
    for (int q = blockIdx.x; q < npend; q += gridDim.x) {
        const int slot = run.pp_list[q];
        const int mode = run.pp_mode[slot];
        const int k = run.iter[slot];
        const int group = slot / kGroup, b = slot % kGroup;
        const size_t row = plane + static_cast<size_t>(group) * n;
        for (int v = threadIdx.x; v < n; v += blockDim.x)
            sh.est[v] = static_cast<uint8_t>(((run.estx[row + v] >> b) & 1u) | (((run.estz[row + v] >> b) & 1u) << 1));
        for (int r = threadIdx.x; r < M; r += blockDim.x)
            sh.tgt[r] = static_cast<uint8_t>((run.synm[static_cast<size_t>(r) * G + group] >> b) & 1u);
        if (precision == JBP_PREC_FP64) slot_abs_llr_f64(code, run, msg, slot, llr, llr + n);
        else if (precision == JBP_PREC_FP32) slot_abs_llr_llr<float>(code, run, msg, slot, llr, llr + n);
        else slot_abs_llr_llr<__half>(code, run, msg, slot, llr, llr + n);
        __syncthreads();
        const SlotHistory hist{&run, slot, k};
        const PpOutcome o = blk_pp_stages(code, run.ets, hist, run.flip_hist, run.act_k[slot], k, llr, llr + n, sh, sc);
        const bool in_loop_success = mode == kPpInLoop && o.ok;
        const bool post = !in_loop_success && (mode == kPpPost || k >= run.max_iter);
        if (in_loop_success || post) {
            // write the corrected decisions back into the slot's bits of the current planes
            const unsigned bit = 1u << b;
            for (int v = threadIdx.x; v < n; v += blockDim.x) {
                const unsigned ox = (run.estx[row + v] >> b) & 1u, oz = (run.estz[row + v] >> b) & 1u;
                const unsigned nx = sh.est[v] & 1u, nz = (sh.est[v] >> 1) & 1u;
                if (ox != nx) atomicXor(&run.estx[row + v], bit);
                if (oz != nz) atomicXor(&run.estz[row + v], bit);
            }
        }
        if (threadIdx.x == 0) {
            if (in_loop_success || post) run.res_flags[slot] = pp_result_flags(o, in_loop_success);
            if (in_loop_success) {
                run.res_iters[slot] = k;
                if (k < run.max_iter) {
                    run.flags[slot] = kFinished;
                    run.retired[atomicAdd(run.n_retired, 1)] = slot;
                }
            }
        }
        __syncthreads();
    }
}

}  // namespace jbp
