// jbp_decode_syndromes_noalloc: batched syndrome decoding that allocates no device memory.
//
// Who needs it: callers that cannot call cudaMalloc when they decode.  Examples are
// applications whose device memory is owned by another allocator (a framework's caching
// allocator that must see every byte), and real-time decoding loops that forbid any
// allocation after start-up because an allocation can block for milliseconds and can fail.
// The regular entry points allocate their slot buffers on first use; this one works in a
// fixed scratch area that is part of the library image instead.
//
// The scratch area is the file-scope device array below.  Every GPU that loads the library
// holds it (JBP_NOALLOC_SCRATCH_BYTES) until the process exits.  All calls share it and it
// keeps the last call's contents, so each call clears what must start at zero; calls whose
// work overlaps on the GPU (different streams, or different host threads) race on it and
// must be serialized by the caller.
//
// On the host the array's name is only a host-side stand-in, not a device address: the
// device address is looked up once per device with cudaGetSymbolAddress (with that device
// current) on the first call made on it, so that first call should come before any stream
// capture.  The call itself launches kernels and small copies on the caller's stream and
// waits on that stream; it calls no cudaMalloc, cudaFree or allocating library routine, and
// it leaves the caller's current device as it found it.
//
// It decodes on the slot engine's kernels (the FP64 bit-exact kernels, or the FP32 / FP16
// LLR kernels), so its results equal jbp_decode_syndromes run with engine SLOTS; with engine
// AUTO that call may pick the trial-resident kernels instead, whose FP16 / FP32 arithmetic
// differs slightly.
#include <cstring>
#include <mutex>
#include <sstream>

#include "ctx.hpp"
#include "kernels_bp.cuh"
#include "kernels_slots.cuh"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[JBP_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 128;
void *g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mu;

// Device address of the scratch array on `device` (which must be current).
std::string scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return "device index out of range";
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_addr[device]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return jbp::cuda_err(e, "cudaGetSymbolAddress(scratch)");
        g_scratch_addr[device] = p;
    }
    *out = static_cast<unsigned char *>(g_scratch_addr[device]);
    return "";
}

// Hands out 256-byte aligned pieces of the scratch area.
struct Carver {
    unsigned char *base;
    size_t off = 0;
    template <typename T>
    T *take(size_t count) {
        T *p = reinterpret_cast<T *>(base ? base + off : nullptr);
        off += (sizeof(T) * count + 255) / 256 * 256;
        return p;
    }
};

using CheckFn = void (*)(jbp::DevCode, jbp::DevRun, jbp::DevMsgs);
using VarF64Fn = void (*)(jbp::DevCode, jbp::DevRun, jbp::DevMsgs, double);
using VarLlrFn = void (*)(jbp::DevCode, jbp::DevRun, jbp::DevMsgs, float);

template <int DC, int DV>
void pick(int precision, CheckFn &c, VarF64Fn &v64, VarLlrFn &vl) {
    using namespace jbp;
    if (precision == JBP_PREC_FP64) {
        c = k_check_f64<DC, false>;
        v64 = k_var_f64<DC, DV, false>;
    } else if (precision == JBP_PREC_FP32) {
        c = k_check_llr<float, DC>;
        vl = k_var_llr<float, DC, DV, false>;
    } else {
        c = k_check_llr<__half, DC>;
        vl = k_var_llr<__half, DC, DV, false>;
    }
}

bool pick_kernels(int dc, int dv, int precision, CheckFn &c, VarF64Fn &v64, VarLlrFn &vl) {
    if (dc == 12 && dv == 3) { pick<12, 3>(precision, c, v64, vl); return true; }
    if (dc == 8 && dv == 3) { pick<8, 3>(precision, c, v64, vl); return true; }
    if (dc == 6 && dv == 3) { pick<6, 3>(precision, c, v64, vl); return true; }
    if (dc == 4 && dv == 2) { pick<4, 2>(precision, c, v64, vl); return true; }
    return false;
}

// Carves the run's device state for S slots out of `base` (or only measures it when base
// is null) and returns the bytes used.
size_t layout(const jbp::DevCode &code, int S, int precision, unsigned char *base, jbp::DevRun &r, jbp::DevMsgs &msg) {
    Carver cv{base};
    const size_t es = precision == JBP_PREC_FP64 ? sizeof(double2) : (precision == JBP_PREC_FP32 ? 4 : 2);
    const int n = code.n, M = code.s[0].m + code.s[1].m, G = S / jbp::kGroup;
    for (int s = 0; s < 2; ++s) {
        msg.c2v[s] = cv.take<unsigned char>(es * code.s[s].edges * static_cast<size_t>(S));
        msg.v2c[s] = cv.take<unsigned char>(es * code.s[s].edges * static_cast<size_t>(S));
        msg.v2c_hi[s] = nullptr;
    }
    r.trial = cv.take<long long>(S);
    r.iter = cv.take<int>(S);
    r.flags = cv.take<int>(S);
    r.unsat = cv.take<int>(2 * S);
    r.unsat_mask = cv.take<unsigned>(2 * G);
    r.prior = cv.take<double>(4 * S);
    r.slot_p = cv.take<double>(S);
    r.lprior = cv.take<float>(8 * S);
    r.err = cv.take<uint8_t>(static_cast<size_t>(S) * n);
    r.estx = cv.take<unsigned>(static_cast<size_t>(G) * n);
    r.estz = cv.take<unsigned>(static_cast<size_t>(G) * n);
    r.synm = cv.take<unsigned>(static_cast<size_t>(G) * M);
    r.res_iters = cv.take<int>(S);
    r.res_flags = cv.take<int>(S);
    int *lists = cv.take<int>(3 * S);
    r.retired = lists;
    r.fresh = lists ? lists + S : nullptr;
    r.groups = lists ? lists + 2 * S : nullptr;
    int *counts = cv.take<int>(4);
    r.n_retired = counts;
    r.n_fresh = counts ? counts + 1 : nullptr;
    r.n_groups = counts ? counts + 2 : nullptr;
    r.cnt = cv.take<jbp::DevCounters>(1);
    r.it = cv.take<int>(1);
    r.R = 1;
    return cv.off;
}

// Restores the caller's current device on every return path: embedding callers keep issuing
// runtime calls on their own device after this call.
struct DeviceGuard {
    int saved = -1;
    DeviceGuard() {
        if (cudaGetDevice(&saved) != cudaSuccess) {
            saved = -1;
            cudaGetLastError();
        }
    }
    ~DeviceGuard() {
        if (saved >= 0) cudaSetDevice(saved);
    }
};

}  // namespace

extern "C" int jbp_decode_syndromes_noalloc(jbp_ctx *ctx, const jbp_options *opt, int ntrials, const uint8_t *d_sx,
                                            const uint8_t *d_sz, double p, uint8_t *d_est_out,
                                            jbp_trial_result *d_res, void *stream) {
    using namespace jbp;
    // options first (no CUDA call is needed to reject them), with the checks of every other entry point
    if (!opt) return set_last_error(JBP_ERR_ARG, "jbp_decode_syndromes_noalloc: null options");
    if (std::string bad = validate_options(*opt, p); !bad.empty())
        return set_last_error(JBP_ERR_ARG, "jbp_decode_syndromes_noalloc: " + bad);
    if (opt->engine != JBP_ENGINE_AUTO && opt->engine != JBP_ENGINE_SLOTS)
        return set_last_error(JBP_ERR_UNSUPPORTED,
                              "jbp_decode_syndromes_noalloc runs the slot engine only (engine AUTO or SLOTS)");
    if (opt->enable_pp || opt->freeze_syn || opt->damping > 0.0 || opt->learned_from > 0)
        return set_last_error(JBP_ERR_UNSUPPORTED,
                              "jbp_decode_syndromes_noalloc decodes plain BP only (no post-processing, "
                              "freeze-syn, damping or learned proposals)");
    if (!ctx || !d_sx || !d_sz || !d_res || ntrials < 0)
        return set_last_error(JBP_ERR_ARG, "jbp_decode_syndromes_noalloc: invalid argument");
    if (ntrials == 0) return JBP_OK;
    const Engine &eng = ctx->engine;
    const DevCode &code = eng.dev_code();
    const auto &gx = eng.model().side[0], &gz = eng.model().side[1];
    CheckFn check = nullptr;
    VarF64Fn var64 = nullptr;
    VarLlrFn varllr = nullptr;
    if (!gx.regular || !gz.regular || gx.dc_max != gz.dc_max || gx.dv_max != gz.dv_max ||
        !pick_kernels(gx.dc_max, gx.dv_max, opt->precision, check, var64, varllr))
        return set_last_error(JBP_ERR_UNSUPPORTED, "jbp_decode_syndromes_noalloc: code degrees not built");
    // every trial gets its own slot, so no refill is needed
    const int S = (ntrials + kGroup - 1) / kGroup * kGroup;
    DevRun r{};
    DevMsgs msg{};
    const size_t need = layout(code, S, opt->precision, nullptr, r, msg);
    if (need > JBP_NOALLOC_SCRATCH_BYTES) {
        const size_t per_group = layout(code, kGroup, opt->precision, nullptr, r, msg);
        std::ostringstream os;
        os << "jbp_decode_syndromes_noalloc: " << ntrials << " trials need " << need << " bytes of scratch, more than "
           << "its fixed " << static_cast<size_t>(JBP_NOALLOC_SCRATCH_BYTES) << " bytes (at most about "
           << (JBP_NOALLOC_SCRATCH_BYTES / per_group) * kGroup << " trials of this code at this precision)";
        return set_last_error(JBP_ERR_ARG, os.str());
    }
    const int sm = eng.sm_count(), tpb = 256;
    const int classify_tpb = 128;
    const size_t classify_smem = static_cast<size_t>(classify_tpb / 32) * 2 * code.words * sizeof(uint64_t);
    if (classify_smem > 48 * 1024) return set_last_error(JBP_ERR_UNSUPPORTED, "code too long for this entry point");
    DeviceGuard guard;
    cudaError_t e = cudaSetDevice(eng.device());
    if (e != cudaSuccess) return set_last_error(JBP_ERR_CUDA, cuda_err(e, "cudaSetDevice"));
    unsigned char *base = nullptr;
    std::string err = scratch_address(eng.device(), &base);
    if (!err.empty()) return set_last_error(JBP_ERR_CUDA, err);
    layout(code, S, opt->precision, base, r, msg);
    r.S = S;
    r.max_iter = opt->max_iter;
    r.check_warmup = opt->check_warmup > 0 ? opt->check_warmup : 0;
    r.check_interval = opt->check_interval > 0 ? opt->check_interval : 1;
    r.source = kSrcSyndromes;
    r.use_prior = opt->use_prior ? 1 : 0;
    for (int i = 0; i < 4; ++i) r.prior4[i] = opt->prior[i];
    r.p = p;
    r.first_trial = 0;
    r.ntrials = ntrials;
    r.src_sx = d_sx;
    r.src_sz = d_sz;
    r.est_out = d_est_out;
    r.res_out = d_res;
    r.hist = nullptr;

    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int big_grid = sm * 8;
    const int slot_blocks = (S / kGroup + 7) / 8;
    const int list_grid = (S + tpb - 1) / tpb;
    auto fail_cuda = [](cudaError_t ce) {
        return set_last_error(JBP_ERR_CUDA, cuda_err(ce, "jbp_decode_syndromes_noalloc"));
    };

    // state that must start at zero: counters (the slot flags, lists and masks are
    // re-initialized by the first kernel)
    e = cudaMemsetAsync(r.cnt, 0, sizeof(DevCounters), st);
    if (e != cudaSuccess) return fail_cuda(e);
    k_init_slots<<<list_grid, tpb, 0, st>>>(r);
    e = cudaMemsetAsync(r.n_fresh, 0, sizeof(int), st);
    if (e != cudaSuccess) return fail_cuda(e);
    k_refill<<<list_grid, tpb, 0, st>>>(r, opt->precision);
    k_fresh_syndrome<<<sm * 4, tpb, 0, st>>>(code, r);
    e = cudaMemsetAsync(r.n_groups, 0, sizeof(int), st);
    if (e != cudaSuccess) return fail_cuda(e);
    k_groups<<<slot_blocks, tpb, 0, st>>>(r);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail_cuda(e);
    unsigned long long done = 0;
    for (int it = 0; it < opt->max_iter && done < static_cast<unsigned long long>(ntrials); ++it) {
        check<<<big_grid, tpb, 0, st>>>(code, r, msg);
        if (opt->precision == JBP_PREC_FP64) var64<<<big_grid, tpb, 0, st>>>(code, r, msg, 0.0);
        else varllr<<<big_grid, tpb, 0, st>>>(code, r, msg, 0.0f);
        k_syndrome_check<<<big_grid, tpb, 0, st>>>(code, r);
        e = cudaMemsetAsync(r.n_retired, 0, sizeof(int), st);
        if (e != cudaSuccess) return fail_cuda(e);
        k_retire<<<slot_blocks, tpb, 0, st>>>(r);
        k_classify<<<sm * 2, classify_tpb, classify_smem, st>>>(code, r);
        e = cudaMemsetAsync(r.n_groups, 0, sizeof(int), st);
        if (e != cudaSuccess) return fail_cuda(e);
        k_groups<<<slot_blocks, tpb, 0, st>>>(r);
        e = cudaGetLastError();   // launch errors of this iteration's kernels
        if (e != cudaSuccess) return fail_cuda(e);
        if ((it & 7) == 7 || it + 1 == opt->max_iter) {
            e = cudaMemcpyAsync(&done, &r.cnt->done, sizeof(done), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return fail_cuda(e);
        }
    }
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return fail_cuda(e);
    if (done != static_cast<unsigned long long>(ntrials))
        return set_last_error(JBP_ERR_CUDA, "jbp_decode_syndromes_noalloc: not every trial finished (internal error)");
    return JBP_OK;
}
