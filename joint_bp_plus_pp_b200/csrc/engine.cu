// Batched joint BP engine: device buffers, per-iteration CUDA graph and the run loop.
#include "engine.hpp"

#include <algorithm>
#include <atomic>
#include <memory>
#include <chrono>
#include <cstring>
#include <sstream>

#include "kernels_bp.cuh"
#include "kernels_slots.cuh"
#include "kernels_pp.cuh"
#include "kernels_slot_pp.cuh"
#include "kernels_single.cuh"
#include "kernels_resident.cuh"
#include "kernels_mixed.cuh"
#include "mlp.cuh"

namespace jbp {

std::string cuda_err(cudaError_t e, const char *what) {
    std::ostringstream os;
    os << what << ": " << cudaGetErrorString(e);
    return os.str();
}

namespace {
std::atomic<long long> g_fail_after{-1};

// true when the allocation being made is the one the hook fails
bool take_alloc_failure() {
    long long k = g_fail_after.load();
    while (k >= 0) {
        if (g_fail_after.compare_exchange_weak(k, k - 1)) return k == 0;
    }
    return false;
}
}  // namespace

void set_alloc_failure(long long after) { g_fail_after.store(after < 0 ? -1 : after); }

cudaError_t dev_malloc_bytes(void **p, size_t bytes) {
    if (take_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes);
}

cudaError_t host_malloc_pinned(void **p, size_t bytes) {
    if (take_alloc_failure()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaHostAlloc(p, bytes, cudaHostAllocMapped);
}

#define JBP_CUDA_TRY(expr, what)                                  \
    do {                                                          \
        cudaError_t e_ = (expr);                                  \
        if (e_ != cudaSuccess) return cuda_err(e_, what);         \
    } while (0)

namespace {

template <typename T>
std::string dev_upload(std::vector<void *> &allocs, const std::vector<T> &h, T **out) {
    *out = nullptr;
    size_t bytes = sizeof(T) * std::max<size_t>(h.size(), 1);
    JBP_CUDA_TRY(dev_malloc(reinterpret_cast<void **>(out), bytes), "cudaMalloc(code)");
    allocs.push_back(*out);
    if (!h.empty()) JBP_CUDA_TRY(cudaMemcpy(*out, h.data(), sizeof(T) * h.size(), cudaMemcpyHostToDevice), "upload code");
    return "";
}

// ---------------------------------------------------------------- kernel selection

using CheckFn = void (*)(DevCode, DevRun, DevMsgs);
using VarF64Fn = void (*)(DevCode, DevRun, DevMsgs, double);
using VarLlrFn = void (*)(DevCode, DevRun, DevMsgs, float);
using SingleFn = void (*)(SingleRun);

struct KernelSet {
    CheckFn check = nullptr;
    VarF64Fn var64 = nullptr;
    VarLlrFn varllr = nullptr;
    SingleFn single = nullptr;   // one trial per cooperative launch (FP64, FP32)
};

template <int DC, int DV>
KernelSet kernels_for(int precision, bool damp) {
    KernelSet k;
    if (precision == JBP_PREC_FP64) {
        k.check = damp ? k_check_f64<DC, true> : k_check_f64<DC, false>;
        k.var64 = damp ? k_var_f64<DC, DV, true> : k_var_f64<DC, DV, false>;
        k.single = k_single_f64<DC, DV>;
    } else if (precision == JBP_PREC_FP32) {
        k.check = k_check_llr<float, DC>;
        k.varllr = damp ? k_var_llr<float, DC, DV, true> : k_var_llr<float, DC, DV, false>;
        k.single = k_single_llr<DC, DV>;
    } else {
        k.check = k_check_llr<__half, DC>;
        k.varllr = damp ? k_var_llr<__half, DC, DV, true> : k_var_llr<__half, DC, DV, false>;
    }
    return k;
}

// Regular (dc, dv) pairs built for the GPU.
bool select_kernels(int dc, int dv, int precision, bool damp, KernelSet &k) {
#define JBP_CASE(DC, DV) \
    if (dc == DC && dv == DV) { k = kernels_for<DC, DV>(precision, damp); return true; }
    JBP_CASE(12, 3)
    JBP_CASE(7, 4)
    JBP_CASE(8, 3)
    JBP_CASE(6, 3)
    JBP_CASE(4, 2)
    JBP_CASE(6, 2)
    JBP_CASE(10, 3)
    JBP_CASE(12, 4)
    JBP_CASE(16, 4)
#undef JBP_CASE
    return false;
}

size_t msg_elem_bytes(int precision) {
    return precision == JBP_PREC_FP64 ? sizeof(double2) : (precision == JBP_PREC_FP32 ? sizeof(float) : sizeof(__half));
}

// Run Summary counters of a finished run.
void fill_stats(const DevCounters &hc, jbp_stats &stats) {
    stats.trials = static_cast<long long>(hc.done);
    stats.failures = static_cast<long long>(hc.failures);
    stats.bp_fail = static_cast<long long>(hc.bp_fail);
    stats.pp_success = static_cast<long long>(hc.pp_success);
    stats.flip_pp_success = static_cast<long long>(hc.flip_pp_success);
    stats.osd_pp_success = static_cast<long long>(hc.osd_pp_success);
    stats.stab_success = static_cast<long long>(hc.stab_success);
    stats.ets_used = static_cast<long long>(hc.ets_used);
    stats.ets_saved = static_cast<long long>(hc.ets_saved);
    stats.ets6_used = static_cast<long long>(hc.ets6_used);
    stats.ets6_saved = static_cast<long long>(hc.ets6_saved);
    stats.ets12_used = static_cast<long long>(hc.ets12_used);
    stats.ets12_saved = static_cast<long long>(hc.ets12_saved);
    stats.exact = static_cast<long long>(hc.exact);
    stats.total_iters = static_cast<long long>(hc.total_iters);
    stats.bp_trial_iterations = static_cast<long long>(hc.bp_trial_iterations);
    stats.learned_attempts = static_cast<long long>(hc.learned_attempts);
    stats.learned_success = static_cast<long long>(hc.learned_success);
    stats.syndrome_tests = static_cast<long long>(hc.syndrome_tests);
}

}  // namespace

Engine::~Engine() {
    if (abort_host_) cudaFreeHost(const_cast<int *>(abort_host_));
    for (void *p : single_msg_) cudaFree(p);
    cudaFree(single_est_);
    cudaFree(single_ctl_);   // single_cnt_ lies in the same allocation
    if (single_host_) cudaFreeHost(single_host_);
    if (slot_graph_.exec) cudaGraphExecDestroy(slot_graph_.exec);
    for (cudaEvent_t ev : run_ev_)
        if (ev) cudaEventDestroy(ev);
    cudaFree(res_c2v_scratch_);
    cudaFree(mix_scratch_);
    cudaFree(mix_cnt_);
    free_buffers();
    delete rcode_;
    cudaFree(res_cnt_);
    cudaFree(res_pp_scratch_);
    cudaFree(mlp_dev_);
    for (void *p : code_allocs_) cudaFree(p);
    for (void *p : ets_allocs_) cudaFree(p);
}

std::string Engine::init(CodeModel model, int device) {
    model_ = std::move(model);
    device_ = device;
    int ndev = 0;
    JBP_CUDA_TRY(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
    if (device < 0 || device >= ndev) return "CUDA device " + std::to_string(device) + " not available";
    JBP_CUDA_TRY(cudaSetDevice(device), "cudaSetDevice");
    JBP_CUDA_TRY(cudaDeviceGetAttribute(&sm_count_, cudaDevAttrMultiProcessorCount, device), "device attributes");
    JBP_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin_, cudaDevAttrMaxSharedMemoryPerBlockOptin, device),
                 "device attributes");
    {
        int coop = 0;
        JBP_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, device), "device attributes");
        coop_launch_ = coop != 0;
    }
    {
        int *flag = nullptr, *dflag = nullptr;
        JBP_CUDA_TRY(host_malloc(&flag, sizeof(int)), "cudaHostAlloc(abort flag)");
        abort_host_ = flag;
        *abort_host_ = 0;
        JBP_CUDA_TRY(cudaHostGetDevicePointer(reinterpret_cast<void **>(&dflag), flag, 0), "abort flag");
        abort_dev_ = dflag;
    }
    dcode_.n = model_.n;
    dcode_.words = (model_.n + 63) / 64;
    for (int s = 0; s < 2; ++s) {
        const SideGraph &g = model_.side[s];
        DevSide &d = dcode_.s[s];
        d.m = g.m;
        d.edges = g.edges;
        d.dc = g.dc_max;
        d.dv = g.dv_max;
        int *p = nullptr;
        std::string e = dev_upload(code_allocs_, g.chk_var, &p);
        if (!e.empty()) return e;
        d.chk_var = p;
        // per-variable edge lists padded to dv_max with -1 (variables of lower degree)
        std::vector<int> ve(static_cast<size_t>(model_.n) * std::max(1, g.dv_max), -1);
        for (int v = 0; v < model_.n; ++v)
            for (int k = g.var_off[v]; k < g.var_off[v + 1]; ++k)
                ve[static_cast<size_t>(v) * g.dv_max + (k - g.var_off[v])] = g.var_edge[k];
        e = dev_upload(code_allocs_, ve, &p);
        if (!e.empty()) return e;
        d.var_edge = p;
        uint64_t *rows = nullptr;
        e = dev_upload(code_allocs_, model_.basis[s].rows, &rows);
        if (!e.empty()) return e;
        dcode_.basis_rows[s] = rows;
        e = dev_upload(code_allocs_, model_.basis[s].pivot_row, &p);
        if (!e.empty()) return e;
        dcode_.pivot_row[s] = p;
    }
    res_code_why_ = build_res_code();
    res_code_ok_ = res_code_why_.empty();
    return "";
}

// ---------------------------------------------------------------- trial-resident tier

namespace {

long long host_mod(long long x, long long m) {
    x %= m;
    return x < 0 ? x + m : x;
}

bool host_inverse(long long a, long long m, long long &inv) {
    long long t0 = 0, t1 = 1, r0 = m, r1 = host_mod(a, m);
    while (r1 != 0) {
        const long long q = r0 / r1;
        long long t = t0 - q * t1; t0 = t1; t1 = t;
        long long r = r0 - q * r1; r0 = r1; r1 = r;
    }
    if (r0 != 1) return false;
    inv = host_mod(t0, m);
    return true;
}

}  // namespace

// Recognises a quasi-cyclic code with affine permutation blocks from its check lists: check
// j*P + x has, at position l, variable l*P + ((fa*x + fb) mod P) on both sides, J = m/P block
// rows and L = n/P block columns.  Returns why not, or "" and fills rcode_.
std::string Engine::build_res_code() {
    const int P = model_.P;
    if (P <= 0) return "the code is not quasi-cyclic (built from check lists)";
    const int n = model_.n, m = model_.side[0].m;
    if (n % P || m % P || model_.side[1].m != m) return "block structure does not match P";
    const int J = m / P, L = n / P;
    if (J > kResMaxJ || L > kResMaxL) return "block dimensions beyond the resident kernels";
    if (P > 65535) return "circulant size too large";
    auto rc = std::make_unique<ResCode>();
    std::memset(rc.get(), 0, sizeof(ResCode));
    rc->P = P; rc->J = J; rc->L = L; rc->n = n; rc->m = m;
    for (int s = 0; s < 2; ++s) {
        const SideGraph &g = model_.side[s];
        if (!g.regular || g.dc_max != L || g.dv_max != J) return "side degrees do not match the block structure";
        for (int j = 0; j < J; ++j)
            for (int l = 0; l < L; ++l) {
                auto var_at = [&](int x) { return g.chk_var[static_cast<size_t>(g.chk_off[j * P + x]) + l]; };
                const long long b = var_at(0) - static_cast<long long>(l) * P;
                const long long a = P > 1 ? host_mod(var_at(1) - static_cast<long long>(l) * P - b, P) : 0;
                if (b < 0 || b >= P) return "block column order does not match";
                for (int x = 0; x < P; ++x)
                    if (var_at(x) != l * P + host_mod(a * x + b, P)) return "a block is not an affine permutation";
                long long ia = 0;
                if (!host_inverse(a, P, ia)) return "a block multiplier has no inverse";
                const long long ib = host_mod(-ia * b, P);
                auto fx = [&](long long c) {   // ceil(c 2^32 / P)
                    return static_cast<unsigned>(((static_cast<unsigned long long>(c) << 32) + P - 1) / P);
                };
                rc->fF[s][j][l] = fx(a);
                rc->fG[s][j][l] = fx(b);
                rc->iF[s][j][l] = fx(ia);
                rc->iG[s][j][l] = fx(ib);
                // the fixed-point maps must reproduce both permutations exactly
                for (unsigned x = 0; x < static_cast<unsigned>(P); ++x) {
                    const unsigned y = static_cast<unsigned>(
                        (static_cast<unsigned long long>(x * rc->fF[s][j][l] + rc->fG[s][j][l]) * P) >> 32);
                    const unsigned xb = static_cast<unsigned>(
                        (static_cast<unsigned long long>(x * rc->iF[s][j][l] + rc->iG[s][j][l]) * P) >> 32);
                    if (y != static_cast<unsigned>(host_mod(a * x + b, P)) ||
                        xb != static_cast<unsigned>(host_mod(ia * x + ib, P)))
                        return "fixed-point block map check failed";
                }
            }
    }
    rc->words = dcode_.words;
    for (int s = 0; s < 2; ++s) {
        rc->basis_rows[s] = dcode_.basis_rows[s];
        rc->pivot_row[s] = dcode_.pivot_row[s];
    }
    if (!(P == 768 && J == 3 && L == 12))
        return "no resident kernel built for P=" + std::to_string(P) + ", J=" + std::to_string(J) + ", L=" +
               std::to_string(L);
    const size_t smem = res_smem_bytes(n, m, L, sizeof(__half), true);
    if (smem > static_cast<size_t>(smem_optin_) - 1024) return "trial state does not fit in shared memory";
    rcode_ = rc.release();
    return "";
}

std::string Engine::set_flip_model(const float *params) {
    if (!params) {
        has_mlp_ = false;
        return "";
    }
    JBP_CUDA_TRY(cudaSetDevice(device_), "cudaSetDevice");
    if (!mlp_dev_) JBP_CUDA_TRY(dev_malloc(&mlp_dev_, sizeof(uint32_t) * kMlpDevWords), "cudaMalloc(mlp)");
    std::vector<uint32_t> packed(kMlpDevWords);
    mlp_pack(params, packed.data());
    JBP_CUDA_TRY(cudaMemcpy(mlp_dev_, packed.data(), sizeof(uint32_t) * kMlpDevWords, cudaMemcpyHostToDevice),
                 "upload mlp");
    has_mlp_ = true;
    return "";
}

bool Engine::resident_applies(const jbp_options &o, std::string *why) const {
    auto no = [&](const std::string &w) {
        if (why) *why = w;
        return false;
    };
    if (!res_code_ok_) return no(res_code_why_);
    if (o.precision == JBP_PREC_FP64) return no("the resident tier computes in FP32 (precision FP16 or FP32)");
    if (o.precision == JBP_PREC_FP32 && o.engine != JBP_ENGINE_RESIDENT)
        return no("FP32 messages run on the resident tier only when it is asked for (engine RESIDENT)");
    if (o.enable_pp && (o.check_interval != 1 || o.check_warmup != 0))
        return no("post-processing needs a syndrome test every iteration");
    if (o.learned_from > 0 && !o.enable_pp) return no("learned flip proposals need post-processing on");
    if (o.damping > 0.0) return no("damping runs on the slot tier");
    if (o.freeze_syn) return no("freeze-syn runs on the slot tier");
    return true;
}

std::string Engine::run_resident(const RunRequest &rq, jbp_stats &stats) {
    std::memset(&stats, 0, sizeof(stats));
    const jbp_options &o = rq.opt;
    JBP_CUDA_TRY(cudaSetDevice(device_), "cudaSetDevice");
    if (!res_cnt_) JBP_CUDA_TRY(dev_malloc(&res_cnt_, sizeof(DevCounters)), "cudaMalloc(counters)");
    const ResCode &rc = *rcode_;
    const bool pp = o.enable_pp != 0;
    // FP16 messages in shared memory; FP32 messages in a per-block global scratch (L2)
    const bool f32 = o.precision == JBP_PREC_FP32;
    auto kern = f32 ? (!pp ? k_resident<768, 3, 12, StoreFloat, false, false, true>
                           : (o.learned_from > 0 ? k_resident<768, 3, 12, StoreFloat, true, true, true>
                                                 : k_resident<768, 3, 12, StoreFloat, true, false, true>))
                    : (!pp ? k_resident<768, 3, 12, StoreHalf, false, false>
                           : (o.learned_from > 0 ? k_resident<768, 3, 12, StoreHalf, true, true>
                                                 : k_resident<768, 3, 12, StoreHalf, true, false>));
    const size_t store = f32 ? sizeof(float) : sizeof(__half);
    const int c2v_sides = f32 ? 1 : 2;   // sides whose c2v live in shared memory
    const size_t smem = res_smem_bytes(rc.n, rc.m, rc.L, store, pp, c2v_sides);
    JBP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                 "smem attribute");
    int per_sm = 0;
    JBP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kResThreads, smem), "occupancy");
    if (per_sm < 1) return "the resident kernel does not fit on an SM";
    const long long want = std::max<long long>(1, std::min<long long>(rq.ntrials, 1LL << 30));
    const int grid = static_cast<int>(std::min<long long>(static_cast<long long>(per_sm) * sm_count_, want));
    const int H = std::max(0, o.flip_hist);
    const bool learned = pp && o.learned_from > 0;
    if (learned && !rq.collect && !has_mlp_ && o.learned_order == 0)
        return "learned flip proposals requested but no model is set";
    const int R = std::max(H + 1, learned ? 6 : 3);   // the kernel's ring size
    size_t stride = 0;
    if (pp) {
        std::string ee = upload_ets();
        if (!ee.empty()) return ee;
        stride = pp_align(res_pp_scratch_bytes(rc.n, rc.m, R));
        const size_t need = stride * grid;
        if (res_pp_bytes_ < need) {
            cudaFree(res_pp_scratch_);
            res_pp_scratch_ = nullptr;
            res_pp_bytes_ = 0;
            JBP_CUDA_TRY(dev_malloc(&res_pp_scratch_, need), "cudaMalloc(post-processing scratch)");
            res_pp_bytes_ = need;
        }
    }
    size_t c2v_stride = 0;
    if (f32) {
        c2v_stride = (1ull * rc.L * rc.m * sizeof(float) + 255) / 256 * 256;   // the Z side
        if (res_c2v_bytes_ < c2v_stride * grid) {
            cudaFree(res_c2v_scratch_);
            res_c2v_scratch_ = nullptr;
            res_c2v_bytes_ = 0;
            JBP_CUDA_TRY(dev_malloc(&res_c2v_scratch_, c2v_stride * grid), "cudaMalloc(message scratch)");
            res_c2v_bytes_ = c2v_stride * grid;
        }
    }
    ResRun r{};
    r.max_iter = o.max_iter;
    r.check_warmup = std::max(0, o.check_warmup);
    r.check_interval = std::max(1, o.check_interval);
    r.source = rq.source;
    r.p = rq.p;
    r.p_max = o.p_max;
    r.use_prior = o.use_prior ? 1 : 0;
    for (int i = 0; i < 4; ++i) r.prior4[i] = o.prior[i];
    r.seed = rq.seed;
    r.first_trial = rq.first_trial;
    r.ntrials = rq.ntrials;
    r.trial_list = nullptr;
    r.src_err = rq.d_err;
    r.src_sx = rq.d_sx;
    r.src_sz = rq.d_sz;
    r.est_out = rq.d_est_out;
    r.llr_out = rq.d_llr_out;
    r.res_out = rq.d_res_out;
    r.hist = rq.d_hist;
    r.cnt = res_cnt_;
    r.flip_hist = H;
    r.dc = dcode_;
    r.ets = dets_;
    r.pp_scratch = pp ? res_pp_scratch_ : nullptr;
    r.pp_scratch_stride = stride;
    r.pp_smem_base = pp_align(res_base_bytes(rc.n, rc.m, rc.L, store, c2v_sides));
    r.c2v_scratch = f32 ? res_c2v_scratch_ : nullptr;
    r.c2v_stride = c2v_stride;
    r.learned_from = learned ? o.learned_from : 0;
    r.learned_order = o.learned_order;
    r.learned_cols = o.learned_cols > 0 ? std::min(o.learned_cols, rc.n) : kLearnedMaxCols;
    r.mlp.w = mlp_dev_;
    r.collect = rq.collect ? 1 : 0;
    r.collect_every = o.collect_every > 0 ? static_cast<unsigned>(o.collect_every) : 32u;
    r.col_x = rq.d_col_x;
    r.col_y = rq.d_col_y;
    r.col_count = rq.d_col_count;
    r.col_cap = rq.col_cap;
    r.budget_ns = o.watchdog_ms > 0 ? static_cast<unsigned long long>(o.watchdog_ms) * 1000000ull : 0ull;
    r.abort_flag = abort_dev_;
    cudaStream_t st = rq.stream;
    cudaEvent_t ev0, ev1;
    JBP_CUDA_TRY(cudaEventCreate(&ev0), "cudaEventCreate");
    JBP_CUDA_TRY(cudaEventCreate(&ev1), "cudaEventCreate");
    std::string err;
    cudaError_t ce = cudaEventRecord(ev0, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(res_cnt_, 0, sizeof(DevCounters), st);
    if (ce == cudaSuccess) {
        kern<<<grid, kResThreads, smem, st>>>(rc, r);
        ce = cudaGetLastError();
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(ev1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
    DevCounters hc{};
    if (ce == cudaSuccess) ce = cudaMemcpy(&hc, res_cnt_, sizeof(hc), cudaMemcpyDeviceToHost);
    float ms = 0.0f;
    if (ce == cudaSuccess) cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (ce != cudaSuccess) return cuda_err(ce, "resident run");
    if (hc.bad_input) return "error vector has invalid value";
    fill_stats(hc, stats);
    stats.device_ms = ms;
    stats.kernel_launches = 1;
    stats.slots = grid;
    if (hc.watchdog)
        return "watchdog expired: the run budget of " + std::to_string(o.watchdog_ms) + " ms ran out on the device after " +
               std::to_string(hc.done) + " of " + std::to_string(rq.ntrials) + " trials";
    if (hc.aborted)
        return "aborted by request after " + std::to_string(hc.done) + " of " + std::to_string(rq.ntrials) + " trials";
    if (hc.done != static_cast<unsigned long long>(rq.ntrials)) return "resident run finished an unexpected number of trials";
    return "";
}

// The single-trial path takes FP64 and FP32 decodes of up to kSingleMaxTrials given syndromes with plain
// undamped BP and no profile, run budget, frozen sides or per-trial error rate -- the calls of
// the drop-in's cuda_bp_decode -- unless the slot engine is asked for by name.  The iteration
// limit keeps a launch's barrier count within the 31 bits of its barrier word.
constexpr int kSingleMaxIter = 1000000;

bool Engine::single_applies(const RunRequest &rq) const {
    const jbp_options &o = rq.opt;
    return coop_launch_ && o.engine == JBP_ENGINE_AUTO && (o.precision == JBP_PREC_FP64 || o.precision == JBP_PREC_FP32) &&
           !o.enable_pp && o.damping <= 0.0 &&
           !o.freeze_syn && !o.profile && o.watchdog_ms <= 0 && !(o.p_max > rq.p) && rq.source == kSrcSyndromes &&
           rq.ntrials >= 1 && rq.ntrials <= kSingleMaxTrials && o.max_iter <= kSingleMaxIter && !rq.d_llr_out &&
           !rq.collect;
}

// Whether every block of a single-trial launch can be resident at once on this device (a
// cooperative launch needs it; a partition with few SMs decodes on the slot engine instead).
bool Engine::single_fits(const void *fn) {
    for (const auto &f : single_fit_)
        if (f.first == fn) return f.second;
    int per_sm = 0;
    const cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kSingleThreads, 0);
    if (e != cudaSuccess) cudaGetLastError();   // the query's own error: the slot engine then decodes
    const bool fits = e == cudaSuccess && static_cast<long long>(per_sm) * sm_count_ >= kSingleBlocks;
    single_fit_.emplace_back(fn, fits);
    return fits;
}

std::string Engine::run_single(const RunRequest &rq, jbp_stats &stats) {
    const jbp_options &o = rq.opt;
    const SideGraph &gx = model_.side[0], &gz = model_.side[1];
    KernelSet ks;
    if (!select_kernels(gx.dc_max, gx.dv_max, o.precision, false, ks) || !ks.single)
        return "no single-trial kernel for this code";
    const int n = model_.n;
    for (int s = 0; s < 2; ++s) {
        const size_t bytes = sizeof(double2) * static_cast<size_t>(model_.side[s].edges);
        if (!single_msg_[s]) JBP_CUDA_TRY(dev_malloc(&single_msg_[s], bytes), "cudaMalloc(single-trial messages)");
        if (!single_msg_[2 + s])
            JBP_CUDA_TRY(dev_malloc(&single_msg_[2 + s], bytes), "cudaMalloc(single-trial messages)");
    }
    constexpr size_t state_bytes = kSingleCntOffset + sizeof(DevCounters);
    static_assert(sizeof(int) * 8 <= kSingleCntOffset, "control words before the counters");
    if (!single_ctl_) {
        JBP_CUDA_TRY(dev_malloc(&single_ctl_, state_bytes), "cudaMalloc(single-trial control)");
        single_cnt_ = reinterpret_cast<DevCounters *>(reinterpret_cast<unsigned char *>(single_ctl_) + kSingleCntOffset);
    }
    if (!single_host_) JBP_CUDA_TRY(host_malloc(&single_host_, state_bytes), "cudaHostAlloc(single-trial control)");
    if (!rq.d_est_out && !single_est_)
        JBP_CUDA_TRY(dev_malloc(&single_est_, static_cast<size_t>(n)), "cudaMalloc(single-trial decisions)");
    SingleRun sr{};
    sr.code = dcode_;
    sr.max_iter = o.max_iter;
    sr.check_warmup = std::max(0, o.check_warmup);
    sr.check_interval = std::max(1, o.check_interval);
    if (o.use_prior) {
        for (int i = 0; i < 4; ++i) sr.prior[i] = o.prior[i];
    } else {
        // normalize(1-p, p/3, p/3, p/3) as the slot engine's refill and jointbp_ets.cpp:5484-5485
        double p0 = 1.0 - rq.p, p1 = rq.p / 3.0, p2 = p1, p3 = p1;
        const double s = ((p0 + p1) + p2) + p3;
        if (s <= 0.0) { p0 = p1 = p2 = p3 = 0.25; }
        else { p0 = p0 / s; p1 = p1 / s; p2 = p2 / s; p3 = p3 / s; }
        sr.prior[0] = p0; sr.prior[1] = p1; sr.prior[2] = p2; sr.prior[3] = p3;
    }
    for (int s = 0; s < 2; ++s) {
        sr.c2v[s] = static_cast<double2 *>(single_msg_[s]);
        sr.v2c[s] = static_cast<double2 *>(single_msg_[2 + s]);
    }
    static_assert(sizeof(unsigned long long) * kSingleMaxTrials <= sizeof(int) * kSingleErrWord &&
                      kSingleErrWord < 8,
                  "barrier words, then the error flag, within the eight control words");
    sr.err = single_ctl_ + kSingleErrWord;
    sr.cnt = single_cnt_;
    sr.hist = rq.d_hist;
    sr.res_out = rq.d_res_out;
    cudaStream_t st = rq.stream;
    if (!run_ev_[0]) {
        for (int i = 0; i < 2; ++i) JBP_CUDA_TRY(cudaEventCreate(&run_ev_[i]), "cudaEventCreate");
        for (int i = 2; i < 4; ++i)
            JBP_CUDA_TRY(cudaEventCreateWithFlags(&run_ev_[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    cudaError_t ce = cudaEventRecord(run_ev_[0], st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(single_ctl_, 0, state_bytes, st);
    const int mx = gx.m, mz = gz.m;
    for (long long t = 0; t < rq.ntrials && ce == cudaSuccess; ++t) {
        sr.sx = rq.d_sx + t * mx;
        sr.sz = rq.d_sz + t * mz;
        sr.est = rq.d_est_out ? rq.d_est_out + t * n : single_est_;
        sr.local = t;
        sr.bar = reinterpret_cast<unsigned long long *>(single_ctl_) + t;   // zeroed above, one per launch
        void *args[] = {&sr};
        ce = cudaLaunchCooperativeKernel(reinterpret_cast<void *>(ks.single), kSingleBlocks, kSingleThreads, args, 0,
                                         st);
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(run_ev_[1], st);
    // control words, counters and the caller's host copies queued behind the launches: one wait
    // for the whole call
    if (ce == cudaSuccess) ce = cudaMemcpyAsync(single_host_, single_ctl_, state_bytes, cudaMemcpyDeviceToHost, st);
    const bool copy_res = rq.h_res_out && rq.d_res_out, copy_est = rq.h_est_out && rq.d_est_out;
    if (ce == cudaSuccess && copy_res)
        ce = cudaMemcpyAsync(rq.h_res_out, rq.d_res_out, sizeof(jbp_trial_result) * rq.ntrials, cudaMemcpyDeviceToHost,
                             st);
    if (ce == cudaSuccess && copy_est)
        ce = cudaMemcpyAsync(rq.h_est_out, rq.d_est_out, static_cast<size_t>(rq.ntrials) * n, cudaMemcpyDeviceToHost,
                             st);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(st);
    if (ce != cudaSuccess) return cuda_err(ce, "single-trial run");
    int ctl[8];
    DevCounters hc;
    std::memcpy(ctl, single_host_, sizeof(ctl));
    std::memcpy(&hc, single_host_ + kSingleCntOffset, sizeof(hc));
    if (ctl[kSingleErrWord])
        return "single-trial run: a grid barrier waited longer than its limit (internal error)";
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, run_ev_[0], run_ev_[1]);
    fill_stats(hc, stats);
    stats.device_ms = ms;
    stats.kernel_launches = rq.ntrials;
    stats.slots = 1;
    if (hc.done != static_cast<unsigned long long>(rq.ntrials)) return "single-trial run finished an unexpected number of trials";
    if (rq.host_copied) *rq.host_copied = (copy_res || !rq.h_res_out) && (copy_est || !rq.h_est_out);
    return "";
}

void Engine::free_buffers() {
    for (void *&p : buf_.msg) { cudaFree(p); p = nullptr; }
    cudaFree(buf_.trial); cudaFree(buf_.iter); cudaFree(buf_.flags); cudaFree(buf_.frz); cudaFree(buf_.unsat);
    cudaFree(buf_.prior); cudaFree(buf_.lprior); cudaFree(buf_.err); cudaFree(buf_.slot_p);
    cudaFree(buf_.unsat_mask); cudaFree(buf_.estx); cudaFree(buf_.estz); cudaFree(buf_.synm);
    cudaFree(buf_.res_iters); cudaFree(buf_.res_flags); cudaFree(buf_.lists); cudaFree(buf_.counts);
    cudaFree(buf_.cnt);
    cudaFree(buf_.it);
    cudaFree(buf_.act_k); cudaFree(buf_.pstate); cudaFree(buf_.stall_same);
    cudaFree(buf_.pp_list); cudaFree(buf_.pp_mode); cudaFree(buf_.us_hist); cudaFree(buf_.dprev);
    cudaFree(buf_.dpprev); cudaFree(buf_.pp_scratch);
    if (buf_.h_done) cudaFreeHost(buf_.h_done);
    buf_ = Buffers{};
}

// Flattens the loaded ETS groups into device arrays (DevEts), in load order.
std::string Engine::upload_ets() {
    if (ets_uploaded_ == model_.ets.size()) return "";
    for (void *p : ets_allocs_) cudaFree(p);
    ets_allocs_.clear();
    dets_ = DevEts{};
    if (model_.ets.size() > static_cast<size_t>(kMaxEtsGroups)) return "too many ETS groups";
    std::vector<unsigned long long> keys;
    std::vector<int> vars, var_first;
    dets_.ngroups = static_cast<int>(model_.ets.size());
    for (int g = 0; g < dets_.ngroups; ++g) {
        const EtsGroup &grp = model_.ets[g];
        dets_.size[g] = grp.size;
        for (int s = 0; s < 2; ++s) {
            dets_.first[g][s] = static_cast<int>(keys.size());
            dets_.count[g][s] = grp.loaded[s] ? grp.tab[s].count() : 0;
            if (!grp.loaded[s]) continue;
            for (int e = 0; e < grp.tab[s].count(); ++e) {
                keys.push_back(grp.tab[s].key[e]);
                var_first.push_back(static_cast<int>(vars.size()));
                const int *v = grp.tab[s].vars.data() + static_cast<size_t>(e) * grp.tab[s].var_count;
                vars.insert(vars.end(), v, v + grp.tab[s].var_count);
            }
        }
    }
    unsigned long long *dk = nullptr;
    int *dv = nullptr, *df = nullptr;
    std::string e = dev_upload(ets_allocs_, keys, &dk);
    if (e.empty()) e = dev_upload(ets_allocs_, vars, &dv);
    if (e.empty()) e = dev_upload(ets_allocs_, var_first, &df);
    if (!e.empty()) return e;
    dets_.key = dk;
    dets_.vars = dv;
    dets_.var_first = df;
    ets_uploaded_ = model_.ets.size();
    return "";
}

std::string Engine::ensure_buffers(int S, int precision, bool damp, bool pp, int R, cudaStream_t st) {
    if (buf_.S == S && buf_.precision == precision && buf_.damp == damp && buf_.pp == pp && buf_.R == R) return "";
    free_buffers();
    const int n = model_.n, M = model_.side[0].m + model_.side[1].m;
    const size_t es = msg_elem_bytes(precision);
    for (int s = 0; s < 2; ++s) {
        const size_t bytes = es * static_cast<size_t>(model_.side[s].edges) * S;
        JBP_CUDA_TRY(dev_malloc(&buf_.msg[s], bytes), "cudaMalloc(c2v)");
        JBP_CUDA_TRY(dev_malloc(&buf_.msg[2 + s], bytes), "cudaMalloc(v2c)");
        if (precision == JBP_PREC_FP64 && damp) JBP_CUDA_TRY(dev_malloc(&buf_.msg[4 + s], bytes), "cudaMalloc(v2c hi)");
        buf_.msg_bytes += bytes * (precision == JBP_PREC_FP64 && damp ? 3 : 2);
    }
    JBP_CUDA_TRY(dev_malloc(&buf_.trial, sizeof(long long) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.iter, sizeof(int) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.flags, sizeof(int) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.frz, sizeof(int) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.unsat, sizeof(int) * 2 * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.prior, sizeof(double) * 4 * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.slot_p, sizeof(double) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.lprior, sizeof(float) * 8 * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.err, static_cast<size_t>(n) * S), "cudaMalloc(err)");
    const size_t G = static_cast<size_t>(S) / kGroup;
    JBP_CUDA_TRY(dev_malloc(&buf_.estx, sizeof(unsigned) * R * G * n), "cudaMalloc(est)");
    JBP_CUDA_TRY(dev_malloc(&buf_.estz, sizeof(unsigned) * R * G * n), "cudaMalloc(est)");
    JBP_CUDA_TRY(dev_malloc(&buf_.it, sizeof(int)), "cudaMalloc(it)");
    if (pp) {
        const int mmax = std::max(model_.side[0].m, model_.side[1].m);
        JBP_CUDA_TRY(dev_malloc(&buf_.act_k, sizeof(int) * S), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.pstate, sizeof(int) * S), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.stall_same, sizeof(int) * S), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.pp_list, sizeof(int) * S), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.pp_mode, sizeof(int) * S), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.us_hist, sizeof(unsigned short) * 100 * S), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.dprev, sizeof(unsigned) * G), "cudaMalloc(pp)");
        JBP_CUDA_TRY(dev_malloc(&buf_.dpprev, sizeof(unsigned) * G), "cudaMalloc(pp)");
        JBP_CUDA_TRY(cudaMemsetAsync(buf_.dprev, 0, sizeof(unsigned) * G, st), "memset(pp)");
        JBP_CUDA_TRY(cudaMemsetAsync(buf_.dpprev, 0, sizeof(unsigned) * G, st), "memset(pp)");
        buf_.pp_stride = slot_pp_scratch_bytes(n, mmax);
        buf_.pp_blocks = std::min(sm_count_, static_cast<int>(S));
        JBP_CUDA_TRY(dev_malloc(&buf_.pp_scratch, buf_.pp_stride * buf_.pp_blocks), "cudaMalloc(pp scratch)");
    }
    JBP_CUDA_TRY(dev_malloc(&buf_.synm, sizeof(unsigned) * G * M), "cudaMalloc(syn)");
    JBP_CUDA_TRY(cudaMemsetAsync(buf_.synm, 0, sizeof(unsigned) * G * M, st), "memset(syn)");
    JBP_CUDA_TRY(dev_malloc(&buf_.unsat_mask, sizeof(unsigned) * 2 * G), "cudaMalloc(unsat)");
    JBP_CUDA_TRY(dev_malloc(&buf_.res_iters, sizeof(int) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.res_flags, sizeof(int) * S), "cudaMalloc(slots)");
    JBP_CUDA_TRY(dev_malloc(&buf_.lists, sizeof(int) * (3 * S)), "cudaMalloc(lists)");
    JBP_CUDA_TRY(dev_malloc(&buf_.counts, sizeof(int) * 4), "cudaMalloc(lists)");
    JBP_CUDA_TRY(dev_malloc(&buf_.cnt, sizeof(DevCounters)), "cudaMalloc(counters)");
    JBP_CUDA_TRY(host_malloc(&buf_.h_done, sizeof(unsigned long long) * 2), "cudaMallocHost");
    // the memsets above are ordered on the run's stream (no device-wide synchronization: another
    // context may be capturing a graph on another host thread)
    buf_.S = S;
    buf_.precision = precision;
    buf_.damp = damp;
    buf_.pp = pp;
    buf_.R = R;
    return "";
}

int Engine::choose_slots(const jbp_options &opt, long long ntrials) const {
    long long S = opt.slots;
    if (S <= 0) S = opt.precision == JBP_PREC_FP64 ? 8192 : 16384;
    long long need = (std::max<long long>(ntrials, 1) + kGroup - 1) / kGroup * kGroup;
    S = std::min(S, need);
    S = (S + kGroup - 1) / kGroup * kGroup;
    return static_cast<int>(std::max<long long>(S, kGroup));
}

std::string validate_options(const jbp_options &o, double p) {
    if (o.max_iter < 1) return "max_iter must be >= 1";
    if (o.precision < JBP_PREC_FP64 || o.precision > JBP_PREC_FP16) return "unknown precision";
    if (o.use_prior) {
        for (int i = 0; i < 4; ++i)
            if (!(o.prior[i] >= 0.0 && o.prior[i] <= 1.0)) return "prior entries must be in [0, 1]";
    } else if (!(p > 0.0 && p < 1.0)) {
        return "p must be in (0, 1)";
    }
    if (o.damping < 0.0 || o.damping > 1.0) return "damping must be in [0, 1]";
    if (o.p_max > p && !(o.p_max < 1.0)) return "p_max must be below 1";
    if (o.engine < JBP_ENGINE_AUTO || o.engine > JBP_ENGINE_TABLE) return "unknown engine";
    if (o.watchdog_ms < 0) return "watchdog_ms must be >= 0";
    if (o.learned_order < 0 || o.learned_order > 1) return "learned_order must be 0 (model) or 1 (|LLR|)";
    if (o.learned_cols < 0) return "learned_cols must be >= 0";
    if (o.collect_every < 0) return "collect_every must be >= 0";
    return "";
}

// A request to abort applies to the run in progress (or the next run): it is cleared when that
// run returns, on every path.
std::string Engine::run(const RunRequest &rq, jbp_stats &stats) {
    std::string e = run_dispatch(rq, stats);
    clear_abort();
    return e;
}

std::string Engine::run_mixed(const MixedRequest &rq, std::vector<jbp_stats> &stats) {
    std::string e = run_mixed_impl(rq, stats);
    for (Engine *eng : rq.engines)
        if (eng) eng->clear_abort();
    return e;
}

std::string Engine::run_dispatch(const RunRequest &rq, jbp_stats &stats) {
    std::memset(&stats, 0, sizeof(stats));
    const jbp_options &o = rq.opt;
    if (rq.ntrials <= 0) return "";
    if (std::string bad = validate_options(o, rq.p); !bad.empty()) return bad;
    if (o.engine == JBP_ENGINE_TABLE) {
        if ((rq.source != kSrcPhilox && rq.source != kSrcErrors) || rq.collect)
            return "the table engine is not available for syndrome inputs or the mt19937 sampler "
                   "(it decodes Philox Monte Carlo and given errors)";
        MixedRequest mr;
        mr.engines = {this};
        mr.opt = o;
        mr.seeds = {rq.seed};
        mr.first_trial = {rq.first_trial};
        mr.ntrials = {rq.ntrials};
        mr.p = rq.p;
        mr.d_res = {rq.d_res_out};
        mr.d_hist = {rq.d_hist};
        mr.d_err = {rq.source == kSrcErrors ? rq.d_err : nullptr};
        mr.d_est = {rq.d_est_out};
        mr.d_llr = {rq.d_llr_out};
        mr.stream = rq.stream;
        std::vector<jbp_stats> st;
        std::string e = run_mixed_impl(mr, st);
        if (!st.empty()) stats = st[0];   // also on a run-budget stop: the trials that finished
        return e;
    }
    if (o.engine != JBP_ENGINE_SLOTS) {
        std::string why;
        if (resident_applies(o, &why)) return run_resident(rq, stats);
        if (o.engine == JBP_ENGINE_RESIDENT || o.learned_from > 0 || rq.collect)
            return "resident engine not available: " + why;
    }
    if (o.learned_from > 0 || rq.collect) return "learned flip proposals are not available on the slot engine";
    const SideGraph &gx = model_.side[0], &gz = model_.side[1];
    if (!gx.checks_regular || !gz.checks_regular || gx.dc_max != gz.dc_max || gx.dv_max != gz.dv_max)
        return "the GPU kernels need a code whose checks all have one degree and whose sides have equal degrees";
    const bool pp = o.enable_pp != 0;
    if (pp && (o.check_interval != 1 || o.check_warmup != 0))
        return "post-processing needs a syndrome test every iteration (check interval 1, warmup 0)";
    const bool damp = o.damping > 0.0;
    KernelSet ks;
    if (!select_kernels(gx.dc_max, gx.dv_max, o.precision, damp, ks))
        return "no GPU kernel built for check degree " + std::to_string(gx.dc_max) + " / variable degree " +
               std::to_string(gx.dv_max);
    JBP_CUDA_TRY(cudaSetDevice(device_), "cudaSetDevice");
    if (ks.single && single_applies(rq) && single_fits(reinterpret_cast<const void *>(ks.single)))
        return run_single(rq, stats);
    const int S = choose_slots(o, rq.ntrials);
    const int H = std::max(0, o.flip_hist);
    const int R = pp ? std::max(H + 1, 3) : 1;
    if (pp) {
        const int mmax = std::max(gx.m, gz.m);
        const size_t smem = pp_smem_bytes(model_.n, gx.m + gz.m, mmax);
        if (smem > 200 * 1024) return "code too large for GPU post-processing";
        JBP_CUDA_TRY(cudaFuncSetAttribute(k_postprocess, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(smem)), "smem attribute");
        std::string ee = upload_ets();
        if (!ee.empty()) return ee;
    }
    std::string e = ensure_buffers(S, o.precision, damp, pp, R, rq.stream);
    if (!e.empty()) return e;

    cudaStream_t st = rq.stream;
    const int n = model_.n, M = gx.m + gz.m;
    DevRun r{};
    r.S = S;
    r.max_iter = o.max_iter;
    r.check_warmup = std::max(0, o.check_warmup);
    r.check_interval = std::max(1, o.check_interval);
    r.source = rq.source;
    r.p = rq.p;
    r.p_max = o.p_max;
    r.slot_p = buf_.slot_p;
    r.seed = rq.seed;
    r.first_trial = rq.first_trial;
    r.ntrials = rq.ntrials;
    r.src_err = rq.d_err;
    r.src_sx = rq.d_sx;
    r.src_sz = rq.d_sz;
    r.est_out = rq.d_est_out;
    r.llr_out = rq.d_llr_out;
    r.res_out = rq.d_res_out;
    r.hist = rq.d_hist;
    r.trial = buf_.trial;
    r.iter = buf_.iter;
    r.flags = buf_.flags;
    r.freeze_syn = o.freeze_syn ? 1 : 0;
    r.frz = buf_.frz;
    r.use_prior = o.use_prior ? 1 : 0;
    for (int i = 0; i < 4; ++i) r.prior4[i] = o.prior[i];
    r.unsat = buf_.unsat;
    r.prior = buf_.prior;
    r.lprior = buf_.lprior;
    r.err = buf_.err;
    r.estx = buf_.estx;
    r.estz = buf_.estz;
    r.synm = buf_.synm;
    r.unsat_mask = buf_.unsat_mask;
    r.res_iters = buf_.res_iters;
    r.res_flags = buf_.res_flags;
    r.retired = buf_.lists;
    r.fresh = buf_.lists + S;
    r.groups = buf_.lists + 2 * S;
    r.n_retired = buf_.counts;
    r.n_fresh = buf_.counts + 1;
    r.n_groups = buf_.counts + 2;
    r.cnt = buf_.cnt;
    r.R = R;
    r.it = buf_.it;
    r.pp = pp ? 1 : 0;
    r.flip_hist = H;
    r.llr_from = std::min(100, o.max_iter);
    if (pp) {
        r.act_k = buf_.act_k;
        r.pstate = buf_.pstate;
        r.stall_same = buf_.stall_same;
        r.us_hist = buf_.us_hist;
        r.dprev = buf_.dprev;
        r.dpprev = buf_.dpprev;
        r.pp_list = buf_.pp_list;
        r.n_pp = buf_.counts + 3;
        r.pp_mode = buf_.pp_mode;
        r.ets = dets_;
        r.pp_scratch = buf_.pp_scratch;
        r.pp_scratch_stride = buf_.pp_stride;
    }
    DevMsgs msg{};
    for (int s = 0; s < 2; ++s) {
        msg.c2v[s] = buf_.msg[s];
        msg.v2c[s] = buf_.msg[2 + s];
        msg.v2c_hi[s] = buf_.msg[4 + s];
    }

    // launch shapes
    const int tpb = 256;
    const int big_grid = sm_count_ * 8;                         // grid-stride message kernels
    const int slot_blocks = (S / kGroup + (tpb / 32) - 1) / (tpb / 32);
    const int classify_tpb = 128;
    const size_t classify_smem = static_cast<size_t>(classify_tpb / 32) * 2 * dcode_.words * sizeof(uint64_t);
    if (classify_smem > 48 * 1024) {
        JBP_CUDA_TRY(cudaFuncSetAttribute(k_classify, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(classify_smem)), "smem attribute");
    }
    const int list_grid = std::max(1, std::min((S + tpb - 1) / tpb, sm_count_ * 4));
    const int sample_grid = sm_count_ * 4;
    long long launches = 0;

    if (!run_ev_[0]) {
        for (int i = 0; i < 2; ++i) JBP_CUDA_TRY(cudaEventCreate(&run_ev_[i]), "cudaEventCreate");
        for (int i = 2; i < 4; ++i)
            JBP_CUDA_TRY(cudaEventCreateWithFlags(&run_ev_[i], cudaEventDisableTiming), "cudaEventCreate");
    }
    cudaEvent_t ev0 = run_ev_[0], ev1 = run_ev_[1];
    cudaEvent_t poll_ev[2] = {run_ev_[2], run_ev_[3]};

    auto enqueue_refill = [&](cudaStream_t s) {
        cudaMemsetAsync(r.n_fresh, 0, sizeof(int), s);
        k_refill<<<list_grid, tpb, 0, s>>>(r, o.precision);
        if (rq.source == kSrcMt19937) k_sample_mt<<<sample_grid, 256, 0, s>>>(dcode_, r);
        else if (rq.source != kSrcSyndromes) k_sample<<<sample_grid, tpb, 0, s>>>(dcode_, r);
        k_fresh_syndrome<<<sample_grid, tpb, 0, s>>>(dcode_, r);
        cudaMemsetAsync(r.n_groups, 0, sizeof(int), s);
        k_groups<<<slot_blocks, tpb, 0, s>>>(r);
        launches += rq.source == kSrcSyndromes ? 3 : 4;
    };
    auto enqueue_iteration = [&](cudaStream_t s, cudaEvent_t *e3) {
        if (e3) cudaEventRecordWithFlags(e3[0], s, cudaEventRecordExternal);
        ks.check<<<big_grid, tpb, 0, s>>>(dcode_, r, msg);
        if (e3) cudaEventRecordWithFlags(e3[1], s, cudaEventRecordExternal);
        if (o.precision == JBP_PREC_FP64) ks.var64<<<big_grid, tpb, 0, s>>>(dcode_, r, msg, o.damping);
        else ks.varllr<<<big_grid, tpb, 0, s>>>(dcode_, r, msg, static_cast<float>(o.damping));
        if (e3) cudaEventRecordWithFlags(e3[2], s, cudaEventRecordExternal);
        if (pp) {
            k_stall_compare<<<big_grid, tpb, 0, s>>>(dcode_, r);
            launches += 1;
        }
        if (e3) cudaEventRecordWithFlags(e3[3], s, cudaEventRecordExternal);
        k_syndrome_check<<<big_grid, tpb, 0, s>>>(dcode_, r);
        if (e3) cudaEventRecordWithFlags(e3[4], s, cudaEventRecordExternal);
        cudaMemsetAsync(r.n_retired, 0, sizeof(int), s);
        if (pp) cudaMemsetAsync(r.n_pp, 0, sizeof(int), s);
        k_retire<<<slot_blocks, tpb, 0, s>>>(r);
        if (pp) {
            k_postprocess<<<buf_.pp_blocks, kPpThreads,
                            pp_smem_bytes(n, M, std::max(gx.m, gz.m)), s>>>(dcode_, r, msg, o.precision);
            launches += 1;
        }
        if (rq.d_llr_out) {
            if (o.precision == JBP_PREC_FP64) k_llr_out<double2><<<sm_count_ * 2, 256, 0, s>>>(dcode_, r, msg);
            else if (o.precision == JBP_PREC_FP32) k_llr_out<float><<<sm_count_ * 2, 256, 0, s>>>(dcode_, r, msg);
            else k_llr_out<__half><<<sm_count_ * 2, 256, 0, s>>>(dcode_, r, msg);
            launches += 1;
        }
        k_classify<<<sm_count_ * 2, classify_tpb, classify_smem, s>>>(dcode_, r);
        launches += 5;
        enqueue_refill(s);
    };

    JBP_CUDA_TRY(cudaEventRecord(ev0, st), "cudaEventRecord");
    JBP_CUDA_TRY(cudaMemsetAsync(buf_.cnt, 0, sizeof(DevCounters), st), "memset counters");
    JBP_CUDA_TRY(cudaMemsetAsync(buf_.it, 0, sizeof(int), st), "memset it");
    k_init_slots<<<list_grid, tpb, 0, st>>>(r);
    launches += 1;
    enqueue_refill(st);
    JBP_CUDA_TRY(cudaGetLastError(), "initial launches");

    // CUDA graph of GI iterations.  With profiling on, every captured iteration also records
    // event nodes around the check and variable kernels; two graph instances alternate so
    // that the events of a finished graph are read while the next one runs.
    int GI = o.iters_per_launch > 0 ? o.iters_per_launch : 4;
    GI = std::min(GI, o.max_iter);
    const bool prof = o.profile != 0;
    // Without profiling (events) or a run budget (a host check between launches), the whole run
    // is one launch: a graph whose while node repeats one BP iteration until every trial is
    // classified (k_loop_cond), so the host neither polls nor launches graphs that find nothing
    // left to do -- what a one-trial call (cuda_bp_decode) spends most of its time on otherwise.
    const bool device_loop = !prof && o.watchdog_ms <= 0;
    if (device_loop) GI = 1;
    const long long max_iters_total =
        (rq.ntrials * static_cast<long long>(o.max_iter)) / std::max(1, S) + 2LL * o.max_iter + 2 * GI + 8;
    const int nsets = prof ? 2 : 1;
    // events per iteration: before the check kernel, before the variable kernel, after it, and
    // around the syndrome-test kernel
    constexpr int kEv = 5;
    std::vector<cudaEvent_t> pev(prof ? 2 * GI * kEv : 0);
    for (auto &ev : pev) JBP_CUDA_TRY(cudaEventCreate(&ev), "cudaEventCreate");
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    const long long launches_before = launches;
    long long per_graph = 0;
    cudaError_t ce = cudaSuccess;
    // reuse the last run's graph when every launch parameter is the same
    SlotGraph &sg = slot_graph_;
    const bool reuse = !prof && sg.valid && sg.precision == o.precision && sg.damping == o.damping && sg.GI == GI &&
                       sg.device_loop == device_loop && sg.llr_out == (rq.d_llr_out != nullptr) &&
                       std::memcmp(&sg.r, &r, sizeof(DevRun)) == 0 && std::memcmp(&sg.msg, &msg, sizeof(DevMsgs)) == 0;
    cudaStream_t cap = nullptr;
    if (reuse) {
        exec[0] = sg.exec;
        per_graph = sg.per_graph;
    } else {
        JBP_CUDA_TRY(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "cudaStreamCreate");
    }
    if (!reuse && device_loop) {
        // graph = while(cond) { one iteration; k_loop_cond }
        cudaGraph_t g = nullptr;
        cudaGraphConditionalHandle h{};
        ce = cudaGraphCreate(&g, 0);
        if (ce == cudaSuccess) ce = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
        cudaGraphNodeParams np{};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t wn = nullptr;
        if (ce == cudaSuccess) ce = cudaGraphAddNode(&wn, g, nullptr, 0, &np);
        if (ce == cudaSuccess) {
            cudaGraph_t body = np.conditional.phGraph_out[0];
            launches = launches_before;
            ce = cudaStreamBeginCaptureToGraph(cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
            if (ce == cudaSuccess) {
                enqueue_iteration(cap, nullptr);
                k_loop_cond<<<1, 32, 0, cap>>>(h, r.cnt, r.it, static_cast<unsigned long long>(rq.ntrials),
                                               static_cast<int>(std::min<long long>(max_iters_total + 2, 1 << 30)),
                                               abort_dev_);
                launches += 1;
                cudaGraph_t captured = nullptr;
                ce = cudaStreamEndCapture(cap, &captured);
            }
            per_graph = launches - launches_before;   // kernels per iteration
        }
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec[0], g, 0);
        if (g) cudaGraphDestroy(g);
    }
    for (int set = 0; set < nsets && ce == cudaSuccess && !reuse && !device_loop; ++set) {
        launches = launches_before;
        ce = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
        if (ce != cudaSuccess) break;
        for (int i = 0; i < GI; ++i) {
            cudaEvent_t *e3 = prof ? &pev[(set * GI + i) * kEv] : nullptr;
            enqueue_iteration(cap, e3);
        }
        ce = cudaStreamEndCapture(cap, &graph[set]);
        if (ce == cudaSuccess) ce = cudaGraphInstantiate(&exec[set], graph[set], 0);
        per_graph = launches - launches_before;
    }
    if (!reuse && !prof && ce == cudaSuccess) {
        // keep this graph for the next run with the same parameters
        if (sg.exec) cudaGraphExecDestroy(sg.exec);
        sg.valid = true;
        sg.r = r;
        sg.msg = msg;
        sg.precision = o.precision;
        sg.damping = o.damping;
        sg.GI = GI;
        sg.device_loop = device_loop;
        sg.llr_out = rq.d_llr_out != nullptr;
        sg.exec = exec[0];
        sg.per_graph = per_graph;
    }
    launches = launches_before;
    double check_ms = 0.0, var_ms = 0.0, test_ms = 0.0;
    long long prof_iters = 0;
    auto read_profile = [&](long long gidx) {
        if (!prof) return;
        const int set = static_cast<int>(gidx & 1);
        for (int i = 0; i < GI; ++i) {
            float a = 0.0f, b = 0.0f;
            float c = 0.0f;
            cudaEvent_t *e3 = &pev[(set * GI + i) * kEv];
            if (cudaEventElapsedTime(&a, e3[0], e3[1]) == cudaSuccess &&
                cudaEventElapsedTime(&b, e3[1], e3[2]) == cudaSuccess &&
                cudaEventElapsedTime(&c, e3[3], e3[4]) == cudaSuccess) {
                test_ms += c;
                check_ms += a;
                var_ms += b;
                prof_iters++;
            }
        }
    };

    const long long max_graphs = max_iters_total / GI + 2;
    auto t0 = std::chrono::steady_clock::now();
    std::string err;
    bool timed_out = false, aborted = false;
    if (ce != cudaSuccess) err = cuda_err(ce, "graph capture");
    long long g = 0;
    bool finished = false;
    if (device_loop && err.empty()) {
        // one launch; the iterations it ran are read back with the completion count
        int *h_it = reinterpret_cast<int *>(&buf_.h_done[1]);
        ce = cudaGraphLaunch(exec[0], st);
        if (ce == cudaSuccess)
            ce = cudaMemcpyAsync(&buf_.h_done[0], &buf_.cnt->done, sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 st);
        if (ce == cudaSuccess) ce = cudaMemcpyAsync(h_it, buf_.it, sizeof(int), cudaMemcpyDeviceToHost, st);
        if (ce == cudaSuccess) ce = cudaEventRecord(poll_ev[0], st);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(poll_ev[0]);
        if (ce != cudaSuccess) {
            err = cuda_err(ce, "run");
        } else {
            launches += per_graph * std::max(0, *h_it - 1);
            finished = buf_.h_done[0] >= static_cast<unsigned long long>(rq.ntrials);
            if (!finished && abort_requested()) aborted = true;   // k_loop_cond saw the flag
            else if (!finished) err = "run did not complete within the iteration bound (internal error)";
        }
        g = max_graphs;   // the polling loop below has nothing to do
    }
    for (; err.empty() && g < max_graphs && !finished; ++g) {
        ce = cudaGraphLaunch(exec[g % nsets], st);
        if (ce != cudaSuccess) { err = cuda_err(ce, "graph launch"); break; }
        launches += per_graph;
        cudaMemcpyAsync(&buf_.h_done[g & 1], &buf_.cnt->done, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
        cudaEventRecord(poll_ev[g & 1], st);
        if (g >= 1) {
            ce = cudaEventSynchronize(poll_ev[(g - 1) & 1]);
            if (ce != cudaSuccess) { err = cuda_err(ce, "run"); break; }
            read_profile(g - 1);
            if (buf_.h_done[(g - 1) & 1] >= static_cast<unsigned long long>(rq.ntrials)) finished = true;
        }
        if (o.watchdog_ms > 0) {
            double wall = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
            if (wall > o.watchdog_ms) {
                // the graphs already launched finish; the counters below say how far the run got
                timed_out = true;
                break;
            }
        }
        if (!finished && abort_requested()) {
            aborted = true;
            break;
        }
    }
    if (err.empty() && !finished && !timed_out && !aborted && g >= 1 && !device_loop) {
        ce = cudaEventSynchronize(poll_ev[(g - 1) & 1]);
        if (ce == cudaSuccess && buf_.h_done[(g - 1) & 1] >= static_cast<unsigned long long>(rq.ntrials)) finished = true;
        if (!finished) err = "run did not complete within the iteration bound (internal error)";
    }
    cudaEventRecord(ev1, st);
    ce = cudaEventSynchronize(ev1);
    if (err.empty() && ce != cudaSuccess) err = cuda_err(ce, "run");
    if (err.empty() && g >= 1 && prof) read_profile(g - 1);
    if (err.empty()) {
        ce = cudaGetLastError();
        if (ce != cudaSuccess) err = cuda_err(ce, "run");
    }
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ev0, ev1);
    DevCounters hc{};
    if (err.empty()) {
        ce = cudaMemcpy(&hc, buf_.cnt, sizeof(hc), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) err = cuda_err(ce, "read counters");
    }
    const bool timeout_err = err.empty() && timed_out && hc.done < static_cast<unsigned long long>(rq.ntrials);
    if (timeout_err)
        err = "watchdog expired: the run budget of " + std::to_string(o.watchdog_ms) + " ms ran out (host check) after " +
              std::to_string(hc.done) + " of " + std::to_string(rq.ntrials) + " trials";
    const bool abort_err = err.empty() && aborted && hc.done < static_cast<unsigned long long>(rq.ntrials);
    if (abort_err)
        err = "aborted by request after " + std::to_string(hc.done) + " of " + std::to_string(rq.ntrials) + " trials";
    for (int set = 0; set < 2; ++set) {
        if (exec[set] && !(sg.valid && exec[set] == sg.exec)) cudaGraphExecDestroy(exec[set]);
        if (graph[set]) cudaGraphDestroy(graph[set]);
    }
    for (auto &ev : pev) cudaEventDestroy(ev);
    if (cap) cudaStreamDestroy(cap);
    if (!err.empty() && !timeout_err && !abort_err) return err;
    if (hc.bad_input) return "error vector has invalid value";
    fill_stats(hc, stats);
    stats.device_ms = ms;
    stats.kernel_launches = launches;
    stats.check_ms = check_ms;
    stats.var_ms = var_ms;
    stats.test_ms = test_ms;
    stats.profiled_iterations = prof_iters;
    stats.slots = S;
    if (!err.empty()) return err;
    (void)n;
    (void)M;
    return "";
}

std::string Engine::sample_errors(unsigned long long seed, long long first, long long count, double p, int source,
                                  uint8_t *d_out) {
    if (count <= 0) return "";
    if (!(p > 0.0 && p < 1.0)) return "p must be in (0, 1)";
    JBP_CUDA_TRY(cudaSetDevice(device_), "cudaSetDevice");
    k_sample_out<<<sm_count_ * 4, 256>>>(model_.n, seed, first, count, p, source, d_out);
    JBP_CUDA_TRY(cudaGetLastError(), "sample launch");
    JBP_CUDA_TRY(cudaStreamSynchronize(nullptr), "sample");
    return "";
}


// ---------------------------------------------------------------- mixed-size launch

std::string Engine::mixed_slots() {
    if (mix_slot_[0] && mix_slot_[1]) return "";
    // both sides' tables are published together, only when every upload succeeded (a failed
    // upload leaves none set, and the next call builds them again)
    uint16_t *slot_tab[2] = {nullptr, nullptr}, *chk_tab[2] = {nullptr, nullptr};
    for (int s = 0; s < 2; ++s) {
        const SideGraph &g = model_.side[s];
        const int dv = std::max(1, g.dv_max), dc = g.dc_max, m = g.m, n = model_.n;
        if (n > 65535 || static_cast<long long>(dc) * m > 65535)
            return "codes above 65,535 variables or message slots per side are not available in the mixed launch";
        // variable -> c2v slot, k-major; check -> variable, i-major (both 16-bit, read coalesced)
        std::vector<uint16_t> sl(static_cast<size_t>(n) * dv, static_cast<uint16_t>(kMixNone)),
            ck(static_cast<size_t>(m) * dc);
        for (int v = 0; v < n; ++v)
            for (int k = g.var_off[v]; k < g.var_off[v + 1]; ++k) {
                const int e = g.var_edge[k], c = e / dc, pos = e - c * dc;
                sl[static_cast<size_t>(k - g.var_off[v]) * n + v] = static_cast<uint16_t>(pos * m + c);
            }
        for (int c = 0; c < m; ++c)
            for (int i = 0; i < dc; ++i)
                ck[static_cast<size_t>(i) * m + c] = static_cast<uint16_t>(g.chk_var[static_cast<size_t>(c) * dc + i]);
        std::string e = dev_upload(code_allocs_, sl, &slot_tab[s]);
        if (e.empty()) e = dev_upload(code_allocs_, ck, &chk_tab[s]);
        if (!e.empty()) return e;
    }
    for (int s = 0; s < 2; ++s) {
        mix_slot_[s] = slot_tab[s];
        mix_chk_[s] = chk_tab[s];
    }
    return "";
}

namespace {
template <int DC>
void *mixed_kernel(int precision) {
    return precision == JBP_PREC_FP16 ? reinterpret_cast<void *>(k_mixed<DC, StoreHalf>)
                                      : reinterpret_cast<void *>(k_mixed<DC, StoreFloat>);
}
}  // namespace

std::string Engine::run_mixed_impl(const MixedRequest &rq, std::vector<jbp_stats> &stats) {
    const int nc = static_cast<int>(rq.engines.size());
    stats.assign(static_cast<size_t>(std::max(nc, 0)), jbp_stats{});
    for (jbp_stats &s : stats) std::memset(&s, 0, sizeof(s));
    if (nc < 1 || nc > kMixMaxCodes) return "the mixed launch takes 1 to 8 codes";
    if (rq.seeds.size() != static_cast<size_t>(nc) || rq.ntrials.size() != static_cast<size_t>(nc) ||
        rq.first_trial.size() != static_cast<size_t>(nc))
        return "one seed, first trial and trial count per code";
    const jbp_options &o = rq.opt;
    if (o.precision != JBP_PREC_FP32 && o.precision != JBP_PREC_FP16)
        return "FP64 is not available in the mixed launch (FP32 arithmetic: precision FP32, or FP16 storage)";
    if (o.enable_pp) return "post-processing is not available in the mixed launch (plain BP)";
    if (o.damping > 0.0 || o.freeze_syn || o.learned_from > 0)
        return "damping, freeze-syn and the learned proposal are not available in the mixed launch";
    if (o.max_iter < 1) return "max_iter must be >= 1";
    if (o.use_prior) {
        for (int i = 0; i < 4; ++i)
            if (!(o.prior[i] >= 0.0 && o.prior[i] <= 1.0)) return "prior entries must be in [0, 1]";
    } else if (!(rq.p > 0.0 && rq.p < 1.0)) {
        return "p must be in (0, 1)";
    }
    if (o.p_max > rq.p && !(o.p_max < 1.0)) return "p_max must be below 1";
    Engine &e0 = *rq.engines[0];
    const int DC = e0.model_.side[0].dc_max;
    for (Engine *e : rq.engines) {
        if (!e || e->device_ != e0.device_) return "the codes of a mixed launch must be on one device";
        for (int s = 0; s < 2; ++s) {
            if (!e->model_.side[s].checks_regular || e->model_.side[s].dc_max != DC)
                return "the codes of a mixed launch need a code-wide check degree, the same for every code";
            if (e->model_.side[s].dv_max > kMixMaxDv)
                return "variable degrees above 4 are not available in the mixed launch";
        }
    }
    void *kern = DC == 6    ? mixed_kernel<6>(o.precision)
                 : DC == 7  ? mixed_kernel<7>(o.precision)
                 : DC == 8  ? mixed_kernel<8>(o.precision)
                 : DC == 12 ? mixed_kernel<12>(o.precision)
                            : nullptr;
    if (!kern) return "check degrees other than 6, 7, 8 and 12 are not available in the mixed launch";
    JBP_CUDA_TRY(cudaSetDevice(e0.device_), "cudaSetDevice");
    cudaFuncAttributes fa{};
    JBP_CUDA_TRY(cudaFuncGetAttributes(&fa, kern), "kernel attributes");
    const size_t limit = static_cast<size_t>(e0.smem_optin_) - fa.sharedSizeBytes;
    const size_t es = o.precision == JBP_PREC_FP16 ? 2 : 4;
    // largest codes first: the launch's tail is made of the shortest trials
    std::vector<int> order(nc);
    for (int i = 0; i < nc; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return rq.engines[a]->model_.n > rq.engines[b]->model_.n; });
    size_t smem = 0, scratch = 0;
    std::vector<size_t> base(nc), full(nc);
    for (int i = 0; i < nc; ++i) {
        const CodeModel &m = rq.engines[i]->model_;
        base[i] = mix_state_bytes(m.n, m.side[0].m, m.side[1].m);
        full[i] = base[i] + mix_c2v_bytes(m.side[0].m, m.side[1].m, DC, es);
        if (base[i] > limit) return "a code of the mixed launch is too large for one block's shared memory";
        if (full[i] - base[i] < 16ull * ((m.n + 63) / 64))
            return "codes with fewer check edges than 2 bits per variable are not available in the mixed launch";
        smem = std::max(smem, full[i] <= limit ? full[i] : base[i]);
    }
    for (int i = 0; i < nc; ++i)
        if (full[i] > smem) scratch = std::max(scratch, (full[i] - base[i] + 255) / 256 * 256);
    JBP_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)),
                 "smem attribute");
    int per_sm = 0;
    JBP_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kMixThreads, smem), "occupancy");
    if (per_sm < 1) return "the mixed kernel does not fit on an SM";
    long long total = 0;
    for (int i = 0; i < nc; ++i) {
        if (rq.ntrials[i] < 0) return "invalid trial count";
        total += rq.ntrials[i];
    }
    if (total == 0) return "";
    const int grid = static_cast<int>(std::min<long long>(static_cast<long long>(per_sm) * e0.sm_count_, total));
    if (scratch * grid > e0.mix_scratch_bytes_) {
        cudaFree(e0.mix_scratch_);
        e0.mix_scratch_ = nullptr;
        e0.mix_scratch_bytes_ = 0;
        JBP_CUDA_TRY(dev_malloc(&e0.mix_scratch_, scratch * grid), "cudaMalloc(mixed scratch)");
        e0.mix_scratch_bytes_ = scratch * grid;
    }
    if (!e0.mix_cnt_) JBP_CUDA_TRY(dev_malloc(&e0.mix_cnt_, sizeof(DevCounters) * (kMixMaxCodes + 1)),
                                   "cudaMalloc(mixed counters)");
    MixRun r{};
    r.ncodes = nc;
    r.next = reinterpret_cast<unsigned long long *>(e0.mix_cnt_ + kMixMaxCodes);
    r.max_iter = o.max_iter;
    r.check_warmup = std::max(0, o.check_warmup);
    r.check_interval = std::max(1, o.check_interval);
    r.p = rq.p;
    r.p_max = o.p_max;
    r.use_prior = o.use_prior ? 1 : 0;
    for (int i = 0; i < 4; ++i) r.prior4[i] = o.prior[i];
    r.scratch = e0.mix_scratch_;
    r.scratch_stride = scratch;
    r.budget_ns = o.watchdog_ms > 0 ? static_cast<unsigned long long>(o.watchdog_ms) * 1000000ull : 0ull;
    r.abort_flag = e0.abort_dev_;
    long long end = 0;
    for (int k = 0; k < nc; ++k) {
        const int i = order[k];
        Engine &e = *rq.engines[i];
        std::string err = e.mixed_slots();
        if (!err.empty()) return err;
        MixCode &mc = r.code[k];
        mc.dc = e.dcode_;
        mc.slot[0] = e.mix_slot_[0];
        mc.slot[1] = e.mix_slot_[1];
        mc.chk[0] = e.mix_chk_[0];
        mc.chk[1] = e.mix_chk_[1];
        mc.seed = rq.seeds[i];
        mc.first_trial = rq.first_trial[i];
        mc.ntrials = rq.ntrials[i];
        end += rq.ntrials[i];
        mc.item_end = end;
        mc.cnt = e0.mix_cnt_ + k;
        mc.res_out = i < static_cast<int>(rq.d_res.size()) ? rq.d_res[i] : nullptr;
        mc.hist = i < static_cast<int>(rq.d_hist.size()) ? rq.d_hist[i] : nullptr;
        mc.src_err = i < static_cast<int>(rq.d_err.size()) ? rq.d_err[i] : nullptr;
        mc.est_out = i < static_cast<int>(rq.d_est.size()) ? rq.d_est[i] : nullptr;
        mc.llr_out = i < static_cast<int>(rq.d_llr.size()) ? rq.d_llr[i] : nullptr;
        mc.c2v_in_smem = full[i] <= smem ? 1 : 0;
    }
    cudaStream_t st = rq.stream;
    cudaEvent_t ev0, ev1;
    JBP_CUDA_TRY(cudaEventCreate(&ev0), "cudaEventCreate");
    JBP_CUDA_TRY(cudaEventCreate(&ev1), "cudaEventCreate");
    cudaError_t ce = cudaEventRecord(ev0, st);
    if (ce == cudaSuccess) ce = cudaMemsetAsync(e0.mix_cnt_, 0, sizeof(DevCounters) * (kMixMaxCodes + 1), st);
    if (ce == cudaSuccess) {
        void *args[] = {&r};
        ce = cudaLaunchKernel(kern, dim3(grid), dim3(kMixThreads), args, smem, st);
    }
    if (ce == cudaSuccess) ce = cudaEventRecord(ev1, st);
    if (ce == cudaSuccess) ce = cudaEventSynchronize(ev1);
    std::vector<DevCounters> hc(kMixMaxCodes);
    if (ce == cudaSuccess)
        ce = cudaMemcpy(hc.data(), e0.mix_cnt_, sizeof(DevCounters) * kMixMaxCodes, cudaMemcpyDeviceToHost);
    float ms = 0.0f;
    if (ce == cudaSuccess) cudaEventElapsedTime(&ms, ev0, ev1);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (ce != cudaSuccess) return cuda_err(ce, "mixed run");
    for (int k = 0; k < nc; ++k)
        if (hc[k].bad_input) return "error vector has invalid value";
    long long done = 0;
    for (int k = 0; k < nc; ++k) {
        const int i = order[k];
        fill_stats(hc[k], stats[i]);
        stats[i].device_ms = ms;
        stats[i].kernel_launches = 1;
        stats[i].slots = grid;
        done += static_cast<long long>(hc[k].done);
    }
    if (hc[0].watchdog)
        return "watchdog expired: the run budget of " + std::to_string(o.watchdog_ms) + " ms ran out on the device after " +
               std::to_string(done) + " of " + std::to_string(total) + " trials";
    if (hc[0].aborted)
        return "aborted by request after " + std::to_string(done) + " of " + std::to_string(total) + " trials";
    for (int k = 0; k < nc; ++k)
        if (hc[k].done != static_cast<unsigned long long>(rq.ntrials[order[k]]))
            return "mixed run finished an unexpected number of trials";
    return "";
}

}  // namespace jbp
