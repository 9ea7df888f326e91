// C ABI (include/jbp_b200.h) over the batched engine.
#include <algorithm>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "../../include/jbp_b200.h"
#include "ctx.hpp"
#include "engine.hpp"
#include "mlp.cuh"

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

// Statuses whose jbp_stats hold the trials that finished before the run stopped.
bool partial_stats(int rc) { return rc == JBP_ERR_TIMEOUT || rc == JBP_ERR_ABORTED; }

int engine_fail(const std::string &msg) {
    if (msg.find("not available") != std::string::npos || msg.find("no GPU kernel") != std::string::npos ||
        msg.find("need a code") != std::string::npos)
        return fail(JBP_ERR_UNSUPPORTED, msg);
    if (msg.find("watchdog") != std::string::npos) return fail(JBP_ERR_TIMEOUT, msg);
    if (msg.find("aborted by request") != std::string::npos) return fail(JBP_ERR_ABORTED, msg);
    if (msg.find(':') != std::string::npos && msg.find("must") == std::string::npos) return fail(JBP_ERR_CUDA, msg);
    return fail(JBP_ERR_ARG, msg);
}

template <typename T>
int grow(T **p, size_t *have, size_t need) {
    if (*have >= need && *p) return JBP_OK;
    cudaFree(*p);
    *p = nullptr;
    *have = 0;
    cudaError_t e = jbp::dev_malloc(reinterpret_cast<void **>(p), std::max<size_t>(need, 1) * sizeof(T));
    if (e != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(e, "cudaMalloc(staging)"));
    *have = need;
    return JBP_OK;
}

jbp_options normalized(const jbp_options *opt) {
    jbp_options o;
    jbp_default_options(&o);
    if (opt) o = *opt;
    if (o.flip_hist < 0) o.flip_hist = 0;
    if (o.check_warmup < 0) o.check_warmup = 0;
    if (o.check_interval <= 0) o.check_interval = 1;
    return o;
}

int finish_create(jbp::CodeModel &&m, const std::string &ets_dir, int device, jbp_ctx **out) {
    if (!ets_dir.empty()) {
        std::string e = m.load_ets_dir(ets_dir);
        if (!e.empty()) return fail(JBP_ERR_IO, e);
    }
    auto ctx = std::make_unique<jbp_ctx>();
    std::string e = ctx->engine.init(std::move(m), device);
    if (!e.empty()) return fail(JBP_ERR_CUDA, e);
    cudaError_t ce = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "cudaStreamCreate"));
    *out = ctx.release();
    return JBP_OK;
}

}  // namespace

int jbp::set_last_error(int code, const std::string &msg) { return fail(code, msg); }

extern "C" {

void jbp_default_options(jbp_options *o) {
    std::memset(o, 0, sizeof(*o));
    o->precision = JBP_PREC_FP64;
    o->max_iter = 50;
    o->damping = 0.0;
    o->flip_hist = 5;
    o->enable_pp = 1;
    o->freeze_syn = 0;
    o->check_warmup = 0;
    o->check_interval = 1;
    o->slots = 0;
    o->iters_per_launch = 0;
    o->watchdog_ms = 0;
    o->profile = 0;
}

const char *jbp_last_error(void) { return g_last_error.c_str(); }

const char *jbp_version(void) { return "jbp_b200 0.1 (sm_100a)"; }

int jbp_request_abort(jbp_ctx *ctx) {
    if (!ctx) return fail(JBP_ERR_ARG, "null context");
    ctx->engine.request_abort();
    return JBP_OK;
}

int jbp_debug_fail_allocation(long long after) {
    jbp::set_alloc_failure(after);
    return JBP_OK;
}

int jbp_create_from_params(const char *params_path, const char *ets_dir, int device, jbp_ctx **out) {
    if (!params_path || !out) return fail(JBP_ERR_ARG, "null argument");
    *out = nullptr;
    jbp::CodeModel m;
    std::string e = m.build_from_params(params_path);
    if (!e.empty()) return fail(JBP_ERR_IO, e);
    return finish_create(std::move(m), ets_dir ? ets_dir : "", device, out);
}

int jbp_create_from_checks(int n, int mx, const int *x_off, const int *x_var, int mz, const int *z_off,
                           const int *z_var, int device, jbp_ctx **out) {
    if (!out || !x_off || !z_off || n <= 0 || mx < 0 || mz < 0) return fail(JBP_ERR_ARG, "invalid code arguments");
    *out = nullptr;
    std::vector<int> xo(x_off, x_off + mx + 1), zo(z_off, z_off + mz + 1);
    if (xo[mx] < 0 || zo[mz] < 0) return fail(JBP_ERR_ARG, "invalid check offsets");
    std::vector<int> xv(x_var, x_var + xo[mx]), zv(z_var, z_var + zo[mz]);
    jbp::CodeModel m;
    std::string e = m.build_from_checks(n, xo, xv, zo, zv);
    if (!e.empty()) return fail(JBP_ERR_ARG, e);
    return finish_create(std::move(m), "", device, out);
}

int jbp_add_ets_group(jbp_ctx *ctx, int size, const char *label, const char *path_x, const char *path_z) {
    if (!ctx) return fail(JBP_ERR_ARG, "null context");
    auto &m = const_cast<jbp::CodeModel &>(ctx->engine.model());
    std::string e = m.add_ets_group(size, label ? label : std::to_string(size), path_x ? path_x : "",
                                    path_z ? path_z : "");
    if (!e.empty()) return fail(JBP_ERR_IO, e);
    return JBP_OK;
}

void jbp_destroy(jbp_ctx *ctx) { delete ctx; }

static void put_graph_checks(const jbp::GraphChecks &g, long long *odd_pairs, int *girth_x, int *girth_z) {
    if (odd_pairs) *odd_pairs = g.odd_pairs;
    if (girth_x) *girth_x = g.girth[0];
    if (girth_z) *girth_z = g.girth[1];
}

int jbp_code_graph_checks(jbp_ctx *ctx, long long *odd_pairs, int *girth_x, int *girth_z) {
    if (!ctx) return fail(JBP_ERR_ARG, "null context");
    put_graph_checks(jbp::graph_checks(ctx->engine.model()), odd_pairs, girth_x, girth_z);
    return JBP_OK;
}

int jbp_graph_checks(int n, int mx, const int *x_off, const int *x_var, int mz, const int *z_off, const int *z_var,
                     long long *odd_pairs, int *girth_x, int *girth_z) {
    if (!x_off || !z_off || n <= 0 || mx < 0 || mz < 0) return fail(JBP_ERR_ARG, "invalid code arguments");
    std::vector<int> xo(x_off, x_off + mx + 1), zo(z_off, z_off + mz + 1);
    if (xo[mx] < 0 || zo[mz] < 0) return fail(JBP_ERR_ARG, "invalid check offsets");
    std::vector<int> xv(x_var, x_var + xo[mx]), zv(z_var, z_var + zo[mz]);
    jbp::CodeModel m;
    std::string e = m.build_from_checks(n, xo, xv, zo, zv);
    if (!e.empty()) return fail(JBP_ERR_ARG, e);
    put_graph_checks(jbp::graph_checks(m), odd_pairs, girth_x, girth_z);
    return JBP_OK;
}

int jbp_code_info(jbp_ctx *ctx, int *n, int *mx, int *mz, int *rank_x, int *rank_z, int *ets_groups) {
    if (!ctx) return fail(JBP_ERR_ARG, "null context");
    const auto &m = ctx->engine.model();
    if (n) *n = m.n;
    if (mx) *mx = m.side[0].m;
    if (mz) *mz = m.side[1].m;
    if (rank_x) *rank_x = m.basis[0].rank;
    if (rank_z) *rank_z = m.basis[1].rank;
    if (ets_groups) *ets_groups = static_cast<int>(m.ets.size());
    return JBP_OK;
}

int jbp_code_checks(jbp_ctx *ctx, int side, int *off, int *var) {
    if (!ctx || side < 0 || side > 1) return fail(JBP_ERR_ARG, "invalid argument");
    const auto &g = ctx->engine.model().side[side];
    if (off) std::copy(g.chk_off.begin(), g.chk_off.end(), off);
    if (var) std::copy(g.chk_var.begin(), g.chk_var.end(), var);
    return JBP_OK;
}

int jbp_simulate(jbp_ctx *ctx, const jbp_options *opt, uint64_t seed, long long first_trial, long long ntrials,
                 double p, int sampler, jbp_stats *stats, jbp_trial_result *per_trial, long long *iter_hist) {
    if (!ctx || ntrials < 0) return fail(JBP_ERR_ARG, "invalid argument");
    if (sampler != JBP_SAMPLER_PHILOX && sampler != JBP_SAMPLER_MT19937) return fail(JBP_ERR_ARG, "unknown sampler");
    jbp::RunRequest rq;
    rq.opt = normalized(opt);
    rq.source = sampler == JBP_SAMPLER_PHILOX ? jbp::kSrcPhilox : jbp::kSrcMt19937;
    rq.seed = seed;
    rq.first_trial = first_trial;
    rq.ntrials = ntrials;
    rq.p = p;
    rq.stream = ctx->stream;
    cudaSetDevice(ctx->engine.device());
    if (per_trial) {
        if (int rc = grow(&ctx->d_res, &ctx->res_count, static_cast<size_t>(ntrials))) return rc;
        rq.d_res_out = ctx->d_res;
    }
    if (iter_hist) {
        if (rq.opt.max_iter < 1) return fail(JBP_ERR_ARG, "max_iter must be >= 1");
        if (int rc = grow(&ctx->d_hist, &ctx->hist_count, static_cast<size_t>(rq.opt.max_iter) + 1)) return rc;
        cudaMemsetAsync(ctx->d_hist, 0, sizeof(unsigned long long) * (rq.opt.max_iter + 1), ctx->stream);
        rq.d_hist = ctx->d_hist;
    }
    jbp_stats st;
    std::string e = ctx->engine.run(rq, st);
    auto copy_hist = [&]() -> int {
        std::vector<unsigned long long> h(rq.opt.max_iter + 1);
        cudaError_t ce = cudaMemcpy(h.data(), ctx->d_hist, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy histogram"));
        for (size_t i = 0; i < h.size(); ++i) iter_hist[i] = static_cast<long long>(h[i]);
        return JBP_OK;
    };
    if (!e.empty()) {
        const int rc = engine_fail(e);
        if (partial_stats(rc)) {
            // the trials finished before the stop: their counters and iteration histogram (the
            // per-trial records of the trials that did not finish are not defined, so none are copied)
            if (iter_hist)
                if (int hc = copy_hist()) return hc;
            if (stats) *stats = st;
        }
        return rc;
    }
    if (per_trial && ntrials > 0) {
        cudaError_t ce = cudaMemcpy(per_trial, ctx->d_res, sizeof(jbp_trial_result) * ntrials, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy results"));
    }
    if (iter_hist)
        if (int rc = copy_hist()) return rc;
    if (stats) *stats = st;
    return JBP_OK;
}

int jbp_simulate_mixed(jbp_ctx *const *ctxs, int nctx, const jbp_options *opt, const uint64_t *seeds,
                       const long long *first_trial, const long long *ntrials, double p, jbp_stats *stats,
                       jbp_trial_result *const *per_trial) {
    if (!ctxs || nctx < 1 || !seeds || !ntrials || !stats) return fail(JBP_ERR_ARG, "invalid argument");
    jbp::MixedRequest rq;
    rq.opt = normalized(opt);
    rq.p = p;
    for (int i = 0; i < nctx; ++i) {
        if (!ctxs[i] || ntrials[i] < 0) return fail(JBP_ERR_ARG, "invalid argument");
        rq.engines.push_back(&ctxs[i]->engine);
        rq.seeds.push_back(seeds[i]);
        rq.first_trial.push_back(first_trial ? first_trial[i] : 1);
        rq.ntrials.push_back(ntrials[i]);
    }
    cudaSetDevice(ctxs[0]->engine.device());
    rq.stream = ctxs[0]->stream;
    rq.d_res.assign(static_cast<size_t>(nctx), nullptr);
    if (per_trial)
        for (int i = 0; i < nctx; ++i)
            if (per_trial[i] && ntrials[i] > 0) {
                if (int rc = grow(&ctxs[i]->d_res, &ctxs[i]->res_count, static_cast<size_t>(ntrials[i]))) return rc;
                rq.d_res[i] = ctxs[i]->d_res;
            }
    std::vector<jbp_stats> st;
    std::string e = jbp::Engine::run_mixed(rq, st);
    if (!e.empty()) {
        const int rc = engine_fail(e);
        if (partial_stats(rc))
            for (int i = 0; i < nctx && i < static_cast<int>(st.size()); ++i) stats[i] = st[i];
        return rc;
    }
    for (int i = 0; i < nctx; ++i) {
        if (rq.d_res[i]) {
            cudaError_t ce = cudaMemcpy(per_trial[i], rq.d_res[i], sizeof(jbp_trial_result) * ntrials[i],
                                        cudaMemcpyDeviceToHost);
            if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy results"));
        }
        stats[i] = st[i];
    }
    return JBP_OK;
}

// Adds the counters and times of one engine run to a running total.
static void add_stats(jbp_stats &total, const jbp_stats &st) {
    long long *a = &total.trials;
    const long long *b = &st.trials;
    for (int i = 0; i < 15; ++i) a[i] += b[i];
    total.device_ms += st.device_ms;
    total.kernel_launches += st.kernel_launches;
    total.bp_trial_iterations += st.bp_trial_iterations;
    total.check_ms += st.check_ms;
    total.var_ms += st.var_ms;
    total.profiled_iterations += st.profiled_iterations;
    total.slots = std::max(total.slots, st.slots);
    total.learned_attempts += st.learned_attempts;
    total.learned_success += st.learned_success;
    total.test_ms += st.test_ms;
    total.syndrome_tests += st.syndrome_tests;
}

// Calls of at most this many trials from unmapped host syndromes stage through pinned memory.
constexpr long long kStagedTrials = 3;

static int decode_host(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *err, const uint8_t *sx,
                       const uint8_t *sz, double p, uint8_t *est_out, jbp_trial_result *res, jbp_stats *stats,
                       float *llr_out = nullptr) {
    if (!ctx || ntrials < 0 || !res) return fail(JBP_ERR_ARG, "invalid argument");
    const auto &m = ctx->engine.model();
    const long long n = m.n, mx = m.side[0].m, mz = m.side[1].m;
    cudaSetDevice(ctx->engine.device());
    jbp_stats total;
    std::memset(&total, 0, sizeof(total));
    // Inputs in pinned host memory the device can address (cudaHostAlloc / cudaHostRegister)
    // are read by the kernels in place: each trial's data crosses PCIe when a block starts the
    // trial, overlapping the decoding of the others, and no staging copy is made.
    auto mapped = [](const void *h) -> const uint8_t * {
        if (!h) return nullptr;
        cudaPointerAttributes at;
        if (cudaPointerGetAttributes(&at, h) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return at.type == cudaMemoryTypeHost && at.devicePointer ? static_cast<const uint8_t *>(at.devicePointer)
                                                                 : nullptr;
    };
    const uint8_t *m_err = mapped(err), *m_sx = mapped(sx), *m_sz = mapped(sz);
    // chunks bound the staging memory; each chunk is one engine run
    const bool in_place = (err && m_err) || (!err && m_sx && m_sz);
    const long long chunk = std::max<long long>(
        1, std::min<long long>(ntrials, llr_out ? 4096 : (in_place && !est_out ? 1LL << 20 : 1LL << 17)));
    for (long long base = 0; base < ntrials; base += chunk) {
        const long long cnt = std::min(chunk, ntrials - base);
        jbp::RunRequest rq;
        rq.opt = normalized(opt);
        rq.opt.p_max = 0.0;   // known inputs: every trial decodes with the given p
        rq.p = p;
        rq.stream = ctx->stream;
        rq.first_trial = 0;
        rq.ntrials = cnt;
        cudaError_t ce;
        bool host_copied = false;
        if (err && m_err) {
            rq.source = jbp::kSrcErrors;
            rq.d_err = m_err + base * n;
        } else if (err) {
            if (int rc = grow(&ctx->d_in, &ctx->in_bytes, static_cast<size_t>(cnt * n))) return rc;
            ce = cudaMemcpy(ctx->d_in, err + base * n, static_cast<size_t>(cnt * n), cudaMemcpyHostToDevice);
            if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy errors"));
            rq.source = jbp::kSrcErrors;
            rq.d_err = ctx->d_in;
        } else if (m_sx && m_sz) {
            rq.source = jbp::kSrcSyndromes;
            rq.d_sx = m_sx + base * mx;
            rq.d_sz = m_sz + base * mz;
        } else if (cnt <= kStagedTrials && !llr_out) {
            // a call of a few trials (the drop-in decodes one per call): inputs through pinned
            // staging on the context's stream, and the results, when the engine's single-trial
            // path runs, copied back behind its launches, so that the call waits once
            if (!sx || !sz) return fail(JBP_ERR_ARG, "null syndrome");
            const size_t in = static_cast<size_t>(cnt * (mx + mz)), in_al = (in + 15) / 16 * 16;
            const size_t res_b = sizeof(jbp_trial_result) * cnt, res_al = (res_b + 15) / 16 * 16;
            const size_t need = in_al + res_al + (est_out ? static_cast<size_t>(cnt * n) : 0);
            if (ctx->h_stage_bytes < need) {
                if (ctx->h_stage) cudaFreeHost(ctx->h_stage);
                ctx->h_stage = nullptr;
                ctx->h_stage_bytes = 0;
                ce = jbp::host_malloc(&ctx->h_stage, need);
                if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "cudaHostAlloc(staging)"));
                ctx->h_stage_bytes = need;
            }
            if (int rc = grow(&ctx->d_in, &ctx->in_bytes, in)) return rc;
            std::memcpy(ctx->h_stage, sx + base * mx, static_cast<size_t>(cnt * mx));
            std::memcpy(ctx->h_stage + cnt * mx, sz + base * mz, static_cast<size_t>(cnt * mz));
            ce = cudaMemcpyAsync(ctx->d_in, ctx->h_stage, in, cudaMemcpyHostToDevice, ctx->stream);
            if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy syndromes"));
            rq.source = jbp::kSrcSyndromes;
            rq.d_sx = ctx->d_in;
            rq.d_sz = ctx->d_in + cnt * mx;
            rq.h_res_out = reinterpret_cast<jbp_trial_result *>(ctx->h_stage + in_al);
            rq.h_est_out = est_out ? ctx->h_stage + in_al + res_al : nullptr;
            rq.host_copied = &host_copied;
        } else {
            if (!sx || !sz) return fail(JBP_ERR_ARG, "null syndrome");
            if (int rc = grow(&ctx->d_in, &ctx->in_bytes, static_cast<size_t>(cnt * mx))) return rc;
            if (int rc = grow(&ctx->d_in2, &ctx->in2_bytes, static_cast<size_t>(cnt * mz))) return rc;
            ce = cudaMemcpy(ctx->d_in, sx + base * mx, static_cast<size_t>(cnt * mx), cudaMemcpyHostToDevice);
            if (ce == cudaSuccess)
                ce = cudaMemcpy(ctx->d_in2, sz + base * mz, static_cast<size_t>(cnt * mz), cudaMemcpyHostToDevice);
            if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy syndromes"));
            rq.source = jbp::kSrcSyndromes;
            rq.d_sx = ctx->d_in;
            rq.d_sz = ctx->d_in2;
        }
        if (est_out) {
            if (int rc = grow(&ctx->d_est, &ctx->est_bytes, static_cast<size_t>(cnt * n))) return rc;
            rq.d_est_out = ctx->d_est;
        }
        if (int rc = grow(&ctx->d_res, &ctx->res_count, static_cast<size_t>(cnt))) return rc;
        rq.d_res_out = ctx->d_res;
        if (llr_out) {
            if (int rc = grow(&ctx->d_llr, &ctx->llr_count, static_cast<size_t>(cnt * n * 2))) return rc;
            rq.d_llr_out = ctx->d_llr;
        }
        jbp_stats st;
        std::string e = ctx->engine.run(rq, st);
        if (!e.empty()) {
            // a run that stopped before its launches leaves the staged input copy to finish
            // before the staging is reused
            if (rq.host_copied) cudaStreamSynchronize(ctx->stream);
            const int rc = engine_fail(e);
            if (partial_stats(rc) && stats) {
                add_stats(total, st);
                *stats = total;   // the trials finished within the budget
            }
            return rc;
        }
        if (host_copied) {
            std::memcpy(res + base, rq.h_res_out, sizeof(jbp_trial_result) * cnt);
            if (est_out) std::memcpy(est_out + base * n, rq.h_est_out, static_cast<size_t>(cnt * n));
            add_stats(total, st);
            continue;
        }
        ce = cudaMemcpy(res + base, ctx->d_res, sizeof(jbp_trial_result) * cnt, cudaMemcpyDeviceToHost);
        if (ce == cudaSuccess && est_out)
            ce = cudaMemcpy(est_out + base * n, ctx->d_est, static_cast<size_t>(cnt * n), cudaMemcpyDeviceToHost);
        if (ce == cudaSuccess && llr_out)
            ce = cudaMemcpy(llr_out + base * n * 2, ctx->d_llr, sizeof(float) * cnt * n * 2, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy results"));
        add_stats(total, st);
    }
    if (stats) *stats = total;
    return JBP_OK;
}

int jbp_collect_stall_states(jbp_ctx *ctx, const jbp_options *opt, uint64_t seed, long long first_trial,
                             long long ntrials, double p, int sampler, long long capacity, float *x_out, float *y_out,
                             long long *count_out, jbp_stats *stats) {
    if (!ctx || ntrials < 0 || capacity <= 0 || !x_out || !y_out || !count_out)
        return fail(JBP_ERR_ARG, "invalid argument");
    if (sampler != JBP_SAMPLER_PHILOX && sampler != JBP_SAMPLER_MT19937) return fail(JBP_ERR_ARG, "unknown sampler");
    jbp::RunRequest rq;
    rq.opt = normalized(opt);
    if (rq.opt.learned_from <= 0) return fail(JBP_ERR_ARG, "learned_from must be > 0 to define the stalls");
    rq.source = sampler == JBP_SAMPLER_PHILOX ? jbp::kSrcPhilox : jbp::kSrcMt19937;
    rq.seed = seed;
    rq.first_trial = first_trial;
    rq.ntrials = ntrials;
    rq.p = p;
    rq.stream = ctx->stream;
    rq.collect = true;
    rq.col_cap = capacity;
    cudaSetDevice(ctx->engine.device());
    float *dx = nullptr, *dy = nullptr;
    unsigned long long *dc = nullptr;
    cudaError_t ce = jbp::dev_malloc(&dx, sizeof(float) * jbp::kMlpIn * capacity);
    if (ce == cudaSuccess) ce = jbp::dev_malloc(&dy, sizeof(float) * 2 * capacity);
    if (ce == cudaSuccess) ce = jbp::dev_malloc(&dc, sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMemsetAsync(dc, 0, sizeof(unsigned long long), ctx->stream);
    std::string e;
    jbp_stats st;
    std::memset(&st, 0, sizeof(st));
    unsigned long long cnt = 0;
    if (ce != cudaSuccess) e = jbp::cuda_err(ce, "cudaMalloc(collection)");
    if (e.empty()) {
        rq.d_col_x = dx;
        rq.d_col_y = dy;
        rq.d_col_count = dc;
        e = ctx->engine.run(rq, st);
    }
    if (e.empty()) {
        ce = cudaMemcpy(&cnt, dc, sizeof(cnt), cudaMemcpyDeviceToHost);
        const long long keep = std::min<long long>(static_cast<long long>(cnt), capacity);
        if (ce == cudaSuccess && keep > 0) ce = cudaMemcpy(x_out, dx, sizeof(float) * jbp::kMlpIn * keep, cudaMemcpyDeviceToHost);
        if (ce == cudaSuccess && keep > 0) ce = cudaMemcpy(y_out, dy, sizeof(float) * 2 * keep, cudaMemcpyDeviceToHost);
        if (ce != cudaSuccess) e = jbp::cuda_err(ce, "copy collection");
        *count_out = keep;
    }
    cudaFree(dx);
    cudaFree(dy);
    cudaFree(dc);
    if (!e.empty()) return engine_fail(e);
    if (stats) *stats = st;
    return JBP_OK;
}

int jbp_decode_errors(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *err, double p,
                      uint8_t *est_out, jbp_trial_result *res, jbp_stats *stats) {
    if (!err) return fail(JBP_ERR_ARG, "null error buffer");
    // values outside 0..3 are detected on the device while the errors are read
    return decode_host(ctx, opt, ntrials, err, nullptr, nullptr, p, est_out, res, stats);
}

int jbp_decode_errors_llr(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *err, double p,
                          float *llr_out, jbp_trial_result *res, jbp_stats *stats) {
    if (!err || !llr_out) return fail(JBP_ERR_ARG, "null buffer");
    return decode_host(ctx, opt, ntrials, err, nullptr, nullptr, p, nullptr, res, stats, llr_out);
}

int jbp_decode_syndromes(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *sx,
                         const uint8_t *sz, double p, uint8_t *est_out, jbp_trial_result *res, jbp_stats *stats) {
    return decode_host(ctx, opt, ntrials, nullptr, sx, sz, p, est_out, res, stats);
}

int jbp_decode_errors_device(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *d_err, double p,
                             uint8_t *d_est_out, jbp_trial_result *d_res, jbp_stats *stats, void *stream) {
    if (!ctx || !d_err || !d_res || ntrials < 0) return fail(JBP_ERR_ARG, "invalid argument");
    jbp::RunRequest rq;
    rq.opt = normalized(opt);
    rq.opt.p_max = 0.0;
    rq.source = jbp::kSrcErrors;
    rq.first_trial = 0;
    rq.ntrials = ntrials;
    rq.p = p;
    rq.d_err = d_err;
    rq.d_est_out = d_est_out;
    rq.d_res_out = d_res;
    rq.stream = static_cast<cudaStream_t>(stream);
    cudaSetDevice(ctx->engine.device());
    jbp_stats st;
    std::string e = ctx->engine.run(rq, st);
    if (!e.empty()) {
        const int rc = engine_fail(e);
        if (partial_stats(rc) && stats) *stats = st;
        return rc;
    }
    if (stats) *stats = st;
    return JBP_OK;
}

int jbp_autotune(jbp_ctx *ctx, const jbp_options *opt, double p, long long probe_trials, jbp_options *best,
                 double *best_trials_per_s) {
    if (!ctx || !best || probe_trials <= 0) return fail(JBP_ERR_ARG, "invalid argument");
    const jbp_options base = normalized(opt);
    // check_interval 0 (asked for explicitly) admits the choices that change results: the
    // interval of the syndrome test, among 1, 2 and 4, where post-processing is off (it needs a
    // test every iteration) -- trials then stop at a multiple of the interval -- and, for FP32
    // messages, the resident engine, whose arithmetic differs slightly from the slot engine's
    // that AUTO uses for FP32.  Otherwise every candidate decodes as AUTO does.
    const bool result_changing = opt && opt->check_interval == 0;
    const bool tune_ci = result_changing && !base.enable_pp;
    const bool resident_ok = base.precision != JBP_PREC_FP32 || result_changing;
    std::vector<int> intervals = tune_ci ? std::vector<int>{1, 2, 4} : std::vector<int>{base.check_interval};
    std::vector<jbp_options> cand;
    for (int ci : intervals) {
        jbp_options c = base;
        c.check_interval = ci;
        c.engine = JBP_ENGINE_RESIDENT;
        if (resident_ok) cand.push_back(c);
        for (int S : {4096, 8192, 16384, 32768})
            for (int gi : {2, 4, 8}) {
                c = base;
                c.check_interval = ci;
                c.engine = JBP_ENGINE_SLOTS;
                c.slots = S;
                c.iters_per_launch = gi;
                cand.push_back(c);
            }
    }
    double best_rate = -1.0;
    for (const jbp_options &o : cand) {
        jbp_stats st;
        // a short run first (buffers, graphs), then the timed probe
        int rc = jbp_simulate(ctx, &o, 1, 1, std::max<long long>(64, probe_trials / 8), p, JBP_SAMPLER_PHILOX, &st,
                              nullptr, nullptr);
        if (rc == JBP_ERR_UNSUPPORTED) continue;   // e.g. the resident engine does not apply
        if (rc != JBP_OK) return rc;
        rc = jbp_simulate(ctx, &o, 1, 1, probe_trials, p, JBP_SAMPLER_PHILOX, &st, nullptr, nullptr);
        if (rc != JBP_OK) return rc;
        const double rate = st.device_ms > 0.0 ? st.trials / (st.device_ms / 1000.0) : 0.0;
        if (rate > best_rate) {
            best_rate = rate;
            *best = o;
        }
    }
    if (best_rate < 0.0) return fail(JBP_ERR_UNSUPPORTED, "no engine configuration applies");
    if (best_trials_per_s) *best_trials_per_s = best_rate;
    return JBP_OK;
}

int jbp_sample_errors(jbp_ctx *ctx, uint64_t seed, long long first_trial, long long ntrials, double p, int sampler,
                      uint8_t *err) {
    if (!ctx || !err || ntrials < 0) return fail(JBP_ERR_ARG, "invalid argument");
    if (sampler != JBP_SAMPLER_PHILOX && sampler != JBP_SAMPLER_MT19937) return fail(JBP_ERR_ARG, "unknown sampler");
    const long long n = ctx->engine.model().n;
    cudaSetDevice(ctx->engine.device());
    if (int rc = grow(&ctx->d_in, &ctx->in_bytes, static_cast<size_t>(ntrials * n))) return rc;
    std::string e = ctx->engine.sample_errors(seed, first_trial, ntrials, p,
                                              sampler == JBP_SAMPLER_PHILOX ? jbp::kSrcPhilox : jbp::kSrcMt19937,
                                              ctx->d_in);
    if (!e.empty()) return engine_fail(e);
    cudaError_t ce = cudaMemcpy(err, ctx->d_in, static_cast<size_t>(ntrials * n), cudaMemcpyDeviceToHost);
    if (ce != cudaSuccess) return fail(JBP_ERR_CUDA, jbp::cuda_err(ce, "copy errors"));
    return JBP_OK;
}

// The reference sampler, run on the host with libstdc++'s mt19937_64 and
// uniform_real_distribution<double> (jointbp_ets.cpp:4401-4411, 5931-5946).
int jbp_sample_reference_errors(int n, uint64_t seed, long long first_trial, long long ntrials, double p,
                                uint8_t *err, int threads) {
    if (n <= 0 || ntrials < 0 || !err) return fail(JBP_ERR_ARG, "invalid argument");
    if (threads <= 0) threads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    threads = static_cast<int>(std::min<long long>(threads, std::max<long long>(ntrials, 1)));
    auto work = [&](long long lo, long long hi) {
        std::uniform_real_distribution<double> dist(0.0, 1.0);
        for (long long t = lo; t < hi; ++t) {
            const unsigned long long idx = static_cast<unsigned long long>(first_trial + t);
            std::mt19937_64 rng(jbp::splitmix64(seed ^ (idx * 0x9e3779b97f4a7c15ull)));
            uint8_t *e = err + t * n;
            for (int i = 0; i < n; ++i) {
                const double u = dist(rng);
                if (u < 1.0 - p) {
                    e[i] = 0;
                } else {
                    const double v = (u - (1.0 - p)) / p;
                    e[i] = v < 1.0 / 3.0 ? 1 : (v < 2.0 / 3.0 ? 2 : 3);
                }
            }
        }
    };
    std::vector<std::thread> pool;
    const long long per = (ntrials + threads - 1) / threads;
    for (int k = 0; k < threads; ++k) {
        const long long lo = k * per, hi = std::min(ntrials, lo + per);
        if (lo < hi) pool.emplace_back(work, lo, hi);
    }
    for (auto &t : pool) t.join();
    return JBP_OK;
}

}  // extern "C"
