// jointbp_cuda.h over the C ABI (include/jbp_b200.h): the reference host program links this
// library in place of its jointbp_cuda.cu.  Contract and differences: include/jointbp_cuda.h.
#include "jointbp_cuda.h"

#include <chrono>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "jbp_b200.h"

struct CudaBPContext {
    jbp_ctx *ctx = nullptr;
    int nvars = 0, mx = 0, mz = 0;
    int precision = JBP_PREC_FP64;
    std::vector<uint8_t> sx8, sz8, est8;
};

namespace {

bool fail(std::string *err, const std::string &msg) {
    if (err) *err = msg;
    return false;
}

// check lists of one side from the CSR graph (check c: x_edge_var of its edges, in order)
bool side_lists(int m, int nvars, int edges, const std::vector<int> &off, const std::vector<int> &chk_edges,
                const std::vector<int> &edge_var, std::vector<int> &o, std::vector<int> &v, std::string *err,
                const char *name) {
    if (static_cast<int>(off.size()) != m + 1 || off[0] != 0 || off[m] != edges ||
        static_cast<int>(chk_edges.size()) != edges || static_cast<int>(edge_var.size()) != edges)
        return fail(err, std::string("CUDA graph: inconsistent ") + name + " CSR sizes");
    o.assign(off.begin(), off.end());
    v.resize(edges);
    for (int k = 0; k < edges; ++k) {
        const int e = chk_edges[k];
        if (e < 0 || e >= edges) return fail(err, std::string("CUDA graph: ") + name + " edge id out of range");
        const int var = edge_var[e];
        if (var < 0 || var >= nvars) return fail(err, std::string("CUDA graph: ") + name + " variable out of range");
        v[k] = var;
    }
    for (int c = 0; c < m; ++c)
        if (o[c + 1] < o[c]) return fail(err, std::string("CUDA graph: ") + name + " offsets decrease");
    return true;
}

int precision_from_env() {
    const char *p = std::getenv("JBP_CUDA_PRECISION");
    if (!p || !*p || !std::strcmp(p, "fp64")) return JBP_PREC_FP64;
    if (!std::strcmp(p, "fp32")) return JBP_PREC_FP32;
    if (!std::strcmp(p, "fp16")) return JBP_PREC_FP16;
    return -1;
}

bool check_due(int k1, int max_iter, int warmup, int interval) {
    return k1 >= max_iter || (k1 > warmup && (k1 - warmup) % interval == 0);
}

}  // namespace

CudaBPContext *cuda_bp_create(const CudaBPGraph &g, int device_id, std::string *error_out) {
    if (g.nvars <= 0 || g.mX <= 0 || g.mZ <= 0) {
        fail(error_out, "CUDA graph: empty code");
        return nullptr;
    }
    const int prec = precision_from_env();
    if (prec < 0) {
        fail(error_out, "JBP_CUDA_PRECISION must be fp64, fp32 or fp16");
        return nullptr;
    }
    std::vector<int> xo, xv, zo, zv;
    if (!side_lists(g.mX, g.nvars, g.x_edges, g.x_check_offsets, g.x_check_edges, g.x_edge_var, xo, xv, error_out,
                    "X") ||
        !side_lists(g.mZ, g.nvars, g.z_edges, g.z_check_offsets, g.z_check_edges, g.z_edge_var, zo, zv, error_out,
                    "Z"))
        return nullptr;
    jbp_ctx *ctx = nullptr;
    if (jbp_create_from_checks(g.nvars, g.mX, xo.data(), xv.data(), g.mZ, zo.data(), zv.data(), device_id, &ctx) !=
        JBP_OK) {
        fail(error_out, jbp_last_error());
        return nullptr;
    }
    auto *c = new CudaBPContext;
    c->ctx = ctx;
    c->nvars = g.nvars;
    c->mx = g.mX;
    c->mz = g.mZ;
    c->precision = prec;
    return c;
}

void cuda_bp_destroy(CudaBPContext *ctx) {
    if (!ctx) return;
    jbp_destroy(ctx->ctx);
    delete ctx;
}

bool cuda_bp_decode(CudaBPContext *ctx, const std::vector<int> &sx, const std::vector<int> &sz, const CudaMsg &prior,
                    int max_iter, int check_warmup, int check_interval, bool measure_costs, bool use_graph,
                    bool freeze_syn, double damping, CudaBPResult &out, std::string *error_out) {
    (void)use_graph;
    const auto t0 = std::chrono::steady_clock::now();
    if (!ctx) return fail(error_out, "CUDA context not initialized");
    if (static_cast<int>(sx.size()) != ctx->mx || static_cast<int>(sz.size()) != ctx->mz)
        return fail(error_out, "CUDA input syndrome size mismatch");
    if (check_warmup < 0) check_warmup = 0;
    if (check_interval <= 0) check_interval = 1;
    jbp_options o;
    jbp_default_options(&o);
    o.precision = ctx->precision;
    o.max_iter = max_iter;
    o.damping = damping;
    o.enable_pp = 0;
    o.freeze_syn = freeze_syn ? 1 : 0;
    o.check_warmup = check_warmup;
    o.check_interval = check_interval;
    o.profile = measure_costs ? 1 : 0;
    o.use_prior = 1;
    for (int i = 0; i < 4; ++i) o.prior[i] = prior.v[i];
    ctx->sx8.resize(ctx->mx);
    ctx->sz8.resize(ctx->mz);
    for (int i = 0; i < ctx->mx; ++i) ctx->sx8[i] = static_cast<uint8_t>(sx[i] & 1);
    for (int i = 0; i < ctx->mz; ++i) ctx->sz8[i] = static_cast<uint8_t>(sz[i] & 1);
    ctx->est8.resize(ctx->nvars);
    jbp_trial_result res;
    jbp_stats st;
    if (jbp_decode_syndromes(ctx->ctx, &o, 1, ctx->sx8.data(), ctx->sz8.data(), 0.0, ctx->est8.data(), &res, &st) !=
        JBP_OK)
        return fail(error_out, jbp_last_error());
    out.est.assign(ctx->est8.begin(), ctx->est8.end());
    out.iterations = res.iterations;
    out.syndrome_match = res.syndrome_ok != 0;
    // the reference loop's syndrome tests up to the last iteration, plus its final test when
    // the loop ran out (jointbp_cuda.cu:970-1071)
    int checks = 0;
    for (int k = 1; k <= res.iterations; ++k) checks += check_due(k, max_iter, check_warmup, check_interval);
    if (!res.syndrome_ok) checks += 1;
    out.check_count = checks;
    out.kernel_ms = st.device_ms;
    out.memcpy_ms = 0.0;
    out.check_kernel_ms = 0.0;
    out.check_memcpy_ms = 0.0;
    out.init_kernel_ms = 0.0;
    const double total = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    out.host_ms = total > st.device_ms ? total - st.device_ms : 0.0;
    return true;
}
