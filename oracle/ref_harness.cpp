// Test infrastructure only: a C-ABI harness around the UNMODIFIED reference decoder.
//
// This translation unit textually includes the reference source file jointbp_ets.cpp
// (path supplied by the build recipe with -I) after renaming its `main`, so that the
// reference's own file-local functions (joint_bp_decode, compute_syndrome,
// attempt_ets_fix_side_multi, attempt_flip_pp_side, attempt_osd_pp_side, in_row_space,
// read_ets_file, trial_seed_from_base, ...) become callable from tests.  No reference
// code is copied into this repository; the build output lives in oracle/_ref/ only.
//
// The per-trial driver below (ref_simulate_trial) calls those functions in the order the
// reference's --simulate loop does (jointbp_ets.cpp:5931-6245): sample, syndrome,
// joint_bp_decode, post-BP ETS -> flip -> OSD, success classification.  Logging-only
// branches of that loop are omitted because they never change `est` or a counter.
//
// Only tests/, bench.py's CPU baseline leg and __graft_entry__.smoke() may use this.

#define main jointbp_reference_main
#include "jointbp_ets.cpp"
#undef main

#include <cstring>

namespace refh {

struct Code {
    bool ready = false;
    Params params;
    int nvars = 0;
    std::vector<std::vector<int>> x_checks, z_checks;
    std::vector<std::vector<EdgeRef>> var_to_x, var_to_z;
    RowBasis hx_basis, hz_basis;
    // ETS groups in the reference load order: 6, 8, 8p4, 10, 12, 14, 16, 18, 20, 22
    struct Group {
        int size = 0;
        std::string label;
        ETSIndex x, z;
        bool x_loaded = false, z_loaded = false;
    };
    std::vector<Group> groups;  // only groups with at least one side loaded
    std::vector<ETSIndexRef> refs;
};

Code g;

// Mirrors the reference's load_ets lambda (jointbp_ets.cpp:5242-5293) without printing.
static bool load_one(int size, const std::string &path, char side, ETSIndex &out) {
    std::string resolved = resolve_existing_path(path);
    if (resolved.empty()) return false;
    std::error_code ec;
    auto fsz = std::filesystem::file_size(resolved, ec);
    if (!ec && fsz == 0) return false;
    if (!read_ets_file(resolved, static_cast<int>(g.params.P), size, side, out)) return false;
    return !out.entries.empty();
}

}  // namespace refh

extern "C" {

struct RefTrialRecord {
    long long trial_idx;
    int iterations;
    int bp_ok;            // res.bp_syndrome_match
    int syndrome_ok;      // final syndrome match after all PP
    int success;          // syndrome_ok && stabilizer-equivalent
    int exact;            // est == err
    int stab_equiv;
    int pp_in_decode;     // res.pp_success (in-loop PP)
    int pp_in_ets;        // res.pp_success_ets
    int pp_in_flip;       // res.pp_success_flip
    int ets_pp_ok;        // final (in-loop or post-BP) ETS success flag
    int flip_pp_ok;
    int osd_pp_ok;        // post-BP OSD success flag
    int used_any;         // ETS used (any)
    int used6;
    int used12;
    int ets_applied_post; // post-BP ETS applied on either side
    int pp_success_this;  // counted in pp_success
    int osd_success;      // counted in osd_pp_success (reference definition)
};

// Builds the code from a params file and loads ETS tables the way the reference does with
// default paths (directory named after the params basename).  ets_dir overrides that
// directory when non-null.  Returns 0 on success.
int ref_init(const char *params_path, const char *ets_dir) {
    using namespace refh;
    g = Code{};
    if (!read_params(params_path, g.params)) return 1;
    auto hx_blocks = build_block_matrix_hx(g.params.P, g.params.J, g.params.L2, g.params.a, g.params.b,
                                           g.params.c, g.params.d);
    auto hz_blocks = build_block_matrix_hz(g.params.P, g.params.J, g.params.L2, g.params.a, g.params.b,
                                           g.params.c, g.params.d);
    g.x_checks = build_check_neighbors(hx_blocks, g.params.P);
    g.z_checks = build_check_neighbors(hz_blocks, g.params.P);
    g.nvars = g.params.L * static_cast<int>(g.params.P);
    g.var_to_x = build_var_adjacency(g.x_checks, g.nvars);
    g.var_to_z = build_var_adjacency(g.z_checks, g.nvars);
    g.hx_basis = build_row_basis(g.x_checks, g.nvars);
    g.hz_basis = build_row_basis(g.z_checks, g.nvars);

    std::string dir = ets_dir ? std::string(ets_dir) : basename_no_ext(params_path);
    if (!ets_dir) {
        // the reference resolves the directory relative to the CWD; tests pass absolute dirs
        std::string pp(params_path);
        size_t slash = pp.find_last_of('/');
        if (slash != std::string::npos) dir = pp.substr(0, slash + 1) + basename_no_ext(params_path);
    }
    const int sizes[] = {6, 8, 10, 12, 14, 16, 18, 20, 22};
    auto add_group = [&](int size, const std::string &label, const std::string &path) {
        Code::Group grp;
        grp.size = size;
        grp.label = label;
        grp.x_loaded = load_one(size, path, 'X', grp.x);
        grp.z_loaded = load_one(size, path, 'Z', grp.z);
        if (grp.x_loaded || grp.z_loaded) g.groups.push_back(std::move(grp));
    };
    for (int size : sizes) {
        add_group(size, std::to_string(size), dir + "/ets_" + std::to_string(size) + "_2.txt");
        if (size == 8) add_group(8, "8p4", dir + "/ets_8_2_path4.txt");
    }
    for (auto &grp : g.groups) {
        ETSIndexRef r;
        r.size = grp.size;
        r.label = grp.label;
        r.x = grp.x_loaded ? &grp.x : nullptr;
        r.z = grp.z_loaded ? &grp.z : nullptr;
        g.refs.push_back(r);
    }
    g.ready = true;
    return 0;
}

int ref_nvars(void) { return refh::g.nvars; }
int ref_mx(void) { return static_cast<int>(refh::g.x_checks.size()); }
int ref_mz(void) { return static_cast<int>(refh::g.z_checks.size()); }
int ref_rank_x(void) { return static_cast<int>(refh::g.hx_basis.rows.size()); }
int ref_rank_z(void) { return static_cast<int>(refh::g.hz_basis.rows.size()); }
int ref_girth(int side) {
    return side == 0 ? compute_girth(refh::g.x_checks, refh::g.var_to_x)
                     : compute_girth(refh::g.z_checks, refh::g.var_to_z);
}

// ETS entry counts per loaded group, in load order: out[2*i] = X count, out[2*i+1] = Z count.
int ref_ets_counts(int *out, int max_groups, char *labels, int label_stride) {
    int n = 0;
    for (auto &grp : refh::g.groups) {
        if (n >= max_groups) break;
        out[2 * n] = grp.x_loaded ? static_cast<int>(grp.x.entries.size()) : 0;
        out[2 * n + 1] = grp.z_loaded ? static_cast<int>(grp.z.entries.size()) : 0;
        if (labels) std::strncpy(labels + n * label_stride, grp.label.c_str(), label_stride - 1);
        ++n;
    }
    return n;
}

// Neighbour lists, check-major: out[c*deg + i] (deg = 12 for the shipped code).
int ref_checks(int side, int *out) {
    const auto &ch = side == 0 ? refh::g.x_checks : refh::g.z_checks;
    int k = 0;
    for (const auto &row : ch)
        for (int v : row) out[k++] = v;
    return k;
}

// Reference per-trial sampler (jointbp_ets.cpp:5932-5946).
void ref_sample(unsigned long long seed, long long trial_idx, double p, int *err) {
    uint64_t s = trial_seed_from_base(seed, static_cast<uint64_t>(trial_idx));
    std::mt19937_64 rng(s);
    std::uniform_real_distribution<double> dist(0.0, 1.0);
    for (int i = 0; i < refh::g.nvars; ++i) {
        double u = dist(rng);
        if (u < (1.0 - p)) {
            err[i] = 0;
        } else {
            double v = (u - (1.0 - p)) / p;
            err[i] = v < 1.0 / 3.0 ? 1 : (v < 2.0 / 3.0 ? 2 : 3);
        }
    }
}

void ref_syndrome(const int *err, int *sx, int *sz) {
    std::vector<int> e(err, err + refh::g.nvars);
    auto a = compute_syndrome(refh::g.x_checks, e, true);
    auto b = compute_syndrome(refh::g.z_checks, e, false);
    std::copy(a.begin(), a.end(), sx);
    std::copy(b.begin(), b.end(), sz);
}

// Plain joint BP (no PP) on a syndrome: est, iterations, syndrome match and the final
// |LLR| vectors (collected on the last iteration, as collect_llr_final does).
int ref_bp_decode(const int *sx_in, const int *sz_in, double p, int max_iter, double damping,
                  int freeze_syn, int *est, int *syndrome_ok, double *abs_llr_x, double *abs_llr_z) {
    using namespace refh;
    std::vector<int> sx(sx_in, sx_in + g.x_checks.size());
    std::vector<int> sz(sz_in, sz_in + g.z_checks.size());
    Msg prior{1.0 - p, p / 3.0, p / 3.0, p / 3.0};
    normalize_msg(prior);
    JointBPResult res = joint_bp_decode(g.x_checks, g.z_checks, g.var_to_x, g.var_to_z, sx, sz, prior,
                                        max_iter, 5, freeze_syn != 0, damping, false, false,
                                        abs_llr_x != nullptr, nullptr, nullptr, nullptr, nullptr,
                                        nullptr, nullptr);
    std::copy(res.est.begin(), res.est.end(), est);
    if (syndrome_ok) *syndrome_ok = res.syndrome_match ? 1 : 0;
    if (abs_llr_x && res.abs_llr_x.size() == static_cast<size_t>(g.nvars)) {
        std::copy(res.abs_llr_x.begin(), res.abs_llr_x.end(), abs_llr_x);
        std::copy(res.abs_llr_z.begin(), res.abs_llr_z.end(), abs_llr_z);
    }
    return res.iterations;
}

// The body of one Monte-Carlo trial from a known error, as the reference --simulate loop
// runs it after sampling.
int ref_error_trial(const int *err_in, long long trial_idx, double p, int max_iter, int flip_hist, double damping,
                    int freeze_syn, int enable_pp, RefTrialRecord *rec, int *est_out) {
    using namespace refh;
    if (!g.ready) return 1;
    std::vector<int> err(err_in, err_in + g.nvars);
    auto sx = compute_syndrome(g.x_checks, err, true);
    auto sz = compute_syndrome(g.z_checks, err, false);
    Msg prior{1.0 - p, p / 3.0, p / 3.0, p / 3.0};
    normalize_msg(prior);
    PPEarlyContext pp_ctx{enable_pp != 0, false, g.refs, nullptr};
    JointBPResult res = joint_bp_decode(g.x_checks, g.z_checks, g.var_to_x, g.var_to_z, sx, sz, prior,
                                        max_iter, flip_hist, freeze_syn != 0, damping, false, false,
                                        enable_pp != 0, enable_pp ? &pp_ctx : nullptr, &err, &g.hx_basis,
                                        &g.hz_basis, nullptr, nullptr);
    bool bp_ok = res.bp_syndrome_match;
    bool used6 = res.pp_used_ets6, used12 = res.pp_used_ets12;
    bool used_any = res.pp_used_ets_any || used6 || used12;
    bool ok = res.syndrome_match;
    bool ets_pp_ok = res.pp_success_ets, flip_pp_ok = res.pp_success_flip, osd_pp_ok = false;
    bool ets_applied = false;
    if (!ok && enable_pp) {
        ETSFixResult ex = attempt_ets_fix_side_multi("X", g.refs, g.x_checks, g.var_to_x, sx, true, res.est, false);
        ETSFixResult ez = attempt_ets_fix_side_multi("Z", g.refs, g.z_checks, g.var_to_z, sz, false, res.est, false);
        ets_applied = ex.applied || ez.applied;
        used_any = used_any || ets_applied;
        used6 = used6 || ex.size == 6 || ez.size == 6;
        used12 = used12 || ex.size == 12 || ez.size == 12;
        if (ets_applied) {
            ok = compute_syndrome(g.x_checks, res.est, true) == sx && compute_syndrome(g.z_checks, res.est, false) == sz;
            if (ok) ets_pp_ok = true;
        }
    }
    if (!ok && enable_pp) {
        bool fx = false, fz = false;
        for (const auto &set : build_flip_sets(res.flip_x_history, res.flip_x_window, res.flip_x)) {
            if (!set.vars || set.vars->empty()) continue;
            if (attempt_flip_pp_side("X", *set.vars, g.x_checks, sx, true, res.est, false, nullptr, set.tag)) {
                fx = true;
                break;
            }
        }
        for (const auto &set : build_flip_sets(res.flip_z_history, res.flip_z_window, res.flip_z)) {
            if (!set.vars || set.vars->empty()) continue;
            if (attempt_flip_pp_side("Z", *set.vars, g.z_checks, sz, false, res.est, false, nullptr, set.tag)) {
                fz = true;
                break;
            }
        }
        if (fx || fz) {
            ok = compute_syndrome(g.x_checks, res.est, true) == sx && compute_syndrome(g.z_checks, res.est, false) == sz;
            if (ok) flip_pp_ok = true;
        }
    }
    if (!ok && enable_pp) {
        auto shx = compute_syndrome(g.x_checks, res.est, true);
        auto shz = compute_syndrome(g.z_checks, res.est, false);
        int us = std::max(unsatisfied_count(shx, sx), unsatisfied_count(shz, sz));
        if (us <= 20) {
            bool ox = attempt_osd_pp_side("X", res.abs_llr_x, g.x_checks, sx, true, res.est, false, &err);
            bool oz = attempt_osd_pp_side("Z", res.abs_llr_z, g.z_checks, sz, false, res.est, false, &err);
            if (ox || oz) {
                ok = compute_syndrome(g.x_checks, res.est, true) == sx &&
                     compute_syndrome(g.z_checks, res.est, false) == sz;
                if (ok) osd_pp_ok = true;
            }
        }
    }
    bool exact = (res.est == err);
    bool stab = false, success = ok;
    if (ok) {
        std::vector<uint64_t> dx(g.hz_basis.words, 0), dz(g.hx_basis.words, 0);
        fill_diff_bits(dx, err, res.est, true);
        fill_diff_bits(dz, err, res.est, false);
        stab = in_row_space(g.hz_basis, dx) && in_row_space(g.hx_basis, dz);
        success = ok && stab;
    }
    bool osd_success = osd_pp_ok || (res.pp_success && !res.pp_success_ets && !res.pp_success_flip);
    rec->trial_idx = trial_idx;
    rec->iterations = res.iterations;
    rec->bp_ok = bp_ok;
    rec->syndrome_ok = ok;
    rec->success = success;
    rec->exact = exact;
    rec->stab_equiv = stab;
    rec->pp_in_decode = res.pp_success;
    rec->pp_in_ets = res.pp_success_ets;
    rec->pp_in_flip = res.pp_success_flip;
    rec->ets_pp_ok = ets_pp_ok;
    rec->flip_pp_ok = flip_pp_ok;
    rec->osd_pp_ok = osd_pp_ok;
    rec->used_any = used_any;
    rec->used6 = used6;
    rec->used12 = used12;
    rec->ets_applied_post = ets_applied;
    rec->pp_success_this = success && (res.pp_success || ets_pp_ok || flip_pp_ok || osd_pp_ok);
    rec->osd_success = osd_success;
    if (est_out) std::copy(res.est.begin(), res.est.end(), est_out);
    return 0;
}

// One Monte-Carlo trial exactly as the reference --simulate loop runs it.
int ref_simulate_trial(unsigned long long seed, long long trial_idx, double p, int max_iter, int flip_hist,
                       double damping, int freeze_syn, int enable_pp, RefTrialRecord *rec, int *err_out,
                       int *est_out) {
    if (!refh::g.ready) return 1;
    std::vector<int> err(refh::g.nvars);
    ref_sample(seed, trial_idx, p, err.data());
    int rc = ref_error_trial(err.data(), trial_idx, p, max_iter, flip_hist, damping, freeze_syn, enable_pp, rec,
                             est_out);
    if (err_out) std::copy(err.begin(), err.end(), err_out);
    return rc;
}

}  // extern "C"
