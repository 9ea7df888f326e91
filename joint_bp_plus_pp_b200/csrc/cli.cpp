// jointbp_b200: the reference command line (jointbp_ets.cpp:4733-6449) over the batched GPU
// decoder of include/jbp_b200.h.
//
// Same flags, params/ETS/vector file formats, modes (--simulate, --err, --sx/--sz) and exit
// codes (0 ok, 2 single decode failed, 1 usage or input error), and the same Run Summary line
// (jointbp_ets.cpp:6427-6448).  Unlike the reference, --cuda is not required and post-
// processing runs on the GPU too (the reference allows --cuda only with --no-pp,
// jointbp_ets.cpp:5408).  Monte Carlo trials run in batches of --batch trials on the device;
// by default they use the reference's error stream (splitmix64 + mt19937_64 per trial index)
// and FP64 messages, so counts equal the reference CPU run's.
//
// Extra flags: --precision fp64|fp32|fp16, --sampler mt19937|philox, --slots N, --batch N,
// --ets-dir DIR.  Flags of the reference's per-iteration CPU diagnostics (--verbose,
// --verbose-all, --report-ets, --report-fail, --save-fail-prefix) are accepted and ignored.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <csignal>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <sstream>
#include <string>
#include <sys/stat.h>
#include <thread>
#include <vector>

#include "jbp_b200.h"

namespace {

// Ctrl-C during a simulation: every context is asked to stop (jbp_request_abort, a store to a
// pinned host word); each run returns the trials that finished, and the Run Summary of those is
// printed (exit status 130).  The context list is filled before the handler is installed.
std::vector<jbp_ctx *> g_abort_ctxs;
volatile std::sig_atomic_t g_interrupted = 0;

extern "C" void on_interrupt(int) {
    g_interrupted = 1;
    for (jbp_ctx *c : g_abort_ctxs) jbp_request_abort(c);
}

void install_interrupt(const std::vector<jbp_ctx *> &ctxs) {
    g_abort_ctxs = ctxs;
    std::signal(SIGINT, on_interrupt);
}

struct Args {
    std::string params, sx_path, sz_path, err_path, est_path, hist_out, progress_tsv, ets_dir;
    std::vector<int> devices;   // --cuda-devices: one context and host thread per entry
    int learned_order = 0;      // --learned-order: 0 the model's scores, 1 |LLR| order
    std::string ets6_x, ets6_z, ets12_x, ets12_z, ets8_path4;
    double p = 0.05, damping = 0.0;
    int max_iter = 50, flip_hist = 5, device = 0, check_warmup = 0, check_interval = 1;
    bool freeze_syn = false, simulate = false, enable_pp = true, seed_set = false;
    unsigned long long seed = 0;
    long long trials = 1, min_fails = 0, report_every = 100, progress_every = 100, trial_index = -1;
    int precision = JBP_PREC_FP64, sampler = JBP_SAMPLER_MT19937, slots = 0;
    long long batch = 1 << 18;
    int engine = JBP_ENGINE_AUTO, learned_from = 0;
    std::string flip_model, checks, mixed;
    double p_max = 0.0;
    bool autotune = false;
};

void usage(const char *prog) {
    std::cout << "Usage: " << prog << " --params FILE [mode] [options]\n"
              << "Modes:\n"
              << "  --simulate               Monte Carlo over seeded depolarizing errors\n"
              << "  --err FILE               decode the syndrome of an error vector (0..3 per qubit)\n"
              << "  --sx FILE --sz FILE      decode a syndrome pair (one bit per check)\n"
              << "Options (reference defaults):\n"
              << "  --p P (0.05)  --max-iter N (50)  --flip-hist H (5)  --damping D (0)  --freeze-syn\n"
              << "  --no-pp  --seed S  --trials N (1)  --trial-index I  --min-fails N  --est FILE\n"
              << "  --report-every N (100)  --progress-every N (100)  --progress-tsv FILE  --iter-hist-out FILE\n"
              << "  --ets6-x F --ets6-z F --ets12-x F --ets12-z F --ets-x F --ets-z F --ets8-path4 F\n"
              << "  --cuda --cuda-graph (accepted; decoding always runs on the GPU)  --cuda-device D\n"
              << "  --cuda-devices D0,D1,... (with --simulate: one context and host thread per listed device, each\n"
              << "  decoding a contiguous part of the trial range; one Run Summary of the whole run)\n"
              << "  --cuda-check-warmup N (0)  --cuda-check-interval N (1; 0 with --autotune: tuned)\n"
              << "Extra options:\n"
              << "  --precision fp64|fp32|fp16 (fp64)  --sampler mt19937|philox (mt19937)\n"
              << "  --slots N (trials in flight, 0 = auto)  --batch N (trials per GPU call, 262144)\n"
              << "  --ets-dir DIR (default: the params path without extension)\n"
              << "  --engine auto|resident|slots|table (auto)  --learned-from N (0 = off; learned flip proposal at\n"
              << "  stalls from iteration N, resident engine with FP32 or FP16 messages)  --learned-order model|llr (model:\n"
              << "  columns by the network's scores; llr: by |LLR|, the baseline)  --flip-model FILE.npy (default: the\n"
              << "  shipped data/flip_mlp_params.npy next to the library)\n"
              << "  --checks FILE (a code as check lists instead of --params: 'n mx mz', then one line of\n"
              << "  variables per X check and per Z check)  --p-max P (per-trial p uniform in [p, P))\n"
              << "  --autotune (time short probes and keep the fastest engine / slots / graph length)\n"
              << "  --mixed FILE1,FILE2,... (with --simulate --no-pp: the codes of these check-list files, --trials\n"
              << "  trials each with seed --seed + i, in one kernel launch; one Run Summary per code)\n";
}

// format_scaled_unit / format_latency (jointbp_ets.cpp:203-237)
std::string scaled_unit(double value, double scale, const char *suffix) {
    const double s = value / scale, a = std::fabs(s);
    const int prec = a < 10.0 ? 2 : (a < 100.0 ? 1 : 0);
    std::ostringstream o;
    o << std::fixed << std::setprecision(prec) << s << suffix;
    return o.str();
}
std::string latency_str(double sec) {
    return std::fabs(sec) < 1e-3 ? scaled_unit(sec, 1e-6, "us") : scaled_unit(sec, 1e-3, "ms");
}

// Wilson score interval (jointbp_ets.cpp:4388-4399)
bool wilson(long long n, long long k, double z, double &lo, double &hi) {
    if (n <= 0) return false;
    const double ph = static_cast<double>(k) / n, z2 = z * z;
    const double den = 1.0 + z2 / n;
    const double c = (ph + z2 / (2.0 * n)) / den;
    const double m = z * std::sqrt(ph * (1.0 - ph) / n + z2 / (4.0 * n * n)) / den;
    lo = std::max(0.0, c - m);
    hi = std::min(1.0, c + m);
    return true;
}

std::string basename_no_ext(const std::string &path) {
    const size_t dot = path.find_last_of('.'), slash = path.find_last_of('/');
    if (dot == std::string::npos || (slash != std::string::npos && dot < slash)) return path;
    return path.substr(0, dot);
}

bool exists(const std::string &p) {
    struct stat st;
    return stat(p.c_str(), &st) == 0;
}

bool read_ints(const std::string &path, std::vector<int> &out) {
    std::ifstream in(path);
    if (!in) return false;
    out.clear();
    int v = 0;
    while (in >> v) out.push_back(v);
    return true;
}

bool write_vector(const std::string &path, const uint8_t *v, int n) {
    std::ofstream o(path);
    if (!o) return false;
    for (int i = 0; i < n; ++i) o << static_cast<int>(v[i]) << "\n";
    return true;
}

const char *tf(bool b) { return b ? "true" : "false"; }

// returns 0 on success, 1 on a usage error (message printed)
int parse(int argc, char **argv, Args &a) {
    auto need = [&](int &i, const char *flag) -> const char * {
        if (i + 1 >= argc) {
            std::cerr << "Missing value for " << flag << "\n";
            return nullptr;
        }
        return argv[++i];
    };
    for (int i = 1; i < argc; ++i) {
        const std::string f = argv[i];
        const char *v = nullptr;
#define VAL()                             \
    do {                                  \
        if (!(v = need(i, f.c_str()))) { \
            return 1;                     \
        }                                 \
    } while (0)
        try {
            if (f == "--help" || f == "-h") { usage(argv[0]); return 2; }
            else if (f == "--params") { VAL(); a.params = v; }
            else if (f == "--sx") { VAL(); a.sx_path = v; }
            else if (f == "--sz") { VAL(); a.sz_path = v; }
            else if (f == "--err") { VAL(); a.err_path = v; }
            else if (f == "--est") { VAL(); a.est_path = v; }
            else if (f == "--p") { VAL(); a.p = std::stod(v); }
            else if (f == "--max-iter") { VAL(); a.max_iter = std::stoi(v); }
            else if (f == "--flip-hist") { VAL(); a.flip_hist = std::max(0, std::stoi(v)); }
            else if (f == "--freeze-syn") a.freeze_syn = true;
            else if (f == "--damping") { VAL(); a.damping = std::stod(v); }
            else if (f == "--simulate") a.simulate = true;
            else if (f == "--verbose") { if (i + 1 < argc && argv[i + 1][0] != '-') ++i; }
            else if (f == "--verbose-all" || f == "--report-fail" || f == "--report-ets") {}
            else if (f == "--seed") { VAL(); a.seed = std::stoull(v); a.seed_set = true; }
            else if (f == "--ets6-x") { VAL(); a.ets6_x = v; }
            else if (f == "--ets6-z") { VAL(); a.ets6_z = v; }
            else if (f == "--ets12-x" || f == "--ets-x") { VAL(); a.ets12_x = v; }
            else if (f == "--ets12-z" || f == "--ets-z") { VAL(); a.ets12_z = v; }
            else if (f == "--ets8-path4") { VAL(); a.ets8_path4 = v; }
            else if (f == "--trials") { VAL(); a.trials = std::stoll(v); }
            else if (f == "--min-fails") { VAL(); a.min_fails = std::stoll(v); }
            else if (f == "--report-every") { VAL(); a.report_every = std::stoll(v); }
            else if (f == "--progress-every") { VAL(); a.progress_every = std::stoll(v); }
            else if (f == "--iter-hist-out") { VAL(); a.hist_out = v; }
            else if (f == "--save-fail-prefix") { VAL(); }
            else if (f == "--progress-tsv") { VAL(); a.progress_tsv = v; }
            else if (f == "--no-pp") a.enable_pp = false;
            else if (f == "--cuda" || f == "--cuda-graph") {}
            else if (f == "--cuda-device") { VAL(); a.device = std::stoi(v); }
            else if (f == "--learned-order") {
                VAL();
                if (v == "model") a.learned_order = 0;
                else if (v == "llr") a.learned_order = 1;
                else {
                    std::cerr << "--learned-order must be model or llr\n";
                    return 1;
                }
            }
            else if (f == "--cuda-devices") {
                VAL();
                a.devices.clear();
                std::stringstream ds(v);
                for (std::string t; std::getline(ds, t, ',');)
                    if (!t.empty()) a.devices.push_back(std::stoi(t));
                if (a.devices.empty()) {
                    std::cerr << "--cuda-devices needs a list of device indices (e.g. 0,1,2,3)\n";
                    return 1;
                }
            }
            else if (f == "--cuda-check-warmup") { VAL(); a.check_warmup = std::max(0, std::stoi(v)); }
            else if (f == "--cuda-check-interval") { VAL(); a.check_interval = std::max(0, std::stoi(v)); }
            else if (f == "--trial-index") { VAL(); a.trial_index = std::stoll(v); }
            else if (f == "--precision") {
                VAL();
                const std::string s = v;
                if (s == "fp64") a.precision = JBP_PREC_FP64;
                else if (s == "fp32") a.precision = JBP_PREC_FP32;
                else if (s == "fp16") a.precision = JBP_PREC_FP16;
                else { std::cerr << "--precision must be fp64, fp32 or fp16\n"; return 1; }
            } else if (f == "--sampler") {
                VAL();
                const std::string s = v;
                if (s == "mt19937") a.sampler = JBP_SAMPLER_MT19937;
                else if (s == "philox") a.sampler = JBP_SAMPLER_PHILOX;
                else { std::cerr << "--sampler must be mt19937 or philox\n"; return 1; }
            } else if (f == "--engine") {
                VAL();
                const std::string s = v;
                if (s == "auto") a.engine = JBP_ENGINE_AUTO;
                else if (s == "resident") a.engine = JBP_ENGINE_RESIDENT;
                else if (s == "slots") a.engine = JBP_ENGINE_SLOTS;
                else if (s == "table") a.engine = JBP_ENGINE_TABLE;
                else { std::cerr << "--engine must be auto, resident, slots or table\n"; return 1; }
            } else if (f == "--learned-from") { VAL(); a.learned_from = std::max(0, std::stoi(v)); }
            else if (f == "--flip-model") { VAL(); a.flip_model = v; }
            else if (f == "--checks") { VAL(); a.checks = v; }
            else if (f == "--mixed") { VAL(); a.mixed = v; }
            else if (f == "--autotune") a.autotune = true;
            else if (f == "--p-max") { VAL(); a.p_max = std::stod(v); }
            else if (f == "--slots") { VAL(); a.slots = std::stoi(v); }
            else if (f == "--batch") { VAL(); a.batch = std::max(1LL, std::stoll(v)); }
            else if (f == "--ets-dir") { VAL(); a.ets_dir = v; }
            else {
                std::cerr << "Unknown argument: " << f << "\n";
                usage(argv[0]);
                return 1;
            }
        } catch (const std::exception &) {
            std::cerr << "Invalid value for " << f << "\n";
            return 1;
        }
#undef VAL
    }
    return 0;
}

// ETS groups in the reference order and default paths (jointbp_ets.cpp:5031-5337), with the
// per-file overrides of --ets6-x/-z, --ets12-x/-z and --ets8-path4.
int load_ets(jbp_ctx *ctx, const Args &a) {
    const std::string dir = a.ets_dir.empty() ? basename_no_ext(a.params) : a.ets_dir;
    const int sizes[] = {6, 8, 10, 12, 14, 16, 18, 20, 22};
    for (int s : sizes) {
        const std::string def = dir + "/ets_" + std::to_string(s) + "_2.txt";
        std::string px = def, pz = def;
        if (s == 6) {
            if (!a.ets6_x.empty()) px = a.ets6_x;
            if (!a.ets6_z.empty()) pz = a.ets6_z;
        } else if (s == 12) {
            if (!a.ets12_x.empty()) px = a.ets12_x;
            if (!a.ets12_z.empty()) pz = a.ets12_z;
        }
        if (jbp_add_ets_group(ctx, s, std::to_string(s).c_str(), px.c_str(), pz.c_str()) != JBP_OK) return 1;
        if (s == 8) {
            const std::string p4 = a.ets8_path4.empty() ? dir + "/ets_8_2_path4.txt" : a.ets8_path4;
            if (jbp_add_ets_group(ctx, 8, "8p4", p4.c_str(), p4.c_str()) != JBP_OK) return 1;
        }
    }
    return 0;
}

jbp_options options(const Args &a) {
    jbp_options o;
    jbp_default_options(&o);
    o.precision = a.precision;
    o.max_iter = a.max_iter;
    o.damping = a.damping;
    o.flip_hist = a.flip_hist;
    o.enable_pp = a.enable_pp ? 1 : 0;
    o.freeze_syn = a.freeze_syn ? 1 : 0;
    o.check_warmup = a.check_warmup;
    o.check_interval = a.check_interval;
    o.slots = a.slots;
    o.engine = a.engine;
    o.learned_from = a.learned_from;
    o.learned_order = a.learned_order;
    o.p_max = a.p_max;
    // --iter-hist-out reports measured per-phase costs: time the slot engine's kernels
    if (!a.hist_out.empty()) o.profile = 1;
    return o;
}

// Learned flip-proposal parameters from a NumPy .npy file (format 1.0/2.0, little-endian
// float32 '<f4', C order, jbp_mlp_param_count() values).  Returns an error or "".
std::string load_npy_f32(const std::string &path, std::vector<float> &out, size_t count) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return "cannot open " + path;
    char magic[8];
    if (!in.read(magic, 8) || std::memcmp(magic, "\x93NUMPY", 6) != 0) return path + ": not a .npy file";
    size_t hlen = 0;
    if (magic[6] == 1) {
        unsigned char b[2];
        if (!in.read(reinterpret_cast<char *>(b), 2)) return path + ": truncated header";
        hlen = b[0] | (b[1] << 8);
    } else {
        unsigned char b[4];
        if (!in.read(reinterpret_cast<char *>(b), 4)) return path + ": truncated header";
        hlen = b[0] | (b[1] << 8) | (b[2] << 16) | (static_cast<size_t>(b[3]) << 24);
    }
    std::string hdr(hlen, '\0');
    if (!in.read(&hdr[0], static_cast<std::streamsize>(hlen))) return path + ": truncated header";
    if (hdr.find("'<f4'") == std::string::npos || hdr.find("True") != std::string::npos)
        return path + ": expected little-endian float32 in C order";
    out.resize(count);
    if (!in.read(reinterpret_cast<char *>(out.data()), static_cast<std::streamsize>(count * sizeof(float))))
        return path + ": fewer than " + std::to_string(count) + " values";
    return "";
}

// Sets the learned flip model when --learned-from is given (the shipped model by default).
int setup_flip_model(jbp_ctx *ctx, const Args &a, const char *argv0) {
    if (a.learned_from <= 0 || a.learned_order == 1) return 0;   // the |LLR| order needs no model
    std::string path = a.flip_model;
    if (path.empty()) {
        // <repo>/joint_bp_plus_pp_b200/bin/jointbp_b200 -> ../data/flip_mlp_params.npy
        std::string self = argv0;
        const size_t sl = self.find_last_of('/');
        path = (sl == std::string::npos ? std::string(".") : self.substr(0, sl)) + "/../data/flip_mlp_params.npy";
    }
    std::vector<float> prm;
    const std::string e = load_npy_f32(path, prm, static_cast<size_t>(jbp_mlp_param_count()));
    if (!e.empty()) {
        std::cerr << e << "\n";
        return 1;
    }
    if (jbp_set_flip_model(ctx, prm.data()) != JBP_OK) {
        std::cerr << jbp_last_error() << "\n";
        return 1;
    }
    return 0;
}

void add_stats(jbp_stats &acc, const jbp_stats &s) {
    acc.trials += s.trials;
    acc.failures += s.failures;
    acc.bp_fail += s.bp_fail;
    acc.pp_success += s.pp_success;
    acc.flip_pp_success += s.flip_pp_success;
    acc.osd_pp_success += s.osd_pp_success;
    acc.stab_success += s.stab_success;
    acc.ets_used += s.ets_used;
    acc.ets_saved += s.ets_saved;
    acc.ets6_used += s.ets6_used;
    acc.ets6_saved += s.ets6_saved;
    acc.ets12_used += s.ets12_used;
    acc.ets12_saved += s.ets12_saved;
    acc.exact += s.exact;
    acc.total_iters += s.total_iters;
    acc.device_ms += s.device_ms;
    acc.kernel_launches += s.kernel_launches;
    acc.bp_trial_iterations += s.bp_trial_iterations;
    acc.check_ms += s.check_ms;
    acc.var_ms += s.var_ms;
    acc.profiled_iterations += s.profiled_iterations;
    acc.learned_attempts += s.learned_attempts;
    acc.learned_success += s.learned_success;
    acc.test_ms += s.test_ms;
    acc.syndrome_tests += s.syndrome_tests;
}

// --iter-hist-out (write_hist_out, jointbp_ets.cpp:4623-4643): "# costs <iter_cost_ms>
// <check_cost_ms>", then "iterations fraction" lines.  The reference's costs are the CUDA path's
// BP kernel time per iteration and syndrome-check time per check, and are always 0 there
// (cuda_costs is never set, jointbp_ets.cpp:4866).  Here they are measured with CUDA events:
// on the slot engine, the check- and variable-node kernels' device time per trial-iteration and
// the syndrome-test kernel's device time per trial test, amortized over the batch; on the
// trial-resident and table kernels, whose phases run inside one launch, the whole kernel's
// device time per trial-iteration, with no separate syndrome-test cost (the test rides in the
// next check phase).  A third comment line says which; '#' lines are skipped by readers of the
// format (visualize_costs.py).
bool write_hist_out(const std::string &path, const std::vector<long long> &hist, long long total, const jbp_stats &s) {
    if (path.empty() || total <= 0 || hist.size() <= 1) return true;
    std::ofstream h(path);
    if (!h) return false;
    const bool slots = s.check_ms + s.var_ms > 0.0;
    const double ti = static_cast<double>(std::max(1LL, s.bp_trial_iterations));
    const double iter_cost = slots ? (s.check_ms + s.var_ms) / ti : s.device_ms / ti;
    const double check_cost = slots && s.syndrome_tests > 0 ? s.test_ms / static_cast<double>(s.syndrome_tests) : 0.0;
    h << "# costs " << std::fixed << std::setprecision(8) << iter_cost << " " << std::setprecision(8) << check_cost
      << "\n";
    if (slots)
        h << "# cost_source slots: check + variable node kernels, device ms per trial-iteration; syndrome-test "
             "kernel, device ms per trial test (CUDA events, amortized over the batch)\n";
    else
        h << "# cost_source resident: whole kernel, device ms per trial-iteration (sampling, BP, post-processing, "
             "classification); the syndrome test rides in the check phase and has no separate cost\n";
    h << "# iter fraction\n";
    for (size_t i = 1; i < hist.size(); ++i)
        if (hist[i]) h << i << " " << std::setprecision(10) << static_cast<double>(hist[i]) / total << "\n";
    return true;
}

void print_section(const char *name) { std::cout << "== " << name << " ==\n"; }

int decode_single(jbp_ctx *ctx, const Args &a, int n, int mx, int mz) {
    const jbp_options o = options(a);
    std::vector<uint8_t> est(n);
    jbp_trial_result r{};
    jbp_stats st{};
    const auto t0 = std::chrono::steady_clock::now();
    int rc;
    if (!a.err_path.empty()) {
        std::vector<int> e;
        if (!read_ints(a.err_path, e)) {
            std::cerr << "Failed to read error vector from " << a.err_path << "\n";
            return 1;
        }
        if (static_cast<int>(e.size()) != n) {
            std::cerr << "Error vector size mismatch\n";
            return 1;
        }
        std::vector<uint8_t> e8(n);
        for (int i = 0; i < n; ++i) {
            if (e[i] < 0 || e[i] > 3) {
                std::cerr << "Error vector has invalid value\n";
                return 1;
            }
            e8[i] = static_cast<uint8_t>(e[i]);
        }
        rc = jbp_decode_errors(ctx, &o, 1, e8.data(), a.p, est.data(), &r, &st);
    } else {
        if (a.sx_path.empty() || a.sz_path.empty()) {
            std::cerr << "--sx and --sz are required unless --simulate is set\n";
            return 1;
        }
        std::vector<int> sx, sz;
        if (!read_ints(a.sx_path, sx) || !read_ints(a.sz_path, sz)) {
            std::cerr << "Failed to read syndrome files\n";
            return 1;
        }
        if (static_cast<int>(sx.size()) != mx || static_cast<int>(sz.size()) != mz) {
            std::cerr << "Syndrome size mismatch\n";
            return 1;
        }
        std::vector<uint8_t> sx8(mx), sz8(mz);
        for (int i = 0; i < mx; ++i) sx8[i] = sx[i] ? 1 : 0;
        for (int i = 0; i < mz; ++i) sz8[i] = sz[i] ? 1 : 0;
        rc = jbp_decode_syndromes(ctx, &o, 1, sx8.data(), sz8.data(), a.p, est.data(), &r, &st);
    }
    if (rc != JBP_OK) {
        std::cerr << "decode failed: " << jbp_last_error() << "\n";
        return 1;
    }
    const double lat = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    const bool ok = r.syndrome_ok;
    const bool with_err = !a.err_path.empty();
    const bool success = with_err ? r.success != 0 : ok;
    // single-decode flags (jointbp_ets.cpp:5732-5735): ets_pp_ok / flip_pp_ok of this decode
    const bool ets_ok = r.pp_ets, flip_ok = r.pp_flip, osd_ok = r.reserved;
    const bool pp_success = success && (r.pp_in_decode || ets_ok || flip_ok || osd_ok);
    print_section("Decode Result");
    std::cout << "iterations=" << r.iterations << " syndrome_match=" << tf(ok) << "\n";
    std::cout << "decode_success=" << tf(success) << "\n";
    std::cout << "pp_enabled=" << tf(a.enable_pp) << "\n";
    std::cout << "pp_success=" << tf(pp_success) << "\n";
    std::cout << "pp_success_ets=" << tf(success && ets_ok) << "\n";
    std::cout << "pp_success_flip=" << tf(success && flip_ok) << "\n";
    std::cout << "avg_latency=" << latency_str(lat) << "\n";
    if (with_err) {
        std::cout << "exact_match=" << tf(r.exact) << "\n";
        std::cout << "stabilizer_equiv=" << tf(r.stab_equiv) << "\n";
    }
    if (!a.est_path.empty()) {
        if (!write_vector(a.est_path, est.data(), n)) {
            std::cerr << "Failed to write estimate to " << a.est_path << "\n";
            return 1;
        }
        std::cout << "Saved estimate: " << a.est_path << "\n";
    }
    if (!a.hist_out.empty() && a.max_iter >= 1 && r.iterations >= 1 && r.iterations <= a.max_iter) {
        std::vector<long long> h1(static_cast<size_t>(a.max_iter) + 1, 0);
        h1[r.iterations] = 1;
        if (!write_hist_out(a.hist_out, h1, 1, st)) std::cerr << "Failed to write histogram output: " << a.hist_out << "\n";
    }
    return success ? 0 : 2;
}

// --progress-tsv (write_progress_tsv, jointbp_ets.cpp:5085-5122): the file holds the latest
// progress line only (rewritten each time), tab-separated: epoch seconds, trials, failures,
// pp_success, ETS saves, flip saves, stab_success, avg_iter, iterations, FER, trials/s, and the
// "PROGRESS | ..." text of format_progress_line (jointbp_ets.cpp:4575-4602).  Written after
// every GPU batch.
bool write_progress_tsv(const std::string &path, const jbp_stats &s, double elapsed) {
    if (s.trials <= 0) return true;
    std::ofstream out(path, std::ios::trunc);
    if (!out) return false;
    const double fer = static_cast<double>(s.failures) / static_cast<double>(s.trials);
    const double fps = elapsed > 0.0 ? static_cast<double>(s.trials) / elapsed : 0.0;
    const double avg = static_cast<double>(s.total_iters) / static_cast<double>(s.trials);
    std::ostringstream line;
    line << "PROGRESS | trials=" << s.trials << " | failures=" << s.failures << " | pp_success=" << s.pp_success
         << " | ets_success=" << s.ets_saved << " | flip_success=" << s.flip_pp_success
         << " | stab_success=" << s.stab_success << " | avg_iter=" << std::setprecision(2) << std::fixed << avg
         << " | iters=" << s.total_iters << " | FER=" << std::setprecision(6) << fer
         << " | trials/sec=" << std::setprecision(2) << fps;
    out << static_cast<long long>(std::time(nullptr)) << "\t" << s.trials << "\t" << s.failures << "\t"
        << s.pp_success << "\t" << s.ets_saved << "\t" << s.flip_pp_success << "\t" << s.stab_success << "\t"
        << std::setprecision(2) << std::fixed << avg << "\t" << s.total_iters << "\t" << std::setprecision(6) << fer
        << "\t" << std::setprecision(2) << fps << "\t" << line.str() << "\n";
    return static_cast<bool>(out);
}

void progress_line(std::ostream &os, const jbp_stats &s, double elapsed) {
    const double fer = s.trials ? static_cast<double>(s.failures) / s.trials : 0.0;
    os << "progress trials=" << s.trials << " failures=" << s.failures << " bp_fail=" << s.bp_fail
       << " pp_success=" << s.pp_success << " fer=" << std::fixed << std::setprecision(6) << fer
       << " fps=" << std::setprecision(2) << (elapsed > 0 ? s.trials / elapsed : 0.0) << " avg_iter="
       << (s.trials ? static_cast<double>(s.total_iters) / s.trials : 0.0) << " gpu_ms=" << s.device_ms << "\n";
}

// Run Summary (jointbp_ets.cpp:6419-6448), the gpu line and --iter-hist-out of a finished run.
void print_run_summary(const Args &a, const jbp_stats &acc, const std::vector<long long> &hist, double elapsed) {
    const long long d = acc.trials;
    const double fer = d ? static_cast<double>(acc.failures) / d : 0.0;
    double lo = 0.0, hi = 0.0;
    const bool ci = wilson(d, acc.failures, 1.96, lo, hi);
    print_section("Run Summary");
    std::cout << "trials=" << d << " failures=" << acc.failures << " bp_fail=" << acc.bp_fail
              << " pp_success=" << acc.pp_success << " flip_pp_success=" << acc.flip_pp_success
              << " stab_success=" << acc.stab_success << " ets_used=" << acc.ets_used << " ets_saved=" << acc.ets_saved
              << " ets6_used=" << acc.ets6_used << " ets6_saved=" << acc.ets6_saved << " ets12_used=" << acc.ets12_used
              << " ets12_saved=" << acc.ets12_saved << " fer=" << std::setprecision(8) << std::fixed << fer;
    if (ci) std::cout << " ci95=[" << std::setprecision(8) << lo << "," << hi << "]";
    std::cout << " iters=" << acc.total_iters << " avg_iter=" << std::setprecision(2)
              << (d ? static_cast<double>(acc.total_iters) / d : 0.0)
              << " avg_latency=" << latency_str(d ? elapsed / d : 0.0) << " exact_rate=" << std::setprecision(6)
              << (d ? static_cast<double>(acc.exact) / d : 0.0) << " elapsed_s=" << std::setprecision(2) << elapsed
              << "s\n";
    std::cout << "gpu: precision=" << (a.precision == JBP_PREC_FP64 ? "fp64" : a.precision == JBP_PREC_FP32 ? "fp32"
                                                                                                               : "fp16")
              << " sampler=" << (a.sampler == JBP_SAMPLER_MT19937 ? "mt19937" : "philox") << " device_ms="
              << std::setprecision(2) << acc.device_ms << " trials_per_s=" << (elapsed > 0 ? d / elapsed : 0.0)
              << "\n";
    if (!a.hist_out.empty() && d > 0 && !write_hist_out(a.hist_out, hist, d, acc))
        std::cerr << "Failed to write histogram output: " << a.hist_out << "\n";
}

int simulate(jbp_ctx *ctx, const Args &a, int n) {
    if (a.trials <= 0) {
        std::cerr << "--trials must be positive in --simulate mode\n";
        return 1;
    }
    if (a.trials != 1 && !a.est_path.empty()) {
        std::cerr << "--est is only supported with --trials 1\n";
        return 1;
    }
    jbp_options o = options(a);
    if (a.autotune) {
        jbp_options best;
        double rate = 0.0;
        if (jbp_autotune(ctx, &o, a.p, std::min<long long>(16384, std::max<long long>(1024, a.trials)), &best, &rate) !=
            JBP_OK) {
            std::cerr << "autotune failed: " << jbp_last_error() << "\n";
            return 1;
        }
        o = best;
        std::cout << "autotune: engine=" << (o.engine == JBP_ENGINE_RESIDENT ? "resident" : "slots")
                  << " slots=" << o.slots << " iters_per_launch=" << o.iters_per_launch
                  << " check_interval=" << o.check_interval << " probe_trials_per_s="
                  << std::fixed << std::setprecision(0) << rate << "\n";
    }
    const long long first = a.trial_index >= 0 ? a.trial_index : 1;
    std::vector<long long> hist(static_cast<size_t>(a.max_iter) + 1, 0), chunk_hist(hist.size());
    std::vector<jbp_trial_result> per;
    jbp_stats acc{};
    const auto t0 = std::chrono::steady_clock::now();
    long long done = 0, next_report = a.report_every > 0 ? a.report_every : -1;
    while (done < a.trials && !g_interrupted) {
        const long long cnt = std::min(a.batch, a.trials - done);
        jbp_stats st{};
        std::fill(chunk_hist.begin(), chunk_hist.end(), 0);
        if (a.min_fails > 0) per.resize(cnt);
        const int rc = jbp_simulate(ctx, &o, a.seed, first + done, cnt, a.p, a.sampler, &st,
                                    a.min_fails > 0 ? per.data() : nullptr, chunk_hist.data());
        if (rc == JBP_ERR_ABORTED) {   // interrupted: keep the trials that finished
            add_stats(acc, st);
            for (size_t i = 0; i < hist.size(); ++i) hist[i] += chunk_hist[i];
            done += st.trials;
            break;
        }
        if (rc != JBP_OK) {
            std::cerr << "simulate failed: " << jbp_last_error() << "\n";
            return 1;
        }
        if (a.min_fails > 0 && acc.failures + st.failures >= a.min_fails) {
            // stop at the trial that reaches --min-fails, as the reference loop does: decode the
            // prefix again (same trial indices, same errors) for its exact counters
            long long need = a.min_fails - acc.failures, cut = 0;
            for (long long t = 0; t < cnt && need > 0; ++t, ++cut) need -= per[t].success ? 0 : 1;
            std::fill(chunk_hist.begin(), chunk_hist.end(), 0);
            if (jbp_simulate(ctx, &o, a.seed, first + done, cut, a.p, a.sampler, &st, nullptr, chunk_hist.data()) !=
                JBP_OK) {
                std::cerr << "simulate failed: " << jbp_last_error() << "\n";
                return 1;
            }
            add_stats(acc, st);
            for (size_t i = 0; i < hist.size(); ++i) hist[i] += chunk_hist[i];
            done += cut;
            break;
        }
        add_stats(acc, st);
        for (size_t i = 0; i < hist.size(); ++i) hist[i] += chunk_hist[i];
        done += cnt;
        const double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (next_report > 0 && done >= next_report) {
            progress_line(std::cout, acc, el);
            while (next_report <= done) next_report += a.report_every;
        }
        if (!a.progress_tsv.empty() && !write_progress_tsv(a.progress_tsv, acc, el)) {
            std::cerr << "Failed to write progress TSV: " << a.progress_tsv << "\n";
            return 1;
        }
    }
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!a.est_path.empty()) {
        std::vector<uint8_t> err(n), est(n);
        jbp_trial_result r{};
        jbp_stats st{};
        if (jbp_sample_errors(ctx, a.seed, first, 1, a.p, a.sampler, err.data()) != JBP_OK ||
            jbp_decode_errors(ctx, &o, 1, err.data(), a.p, est.data(), &r, &st) != JBP_OK) {
            std::cerr << "decode failed: " << jbp_last_error() << "\n";
            return 1;
        }
        if (!write_vector(a.est_path, est.data(), n)) {
            std::cerr << "Failed to write estimate to " << a.est_path << "\n";
            return 1;
        }
        std::cout << "Saved estimate: " << a.est_path << "\n";
    }
    if (g_interrupted) std::cerr << "interrupted: " << done << " of " << a.trials << " trials decoded\n";
    print_run_summary(a, acc, hist, elapsed);
    return g_interrupted ? 130 : 0;
}

// --cuda-devices: the trial range split into contiguous parts, one per listed device (a device
// may be listed twice), each decoded by its own context on its own host thread in batches of
// --batch; the counters and histograms are summed into one Run Summary.  Trials are keyed by
// (seed, trial index), so the summary equals that of one device decoding the whole range.
int simulate_multi(const std::vector<jbp_ctx *> &ctxs, const Args &a) {
    if (a.trials <= 0) {
        std::cerr << "--trials must be positive in --simulate mode\n";
        return 1;
    }
    if (a.min_fails > 0 || !a.est_path.empty() || a.autotune || !a.progress_tsv.empty()) {
        std::cerr << "--cuda-devices does not take --min-fails, --est, --autotune or --progress-tsv\n";
        return 1;
    }
    const jbp_options o = options(a);
    const long long first = a.trial_index >= 0 ? a.trial_index : 1;
    const int D = static_cast<int>(ctxs.size());
    std::vector<jbp_stats> st(D);
    std::vector<std::vector<long long>> hist(D, std::vector<long long>(static_cast<size_t>(a.max_iter) + 1, 0));
    std::vector<std::string> errs(D);
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> pool;
    for (int d = 0; d < D; ++d) {
        pool.emplace_back([&, d]() {
            const long long lo = first + a.trials * d / D, hi = first + a.trials * (d + 1) / D;
            std::vector<long long> h(hist[d].size());
            std::memset(&st[d], 0, sizeof(jbp_stats));
            for (long long b = lo; b < hi; b += a.batch) {
                const long long cnt = std::min(a.batch, hi - b);
                jbp_stats s{};
                std::fill(h.begin(), h.end(), 0);
                if (g_interrupted) return;
                const int rc = jbp_simulate(ctxs[d], &o, a.seed, b, cnt, a.p, a.sampler, &s, nullptr, h.data());
                if (rc == JBP_ERR_ABORTED) {   // interrupted: keep the trials that finished
                    add_stats(st[d], s);
                    for (size_t i = 0; i < h.size(); ++i) hist[d][i] += h[i];
                    return;
                }
                if (rc != JBP_OK) {
                    errs[d] = jbp_last_error();
                    return;
                }
                add_stats(st[d], s);
                for (size_t i = 0; i < h.size(); ++i) hist[d][i] += h[i];
            }
        });
    }
    for (auto &t : pool) t.join();
    for (int d = 0; d < D; ++d)
        if (!errs[d].empty()) {
            std::cerr << "simulate failed on device " << a.devices[d] << ": " << errs[d] << "\n";
            return 1;
        }
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    jbp_stats acc{};
    std::vector<long long> all(hist[0].size(), 0);
    for (int d = 0; d < D; ++d) {
        add_stats(acc, st[d]);
        for (size_t i = 0; i < all.size(); ++i) all[i] += hist[d][i];
    }
    std::cout << "devices=" << D << " trials_per_device=" << (a.trials + D - 1) / D << "\n";
    if (g_interrupted) std::cerr << "interrupted: " << acc.trials << " of " << a.trials << " trials decoded\n";
    print_run_summary(a, acc, all, elapsed);
    return g_interrupted ? 130 : 0;
}

// A code as check lists ('n mx mz', then the variables of each X check and of each Z check, one
// check per line).  Returns false (after a message) when the file cannot be read.
bool read_checks_file(const std::string &path, int &n, int m[2], std::vector<int> off[2], std::vector<int> var[2]) {
    std::ifstream in(path);
    n = 0;
    m[0] = m[1] = 0;
    if (!in || !(in >> n >> m[0] >> m[1]) || n <= 0 || m[0] <= 0 || m[1] <= 0) {
        std::cerr << "Failed to read checks: " << path << "\n";
        return false;
    }
    std::string line;
    std::getline(in, line);
    for (int s = 0; s < 2; ++s) {
        off[s].assign(1, 0);
        var[s].clear();
        for (int c = 0; c < m[s]; ++c) {
            if (!std::getline(in, line)) {
                std::cerr << "Failed to read checks: " << path << " (too few lines)\n";
                return false;
            }
            std::istringstream ls(line);
            int v;
            while (ls >> v) var[s].push_back(v);
            off[s].push_back(static_cast<int>(var[s].size()));
        }
    }
    return true;
}

// --mixed: the codes of several check-list files decoded in one launch (jbp_simulate_mixed).
int simulate_mixed_files(const Args &a) {
    if (!a.simulate) {
        std::cerr << "--mixed requires --simulate\n";
        return 1;
    }
    if (a.enable_pp) {
        std::cerr << "--mixed decodes with plain BP: add --no-pp\n";
        return 1;
    }
    std::vector<std::string> files;
    std::stringstream ss(a.mixed);
    for (std::string f; std::getline(ss, f, ',');)
        if (!f.empty()) files.push_back(f);
    std::vector<jbp_ctx *> ctxs;
    auto cleanup = [&]() {
        for (jbp_ctx *c : ctxs) jbp_destroy(c);
    };
    std::vector<int> ns;
    for (const std::string &f : files) {
        int n = 0, m[2];
        std::vector<int> off[2], var[2];
        if (!read_checks_file(f, n, m, off, var)) {
            cleanup();
            return 1;
        }
        jbp_ctx *c = nullptr;
        if (jbp_create_from_checks(n, m[0], off[0].data(), var[0].data(), m[1], off[1].data(), var[1].data(),
                                   a.device, &c) != JBP_OK) {
            std::cerr << "init failed: " << f << ": " << jbp_last_error() << "\n";
            cleanup();
            return 1;
        }
        ctxs.push_back(c);
        ns.push_back(n);
    }
    const int k = static_cast<int>(ctxs.size());
    std::vector<uint64_t> seeds(k);
    std::vector<long long> first(k, a.trial_index >= 0 ? a.trial_index : 1), ntrials(k, a.trials);
    for (int i = 0; i < k; ++i) seeds[i] = a.seed + static_cast<uint64_t>(i);
    std::vector<jbp_stats> st(k);
    const jbp_options o = options(a);
    const auto t0 = std::chrono::steady_clock::now();
    const int rc = jbp_simulate_mixed(ctxs.data(), k, &o, seeds.data(), first.data(), ntrials.data(), a.p, st.data(),
                                      nullptr);
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != JBP_OK) {
        std::cerr << "mixed run failed: " << jbp_last_error() << "\n";
        cleanup();
        return 1;
    }
    long long total = 0;
    for (int i = 0; i < k; ++i) {
        const long long d = st[i].trials;
        total += d;
        double lo = 0.0, hi = 0.0;
        const bool ci = wilson(d, st[i].failures, 1.96, lo, hi);
        print_section(("Run Summary (" + files[i] + ")").c_str());
        std::cout << "n=" << ns[i] << " trials=" << d << " failures=" << st[i].failures << " fer=" << std::fixed
                  << std::setprecision(8) << (d ? static_cast<double>(st[i].failures) / d : 0.0);
        if (ci) std::cout << " ci95=[" << lo << "," << hi << "]";
        std::cout << " iters=" << st[i].total_iters << " avg_iter=" << std::setprecision(2)
                  << (d ? static_cast<double>(st[i].total_iters) / d : 0.0) << " exact_rate=" << std::setprecision(6)
                  << (d ? static_cast<double>(st[i].exact) / d : 0.0) << "\n";
    }
    std::cout << "gpu: mixed launch of " << k << " codes, kernel_launches=" << (k ? st[0].kernel_launches : 0)
              << " device_ms=" << std::setprecision(2) << (k ? st[0].device_ms : 0.0)
              << " trials_per_s=" << (elapsed > 0 ? total / elapsed : 0.0) << "\n";
    cleanup();
    return 0;
}

}  // namespace

// One decoding context on `device`: the code (params file or check lists), the ETS tables when
// post-processing is on, and the learned flip model when asked for.  Returns 0, or 1 after a
// message.
int create_context(const Args &a, int device, const char *argv0, jbp_ctx **out) {
    jbp_ctx *ctx = nullptr;
    if (!a.checks.empty()) {
        // a code given as check lists (no ETS tables)
        int n = 0, m[2];
        std::vector<int> off[2], var[2];
        if (!read_checks_file(a.checks, n, m, off, var)) return 1;
        if (jbp_create_from_checks(n, m[0], off[0].data(), var[0].data(), m[1], off[1].data(), var[1].data(),
                                   device, &ctx) != JBP_OK) {
            std::cerr << "init failed: " << jbp_last_error() << "\n";
            return 1;
        }
    } else {
        if (!exists(a.params)) {
            std::cerr << "Failed to read params: " << a.params << "\n";
            return 1;
        }
        if (jbp_create_from_params(a.params.c_str(), nullptr, device, &ctx) != JBP_OK) {
            std::cerr << "init failed: " << jbp_last_error() << "\n";
            return 1;
        }
    }
    if (a.enable_pp && a.checks.empty() && load_ets(ctx, a)) {
        std::cerr << "ETS load failed: " << jbp_last_error() << "\n";
        jbp_destroy(ctx);
        return 1;
    }
    if (setup_flip_model(ctx, a, argv0)) {
        jbp_destroy(ctx);
        return 1;
    }
    *out = ctx;
    return 0;
}

int main(int argc, char **argv) {
    Args a;
    const int prc = parse(argc, argv, a);
    if (prc == 2) return 0;
    if (prc) return 1;
    if (!a.seed_set) {
        a.seed = static_cast<unsigned long long>(std::chrono::duration_cast<std::chrono::microseconds>(
                                                     std::chrono::system_clock::now().time_since_epoch())
                                                     .count());
    }
    if (!a.mixed.empty()) return simulate_mixed_files(a);
    if (a.params.empty() && a.checks.empty()) {
        std::cerr << "--params is required\n";
        return 1;
    }
    if (a.simulate && !a.err_path.empty()) {
        std::cerr << "--err cannot be used with --simulate\n";
        return 1;
    }
    if (a.simulate && a.trial_index >= 0 && (a.trials != 1 || a.min_fails > 0)) {
        std::cerr << "--trial-index requires --trials 1 and no --min-fails\n";
        return 1;
    }
    if (!a.simulate) {
        if (a.trials != 1 || a.min_fails > 0) {
            std::cerr << "--trials/--min-fails are only valid with --simulate\n";
            return 1;
        }
        if (!a.err_path.empty() && (!a.sx_path.empty() || !a.sz_path.empty())) {
            std::cerr << "--err cannot be combined with --sx/--sz\n";
            return 1;
        }
    }
    if (!a.devices.empty() && !a.simulate) {
        std::cerr << "--cuda-devices requires --simulate\n";
        return 1;
    }
    std::vector<int> devs = a.devices.empty() ? std::vector<int>{a.device} : a.devices;
    std::vector<jbp_ctx *> ctxs;
    auto destroy_all = [&]() {
        for (jbp_ctx *c : ctxs) jbp_destroy(c);
    };
    for (int dev : devs) {
        jbp_ctx *c = nullptr;
        if (create_context(a, dev, argv[0], &c)) {
            destroy_all();
            return 1;
        }
        ctxs.push_back(c);
    }
    jbp_ctx *ctx = ctxs[0];
    int n = 0, mx = 0, mz = 0, rx = 0, rz = 0, ng = 0;
    jbp_code_info(ctx, &n, &mx, &mz, &rx, &rz, &ng);
    print_section("Code Summary");
    const int k = n - rx - rz;
    std::cout << "p=" << std::fixed << std::setprecision(6) << a.p << " n=" << n << " mx=" << mx << " mz=" << mz
              << " rank_x=" << rx << " rank_z=" << rz << " stab_rank=" << rx + rz << " k=" << k
              << " rate=" << (n ? static_cast<double>(k) / n : 0.0) << " ets_groups=" << ng << "\n";
    {
        long long odd = 0;
        int gx = 0, gz = 0;
        if (jbp_code_graph_checks(ctx, &odd, &gx, &gz) == JBP_OK) {
            print_section("Graph Checks");
            std::cout << "hx_hz_orthogonal=" << (odd == 0 ? "true" : "false") << "  hx_hz_odd_pairs=" << odd
                      << "  girth_x=" << gx << "  girth_z=" << gz << "\n";
        }
    }
    install_interrupt(ctxs);
    const int rc = !a.devices.empty() ? simulate_multi(ctxs, a)
                   : (a.simulate ? simulate(ctx, a, n) : decode_single(ctx, a, n, mx, mz));
    std::signal(SIGINT, SIG_DFL);   // no abort request may reach a destroyed context
    g_abort_ctxs.clear();
    destroy_all();
    return rc;
}
