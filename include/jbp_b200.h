/* jbp_b200.h -- C ABI of the B200 joint X/Z BP + post-processing decoder.
 *
 * Plain C types only.  One context per code and device; a context is not thread-safe
 * (calls on one context must not overlap).  Every entry point returns JBP_OK (0) or an
 * error code; jbp_last_error() gives the message of the calling thread's last failure.
 * No entry point falls back to the CPU: a missing or failing GPU is an error.
 *
 * Reference interfaces replaced (file:line in NagatsukiSep/joint_BP_plus_PP):
 *   jbp_create_*      <- cuda_bp_create            jointbp_cuda.h:46, jointbp_cuda.cu:589-642
 *                        + code construction       jointbp_ets.cpp:162-180, 98-160, 628-648
 *   jbp_add_ets_group <- read_ets_file / ETS load  jointbp_ets.cpp:3199-3258, 5212-5337
 *   jbp_destroy       <- cuda_bp_destroy           jointbp_cuda.h:47, jointbp_cuda.cu:644-679
 *   jbp_decode_*      <- cuda_bp_decode            jointbp_cuda.h:48-62, jointbp_cuda.cu:681-1104
 *                        (batched; + post-processing and success test the reference
 *                        runs on the CPU: jointbp_ets.cpp:5487-5730)
 *   jbp_simulate      <- the --simulate trial loop jointbp_ets.cpp:5931-6449
 */
#ifndef JBP_B200_H
#define JBP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JBP_OK 0
#define JBP_ERR_ARG 1          /* invalid argument or size mismatch */
#define JBP_ERR_CUDA 2         /* CUDA runtime error or no usable device */
#define JBP_ERR_IO 3           /* file missing or malformed */
#define JBP_ERR_UNSUPPORTED 4  /* combination not built for the GPU */
#define JBP_ERR_TIMEOUT 5      /* device watchdog expired (see jbp_options.watchdog_ms) */
#define JBP_ERR_ABORTED 6      /* stopped by jbp_request_abort; stats hold the trials finished */

#define JBP_PREC_FP64 0        /* probability-domain messages, bit-exact with the reference CPU */
#define JBP_PREC_FP32 1        /* LLR messages in FP32 */
#define JBP_PREC_FP16 2        /* LLR messages stored in FP16, FP32 arithmetic */

/* Decoding engines.  RESIDENT: one persistent thread block per SM keeps a whole trial's BP
 * state in shared memory (FP16 precision on quasi-cyclic affine codes such as the shipped APM
 * code).  SLOTS: trials in HBM-resident slots, one kernel per BP phase (every precision and
 * option).  AUTO picks RESIDENT where it applies, else SLOTS.  TABLE (explicit only): the
 * table-driven persistent kernel of jbp_simulate_mixed on this one code -- plain BP on Philox
 * noise or given errors (not syndromes), FP32 arithmetic with FP32 or FP16 message storage, any
 * code whose checks have one degree (6, 7, 8 or 12) and whose variables have degree <= 4 per
 * side. */
#define JBP_ENGINE_AUTO 0
#define JBP_ENGINE_RESIDENT 1
#define JBP_ENGINE_SLOTS 2
#define JBP_ENGINE_TABLE 3

#define JBP_SAMPLER_PHILOX 0   /* counter-based Philox4x32-10 keyed by (seed, trial index) */
#define JBP_SAMPLER_MT19937 1  /* the reference stream: splitmix64 seed -> mt19937_64 per trial */

typedef struct jbp_ctx jbp_ctx;

typedef struct {
    int precision;         /* JBP_PREC_* (default FP64) */
    int max_iter;          /* >= 1 (default 50, as --max-iter) */
    double damping;        /* 0..1 (default 0, as --damping) */
    int flip_hist;         /* flip-history window (default 5, as --flip-hist; clamped >= 0) */
    int enable_pp;         /* ETS / flip / OSD post-processing (default 1; 0 = --no-pp) */
    int freeze_syn;        /* --freeze-syn */
    int check_warmup;      /* --cuda-check-warmup (default 0) */
    int check_interval;    /* --cuda-check-interval (default 1, clamped >= 1) */
    int slots;             /* trials in flight; 0 = automatic */
    int iters_per_launch;  /* BP iterations per CUDA-graph launch; 0 = automatic */
    int watchdog_ms;       /* run budget (0 = none): a run that takes longer stops early with
                              JBP_ERR_TIMEOUT and its stats hold the trials finished within it.
                              Persistent kernels (resident, table, mixed) check the GPU's global
                              timer between trials and every 16 BP iterations of a trial, and
                              abandon unfinished trials; the slot engine checks on the host
                              between CUDA-graph launches */
    int profile;           /* time the check and variable kernels with CUDA events (jbp_stats) */
    int use_prior;         /* 1: decode with `prior` below instead of normalize(1-p, p/3, p/3, p/3) */
    double prior[4];       /* probabilities of I, X, Z, Y (used as given, as cuda_bp_decode does) */
    int engine;            /* JBP_ENGINE_* (default AUTO) */
    double p_max;          /* > p: each trial's error rate is drawn uniformly from [p, p_max), keyed by
                              (seed, trial index); jbp_simulate only; 0 = every trial at p */
    int learned_from;      /* > 0: from this iteration on, a stalled trial (decisions unchanged or
                              oscillating) first tries the learned flip proposal set with
                              jbp_set_flip_model (resident engine, post-processing on); 0 = off */
    int learned_order;     /* column order of that proposal: 0 = the model's scores (default);
                              1 = the decoder's own |LLR| order (least reliable first), the same
                              trigger, elimination and acceptance without the network -- the
                              baseline the network is measured against; needs no model */
    int learned_cols;      /* qubits (columns) of that proposal's GF(2) elimination, taken in the
                              column order above (0 = 512) */
    int collect_every;     /* jbp_collect_stall_states: of the qubits that are next to no
                              unsatisfied check and whose estimate is right, record 1 in this many
                              (0 = 32; 1 = every qubit, a sample without selection bias) */
} jbp_options;

/* Per-trial outcome (16 bytes). */
typedef struct {
    int32_t iterations;    /* as the reference CPU reports: convergence iteration, else max_iter */
    uint8_t syndrome_ok;   /* final estimate reproduces the syndrome */
    uint8_t bp_ok;         /* plain BP converged */
    uint8_t success;       /* syndrome_ok and residual is a stabilizer (needs the true error) */
    uint8_t exact;         /* estimate equals the true error */
    uint8_t stab_equiv;    /* residual in the stabilizer row space */
    uint8_t pp_success;    /* counted in pp_success */
    uint8_t pp_ets;        /* ETS stage produced the final estimate */
    uint8_t pp_flip;       /* flip stage produced the final estimate */
    uint8_t pp_osd;        /* OSD counted (reference osd_success) */
    uint8_t ets_used_flags;/* bit0 ETS used, bit1 size 6, bit2 size 12, bit3 post-BP ETS applied,
                              bit4 post-BP stages ran, bit5 a learned flip proposal was accepted */
    uint8_t pp_in_decode;  /* post-processing succeeded inside the BP loop */
    uint8_t reserved;
} jbp_trial_result;

/* Run counters with the reference Run Summary keys (jointbp_ets.cpp:6428-6449). */
typedef struct {
    long long trials, failures, bp_fail, pp_success, flip_pp_success, osd_pp_success, stab_success;
    long long ets_used, ets_saved, ets6_used, ets6_saved, ets12_used, ets12_saved;
    long long exact, total_iters;
    double device_ms;          /* device time of the run (CUDA events) */
    long long kernel_launches; /* this library's kernels launched by the run */
    long long bp_trial_iterations; /* BP iterations summed over trials */
    double check_ms;           /* with profile: device time of all check-node kernel launches */
    double var_ms;             /* with profile: device time of all variable-node kernel launches */
    long long profiled_iterations; /* with profile: BP iterations (launch pairs) timed */
    long long slots;           /* trials in flight used by the run */
    long long learned_attempts;/* learned flip proposals evaluated */
    long long learned_success; /* trials whose accepted learned proposal was a success */
    double test_ms;            /* with profile (slot engine): device time of all syndrome-test kernel launches */
    long long syndrome_tests;  /* slot engine: per-trial syndrome tests run (the resident and table kernels
                                  fuse the test into the next check phase and do not count it) */
} jbp_stats;

void jbp_default_options(jbp_options *opt);
const char *jbp_last_error(void);
const char *jbp_version(void);
/* Test hook (fault injection on the host): the device or pinned-host allocation `after`
 * allocations from now (0 = the next one) fails with JBP_ERR_CUDA ("out of memory"), once,
 * without calling the CUDA runtime; after < 0 turns the hook off.  Process-wide.  Every
 * allocation failure leaves the context usable: the next call allocates again.  No counterpart
 * in the reference (whose allocation failures end in its CPU fallback). */
int jbp_debug_fail_allocation(long long after);
/* Asks the run in progress on ctx (from any host thread), or the next run if none is in
 * progress, to stop: the persistent kernels claim no further trial (they look at the flag, a
 * pinned host word, at every 8th trial they claim and every 16 iterations of a trial past
 * iteration 64), the slot engine ends its iteration loop, and the run returns JBP_ERR_ABORTED
 * with the counters of the trials that finished (jbp_stats is filled as for JBP_ERR_TIMEOUT).
 * The flag clears when that run returns.  No counterpart in the reference. */
int jbp_request_abort(jbp_ctx *ctx);

int jbp_create_from_params(const char *params_path, const char *ets_dir, int device, jbp_ctx **out);
int jbp_create_from_checks(int n, int mx, const int *x_off, const int *x_var, int mz, const int *z_off,
                           const int *z_var, int device, jbp_ctx **out);
int jbp_add_ets_group(jbp_ctx *ctx, int size, const char *label, const char *path_x, const char *path_z);
void jbp_destroy(jbp_ctx *ctx);

/* n, mx, mz, rank_x, rank_z, number of ETS groups loaded (any pointer may be null). */
int jbp_code_info(jbp_ctx *ctx, int *n, int *mx, int *mz, int *rank_x, int *rank_z, int *ets_groups);
/* Check lists (check-major, x_var has x_off[mx] entries); sizes from jbp_code_info. */
int jbp_code_checks(jbp_ctx *ctx, int side, int *off, int *var);

/* Start-up graph checks (check_hx_hz_orthogonality and compute_girth, jointbp_ets.cpp:1070-1171):
 * odd_pairs = the (X check, Z check) pairs sharing an odd number of variables (0: Hx Hz^T = 0),
 * girth_x / girth_z = the girth of each side's Tanner graph (0 without a cycle).  Any pointer
 * may be null.  jbp_graph_checks takes check lists (as jbp_create_from_checks) and needs no GPU. */
int jbp_code_graph_checks(jbp_ctx *ctx, long long *odd_pairs, int *girth_x, int *girth_z);
int jbp_graph_checks(int n, int mx, const int *x_off, const int *x_var, int mz, const int *z_off, const int *z_var,
                     long long *odd_pairs, int *girth_x, int *girth_z);

/* Monte Carlo: trials first_trial .. first_trial+ntrials-1 of base seed `seed` at error rate p.
 * per_trial (host, ntrials entries) and iter_hist (host, max_iter+1 entries) may be null. */
int jbp_simulate(jbp_ctx *ctx, const jbp_options *opt, uint64_t seed, long long first_trial, long long ntrials,
                 double p, int sampler, jbp_stats *stats, jbp_trial_result *per_trial, long long *iter_hist);

/* Decode known errors (host buffers): err is ntrials x n bytes in {0,1,2,3}; the syndromes
 * are computed on the device.  est_out (ntrials x n, may be null) receives the estimates. */
int jbp_decode_errors(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *err, double p,
                      uint8_t *est_out, jbp_trial_result *res, jbp_stats *stats);

/* Decode syndromes (host buffers): sx is ntrials x mx bits (one byte each), sz ntrials x mz.
 * success/exact/stab fields stay 0 (no true error).  Calls of at most three trials (the
 * drop-in's cuda_bp_decode decodes one) copy their inputs through pinned memory the context
 * keeps; FP64 and FP32 ones without post-processing, damping, frozen sides, profile or run
 * budget decode each trial in one cooperative launch and wait once for the whole call. */
int jbp_decode_syndromes(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *sx,
                         const uint8_t *sz, double p, uint8_t *est_out, jbp_trial_result *res, jbp_stats *stats);

/* jbp_decode_errors with the final LLRs of every trial (precision diagnostics): llr_out is
 * ntrials x n x 2 floats, the natural log of P(bit = 1) / P(bit = 0) of each qubit's x bit and
 * z bit from the check-to-variable messages the trial ends with.  With the syndrome tested only
 * at max_iter (check_warmup >= max_iter) these are the messages of its last iteration for every
 * trial; a trial that stops earlier may end with one more check update. */
int jbp_decode_errors_llr(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *err, double p,
                          float *llr_out, jbp_trial_result *res, jbp_stats *stats);

/* Device-resident variants: every pointer is device memory of the context's device and
 * the call is ordered on `stream` (a cudaStream_t, 0 = legacy default stream). */
int jbp_decode_errors_device(jbp_ctx *ctx, const jbp_options *opt, long long ntrials, const uint8_t *d_err,
                             double p, uint8_t *d_est_out, jbp_trial_result *d_res, jbp_stats *stats, void *stream);

/* Allocation-free decoding.  No counterpart in the reference: it is for callers that cannot
 * call cudaMalloc while they decode (device memory owned by another allocator, or decoding
 * loops that must not allocate after start-up).  It runs the slot engine's kernels: its results
 * equal jbp_decode_syndromes with engine JBP_ENGINE_SLOTS (engine must be AUTO or SLOTS; plain BP:
 * enable_pp, freeze_syn, damping and learned_from must be off), but d_sx (ntrials x mx),
 * d_sz (ntrials x mz), d_est_out (ntrials x n, may be null) and d_res (ntrials) are device
 * memory, the work is ordered on `stream`, and all temporary state lives in a fixed device
 * array of JBP_NOALLOC_SCRATCH_BYTES that the library holds on every GPU that loads it until
 * the process exits; the call allocates nothing.  Requests that do not fit (about 32 trials
 * of the shipped code in FP64, 128 in FP32) are rejected with JBP_ERR_ARG.  The first call on
 * a device looks up the array's device address, so make it before any stream capture.  All
 * calls share the array: calls that overlap on the GPU race and must be serialized.  The
 * options are checked before any CUDA call; the caller's current device is left unchanged. */
#define JBP_NOALLOC_SCRATCH_BYTES (64u << 20)
int jbp_decode_syndromes_noalloc(jbp_ctx *ctx, const jbp_options *opt, int ntrials, const uint8_t *d_sx,
                                 const uint8_t *d_sz, double p, uint8_t *d_est_out, jbp_trial_result *d_res,
                                 void *stream);

/* Learned flip proposal (no counterpart in the reference): a 3-layer MLP (8 -> 64 -> 64 -> 2,
 * ReLU) over per-qubit features of a stalled BP state -- the four normalized log2 weights of
 * I, X, Z, Y, the x-bit and z-bit flips over the last 5 iterations, and the unsatisfied X and
 * Z checks at the qubit -- whose two logits propose flipping the qubit's x-bit and z-bit.  A
 * proposal is applied only if both syndromes then match exactly.  Parameters: FP32, the
 * layout W1[64][8], b1[64], W2[64][64], b2[64], W3[2][64], b3[2] (jbp_mlp_param_count()).
 * Features x are nsamples x 8 floats, labels y nsamples x 2 floats (0/1), host buffers. */
int jbp_mlp_param_count(void);

/* Measured FP32 special-function throughput of a device (G results/s for the whole GPU) for
 * ex2, lg2 and rcp (approx, flush-to-zero), the operations of the BP check and variable
 * rules: the denominators of the SFU roofline the resident and table-driven kernels report.
 * No counterpart in the reference.  About 10 ms of GPU time. */
int jbp_measure_sfu(int device, double *ex2_gops, double *lg2_gops, double *rcp_gops);
/* Device self-check of the FP64 kernels' branch-free reciprocal (three Newton steps from the
 * hardware approximation and an exact-remainder choice of the nearest double) against the
 * correctly rounded division 1.0 / s, on n divisors in [2^-900, 2^900] drawn from seed (random
 * significands, all-ones significands, powers of two and their neighbours).  mismatches gets
 * the count, first_mismatch (may be null) the index of the first, or -1.  No counterpart in the
 * reference: the bit-exact FP64 decoder depends on it.  About 1 ms of GPU time per 10^8. */
int jbp_check_reciprocal(int device, unsigned long long seed, long long n, long long *mismatches,
                         long long *first_mismatch);
/* Device self-check of the us-signal oscillation test of the post-processing trigger
 * (detect_us_oscillation, jointbp_ets.cpp:2021-2053): the one-pass form the slot engine uses
 * and the warp-parallel form of the trial-resident kernel against the rule as written, on n
 * seeded histories (constant, noisy, alternating, ramps, spikes, steps).  mismatches gets the
 * disagreements, fired (may be null) how many histories the rule accepts. */
int jbp_check_us_oscillation(int device, unsigned long long seed, long long n, long long *mismatches,
                             long long *fired);
/* Gradient of the mean loss (binary cross-entropy with logits, positives weighted by
 * pos_weight, summed over the two outputs) on the GPU; grad_out has jbp_mlp_param_count()
 * entries. */
int jbp_mlp_grad(jbp_ctx *ctx, const float *params, long long nsamples, const float *x, const float *y,
                 float pos_weight, float *grad_out, double *loss_out);
/* Adam training on the GPU (minibatches of `batch`, reshuffled each epoch from `seed`);
 * params is updated in place; epoch_loss (epochs entries, may be null) gets each epoch's
 * mean loss. */
int jbp_mlp_train(jbp_ctx *ctx, float *params, long long nsamples, const float *x, const float *y, int epochs,
                  int batch, float lr, float pos_weight, uint64_t seed, double *epoch_loss);
/* BF16 tensor-core inference (the kernel code the decoder runs after a stall): logits is
 * nsamples x 2. */
int jbp_mlp_infer(jbp_ctx *ctx, const float *params, long long nsamples, const float *x, float *logits);
/* The model used when jbp_options.learned_from > 0 (params = NULL removes it). */
int jbp_set_flip_model(jbp_ctx *ctx, const float *params);
/* Training data: runs the Monte Carlo like jbp_simulate (resident engine, post-processing on,
 * opt->learned_from > 0 gives the first stall iteration) and, at every stall where the learned
 * proposal would run, records the features and labels (x-bit / z-bit of error xor estimate) of
 * the qubits next to an unsatisfied check, the qubits whose estimate is wrong and 1 in
 * opt->collect_every (0 = 32) of the others, up to `capacity` samples; stats->learned_attempts
 * counts the stalls recorded.  Decoding itself is unchanged. */
int jbp_collect_stall_states(jbp_ctx *ctx, const jbp_options *opt, uint64_t seed, long long first_trial,
                             long long ntrials, double p, int sampler, long long capacity, float *x_out, float *y_out,
                             long long *count_out, jbp_stats *stats);

/* Autotuner: times short Monte-Carlo probes (probe_trials trials of seed 1 at error rate p, the
 * options in *opt) over the launch choices that do not change any decoding result -- the
 * engine (resident where it applies, else slots), the slot engine's trials in flight (4096 ..
 * 32768) and its BP iterations per CUDA-graph launch (2, 4, 8) -- and writes the fastest into
 * *best (a copy of *opt with engine, slots and iters_per_launch set).  With
 * opt->check_interval == 0 it also considers the choices that change results: the syndrome-test
 * interval among 1, 2 and 4 when post-processing is off (trials stop at a multiple of the
 * interval, as with the reference's --cuda-check-interval), and for FP32 messages the resident
 * engine, whose arithmetic differs slightly from the slot engine's.  best_trials_per_s may be
 * null. */
int jbp_autotune(jbp_ctx *ctx, const jbp_options *opt, double p, long long probe_trials, jbp_options *best,
                 double *best_trials_per_s);

/* Mixed-size Monte Carlo in one kernel launch (no counterpart in the reference): the trials of
 * the codes of nctx contexts on one device -- code i decodes trials first_trial[i] ..
 * first_trial[i] + ntrials[i] - 1 of seed seeds[i] (Philox noise, per-trial p uniform in
 * [p, opt->p_max) when p_max > p) -- taken by one persistent kernel from one work queue, largest
 * code first.  Plain BP (opt->enable_pp = 0), FP32 arithmetic with FP32 (JBP_PREC_FP32) or FP16
 * (JBP_PREC_FP16) message storage; the codes' checks must all have one degree (6, 7, 8 or 12), the
 * same for every code; variables of degree <= 4 per side.  first_trial may be null (every code from trial 1); stats receives one
 * entry per code; per_trial, if not null, holds nctx host arrays (each null or ntrials[i]
 * records).  Runs on the first context's stream. */
int jbp_simulate_mixed(jbp_ctx *const *ctxs, int nctx, const jbp_options *opt, const uint64_t *seeds,
                       const long long *first_trial, const long long *ntrials, double p, jbp_stats *stats,
                       jbp_trial_result *const *per_trial);

/* Errors of trials first_trial.. drawn by a device sampler (JBP_SAMPLER_*), copied to the host
 * buffer err (ntrials x n).  The same streams jbp_simulate decodes. */
int jbp_sample_errors(jbp_ctx *ctx, uint64_t seed, long long first_trial, long long ntrials, double p, int sampler,
                      uint8_t *err);

/* Host-side sampler of the reference stream (splitmix64 + mt19937_64 + libstdc++ uniform),
 * for feeding reference-sampled errors: trials first_trial.. into err (ntrials x n). */
int jbp_sample_reference_errors(int n, uint64_t seed, long long first_trial, long long ntrials, double p,
                                uint8_t *err, int threads);

#ifdef __cplusplus
}
#endif
#endif
