// Host side of the batched engine.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "code_model.hpp"
#include "engine.cuh"

namespace jbp {

struct ResCode;

struct RunRequest {
    jbp_options opt{};
    int source = kSrcPhilox;
    unsigned long long seed = 0;
    long long first_trial = 1;
    long long ntrials = 0;
    double p = 0.05;
    const uint8_t *d_err = nullptr;     // source buffers (device)
    const uint8_t *d_sx = nullptr;
    const uint8_t *d_sz = nullptr;
    uint8_t *d_est_out = nullptr;       // outputs (device, optional)
    float *d_llr_out = nullptr;         // [ntrials][n][2] final LLRs (diagnostics)
    jbp_trial_result *d_res_out = nullptr;
    unsigned long long *d_hist = nullptr;
    cudaStream_t stream = nullptr;
    // Optional pinned host buffers for copies of d_res_out / d_est_out.  The single-trial path
    // queues those copies behind its launches and waits once for all of them, then sets
    // *host_copied; other paths leave the buffers and the flag alone.
    jbp_trial_result *h_res_out = nullptr;
    uint8_t *h_est_out = nullptr;
    bool *host_copied = nullptr;
    // stall-state collection for training the learned proposal (device buffers)
    bool collect = false;
    float *d_col_x = nullptr, *d_col_y = nullptr;
    unsigned long long *d_col_count = nullptr;
    long long col_cap = 0;
};

class Engine;

// Mixed-size Monte Carlo in one launch (kernels_mixed.cuh): the codes of several engines on
// one device, trials first_trial[i] .. of code i with seed seeds[i].
struct MixedRequest {
    std::vector<Engine *> engines;
    jbp_options opt{};
    std::vector<unsigned long long> seeds;
    std::vector<long long> first_trial, ntrials;
    double p = 0.05;
    std::vector<jbp_trial_result *> d_res;   // per code, optional device buffers
    std::vector<unsigned long long *> d_hist;  // per code, optional iteration histograms [max_iter + 1]
    std::vector<const uint8_t *> d_err;        // per code, optional given errors instead of Philox noise
    std::vector<uint8_t *> d_est;              // per code, optional estimates
    std::vector<float *> d_llr;                // per code, optional final LLRs
    cudaStream_t stream = nullptr;
};

class Engine {
public:
    Engine() = default;
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    std::string init(CodeModel model, int device);
    const CodeModel &model() const { return model_; }
    int device() const { return device_; }
    std::string run(const RunRequest &rq, jbp_stats &stats);
    // Device sampler output (trial-major) into a device buffer.
    std::string sample_errors(unsigned long long seed, long long first, long long count, double p, int source,
                              uint8_t *d_out);
    const DevCode &dev_code() const { return dcode_; }
    // Learned flip proposal parameters (FP32, mlp.cuh layout); null removes the model.
    std::string set_flip_model(const float *params);
    int sm_count() const { return sm_count_; }
    // Asks the run in progress (or the next run) to stop; any host thread (jbp_request_abort).
    void request_abort() {
        if (abort_host_) *abort_host_ = 1;
    }
    bool abort_requested() const { return abort_host_ && *abort_host_ != 0; }
    void clear_abort() {
        if (abort_host_) *abort_host_ = 0;
    }
    // One launch over the codes of rq.engines; stats[i] for code i.
    static std::string run_mixed(const MixedRequest &rq, std::vector<jbp_stats> &stats);

private:
    struct Buffers {
        int S = 0, precision = -1;
        bool damp = false;
        size_t msg_bytes = 0;
        void *msg[6] = {};            // c2v x/z, v2c x/z, v2c_hi x/z
        long long *trial = nullptr;
        int *iter = nullptr, *flags = nullptr, *frz = nullptr, *unsat = nullptr;
        unsigned *unsat_mask = nullptr, *estx = nullptr, *estz = nullptr, *synm = nullptr;
        double *prior = nullptr, *slot_p = nullptr;
        float *lprior = nullptr;
        uint8_t *err = nullptr;
        int *res_iters = nullptr, *res_flags = nullptr;
        int *lists = nullptr;         // retired | fresh | groups
        int *counts = nullptr;        // n_retired, n_fresh, n_groups, n_pp
        DevCounters *cnt = nullptr;
        unsigned long long *h_done = nullptr;  // pinned
        int *it = nullptr;            // global iteration counter
        // post-processing state (allocated when a run enables it)
        bool pp = false;
        int R = 1;
        int *act_k = nullptr, *pstate = nullptr, *stall_same = nullptr, *pp_list = nullptr, *pp_mode = nullptr;
        unsigned short *us_hist = nullptr;
        unsigned *dprev = nullptr, *dpprev = nullptr;
        unsigned char *pp_scratch = nullptr;
        size_t pp_stride = 0;
        int pp_blocks = 0;
    };

    // Trial-resident tier (kernels_resident.cuh): whether a run can use it, and the run.
    bool resident_applies(const jbp_options &o, std::string *why) const;
    std::string run_resident(const RunRequest &rq, jbp_stats &stats);
    std::string run_dispatch(const RunRequest &rq, jbp_stats &stats);
    // one or a few FP64 trials, each in one cooperative launch (kernels_single.cuh)
    bool single_applies(const RunRequest &rq) const;
    bool single_fits(const void *fn);
    std::vector<std::pair<const void *, bool>> single_fit_;   // per kernel: all blocks co-resident
    static constexpr size_t kSingleCntOffset = 64;   // single_cnt_ within the control allocation
    std::string run_single(const RunRequest &rq, jbp_stats &stats);
    static std::string run_mixed_impl(const MixedRequest &rq, std::vector<jbp_stats> &stats);
    std::string build_res_code();

    std::string ensure_buffers(int S, int precision, bool damp, bool pp, int R, cudaStream_t st);
    std::string upload_ets();
    void free_buffers();
    int choose_slots(const jbp_options &opt, long long ntrials) const;

    // the neighbour tables of the mixed launch, built on first use
    std::string mixed_slots();

    // The slot engine's instantiated CUDA graph of its last run without profiling, reused by a
    // run whose launch parameters are byte for byte the same (the per-trial calls of a
    // cuda_bp_decode loop decode through the same staging buffers): capturing and
    // instantiating a graph costs more than decoding one trial.
    struct SlotGraph {
        bool valid = false;
        DevRun r{};
        DevMsgs msg{};
        int precision = -1, GI = 0;
        double damping = 0.0;
        bool llr_out = false, device_loop = false;
        cudaGraphExec_t exec = nullptr;
        long long per_graph = 0;
    };
    SlotGraph slot_graph_;
    cudaEvent_t run_ev_[4] = {nullptr, nullptr, nullptr, nullptr};   // start, end, two polls

    int device_ = 0;
    int sm_count_ = 0;
    volatile int *abort_host_ = nullptr;   // jbp_request_abort's flag, mapped pinned host memory
    // the single-trial FP64 path: messages [c2v x, c2v z, v2c x, v2c z], decisions when the caller
    // gives no buffer, barrier / test counters / error flag, counters
    bool coop_launch_ = false;   // the device runs cooperative launches (the single-trial path)
    void *single_msg_[4] = {};
    uint8_t *single_est_ = nullptr;
    // the single-trial path's barrier, test counts and error flag (single_ctl_, 8 ints) and its
    // counters (single_cnt_) in one allocation, copied back in one transfer to single_host_
    int *single_ctl_ = nullptr;
    DevCounters *single_cnt_ = nullptr;
    unsigned char *single_host_ = nullptr;   // pinned
    const volatile int *abort_dev_ = nullptr;   // ... the device's address of it (the kernels poll it)
    const uint16_t *mix_slot_[2] = {nullptr, nullptr};   // [dv][n] message slot of each variable's edges
    const uint16_t *mix_chk_[2] = {nullptr, nullptr};    // [dc][m] variable of each check's edges
    unsigned char *mix_scratch_ = nullptr;   // per-block c2v of the codes that do not fit shared memory
    size_t mix_scratch_bytes_ = 0;
    DevCounters *mix_cnt_ = nullptr;         // kMixMaxCodes counters + the work counter
    int smem_optin_ = 0;
    bool res_code_ok_ = false;
    std::string res_code_why_;
    ResCode *rcode_ = nullptr;
    DevCounters *res_cnt_ = nullptr;
    unsigned char *res_pp_scratch_ = nullptr;
    size_t res_pp_bytes_ = 0;
    unsigned char *res_c2v_scratch_ = nullptr;   // FP32 messages of the resident tier, per block
    size_t res_c2v_bytes_ = 0;
    uint32_t *mlp_dev_ = nullptr;
    bool has_mlp_ = false;
    CodeModel model_;
    DevCode dcode_{};
    std::vector<void *> code_allocs_;
    Buffers buf_;
    DevEts dets_{};
    size_t ets_uploaded_ = static_cast<size_t>(-1);  // ETS groups in dets_
    std::vector<void *> ets_allocs_;
};

std::string cuda_err(cudaError_t e, const char *what);

// Every device and (mapped) pinned-host allocation of the library goes through these, so that the test
// hook jbp_debug_fail_allocation can make the n-th one fail (cudaErrorMemoryAllocation, without
// calling the runtime): the failure path of each allocation site is exercised from the host.
cudaError_t dev_malloc_bytes(void **p, size_t bytes);
cudaError_t host_malloc_pinned(void **p, size_t bytes);
template <class T>
inline cudaError_t dev_malloc(T **p, size_t bytes) {
    return dev_malloc_bytes(reinterpret_cast<void **>(p), bytes);
}
template <class T>
inline cudaError_t host_malloc(T **p, size_t bytes) {
    return host_malloc_pinned(reinterpret_cast<void **>(p), bytes);
}
// after >= 0: the allocation that many allocations from now fails (0 = the next), once; < 0: off.
void set_alloc_failure(long long after);

// The option checks every decoding entry point shares (error rate, prior, precision, damping,
// engine, iteration and time limits): "" when the options are valid, else why not.
std::string validate_options(const jbp_options &o, double p);

}  // namespace jbp
