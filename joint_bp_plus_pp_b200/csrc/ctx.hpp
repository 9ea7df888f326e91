// The C-ABI context (opaque jbp_ctx in include/jbp_b200.h) and the shared error reporting
// of the C entry points.
#pragma once

#include <cuda_runtime.h>

#include <string>

#include "../../include/jbp_b200.h"
#include "engine.hpp"

struct jbp_ctx {
    jbp::Engine engine;
    // the context's own non-blocking stream for the host-buffer calls, so that contexts used
    // from different host threads decode concurrently on one device
    cudaStream_t stream = nullptr;
    // cached device staging for host-buffer calls
    uint8_t *d_in = nullptr, *d_in2 = nullptr, *d_est = nullptr;
    size_t in_bytes = 0, in2_bytes = 0, est_bytes = 0;
    jbp_trial_result *d_res = nullptr;
    size_t res_count = 0;
    unsigned long long *d_hist = nullptr;
    size_t hist_count = 0;
    float *d_llr = nullptr;
    size_t llr_count = 0;
    // pinned host staging of calls of a few trials (inputs, then results)
    unsigned char *h_stage = nullptr;
    size_t h_stage_bytes = 0;
    ~jbp_ctx() {
        if (stream) cudaStreamDestroy(stream);
        cudaFree(d_in);
        cudaFree(d_in2);
        cudaFree(d_est);
        cudaFree(d_res);
        cudaFree(d_hist);
        cudaFree(d_llr);
        if (h_stage) cudaFreeHost(h_stage);
    }
};

namespace jbp {
// Records msg as the calling thread's last error (jbp_last_error) and returns code.
int set_last_error(int code, const std::string &msg);
}  // namespace jbp
