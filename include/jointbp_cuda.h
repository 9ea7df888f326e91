/* The reference's GPU boundary (jointbp_cuda.h:1-93 of NagatsukiSep/joint_BP_plus_PP),
 * implemented by lib/libjointbp_cuda.so over the C ABI of jbp_b200.h.
 *
 * The types must stay layout-compatible with the reference header, because the reference
 * host program (jointbp_ets.cpp, built with -DUSE_CUDA) includes its own copy of the header
 * and links against this library instead of jointbp_cuda.cu.  Member names, types and order
 * therefore follow the reference; the semantics of each call are described below.
 *
 *   cuda_bp_create   jointbp_cuda.h:46   builds a decoder from the CSR graph (check-major
 *                                        edge numbering of build_cuda_graph,
 *                                        jointbp_ets.cpp:937-1016)
 *   cuda_bp_destroy  jointbp_cuda.h:47
 *   cuda_bp_decode   jointbp_cuda.h:48-62  one decode from a syndrome pair
 *
 * Differences from the reference implementation (jointbp_cuda.cu):
 *   - the arithmetic is the reference CPU decoder's (bit-exact in FP64, the default), not the
 *     reference GPU kernels'; JBP_CUDA_PRECISION=fp32|fp16 in the environment selects the
 *     LLR decoders instead;
 *   - `iterations` of a trial that does not converge is max_iter, as the CPU path reports
 *     (jointbp_cuda.cu:1077 reports max_iter + 1);
 *   - use_graph is accepted and ignored: every decode runs from CUDA graphs;
 *   - check_kernel_ms, check_memcpy_ms and init_kernel_ms are 0; kernel_ms is the device time
 *     of the decode and host_ms the rest of the call's wall time.
 */
#pragma once

#include <string>
#include <vector>

struct CudaMsg {
    double v[4];  /* probabilities of I, X, Z, Y */
};

struct CudaBPGraph {
    int nvars = 0;
    int mX = 0;
    int mZ = 0;
    int x_edges = 0;
    int z_edges = 0;
    std::vector<int> x_check_offsets;  /* mX + 1 */
    std::vector<int> x_check_edges;    /* edge ids of each check, in check order */
    std::vector<int> x_edge_var;       /* variable of each edge */
    std::vector<int> x_edge_check;
    std::vector<int> x_edge_pos;
    std::vector<int> x_var_offsets;
    std::vector<int> x_var_edges;
    std::vector<int> z_check_offsets;
    std::vector<int> z_check_edges;
    std::vector<int> z_edge_var;
    std::vector<int> z_edge_check;
    std::vector<int> z_edge_pos;
    std::vector<int> z_var_offsets;
    std::vector<int> z_var_edges;
};

struct CudaBPResult {
    std::vector<int> est;       /* nvars Pauli indices 0..3 */
    int iterations = 0;
    int check_count = 0;        /* syndrome tests made (schedule of check_warmup / check_interval) */
    bool syndrome_match = false;
    double kernel_ms = 0.0;
    double memcpy_ms = 0.0;
    double check_kernel_ms = 0.0;
    double check_memcpy_ms = 0.0;
    double init_kernel_ms = 0.0;
    double host_ms = 0.0;
};

struct CudaBPContext;

CudaBPContext *cuda_bp_create(const CudaBPGraph &graph, int device_id, std::string *error_out);
void cuda_bp_destroy(CudaBPContext *ctx);
bool cuda_bp_decode(CudaBPContext *ctx, const std::vector<int> &sx, const std::vector<int> &sz, const CudaMsg &prior,
                    int max_iter, int check_warmup, int check_interval, bool measure_costs, bool use_graph,
                    bool freeze_syn, double damping, CudaBPResult &out, std::string *error_out);
