// Symmetric indefinite multifrontal LDLᵀ on the GPU (1×1 and 2×2 pivots with the
// reference's threshold rule, delayed pivots passed to the parent, Bunch–Kaufman
// at the root), following src/sparse/indef.rs.
//
// The tree is the positive definite one (same symbolic analysis), but a front's
// fully summed set grows by the pivots its children delayed, which are known
// only after the children are factored. So the level loop runs on the host: for
// each level it gathers the children's delayed variables (a small device→host
// copy per level), sizes and allocates the dense fronts, and launches
//   k_indef_asm_*      the level's fronts zeroed, then on all SMs: original entries, the
//                      children's update matrices (one launch per child slot, child order
//                      kept), the mirror of the fully summed blocks;
//   k_indef_block      in rounds, one CTA per front (k_indef_block_cl: a cluster of 8
//                      CTAs for fronts of 768 rows and more): the pivot search, swaps and
//                      eager updates of one block (src/sparse/indef.rs:416-500);
//   k_indef_trailing   after each round, on all SMs: the trailing update of each
//                      front's block in 64×64 tiles (src/sparse/indef.rs:504-532).
// The file is compiled without multiply-add contraction so that every product
// and sum the reference does separately is rounded separately; the trailing
// update uses the reference's fused multiply-add chain (src/sparse.rs:329-335).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "symbolic.h"

namespace rfg {

struct IndefStats {
    int64_t neg = 0, zero = 0, pos = 0;
    int64_t delayed = 0, two_by_two = 0;
    int64_t factor_size = 0;
    double t_factor_ms = 0.0;
    int64_t launches = 0;
};

class IndefEngine {
   public:
    // S: the symbolic analysis; colptr/rowidx: the lower CSC pattern (internal numbering)
    IndefEngine(const Symbolic& S, const std::vector<int64_t>& colptr, const std::vector<int64_t>& rowidx,
                double threshold);
    ~IndefEngine();
    // Factors the values val (host, lower CSC). Returns -1, or the internal equation at
    // which the matrix is singular (src/sparse/indef.rs:110-114).
    int64_t factor(const double* val);
    // Solves in place, X[q·nrhs + j] on the device (internal numbering).
    void solve_device(double* X, int64_t nrhs);
    const IndefStats& stats() const { return stats_; }
    cudaStream_t stream() const { return stream_; }

   private:
    void release_fronts();
    const Symbolic& S_;
    std::vector<int64_t> colptr_, rowidx_;
    double thr_;
    cudaStream_t stream_ = nullptr;
    std::vector<int64_t> level_off_, level_order_;
    int64_t nlevels_ = 0;
    // device
    int64_t* d_colptr_ = nullptr;
    int64_t* d_rowidx_ = nullptr;
    double* d_val_ = nullptr;
    double* d_scale_ = nullptr;
    int64_t* d_tpre_ = nullptr;    // prefix of trailing-update tiles over a level's fronts
    int64_t* d_active_ = nullptr;  // fronts of the level not yet done
    int num_sms_ = 148;
    int64_t cluster_rows_ = 768;  // fronts from this size: block rounds on a cluster of CTAs
    void* d_desc_ = nullptr;     // IFrontDesc[nfronts]
    std::vector<void*> front_bufs_;
    std::vector<void*> level_bufs_;
    // host copies after factorization
    std::vector<int64_t> npiv_, kf_, m_;
    // host copies of each level's D (d then e) and pivot kinds, and each front's place in them
    std::vector<std::vector<double>> lvl_d_;
    std::vector<std::vector<int8_t>> lvl_kind_;
    std::vector<int64_t> front_lvl_, front_vo_, front_vb_;
    IndefStats stats_;
};

}  // namespace rfg
