// Unsymmetric multifrontal LU on the GPU, following src/sparse/lu.rs: the same
// tree as LDLᵀ with full fronts (both triangles), diagonal pivoting with the
// threshold test |a_jj| >= u·max_{i≠j} |a_ij| (u = 0.01) over the column, symmetric
// swaps, variables that fail delayed to the parent, and at the root the rest
// factored with partial pivoting (row swaps).
//
// As for the indefinite path, a front's fully summed set grows by its children's
// delayed variables, known only after the children are factored: the level loop
// runs on the host, and per level
//   k_lu_asm_orig   the level's fronts zeroed, then on all SMs the original entries
//   k_lu_asm_child  (lower triangle and transposed upper partners), then the children's
//                   full update matrices, one launch per child slot (child order kept);
//   k_lu_block      in rounds, one CTA per front (k_lu_block_cl: a cluster of 8 CTAs
//                   for fronts of 768 rows and more): the pivot search, swaps and eager
//                   updates of the block's columns (src/sparse/lu.rs:292-330); at the
//                   root, once no candidate passes, the partial-pivoting LU of the rest
//                   (:246-270);
//   k_lu_rowblock   after each round, on all SMs: the columns beyond the block of the
//                   block's rows, each entry with the reference's sequence of updates;
//   k_lu_trailing   then F[b1.., b1..] −= L·U of the block's pivots in 64×64 tiles
//                   (:331-350).
// The file is compiled without multiply-add contraction; the trailing update uses the
// reference's fused multiply-add chain per entry (src/sparse.rs:329-343).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

#include "symbolic.h"

namespace rfg {

struct LuStats {
    int64_t delayed = 0;      // delayed pivots (src/sparse/lu.rs:108-110)
    int64_t factor_size = 0;  // values of L and U (:404-406)
    double t_factor_ms = 0.0;
    int64_t launches = 0;
};

class LuEngine {
   public:
    // S: the symbolic analysis; colptr/rowidx: the lower CSC pattern (internal numbering),
    // shared by the lower triangle and the transposed strict upper triangle
    LuEngine(const Symbolic& S, const std::vector<int64_t>& colptr, const std::vector<int64_t>& rowidx,
             double threshold);
    ~LuEngine();
    // Factors A with lower values lval and transposed upper values uval (host, the pattern's
    // order: uval[p] = A(c, r) for the lower entry (r, c)). Returns -1, or the internal
    // equation at which the matrix is singular.
    int64_t factor(const double* lval, const double* uval);
    // Solves A X = B in place, X[q·nrhs + j] on the device (internal numbering).
    void solve_device(double* X, int64_t nrhs);
    const LuStats& stats() const { return stats_; }
    cudaStream_t stream() const { return stream_; }

   private:
    void release_fronts();
    const Symbolic& S_;
    std::vector<int64_t> colptr_, rowidx_;
    double thr_;
    cudaStream_t stream_ = nullptr;
    std::vector<int64_t> level_off_, level_order_;
    int64_t nlevels_ = 0;
    double* d_lval_ = nullptr;
    double* d_uval_ = nullptr;
    double* d_scale_ = nullptr;
    int64_t* d_tpre_ = nullptr;   // prefix of the trailing-update tiles over a level's fronts
    int64_t* d_rpre_ = nullptr;   // prefix of the row-block-update tiles
    int64_t* d_active_ = nullptr;
    int num_sms_ = 148;
    int64_t cluster_rows_ = 768;  // fronts from this size: block rounds on a cluster of CTAs
    void* d_desc_ = nullptr;  // LFrontDesc[nfronts]
    std::vector<void*> front_bufs_, level_bufs_;
    std::vector<int64_t> npiv_, kf_, m_;
    LuStats stats_;
};

}  // namespace rfg
