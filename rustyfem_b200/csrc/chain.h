// Solve chains: the sweeps of the top levels of the tree (levels with few fronts) in one
// chain launch per level and direction (chain.cu), plus one fully parallel launch for the
// fronts' later rows (after the forward chain, before the backward one). The plan's chain
// items say which WS-wide diagonal blocks a level has; each is done by a cluster of four
// CTAs, which takes items in the plan's order from a counter and waits (bounded) on the
// flags of the blocks the item depends on.
//
// Flag region of a sweep (int words, zeroed before the sweep): forward block flags
// [0, chain_blocks), backward block flags [chain_blocks, 2·chain_blocks), then the work
// counter of each level and direction (2·nlevels). A block's flag counts the CTAs of its
// cluster that have published their part of y (four when the block is done).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "plan.h"

namespace rfg {

inline int64_t chain_flag_words(const Plan& P) { return 2 * P.chain_blocks + 2 * P.nlevels; }

// The inverse of every chain block's unit-lower diagonal block, WS × WS in FP64 (row-major,
// zero above the diagonal and beyond the block's width), from the NB × NB inverses of the
// factorization and the FP32 factor: cinv[(cb·WS + r)·WS + c].
void launch_chain_inverse(double* cinv, const float* panel, const double* linv, const DFront* fronts,
                          const int64_t* chain_blk, const int64_t* chain_bfront, int64_t nblocks, cudaStream_t st);

// Forward chain of one level: Y[pivot rows] = L⁻¹ x for the level's fronts, X (with the
// children's update vectors added) as the right-hand side. items: the level's (front,
// block) pairs; flags: the forward block flags; counter: the level's work counter; err: set
// to 1 when a wait gave up (sticky).
void launch_chain_fwd(int nrhs, int64_t nitems, const double* X, double* Y, const float* panel, const double* cinv,
                      const DFront* fronts, const int64_t* chain_blk, const int64_t* items, int* flags, int* counter,
                      int* err, cudaStream_t st);

// After a level's forward chain: V[later rows] −= L21·y, items the (front, piece) pairs of
// the level's later rows.
void launch_chain_rows(int nrhs, int64_t nitems, const double* Y, double* V, const float* panel, const DFront* fronts,
                       const int64_t* items, cudaStream_t st);

// Before a level's backward chain: the solution of the fronts' later rows gathered into V
// (gather_items: the level's later-row pieces), then z[pivot columns] −= L21ᵀ·y_later
// (items: the level's pivot-column pieces), z the scaled forward result in Y; part holds
// the row groups' partial sums (CHAIN_GROUPS · CHAIN_PIECE · nrhs values per item).
void launch_chain_cols(int nrhs, int64_t ngather, const int64_t* gather_items, int64_t nitems, const int64_t* items,
                       double* Y, double* V, double* part, const float* panel, const DFront* fronts,
                       const int64_t* rows, cudaStream_t st);

// Backward chain of one level: Y[pivot rows] = L11⁻ᵀ z.
void launch_chain_bwd(int nrhs, int64_t nitems, double* Y, const float* panel, const double* cinv,
                      const DFront* fronts, const int64_t* chain_blk, const int64_t* items, int* flags, int* counter,
                      int* err, cudaStream_t st);

}  // namespace rfg
