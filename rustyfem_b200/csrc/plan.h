// Device plan of the multifrontal factorization: where each front lives in
// HBM, the level-by-level schedule of the numeric phase and the index maps that
// let the GPU assemble fronts without searching.
//
// Layout. Front t (m = k + u rows) is the symmetric matrix
//     F = [F11 .; F21 F22],  F11 k×k, F21 u×k, F22 u×u,
// stored as two row-major pieces:
//   * the panel P_t = [F11; F21] (m × k, row stride ldp) in the panel arena —
//     after factorization it holds L11 (strictly lower) and L21, i.e. the factor,
//     and stays resident for the solves;
//   * the update block U_t = F22 (u × u, row stride ldu, lower triangle) in the
//     update arena — it becomes the Schur complement that the parent consumes,
//     and its memory is reused once the parent has been assembled.
// Rows are the K-major operand layout of the Schur update
// F22 −= (L21·D)·L21ᵀ: both operands are read along the pivot index.
//
// Schedule. Fronts are grouped by level (leaves at level 0, a parent one level
// above its highest child). All fronts of a level are assembled together, then
// factored together in steps of NB pivots: step s handles the pivot block
// [s·NB, min((s+1)·NB, k)) of every front of the level whose k exceeds s·NB.
// Steps come in outer blocks of NBO = 4·NB pivots [J0, J1): inside an outer
// block, a step updates only the block's remaining pivot columns (the "inner"
// update, K = NB); the step that completes the block applies the whole block to
// the trailing matrix [J1, m) at once (the "outer" update, K up to NBO), so that
// the largest updates stream the trailing matrix once per NBO pivots.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <utility>
#include <vector>

#include "symbolic.h"

namespace rfg {

constexpr int NB = 64;        // pivot block width (factor and solve steps)
constexpr int NBO = 256;      // outer block: pivots applied together to the trailing matrix
constexpr int KO = NBO / NB;
constexpr int UT = 64;        // Schur-update tile (UT × UT of F)
constexpr int PR = 128;       // panel rows per CTA
constexpr int XR = 256;       // solve: update-vector rows of one warp's extend-add task
constexpr int XT = 32;        // factor: tile (XT × XT of a child's update matrix) of one warp of the extend-add

// per-front descriptor used by the kernels (int64 everywhere: offsets exceed 2^31)
struct DFront {
    int64_t start, k, u, m;
    int64_t ldp, ldu;
    int64_t poff, uoff;       // element offsets in the panel / update arena
    int64_t parent;           // -1 for a root
    int64_t rows_off;         // rows[] offset (global equation of each later row)
    int64_t emap_off;         // emap[] offset: local index in the parent of each later row
    int64_t vuoff;            // offset (in rows) of the front's solve update vector
    int64_t blk_off;          // first of the front's NB×NB diagonal blocks in the inverse store
};

// one step s of one level: the active fronts are the first nact of the level's
// fronts sorted by decreasing k
struct DStep {
    int64_t level;
    int64_t s;                // step index: pivots [s·NB, ...)
    int64_t fr_off;           // offset in level_order (the level's sorted fronts)
    int64_t nact;
    int64_t pre_off;          // offset of this step's prefix arrays (nact + 1 entries each)
    int64_t scr_off;          // offset of the outer block's scratch prefix (rows m − J0 per front)
    int64_t out_lo;           // active fronts [out_lo, nact) complete their outer block in this step
    int64_t n_panel;          // total panel CTAs
    int64_t n_inner;          // inner-update tiles of the small-tile kernel (UT×UT)
    int64_t n_inner_tc;       // inner-update 128×128 tiles on the tensor cores (mixed, large fronts)
    int64_t n_outer;          // outer-update tiles of the small-tile kernel (UT×UT)
    int64_t n_outer_tc;       // outer-update tiles of the large-tile kernels (128×128: tensor
                              // cores in the mixed path, CUDA cores in the FP64 path)
    int64_t n_outer_tc2;      // the same trailing matrices in 128×256 tiles (persistent
                              // tensor-core kernel)
    int64_t scr_rows;         // scratch rows of the outer block
    int64_t scr_off_prev;     // the previous outer block's scratch prefix (two-block passes)
    double inner_flops;       // algorithmic flops of the inner updates
    double outer_flops;       // algorithmic flops of the outer updates
};

// One step of the solves: WS = 4·NB pivots [S·WS, min(k, (S+1)·WS)) of the active fronts
// of a level (the first nact of the level's fronts, sorted by decreasing k).
constexpr int WS = 4 * NB;
struct WStep {
    int64_t level;
    int64_t S;
    int64_t fr_off;           // offset in level_order
    int64_t nact;
    int64_t pre_off;          // offset of this step's prefix arrays (nact + 1 entries each)
    int64_t n_rows;           // CTAs of the row kernels: max(1, ⌈(m − J1)/PR⌉) per front
    int64_t n_part;           // partial-sum columns of the backward row kernel: Σ CTAs × width
};

// extend-add work of one level and one child rank
struct DXadd {
    int64_t off;              // offset into xadd_child
    int64_t task_off;         // offset (in tasks) into xadd_task
    int64_t ntask;            // solve: warp tasks (XR rows of one child each)
    int64_t nchild;
    int64_t nblk;             // solve: CTAs (eight warp tasks each)
    int64_t fpre_off;         // offset into xadd_fpre (nchild + 1 entries)
    int64_t fnblk;            // total CTAs of the factor's extend-add (eight XT × XT tiles each)
};


constexpr uint8_t PANEL_SCR = 1, PANEL_SPLIT = 2;
constexpr uint8_t OUT_NONE = 0, OUT_FULL = 1, OUT_STRIP = 2, OUT_PAIR = 3;
constexpr int TC_TILE = 128;          // tile of the large-front Schur update (tensor cores or FP64 128-tiles)
constexpr int TC_WIDE = 256;          // tile columns of the persistent tensor-core outer update (128×256)
constexpr int64_t TC_INNER_MIN_ROWS = 512;  // mixed path: rows below the step from which an inner
                                            // update runs on the tensor cores
constexpr int64_t TC_MIN_ROWS = 256;  // default: trailing rows from which an outer update uses it

struct Plan {
    int64_t nfronts = 0, nlevels = 0, n = 0;
    std::vector<DFront> fronts;
    std::vector<int64_t> level_off;     // nlevels+1 into level_order
    std::vector<int64_t> level_order;   // fronts of each level, by decreasing k
    std::vector<int64_t> level_maxk;
    std::vector<DStep> steps;           // all steps, level by level
    std::vector<int64_t> step_off;      // nlevels+1 into steps
    // prefix arrays (per step, nact+1 entries each, concatenated): panel CTAs,
    // inner tiles, outer tiles (0 for fronts before out_lo); pre_scr per outer block
    std::vector<int64_t> pre_panel, pre_inner, pre_inner_tc, pre_outer, pre_outer_tc, pre_outer_tc2, pre_scr;
    std::vector<uint8_t> front_tc_inner;  // fronts whose inner updates may run on the tensor cores
    // per step and active front (the layout of pre_panel): what the panel kernel writes
    // besides L — PANEL_SCR: the W and L rows in the storage precision (read by the
    // CUDA-core and FP64 updates), PANEL_SPLIT: their TF32 head/tail splits (read by the
    // tensor-core updates). A kind is written only when an update of the step or of the
    // step's outer block reads it.
    std::vector<uint8_t> panel_mode;
    // per step and active front (the layout of pre_panel): the kind of the front's tensor-core
    // outer update at this step (OUT_*). Two outer blocks of a front pass over its trailing
    // matrix once: the first updates only the next block's columns (OUT_STRIP), the second
    // the rest with both blocks' pivots, K up to 2·NBO (OUT_PAIR, the first block's operands
    // from the other scratch buffer: the split operands are double-buffered by the parity of
    // the outer block).
    std::vector<uint8_t> outer_mode;
    // solve steps (WS pivots wide), per level in order; prefix of row-kernel CTAs and of
    // partial-sum columns (CTAs × step width) per active front
    std::vector<WStep> wsteps;
    std::vector<int64_t> wstep_off;     // nlevels + 1
    std::vector<int64_t> pre_wrows, pre_wpart;
    int64_t max_wrows = 0, max_wpart = 0;
    // Solve chains. On the levels with at most chain_fronts fronts (the top of the tree,
    // where a step's launches have a few CTAs of work) a sweep of the FP32 factor with at
    // most four right-hand sides runs as one launch per level and direction instead of
    // two per WS-wide step: each WS-wide diagonal block of a front is one work item, done
    // by a cluster of four CTAs that waits for the blocks it depends on (chain.cu). The
    // block's solve multiplies by the inverse of its unit-lower diagonal block (WS × WS,
    // FP64), formed from the factor before the first sweep.
    std::vector<uint8_t> level_chain;    // per level: 1 when its sweeps run as chains
    std::vector<int64_t> chain_blk;      // per front: its first chain block, or -1
    std::vector<int64_t> chain_bfront;   // per chain block: its front
    int64_t chain_blocks = 0;
    // work items per level as pairs (front, diagonal block) in dependency order
    std::vector<int64_t> chain_fwd_off, chain_bwd_off;  // nlevels + 1, in items
    std::vector<int64_t> chain_fwd, chain_bwd;
    // the later rows of a chain level's fronts, one CTA per pair (front, piece of CHAIN_PIECE):
    // forward, rows k + CHAIN_PIECE·i ... (V −= L21·y after the level's chain); backward,
    // pivot columns CHAIN_PIECE·i ... (z −= L21ᵀ·y_later before it)
    std::vector<int64_t> chain_rows_off, chain_cols_off;  // nlevels + 1, in pairs
    std::vector<int64_t> chain_rows, chain_cols;
    int64_t chain_colpart = 0;  // partial sums of a level's column pieces (CHAIN_GROUPS row groups), per rhs
    std::vector<uint8_t> front_tc;      // fronts whose large outer updates run on the tensor cores
    // extend-add lists, per level and rank (2 ranks)
    std::vector<DXadd> xadd;            // 2·nlevels
    std::vector<int64_t> xadd_child;    // child ids
    std::vector<int64_t> xadd_task;     // solve: (child, parent, first row, rows) per warp task
    std::vector<int64_t> xadd_fpre;     // the same for the factor's area-balanced chunks
    SegVec rows;                        // global equation of the later rows (Symbolic::rows)
    std::vector<int32_t> emap;          // local index in the parent of each later row
    int64_t panel_elems = 0, upd_elems = 0, vu_rows = 0;
    int64_t max_scr_rows = 0;           // largest scratch over all steps
    int64_t max_nact = 0;               // largest number of active fronts of a step
    int64_t nblocks = 0;                // NB×NB diagonal blocks of all fronts
    std::vector<int64_t> front_of_dof;  // front owning each equation
    double work = 0.0;
    double inner_flops = 0.0, outer_flops = 0.0;  // Σ over all steps
    double outer_big_flops = 0.0;                 // the part of outer_flops on 128-tiles
    double outer_big_entries = 0.0;               // their trailing entries updated (Σ R(R+1)/2)
    double outer_big_opvals = 0.0;                // their operand values (Σ R·K)
    int64_t upd_peak_elems = 0;         // update arena size with reuse
    int64_t big_min_rows = 0;           // the cutover this plan was built with
    int outer_tn = TC_WIDE;             // the tensor-core outer-update tile width it was built with
    int64_t big_tiles = 0, small_tiles = 0;  // outer-update tiles of each kind, all steps
};

// Plan choices an autotuner may change; the defaults are the built-in ones.
struct Tuning {
    int64_t big_min_rows = TC_MIN_ROWS;  // small-front / large-front cutover of the outer update
    int outer_tn = TC_WIDE;              // tensor-core outer-update tile width: 128 or 256 columns
    bool pair_blocks = true;             // tensor-core outer updates in two-block passes
    int64_t chain_fronts = -1;           // solve chains on levels of at most this many fronts
                                         // (-1: RFG_SOLVE_CHAIN, else CHAIN_FRONTS; 0: none)
};
constexpr int64_t CHAIN_FRONTS = 16;
constexpr int64_t CHAIN_PIECE = 64;  // rows or columns of a later-rows CTA of the solve chains
constexpr int CHAIN_GROUPS = 4;      // row groups of a column piece (each its own CTA and partial sums)

// Builds the plan from the symbolic analysis. The update arena is shared by
// fronts whose update matrices are not alive at the same time (first fit in
// level order).
// Large outer updates (trailing rows >= tun.big_min_rows, u = 0 or u >= TC_TILE) use 128×128
// tiles; use_tc marks their fronts for the tensor-core kernel (mixed precision).
Plan build_plan(const Symbolic& S, bool use_tc = false, const Tuning& tun = Tuning());

// Original entries. For each destination position in the panel arena (a
// front's P_t entry), the sum of the source values src[seg_src[j]] for j in
// [seg_ptr[i], seg_ptr[i+1]) is stored there (the C interface may give the same
// entry more than once; it is then summed in the caller's order).

struct Scatter {
    SegVec dst;                         // panel-arena offset per segment
    std::vector<int64_t> seg_ptr;       // nseg+1
    SegVec src;                         // source index per entry
    std::vector<int64_t> level_seg;     // nlevels+1: segments of each level are contiguous
    std::vector<int64_t> front_seg;     // nfronts+1: segments of the j-th front in level order
};

// The caller's CSC pattern (host arrays), from which an engine builds the scatter of
// the original entries on the device (Engine's CallerPattern constructor). eq maps a
// caller DOF to its internal equation or -1.
struct CallerPattern {
    int64_t ncaller = 0;
    const int64_t* indptr = nullptr;
    const int64_t* indices = nullptr;
    const std::vector<int64_t>* eq = nullptr;
    const Symbolic* sym = nullptr;  // for the host lists when the pattern needs them
    // the row indices already on the device (nullptr: uploaded by the engine), and the
    // call that orders a stream (cudaStream_t) after their copy
    const int64_t* indices_dev = nullptr;
    std::function<void(void*)> wait_indices;
};

// Scatter of the internal lower CSC (engine API: one segment per entry).
Scatter scatter_from_lower(const Plan& P, const Symbolic& S, const std::vector<int64_t>& colptr,
                           const std::vector<int64_t>& rowidx);

// Scatter of a caller CSC through eq (caller DOF -> internal equation or -1):
// the entries with eq[row] >= eq[col] (ffi/src/lib.rs:216-224).
Scatter scatter_from_caller(const Plan& P, const Symbolic& S, int64_t ncaller, const int64_t* indptr,
                            const int64_t* indices, const std::vector<int64_t>& eq);

}  // namespace rfg
