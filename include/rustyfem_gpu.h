/*
 * rustyfem_gpu.h — C interface of the B200 multifrontal sparse LDLᵀ solver.
 *
 * librustyfem_gpu.so is a drop-in for RustyFEM's C interface (the cdylib
 * rustyfem_ffi, ffi/src/lib.rs): the rustyfem_* functions below keep the
 * reference's names, argument meaning, ownership and error behaviour. The
 * symbolic stage (nested dissection, elimination tree, front patterns) runs on
 * the host and reproduces the reference's analysis; the numeric factorization
 * and the solves run on the GPU (sm_100a). The rfg_* functions are additions.
 *
 * Conventions (as in the reference):
 *  - the matrix is symmetric, in CSC (indptr[n+1], indices/data[indptr[n]]) in
 *    the caller's numbering; loc[i] is the node of DOF i, coords the 3·nn node
 *    coordinates. The positive definite factorization uses the entries whose
 *    internal row is not above the internal column, so it needs both triangles;
 *    the indefinite one reads the lower triangle (ffi/src/lib.rs:193-224);
 *  - DOFs without couplings (diagonal only) are split off and solved by
 *    division (ffi/src/lib.rs:105-128);
 *  - on error a factorization returns NULL and sets *err_dof to the caller's DOF
 *    of the failing pivot, or to -1 for invalid input or an internal error
 *    (rfg_last_error() then describes it);
 *  - the caller owns every array; the library owns the handle until
 *    rustyfem_free.
 */
#ifndef RUSTYFEM_GPU_H
#define RUSTYFEM_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct RustyfemHandle RustyfemHandle;

/* ---------------------------------------------------------------------------
 * The reference's C interface
 * ------------------------------------------------------------------------- */

/* Positive definite LDLᵀ. d_out (n, may be NULL) receives the pivots D in the
 * caller's numbering. Replaces rustyfem_factor, ffi/src/lib.rs:64-97. */
RustyfemHandle* rustyfem_factor(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                                const int64_t* indices, const double* data, double* d_out, int64_t* err_dof);

/* Symmetric indefinite LDLᵀ (1×1/2×2 pivots, delayed pivots). inertia_out (3,
 * may be NULL) receives [negative, zero, positive]. Replaces
 * rustyfem_factor_indef, ffi/src/lib.rs:273-290. */
RustyfemHandle* rustyfem_factor_indef(size_t n, size_t nn, const int64_t* loc, const double* coords,
                                      const int64_t* indptr, const int64_t* indices, const double* data,
                                      int64_t* inertia_out, int64_t* err_dof);

/* Unsymmetric LU. Replaces rustyfem_factor_unsym, ffi/src/lib.rs:300-311.
 * Not provided by this library: always returns NULL with *err_dof = -1. */
RustyfemHandle* rustyfem_factor_unsym(size_t n, size_t nn, const int64_t* loc, const double* coords,
                                      const int64_t* indptr, const int64_t* indices, const double* data,
                                      int64_t* err_dof);

/* Inertia [negative, zero, positive]; 0, or -1 if not available.
 * Replaces rustyfem_inertia, ffi/src/lib.rs:320-329. */
int32_t rustyfem_inertia(const RustyfemHandle* h, int64_t* out);

/* Solves K X = B in place for nrhs right-hand sides stored one after another
 * (column-major n × nrhs). 0, or -1 on error. Replaces rustyfem_solve,
 * ffi/src/lib.rs:337-371. */
int32_t rustyfem_solve(const RustyfemHandle* h, size_t nrhs, double* b);

/* out[0] = estimated flops of the factorization, out[1] = stored entries of L.
 * Replaces rustyfem_info, ffi/src/lib.rs:378-383. */
void rustyfem_info(const RustyfemHandle* h, double* out);

/* Internal equation of each caller DOF; uncoupled DOFs numbered last.
 * Replaces rustyfem_order, ffi/src/lib.rs:391-398. */
void rustyfem_order(const RustyfemHandle* h, int64_t* out);

/* Frees a handle (NULL allowed). Replaces rustyfem_free, ffi/src/lib.rs:403-407. */
void rustyfem_free(RustyfemHandle* h);

/* ---------------------------------------------------------------------------
 * Additions
 * ------------------------------------------------------------------------- */

/* RFG_AUTO: the library chooses per model at the factorization — RFG_MIXED when at least
 * half of the factorization's flops fall in fronts of 1024 rows or more (where the
 * tensor-core Schur updates carry the work and refinement pays off), RFG_FP64 otherwise
 * (small fronts, as in 2D or batched small models: the FP32 factor would need many
 * refinement sweeps for little speed). rfg_factor_stats reports the choice. */
enum { RFG_FP64 = 0, RFG_MIXED = 1, RFG_AUTO = 2 };

typedef struct rfg_options {
    int32_t precision;        /* RFG_FP64 or RFG_MIXED (FP32 fronts and Schur updates, FP64 D and refinement) */
    int32_t leaf;             /* nodes per dissection leaf; 0 = 16 as the reference's C interface */
    int32_t refine_max_iter;  /* refinement steps of rfg_solve_ex / rustyfem_solve; -1 = default
                                 (0 for RFG_FP64, 10 for RFG_MIXED) */
    int32_t flags;            /* RFG_FLAG_* */
    double refine_tol;        /* stop when the normwise backward error is at most this; 0 = 1e-12 */
} rfg_options;

/* rfg_options.flags: keep the large Schur updates of the mixed path on the FP32
 * CUDA cores instead of the tensor cores (3×TF32). */
#define RFG_FLAG_NO_TENSOR_CORES 1
/* rfg_options.flags: choose the small-front / large-front cutover of the Schur update
 * (trailing rows from which 128-row tiles are used) and, with tensor cores, the width
 * of their tiles (128 or 256 columns) by measuring the numeric phase of this model for
 * each candidate before the factorization (rfg_tune_report_ex lists them). Costs a
 * number of numeric phases once per analysis and device; cached for the life of the
 * process. */
#define RFG_FLAG_AUTOTUNE 2

typedef struct rfg_solve_stats {
    int32_t iterations;       /* refinement steps done */
    int32_t launches;         /* kernels launched by the call */
    double backward_error;    /* max over RHS of ‖b − Ax‖∞ / (‖A‖∞‖x‖∞ + ‖b‖∞); for a batched
                                 handle each model's own (A, b, x), the max over models */
    double rel_residual;      /* max over RHS (and models) of ‖b − Ax‖₂ / ‖b‖₂ */
    double t_solve_ms;        /* wall time of the call */
} rfg_solve_stats;

typedef struct rfg_factor_stats {
    double work;              /* flops of the factorization (Symbolic::work) */
    double factor_size;       /* entries of L */
    double t_analyse_ms;      /* host symbolic stage and plan */
    double t_factor_ms;       /* device time of the numeric phase */
    int64_t nfronts, nlevels, nsteps, launches;
    int64_t panel_bytes, update_bytes;  /* device arenas */
    int64_t largest_k, largest_u;
    double schur_ms;          /* device time of the 128-tile outer Schur-update launches (tensor
                                 cores in RFG_MIXED, FP64 128-tiles otherwise; profiling on) */
    double schur_flops;       /* their algorithmic flops: Σ over their steps of 2·K·R(R+1)/2 */
    int64_t schur_launches;   /* their number */
    int64_t h2d_bytes;        /* host-to-device bytes of the factorization call (plan + values) */
    double phase_ms[7];       /* with profiling on: device time of assembly, extend-add, pivot
                                 blocks, panels, inner updates, outer updates on 64-tiles, outer
                                 updates on 128-tiles */
    int64_t tile_cutover_rows; /* trailing rows from which the Schur update uses 128×128 tiles */
    int64_t tc_kind;          /* tensor-core Schur updates of the last numeric phase: 0 none, 1 the
                                 TF32 split of W and L, 2 the FP16 split of U = L·D^(1/2) with
                                 power-of-two row scales (RFG_MIXED default) */
    int64_t outer_tile_n;     /* columns of the tensor-core outer-update tiles (128 or 256; 0 without
                                 tensor-core updates) */
    int64_t precision;        /* RFG_FP64 or RFG_MIXED: the precision factored in (RFG_AUTO resolved) */
    double schur_entries;     /* trailing-matrix entries the 128-tile outer updates read and write
                                 (Σ R(R+1)/2): their least memory traffic with schur_opvals */
    double schur_opvals;      /* operand values those updates read at least once (Σ R·K) */
    int64_t delayed;          /* indefinite and LU handles: pivots delayed to a parent front */
} rfg_factor_stats;

/* rustyfem_factor with options (precision, leaf). NULL opt = defaults. */
RustyfemHandle* rfg_factor_ex(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                              const int64_t* indices, const double* data, const rfg_options* opt, double* d_out,
                              int64_t* err_dof);

/* Factors nmodels independent positive definite systems as one batched
 * factorization: each model is analysed on its own, their elimination trees form
 * one forest whose fronts are factored level by level across all models (one CUDA
 * graph for the whole numeric phase). The arrays of model i are given as in
 * rustyfem_factor. The returned handle numbers the DOFs model after model (model
 * i's DOFs start at n[0] + … + n[i-1]); rustyfem_solve / rfg_solve_ex take the
 * right-hand sides in that stacked layout, rfg_refactor the stacked values.
 * On error NULL, *err_model = the model (or -1) and *err_dof its DOF (or -1). */
RustyfemHandle* rfg_batch_factor(size_t nmodels, const size_t* n, const size_t* nn, const int64_t* const* loc,
                                 const double* const* coords, const int64_t* const* indptr,
                                 const int64_t* const* indices, const double* const* data, const rfg_options* opt,
                                 int64_t* err_model, int64_t* err_dof);

/* New values (same n, loc, coords and CSC pattern as the handle's factorization):
 * numeric phase only, the symbolic stage and the plan are reused. Returns -1 on
 * success, the caller's DOF of the failing pivot, or -2 on another error. */
int64_t rfg_refactor(RustyfemHandle* h, const double* data);

/* rustyfem_solve with refinement per the handle's options and statistics. */
int32_t rfg_solve_ex(const RustyfemHandle* h, size_t nrhs, double* b, rfg_solve_stats* stats);

/* Stream order of the entry points that take device pointers (rfg_refactor_device,
 * rfg_solve_device, rfg_solve_device_noalloc): their kernels run on the handle's own
 * non-blocking stream (rfg_stream). On entry that stream waits for the work queued before
 * the call on the legacy default stream (and so on every blocking stream) and on the
 * calling thread's per-thread default stream. Work that produces the inputs on another
 * non-blocking stream (a framework's side stream) must be complete before the call, or
 * the caller makes rfg_stream(h) wait on it. Each call returns when its results are in
 * place (it synchronizes the handle's stream). */

/* rfg_refactor with the values already in device memory (same order as the caller CSC). */
int64_t rfg_refactor_device(RustyfemHandle* h, const double* data_device);

/* rfg_solve_ex with the right-hand sides in device memory (caller numbering, column-major
 * n × nrhs), solved in place. */
int32_t rfg_solve_device(const RustyfemHandle* h, size_t nrhs, double* b_device, rfg_solve_stats* stats);

/* rfg_solve_device that allocates no memory: no counterpart in the reference (it is
 * not a rustyfem_* FFI function). For callers that cannot allocate on the device at
 * solve time: a host framework whose caching allocator has already taken the free
 * device memory, or a time-step loop where cudaMalloc/cudaFree would stall it
 * (cudaFree waits for the whole device). rfg_solve_device allocates its buffers on
 * first use and grows them for more right-hand sides; this call uses only the
 * handle's resident factor and caller-numbering maps (uploaded when the handle was
 * built) and a fixed 16 MiB scratch array compiled into the library (the driver
 * reserves it when the library's kernels are loaded on a device), so it serves small
 * and medium models only.
 *  - Same input and result as rfg_solve_device on a positive definite handle (b_device:
 *    caller numbering, column-major n × nrhs, solved in place), but with no iterative
 *    refinement and no statistics: the result is the handle's factor applied once, the
 *    same values rfg_solve_device gives with refine_max_iter = 0 and stats = NULL.
 *  - Returns 0, or -1 with rfg_last_error() set: an indefinite handle, or a handle whose
 *    scratch need (n × min(nrhs, 32) values twice, the per-front update vectors and
 *    per-CTA partial sums of one 32-column sweep) exceeds 16 MiB; then nothing was
 *    launched.
 *  - Nothing in the scratch need be zero beforehand: every call zeroes the update
 *    vectors and the ticket counters itself.
 *  - Stream order as for rfg_solve_device (above); the call returns when its result is
 *    in b_device: it synchronizes the handle's stream.
 *  - The scratch is one per device and shared by every handle: two calls that overlap
 *    in time on one device (from two host threads, on any handles) race on it and give
 *    wrong results. Make such calls one after another.
 *  - The first call on each device does set-up (it looks up the scratch address and
 *    sets kernel attributes); make it before any stream capture. */
int32_t rfg_solve_device_noalloc(const RustyfemHandle* h, size_t nrhs, double* b_device);

/* The autotuner's measurements of a handle factored with RFG_FLAG_AUTOTUNE: up to cap
 * (cutover, numeric-phase ms) pairs; returns how many were measured (0 without the
 * flag). */
size_t rfg_tune_report(const RustyfemHandle* h, int64_t* cutover, double* ms, size_t cap);
/* The same with the tensor-core outer-update tile width of each candidate (128 or 256
 * columns; the mixed path tunes both with every cutover). */
size_t rfg_tune_report_ex(const RustyfemHandle* h, int64_t* cutover, int64_t* tile_n, double* ms, size_t cap);

/* Device memory of handles is taken from a per-device pool that keeps freed blocks for
 * the next handle (factorizations done one after another skip cudaMalloc/cudaFree of
 * their arenas), and the host stages' large scratch arrays (1 MB and more) from a
 * process-wide cache of freed host blocks (at most 4 GB). This returns the cached device
 * blocks to the driver and frees the cached host blocks; live handles keep theirs.
 * No counterpart in the reference. */
void rfg_release_cached_memory(void);

/* The CUDA stream (cudaStream_t) the handle's kernels run on. */
void* rfg_stream(const RustyfemHandle* h);

/* Profiling of later factorizations with CUDA events recorded on the handle's stream:
 * on = 1 an event after every launch (rfg_factor_stats.phase_ms and schur_ms); on = 2
 * events around the 128-tile outer Schur updates only (schur_ms; the other launches keep
 * their programmatic overlap, so the factorization's own time is hardly changed); 0 off. */
void rfg_set_profiling(RustyfemHandle* h, int32_t on);

/* Statistics of the handle's factorization. 0, or -1. */
int32_t rfg_factor_stats_get(const RustyfemHandle* h, rfg_factor_stats* out);

/* The handle's front list (start, k, u, children per front; the RUSTYFEM_FRONTS dump). */
size_t rfg_handle_nfronts(const RustyfemHandle* h);
void rfg_handle_fronts(const RustyfemHandle* h, int64_t* out4);

/* Message of the last error of this thread ("" if none). */
const char* rfg_last_error(void);

/* Number of CUDA devices visible to the library (0 when there is none). */
int32_t rfg_device_count(void);

/* Self-test of the reciprocal the pivot blocks use (a Newton–Raphson refinement of the
 * hardware's approximate reciprocal): r[i] = 1/x[i] on the current device for n host
 * values x[i] > 0. 0, or -1 on a CUDA error. */
int32_t rfg_selftest_reciprocal(const double* x, double* r, size_t n);

/* Self-test of the host symbolic stage's coordinate sort, the restatement of Rust's
 * slice::sort_unstable_by that src/sparse.rs:108 calls: perm receives the indices 0..n-1
 * in the order that sort leaves them in when sorting by keys[] (keys < 2^32). limit >= 0
 * replaces the quicksort's imbalance budget (0: heapsort for more than 32 elements). */
void rfg_selftest_sort_unstable(const int64_t* keys, int64_t n, int64_t limit, int64_t* perm);

/* --- engine-level matrix (the LinearSolver / SystemMatrix API of
 *     src/solver/api.rs:21-60: prepare, zero, add, factor, solve) --- */
typedef struct RfgMatrix RfgMatrix;

/* Symbolic analysis of the node graph (nb blocks; sorted neighbour lists without
 * the block itself; DOFs per block); leaf 0 = 48 as the engine's direct solver. */
RfgMatrix* rfg_matrix_prepare(size_t nb, const double* coords, const int64_t* adj_ptr, const int64_t* adj_idx,
                              const int64_t* ndof, int32_t leaf, int32_t precision);
size_t rfg_matrix_n(const RfgMatrix* m);
void rfg_matrix_first_dof(const RfgMatrix* m, int64_t* out);
void rfg_matrix_zero(RfgMatrix* m);
/* Adds v at (r, c), r >= c, internal numbering. 0, or -1 if (r, c) is not in the pattern. */
int32_t rfg_matrix_add(RfgMatrix* m, size_t r, size_t c, double v);
int32_t rfg_matrix_add_many(RfgMatrix* m, size_t cnt, const int64_t* r, const int64_t* c, const double* v);
/* -1 on success, else the internal equation of the failing pivot; -2 on another error. */
int64_t rfg_matrix_factor(RfgMatrix* m);
/* Solves in place (internal numbering, one right-hand side). 0, or -1. */
int32_t rfg_matrix_solve(const RfgMatrix* m, double* b);
void rfg_matrix_free(RfgMatrix* m);
/* Number of stored entries of the lower pattern, and a copy of their current values
 * (host or device assembled; internal lower CSC order). 0, or -1. */
size_t rfg_matrix_nnz(const RfgMatrix* m);
int32_t rfg_matrix_values(RfgMatrix* m, double* out);

/* --- assembly of K on the device (replaces the element loop of `internal`,
 *     src/fem/assembly.rs:315-420: the tangent of a symmetric system matrix without
 *     constraints, K = zero, then for every element e and local DOFs a, b with
 *     equations ia >= ib: K[ia, ib] += (ke[a,b] + ke[b,a]) / 2 through
 *     SystemMatrix::add, src/sparse.rs:47-51) ---
 * The values land on the matrix's device and stay there: the next rfg_matrix_factor
 * factors them without a host copy. Every entry is summed in the reference's order
 * (element by element, then (a, b)), so the values equal a host assembly of the same
 * element matrices bit for bit. rfg_matrix_zero / rfg_matrix_add afterwards work on the
 * host values again (the device values are copied down first). An assembly refers to
 * its matrix: free it before the matrix. Calls on one matrix are serialised. */
typedef struct RfgAssembly RfgAssembly;

/* Maps the element pairs onto the matrix's pattern once: nelem elements of nd DOFs,
 * edof[e·nd + a] = the internal equation of local DOF a (dm.eq, src/fem/assembly.rs:
 * 289-301), -1 for a constrained DOF. NULL on error (rfg_last_error names the first
 * pair missing in the pattern, where the reference panics: src/sparse.rs:49). */
RfgAssembly* rfg_assembly_prepare(RfgMatrix* m, size_t nelem, size_t nd, const int64_t* edof);
/* K from element matrices ke (nelem·nd·nd doubles, row-major per element) in host
 * memory, or in the matrix's device memory. 0, or -1. */
int32_t rfg_assembly_set(RfgAssembly* a, const double* ke);
int32_t rfg_assembly_set_device(RfgAssembly* a, const double* d_ke);
/* C3D8 linear-elastic elements computed on the device and assembled: K_e of
 * src/elements/continuum3d.rs:39-131 (2×2×2 Gauss points, volumetric B-bar of
 * src/elements/common.rs:174-200, K_e = Σ Bᵀ D B w of :264-289) with isotropic D
 * (src/materials/elastic.rs:57-70). Needs nd = 24 (node-major U1 U2 U3); conn: nelem × 8
 * node ids (the C3D8 corner order), xyz: nn × 3 coordinates, emod: E per element.
 * -1 on success; the element index when an element is distorted (det J <= 0,
 * src/elements/continuum3d.rs:55-57; K unchanged); -2 on another error. */
int64_t rfg_assembly_hex8(RfgAssembly* a, size_t nn, const double* xyz, const int64_t* conn, const double* emod,
                          double nu);
/* Device time of the last element kernel and of the last assembly gather (ms). */
void rfg_assembly_times(const RfgAssembly* a, double* out2);
/* Number of (element, a, b) contributions mapped onto the pattern. */
size_t rfg_assembly_contributions(const RfgAssembly* a);
void rfg_assembly_free(RfgAssembly* a);

/* --- host symbolic stage alone (no GPU needed) --- */
typedef struct RfgSymbolic RfgSymbolic;
RfgSymbolic* rfg_sym_analyse(size_t nb, const double* coords, const int64_t* adj_ptr, const int64_t* adj_idx,
                             const int64_t* ndof, int32_t leaf);
size_t rfg_sym_n(const RfgSymbolic* s);
size_t rfg_sym_nfronts(const RfgSymbolic* s);
double rfg_sym_work(const RfgSymbolic* s);
size_t rfg_sym_factor_size(const RfgSymbolic* s);
size_t rfg_sym_total_rows(const RfgSymbolic* s);
void rfg_sym_fronts(const RfgSymbolic* s, int64_t* out4);
void rfg_sym_first_dof(const RfgSymbolic* s, int64_t* out);
void rfg_sym_rows(const RfgSymbolic* s, int64_t* out);
void rfg_sym_children(const RfgSymbolic* s, int64_t* out);
size_t rfg_sym_nnz(const RfgSymbolic* s);
void rfg_sym_pattern(const RfgSymbolic* s, int64_t* colptr, int64_t* rowidx);
/* plan figures: levels, steps, panel / peak update arena elements */
void rfg_sym_plan_stats(const RfgSymbolic* s, int64_t* out4);
/* Schur-update flops of the plan with a given cutover (0 = default): inner, outer, the
 * outer part on 128×128 tiles, and the number of those tiles */
void rfg_sym_plan_flops(const RfgSymbolic* s, int64_t cutover_rows, double* out4);
void rfg_sym_free(RfgSymbolic* s);

#ifdef __cplusplus
}
#endif

#endif /* RUSTYFEM_GPU_H */
