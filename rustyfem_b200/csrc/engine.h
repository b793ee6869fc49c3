// The device-resident numeric factorization: plan arrays in HBM, the panel and
// update arenas, the pivots, and the numeric phase / solve drivers. Used by the
// C interface (capi.cpp); implemented in numeric.cu and solve.cu.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdlib>
#include <string>
#include <vector>

#include "plan.h"

namespace rfg {

enum Precision : int32_t {
    PREC_FP64 = 0,   // fronts, factor and Schur updates in FP64
    PREC_MIXED = 1,  // fronts and factor in FP32, FP32 Schur updates, pivots D in FP64
};

struct CudaError : std::exception {
    std::string msg;
    explicit CudaError(std::string m) : msg(std::move(m)) {}
    const char* what() const noexcept override { return msg.c_str(); }
};

#define RFG_CUDA(x)                                                                                        \
    do {                                                                                                   \
        cudaError_t e_ = (x);                                                                              \
        if (e_ != cudaSuccess)                                                                             \
            throw ::rfg::CudaError(std::string(#x) + ": " + cudaGetErrorString(e_) + " (" + __FILE__ + ")"); \
    } while (0)

// Programmatic dependent launch (PDL) of a kernel after the previous one in the stream.
// Every kernel launched this way calls pdl_wait() before it touches data that the
// previous kernel produces or reads (tiles.cuh). RFG_PDL=0 launches plainly.
inline bool pdl_enabled() {
    static const bool on = [] {
        const char* e = std::getenv("RFG_PDL");
        return !(e && e[0] == '0');
    }();
    return on;
}
template <typename... KArgs, typename... Args>
inline void launch_pdl(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                       Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl && pdl_enabled() ? 1 : 0;
    RFG_CUDA(cudaLaunchKernelEx(&cfg, kern, args...));
}

// Device utilities (devutil.cu). exclusive_scan_i64: in-place exclusive prefix sum of
// n counts, tmp holding scan_tmp_elems(n) values. sort_rows_u64: sorts each row
// [rp[r], rp[r+1]) of key ascending (keys distinct within a row).
int64_t scan_tmp_elems(int64_t n);
void exclusive_scan_i64(int64_t* d, int64_t n, int64_t* tmp, cudaStream_t st);
void sort_rows_u64(uint64_t* key, const int64_t* rp, int64_t nrows, cudaStream_t st);

// TMA descriptors of the split Schur-update operands (tensor-core path), one set per
// scratch buffer (the buffers alternate with the parity of the outer block)
struct TcMaps {
    CUtensorMap whi[2], wlo[2], lhi[2], llo[2];  // TF32 split of W and L: boxes of 32 × 128
    CUtensorMap lhi2[2], llo2[2];                // L operands in boxes of 32 × 256 (128×256 tiles)
    CUtensorMap uhi[2], ulo[2];                  // FP16 split of the scaled U = L·D^(1/2): 64 × 128
    CUtensorMap uhi2[2], ulo2[2];                // the same in boxes of 64 × 256
};

// device copies of the plan
struct DevPlan {
    DFront* fronts = nullptr;
    int64_t* level_order = nullptr;
    int64_t* pre_panel = nullptr;
    int64_t* pre_inner = nullptr;
    int64_t* pre_inner_tc = nullptr;
    int64_t* pre_outer = nullptr;
    int64_t* pre_outer_tc = nullptr;
    int64_t* pre_outer_tc2 = nullptr;
    uint8_t* panel_mode = nullptr;    // Plan::panel_mode
    uint8_t* outer_mode = nullptr;    // Plan::outer_mode
    int64_t* pre_scr = nullptr;
    int64_t* xadd_child = nullptr;
    int64_t* xadd_task = nullptr;
    int64_t* xadd_fpre = nullptr;
    int64_t* pre_wrows = nullptr;
    int64_t* pre_wpart = nullptr;
    int64_t* rows = nullptr;
    int32_t* emap = nullptr;
    int64_t* seg_dst = nullptr;
    int64_t* seg_ptr = nullptr;  // null when every segment has one source (seg i -> src i)
    int64_t* seg_src = nullptr;
    int64_t* front_seg = nullptr;  // segments of each front, in level order
    int64_t* chain_blk = nullptr;     // Plan::chain_blk
    int64_t* chain_bfront = nullptr;  // Plan::chain_bfront
    int64_t* chain_fwd = nullptr;     // Plan::chain_fwd
    int64_t* chain_bwd = nullptr;     // Plan::chain_bwd
    int64_t* chain_rows = nullptr;    // Plan::chain_rows
    int64_t* chain_cols = nullptr;    // Plan::chain_cols
};

struct FactorStats {
    double t_factor_ms = 0.0;     // device time of the numeric phase
    int64_t launches = 0;         // kernels launched by the numeric phase
    double schur_ms = 0.0;        // device time of the 128-tile outer-update launches (profiling on)
    int64_t schur_launches = 0;   // their number
    double schur_flops = 0.0;     // their algorithmic flops
    double schur_entries = 0.0;   // trailing entries they update (Σ R(R+1)/2)
    double schur_opvals = 0.0;    // operand values they read at least once (Σ R·K)
    int64_t h2d_bytes = 0;        // host-to-device bytes of the call
    // device time by phase (profiling on): assembly, extend-add, pivot blocks, panels,
    // inner updates, outer updates on 64-tiles, outer updates on 128-tiles
    double phase_ms[7] = {0, 0, 0, 0, 0, 0, 0};
};

struct SolveStats {
    int32_t iterations = 0;       // refinement iterations done
    double backward_error = 0.0;  // ‖b − A x‖∞ / (‖A‖∞ ‖x‖∞ + ‖b‖∞), max over the right-hand sides
    double rel_residual = 0.0;    // ‖b − A x‖₂ / ‖b‖₂, max over the right-hand sides
    int64_t launches = 0;
};

class Engine {
   public:
    Engine(Plan&& plan, Scatter&& scatter, int64_t nsrc, Precision prec, bool use_tc);
    // The scatter of the caller's entries built on the device from its CSC pattern: the
    // pattern is uploaded and mapped by two kernels instead of host lists (the host
    // lists of scatter_from_caller are used when a column's rows are not strictly
    // increasing).
    Engine(Plan&& plan, const CallerPattern& pattern, int64_t nsrc, Precision prec, bool use_tc);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Numeric factorization of the source values src (host pointer, nsrc values, or a
    // device pointer when on_device). Returns -1, or the internal equation of the first
    // pivot that breaks the positive definite rule (src/sparse.rs:528-531) in postorder.
    int64_t factor(const double* src, bool on_device);

    // Solves in place for nrhs right-hand sides in the internal numbering, stored as
    // X[q·nrhs + j] on the device.
    // (allow_graph = false: launch directly, capture nothing)
    void solve_device(double* X, int64_t nrhs, bool allow_graph = true);

    // The sweep of solve_device for nrhs ≤ 32 right-hand sides, launched directly (no
    // CUDA graph) on workspace the caller provides instead of the engine's own. The
    // workspace is sweep_workspace_bytes(nrhs) bytes at a 256-byte aligned address. It
    // need hold nothing on entry: the sweep zeroes the ticket words and the update rows
    // (v) itself, with memsets on the engine's stream. Allocates nothing.
    struct SweepWorkspace {
        double* y;        // n · nrhs
        double* v;        // vu_rows · nrhs
        double* partial;  // partial_rows() · nrhs
        int* tickets;     // max_nact, then the flag words of the solve chains
    };
    int64_t sweep_workspace_bytes(int64_t nrhs) const;
    SweepWorkspace carve_sweep_workspace(void* base, int64_t nrhs) const;
    void solve_sweep_on(double* X, int64_t nrhs, const SweepWorkspace& ws);

    // Pivots D in the internal numbering (device array of n doubles).
    const double* pivots() const { return d_; }
    void pivots_to_host(double* out) const;

    // y = A x for the symmetric matrix that was factored (FP64, both triangles as a CSR in
    // the internal numbering, built on the device from the scatter lists on first use).
    // X, Y laid out as in solve_device.
    void matvec(const double* X, double* Y, int64_t nrhs);
    double norm_inf_A() const { return anorm_; }

    // Throws CudaError (and clears the record) when a wait of a solve chain gave up since
    // the last check: the solutions of the sweeps since then are invalid. Waits for the
    // engine's stream.
    void chain_check();

    // Refined solve: x = A⁻¹ b by the factor and FP64 iterative refinement until the
    // backward error is at most tol or max_iter steps were done.
    SolveStats solve_refined(double* X, const double* B, int64_t nrhs, double tol, int max_iter);

    // Splits the internal rows into independent systems (offsets off[0] = 0 < ... <=
    // off[g] ... = n, one per model of a batched factorization): the refined solve
    // then measures the backward error of every system on its own and iterates until
    // the worst one meets the tolerance. Without it the rows form one system.
    void set_segments(const std::vector<int64_t>& off);

    const Plan& plan() const { return plan_; }
    // 0 off; 1 an event after every launch (phase_ms); 2 events around the 128-tile outer
    // updates only (schur_ms), which leave the other launches' programmatic overlap alone
    void set_profiling(int level) { profile_ = level >= 0 && level <= 2 ? level : 0; }
    // replay the numeric phase and the solve sweeps from captured CUDA graphs
    void set_graphs(bool on) { use_graphs_ = on; }
    int64_t plan_bytes() const { return plan_bytes_; }
    Precision precision() const { return prec_; }
    // 0: no tensor-core updates, 1: TF32 split, 2: FP16 split of the scaled U
    int tc_kind() const { return use_tc_ ? (h16_ ? 2 : 1) : 0; }
    cudaStream_t stream() const { return stream_; }
    FactorStats last_factor;
    int64_t solve_launches = 0;

   private:
    template <typename T>
    void factor_impl();
    template <typename T>
    void solve_impl(double* X, int64_t nrhs);
    template <typename T>
    void solve_sweep_impl(double* X, int64_t nrhs, const SweepWorkspace& ws);
    template <typename T>
    int64_t forward_steps(int64_t level, double* X, double* Y, double* V, int nrhs, int* chain);
    template <typename T>
    int64_t backward_steps(int64_t level, double* Y, double* V, int nrhs, double* partial, int* tickets, int* chain);
    // the sweeps of nrhs right-hand sides run the solve chains of the plan's chain levels
    bool chain_on(int64_t nrhs) const;
    void ensure_chain_inverse();
    int64_t ticket_words() const;
    int64_t partial_rows() const;  // partial-sum values per right-hand side of a sweep
    void init(bool use_tc);
    void upload_plan();
    void upload_scatter();
    void build_scatter_device(const CallerPattern& cp);
    void build_matrix();
    void setup_tc();
    void launch_schur_tc(const DStep& st);
    void launch_schur_tc_inner(const DStep& st);

    Plan plan_;
    Scatter scatter_;  // host lists (level_seg, front_seg kept; dst/src released after upload)
    int64_t nseg_ = 0;  // scatter segments (entries read from the caller's values)
    int64_t nsrc_;
    Precision prec_;
    cudaStream_t stream_ = nullptr;
    DevPlan dp_;
    std::vector<int64_t> level_poff_;  // panel-arena range of each level
    void* panel_ = nullptr;
    void* upd_ = nullptr;
    void* scr_w_ = nullptr;
    void* scr_l_ = nullptr;
    bool use_tc_ = false;
    void* scr_whi_ = nullptr;
    void* scr_wlo_ = nullptr;
    void* scr_lhi_ = nullptr;
    void* scr_llo_ = nullptr;
    void* scr_uhi_ = nullptr;     // FP16 split of the scaled U rows (tensor cores, FP16 kind)
    void* scr_ulo_ = nullptr;
    void* scr_uscale_ = nullptr;  // power-of-two scale of each scratch row (float)
    bool h16_ = false;            // tensor-core updates with the FP16 split (else TF32 split)
    int64_t* diag_src_ = nullptr;  // caller index of each equation's diagonal entry (or -1)
    double* adiag0_ = nullptr;     // the original diagonal per equation (FP16 split scales)
    TcMaps tc_maps_{};
    CUtensorMap* d_cmaps_ = nullptr;
    int* tc_err_ = nullptr;
    int num_sms_ = 148;
    bool tc_persistent_ = true;
    double* d_ = nullptr;
    double* linv_ = nullptr;      // inverse of each unit-lower NB×NB diagonal block (solves)
    double* chain_inv_ = nullptr; // inverse of each solve-chain block (WS × WS), mixed precision
    int* chain_err_ = nullptr;    // set by a solve-chain wait that gave up
    int64_t chain_inv_at_ = -1;   // the numeric phase (factor_calls_) chain_inv_ was formed for
    double* adiag_ = nullptr;
    int64_t* status_ = nullptr;
    double* src_ = nullptr;
    // solve workspace
    double* vupd_ = nullptr;
    double* partial_ = nullptr;
    double* ybuf_ = nullptr;
    int* counters_ = nullptr;
    int64_t ws_nrhs_ = 0;
    int64_t factor_calls_ = 0;                           // numeric phases run so far
    int64_t refined_calls_ = 0;                          // refined solves run so far
    std::vector<std::pair<std::pair<double*, int64_t>, int64_t>> solve_seen_;  // (X, nrhs) -> sweeps run
    // matrix for refinement (full CSR over the internal numbering)
    int64_t* a_rowptr_ = nullptr;
    int64_t* a_col_ = nullptr;
    int64_t* a_src_ = nullptr;
    double* a_val_ = nullptr;
    int64_t a_nnz_ = 0;
    bool matrix_built_ = false;  // a_* hold the FP64 matrix of the refinement
    double anorm_ = 0.0;
    double* ref_r_ = nullptr;
    double* ref_dx_ = nullptr;
    double* ref_red_ = nullptr;
    int64_t ref_nrhs_ = 0;
    std::vector<int64_t> seg_off_;  // independent systems of the refined solve
    int64_t seg_blocks_ = 0;
    int64_t* d_seg_off_ = nullptr;
    int64_t* d_seg_blk_ = nullptr;
    std::vector<void*> allocs_;
    void* dalloc(size_t bytes);
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    int profile_ = 0;
    bool use_graphs_ = true;
    cudaGraphExec_t factor_graph_[3] = {nullptr, nullptr, nullptr};  // per profiling level
    struct SolveGraph {
        double* X;
        int64_t nrhs;
        cudaGraphExec_t exec;
    };
    std::vector<SolveGraph> solve_graphs_;
    int64_t solve_graph_launches_ = 0;
    void set_attributes();
   public:
    bool uses_tc() const { return use_tc_; }
    int tc_error() const;
   private:
    std::vector<cudaEvent_t> prof_ev_;
    std::vector<int> prof_phase_;
    std::vector<int> prof_phase_graph_[3];  // the phases of the events in each profiling graph
    int64_t plan_bytes_ = 0;
};

// kernels shared with capi.cpp: caller <-> internal permutation of right-hand sides
void launch_gather_rhs(const double* b, double* X, const int64_t* eq, int64_t ncaller, int64_t nsym, int64_t nrhs,
                       cudaStream_t st);
void launch_scatter_rhs(double* b, const double* X, const int64_t* eq, const int64_t* iso_idx, const double* iso_d,
                        int64_t niso, int64_t ncaller, int64_t nsym, int64_t nrhs, cudaStream_t st);

// Stream-ordered device memory from a per-device pool that keeps freed blocks cached
// (devmem.cpp); release_cached_memory() returns the cached blocks to the driver.
void* dev_alloc(size_t bytes, cudaStream_t st);
void dev_free(void* p, cudaStream_t st);
void host_upload(void* dst, const void* src, size_t bytes, cudaStream_t st);  // pinned, multithreaded staging
void release_cached_memory();

// Size of the fixed device scratch behind rfg_solve_device_noalloc (16 MiB).
constexpr int64_t NOALLOC_SCRATCH_BYTES = int64_t(16) << 20;
// Device address of that scratch on the current device. The first call on a device
// looks it up with cudaGetSymbolAddress and keeps it; throws CudaError if the lookup
// fails. Allocates nothing.
void* noalloc_scratch();

}  // namespace rfg
