// The C interface (include/rustyfem_gpu.h): RustyFEM's rustyfem_* functions
// (ffi/src/lib.rs) on top of the host symbolic stage and the GPU engine, plus
// the rfg_* additions.

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <exception>
#include <string>
#include <thread>
#include <vector>

#include "assembly.h"
#include "autotune.h"
#include "engine.h"
#include "indef.h"
#include "lu.h"
#include "par.h"
#include "sort_unstable.h"
#include "plan.h"
#include "rustyfem_gpu.h"
#include "symbolic.h"

using namespace rfg;

namespace {

thread_local std::string g_err;

void set_error(const std::string& s) { g_err = s; }

double ms_since(std::chrono::steady_clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

const int64_t FFI_LEAF = 16;  // ffi/src/lib.rs:17
const int64_t ENGINE_LEAF = 48;  // src/sparse.rs:14

bool have_device() {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return n > 0;
}

enum class Mode { Pd, Indef, Lu };

}  // namespace

struct RustyfemHandle {
    Mode mode = Mode::Pd;
    rfg_options opt{};
    Symbolic sym;
    std::unique_ptr<Engine> eng;
    std::unique_ptr<IndefEngine> ieng;
    std::unique_ptr<LuEngine> leng;
    std::vector<int64_t> lcolptr, lrowidx;  // indefinite and LU: the lower pattern (internal numbering)
    int64_t ncaller = 0, nn = 0, nnz = 0;
    std::vector<int64_t> eq;  // caller DOF -> internal equation, -1 = uncoupled
    std::vector<int64_t> owner;
    std::vector<std::pair<int64_t, double>> iso;
    int64_t n_sym = 0;
    double work = 0.0;
    int64_t factor_size = 0;
    int64_t inertia[3] = {0, 0, 0};
    double t_analyse_ms = 0.0;
    std::vector<int64_t> batch_dof_off;  // batched handle: first caller DOF of each model
    TuneResult tune;                      // RFG_FLAG_AUTOTUNE: the candidates measured
    int64_t first_h2d_bytes = 0;  // plan upload of the factorization call (0 after rfg_refactor)
    // solve buffers on the device
    mutable std::mutex mu;
    mutable int64_t* d_eq = nullptr;
    mutable int64_t* d_iso_idx = nullptr;
    mutable double* d_iso_d = nullptr;
    mutable double* d_b = nullptr;
    mutable double* d_X = nullptr;
    mutable double* d_B = nullptr;
    mutable int64_t buf_cap = 0;
    mutable double* h_pinned = nullptr;
    mutable int64_t pinned_cap = 0;
    mutable cudaEvent_t caller_ev = nullptr;  // orders the handle's stream after the caller's work
    ~RustyfemHandle() {
        if (caller_ev) cudaEventDestroy(caller_ev);
        eng.reset();
        ieng.reset();
        leng.reset();
        for (void* p : {(void*)d_eq, (void*)d_iso_idx, (void*)d_iso_d, (void*)d_b, (void*)d_X, (void*)d_B})
            if (p) dev_free(p, 0);
        if (h_pinned) cudaFreeHost(h_pinned);
    }
};

namespace {

void ensure_maps(const RustyfemHandle* h);

// Host half of the reference's build (ffi/src/lib.rs:100-172): validation, the
// uncoupled DOFs, the node graph from the pattern, the symbolic analysis and the
// equation numbering. Fills h; false (with *err_dof) on invalid input.
bool prepare_model(RustyfemHandle* h, size_t n, size_t nn, const int64_t* loc, const double* coords,
                   const int64_t* indptr, const int64_t* indices, const double* data, Mode mode,
                   std::vector<double>& diag_out, std::vector<char>& coupled_out, int64_t* err_dof) {
    HostTimer timer("prepare_model");
    int64_t N = (int64_t)n;
    int64_t nnz = N > 0 ? indptr[N] : 0;
    for (int64_t i = 0; i < N; i++)
        if (loc[i] < 0 || (size_t)loc[i] >= nn) {
            set_error("invalid input: loc out of range");
            return false;
        }
    h->mode = mode;
    h->ncaller = N;
    h->nn = (int64_t)nn;
    h->nnz = nnz;
    std::vector<char>& coupled = coupled_out;
    std::vector<double>& diag = diag_out;
    coupled.assign(N, 0);
    diag.assign(N, 0.0);
    // diagonal sums and couplings (ffi/src/lib.rs:108-120); a column marks its rows too.
    // Row indices are validated in the same pass.
    std::atomic<bool> bad_index{false};
    parallel_chunks(N, 4096, [&](int64_t a, int64_t b) {
        for (int64_t c = a; c < b; c++) {
            double dsum = 0.0;
            for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                int64_t r = indices[p];
                if (r < 0 || r >= N) {
                    bad_index.store(true, std::memory_order_relaxed);
                    continue;
                }
                if (r == c)
                    dsum += data[p];
                else if (data[p] != 0.0) {
                    // stores only where the mark is not set yet: the lines stay shared
                    if (!__atomic_load_n(&coupled[c], __ATOMIC_RELAXED)) __atomic_store_n(&coupled[c], 1, __ATOMIC_RELAXED);
                    if (!__atomic_load_n(&coupled[r], __ATOMIC_RELAXED)) __atomic_store_n(&coupled[r], 1, __ATOMIC_RELAXED);
                }
            }
            diag[c] = dsum;
        }
    });
    if (bad_index.load()) {
        set_error("invalid input: row index out of range");
        return false;
    }
    timer.lap("validation, couplings");
    for (int64_t i = 0; i < N; i++) {
        if (coupled[i]) continue;
        bool ok = mode == Mode::Pd ? diag[i] > 0.0 : (diag[i] != 0.0 && std::isfinite(diag[i]));
        if (!ok) {
            *err_dof = i;
            set_error("non-positive or zero pivot at an uncoupled DOF");
            return false;
        }
        h->iso.push_back({i, diag[i]});
    }
    // nodes with a coupled DOF, compact numbering in order of their first DOF (:129-138)
    HostVec<int64_t> nid(nn, -1);
    HostVec<double> xyz;
    xyz.reserve(3 * nn);
    for (int64_t i = 0; i < N; i++) {
        if (!coupled[i]) continue;
        int64_t v = loc[i];
        if (nid[v] < 0) {
            nid[v] = (int64_t)(xyz.size() / 3);
            xyz.push_back(coords[3 * v]);
            xyz.push_back(coords[3 * v + 1]);
            xyz.push_back(coords[3 * v + 2]);
        }
    }
    int64_t nc = (int64_t)(xyz.size() / 3);
    Graph g;
    g.nn = nc;
    g.coords = xyz.data();
    g.ndof.assign(nc, 0);
    HostVec<int64_t> local(N, 0), dnode(N, -1);
    for (int64_t i = 0; i < N; i++) {
        if (!coupled[i]) continue;
        int64_t v = nid[loc[i]];
        dnode[i] = v;
        local[i] = g.ndof[v]++;
    }
    // node adjacency from the pattern, explicit zeros included (:148-161): the
    // neighbours found from each node's own columns, united with the transpose
    // (a lower-only pattern gives each pair in one direction only)
    {
        HostVec<int64_t> dptr(nc + 1, 0), dofs(N);
        timer.lap("uncoupled DOFs, node numbering");
        for (int64_t i = 0; i < N; i++)
            if (dnode[i] >= 0) dptr[dnode[i] + 1]++;
        for (int64_t v = 0; v < nc; v++) dptr[v + 1] += dptr[v];
        {
            HostVec<int64_t> fill(dptr.begin(), dptr.end() - 1);
            for (int64_t i = 0; i < N; i++)
                if (dnode[i] >= 0) dofs[fill[dnode[i]]++] = i;
        }
        // Per-thread marks: stamp[w] == key means w was taken for the current (pass, node).
        // Every call reserves 4·nc fresh keys from a process-wide counter, so marks left by
        // other passes, calls or threads never match.
        static std::atomic<int64_t> key_counter{0};
        const int64_t key0 = key_counter.fetch_add(4 * nc);
        auto with_stamp = [&](int pass, auto&& body) {
            parallel_chunks(nc, 256, [&](int64_t a0, int64_t a1) {
                thread_local std::vector<int64_t> stamp;
                if ((int64_t)stamp.size() < nc) stamp.assign(nc, -1);
                const int64_t base = key0 + pass * nc;
                for (int64_t v = a0; v < a1; v++) body(v, stamp.data(), base + v);
            });
        };
        // forward lists: the nodes of the rows of each node's own columns
        auto scan_fwd = [&](int64_t v, int64_t* stamp, int64_t key, auto&& emit) {
            for (int64_t z = dptr[v]; z < dptr[v + 1]; z++) {
                int64_t c = dofs[z];
                for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                    int64_t w = dnode[indices[p]];
                    if (w < 0 || w == v || stamp[w] == key) continue;
                    stamp[w] = key;
                    emit(w);
                }
            }
        };
        HostVec<int64_t> fptr(nc + 1, 0);
        with_stamp(0, [&](int64_t v, int64_t* st, int64_t key) {
            int64_t c = 0;
            scan_fwd(v, st, key, [&](int64_t) { c++; });
            fptr[v + 1] = c;
        });
        for (int64_t v = 0; v < nc; v++) fptr[v + 1] += fptr[v];
        SegVec fidx(fptr[nc]);
        with_stamp(1, [&](int64_t v, int64_t* st, int64_t key) {
            int64_t o = fptr[v];
            scan_fwd(v, st, key, [&](int64_t w) { fidx[o++] = w; });
        });
        timer.lap("node neighbours");
        // transpose, then each node's list united with its transposed list (a lower-only
        // pattern gives each pair in one direction only); the lists need no order
        // (in parallel over blocks of source nodes, each block filling its own slots, so the
        // transposed lists come out in increasing source order as a serial fill gives them)
        HostVec<int64_t> tptr(nc + 1, 0);
        SegVec tidx;
        {
            const int64_t nb = std::max<int64_t>(1, std::min<int64_t>(16, nc / 4096));
            const int64_t bs = (nc + nb - 1) / nb;
            HostVec<int32_t> cnt((size_t)nb * nc, 0);
            parallel_chunks(nb, 1, [&](int64_t b0, int64_t b1) {
                for (int64_t bk = b0; bk < b1; bk++) {
                    int32_t* c = cnt.data() + bk * nc;
                    for (int64_t v = bk * bs; v < std::min(nc, (bk + 1) * bs); v++)
                        for (int64_t e = fptr[v]; e < fptr[v + 1]; e++) c[fidx[e]]++;
                }
            });
            // per target: the blocks' counts become their first slots; tptr the list starts
            HostVec<int64_t> tot(nc, 0);
            parallel_chunks(nc, 8192, [&](int64_t w0, int64_t w1) {
                for (int64_t w = w0; w < w1; w++) {
                    int64_t sum = 0;
                    for (int64_t bk = 0; bk < nb; bk++) {
                        const int32_t x = cnt[bk * nc + w];
                        cnt[bk * nc + w] = (int32_t)sum;
                        sum += x;
                    }
                    tot[w] = sum;
                }
            });
            for (int64_t w = 0; w < nc; w++) tptr[w + 1] = tptr[w] + tot[w];
            tidx.resize(tptr[nc]);
            parallel_chunks(nb, 1, [&](int64_t b0, int64_t b1) {
                for (int64_t bk = b0; bk < b1; bk++) {
                    int32_t* c = cnt.data() + bk * nc;
                    for (int64_t v = bk * bs; v < std::min(nc, (bk + 1) * bs); v++)
                        for (int64_t e = fptr[v]; e < fptr[v + 1]; e++) {
                            const int64_t w = fidx[e];
                            tidx[tptr[w] + c[w]++] = v;
                        }
                }
            });
        }
        timer.lap("transpose");
        auto scan_union = [&](int64_t v, int64_t* stamp, int64_t key, auto&& emit) {
            for (int64_t e = fptr[v]; e < fptr[v + 1]; e++) {
                stamp[fidx[e]] = key;
                emit(fidx[e]);
            }
            for (int64_t e = tptr[v]; e < tptr[v + 1]; e++)
                if (stamp[tidx[e]] != key) {
                    stamp[tidx[e]] = key;
                    emit(tidx[e]);
                }
        };
        g.adj_ptr.assign(nc + 1, 0);
        with_stamp(2, [&](int64_t v, int64_t* st, int64_t key) {
            int64_t c = 0;
            scan_union(v, st, key, [&](int64_t) { c++; });
            g.adj_ptr[v + 1] = c;
        });
        for (int64_t v = 0; v < nc; v++) g.adj_ptr[v + 1] += g.adj_ptr[v];
        g.adj_idx.resize(g.adj_ptr[nc]);
        with_stamp(3, [&](int64_t v, int64_t* st, int64_t key) {
            int64_t o = g.adj_ptr[v];
            scan_union(v, st, key, [&](int64_t w) { g.adj_idx[o++] = w; });
        });
    }
    timer.lap("validation, uncoupled DOFs, node graph");
    h->sym = analyse(g, h->opt.leaf);
    timer.lap("symbolic analysis");
    const Symbolic& S = h->sym;
    if (mode == Mode::Indef || mode == Mode::Lu) lower_pattern(S, g, h->lcolptr, h->lrowidx);
    if (getenv("RUSTYFEM_FRONTS"))
        for (auto& f : S.fronts) fprintf(stderr, "front %lld %lld %lld %lld\n", (long long)f.start, (long long)f.k,
                                         (long long)f.u, (long long)f.nchild);
    h->eq.assign(N, -1);
    for (int64_t i = 0; i < N; i++)
        if (coupled[i]) h->eq[i] = S.first_dof[nid[loc[i]]] + local[i];
    h->owner.assign(S.n, 0);
    for (int64_t i = 0; i < N; i++)
        if (h->eq[i] >= 0) h->owner[h->eq[i]] = i;
    h->n_sym = S.n;
    h->work = S.work();
    h->factor_size = S.factor_size();
    return true;
}

void apply_options(RustyfemHandle* h, const rfg_options* opt) {
    if (opt) h->opt = *opt;
    if (h->opt.leaf <= 0) h->opt.leaf = (int32_t)FFI_LEAF;
    if (h->opt.refine_tol <= 0) h->opt.refine_tol = 1e-12;
    if (h->opt.precision != RFG_MIXED && h->opt.precision != RFG_AUTO) h->opt.precision = RFG_FP64;
    if (h->opt.refine_max_iter < 0 && h->opt.precision != RFG_AUTO)
        h->opt.refine_max_iter = h->opt.precision == RFG_MIXED ? 10 : 0;
}

// RFG_AUTO: mixed precision when at least half of the flops fall in fronts of 1024 rows
// or more, FP64 otherwise; the default number of refinement steps follows the choice.
void resolve_precision(RustyfemHandle* h) {
    if (h->opt.precision == RFG_AUTO) {
        const Symbolic& S = h->sym;
        double big = 0.0, all = 0.0;
        for (const SymFront& f : S.fronts) {
            double own = f.work;
            for (int64_t c = f.child_off; c < f.child_off + f.nchild; c++) own -= S.fronts[S.children[c]].work;
            all += own;
            if (f.k + f.u >= 1024) big += own;
        }
        h->opt.precision = (all > 0.0 && big >= 0.5 * all) ? RFG_MIXED : RFG_FP64;
    }
    if (h->opt.refine_max_iter < 0) h->opt.refine_max_iter = h->opt.precision == RFG_MIXED ? 10 : 0;
}

// The caller's values and row indices copied to the device by a thread of their own
// from the start of a factorization call, so that the copies overlap the host stages
// (validation, node graph, analysis, plan) instead of following them. The buffers come
// from the handle's memory pool on a stream of their own; wait() orders a consumer
// stream after the copies.
struct EarlyUpload {
    cudaStream_t st = nullptr;
    cudaEvent_t done = nullptr;
    double* vals = nullptr;
    int64_t* idx = nullptr;
    std::thread th;
    std::exception_ptr err;
    bool joined = false;

    void start(const double* data, const int64_t* indices, int64_t nnz) {
        int dev = 0;
        RFG_CUDA(cudaGetDevice(&dev));
        RFG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        RFG_CUDA(cudaEventCreateWithFlags(&done, cudaEventDisableTiming));
        vals = (double*)dev_alloc((size_t)std::max<int64_t>(nnz, 1) * 8, st);
        idx = (int64_t*)dev_alloc((size_t)std::max<int64_t>(nnz, 1) * 8, st);
        th = std::thread([=] {
            try {
                RFG_CUDA(cudaSetDevice(dev));
                if (nnz > 0) {
                    host_upload(vals, data, (size_t)nnz * 8, st);
                    host_upload(idx, indices, (size_t)nnz * 8, st);
                }
                RFG_CUDA(cudaEventRecord(done, st));
            } catch (...) {
                err = std::current_exception();
            }
        });
    }
    void join() {
        if (!joined && th.joinable()) th.join();
        joined = true;
    }
    // the copies are queued (and ordered before later work on `consumer`)
    void wait(cudaStream_t consumer) {
        join();
        if (err) std::rethrow_exception(err);
        RFG_CUDA(cudaStreamWaitEvent(consumer, done, 0));
    }
    // frees the buffers after the work queued on `last` (the stream that used them)
    void release(cudaStream_t last) {
        join();
        if (vals) dev_free(vals, last);
        if (idx) dev_free(idx, last);
        vals = nullptr;
        idx = nullptr;
    }
    ~EarlyUpload() {
        join();
        if (st) {
            // not released (an error before the numeric phase): kernels of another stream
            // may still read the buffers
            if (vals || idx) cudaDeviceSynchronize();
            if (vals) dev_free(vals, st);
            if (idx) dev_free(idx, st);
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
        if (done) cudaEventDestroy(done);
    }
};

// Device half: plan, engine, refinement matrix and the numeric factorization.
// Returns false with *err_dof (caller DOF) on a failing pivot. With `early`, the
// caller's values and row indices are already on their way to the device.
bool finish_model(RustyfemHandle* h, const int64_t* indptr, const int64_t* indices, const double* data,
                  std::chrono::steady_clock::time_point t0, int64_t* err_dof, EarlyUpload* early = nullptr) {
    const Symbolic& S = h->sym;
    int64_t N = h->ncaller, nnz = h->nnz;
    if (!have_device()) {
        set_error("no CUDA device: the numeric phase of librustyfem_gpu runs on the GPU only");
        return false;
    }
    resolve_precision(h);
    bool use_tc = h->opt.precision == RFG_MIXED && !(h->opt.flags & RFG_FLAG_NO_TENSOR_CORES);
    Precision prec = h->opt.precision == RFG_MIXED ? PREC_MIXED : PREC_FP64;
    Tuning tun;
    if (const char* e = getenv("RFG_TC_OUTER_TN")) tun.outer_tn = atoi(e) == 128 ? 128 : TC_WIDE;
    // two-block passes of the tensor-core outer update (the persistent kernel only)
    if (const char* e = getenv("RFG_TC_PAIR")) tun.pair_blocks = e[0] != '0';
    if (const char* e = getenv("RFG_TC_PERSISTENT"))
        if (e[0] == '0') tun.pair_blocks = false;
    CallerPattern cp;
    cp.ncaller = N;
    cp.indptr = indptr;
    cp.indices = indices;
    cp.eq = &h->eq;
    cp.sym = &S;
    if (early) {
        cp.indices_dev = early->idx;
        cp.wait_indices = [early](void* stream) { early->wait((cudaStream_t)stream); };
    }
    if (h->opt.flags & RFG_FLAG_AUTOTUNE) {
        auto mk = [&](Plan&& Pc) { return std::unique_ptr<Engine>(new Engine(std::move(Pc), cp, nnz, prec, use_tc)); };
        h->tune = autotune_cutover(S, mk, data, prec, use_tc, tun);
        tun = h->tune.best;
    }
    HostTimer timer("finish_model");
    Plan P = build_plan(S, use_tc, tun);
    timer.lap("plan");
    // the scatter of the original entries is mapped on the device from the pattern
    h->eng.reset(new Engine(std::move(P), cp, nnz, prec, use_tc));
    timer.lap("engine (device arenas, plan and pattern upload, scatter map)");
    h->t_analyse_ms = ms_since(t0);
    h->first_h2d_bytes = h->eng->plan_bytes() + (early ? nnz * (int64_t)sizeof(int64_t) : 0);
    int64_t e;
    if (early) {
        early->wait(h->eng->stream());
        e = h->eng->factor(early->vals, true);
        early->release(h->eng->stream());
        h->first_h2d_bytes += nnz * (int64_t)sizeof(double);
    } else {
        e = h->eng->factor(data, false);
    }
    timer.lap("first numeric phase (values upload, graph capture)");
    if (e >= 0) {
        *err_dof = h->owner[e];
        set_error("not positive definite");
        return false;
    }
    return true;
}

// The reference's build (ffi/src/lib.rs:100-229) for the symmetric modes.
RustyfemHandle* build(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                      const int64_t* indices, const double* data, Mode mode, const rfg_options* opt, double* d_out,
                      int64_t* err_dof) {
    *err_dof = -1;
    set_error("");
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<RustyfemHandle> h(new RustyfemHandle());
    apply_options(h.get(), opt);
    std::vector<double> diag;
    std::vector<char> coupled;
    // large positive definite systems: the values and row indices start their way to the
    // device now, beside the host stages
    std::unique_ptr<EarlyUpload> early;
    const int64_t nnz0 = n > 0 ? indptr[n] : 0;
    if (mode == Mode::Pd && nnz0 >= ((int64_t)1 << 20) && nnz0 < ((int64_t)1 << 40) && have_device()) {
        early.reset(new EarlyUpload());
        early->start(data, indices, nnz0);
    }
    if (!prepare_model(h.get(), n, nn, loc, coords, indptr, indices, data, mode, diag, coupled, err_dof)) return nullptr;
    if (mode == Mode::Indef) {
        if (!have_device()) {
            set_error("no CUDA device: the numeric phase of librustyfem_gpu runs on the GPU only");
            return nullptr;
        }
        // the caller's lower triangle into the internal lower CSC (ffi/src/lib.rs:191-202)
        const Symbolic& S = h->sym;
        std::vector<double> val(h->lrowidx.size(), 0.0);
        for (int64_t c = 0; c < h->ncaller; c++) {
            int64_t qc = h->eq[c];
            if (qc < 0) continue;
            for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                int64_t r = indices[p], qr = h->eq[r];
                if (qr < 0 || r < c) continue;
                int64_t rr = std::max(qr, qc), cc = std::min(qr, qc);
                auto b = h->lrowidx.begin() + h->lcolptr[cc], e = h->lrowidx.begin() + h->lcolptr[cc + 1];
                auto it = std::lower_bound(b, e, rr);
                val[it - h->lrowidx.begin()] += data[p];
            }
        }
        h->ieng.reset(new IndefEngine(S, h->lcolptr, h->lrowidx, 0.01));
        h->t_analyse_ms = ms_since(t0);
        int64_t e = h->ieng->factor(val.data());
        if (e >= 0) {
            *err_dof = h->owner[e];
            set_error("singular matrix");
            return nullptr;
        }
        const IndefStats& st = h->ieng->stats();
        int64_t neg = st.neg, pos = st.pos;
        for (auto& pr : h->iso) {
            if (pr.second < 0.0)
                neg++;
            else
                pos++;
        }
        h->inertia[0] = neg;
        h->inertia[1] = st.zero;
        h->inertia[2] = pos;
        h->factor_size = st.factor_size;
        return h.release();
    }
    if (mode == Mode::Lu) {
        if (!have_device()) {
            set_error("no CUDA device: the numeric phase of librustyfem_gpu runs on the GPU only");
            return nullptr;
        }
        // all of the caller's entries into the full matrix of the lower pattern: the lower
        // triangle, and the strict upper triangle transposed (ffi/src/lib.rs:176-187,
        // src/sparse/lu.rs:40-47)
        const Symbolic& S = h->sym;
        std::vector<double> lval(h->lrowidx.size(), 0.0), uval(h->lrowidx.size(), 0.0);
        for (int64_t c = 0; c < h->ncaller; c++) {
            int64_t qc = h->eq[c];
            if (qc < 0) continue;
            for (int64_t p = indptr[c]; p < indptr[c + 1]; p++) {
                int64_t qr = h->eq[indices[p]];
                if (qr < 0) continue;
                // A(qr, qc): lower (qr, qc), or upper_t at row qc of column qr
                const int64_t rr = qr >= qc ? qr : qc, cc = qr >= qc ? qc : qr;
                auto b = h->lrowidx.begin() + h->lcolptr[cc], e = h->lrowidx.begin() + h->lcolptr[cc + 1];
                auto it = std::lower_bound(b, e, rr);
                (qr >= qc ? lval : uval)[it - h->lrowidx.begin()] += data[p];
            }
        }
        h->leng.reset(new LuEngine(S, h->lcolptr, h->lrowidx, 0.01));
        h->t_analyse_ms = ms_since(t0);
        int64_t e = h->leng->factor(lval.data(), uval.data());
        if (e >= 0) {
            *err_dof = h->owner[e];
            set_error("singular matrix");
            return nullptr;
        }
        h->inertia[0] = h->inertia[1] = h->inertia[2] = -1;
        h->factor_size = h->leng->stats().factor_size;
        return h.release();
    }
    if (!finish_model(h.get(), indptr, indices, data, t0, err_dof, early.get())) return nullptr;
    int64_t N = h->ncaller;
    if (d_out) {
        std::vector<double> dq(h->n_sym);
        if (h->n_sym > 0) h->eng->pivots_to_host(dq.data());
        for (int64_t i = 0; i < N; i++) d_out[i] = coupled[i] ? dq[h->eq[i]] : diag[i];
    }
    h->inertia[0] = 0;
    h->inertia[1] = 0;
    h->inertia[2] = N;
    ensure_maps(h.get());
    return h.release();
}

// Many independent models as one factorization: their trees form a forest whose
// levels are factored together (the combined handle numbers the models' DOFs one
// model after the other).
RustyfemHandle* build_batch(size_t nmodels, const size_t* n, const size_t* nn, const int64_t* const* loc,
                            const double* const* coords, const int64_t* const* indptr, const int64_t* const* indices,
                            const double* const* data, const rfg_options* opt, int64_t* err_model, int64_t* err_dof) {
    *err_dof = -1;
    *err_model = -1;
    set_error("");
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<RustyfemHandle> h(new RustyfemHandle());
    apply_options(h.get(), opt);
    std::vector<int64_t> cdof(nmodels + 1, 0), cnnz(nmodels + 1, 0), cnode(nmodels + 1, 0);
    std::vector<std::unique_ptr<RustyfemHandle>> parts(nmodels);
    for (size_t i = 0; i < nmodels; i++) {
        parts[i].reset(new RustyfemHandle());
        parts[i]->opt = h->opt;
        std::vector<double> diag;
        std::vector<char> coupled;
        if (!prepare_model(parts[i].get(), n[i], nn[i], loc[i], coords[i], indptr[i], indices[i], data[i], Mode::Pd,
                           diag, coupled, err_dof)) {
            *err_model = (int64_t)i;
            return nullptr;
        }
        cdof[i + 1] = cdof[i] + (int64_t)n[i];
        cnnz[i + 1] = cnnz[i] + parts[i]->nnz;
        cnode[i + 1] = cnode[i] + (int64_t)nn[i];
    }
    // merged forest, combined caller numbering and CSC
    Symbolic& S = h->sym;
    S.n = 0;
    std::vector<int64_t> nsym_off(nmodels + 1, 0);
    std::vector<int64_t> cindptr(cdof[nmodels] + 1, 0), cindices(cnnz[nmodels]);
    h->eq.assign(cdof[nmodels], -1);
    for (size_t i = 0; i < nmodels; i++) {
        const Symbolic& P = parts[i]->sym;
        int64_t noff = S.n, foff = (int64_t)S.fronts.size(), roff = (int64_t)S.rows.size(),
                coff = (int64_t)S.children.size();
        for (SymFront f : P.fronts) {
            f.start += noff;
            f.rows_off += roff;
            f.child_off += coff;
            if (f.parent >= 0) f.parent += foff;
            S.fronts.push_back(f);
        }
        for (int64_t r : P.rows) S.rows.push_back(r + noff);
        for (int64_t c : P.children) S.children.push_back(c + foff);
        for (int64_t r : P.roots) S.roots.push_back(r + foff);
        S.n += P.n;
        nsym_off[i + 1] = S.n;
        for (int64_t c = 0; c < (int64_t)n[i]; c++) {
            cindptr[cdof[i] + c + 1] = cnnz[i] + indptr[i][c + 1];
            int64_t q = parts[i]->eq[c];
            h->eq[cdof[i] + c] = q >= 0 ? q + noff : -1;
        }
        for (int64_t p = 0; p < parts[i]->nnz; p++) cindices[cnnz[i] + p] = indices[i][p] + cdof[i];
        for (auto& pr : parts[i]->iso) h->iso.push_back({pr.first + cdof[i], pr.second});
    }
    h->mode = Mode::Pd;
    h->ncaller = cdof[nmodels];
    h->nn = cnode[nmodels];
    h->nnz = cnnz[nmodels];
    h->n_sym = S.n;
    h->owner.assign(S.n, 0);
    for (int64_t i = 0; i < h->ncaller; i++)
        if (h->eq[i] >= 0) h->owner[h->eq[i]] = i;
    h->work = S.work();
    h->factor_size = S.factor_size();
    std::vector<double> cdata(cnnz[nmodels]);
    for (size_t i = 0; i < nmodels; i++)
        std::copy(data[i], data[i] + parts[i]->nnz, cdata.begin() + cnnz[i]);
    parts.clear();
    int64_t e = -1;
    if (!finish_model(h.get(), cindptr.data(), cindices.data(), cdata.data(), t0, &e)) {
        if (e >= 0) {
            int64_t m = (int64_t)(std::upper_bound(cdof.begin(), cdof.end(), e) - cdof.begin()) - 1;
            *err_model = m;
            *err_dof = e - cdof[m];
        }
        return nullptr;
    }
    h->inertia[2] = h->ncaller;
    h->batch_dof_off = cdof;
    // refinement judges every model on its own backward error
    if (h->eng) h->eng->set_segments(nsym_off);
    ensure_maps(h.get());
    return h.release();
}

RustyfemHandle* guarded_build(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                              const int64_t* indices, const double* data, Mode mode, const rfg_options* opt,
                              double* d_out, int64_t* err_dof) {
    try {
        return build(n, nn, loc, coords, indptr, indices, data, mode, opt, d_out, err_dof);
    } catch (const std::exception& ex) {
        *err_dof = -1;
        set_error(ex.what());
        return nullptr;
    }
}

// The caller-numbering maps of a handle on the device (caller DOF -> internal equation,
// the uncoupled DOFs and their pivots): uploaded once, when the handle is built.
void ensure_maps(const RustyfemHandle* h) {
    if (h->d_eq) return;
    h->d_eq = (decltype(h->d_eq))dev_alloc(std::max<int64_t>(h->ncaller, 1) * sizeof(int64_t), 0);
    if (h->ncaller > 0)
        RFG_CUDA(cudaMemcpy(h->d_eq, h->eq.data(), h->ncaller * sizeof(int64_t), cudaMemcpyHostToDevice));
    int64_t ni = (int64_t)h->iso.size();
    h->d_iso_idx = (decltype(h->d_iso_idx))dev_alloc(std::max<int64_t>(ni, 1) * sizeof(int64_t), 0);
    h->d_iso_d = (decltype(h->d_iso_d))dev_alloc(std::max<int64_t>(ni, 1) * sizeof(double), 0);
    std::vector<int64_t> ii(ni);
    std::vector<double> dd(ni);
    for (int64_t i = 0; i < ni; i++) {
        ii[i] = h->iso[i].first;
        dd[i] = h->iso[i].second;
    }
    if (ni > 0) {
        RFG_CUDA(cudaMemcpy(h->d_iso_idx, ii.data(), ni * sizeof(int64_t), cudaMemcpyHostToDevice));
        RFG_CUDA(cudaMemcpy(h->d_iso_d, dd.data(), ni * sizeof(double), cudaMemcpyHostToDevice));
    }
}

// Entry points that take device pointers run on the handle's stream, a non-blocking
// stream. On entry it waits for the work queued before the call on the legacy default
// stream (with which every blocking stream synchronizes) and on the calling thread's
// per-thread default stream, so that data the caller produced there is complete.
void order_after_caller(const RustyfemHandle* h, cudaStream_t st) {
    if (!h->caller_ev) RFG_CUDA(cudaEventCreateWithFlags(&h->caller_ev, cudaEventDisableTiming));
    RFG_CUDA(cudaEventRecord(h->caller_ev, cudaStreamLegacy));
    RFG_CUDA(cudaStreamWaitEvent(st, h->caller_ev, 0));
    RFG_CUDA(cudaEventRecord(h->caller_ev, cudaStreamPerThread));
    RFG_CUDA(cudaStreamWaitEvent(st, h->caller_ev, 0));
}

void ensure_buffers(const RustyfemHandle* h, int64_t nrhs) {
    int64_t need = std::max<int64_t>(1, nrhs);
    ensure_maps(h);
    if (h->buf_cap < need) {
        for (double** p : {&h->d_b, &h->d_X, &h->d_B})
            if (*p) dev_free(*p, 0);
        h->d_b = (decltype(h->d_b))dev_alloc(std::max<int64_t>(h->ncaller * need, 1) * sizeof(double), 0);
        h->d_X = (decltype(h->d_X))dev_alloc(std::max<int64_t>(h->n_sym * need, 1) * sizeof(double), 0);
        h->d_B = (decltype(h->d_B))dev_alloc(std::max<int64_t>(h->n_sym * need, 1) * sizeof(double), 0);
        h->buf_cap = need;
    }
}

int32_t solve_impl(const RustyfemHandle* h, size_t nrhs_, double* b, rfg_solve_stats* stats, bool on_device = false) {
    auto t0 = std::chrono::steady_clock::now();
    int64_t n = h->ncaller, nrhs = (int64_t)nrhs_;
    if (stats) memset(stats, 0, sizeof(*stats));
    if (n == 0 || nrhs == 0) return 0;
    std::lock_guard<std::mutex> lock(h->mu);
    if (h->ieng || h->leng) {
        // the indefinite and LU paths: their own sweeps, no refinement (ffi/src/lib.rs:337-371)
        cudaStream_t st = h->ieng ? h->ieng->stream() : h->leng->stream();
        ensure_buffers(h, std::min<int64_t>(nrhs, 32));
        if (on_device) order_after_caller(h, st);
        for (int64_t j0 = 0; j0 < nrhs; j0 += 32) {
            int64_t nr = std::min<int64_t>(32, nrhs - j0);
            double* bj = b + j0 * n;
            double* db = on_device ? bj : h->d_b;
            if (!on_device) RFG_CUDA(cudaMemcpyAsync(h->d_b, bj, n * nr * sizeof(double), cudaMemcpyHostToDevice, st));
            launch_gather_rhs(db, h->d_X, h->d_eq, n, h->n_sym, nr, st);
            if (h->ieng)
                h->ieng->solve_device(h->d_X, nr);
            else
                h->leng->solve_device(h->d_X, nr);
            launch_scatter_rhs(db, h->d_X, h->d_eq, h->d_iso_idx, h->d_iso_d, (int64_t)h->iso.size(), n, h->n_sym, nr, st);
            if (!on_device) RFG_CUDA(cudaMemcpyAsync(bj, h->d_b, n * nr * sizeof(double), cudaMemcpyDeviceToHost, st));
            RFG_CUDA(cudaStreamSynchronize(st));
        }
        if (stats) stats->t_solve_ms = ms_since(t0);
        return 0;
    }
    if (!h->eng) {
        if (on_device) {
            ensure_buffers(h, 1);
            // the legacy default stream: ordered after the caller's work on it
            launch_scatter_rhs(b, nullptr, nullptr, h->d_iso_idx, h->d_iso_d, (int64_t)h->iso.size(), n, 0, nrhs, 0);
            RFG_CUDA(cudaStreamSynchronize(0));
            return 0;
        }
        // no coupled DOF: only the uncoupled ones
        for (int64_t j = 0; j < nrhs; j++)
            for (auto& pr : h->iso) b[pr.first + j * n] /= pr.second;
        return 0;
    }
    Engine& E = *h->eng;
    cudaStream_t st = E.stream();
    // chunks of at most 32 right-hand sides for the refined path
    const int64_t CH = 32;
    ensure_buffers(h, std::min(nrhs, CH));
    if (on_device) order_after_caller(h, st);
    int32_t iters = 0;
    double eta = 0.0, rr = 0.0;
    int64_t l0 = E.solve_launches;
    for (int64_t j0 = 0; j0 < nrhs; j0 += CH) {
        int64_t nr = std::min(CH, nrhs - j0);
        double* bj = b + j0 * n;
        double* db = on_device ? bj : h->d_b;
        if (!on_device) RFG_CUDA(cudaMemcpyAsync(h->d_b, bj, n * nr * sizeof(double), cudaMemcpyHostToDevice, st));
        launch_gather_rhs(db, h->d_B, h->d_eq, n, h->n_sym, nr, st);
        if (h->opt.refine_max_iter > 0 || stats) {
            SolveStats s = E.solve_refined(h->d_X, h->d_B, nr, h->opt.refine_tol, h->opt.refine_max_iter);
            iters = std::max(iters, s.iterations);
            eta = std::max(eta, s.backward_error);
            rr = std::max(rr, s.rel_residual);
        } else {
            RFG_CUDA(cudaMemcpyAsync(h->d_X, h->d_B, h->n_sym * nr * sizeof(double), cudaMemcpyDeviceToDevice, st));
            E.solve_device(h->d_X, nr);
        }
        launch_scatter_rhs(db, h->d_X, h->d_eq, h->d_iso_idx, h->d_iso_d, (int64_t)h->iso.size(), n, h->n_sym, nr, st);
        if (!on_device) RFG_CUDA(cudaMemcpyAsync(bj, h->d_b, n * nr * sizeof(double), cudaMemcpyDeviceToHost, st));
        RFG_CUDA(cudaStreamSynchronize(st));
    }
    E.chain_check();
    if (stats) {
        stats->iterations = iters;
        stats->backward_error = eta;
        stats->rel_residual = rr;
        stats->t_solve_ms = ms_since(t0);
        stats->launches = (int32_t)(E.solve_launches - l0);
    }
    return 0;
}

}  // namespace

extern "C" {

RustyfemHandle* rustyfem_factor(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                                const int64_t* indices, const double* data, double* d_out, int64_t* err_dof) {
    return guarded_build(n, nn, loc, coords, indptr, indices, data, Mode::Pd, nullptr, d_out, err_dof);
}

RustyfemHandle* rfg_factor_ex(size_t n, size_t nn, const int64_t* loc, const double* coords, const int64_t* indptr,
                              const int64_t* indices, const double* data, const rfg_options* opt, double* d_out,
                              int64_t* err_dof) {
    rfg_options o{};
    o.refine_max_iter = -1;
    if (opt) o = *opt;
    return guarded_build(n, nn, loc, coords, indptr, indices, data, Mode::Pd, &o, d_out, err_dof);
}

RustyfemHandle* rustyfem_factor_indef(size_t n, size_t nn, const int64_t* loc, const double* coords,
                                      const int64_t* indptr, const int64_t* indices, const double* data,
                                      int64_t* inertia_out, int64_t* err_dof) {
    RustyfemHandle* h = guarded_build(n, nn, loc, coords, indptr, indices, data, Mode::Indef, nullptr, nullptr, err_dof);
    if (h && inertia_out) std::copy(h->inertia, h->inertia + 3, inertia_out);
    return h;
}

RustyfemHandle* rustyfem_factor_unsym(size_t n, size_t nn, const int64_t* loc, const double* coords,
                                      const int64_t* indptr, const int64_t* indices, const double* data,
                                      int64_t* err_dof) {
    return guarded_build(n, nn, loc, coords, indptr, indices, data, Mode::Lu, nullptr, nullptr, err_dof);
}

RustyfemHandle* rfg_batch_factor(size_t nmodels, const size_t* n, const size_t* nn, const int64_t* const* loc,
                                 const double* const* coords, const int64_t* const* indptr,
                                 const int64_t* const* indices, const double* const* data, const rfg_options* opt,
                                 int64_t* err_model, int64_t* err_dof) {
    rfg_options o{};
    o.refine_max_iter = -1;
    if (opt) o = *opt;
    try {
        return build_batch(nmodels, n, nn, loc, coords, indptr, indices, data, &o, err_model, err_dof);
    } catch (const std::exception& ex) {
        *err_dof = -1;
        *err_model = -1;
        set_error(ex.what());
        return nullptr;
    }
}

int32_t rustyfem_inertia(const RustyfemHandle* h, int64_t* out) {
    if (!h || h->leng) return -1;  // no inertia for an LU handle (ffi/src/lib.rs:320-329)
    // a positive definite handle reports [0, 0, n] (ffi/src/lib.rs:228), an indefinite one its inertia
    std::copy(h->inertia, h->inertia + 3, out);
    return 0;
}

int32_t rustyfem_solve(const RustyfemHandle* h, size_t nrhs, double* b) {
    try {
        return solve_impl(h, nrhs, b, nullptr);
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t rfg_solve_ex(const RustyfemHandle* h, size_t nrhs, double* b, rfg_solve_stats* stats) {
    try {
        return solve_impl(h, nrhs, b, stats);
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

void rustyfem_info(const RustyfemHandle* h, double* out) {
    out[0] = h->work;
    out[1] = (double)h->factor_size;
}

void rustyfem_order(const RustyfemHandle* h, int64_t* out) {
    int64_t next = h->n_sym;
    for (int64_t i = 0; i < h->ncaller; i++) out[i] = h->eq[i] >= 0 ? h->eq[i] : next++;
}

void rustyfem_free(RustyfemHandle* h) { delete h; }

static int64_t refactor_impl(RustyfemHandle* h, const double* data, bool on_device) {
    try {
        set_error("");
        if (!h->eng) return -1;
        std::lock_guard<std::mutex> lock(h->mu);
        if (on_device) order_after_caller(h, h->eng->stream());
        int64_t e = h->eng->factor(data, on_device);
        if (e >= 0) {
            set_error("not positive definite");
            return h->owner[e];
        }
        return -1;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -2;
    }
}

int64_t rfg_refactor(RustyfemHandle* h, const double* data) { return refactor_impl(h, data, false); }

int64_t rfg_refactor_device(RustyfemHandle* h, const double* data_device) { return refactor_impl(h, data_device, true); }

int32_t rfg_solve_device(const RustyfemHandle* h, size_t nrhs, double* b_device, rfg_solve_stats* stats) {
    try {
        return solve_impl(h, nrhs, b_device, stats, true);
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t rfg_solve_device_noalloc(const RustyfemHandle* h, size_t nrhs_, double* b) {
    try {
        set_error("");
        if (!h) {
            set_error("rfg_solve_device_noalloc: null handle");
            return -1;
        }
        if (h->ieng || h->leng) {
            set_error("rfg_solve_device_noalloc: positive definite handles only (solve indefinite and LU ones "
                      "with rfg_solve_device)");
            return -1;
        }
        int64_t n = h->ncaller, nrhs = (int64_t)nrhs_;
        if (n == 0 || nrhs == 0) return 0;
        std::lock_guard<std::mutex> lock(h->mu);
        if (!h->d_eq) {
            set_error("rfg_solve_device_noalloc: the handle has no device maps");
            return -1;
        }
        const int64_t CH = 32;
        const int64_t nr_max = std::min(nrhs, CH);
        const int64_t niso = (int64_t)h->iso.size();
        auto r256 = [](int64_t b) { return (std::max<int64_t>(b, 1) + 255) / 256 * 256; };
        // scratch layout: X (n_sym · nr_max double), then the sweep workspace; the
        // caller-numbering maps live with the handle (uploaded when it was built)
        int64_t need = 0;
        if (h->eng) need += r256(h->n_sym * nr_max * 8) + h->eng->sweep_workspace_bytes(nr_max);
        if (need > NOALLOC_SCRATCH_BYTES) {
            set_error("rfg_solve_device_noalloc: this handle needs " + std::to_string(need) + " bytes of scratch for " +
                      std::to_string(nr_max) + " right-hand side(s) per sweep; the fixed scratch holds " +
                      std::to_string(NOALLOC_SCRATCH_BYTES) + " bytes (use rfg_solve_device)");
            return -1;
        }
        char* p = (char*)noalloc_scratch();
        const int64_t* d_eq = h->d_eq;
        const int64_t* d_iso_idx = h->d_iso_idx;
        const double* d_iso_d = h->d_iso_d;
        cudaStream_t st = h->eng ? h->eng->stream() : (cudaStream_t)0;
        if (!h->eng) {
            launch_scatter_rhs(b, nullptr, nullptr, d_iso_idx, d_iso_d, niso, n, 0, nrhs, st);
            RFG_CUDA(cudaStreamSynchronize(st));
            return 0;
        }
        Engine& E = *h->eng;
        order_after_caller(h, st);
        double* X = (double*)p;
        p += r256(h->n_sym * nr_max * 8);
        const Engine::SweepWorkspace ws = E.carve_sweep_workspace(p, nr_max);
        for (int64_t j0 = 0; j0 < nrhs; j0 += CH) {
            int64_t nr = std::min(CH, nrhs - j0);
            double* bj = b + j0 * n;
            launch_gather_rhs(bj, X, d_eq, n, h->n_sym, nr, st);
            E.solve_sweep_on(X, nr, ws);
            launch_scatter_rhs(bj, X, d_eq, d_iso_idx, d_iso_d, niso, n, h->n_sym, nr, st);
        }
        RFG_CUDA(cudaStreamSynchronize(st));
        E.chain_check();
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

void rfg_release_cached_memory(void) {
    try {
        release_cached_memory();
        host_release_cached();
    } catch (const std::exception& ex) {
        set_error(ex.what());
    }
}

void* rfg_stream(const RustyfemHandle* h) { return h->eng ? (void*)h->eng->stream() : nullptr; }

void rfg_set_profiling(RustyfemHandle* h, int32_t on) {
    if (h->eng) h->eng->set_profiling(on);
}

int32_t rfg_factor_stats_get(const RustyfemHandle* h, rfg_factor_stats* out) {
    if (!h) return -1;
    memset(out, 0, sizeof(*out));
    out->work = h->work;
    out->factor_size = (double)h->factor_size;
    out->t_analyse_ms = h->t_analyse_ms;
    h->sym.largest_front(&out->largest_k, &out->largest_u);
    out->nfronts = (int64_t)h->sym.fronts.size();
    if (h->eng) {
        const Plan& P = h->eng->plan();
        size_t es = h->eng->precision() == PREC_FP64 ? 8 : 4;
        out->t_factor_ms = h->eng->last_factor.t_factor_ms;
        out->launches = h->eng->last_factor.launches;
        out->nlevels = P.nlevels;
        out->nsteps = (int64_t)P.steps.size();
        out->panel_bytes = P.panel_elems * (int64_t)es;
        out->update_bytes = P.upd_elems * (int64_t)es;
        out->schur_ms = h->eng->last_factor.schur_ms;
        out->schur_flops = h->eng->last_factor.schur_flops;
        out->schur_launches = h->eng->last_factor.schur_launches;
        out->h2d_bytes = h->eng->last_factor.h2d_bytes + h->first_h2d_bytes;
        for (int i = 0; i < 7; i++) out->phase_ms[i] = h->eng->last_factor.phase_ms[i];
        out->tile_cutover_rows = P.big_min_rows;
        out->tc_kind = h->eng->tc_kind();
        out->outer_tile_n = out->tc_kind ? P.outer_tn : 0;
        out->precision = h->eng->precision() == PREC_MIXED ? RFG_MIXED : RFG_FP64;
        out->schur_entries = h->eng->last_factor.schur_entries;
        out->schur_opvals = h->eng->last_factor.schur_opvals;
    }
    if (h->ieng) {
        out->t_factor_ms = h->ieng->stats().t_factor_ms;
        out->launches = h->ieng->stats().launches;
        out->delayed = h->ieng->stats().delayed;
        out->precision = RFG_FP64;
    }
    if (h->leng) {
        out->t_factor_ms = h->leng->stats().t_factor_ms;
        out->launches = h->leng->stats().launches;
        out->delayed = h->leng->stats().delayed;
        out->precision = RFG_FP64;
    }
    return 0;
}

size_t rfg_tune_report(const RustyfemHandle* h, int64_t* cutover, double* ms, size_t cap) {
    return rfg_tune_report_ex(h, cutover, nullptr, ms, cap);
}

size_t rfg_tune_report_ex(const RustyfemHandle* h, int64_t* cutover, int64_t* tile_n, double* ms, size_t cap) {
    if (!h) return 0;
    size_t n = h->tune.cutover.size();
    for (size_t i = 0; i < n && i < cap; i++) {
        if (cutover) cutover[i] = h->tune.cutover[i];
        if (tile_n) tile_n[i] = i < h->tune.tile_n.size() ? h->tune.tile_n[i] : 0;
        if (ms) ms[i] = h->tune.ms[i];
    }
    return n;
}

size_t rfg_handle_nfronts(const RustyfemHandle* h) { return h->sym.fronts.size(); }

void rfg_handle_fronts(const RustyfemHandle* h, int64_t* out4) {
    size_t i = 0;
    for (auto& f : h->sym.fronts) {
        out4[4 * i] = f.start;
        out4[4 * i + 1] = f.k;
        out4[4 * i + 2] = f.u;
        out4[4 * i + 3] = f.nchild;
        i++;
    }
}

const char* rfg_last_error(void) { return g_err.c_str(); }

int32_t rfg_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Engine-level matrix (src/solver/api.rs:21-60, src/solver/direct.rs)
// ---------------------------------------------------------------------------
struct RfgMatrix {
    Symbolic sym;
    std::vector<int64_t> colptr, rowidx;
    std::vector<double> val;
    std::unique_ptr<Engine> eng;
    int32_t precision = RFG_FP64;
    mutable double* d_X = nullptr;
    mutable double* d_B = nullptr;
    // values assembled on the device (rfg_assembly_*); current instead of `val` while dev_current
    double* d_val = nullptr;
    bool dev_current = false;
    mutable std::mutex mu;
    ~RfgMatrix() {
        eng.reset();
        if (d_X) cudaFree(d_X);
        if (d_B) cudaFree(d_B);
        if (d_val) cudaFree(d_val);
    }
    // host values current again (after a device assembly): copy them down once
    void pull_values() {
        if (!dev_current) return;
        if (!val.empty())
            RFG_CUDA(cudaMemcpyAsync(val.data(), d_val, val.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                     eng->stream()));
        RFG_CUDA(cudaStreamSynchronize(eng->stream()));
        dev_current = false;
    }
};

struct RfgAssembly {
    RfgMatrix* m;
    std::unique_ptr<Assembler> a;
};

struct RfgSymbolic {
    Symbolic sym;
    Graph g;
    std::vector<double> coords;
};

namespace {

// RUSTYFEM_TIMING (src/settings.rs:46): the engine-level solver prints its analysis and
// factorization times to stderr in the reference's format (src/solver/direct.rs:27-35,
// :58-60).
bool timing_on() { return getenv("RUSTYFEM_TIMING") != nullptr; }

// Rust's `{:.2e}` (LowerExp with two decimals): "8.73e12", "1.00e-5" — no '+' and no
// zero padding in the exponent.
std::string rust_exp2(double v) {
    char buf[64];
    snprintf(buf, sizeof buf, "%.2e", v);
    std::string t(buf);
    size_t e = t.find('e');
    if (e == std::string::npos) return t;
    return t.substr(0, e) + "e" + std::to_string(atoi(t.c_str() + e + 1));
}

Graph make_graph(size_t nb, const double* coords, const int64_t* adj_ptr, const int64_t* adj_idx, const int64_t* ndof) {
    Graph g;
    g.nn = (int64_t)nb;
    g.coords = coords;
    g.adj_ptr.assign(adj_ptr, adj_ptr + nb + 1);
    g.adj_idx.assign(adj_idx, adj_idx + adj_ptr[nb]);
    g.ndof.assign(ndof, ndof + nb);
    return g;
}

}  // namespace

extern "C" {

RfgMatrix* rfg_matrix_prepare(size_t nb, const double* coords, const int64_t* adj_ptr, const int64_t* adj_idx,
                              const int64_t* ndof, int32_t leaf, int32_t precision) {
    try {
        set_error("");
        auto t0 = std::chrono::steady_clock::now();
        std::unique_ptr<RfgMatrix> m(new RfgMatrix());
        Graph g = make_graph(nb, coords, adj_ptr, adj_idx, ndof);
        m->sym = analyse(g, leaf > 0 ? leaf : ENGINE_LEAF);
        lower_pattern(m->sym, g, m->colptr, m->rowidx);
        if (timing_on()) {
            int64_t lk = 0, lu = 0;
            m->sym.largest_front(&lk, &lu);
            fprintf(stderr, "analysis: %.3f s  flops: %s  factor: %lld MB  largest front: (%lld, %lld)\n",
                    ms_since(t0) / 1e3, rust_exp2(m->sym.work()).c_str(),
                    (long long)((m->sym.factor_size() * 8) >> 20), (long long)lk, (long long)lu);
        }
        m->val.assign(m->rowidx.size(), 0.0);
        m->precision = precision;
        if (!have_device()) {
            set_error("no CUDA device: the numeric phase of librustyfem_gpu runs on the GPU only");
            return nullptr;
        }
        bool use_tc = precision == RFG_MIXED;
        Plan P = build_plan(m->sym, use_tc);
        Scatter X = scatter_from_lower(P, m->sym, m->colptr, m->rowidx);
        m->eng.reset(new Engine(std::move(P), std::move(X), (int64_t)m->val.size(),
                                precision == RFG_MIXED ? PREC_MIXED : PREC_FP64, use_tc));
        return m.release();
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return nullptr;
    }
}

size_t rfg_matrix_n(const RfgMatrix* m) { return (size_t)m->sym.n; }

void rfg_matrix_first_dof(const RfgMatrix* m, int64_t* out) {
    std::copy(m->sym.first_dof.begin(), m->sym.first_dof.end(), out);
}

void rfg_matrix_zero(RfgMatrix* m) {
    std::fill(m->val.begin(), m->val.end(), 0.0);
    m->dev_current = false;
}

int32_t rfg_matrix_add(RfgMatrix* m, size_t r, size_t c, double v) {
    // src/sparse.rs:47-51
    if (c >= (size_t)m->sym.n) return -1;
    if (m->dev_current) {
        try {
            m->pull_values();
        } catch (const std::exception& ex) {
            set_error(ex.what());
            return -1;
        }
    }
    auto b = m->rowidx.begin() + m->colptr[c], e = m->rowidx.begin() + m->colptr[c + 1];
    auto it = std::lower_bound(b, e, (int64_t)r);
    if (it == e || *it != (int64_t)r) return -1;
    m->val[it - m->rowidx.begin()] += v;
    return 0;
}

int32_t rfg_matrix_add_many(RfgMatrix* m, size_t cnt, const int64_t* r, const int64_t* c, const double* v) {
    for (size_t i = 0; i < cnt; i++)
        if (rfg_matrix_add(m, (size_t)r[i], (size_t)c[i], v[i]) != 0) return -1;
    return 0;
}

int64_t rfg_matrix_factor(RfgMatrix* m) {
    try {
        set_error("");
        std::lock_guard<std::mutex> lock(m->mu);
        auto t0 = std::chrono::steady_clock::now();
        int64_t e = m->dev_current ? m->eng->factor(m->d_val, true) : m->eng->factor(m->val.data(), false);
        if (e < 0 && timing_on()) fprintf(stderr, "factorization: %.3f s\n", ms_since(t0) / 1e3);
        return e;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -2;
    }
}

int32_t rfg_matrix_solve(const RfgMatrix* m, double* b) {
    try {
        std::lock_guard<std::mutex> lock(m->mu);
        int64_t n = m->sym.n;
        if (n == 0) return 0;
        Engine& E = *m->eng;
        cudaStream_t st = E.stream();
        if (!m->d_X) {
            RFG_CUDA(cudaMalloc(&m->d_X, n * sizeof(double)));
            RFG_CUDA(cudaMalloc(&m->d_B, n * sizeof(double)));
        }
        RFG_CUDA(cudaMemcpyAsync(m->d_B, b, n * sizeof(double), cudaMemcpyHostToDevice, st));
        if (m->precision == RFG_MIXED) {
            E.solve_refined(m->d_X, m->d_B, 1, 1e-12, 10);
        } else {
            RFG_CUDA(cudaMemcpyAsync(m->d_X, m->d_B, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            E.solve_device(m->d_X, 1);
        }
        RFG_CUDA(cudaMemcpyAsync(b, m->d_X, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        RFG_CUDA(cudaStreamSynchronize(st));
        E.chain_check();
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

void rfg_matrix_free(RfgMatrix* m) { delete m; }

int32_t rfg_matrix_values(RfgMatrix* m, double* out) {
    try {
        set_error("");
        std::lock_guard<std::mutex> lock(m->mu);
        if (m->dev_current) {
            if (!m->val.empty())
                RFG_CUDA(cudaMemcpyAsync(out, m->d_val, m->val.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                         m->eng->stream()));
            RFG_CUDA(cudaStreamSynchronize(m->eng->stream()));
        } else {
            std::copy(m->val.begin(), m->val.end(), out);
        }
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

size_t rfg_matrix_nnz(const RfgMatrix* m) { return m->val.size(); }

// --- assembly of K on the device ---
RfgAssembly* rfg_assembly_prepare(RfgMatrix* m, size_t nelem, size_t nd, const int64_t* edof) {
    try {
        set_error("");
        if (!m || nd == 0 || nd > 4096 || (nelem > 0 && !edof)) {
            set_error("rfg_assembly_prepare: invalid arguments");
            return nullptr;
        }
        if (nelem > ((size_t)1 << 62) / (nd * nd)) {
            set_error("rfg_assembly_prepare: too many element pairs");
            return nullptr;
        }
        const int64_t n = m->sym.n;
        for (size_t i = 0; i < nelem * nd; i++)
            if (edof[i] < -1 || edof[i] >= n) {
                set_error("rfg_assembly_prepare: equation " + std::to_string(edof[i]) + " out of range");
                return nullptr;
            }
        std::lock_guard<std::mutex> lock(m->mu);
        std::unique_ptr<RfgAssembly> a(new RfgAssembly());
        a->m = m;
        a->a.reset(new Assembler(n, m->colptr.data(), m->rowidx.data(), (int64_t)nelem, (int64_t)nd, edof,
                                 m->eng->stream()));
        if (!m->d_val) RFG_CUDA(cudaMalloc(&m->d_val, std::max<size_t>(m->val.size(), 1) * sizeof(double)));
        return a.release();
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return nullptr;
    }
}

int32_t rfg_assembly_set(RfgAssembly* a, const double* ke) {
    try {
        set_error("");
        std::lock_guard<std::mutex> lock(a->m->mu);
        a->a->assemble(ke, false, a->m->d_val);
        a->m->dev_current = true;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int32_t rfg_assembly_set_device(RfgAssembly* a, const double* d_ke) {
    try {
        set_error("");
        std::lock_guard<std::mutex> lock(a->m->mu);
        a->a->assemble(d_ke, true, a->m->d_val);
        a->m->dev_current = true;
        return 0;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -1;
    }
}

int64_t rfg_assembly_hex8(RfgAssembly* a, size_t nn, const double* xyz, const int64_t* conn, const double* emod,
                          double nu) {
    try {
        set_error("");
        std::lock_guard<std::mutex> lock(a->m->mu);
        int64_t bad = a->a->hex8((int64_t)nn, xyz, conn, emod, nu, a->m->d_val);
        if (bad >= 0) {
            set_error("element " + std::to_string(bad) + " is distorted (det J <= 0 at an integration point)");
            return bad;
        }
        a->m->dev_current = true;
        return -1;
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return -2;
    }
}

void rfg_assembly_times(const RfgAssembly* a, double* out2) {
    out2[0] = a->a->element_ms();
    out2[1] = a->a->gather_ms();
}

size_t rfg_assembly_contributions(const RfgAssembly* a) { return (size_t)a->a->contributions(); }

void rfg_assembly_free(RfgAssembly* a) { delete a; }

// --- host symbolic stage alone ---
RfgSymbolic* rfg_sym_analyse(size_t nb, const double* coords, const int64_t* adj_ptr, const int64_t* adj_idx,
                             const int64_t* ndof, int32_t leaf) {
    try {
        std::unique_ptr<RfgSymbolic> s(new RfgSymbolic());
        s->coords.assign(coords, coords + 3 * nb);
        s->g = make_graph(nb, s->coords.data(), adj_ptr, adj_idx, ndof);
        s->sym = analyse(s->g, leaf > 0 ? leaf : ENGINE_LEAF);
        return s.release();
    } catch (const std::exception& ex) {
        set_error(ex.what());
        return nullptr;
    }
}
size_t rfg_sym_n(const RfgSymbolic* s) { return (size_t)s->sym.n; }
size_t rfg_sym_nfronts(const RfgSymbolic* s) { return s->sym.fronts.size(); }
double rfg_sym_work(const RfgSymbolic* s) { return s->sym.work(); }
size_t rfg_sym_factor_size(const RfgSymbolic* s) { return (size_t)s->sym.factor_size(); }
size_t rfg_sym_total_rows(const RfgSymbolic* s) { return s->sym.rows.size(); }
void rfg_sym_fronts(const RfgSymbolic* s, int64_t* out4) {
    size_t i = 0;
    for (auto& f : s->sym.fronts) {
        out4[4 * i] = f.start;
        out4[4 * i + 1] = f.k;
        out4[4 * i + 2] = f.u;
        out4[4 * i + 3] = f.nchild;
        i++;
    }
}
void rfg_sym_first_dof(const RfgSymbolic* s, int64_t* out) {
    std::copy(s->sym.first_dof.begin(), s->sym.first_dof.end(), out);
}
void rfg_sym_rows(const RfgSymbolic* s, int64_t* out) { std::copy(s->sym.rows.begin(), s->sym.rows.end(), out); }
void rfg_sym_children(const RfgSymbolic* s, int64_t* out) {
    std::copy(s->sym.children.begin(), s->sym.children.end(), out);
}
size_t rfg_sym_nnz(const RfgSymbolic* s) {
    std::vector<int64_t> cp, ri;
    lower_pattern(s->sym, s->g, cp, ri);
    return ri.size();
}
void rfg_sym_pattern(const RfgSymbolic* s, int64_t* colptr, int64_t* rowidx) {
    std::vector<int64_t> cp, ri;
    lower_pattern(s->sym, s->g, cp, ri);
    std::copy(cp.begin(), cp.end(), colptr);
    std::copy(ri.begin(), ri.end(), rowidx);
}
void rfg_sym_plan_stats(const RfgSymbolic* s, int64_t* out4) {
    Plan P = build_plan(s->sym);
    out4[0] = P.nlevels;
    out4[1] = (int64_t)P.steps.size();
    out4[2] = P.panel_elems;
    out4[3] = P.upd_elems;
}
void rfg_selftest_sort_unstable(const int64_t* keys, int64_t n, int64_t limit, int64_t* perm) {
    std::vector<uint64_t> kv((size_t)std::max<int64_t>(n, 0));
    for (int64_t i = 0; i < n; i++) kv[i] = ((uint64_t)keys[i] << 32) | (uint64_t)i;
    rfg::unstable_sort::sort(kv.data(), n, [](uint64_t p, uint64_t q) { return (p >> 32) < (q >> 32); },
                             rfg::unstable_sort::NoFork(), limit);
    for (int64_t i = 0; i < n; i++) perm[i] = (int64_t)(kv[i] & 0xffffffffu);
}

void rfg_sym_plan_flops(const RfgSymbolic* s, int64_t cutover_rows, double* out4) {
    Tuning t;
    if (cutover_rows > 0) t.big_min_rows = cutover_rows;
    Plan P = build_plan(s->sym, false, t);
    out4[0] = P.inner_flops;
    out4[1] = P.outer_flops;
    out4[2] = P.outer_big_flops;
    out4[3] = (double)P.big_tiles;
}
void rfg_sym_free(RfgSymbolic* s) { delete s; }

}  // extern "C"
