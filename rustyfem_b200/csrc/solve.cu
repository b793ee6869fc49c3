// Triangular solves over the elimination tree, and FP64 iterative refinement.
//
// The solve follows the factor's level/step schedule (plan.h), for nrhs
// right-hand sides stored as X[q·nrhs + j] (internal numbering):
//  forward  (leaves up)   the children's update vectors are added into the
//                         front (pivot rows into X, later rows into the front's
//                         update vector V_t), then per pivot block: the NB×NB
//                         unit-lower solve (k_fwd_block), and the product of the
//                         panel rows below it with the solved block, subtracted
//                         from X (pivot rows) or V_t (later rows) (k_fwd_panel);
//  diagonal               X /= D;
//  backward (root down)   per pivot block, last first: partial sums of Lᵀ·x over
//                         row chunks below the block (k_bwd_partial), then their
//                         reduction and the NB×NB unit-upper solve (k_bwd_block).
// This is the multifrontal form of Factor::solve (src/sparse.rs:615-652):
// the same three sweeps, with the updates of each front gathered in its update
// vector instead of being subtracted from x row by row.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "engine.h"

namespace rfg {

namespace {

constexpr int MAXR = 32;  // right-hand sides per sweep
constexpr size_t SM_BLOCK = (NB * (NB + 1) + NB * MAXR) * sizeof(double);
constexpr size_t SM_FPANEL = (PR * (NB + 1) + NB * MAXR) * sizeof(double);
constexpr size_t SM_BPART = (PR * (NB + 1) + PR * (MAXR + 1)) * sizeof(double);

__device__ __forceinline__ int64_t find_slot2(const int64_t* pre, int64_t n, int64_t b) {
    int64_t lo = 0, hi = n;
    while (hi - lo > 1) {
        int64_t mid = (lo + hi) >> 1;
        if (pre[mid] <= b)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// children's update vectors into the parent (one launch per child rank)
__global__ void k_vec_extend_add(double* __restrict__ X, double* __restrict__ V, const DFront* __restrict__ fr,
                                 const int64_t* __restrict__ child, const int64_t* __restrict__ pre, int64_t nchild,
                                 const int32_t* __restrict__ emap, int nrhs) {
    int64_t b = blockIdx.x;
    int64_t i = find_slot2(pre, nchild, b);
    int64_t c = child[i];
    int64_t chunk = b - pre[i];
    const DFront fc = fr[c];
    const DFront fp = fr[fc.parent];
    int64_t x0 = chunk * XR, x1 = min(fc.u, x0 + (int64_t)XR);
    for (int64_t e = threadIdx.x; e < (x1 - x0) * nrhs; e += blockDim.x) {
        int64_t x = x0 + e / nrhs;
        int j = (int)(e % nrhs);
        int64_t pos = emap[fc.emap_off + x];
        double v = V[(fc.vuoff + x) * nrhs + j];
        if (pos < fp.k)
            X[(fp.start + pos) * nrhs + j] += v;
        else
            V[(fp.vuoff + pos - fp.k) * nrhs + j] += v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_fwd_block(double* __restrict__ X, const T* __restrict__ panel,
                                                   const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                   int64_t fr_off, int64_t s, int nrhs) {
    extern __shared__ double sm[];
    double(*L)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    double(*y)[MAXR] = reinterpret_cast<double(*)[MAXR]>(sm + NB * (NB + 1));
    const DFront f = fr[order[fr_off + blockIdx.x]];
    int64_t j0 = s * NB;
    int jb = (int)min((int64_t)NB, f.k - j0);
    const T* blk = panel + f.poff + j0 * f.ldp + j0;
    for (int idx = threadIdx.x; idx < jb * jb; idx += blockDim.x) {
        int r = idx / jb, c = idx - r * jb;
        L[r][c] = c < r ? (double)blk[(int64_t)r * f.ldp + c] : 0.0;
    }
    for (int idx = threadIdx.x; idx < jb * nrhs; idx += blockDim.x) {
        int p = idx / nrhs, j = idx - p * nrhs;
        y[p][j] = X[(f.start + j0 + p) * nrhs + j];
    }
    __syncthreads();
    for (int p = 0; p < jb; p++) {
        for (int idx = threadIdx.x; idx < (jb - p - 1) * nrhs; idx += blockDim.x) {
            int q = p + 1 + idx / nrhs, j = idx % nrhs;
            y[q][j] -= L[q][p] * y[p][j];
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < jb * nrhs; idx += blockDim.x) {
        int p = idx / nrhs, j = idx - p * nrhs;
        X[(f.start + j0 + p) * nrhs + j] = y[p][j];
    }
}

// rows r in [j1, m): target(r) −= L[r, j0:j1]·y, target = X (pivot rows) or V_t (later rows)
template <typename T>
__global__ void __launch_bounds__(PR) k_fwd_panel(double* __restrict__ X, double* __restrict__ V,
                                                  const T* __restrict__ panel, const DFront* __restrict__ fr,
                                                  const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                                  const int64_t* __restrict__ pre_panel, int64_t s, int nrhs) {
    extern __shared__ double sm[];
    double(*Lt)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    double(*y)[MAXR] = reinterpret_cast<double(*)[MAXR]>(sm + PR * (NB + 1));
    int64_t b = blockIdx.x;
    int64_t i = find_slot2(pre_panel, nact, b);
    int64_t chunk = b - pre_panel[i];
    const DFront f = fr[order[fr_off + i]];
    int64_t j0 = s * NB;
    int jb = (int)min((int64_t)NB, f.k - j0);
    int64_t j1 = j0 + jb;
    int64_t r0 = j1 + chunk * PR;
    int nr = (int)min((int64_t)PR, f.m - r0);
    for (int idx = threadIdx.x; idx < nr * NB; idx += blockDim.x) {
        int rr = idx / NB, p = idx - rr * NB;
        Lt[rr][p] = p < jb ? (double)panel[f.poff + (r0 + rr) * f.ldp + j0 + p] : 0.0;
    }
    for (int idx = threadIdx.x; idx < NB * nrhs; idx += blockDim.x) {
        int p = idx / nrhs, j = idx - p * nrhs;
        y[p][j] = p < jb ? X[(f.start + j0 + p) * nrhs + j] : 0.0;
    }
    __syncthreads();
    int rr = threadIdx.x;
    if (rr >= nr) return;
    int64_t r = r0 + rr;
    double* tgt = r < f.k ? X + (f.start + r) * nrhs : V + (f.vuoff + r - f.k) * nrhs;
    for (int j = 0; j < nrhs; j++) {
        double acc = 0.0;
#pragma unroll 16
        for (int p = 0; p < NB; p++) acc = fma(Lt[rr][p], y[p][j], acc);
        tgt[j] -= acc;
    }
}

// partial[b][p·nrhs + j] = Σ_{r in chunk b} L[r, j0 + p]·x(r, j)
template <typename T>
__global__ void __launch_bounds__(256) k_bwd_partial(const double* __restrict__ X, const T* __restrict__ panel,
                                                     const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                     int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre_panel,
                                                     const int64_t* __restrict__ rows, int64_t s, int nrhs,
                                                     double* __restrict__ partial) {
    extern __shared__ double sm[];
    double(*Lt)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    double(*xr)[MAXR + 1] = reinterpret_cast<double(*)[MAXR + 1]>(sm + PR * (NB + 1));
    int64_t b = blockIdx.x;
    int64_t i = find_slot2(pre_panel, nact, b);
    int64_t chunk = b - pre_panel[i];
    const DFront f = fr[order[fr_off + i]];
    int64_t j0 = s * NB;
    int jb = (int)min((int64_t)NB, f.k - j0);
    int64_t j1 = j0 + jb;
    int64_t r0 = j1 + chunk * PR;
    int nr = (int)min((int64_t)PR, f.m - r0);
    for (int idx = threadIdx.x; idx < PR * NB; idx += blockDim.x) {
        int rr = idx / NB, p = idx - rr * NB;
        Lt[rr][p] = (rr < nr && p < jb) ? (double)panel[f.poff + (r0 + rr) * f.ldp + j0 + p] : 0.0;
    }
    for (int idx = threadIdx.x; idx < PR * nrhs; idx += blockDim.x) {
        int rr = idx / nrhs, j = idx - rr * nrhs;
        double v = 0.0;
        if (rr < nr) {
            int64_t r = r0 + rr;
            int64_t q = r < f.k ? f.start + r : rows[f.rows_off + r - f.k];
            v = X[q * nrhs + j];
        }
        xr[rr][j] = v;
    }
    __syncthreads();
    double* out = partial + b * (int64_t)NB * nrhs;
    for (int o = threadIdx.x; o < NB * nrhs; o += blockDim.x) {
        int p = o / nrhs, j = o - p * nrhs;
        double acc = 0.0;
        for (int rr = 0; rr < nr; rr++) acc = fma(Lt[rr][p], xr[rr][j], acc);
        out[o] = acc;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_bwd_block(double* __restrict__ X, const T* __restrict__ panel,
                                                   const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                   int64_t fr_off, const int64_t* __restrict__ pre_panel, int64_t s,
                                                   int nrhs, const double* __restrict__ partial) {
    extern __shared__ double sm[];
    double(*L)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    double(*z)[MAXR] = reinterpret_cast<double(*)[MAXR]>(sm + NB * (NB + 1));
    int64_t i = blockIdx.x;
    const DFront f = fr[order[fr_off + i]];
    int64_t j0 = s * NB;
    int jb = (int)min((int64_t)NB, f.k - j0);
    const T* blk = panel + f.poff + j0 * f.ldp + j0;
    for (int idx = threadIdx.x; idx < jb * jb; idx += blockDim.x) {
        int r = idx / jb, c = idx - r * jb;
        L[r][c] = c < r ? (double)blk[(int64_t)r * f.ldp + c] : 0.0;
    }
    int64_t c0 = pre_panel[i], c1 = pre_panel[i + 1];
    for (int idx = threadIdx.x; idx < jb * nrhs; idx += blockDim.x) {
        int p = idx / nrhs, j = idx - p * nrhs;
        double v = X[(f.start + j0 + p) * nrhs + j];
        for (int64_t c = c0; c < c1; c++) v -= partial[c * (int64_t)NB * nrhs + p * nrhs + j];
        z[p][j] = v;
    }
    __syncthreads();
    for (int p = jb - 1; p >= 0; p--) {
        for (int idx = threadIdx.x; idx < p * nrhs; idx += blockDim.x) {
            int q = idx / nrhs, j = idx % nrhs;
            z[q][j] -= L[p][q] * z[p][j];
        }
        __syncthreads();
    }
    for (int idx = threadIdx.x; idx < jb * nrhs; idx += blockDim.x) {
        int p = idx / nrhs, j = idx - p * nrhs;
        X[(f.start + j0 + p) * nrhs + j] = z[p][j];
    }
}

__global__ void k_divide_d(double* __restrict__ X, const double* __restrict__ d, int64_t n, int nrhs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * nrhs; e += (int64_t)gridDim.x * blockDim.x)
        X[e] /= d[e / nrhs];
}

// caller column-major b (ncaller × nrhs) -> internal X (nsym × nrhs, row-major)
__global__ void k_gather_rhs(const double* __restrict__ b, double* __restrict__ X, const int64_t* __restrict__ eq,
                             int64_t ncaller, int nrhs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ncaller * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = e % ncaller;
        int j = (int)(e / ncaller);
        int64_t q = eq[i];
        if (q >= 0) X[q * nrhs + j] = b[e];
    }
}

__global__ void k_scatter_rhs(double* __restrict__ b, const double* __restrict__ X, const int64_t* __restrict__ eq,
                              int64_t ncaller, int nrhs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < ncaller * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = e % ncaller;
        int j = (int)(e / ncaller);
        int64_t q = eq[i];
        if (q >= 0) b[e] = X[q * nrhs + j];
    }
}

__global__ void k_iso_divide(double* __restrict__ b, const int64_t* __restrict__ idx, const double* __restrict__ dv,
                             int64_t niso, int64_t ncaller, int nrhs) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < niso * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = e % niso;
        int j = (int)(e / niso);
        b[idx[i] + j * ncaller] /= dv[i];
    }
}

// ---------------------------------------------------------------------------
// refinement: y = A x on the full CSR, residual norms
// ---------------------------------------------------------------------------
__global__ void k_gather_values(double* __restrict__ val, const double* __restrict__ src, const int64_t* __restrict__ sidx,
                                int64_t nnz) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x)
        val[e] = src[sidx[e]];
}

// one warp per row; also accumulates |a| row sums when rowsum != null
__global__ void k_spmv(const int64_t* __restrict__ rp, const int64_t* __restrict__ col, const double* __restrict__ val,
                       const double* __restrict__ X, double* __restrict__ Y, int64_t n, int nrhs,
                       double* __restrict__ rowsum) {
    int lane = threadIdx.x & 31;
    for (int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; row < n;
         row += ((int64_t)gridDim.x * blockDim.x) >> 5) {
    int64_t e0 = rp[row], e1 = rp[row + 1];
    for (int j = 0; j < nrhs; j++) {
        double acc = 0.0;
        for (int64_t e = e0 + lane; e < e1; e += 32) acc = fma(val[e], X[col[e] * nrhs + j], acc);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if (lane == 0) Y[row * nrhs + j] = acc;
    }
    if (rowsum) {
        double a = 0.0;
        for (int64_t e = e0 + lane; e < e1; e += 32) a += fabs(val[e]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
        if (lane == 0) rowsum[row] = a;
    }
    }
}

// R = B − AX (in R, AX given), per-RHS reductions: red[j·5 + {0..4}] =
// {max|r|, max|x|, max|b|, Σr², Σb²} accumulated with atomics on nonnegative doubles
__device__ __forceinline__ void atomic_max_nonneg(double* a, double v) {
    atomicMax((unsigned long long*)a, (unsigned long long)__double_as_longlong(v));
}

__global__ void k_residual(double* __restrict__ R, const double* __restrict__ AX, const double* __restrict__ B,
                           const double* __restrict__ X, int64_t n, int nrhs, double* __restrict__ red) {
    __shared__ double s[5][MAXR];
    for (int i = threadIdx.x; i < 5 * MAXR; i += blockDim.x) s[i / MAXR][i % MAXR] = 0.0;
    __syncthreads();
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n * nrhs; e += (int64_t)gridDim.x * blockDim.x) {
        int j = (int)(e % nrhs);
        double r = B[e] - AX[e];
        R[e] = r;
        atomic_max_nonneg(&s[0][j], fabs(r));
        atomic_max_nonneg(&s[1][j], fabs(X[e]));
        atomic_max_nonneg(&s[2][j], fabs(B[e]));
        atomicAdd(&s[3][j], r * r);
        atomicAdd(&s[4][j], B[e] * B[e]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 5 * nrhs; i += blockDim.x) {
        int w = i / nrhs, j = i % nrhs;
        double v = s[w][j];
        if (w < 3)
            atomic_max_nonneg(&red[j * 5 + w], v);
        else
            atomicAdd(&red[j * 5 + w], v);
    }
}

__global__ void k_axpy(double* __restrict__ X, const double* __restrict__ D, int64_t cnt) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
        X[e] += D[e];
}

__global__ void k_max_reduce(const double* __restrict__ v, int64_t n, double* __restrict__ out) {
    double m = 0.0;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x)
        m = fmax(m, v[e]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(out, m);
}

unsigned grid_for(int64_t work, int64_t per = 256) {
    int64_t g = (work + per - 1) / per;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(g, 148 * 32));
}

}  // namespace

void launch_gather_rhs(const double* b, double* X, const int64_t* eq, int64_t ncaller, int64_t nsym, int64_t nrhs,
                       cudaStream_t st) {
    RFG_CUDA(cudaMemsetAsync(X, 0, std::max<int64_t>(nsym * nrhs, 1) * sizeof(double), st));
    if (ncaller * nrhs > 0) k_gather_rhs<<<grid_for(ncaller * nrhs), 256, 0, st>>>(b, X, eq, ncaller, (int)nrhs);
}

void launch_scatter_rhs(double* b, const double* X, const int64_t* eq, const int64_t* iso_idx, const double* iso_d,
                        int64_t niso, int64_t ncaller, int64_t nsym, int64_t nrhs, cudaStream_t st) {
    (void)nsym;
    if (X && ncaller * nrhs > 0) k_scatter_rhs<<<grid_for(ncaller * nrhs), 256, 0, st>>>(b, X, eq, ncaller, (int)nrhs);
    if (niso * nrhs > 0) k_iso_divide<<<grid_for(niso * nrhs), 256, 0, st>>>(b, iso_idx, iso_d, niso, ncaller, (int)nrhs);
}

template <typename T>
void Engine::solve_impl(double* X, int64_t nrhs_total) {
    const Plan& P = plan_;
    const T* panel = (const T*)panel_;
    int64_t launches = 0;
    // X is row-major n × nrhs_total; sweeps of at most MAXR right-hand sides work on a
    // contiguous copy when nrhs_total > MAXR
    if (nrhs_total > MAXR) {
        double* tmp = (double*)nullptr;
        RFG_CUDA(cudaMallocAsync((void**)&tmp, P.n * MAXR * sizeof(double), stream_));
        for (int64_t j0 = 0; j0 < nrhs_total; j0 += MAXR) {
            int64_t nr = std::min<int64_t>(MAXR, nrhs_total - j0);
            RFG_CUDA(cudaMemcpy2DAsync(tmp, nr * sizeof(double), X + j0, nrhs_total * sizeof(double), nr * sizeof(double),
                                       P.n, cudaMemcpyDeviceToDevice, stream_));
            solve_impl<T>(tmp, nr);
            RFG_CUDA(cudaMemcpy2DAsync(X + j0, nrhs_total * sizeof(double), tmp, nr * sizeof(double), nr * sizeof(double),
                                       P.n, cudaMemcpyDeviceToDevice, stream_));
        }
        RFG_CUDA(cudaFreeAsync(tmp, stream_));
        return;
    }
    int nrhs = (int)nrhs_total;
    if (ws_nrhs_ < nrhs) {
        if (vupd_) RFG_CUDA(cudaFree(vupd_));
        if (partial_) RFG_CUDA(cudaFree(partial_));
        RFG_CUDA(cudaMalloc(&vupd_, std::max<int64_t>(P.vu_rows * MAXR, 1) * sizeof(double)));
        RFG_CUDA(cudaMalloc(&partial_, std::max<int64_t>(P.max_panel_partials * NB * MAXR, 1) * sizeof(double)));
        ws_nrhs_ = MAXR;
    }
    RFG_CUDA(cudaMemsetAsync(vupd_, 0, std::max<int64_t>(P.vu_rows * nrhs, 1) * sizeof(double), stream_));
    for (int64_t l = 0; l < P.nlevels; l++) {
        for (int r = 0; r < 2; r++) {
            const DXadd& x = P.xadd[2 * l + r];
            if (x.nblk == 0) continue;
            k_vec_extend_add<<<(unsigned)x.nblk, 256, 0, stream_>>>(X, vupd_, dp_.fronts, dp_.xadd_child + x.off,
                                                                   dp_.xadd_pre + x.pre_off, x.nchild, dp_.emap, nrhs);
            launches++;
        }
        for (int64_t si = P.step_off[l]; si < P.step_off[l + 1]; si++) {
            const DStep& st = P.steps[si];
            k_fwd_block<T><<<(unsigned)st.nact, 256, SM_BLOCK, stream_>>>(X, panel, dp_.fronts, dp_.level_order, st.fr_off, st.s,
                                                                    nrhs);
            launches++;
            if (st.n_panel > 0) {
                k_fwd_panel<T><<<(unsigned)st.n_panel, PR, SM_FPANEL, stream_>>>(X, vupd_, panel, dp_.fronts, dp_.level_order,
                                                                          st.fr_off, st.nact, dp_.pre_panel + st.pre_off,
                                                                          st.s, nrhs);
                launches++;
            }
        }
    }
    k_divide_d<<<grid_for(P.n * nrhs), 256, 0, stream_>>>(X, d_, P.n, nrhs);
    launches++;
    for (int64_t l = P.nlevels - 1; l >= 0; l--) {
        for (int64_t si = P.step_off[l + 1] - 1; si >= P.step_off[l]; si--) {
            const DStep& st = P.steps[si];
            if (st.n_panel > 0) {
                k_bwd_partial<T><<<(unsigned)st.n_panel, 256, SM_BPART, stream_>>>(X, panel, dp_.fronts, dp_.level_order,
                                                                             st.fr_off, st.nact, dp_.pre_panel + st.pre_off,
                                                                             dp_.rows, st.s, nrhs, partial_);
                launches++;
            }
            k_bwd_block<T><<<(unsigned)st.nact, 256, SM_BLOCK, stream_>>>(X, panel, dp_.fronts, dp_.level_order, st.fr_off,
                                                                    dp_.pre_panel + st.pre_off, st.s, nrhs, partial_);
            launches++;
        }
    }
    RFG_CUDA(cudaGetLastError());
    solve_launches += launches;
}

void solve_set_attributes() {
    static bool done = false;
    if (done) return;
    RFG_CUDA(cudaFuncSetAttribute(k_fwd_block<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_BLOCK));
    RFG_CUDA(cudaFuncSetAttribute(k_bwd_block<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_BLOCK));
    RFG_CUDA(cudaFuncSetAttribute(k_fwd_panel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_FPANEL));
    RFG_CUDA(cudaFuncSetAttribute(k_bwd_partial<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_BPART));
    RFG_CUDA(cudaFuncSetAttribute(k_fwd_block<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_BLOCK));
    RFG_CUDA(cudaFuncSetAttribute(k_bwd_block<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_BLOCK));
    RFG_CUDA(cudaFuncSetAttribute(k_fwd_panel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_FPANEL));
    RFG_CUDA(cudaFuncSetAttribute(k_bwd_partial<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SM_BPART));
    done = true;
}

void Engine::solve_device(double* X, int64_t nrhs) {
    if (nrhs <= 0 || plan_.n == 0) return;
    solve_set_attributes();
    // the sweep's workspace must exist before a capture
    if (ws_nrhs_ < std::min<int64_t>(nrhs, MAXR)) {
        if (vupd_) RFG_CUDA(cudaFree(vupd_));
        if (partial_) RFG_CUDA(cudaFree(partial_));
        RFG_CUDA(cudaMalloc(&vupd_, std::max<int64_t>(plan_.vu_rows * MAXR, 1) * sizeof(double)));
        RFG_CUDA(cudaMalloc(&partial_, std::max<int64_t>(plan_.max_panel_partials * NB * MAXR, 1) * sizeof(double)));
        ws_nrhs_ = MAXR;
    }
    if (use_graphs_ && nrhs <= MAXR) {
        cudaGraphExec_t ex = nullptr;
        for (auto& g : solve_graphs_)
            if (g.X == X && g.nrhs == nrhs) ex = g.exec;
        if (!ex) {
            cudaGraph_t g;
            int64_t before = solve_launches;
            RFG_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            if (prec_ == PREC_FP64)
                solve_impl<double>(X, nrhs);
            else
                solve_impl<float>(X, nrhs);
            RFG_CUDA(cudaStreamEndCapture(stream_, &g));
            RFG_CUDA(cudaGraphInstantiate(&ex, g, 0));
            RFG_CUDA(cudaGraphDestroy(g));
            solve_graphs_.push_back({X, nrhs, ex});
            solve_graph_launches_ = solve_launches - before;
            solve_launches = before;
        }
        RFG_CUDA(cudaGraphLaunch(ex, stream_));
        solve_launches += solve_graph_launches_;
        return;
    }
    if (prec_ == PREC_FP64)
        solve_impl<double>(X, nrhs);
    else
        solve_impl<float>(X, nrhs);
}

void Engine::set_matrix(const int64_t* row_ptr, const int64_t* col, const int64_t* src_of_entry, int64_t nnz) {
    int64_t n = plan_.n;
    a_nnz_ = nnz;
    a_rowptr_ = (int64_t*)dalloc((n + 1) * sizeof(int64_t));
    a_col_ = (int64_t*)dalloc(std::max<int64_t>(nnz, 1) * sizeof(int64_t));
    a_src_ = (int64_t*)dalloc(std::max<int64_t>(nnz, 1) * sizeof(int64_t));
    a_val_ = (double*)dalloc(std::max<int64_t>(nnz, 1) * sizeof(double));
    RFG_CUDA(cudaMemcpyAsync(a_rowptr_, row_ptr, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    if (nnz > 0) {
        RFG_CUDA(cudaMemcpyAsync(a_col_, col, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        RFG_CUDA(cudaMemcpyAsync(a_src_, src_of_entry, nnz * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    }
    RFG_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::matvec(const double* X, double* Y, int64_t nrhs) {
    int64_t n = plan_.n;
    k_spmv<<<grid_for(n * 32, 256), 256, 0, stream_>>>(a_rowptr_, a_col_, a_val_, X, Y, n, (int)nrhs, nullptr);
}

SolveStats Engine::solve_refined(double* X, const double* B, int64_t nrhs, double tol, int max_iter) {
    SolveStats st;
    int64_t n = plan_.n;
    if (n == 0 || nrhs == 0) return st;
    if (nrhs > MAXR) throw CudaError("solve_refined: at most 32 right-hand sides per call");
    if (!a_val_) throw CudaError("solve_refined: the matrix was not set");
    int64_t l0 = solve_launches;
    // the matrix values of the current factorization and ‖A‖∞
    k_gather_values<<<grid_for(a_nnz_), 256, 0, stream_>>>(a_val_, src_, a_src_, a_nnz_);
    if (ref_nrhs_ < nrhs) {
        if (ref_r_) RFG_CUDA(cudaFree(ref_r_));
        if (ref_dx_) RFG_CUDA(cudaFree(ref_dx_));
        if (ref_red_) RFG_CUDA(cudaFree(ref_red_));
        RFG_CUDA(cudaMalloc(&ref_r_, n * MAXR * sizeof(double)));
        RFG_CUDA(cudaMalloc(&ref_dx_, n * MAXR * sizeof(double)));
        RFG_CUDA(cudaMalloc(&ref_red_, (5 * MAXR + 1) * sizeof(double)));
        ref_nrhs_ = MAXR;
    }
    RFG_CUDA(cudaMemsetAsync(ref_red_, 0, (5 * MAXR + 1) * sizeof(double), stream_));
    k_spmv<<<grid_for(n * 32, 256), 256, 0, stream_>>>(a_rowptr_, a_col_, a_val_, nullptr, nullptr, n, 0, ref_dx_);
    k_max_reduce<<<grid_for(n), 256, 0, stream_>>>(ref_dx_, n, ref_red_ + 5 * MAXR);
    RFG_CUDA(cudaMemcpyAsync(&anorm_, ref_red_ + 5 * MAXR, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    if (X != B) RFG_CUDA(cudaMemcpyAsync(X, B, n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    solve_device(X, nrhs);
    std::vector<double> red(5 * nrhs);
    for (int it = 0;; it++) {
        RFG_CUDA(cudaMemsetAsync(ref_red_, 0, 5 * MAXR * sizeof(double), stream_));
        k_spmv<<<grid_for(n * 32, 256), 256, 0, stream_>>>(a_rowptr_, a_col_, a_val_, X, ref_dx_, n, (int)nrhs, nullptr);
        k_residual<<<grid_for(n * nrhs), 256, 0, stream_>>>(ref_r_, ref_dx_, B, X, n, (int)nrhs, ref_red_);
        solve_launches += 2;
        RFG_CUDA(cudaMemcpyAsync(red.data(), ref_red_, 5 * nrhs * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        RFG_CUDA(cudaStreamSynchronize(stream_));
        double eta = 0.0, rr = 0.0;
        for (int j = 0; j < nrhs; j++) {
            double den = anorm_ * red[5 * j + 1] + red[5 * j + 2];
            double e = den > 0 ? red[5 * j] / den : 0.0;
            double q = red[5 * j + 4] > 0 ? std::sqrt(red[5 * j + 3] / red[5 * j + 4]) : 0.0;
            eta = std::max(eta, e);
            rr = std::max(rr, q);
        }
        st.backward_error = eta;
        st.rel_residual = rr;
        st.iterations = it;
        if (eta <= tol || it >= max_iter) break;
        solve_device(ref_r_, nrhs);
        k_axpy<<<grid_for(n * nrhs), 256, 0, stream_>>>(X, ref_r_, n * nrhs);
        solve_launches += 1;
    }
    st.launches = solve_launches - l0;
    return st;
}

}  // namespace rfg
