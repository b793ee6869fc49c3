// Triangular solves over the elimination tree, and FP64 iterative refinement.
//
// The solve follows the level schedule of the factor (plan.h) in steps of WS = 4·NB
// pivots (WStep), for nrhs right-hand sides stored as X[q·nrhs + j] (internal
// numbering):
//  forward  (leaves up)   per level, the children's update vectors are added into
//                         their parents (k_vec_extend_add: pivot rows into X, later
//                         rows into the parent's update vector V_t); then per step
//                         k_wfwd_diag solves the step's diagonal block with its four
//                         stored NB×NB inverse blocks (y_B → Y) and k_wfwd_rows
//                         subtracts L[r, J0:J1]·y_B from the rows below (X or V_t);
//  diagonal               Y /= D (k_divide_d);
//  backward (root down)   per step, last first: partial sums of Lᵀ·y over row chunks
//                         below the block, then the diagonal block backwards
//                         (k_wbwd_part_pf + k_wbwd_diag_pf for an FP32 factor and up
//                         to four right-hand sides, else k_wbwd, whose last CTA per
//                         front reduces the partials and solves the block).
// Every kernel of a sweep is launched as a programmatic dependent of the one before
// (PDL): the _pf kernels copy their factor data into shared memory before they wait for
// the vectors of the previous kernel.
// This is the multifrontal form of Factor::solve (src/sparse.rs:615-652): the same
// three sweeps, with the updates of each front gathered in its update vector instead
// of being subtracted from x row by row.

#include <cuda_runtime.h>


#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "chain.h"
#include "engine.h"
#include "par.h"
#include "tiles.cuh"

// Scratch of rfg_solve_device_noalloc: a fixed array in the library's device image,
// so that solves through that entry point allocate nothing. The driver reserves it
// when the library's kernels are loaded on a device, once per process and device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[rfg::NOALLOC_SCRATCH_BYTES];

namespace rfg {

namespace {

constexpr int MAXR = 32;  // right-hand sides per sweep
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

// children's update vectors into the parent (one launch per child rank, so that no two
// tasks of a launch add into the same entry): one warp per task of up to XR rows of one
// child; the rows' targets in the parent are staged in shared memory before the wait for
// the previous kernel, then the lanes run over (row, right-hand side) pairs
__global__ void __launch_bounds__(256) k_vec_extend_add(double* __restrict__ X, double* __restrict__ V,
                                                        const DFront* __restrict__ fr,
                                                        const int64_t* __restrict__ tasks, int64_t ntask,
                                                        const int32_t* __restrict__ emap, int nrhs) {
    pdl_launch_dependents();
    __shared__ int32_t spos[8][XR];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t tk = (int64_t)blockIdx.x * 8 + w;
    if (tk >= ntask) return;
    const int64_t c = tasks[4 * tk], p = tasks[4 * tk + 1], x0 = tasks[4 * tk + 2];
    const int nx = (int)tasks[4 * tk + 3];
    const DFront fc = fr[c], fp = fr[p];
    for (int x = lane; x < nx; x += 32) spos[w][x] = emap[fc.emap_off + x0 + x];
    __syncwarp();
    pdl_wait();
    for (int e = lane; e < nx * nrhs; e += 32) {
        const int x = e / nrhs, j = e - x * nrhs;
        const int pos = spos[w][x];
        const double v = V[(fc.vuoff + x0 + x) * nrhs + j];
        if (pos < fp.k)
            X[(fp.start + pos) * nrhs + j] += v;
        else
            V[(fp.vuoff + pos - fp.k) * nrhs + j] += v;
    }
}

// ---------------------------------------------------------------------------
// Solve steps WS = 4·NB pivots wide (WStep). Forward: k_wfwd_diag (one CTA per active
// front) solves the step's diagonal block with its four stored NB×NB inverses and the
// panel pieces between them, writes y_B to Y, and k_wfwd_rows (PR rows per CTA)
// subtracts L[r, J0:J1]·y_B from every row below the block. Backward: k_wbwd sums
// L[r, J0:J1]ᵀ·y(r) over its rows into a per-CTA partial; the last CTA of the front
// (atomic ticket) subtracts all partials from y_B and solves the diagonal block
// backwards. One wide step replaces four NB steps, so the chain of dependent launches
// at the top of the tree is four times shorter.
// ---------------------------------------------------------------------------

// rows of panel pieces the forward diagonal kernel stages for a level (multiple of NB)
inline int wfwd_piece_rows(int64_t maxk_level, int64_t S) {
    const int64_t wbmax = std::min<int64_t>(WS, std::max<int64_t>(0, maxk_level - S * WS));
    const int64_t rows = std::min<int64_t>(3 * NB, std::max<int64_t>(0, wbmax - NB));
    return (int)((rows + NB - 1) / NB * NB);
}
template <typename T>
size_t wfwd_diag_smem(int piece_rows, int nrhs) {
    return NB * (NB + 1) * sizeof(double) + ((size_t)piece_rows * (NB + 1) * sizeof(T) + 7) / 8 * 8 +
           (size_t)(WS + NB) * nrhs * sizeof(double);
}

template <typename T>
__global__ void __launch_bounds__(256) k_wfwd_diag(const double* __restrict__ X, double* __restrict__ Y,
                                                   const T* __restrict__ panel, const double* __restrict__ linv,
                                                   const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                   int64_t fr_off, int64_t S, int nrhs, int piece_rows, int cgrp) {
    pdl_launch_dependents();
    pdl_wait();
    // this CTA: right-hand sides [jc0, jc0 + rc) of front blockIdx.x
    const int jc0 = blockIdx.y * cgrp, rc = min(cgrp, nrhs - jc0);
    extern __shared__ double sm[];
    double(*Li)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    T(*Lp)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(sm + NB * (NB + 1));
    double* xB = sm + NB * (NB + 1) + ((size_t)piece_rows * (NB + 1) * sizeof(T) + 7) / 8;  // [WS][rc]
    double* yb = xB + WS * rc;                                                                // [NB][rc]
    const DFront f = fr[order[fr_off + blockIdx.x]];
    const int64_t J0 = S * WS;
    const int wb = (int)min((int64_t)WS, f.k - J0), nbw = (wb + NB - 1) / NB;
    const double* xs = X + (f.start + J0) * nrhs + jc0;
    for (int idx = threadIdx.x; idx < nbw * NB * rc; idx += blockDim.x) {
        const int q = idx / rc, j = idx - q * rc;
        xB[idx] = q < wb ? xs[(int64_t)q * nrhs + j] : 0.0;
    }
    for (int b = 0; b < nbw; b++) {
        const int jbb = min(NB, wb - b * NB);
        const int nbelow = wb - (b + 1) * NB;  // rows of the block below sub-block b
        __syncthreads();
        load_linv<256>(Li, linv + (f.blk_off + S * 4 + b) * (int64_t)(NB * NB));
        for (int c = 0; c * NB < nbelow; c++)
            load_tile<T, NB, 256>(Lp + c * NB, panel + f.poff + (J0 + (b + 1 + c) * NB) * f.ldp + J0 + b * NB, f.ldp,
                                  min(NB, nbelow - c * NB), jbb);
        __syncthreads();
        for (int idx = threadIdx.x; idx < NB * rc; idx += blockDim.x) {
            const int p = idx / rc, j = idx - p * rc;
            double a0 = 0.0, a1 = 0.0;
            int q = 0;
            for (; q + 1 <= p; q += 2) {
                a0 = fma(Li[p][q], xB[(b * NB + q) * rc + j], a0);
                a1 = fma(Li[p][q + 1], xB[(b * NB + q + 1) * rc + j], a1);
            }
            if (q <= p) a0 = fma(Li[p][q], xB[(b * NB + q) * rc + j], a0);
            yb[idx] = a0 + a1;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < jbb * rc; idx += blockDim.x) {
            const int p = idx / rc, j = idx - p * rc;
            Y[(f.start + J0 + b * NB + p) * nrhs + jc0 + j] = yb[idx];
        }
        for (int idx = threadIdx.x; idx < max(0, nbelow) * rc; idx += blockDim.x) {
            const int i = idx / rc, j = idx - i * rc;
            double a0 = 0.0, a1 = 0.0;
            for (int p = 0; p < NB; p += 2) {
                a0 = fma((double)Lp[i][p], yb[p * rc + j], a0);
                a1 = fma((double)Lp[i][p + 1], yb[(p + 1) * rc + j], a1);
            }
            xB[((b + 1) * NB + i) * rc + j] -= a0 + a1;
        }
    }
}

// rows below the wide block: X (pivot rows) or V (later rows) −= L[r, J0:J1]·y_B
template <typename T>
__global__ void __launch_bounds__(PR) k_wfwd_rows(double* __restrict__ X, double* __restrict__ V,
                                                  const double* __restrict__ Y, const T* __restrict__ panel,
                                                  const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                  int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre,
                                                  int64_t S, int nrhs) {
    pdl_launch_dependents();
    pdl_wait();
    extern __shared__ double sm[];
    double* yB = sm;  // [⌈wb/NB⌉·NB][nrhs]
    const int64_t b = blockIdx.x;
    const int64_t i = find_slot_warp(pre, nact, b);
    const int64_t chunk = b - pre[i];
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS, J1 = min(J0 + WS, f.k);
    const int wb = (int)(J1 - J0), nbw = (wb + NB - 1) / NB;
    const int64_t r0 = J1 + chunk * PR;
    const int nr = (int)max((int64_t)0, min((int64_t)PR, f.m - r0));
    if (nr == 0) return;
    const double* ys = Y + (f.start + J0) * nrhs;
    for (int idx = threadIdx.x; idx < nbw * NB * nrhs; idx += blockDim.x) yB[idx] = idx < wb * nrhs ? ys[idx] : 0.0;
    __syncthreads();
    const int rr = threadIdx.x;
    if (rr >= nr) return;
    const int64_t r = r0 + rr;
    double* tgt = r < f.k ? X + (f.start + r) * nrhs : V + (f.vuoff + r - f.k) * nrhs;
    const T* rowp = panel + f.poff + r * f.ldp + J0;
    constexpr int VEC = 16 / (int)sizeof(T);
    using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    for (int c = 0; c < nbw; c++) {
        const int jc = min(NB, wb - c * NB);
        T lv[NB];
#pragma unroll
        for (int q = 0; q < NB / VEC; q++) {
            const int p = q * VEC;
            if (p + VEC <= jc) {
                *reinterpret_cast<VT*>(&lv[p]) = __ldg(reinterpret_cast<const VT*>(rowp + c * NB + p));
            } else {
#pragma unroll
                for (int e = 0; e < VEC; e++) lv[p + e] = p + e < jc ? rowp[c * NB + p + e] : T(0);
            }
        }
        for (int j = 0; j < nrhs; j++) {
            double acc = 0.0;
#pragma unroll
            for (int p = 0; p < NB; p++) acc = fma((double)lv[p], yB[(c * NB + p) * nrhs + j], acc);
            tgt[j] -= acc;
        }
    }
}

// shared memory of k_wbwd (layout in the kernel)
template <typename T>
constexpr size_t wbwd_smem(int nrhs) {
    return ((std::max<size_t>(PR * (NB + 1) * sizeof(T), NB * (NB + 1) * 8) + 7) / 8 +
            std::max<size_t>(PR * (nrhs + 1), WS * (nrhs + 1) + NB * nrhs + 256) + 256) *
           sizeof(double);
}

template <typename T>
__global__ void __launch_bounds__(256) k_wbwd(double* __restrict__ Y, const T* __restrict__ panel,
                                              const double* __restrict__ linv, const DFront* __restrict__ fr,
                                              const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                              const int64_t* __restrict__ pre, const int64_t* __restrict__ pre_part,
                                              const int64_t* __restrict__ rows, int64_t S, int nrhs,
                                              double* __restrict__ partial, int* __restrict__ tickets) {
    pdl_launch_dependents();
    pdl_wait();
    // region 0: the panel tile (storage type T), later an inverse block or a panel piece;
    // region 1: y of the CTA's rows (row stride nrhs+1), later z_B, y_b and group sums;
    // then 256 doubles for the partial-sum reduction
    extern __shared__ double sm[];
    T(*Lt)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(sm);
    const int region0 = (int)((max(PR * (NB + 1) * (int)sizeof(T), NB * (NB + 1) * 8) + 7) / 8);
    const int xs = nrhs + 1;
    double* xr = sm + region0;
    const int region1 = max(PR * xs, WS * xs + NB * nrhs + 256);
    double* red = xr + region1;
    __shared__ int last;
    const int64_t b = blockIdx.x;
    const int64_t i = find_slot_warp(pre, nact, b);
    const int64_t chunk = b - pre[i];
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS, J1 = min(J0 + WS, f.k);
    const int wb = (int)(J1 - J0), nbw = (wb + NB - 1) / NB;
    const int64_t r0 = J1 + chunk * PR;
    const int nr = (int)max((int64_t)0, min((int64_t)PR, f.m - r0));
#pragma unroll 4
    for (int idx = threadIdx.x; idx < PR * nrhs; idx += 256) {
        int rr = idx / nrhs, j = idx - rr * nrhs;
        double v = 0.0;
        if (rr < nr) {
            int64_t r = r0 + rr;
            int64_t q = r < f.k ? f.start + r : rows[f.rows_off + r - f.k];
            v = Y[q * nrhs + j];
        }
        xr[rr * xs + j] = v;
    }
    // out[p·nrhs + j] = Σ_rr L[r][J0+p]·y(r)[j], column chunk by column chunk; with few
    // outputs, G thread groups take every G-th row, their sums added in group order
    double* out = partial + (pre_part[i] + chunk * wb) * nrhs;
    for (int c = 0; c < nbw; c++) {
        const int jc = min(NB, wb - c * NB);
        __syncthreads();
        load_tile<T, PR, 256>(Lt, panel + f.poff + r0 * f.ldp + J0 + c * NB, f.ldp, nr, jc);
        __syncthreads();
        const int nout = jc * nrhs;
        const int G = nout >= 256 ? 1 : 256 / nout;
        for (int idx = threadIdx.x; idx < nout * G; idx += 256) {
            int g = idx / nout, o = idx - g * nout;
            int p = o / nrhs, j = o - p * nrhs;
            double acc = 0.0;
            for (int rr = g; rr < nr; rr += G) acc = fma((double)Lt[rr][p], xr[rr * xs + j], acc);
            if (G == 1)
                out[c * NB * nrhs + o] = acc;
            else
                red[g * nout + o] = acc;
        }
        if (G > 1) {
            __syncthreads();
            for (int o = threadIdx.x; o < nout; o += 256) {
                double v = 0.0;
                for (int g = 0; g < G; g++) v += red[g * nout + o];
                out[c * NB * nrhs + o] = v;
            }
        }
    }
    __threadfence();
    __syncthreads();
    const int64_t c0 = pre[i], c1 = pre[i + 1];
    if (threadIdx.x == 0) last = (atomicAdd(&tickets[i], 1) == (int)(c1 - c0 - 1));
    __syncthreads();
    if (!last) return;
    __threadfence();
    // the last CTA: z_B = y_B − Σ partials (CTAs in order), then the block solved backwards
    double(*Li)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    double* z = xr;                   // [nbw·NB][xs]
    double* yb = xr + WS * xs;        // [NB][nrhs]
    double* gsum = yb + NB * nrhs;    // [G][nout] when nout < 256
    {
        const int nout = wb * nrhs;
        const int G = nout >= 256 ? 1 : 256 / nout;
        const int64_t nc = c1 - c0, per = (nc + G - 1) / G;
        const double* pbase = partial + pre_part[i] * nrhs;
        for (int idx = threadIdx.x; idx < nout * G; idx += 256) {
            int g = idx / nout, o = idx - g * nout;
            int64_t ca = g * per, cb = min(nc, ca + per);
            double v = 0.0;
#pragma unroll 4
            for (int64_t c = ca; c < cb; c++) v += __ldcg(&pbase[c * nout + o]);
            if (G == 1) {
                int p = o / nrhs, j = o - p * nrhs;
                z[p * xs + j] = Y[(f.start + J0 + p) * nrhs + j] - v;
            } else {
                gsum[g * nout + o] = v;
            }
        }
        if (G > 1) {
            __syncthreads();
            for (int o = threadIdx.x; o < nout; o += 256) {
                double v = 0.0;
                for (int g = 0; g < G; g++) v += gsum[g * nout + o];
                int p = o / nrhs, j = o - p * nrhs;
                z[p * xs + j] = Y[(f.start + J0 + p) * nrhs + j] - v;
            }
        }
        for (int idx = threadIdx.x; idx < (nbw * NB - wb) * nrhs; idx += 256) {
            int p = wb + idx / nrhs, j = idx % nrhs;
            z[p * xs + j] = 0.0;
        }
    }
    for (int bb = nbw - 1; bb >= 0; bb--) {
        const int jbb = min(NB, wb - bb * NB);
        __syncthreads();
        load_linv<256>(Li, linv + (f.blk_off + S * 4 + bb) * (int64_t)(NB * NB));
        __syncthreads();
        // y_b = L_bb⁻ᵀ·z_b
        for (int idx = threadIdx.x; idx < NB * nrhs; idx += 256) {
            const int p = idx / nrhs, j = idx - p * nrhs;
            double acc = 0.0;
            for (int q = p; q < NB; q++) acc = fma(Li[q][p], z[(bb * NB + q) * xs + j], acc);
            yb[idx] = acc;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < jbb * nrhs; idx += 256) Y[(f.start + J0 + bb * NB) * nrhs + idx] = yb[idx];
        // the earlier sub-blocks: z_b2 −= L[rows of bb, columns of b2]ᵀ·y_b
        for (int b2 = 0; b2 < bb; b2++) {
            __syncthreads();
            load_tile<T, NB, 256>(Lt, panel + f.poff + (J0 + bb * NB) * f.ldp + J0 + b2 * NB, f.ldp, jbb, NB);
            __syncthreads();
            for (int idx = threadIdx.x; idx < NB * nrhs; idx += 256) {
                const int c = idx / nrhs, j = idx - c * nrhs;
                double acc = 0.0;
                for (int q = 0; q < jbb; q++) acc = fma((double)Lt[q][c], yb[q * nrhs + j], acc);
                z[(b2 * NB + c) * xs + j] -= acc;
            }
        }
    }
    if (threadIdx.x == 0) tickets[i] = 0;
}

// ---------------------------------------------------------------------------
// Prefetching step kernels for an FP32 factor and at most PF_MAXR right-hand sides.
// Every kernel of a sweep is launched as a programmatic dependent of the one before it:
// it starts while its predecessor runs, copies the factor data it needs (unchanged
// during a solve) into shared memory with cp.async, and only then waits for the
// predecessor's results. At the top of the tree, where a wide step is a chain of small
// launches, a step then costs its arithmetic instead of one global-memory round trip per
// stage plus a launch gap per kernel. The backward step is split in two: k_wbwd_part
// (partial sums of Lᵀ·y over row chunks) and k_wbwd_diag (one CTA per front: the sum of
// the partials in chunk order, then the diagonal block backwards). Shared memory is
// sized per step from the widest front of the step, so the many small fronts of the
// lower levels keep several CTAs per SM.
// ---------------------------------------------------------------------------
constexpr int PF_MAXR = 4;

// row tile of the rows / partial kernels: PF_RPC rows (half of a PR-row chunk of the plan)
// × cols floats (cols = the step's widest block rounded up to 32), row pitch cols + 4
// (16-byte rows, conflict-free row reads); three such CTAs fit on an SM
constexpr int PF_RPC = PR / 2;
inline int pf_cols(int64_t wb_max) { return (int)((wb_max + 31) / 32 * 32); }
inline size_t pf_rows_smem(int cols, int nrhs) {
    return (size_t)PF_RPC * (cols + 4) * sizeof(float) + (size_t)WS * nrhs * sizeof(double);
}
inline size_t pf_part_smem(int cols, int nrhs) {
    return (size_t)PF_RPC * (cols + 4) * sizeof(float) + (size_t)PF_RPC * nrhs * sizeof(double) +
           (size_t)256 * nrhs * sizeof(double);
}
// diagonal kernels: min(nbw, 3) inverse blocks, nbw(nbw−1)/2 panel pieces (NB×NB), the
// block's vectors; nbw = the step's largest number of NB sub-blocks
__host__ __device__ inline int pf_nli(int nbw) { return nbw < 3 ? nbw : 3; }
__host__ __device__ inline int pf_npc(int nbw) { return nbw * (nbw - 1) / 2; }
inline size_t pf_diag_smem(int nbw, int nrhs) {
    return (size_t)pf_nli(nbw) * NB * NB * sizeof(double) + (size_t)pf_npc(nbw) * NB * NB * sizeof(float) +
           (size_t)(WS + NB + 4 * NB) * nrhs * sizeof(double);
}

// Sums of eight rows across a warp: v[i] holds lane's partial of row i; on return every
// lane holds the total of row (lane >> 2) & 7 (three exchange steps that halve the rows
// held, then two plain steps).
template <int R>
__device__ __forceinline__ void warp_sum8(const double (&v)[8][R], double (&out)[R]) {
    const int lane = threadIdx.x & 31;
    const bool b4 = lane & 16, b3 = lane & 8, b2 = lane & 4;
    double w4[4][R], w2[2][R];
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
        for (int r = 0; r < R; r++) {
            const double send = b4 ? v[j][r] : v[j + 4][r], keep = b4 ? v[j + 4][r] : v[j][r];
            w4[j][r] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
        }
#pragma unroll
    for (int j = 0; j < 2; j++)
#pragma unroll
        for (int r = 0; r < R; r++) {
            const double send = b3 ? w4[j][r] : w4[j + 2][r], keep = b3 ? w4[j + 2][r] : w4[j][r];
            w2[j][r] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
        }
#pragma unroll
    for (int r = 0; r < R; r++) {
        const double send = b2 ? w2[0][r] : w2[1][r], keep = b2 ? w2[1][r] : w2[0][r];
        double o = keep + __shfl_xor_sync(0xffffffffu, send, 4);
        o += __shfl_xor_sync(0xffffffffu, o, 2);
        out[r] = o + __shfl_xor_sync(0xffffffffu, o, 1);
    }
}

// Forward diagonal block of a wide step: one CTA (256 threads) per active front. Pieces
// in column-block order ((1,0) (2,0) (3,0) (2,1) (3,1) (3,2) for four sub-blocks); with
// four sub-blocks the inverse block of sub-block 3 is copied into the space of column
// block 0 once stage 0 is done.
template <int R>
__global__ void __launch_bounds__(256) k_wfwd_diag_pf(const double* __restrict__ X, double* __restrict__ Y,
                                                      const float* __restrict__ panel, const double* __restrict__ linv,
                                                      const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                      int64_t fr_off, int64_t S, int nbw_max) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    double* Li = sm;                                                     // [nli][NB][NB]
    float* Pc = reinterpret_cast<float*>(sm + pf_nli(nbw_max) * NB * NB);  // [npc][NB][NB]
    double* xB = sm + pf_nli(nbw_max) * NB * NB + pf_npc(nbw_max) * NB * NB / 2;  // [WS][R]
    double* yb = xB + WS * R;                                                  // [NB][R]
    const DFront f = fr[order[fr_off + blockIdx.x]];
    const int64_t J0 = S * WS;
    const int wb = (int)min((int64_t)WS, f.k - J0), nbw = (wb + NB - 1) / NB;
    const double* lsrc = linv + (f.blk_off + S * 4) * (int64_t)(NB * NB);
    cp_async_flat(Li, lsrc, min(nbw, 3) * NB * NB / 2, 256);
    for (int b = 0; b + 1 < nbw; b++)
        for (int b2 = b + 1; b2 < nbw; b2++) {
            const int pi = b * (nbw - 1) - b * (b - 1) / 2 + (b2 - b - 1);
            cp_async_tile<float>(Pc + pi * NB * NB, NB, panel + f.poff + (J0 + b2 * NB) * f.ldp + J0 + b * NB, f.ldp,
                                 min(NB, wb - b2 * NB), NB, NB, NB, 256);
        }
    cp_async_commit();
    pdl_wait();
    const double* xs = X + (f.start + J0) * R;
    for (int idx = threadIdx.x; idx < nbw * NB * R; idx += 256) xB[idx] = idx < wb * R ? xs[idx] : 0.0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, sel = (lane >> 2) & 7;
    for (int b = 0; b < nbw; b++) {
        const int jbb = min(NB, wb - b * NB);
        if (b == 0 || b == 3) cp_async_wait<0>();
        __syncthreads();
        // y_b = L_bb⁻¹·x_b: warp w takes rows 8w..8w+7, lanes the columns q and q+32
        {
            const double* L = b < 3 ? Li + b * NB * NB : reinterpret_cast<const double*>(Pc);
            double x0[R], x1[R], v[8][R], out[R];
#pragma unroll
            for (int j = 0; j < R; j++) {
                x0[j] = xB[(b * NB + lane) * R + j];
                x1[j] = xB[(b * NB + lane + 32) * R + j];
            }
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const double l0 = L[(8 * warp + i) * NB + lane], l1 = L[(8 * warp + i) * NB + lane + 32];
#pragma unroll
                for (int j = 0; j < R; j++) v[i][j] = fma(l0, x0[j], l1 * x1[j]);
            }
            warp_sum8<R>(v, out);
            if ((lane & 3) == 0) {
                const int p = 8 * warp + sel;
#pragma unroll
                for (int j = 0; j < R; j++) {
                    yb[p * R + j] = out[j];
                    if (p < jbb) Y[(f.start + J0 + b * NB + p) * R + j] = out[j];
                }
            }
        }
        __syncthreads();
        if (b + 1 < nbw) {
            // x_b2 −= L[b2, b]·y_b for the sub-blocks below, eight rows per warp at a time
            double y0[R], y1[R];
#pragma unroll
            for (int j = 0; j < R; j++) {
                y0[j] = yb[lane * R + j];
                y1[j] = yb[(lane + 32) * R + j];
            }
            const int first = b * (nbw - 1) - b * (b - 1) / 2;  // column block b's first piece
            const int ngrp = (nbw - 1 - b) * NB / 8;
            for (int g = warp; g < ngrp; g += 8) {
                double v[8][R], out[R];
#pragma unroll
                for (int i = 0; i < 8; i++) {
                    const float* row = Pc + (first * NB + 8 * g + i) * NB;
                    const double l0 = row[lane], l1 = row[lane + 32];
#pragma unroll
                    for (int j = 0; j < R; j++) v[i][j] = fma(l0, y0[j], l1 * y1[j]);
                }
                warp_sum8<R>(v, out);
                if ((lane & 3) == 0) {
#pragma unroll
                    for (int j = 0; j < R; j++) xB[((b + 1) * NB + 8 * g + sel) * R + j] -= out[j];
                }
            }
            if (b == 0 && nbw == 4) {
                __syncthreads();  // column block 0's pieces are read: the last inverse block goes there
                cp_async_flat(Pc, lsrc + 3 * NB * NB, NB * NB / 2, 256);
                cp_async_commit();
            }
        }
    }
}

// Rows below a wide block: X (pivot rows) or V (later rows) −= L[r, J0:J1]·y_B. Two CTAs
// per PR-row chunk (PF_RPC rows each), two threads per row (half of the columns each),
// the row tile prefetched before the wait for y_B.
template <int R>
__global__ void __launch_bounds__(PR) k_wfwd_rows_pf(double* __restrict__ X, double* __restrict__ V,
                                                     const double* __restrict__ Y, const float* __restrict__ panel,
                                                     const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                     int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre,
                                                     int64_t S, int cols) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    const int pitch = cols + 4;
    float* Lt = reinterpret_cast<float*>(sm);  // [PF_RPC][pitch]
    double* yB = sm + PF_RPC * pitch / 2;      // [WS][R]
    const int64_t b = blockIdx.x >> 1;
    const int64_t i = find_slot_warp(pre, nact, b);
    const int64_t chunk = b - pre[i];
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS, J1 = min(J0 + WS, f.k);
    const int wb = (int)(J1 - J0);
    const int64_t r0 = J1 + chunk * PR + (blockIdx.x & 1) * PF_RPC;
    const int nr = (int)max((int64_t)0, min((int64_t)PF_RPC, f.m - r0));
    if (nr > 0) cp_async_tile<float>(Lt, pitch, panel + f.poff + r0 * f.ldp + J0, f.ldp, nr, wb, nr, cols, PR);
    cp_async_commit();
    pdl_wait();
    if (nr == 0) return;
    const double* ys = Y + (f.start + J0) * R;
    for (int idx = threadIdx.x; idx < cols * R; idx += PR) yB[idx] = idx < wb * R ? ys[idx] : 0.0;
    cp_async_wait<0>();
    __syncthreads();
    const int rr = threadIdx.x >> 1, h = threadIdx.x & 1;
    double acc[R][2];
#pragma unroll
    for (int j = 0; j < R; j++) acc[j][0] = acc[j][1] = 0.0;
    const int q0 = h * (cols / 8), q1 = q0 + cols / 8;
    const float4* row = reinterpret_cast<const float4*>(Lt + rr * pitch);
#pragma unroll 4
    for (int q = q0; q < q1; q++) {
        const float4 l = row[q];
#pragma unroll
        for (int j = 0; j < R; j++) {
            acc[j][0] = fma((double)l.x, yB[(4 * q) * R + j], acc[j][0]);
            acc[j][1] = fma((double)l.y, yB[(4 * q + 1) * R + j], acc[j][1]);
            acc[j][0] = fma((double)l.z, yB[(4 * q + 2) * R + j], acc[j][0]);
            acc[j][1] = fma((double)l.w, yB[(4 * q + 3) * R + j], acc[j][1]);
        }
    }
    double v[R];
#pragma unroll
    for (int j = 0; j < R; j++) {
        v[j] = acc[j][0] + acc[j][1];
        v[j] += __shfl_xor_sync(0xffffffffu, v[j], 1);
    }
    if (h == 0 && rr < nr) {
        const int64_t r = r0 + rr;
        double* tgt = r < f.k ? X + (f.start + r) * R : V + (f.vuoff + r - f.k) * R;
#pragma unroll
        for (int j = 0; j < R; j++) tgt[j] -= v[j];
    }
}

// Backward partial sums: out[p][j] = Σ_rr L[r0+rr][J0+p]·y(r0+rr)[j] over the CTA's PF_RPC
// rows (two CTAs per PR-row chunk, each with its own block of partials); G = 256/cols
// thread groups take every G-th row, their sums added in group order.
template <int R>
__global__ void __launch_bounds__(256) k_wbwd_part_pf(const double* __restrict__ Y, const float* __restrict__ panel,
                                                      const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                      int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre,
                                                      const int64_t* __restrict__ pre_part,
                                                      const int64_t* __restrict__ rows, int64_t S,
                                                      double* __restrict__ partial, int cols) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    const int pitch = cols + 4;
    float* Lt = reinterpret_cast<float*>(sm);  // [PF_RPC][pitch]
    double* yr = sm + PF_RPC * pitch / 2;      // [PF_RPC][R]
    double* red = yr + PF_RPC * R;             // [256][R]
    const int64_t b = blockIdx.x >> 1;
    const int64_t i = find_slot_warp(pre, nact, b);
    const int64_t chunk = b - pre[i];
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS, J1 = min(J0 + WS, f.k);
    const int wb = (int)(J1 - J0);
    const int64_t r0 = J1 + chunk * PR + (blockIdx.x & 1) * PF_RPC;
    const int nr = (int)max((int64_t)0, min((int64_t)PF_RPC, f.m - r0));
    if (nr > 0) cp_async_tile<float>(Lt, pitch, panel + f.poff + r0 * f.ldp + J0, f.ldp, nr, wb, nr, cols, 256);
    cp_async_commit();
    pdl_wait();
    for (int idx = threadIdx.x; idx < PF_RPC * R; idx += 256) {
        const int rr = idx / R, j = idx - rr * R;
        double v = 0.0;
        if (rr < nr) {
            const int64_t r = r0 + rr;
            const int64_t q = r < f.k ? f.start + r : rows[f.rows_off + r - f.k];
            v = Y[q * R + j];
        }
        yr[idx] = v;
    }
    cp_async_wait<0>();
    __syncthreads();
    const int G = 256 / cols, g = threadIdx.x / cols, p = threadIdx.x - g * cols;
    if (g < G) {
        double acc[R][2];
#pragma unroll
        for (int j = 0; j < R; j++) acc[j][0] = acc[j][1] = 0.0;
        int rr = g;
        for (; rr + G < nr; rr += 2 * G) {
            const double l0 = Lt[rr * pitch + p], l1 = Lt[(rr + G) * pitch + p];
#pragma unroll
            for (int j = 0; j < R; j++) {
                acc[j][0] = fma(l0, yr[rr * R + j], acc[j][0]);
                acc[j][1] = fma(l1, yr[(rr + G) * R + j], acc[j][1]);
            }
        }
        if (rr < nr) {
            const double l0 = Lt[rr * pitch + p];
#pragma unroll
            for (int j = 0; j < R; j++) acc[j][0] = fma(l0, yr[rr * R + j], acc[j][0]);
        }
        if (G == 1) {
            if (p < wb) {
                double* out = partial + (2 * (pre_part[i] + chunk * wb) + (blockIdx.x & 1) * wb + p) * R;
#pragma unroll
                for (int j = 0; j < R; j++) out[j] = acc[j][0] + acc[j][1];
            }
            return;
        }
#pragma unroll
        for (int j = 0; j < R; j++) red[(g * cols + p) * R + j] = acc[j][0] + acc[j][1];
    }
    if (G == 1) return;
    __syncthreads();
    double* out = partial + (2 * (pre_part[i] + chunk * wb) + (blockIdx.x & 1) * wb) * R;
    for (int o = threadIdx.x; o < wb * R; o += 256) {
        double v = 0.0;
        for (int gg = 0; gg < G; gg++) v += red[gg * cols * R + o];
        out[o] = v;
    }
}

// Backward diagonal block: one CTA (256 threads) per active front. z_B = y_B − Σ partials
// (chunks in order), then for sub-blocks bb from the last: y_bb = L_bb⁻ᵀ·z_bb and
// z_b2 −= L[bb, b2]ᵀ·y_bb for b2 < bb. Pieces in row-block order (1,0) (2,0) (2,1) (3,0)
// (3,1) (3,2); with four sub-blocks inverse blocks 1..3 are prefetched and block 0 is
// copied into the space of row block 3 once stage 3 is done.
template <int R>
__global__ void __launch_bounds__(256) k_wbwd_diag_pf(double* __restrict__ Y, const float* __restrict__ panel,
                                                      const double* __restrict__ linv, const DFront* __restrict__ fr,
                                                      const int64_t* __restrict__ order, int64_t fr_off,
                                                      const int64_t* __restrict__ pre,
                                                      const int64_t* __restrict__ pre_part, int64_t S,
                                                      const double* __restrict__ partial, int nbw_max) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    double* Li = sm;                                                       // [nli][NB][NB]
    float* Pr = reinterpret_cast<float*>(sm + pf_nli(nbw_max) * NB * NB);  // [npc][NB][NB]
    double* z = sm + pf_nli(nbw_max) * NB * NB + pf_npc(nbw_max) * NB * NB / 2;  // [WS][R]
    double* yb = z + WS * R;                                                     // [NB][R]
    double* red = yb + NB * R;                                                   // [4][NB][R]
    const int64_t i = blockIdx.x;
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS;
    const int wb = (int)min((int64_t)WS, f.k - J0), nbw = (wb + NB - 1) / NB;
    const double* lsrc = linv + (f.blk_off + S * 4) * (int64_t)(NB * NB);
    // inverse block bb in slot bb − shift: with four sub-blocks, blocks 1..3 in slots 0..2
    // and block 0 later in the pieces of row block 3
    const int shift = nbw == 4 ? 1 : 0;
    cp_async_flat(Li, lsrc + shift * NB * NB, (nbw - shift) * NB * NB / 2, 256);
    for (int bb = 1; bb < nbw; bb++)
        for (int b2 = 0; b2 < bb; b2++) {
            const int pi = bb * (bb - 1) / 2 + b2;
            cp_async_tile<float>(Pr + pi * NB * NB, NB, panel + f.poff + (J0 + bb * NB) * f.ldp + J0 + b2 * NB, f.ldp,
                                 min(NB, wb - bb * NB), NB, NB, NB, 256);
        }
    cp_async_commit();
    pdl_wait();
    {
        const int nout = wb * R;
        const int64_t nc = 2 * (pre[i + 1] - pre[i]);  // two partial blocks per chunk
        const double* pbase = partial + 2 * pre_part[i] * R;
        for (int o = threadIdx.x; o < nbw * NB * R; o += 256) {
            double v = 0.0;
            if (o < nout) {
                // blocks added in order; loaded 32 at a time so the loads overlap (the
                // top-of-tree steps have up to two hundred blocks)
                int64_t c = 0;
                for (; c + 32 <= nc; c += 32) {
                    double t[32];
#pragma unroll
                    for (int u = 0; u < 32; u++) t[u] = __ldcg(&pbase[(c + u) * nout + o]);
#pragma unroll
                    for (int u = 0; u < 32; u++) v += t[u];
                }
                for (; c + 8 <= nc; c += 8) {
                    double t[8];
#pragma unroll
                    for (int u = 0; u < 8; u++) t[u] = __ldcg(&pbase[(c + u) * nout + o]);
#pragma unroll
                    for (int u = 0; u < 8; u++) v += t[u];
                }
                for (; c < nc; c++) v += __ldcg(&pbase[c * nout + o]);
                v = Y[(f.start + J0) * R + o] - v;
            }
            z[o] = v;
        }
    }
    cp_async_wait<0>();
    for (int bb = nbw - 1; bb >= 0; bb--) {
        const int jbb = min(NB, wb - bb * NB);
        if (bb == 0 && nbw == 4) cp_async_wait<0>();
        __syncthreads();
        // y_bb = L_bb⁻ᵀ·z_bb: thread (p, g) sums rows q ∈ [16g, 16g+16) of column p
        const double* L = (nbw == 4 && bb == 0) ? reinterpret_cast<const double*>(Pr + 3 * NB * NB)
                                                : Li + (bb - shift) * NB * NB;
        {
            const int p = threadIdx.x & 63, g = threadIdx.x >> 6;
            double acc[R][2];
#pragma unroll
            for (int j = 0; j < R; j++) acc[j][0] = acc[j][1] = 0.0;
#pragma unroll
            for (int q = 16 * g; q < 16 * g + 16; q += 2) {
                const double l0 = L[q * NB + p], l1 = L[(q + 1) * NB + p];
#pragma unroll
                for (int j = 0; j < R; j++) {
                    acc[j][0] = fma(l0, z[(bb * NB + q) * R + j], acc[j][0]);
                    acc[j][1] = fma(l1, z[(bb * NB + q + 1) * R + j], acc[j][1]);
                }
            }
#pragma unroll
            for (int j = 0; j < R; j++) red[(g * NB + p) * R + j] = acc[j][0] + acc[j][1];
        }
        __syncthreads();
        for (int o = threadIdx.x; o < NB * R; o += 256) {
            const double v = red[o] + red[NB * R + o] + red[2 * NB * R + o] + red[3 * NB * R + o];
            yb[o] = v;
            if (o < jbb * R) Y[(f.start + J0 + bb * NB) * R + o] = v;
        }
        if (bb == 0) break;
        __syncthreads();
        // z_b2 −= L[bb, b2]ᵀ·y_bb, one thread per column of row block bb
        if (threadIdx.x < bb * NB) {
            const int b2 = threadIdx.x >> 6, c = threadIdx.x & 63;
            const float* T = Pr + (bb * (bb - 1) / 2 + b2) * NB * NB;
            double acc[R][4];
#pragma unroll
            for (int j = 0; j < R; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0;
#pragma unroll 4
            for (int q = 0; q < NB; q += 4) {
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const double l = T[(q + u) * NB + c];
#pragma unroll
                    for (int j = 0; j < R; j++) acc[j][u] = fma(l, yb[(q + u) * R + j], acc[j][u]);
                }
            }
#pragma unroll
            for (int j = 0; j < R; j++) z[(b2 * NB + c) * R + j] -= (acc[j][0] + acc[j][1]) + (acc[j][2] + acc[j][3]);
        }
        if (bb == 3) {
            __syncthreads();  // row block 3's pieces are read: inverse block 0 goes there
            cp_async_flat(Pr + 3 * NB * NB, lsrc, NB * NB / 2, 256);
            cp_async_commit();
        }
    }
}

// ---------------------------------------------------------------------------
// Step kernels for 5 to 32 right-hand sides (a block of load cases, the subspace
// iteration of an eigen solver): the rows below a wide block and the partial sums of the
// backward step are small GEMMs (PF_RPC rows × up to WS columns × nrhs), register-tiled
// with eight right-hand sides per thread so that every factor entry is converted to FP64
// and read from shared memory once per eight products; the row tile is prefetched
// before the wait for the vectors (PDL). The partial sums of a backward step are added
// (chunks in order) into y_B by k_wred, then k_wbwd_diag_mr solves the diagonal block.
// ---------------------------------------------------------------------------
// rows kernel: the row tile transposed (k-major, PF_RPC + 4 elements per k) in region 0,
// which later holds the four k-groups' partial sums; then Y_B ([cols][MAXR] doubles)
__host__ __device__ inline size_t mr_rows_region0(int cols, size_t elt) {
    const size_t tile = (size_t)cols * (PF_RPC + 4) * elt, sums = (size_t)4 * PF_RPC * MAXR * sizeof(double);
    return tile > sums ? tile : sums;
}
inline size_t mr_rows_smem(int cols, size_t elt) {
    return mr_rows_region0(cols, elt) + (size_t)cols * MAXR * sizeof(double);
}

// Rows below a wide block: X (pivot rows) or V (later rows) −= L[r, J0:J1]·Y_B for PF_RPC
// rows per CTA. The row tile is read into registers before the wait for Y_B and stored
// k-major; thread (k-group of cols/4 columns, 4 rows, 8 right-hand sides) accumulates 32
// products per k from one 4-row load and one 8-vector load; the four k-groups' sums are
// added in order through shared memory.
template <typename T>
__global__ void __launch_bounds__(256) k_wfwd_rows_mr(double* __restrict__ X, double* __restrict__ V,
                                                      const double* __restrict__ Y, const T* __restrict__ panel,
                                                      const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                      int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre,
                                                      int64_t S, int nrhs, int cols) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    constexpr int VEC = 16 / (int)sizeof(T);                 // elements per 16-byte load
    constexpr int LP = PF_RPC + 4;                           // k-major pitch
    constexpr int NPRE = PF_RPC * WS * 4 / 16 / 256;  // 16-byte loads held per thread (an FP32 tile; half an FP64 one)
    using VT = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    T* LT = reinterpret_cast<T*>(sm);                                           // [cols][LP]
    double* red = sm;                                                           // [4][PF_RPC][MAXR] (after use)
    double* yB = sm + mr_rows_region0(cols, sizeof(T)) / sizeof(double);        // [cols][MAXR]
    const int64_t b = blockIdx.x >> 1;
    const int64_t i = find_slot_warp(pre, nact, b);
    const int64_t chunk = b - pre[i];
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS, J1 = min(J0 + WS, f.k);
    const int wb = (int)(J1 - J0);
    const int64_t r0 = J1 + chunk * PR + (blockIdx.x & 1) * PF_RPC;
    const int nr = (int)max((int64_t)0, min((int64_t)PF_RPC, f.m - r0));
    // 16-byte pieces (row rr = idx % PF_RPC, columns VEC·(idx / PF_RPC) ..): a warp reads
    // one column piece of 32 rows and stores it k-major without bank conflicts
    const int npiece = PF_RPC * (cols / VEC);
    const T* src = panel + f.poff + r0 * f.ldp + J0;
    VT pre_v[NPRE];
#pragma unroll
    for (int u = 0; u < NPRE; u++) {
        const int idx = threadIdx.x + 256 * u;
        const int rr = idx % PF_RPC, c = (idx / PF_RPC) * VEC;
        VT v;
        T* ve = reinterpret_cast<T*>(&v);
#pragma unroll
        for (int e = 0; e < VEC; e++) ve[e] = T(0);
        if (idx < npiece && rr < nr) {
            if (c + VEC <= wb)
                v = __ldg(reinterpret_cast<const VT*>(src + (int64_t)rr * f.ldp + c));
            else
#pragma unroll
                for (int e = 0; e < VEC; e++) ve[e] = c + e < wb ? src[(int64_t)rr * f.ldp + c + e] : T(0);
        }
        pre_v[u] = v;
    }
    pdl_wait();
    if (nr == 0) return;
#pragma unroll
    for (int u = 0; u < NPRE; u++) {
        const int idx = threadIdx.x + 256 * u;
        if (idx < npiece) {
            const int rr = idx % PF_RPC, c = (idx / PF_RPC) * VEC;
            const T* ve = reinterpret_cast<const T*>(&pre_v[u]);
#pragma unroll
            for (int e = 0; e < VEC; e++) LT[(c + e) * LP + rr] = ve[e];
        }
    }
    // pieces beyond the registers (FP64 tiles wider than 128 columns)
    for (int idx = threadIdx.x + 256 * NPRE; idx < npiece; idx += 256) {
        const int rr = idx % PF_RPC, c = (idx / PF_RPC) * VEC;
#pragma unroll
        for (int e = 0; e < VEC; e++)
            LT[(c + e) * LP + rr] = (rr < nr && c + e < wb) ? src[(int64_t)rr * f.ldp + c + e] : T(0);
    }
    const double* ys = Y + (f.start + J0) * nrhs;
    for (int idx = threadIdx.x; idx < cols * MAXR; idx += 256) {
        const int p = idx / MAXR, j = idx - p * MAXR;
        yB[idx] = (p < wb && j < nrhs) ? ys[p * nrhs + j] : 0.0;
    }
    __syncthreads();
    const int kg = threadIdx.x >> 6, q = threadIdx.x & 63, rg = q >> 2, g = q & 3;
    const int kq = cols / 4, k0 = kg * kq;
    double acc[4][8];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int u = 0; u < 8; u++) acc[a][u] = 0.0;
    if (8 * g < nrhs) {
#pragma unroll 2
        for (int k = k0; k < k0 + kq; k++) {
            double l[4];
            if constexpr (sizeof(T) == 4) {
                const float4 lv = *reinterpret_cast<const float4*>(LT + k * LP + 4 * rg);
                l[0] = lv.x; l[1] = lv.y; l[2] = lv.z; l[3] = lv.w;
            } else {
                const double2 l01 = *reinterpret_cast<const double2*>(LT + k * LP + 4 * rg);
                const double2 l23 = *reinterpret_cast<const double2*>(LT + k * LP + 4 * rg + 2);
                l[0] = l01.x; l[1] = l01.y; l[2] = l23.x; l[3] = l23.y;
            }
            const double2* y2 = reinterpret_cast<const double2*>(yB + k * MAXR + 8 * g);
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const double2 y = y2[u];
#pragma unroll
                for (int a = 0; a < 4; a++) {
                    acc[a][2 * u] = fma(l[a], y.x, acc[a][2 * u]);
                    acc[a][2 * u + 1] = fma(l[a], y.y, acc[a][2 * u + 1]);
                }
            }
        }
    }
    __syncthreads();  // the tile is read: region 0 takes the k-groups' sums
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int u = 0; u < 8; u++) red[(kg * PF_RPC + 4 * rg + a) * MAXR + 8 * g + u] = acc[a][u];
    __syncthreads();
    for (int o = threadIdx.x; o < PF_RPC * MAXR; o += 256) {
        const int rr = o / MAXR, j = o - rr * MAXR;
        if (rr >= nr || j >= nrhs) continue;
        const double v = ((red[o] + red[PF_RPC * MAXR + o]) + red[2 * PF_RPC * MAXR + o]) + red[3 * PF_RPC * MAXR + o];
        const int64_t r = r0 + rr;
        double* tgt = r < f.k ? X + (f.start + r) * nrhs : V + (f.vuoff + r - f.k) * nrhs;
        tgt[j] -= v;
    }
}

// Backward partial sums for 5 to 32 right-hand sides: out[p][j] = Σ_rr L[r0+rr][J0+p]·
// y(r0+rr)[j] over the CTA's PF_RPC rows; thread (four columns, eight right-hand sides).
template <typename T>
__global__ void __launch_bounds__(256) k_wbwd_part_mr(const double* __restrict__ Y, const T* __restrict__ panel,
                                                      const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                      int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre,
                                                      const int64_t* __restrict__ pre_part,
                                                      const int64_t* __restrict__ rows, int64_t S, int nrhs,
                                                      double* __restrict__ partial, int cols) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    constexpr int VEC = 16 / (int)sizeof(T);
    const int pitch = cols + VEC;
    T* Lt = reinterpret_cast<T*>(sm);                                      // [PF_RPC][pitch]
    double* yr = sm + ((size_t)PF_RPC * pitch * sizeof(T) + 15) / 16 * 2;  // [PF_RPC][MAXR]
    const int64_t b = blockIdx.x >> 1;
    const int64_t i = find_slot_warp(pre, nact, b);
    const int64_t chunk = b - pre[i];
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS, J1 = min(J0 + WS, f.k);
    const int wb = (int)(J1 - J0);
    const int64_t r0 = J1 + chunk * PR + (blockIdx.x & 1) * PF_RPC;
    const int nr = (int)max((int64_t)0, min((int64_t)PF_RPC, f.m - r0));
    // rows beyond nr are zero-filled (they are summed below); with no rows the source is
    // the front's first row, from which nothing is read
    cp_async_tile<T>(Lt, pitch, panel + f.poff + (nr > 0 ? r0 * f.ldp + J0 : 0), f.ldp, nr, wb, PF_RPC, cols, 256);
    cp_async_commit();
    pdl_wait();
    for (int idx = threadIdx.x; idx < PF_RPC * MAXR; idx += 256) {
        const int q = idx / MAXR, j = idx - q * MAXR;
        double v = 0.0;
        if (q < nr && j < nrhs) {
            const int64_t r = r0 + q;
            const int64_t e = r < f.k ? f.start + r : rows[f.rows_off + r - f.k];
            v = Y[e * nrhs + j];
        }
        yr[idx] = v;
    }
    cp_async_wait<0>();
    __syncthreads();
    const int pg = threadIdx.x >> 2, g = threadIdx.x & 3;  // columns 4pg .. 4pg+3, right-hand sides 8g ..
    if (4 * pg >= cols || 8 * g >= nrhs) return;
    double acc[4][8];
#pragma unroll
    for (int c = 0; c < 4; c++)
#pragma unroll
        for (int u = 0; u < 8; u++) acc[c][u] = 0.0;
#pragma unroll 2
    for (int q = 0; q < PF_RPC; q++) {
        double l[4];
#pragma unroll
        for (int c = 0; c < 4; c++) l[c] = (double)Lt[q * pitch + 4 * pg + c];
        const double2* y2 = reinterpret_cast<const double2*>(yr + q * MAXR + 8 * g);
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const double2 y = y2[u];
#pragma unroll
            for (int c = 0; c < 4; c++) {
                acc[c][2 * u] = fma(l[c], y.x, acc[c][2 * u]);
                acc[c][2 * u + 1] = fma(l[c], y.y, acc[c][2 * u + 1]);
            }
        }
    }
    double* out = partial + (2 * (pre_part[i] + chunk * wb) + (blockIdx.x & 1) * wb) * nrhs;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int p = 4 * pg + c;
        if (p >= wb) break;
#pragma unroll
        for (int u = 0; u < 8; u++)
            if (8 * g + u < nrhs) out[p * nrhs + 8 * g + u] = acc[c][u];
    }
}

// y_B −= Σ partial blocks (two per row chunk, in order): grid (front, slice of 256 outputs).
__global__ void __launch_bounds__(256) k_wred(double* __restrict__ Y, const DFront* __restrict__ fr,
                                              const int64_t* __restrict__ order, int64_t fr_off,
                                              const int64_t* __restrict__ pre, const int64_t* __restrict__ pre_part,
                                              int64_t S, int nrhs, const double* __restrict__ partial) {
    pdl_launch_dependents();
    const int64_t i = blockIdx.x;
    const DFront f = fr[order[fr_off + i]];
    const int64_t J0 = S * WS;
    const int wb = (int)min((int64_t)WS, f.k - J0);
    const int nout = wb * nrhs;
    const int o = blockIdx.y * 256 + threadIdx.x;
    pdl_wait();
    if (o >= nout) return;
    const int64_t nc = 2 * (pre[i + 1] - pre[i]);
    const double* pbase = partial + 2 * pre_part[i] * nrhs;
    double v = 0.0;
    int64_t c = 0;
    for (; c + 32 <= nc; c += 32) {
        double t[32];
#pragma unroll
        for (int u = 0; u < 32; u++) t[u] = __ldcg(&pbase[(c + u) * nout + o]);
#pragma unroll
        for (int u = 0; u < 32; u++) v += t[u];
    }
    for (; c + 8 <= nc; c += 8) {
        double t[8];
#pragma unroll
        for (int u = 0; u < 8; u++) t[u] = __ldcg(&pbase[(c + u) * nout + o]);
#pragma unroll
        for (int u = 0; u < 8; u++) v += t[u];
    }
    for (; c < nc; c++) v += __ldcg(&pbase[c * nout + o]);
    Y[(f.start + J0) * nrhs + o] -= v;
}

// Diagonal block of a backward step, y_B already reduced: for sub-blocks bb from the last,
// y_bb = L_bb⁻ᵀ·z_bb and z_b2 −= L[bb, b2]ᵀ·y_bb for b2 < bb. One CTA per front.
template <typename T>
__global__ void __launch_bounds__(256) k_wbwd_diag_mr(double* __restrict__ Y, const T* __restrict__ panel,
                                                      const double* __restrict__ linv, const DFront* __restrict__ fr,
                                                      const int64_t* __restrict__ order, int64_t fr_off, int64_t S,
                                                      int nrhs, int cgrp) {
    pdl_launch_dependents();
    extern __shared__ __align__(16) double sm[];
    // this CTA: right-hand sides [jc0, jc0 + rc) of front blockIdx.x
    const int jc0 = blockIdx.y * cgrp, rc = min(cgrp, nrhs - jc0);
    double(*Li)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    T(*Lt)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(sm + NB * (NB + 1));
    double* z = sm + 2 * NB * (NB + 1);  // [WS][rc]
    double* yb = z + WS * rc;            // [NB][rc]
    const DFront f = fr[order[fr_off + blockIdx.x]];
    const int64_t J0 = S * WS;
    const int wb = (int)min((int64_t)WS, f.k - J0), nbw = (wb + NB - 1) / NB;
    double* yB = Y + (f.start + J0) * nrhs + jc0;
    pdl_wait();
    for (int idx = threadIdx.x; idx < nbw * NB * rc; idx += 256) {
        const int q = idx / rc, j = idx - q * rc;
        z[idx] = q < wb ? yB[(int64_t)q * nrhs + j] : 0.0;
    }
    for (int bb = nbw - 1; bb >= 0; bb--) {
        const int jbb = min(NB, wb - bb * NB);
        __syncthreads();
        load_linv<256>(Li, linv + (f.blk_off + S * 4 + bb) * (int64_t)(NB * NB));
        __syncthreads();
        for (int idx = threadIdx.x; idx < NB * rc; idx += 256) {
            const int p = idx / rc, j = idx - p * rc;
            double a0 = 0.0, a1 = 0.0;
            int q = p;
            for (; q + 1 < NB; q += 2) {
                a0 = fma(Li[q][p], z[(bb * NB + q) * rc + j], a0);
                a1 = fma(Li[q + 1][p], z[(bb * NB + q + 1) * rc + j], a1);
            }
            if (q < NB) a0 = fma(Li[q][p], z[(bb * NB + q) * rc + j], a0);
            yb[idx] = a0 + a1;
        }
        __syncthreads();
        for (int idx = threadIdx.x; idx < jbb * rc; idx += 256) {
            const int p = idx / rc, j = idx - p * rc;
            yB[(int64_t)(bb * NB + p) * nrhs + j] = yb[idx];
        }
        for (int b2 = 0; b2 < bb; b2++) {
            __syncthreads();
            load_tile<T, NB, 256>(Lt, panel + f.poff + (J0 + bb * NB) * f.ldp + J0 + b2 * NB, f.ldp, jbb, NB);
            __syncthreads();
            for (int idx = threadIdx.x; idx < NB * rc; idx += 256) {
                const int c = idx / rc, j = idx - c * rc;
                double a0 = 0.0, a1 = 0.0;
                int q = 0;
                for (; q + 1 < jbb; q += 2) {
                    a0 = fma((double)Lt[q][c], yb[q * rc + j], a0);
                    a1 = fma((double)Lt[q + 1][c], yb[(q + 1) * rc + j], a1);
                }
                if (q < jbb) a0 = fma((double)Lt[q][c], yb[q * rc + j], a0);
                z[(b2 * NB + c) * rc + j] -= a0 + a1;
            }
        }
    }
}
inline size_t mr_diag_smem(int cgrp) {
    return 2 * NB * (NB + 1) * sizeof(double) + (size_t)(WS + NB) * cgrp * sizeof(double);
}
inline size_t mr_part_smem(int cols, size_t elt) {
    const int vec = (int)(16 / elt);
    return ((size_t)PF_RPC * (cols + vec) * elt + 15) / 16 * 16 + (size_t)PF_RPC * MAXR * sizeof(double);
}

__global__ void k_divide_d(double* __restrict__ X, const double* __restrict__ d, int64_t n, int nrhs) {
    pdl_launch_dependents();
    pdl_wait();
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
// refinement: the factored matrix as a full CSR, y = A x, residual norms
// ---------------------------------------------------------------------------
// both triangles of every assembled entry: entry 2i = (row, col) of segment i, entry
// 2i+1 its mirror (or a sentinel row n on the diagonal); value = (col << 32) | segment
__global__ void k_seg_entries(const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                              const int64_t* __restrict__ front_seg, const int64_t* __restrict__ seg_dst,
                              const int64_t* __restrict__ rows, int64_t n, int32_t* __restrict__ key,
                              uint64_t* __restrict__ val) {
    const DFront f = fr[order[blockIdx.x]];
    for (int64_t i = front_seg[blockIdx.x] + threadIdx.x; i < front_seg[blockIdx.x + 1]; i += blockDim.x) {
        int64_t off = seg_dst[i] - f.poff;
        int64_t lr = off / f.ldp, lc = off - lr * f.ldp;
        int64_t qc = f.start + lc;
        int64_t qr = lr < f.k ? f.start + lr : rows[f.rows_off + lr - f.k];
        key[2 * i] = (int32_t)qr;
        val[2 * i] = ((uint64_t)qc << 32) | (uint64_t)i;
        key[2 * i + 1] = (int32_t)(qr != qc ? qc : n);
        val[2 * i + 1] = ((uint64_t)qr << 32) | (uint64_t)i;
    }
}

// counting sort of the entries by row (rows n are the discarded diagonal mirrors): the
// count per row, then (after the prefix sum of the counts) each entry at its row's
// offset plus a ticket; the order inside a row is fixed afterwards by sorting the row
__global__ void k_count_rows(const int32_t* __restrict__ key, int64_t cnt, unsigned long long* __restrict__ rc) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x)
        atomicAdd(rc + key[e], 1ull);
}

__global__ void k_place_rows(const int32_t* __restrict__ key, const uint64_t* __restrict__ val, int64_t cnt,
                             const int64_t* __restrict__ rp, int32_t* __restrict__ ticket,
                             uint64_t* __restrict__ out) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = key[e];
        out[rp[r] + atomicAdd(ticket + r, 1)] = val[e];
    }
}

__global__ void k_split_entries(const uint64_t* __restrict__ val, int64_t cnt, int64_t* __restrict__ col,
                                int64_t* __restrict__ seg) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < cnt; e += (int64_t)gridDim.x * blockDim.x) {
        col[e] = (int64_t)(val[e] >> 32);
        seg[e] = (int64_t)(val[e] & 0xffffffffull);
    }
}

// value of each CSR entry: the sum of its segment's source values
__global__ void k_gather_values(double* __restrict__ val, const double* __restrict__ src, const int64_t* __restrict__ seg,
                                const int64_t* __restrict__ seg_ptr, const int64_t* __restrict__ seg_src, int64_t nnz) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = seg[e];
        double s;
        if (seg_ptr) {
            s = 0.0;
            for (int64_t j = seg_ptr[i]; j < seg_ptr[i + 1]; j++) s += src[seg_src[j]];
        } else {
            s = src[seg_src[i]];
        }
        val[e] = s;
    }
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

// Y = A·X for two or more right-hand sides (X, Y row-major, n × nrhs): groups of L lanes
// (L a power of two, the smallest >= min(nrhs, 32)) take one row each and lane j of a
// group right-hand side j (chunks of L for more), so an X row is read as L consecutive
// doubles and the group's lanes read each matrix entry at the same address (one access).
__global__ void k_spmm(const int64_t* __restrict__ rp, const int64_t* __restrict__ col,
                       const double* __restrict__ val, const double* __restrict__ X, double* __restrict__ Y,
                       int64_t n, int nrhs, int L) {
    const int sub = (int)(threadIdx.x & (L - 1));
    const int64_t ngroups = ((int64_t)gridDim.x * blockDim.x) / L;
    for (int64_t row = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / L; row < n; row += ngroups) {
        const int64_t e0 = rp[row], e1 = rp[row + 1];
        for (int j = sub; j < nrhs; j += L) {
            const double* xj = X + j;
            double a0 = 0.0, a1 = 0.0;
            int64_t e = e0;
            for (; e + 1 < e1; e += 2) {
                a0 = fma(val[e], xj[col[e] * nrhs], a0);
                a1 = fma(val[e + 1], xj[col[e + 1] * nrhs], a1);
            }
            if (e < e1) a0 = fma(val[e], xj[col[e] * nrhs], a0);
            Y[row * nrhs + j] = a0 + a1;
        }
    }
}

// R = B − AX (in R, AX given), per-RHS reductions: red[j·5 + {0..4}] =
// {max|r|, max|x|, max|b|, Σr², Σb²} accumulated with atomics on nonnegative doubles
__device__ __forceinline__ void atomic_max_nonneg(double* a, double v) {
    atomicMax((unsigned long long*)a, (unsigned long long)__double_as_longlong(v));
}

// Per-system reductions of the refinement residual. The internal rows are split into
// segments (one per independent model of a batched factorization, else one), each
// reduced by blocks of SEG_ROWS rows: R = B − AX, and red[(g·nrhs + j)·5 + {0..4}] =
// {max|r|, max|x|, max|b|, Σr², Σb²} of segment g, right-hand side j.
constexpr int64_t SEG_ROWS = 2048;

__global__ void k_residual_seg(double* __restrict__ R, const double* __restrict__ AX, const double* __restrict__ B,
                               const double* __restrict__ X, const int64_t* __restrict__ seg_off,
                               const int64_t* __restrict__ blk_pre, int64_t nseg, int nrhs, double* __restrict__ red) {
    __shared__ double s[5][MAXR];
    for (int i = threadIdx.x; i < 5 * MAXR; i += blockDim.x) s[i / MAXR][i % MAXR] = 0.0;
    __syncthreads();
    int64_t g = find_slot2(blk_pre, nseg, blockIdx.x);
    int64_t r0 = seg_off[g] + (blockIdx.x - blk_pre[g]) * SEG_ROWS;
    int64_t r1 = min(seg_off[g + 1], r0 + SEG_ROWS);
    for (int64_t e = r0 * nrhs + threadIdx.x; e < r1 * nrhs; e += blockDim.x) {
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
        double* dst = &red[(g * nrhs + j) * 5 + w];
        if (w < 3)
            atomic_max_nonneg(dst, v);
        else
            atomicAdd(dst, v);
    }
}

// anorm[g] = max row sum of |A| over the rows of segment g
__global__ void k_seg_max(const double* __restrict__ rowsum, const int64_t* __restrict__ seg_off,
                          const int64_t* __restrict__ blk_pre, int64_t nseg, double* __restrict__ anorm) {
    int64_t g = find_slot2(blk_pre, nseg, blockIdx.x);
    int64_t r0 = seg_off[g] + (blockIdx.x - blk_pre[g]) * SEG_ROWS;
    int64_t r1 = min(seg_off[g + 1], r0 + SEG_ROWS);
    double m = 0.0;
    for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) m = fmax(m, rowsum[r]);
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomic_max_nonneg(&anorm[g], m);
}

// out = {max over (g, j) of the normwise backward error ‖r‖∞ / (‖A_g‖∞‖x‖∞ + ‖b‖∞),
//        max over (g, j) of ‖r‖₂ / ‖b‖₂}; one block of 256 threads
__global__ void k_seg_eta(const double* __restrict__ red, const double* __restrict__ anorm, int64_t nseg, int nrhs,
                          double* __restrict__ out) {
    __shared__ double se[8], sq[8];
    double e = 0.0, q = 0.0;
    for (int64_t i = threadIdx.x; i < nseg * nrhs; i += blockDim.x) {
        const double* v = red + i * 5;
        double den = anorm[i / nrhs] * v[1] + v[2];
        if (den > 0) e = fmax(e, v[0] / den);
        if (v[4] > 0) q = fmax(q, sqrt(v[3] / v[4]));
    }
    for (int o = 16; o > 0; o >>= 1) {
        e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
        q = fmax(q, __shfl_xor_sync(0xffffffffu, q, o));
    }
    if ((threadIdx.x & 31) == 0) {
        se[threadIdx.x >> 5] = e;
        sq[threadIdx.x >> 5] = q;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < (int)(blockDim.x >> 5); w++) {
            e = fmax(e, se[w]);
            q = fmax(q, sq[w]);
        }
        out[0] = e;
        out[1] = q;
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

// a kernel of a sweep, as a programmatic dependent of the previous one when pdl is set
template <typename... KArgs, typename... Args>
void launch_chained(bool pdl, void (*kern)(KArgs...), unsigned grid, unsigned block, size_t smem, cudaStream_t st,
                    Args... args) {
    launch_pdl(pdl, kern, dim3(grid), dim3(block), smem, st, args...);
}

// the sweep of an FP32 factor with at most PF_MAXR right-hand sides runs the prefetching
// kernels, all launched as programmatic dependents; other sweeps launch plainly
template <typename T>
bool pf_path(int64_t nrhs) {
    return std::is_same<T, float>::value && nrhs <= PF_MAXR;
}
// steps with 5 to 32 right-hand sides whose blocks are at least NB wide run the register-
// tiled kernels; narrower ones (the many small fronts of 2D models) the first kernels, whose
// CTAs are sized to the rows they have
inline bool mr_step(int64_t nrhs, int64_t level_maxk, int64_t S) {
    return nrhs > PF_MAXR && std::min<int64_t>(WS, level_maxk - S * WS) >= NB;
}
// sweeps whose step kernels prefetch (and so gain from programmatic dependent launches)
template <typename T>
bool chained_sweep(int64_t nrhs) {
    return pf_path<T>(nrhs) || nrhs > PF_MAXR;
}

template <int R>
void wfwd_pf(const WStep& w, int nbw_max, int cols, double* X, double* Y, double* V, const float* panel,
             const double* linv, const DevPlan& dp, cudaStream_t st) {
    launch_chained(true, k_wfwd_diag_pf<R>, (unsigned)w.nact, 256, pf_diag_smem(nbw_max, R), st, X, Y, panel, linv,
                   dp.fronts, dp.level_order, w.fr_off, w.S, nbw_max);
    launch_chained(true, k_wfwd_rows_pf<R>, (unsigned)(2 * w.n_rows), PR, pf_rows_smem(cols, R), st, X, V, Y, panel, dp.fronts,
                   dp.level_order, w.fr_off, w.nact, dp.pre_wrows + w.pre_off, w.S, cols);
}
template <int R>
void wbwd_pf(const WStep& w, int nbw_max, int cols, double* Y, const float* panel, const double* linv,
             const DevPlan& dp, double* partial, cudaStream_t st) {
    launch_chained(true, k_wbwd_part_pf<R>, (unsigned)(2 * w.n_rows), 256, pf_part_smem(cols, R), st, Y, panel, dp.fronts,
                   dp.level_order, w.fr_off, w.nact, dp.pre_wrows + w.pre_off, dp.pre_wpart + w.pre_off, dp.rows, w.S,
                   partial, cols);
    launch_chained(true, k_wbwd_diag_pf<R>, (unsigned)w.nact, 256, pf_diag_smem(nbw_max, R), st, Y, panel, linv, dp.fronts,
                   dp.level_order, w.fr_off, dp.pre_wrows + w.pre_off, dp.pre_wpart + w.pre_off, w.S, partial,
                   nbw_max);
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
int64_t Engine::forward_steps(int64_t l, double* X, double* Y, double* V, int nrhs, int* chain) {
    const Plan& P = plan_;
    const T* panel = (const T*)panel_;
    int64_t launches = 0;
    if (chain && P.level_chain[l]) {
        const int64_t i0 = P.chain_fwd_off[l], r0 = P.chain_rows_off[l], nr = P.chain_rows_off[l + 1] - r0;
        launch_chain_fwd(nrhs, P.chain_fwd_off[l + 1] - i0, X, Y, (const float*)panel_, chain_inv_, dp_.fronts,
                         dp_.chain_blk, dp_.chain_fwd + 2 * i0, chain, chain + 2 * P.chain_blocks + 2 * l, chain_err_,
                         stream_);
        launch_chain_rows(nrhs, nr, Y, V, (const float*)panel_, dp_.fronts, dp_.chain_rows + 2 * r0, stream_);
        return nr > 0 ? 2 : 1;
    }
    for (int64_t wi = P.wstep_off[l]; wi < P.wstep_off[l + 1]; wi++) {
        const WStep& w = P.wsteps[wi];
        if (pf_path<T>(nrhs)) {
            const float* pf = (const float*)panel_;
            const int64_t wb_max = std::min<int64_t>(WS, P.level_maxk[l] - w.S * WS);
            const int nbw_max = (int)((wb_max + NB - 1) / NB), cols = pf_cols(wb_max);
            if (nrhs == 1) wfwd_pf<1>(w, nbw_max, cols, X, Y, V, pf, linv_, dp_, stream_);
            else if (nrhs == 2) wfwd_pf<2>(w, nbw_max, cols, X, Y, V, pf, linv_, dp_, stream_);
            else if (nrhs == 3) wfwd_pf<3>(w, nbw_max, cols, X, Y, V, pf, linv_, dp_, stream_);
            else wfwd_pf<4>(w, nbw_max, cols, X, Y, V, pf, linv_, dp_, stream_);
        } else if (mr_step(nrhs, P.level_maxk[l], w.S)) {
            const int pr = wfwd_piece_rows(P.level_maxk[l], w.S);
            const int cols = pf_cols(std::min<int64_t>(WS, P.level_maxk[l] - w.S * WS));
            {
                // eight right-hand sides per CTA: the stages of a wide block run in parallel over the columns
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3((unsigned)w.nact, (unsigned)((nrhs + 7) / 8));
                cfg.blockDim = dim3(256);
                cfg.dynamicSmemBytes = wfwd_diag_smem<T>(pr, 8);
                cfg.stream = stream_;
                RFG_CUDA(cudaLaunchKernelEx(&cfg, k_wfwd_diag<T>, (const double*)X, Y, panel, (const double*)linv_,
                                            (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, w.fr_off, w.S,
                                            nrhs, pr, 8));
            }
            launch_chained(true, k_wfwd_rows_mr<T>, (unsigned)(2 * w.n_rows), 256, mr_rows_smem(cols, sizeof(T)), stream_,
                           X, V, Y, panel, dp_.fronts, dp_.level_order, w.fr_off, w.nact, dp_.pre_wrows + w.pre_off, w.S,
                           nrhs, cols);
        } else {
            const int pr = wfwd_piece_rows(P.level_maxk[l], w.S);
            launch_chained(false, k_wfwd_diag<T>, (unsigned)w.nact, 256, wfwd_diag_smem<T>(pr, nrhs), stream_, X, Y, panel,
                           linv_, dp_.fronts, dp_.level_order, w.fr_off, w.S, nrhs, pr, nrhs);
            launch_chained(false, k_wfwd_rows<T>, (unsigned)w.n_rows, PR, (size_t)WS * nrhs * sizeof(double), stream_, X, V, Y,
                           panel, dp_.fronts, dp_.level_order, w.fr_off, w.nact, dp_.pre_wrows + w.pre_off, w.S, nrhs);
        }
        launches += 2;
    }
    return launches;
}

template <typename T>
int64_t Engine::backward_steps(int64_t l, double* Y, double* V, int nrhs, double* partial, int* tickets, int* chain) {
    const Plan& P = plan_;
    const T* panel = (const T*)panel_;
    int64_t launches = 0;
    if (chain && P.level_chain[l]) {
        const int64_t i0 = P.chain_bwd_off[l], r0 = P.chain_rows_off[l], c0 = P.chain_cols_off[l];
        const int64_t nr = P.chain_rows_off[l + 1] - r0, nc = P.chain_cols_off[l + 1] - c0;
        launch_chain_cols(nrhs, nr, dp_.chain_rows + 2 * r0, nc, dp_.chain_cols + 2 * c0, Y, V, partial,
                          (const float*)panel_, dp_.fronts, dp_.rows, stream_);
        launch_chain_bwd(nrhs, P.chain_bwd_off[l + 1] - i0, Y, (const float*)panel_, chain_inv_, dp_.fronts,
                         dp_.chain_blk, dp_.chain_bwd + 2 * i0, chain + P.chain_blocks,
                         chain + 2 * P.chain_blocks + 2 * l + 1, chain_err_, stream_);
        return nc > 0 ? 4 : 1;
    }
    for (int64_t wi = P.wstep_off[l + 1] - 1; wi >= P.wstep_off[l]; wi--) {
        const WStep& w = P.wsteps[wi];
        if (pf_path<T>(nrhs)) {
            const float* pf = (const float*)panel_;
            const int64_t wb_max = std::min<int64_t>(WS, P.level_maxk[l] - w.S * WS);
            const int nbw_max = (int)((wb_max + NB - 1) / NB), cols = pf_cols(wb_max);
            if (nrhs == 1) wbwd_pf<1>(w, nbw_max, cols, Y, pf, linv_, dp_, partial, stream_);
            else if (nrhs == 2) wbwd_pf<2>(w, nbw_max, cols, Y, pf, linv_, dp_, partial, stream_);
            else if (nrhs == 3) wbwd_pf<3>(w, nbw_max, cols, Y, pf, linv_, dp_, partial, stream_);
            else wbwd_pf<4>(w, nbw_max, cols, Y, pf, linv_, dp_, partial, stream_);
            launches += 2;
        } else if (mr_step(nrhs, P.level_maxk[l], w.S)) {
            const int64_t wb_max = std::min<int64_t>(WS, P.level_maxk[l] - w.S * WS);
            const int cols = pf_cols(wb_max);
            launch_chained(true, k_wbwd_part_mr<T>, (unsigned)(2 * w.n_rows), 256, mr_part_smem(cols, sizeof(T)), stream_, Y,
                           panel, dp_.fronts, dp_.level_order, w.fr_off, w.nact, dp_.pre_wrows + w.pre_off,
                           dp_.pre_wpart + w.pre_off, dp_.rows, w.S, nrhs, partial, cols);
            {
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3((unsigned)w.nact, (unsigned)((wb_max * nrhs + 255) / 256));
                cfg.blockDim = dim3(256);
                cfg.stream = stream_;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = at;
                cfg.numAttrs = pdl_enabled() ? 1 : 0;
                RFG_CUDA(cudaLaunchKernelEx(&cfg, k_wred, Y, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order,
                                            w.fr_off, (const int64_t*)(dp_.pre_wrows + w.pre_off),
                                            (const int64_t*)(dp_.pre_wpart + w.pre_off), w.S, nrhs,
                                            (const double*)partial));
            }
            {
                // eight right-hand sides per CTA
                cudaLaunchConfig_t cfg{};
                cfg.gridDim = dim3((unsigned)w.nact, (unsigned)((nrhs + 7) / 8));
                cfg.blockDim = dim3(256);
                cfg.dynamicSmemBytes = mr_diag_smem(8);
                cfg.stream = stream_;
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
                at[0].val.programmaticStreamSerializationAllowed = 1;
                cfg.attrs = at;
                cfg.numAttrs = pdl_enabled() ? 1 : 0;
                RFG_CUDA(cudaLaunchKernelEx(&cfg, k_wbwd_diag_mr<T>, Y, panel, (const double*)linv_,
                                            (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, w.fr_off, w.S,
                                            nrhs, 8));
            }
            launches += 3;
        } else {
            launch_chained(false, k_wbwd<T>, (unsigned)w.n_rows, 256, wbwd_smem<T>(nrhs), stream_, Y, panel, linv_, dp_.fronts,
                           dp_.level_order, w.fr_off, w.nact, dp_.pre_wrows + w.pre_off, dp_.pre_wpart + w.pre_off,
                           dp_.rows, w.S, nrhs, partial, tickets);
            launches++;
        }
    }
    return launches;
}

template <typename T>
void Engine::solve_impl(double* X, int64_t nrhs_total) {
    const Plan& P = plan_;
    int64_t launches = 0;
    // X is row-major n × nrhs_total; sweeps of at most MAXR right-hand sides work on a
    // contiguous copy when nrhs_total > MAXR
    if (nrhs_total > MAXR) {
        double* tmp = (double*)nullptr;
        tmp = (decltype(tmp))dev_alloc(P.n * MAXR * sizeof(double), stream_);
        for (int64_t j0 = 0; j0 < nrhs_total; j0 += MAXR) {
            int64_t nr = std::min<int64_t>(MAXR, nrhs_total - j0);
            RFG_CUDA(cudaMemcpy2DAsync(tmp, nr * sizeof(double), X + j0, nrhs_total * sizeof(double), nr * sizeof(double),
                                       P.n, cudaMemcpyDeviceToDevice, stream_));
            solve_impl<T>(tmp, nr);
            RFG_CUDA(cudaMemcpy2DAsync(X + j0, nrhs_total * sizeof(double), tmp, nr * sizeof(double), nr * sizeof(double),
                                       P.n, cudaMemcpyDeviceToDevice, stream_));
        }
        dev_free(tmp, stream_);
        return;
    }
    int nrhs = (int)nrhs_total;
    RFG_CUDA(cudaMemsetAsync(vupd_, 0, std::max<int64_t>(P.vu_rows * nrhs, 1) * sizeof(double), stream_));
    int* chain = std::is_same<T, float>::value && chain_on(nrhs) ? counters_ + std::max<int64_t>(P.max_nact, 1) : nullptr;
    if (chain) RFG_CUDA(cudaMemsetAsync(chain, 0, chain_flag_words(P) * sizeof(int), stream_));
    for (int64_t l = 0; l < P.nlevels; l++) {
        for (int r = 0; r < 2; r++) {
            const DXadd& x = P.xadd[2 * l + r];
            if (x.nblk == 0) continue;
            launch_chained(chained_sweep<T>(nrhs), k_vec_extend_add, (unsigned)x.nblk, 256, 0, stream_, X, vupd_, dp_.fronts,
                           (const int64_t*)(dp_.xadd_task + 4 * x.task_off), x.ntask, (const int32_t*)dp_.emap, nrhs);
            launches++;
        }
        launches += forward_steps<T>(l, X, ybuf_, vupd_, nrhs, chain);
    }
    launch_chained(chained_sweep<T>(nrhs), k_divide_d, (unsigned)grid_for(P.n * nrhs), 256, 0, stream_, ybuf_, (const double*)d_, P.n, nrhs);
    launches++;
    for (int64_t l = P.nlevels - 1; l >= 0; l--)
        launches += backward_steps<T>(l, ybuf_, vupd_, nrhs, partial_, counters_, chain);
    RFG_CUDA(cudaMemcpyAsync(X, ybuf_, P.n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    RFG_CUDA(cudaGetLastError());
    solve_launches += launches;
}

// Large dynamic shared-memory limits of the sweep kernels. Function attributes belong
// to the current device's context, so they are set once per device (a handle on a
// second device in the same process needs its own), under a lock because handles may
// be used from several host threads.
static void solve_set_attributes_current_device();

void solve_set_attributes() {
    static std::mutex mu;
    static bool done[64] = {};
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw CudaError("solve_set_attributes: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (done[dev]) return;
    solve_set_attributes_current_device();
    done[dev] = true;
}

static void solve_set_attributes_current_device() {
    RFG_CUDA(cudaFuncSetAttribute(k_wfwd_diag<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)wfwd_diag_smem<double>(3 * NB, MAXR)));
    RFG_CUDA(cudaFuncSetAttribute(k_wfwd_diag<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)wfwd_diag_smem<float>(3 * NB, MAXR)));
    RFG_CUDA(cudaFuncSetAttribute(k_wfwd_rows<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(WS * MAXR * sizeof(double))));
    RFG_CUDA(cudaFuncSetAttribute(k_wfwd_rows<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(WS * MAXR * sizeof(double))));
    RFG_CUDA(cudaFuncSetAttribute(k_wbwd<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wbwd_smem<double>(MAXR)));
    auto pf_attrs = [](auto diag_f, auto rows_f, auto part_f, auto diag_b, int r) {
        RFG_CUDA(cudaFuncSetAttribute(diag_f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pf_diag_smem(4, r)));
        RFG_CUDA(cudaFuncSetAttribute(rows_f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pf_rows_smem(WS, r)));
        RFG_CUDA(cudaFuncSetAttribute(part_f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pf_part_smem(WS, r)));
        RFG_CUDA(cudaFuncSetAttribute(diag_b, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pf_diag_smem(4, r)));
    };
    pf_attrs(k_wfwd_diag_pf<1>, k_wfwd_rows_pf<1>, k_wbwd_part_pf<1>, k_wbwd_diag_pf<1>, 1);
    pf_attrs(k_wfwd_diag_pf<2>, k_wfwd_rows_pf<2>, k_wbwd_part_pf<2>, k_wbwd_diag_pf<2>, 2);
    pf_attrs(k_wfwd_diag_pf<3>, k_wfwd_rows_pf<3>, k_wbwd_part_pf<3>, k_wbwd_diag_pf<3>, 3);
    pf_attrs(k_wfwd_diag_pf<4>, k_wfwd_rows_pf<4>, k_wbwd_part_pf<4>, k_wbwd_diag_pf<4>, 4);
    RFG_CUDA(cudaFuncSetAttribute(k_wfwd_rows_mr<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mr_rows_smem(WS, sizeof(float))));
    RFG_CUDA(cudaFuncSetAttribute(k_wfwd_rows_mr<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mr_rows_smem(WS, sizeof(double))));
    RFG_CUDA(cudaFuncSetAttribute(k_wbwd_part_mr<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mr_part_smem(WS, sizeof(float))));
    RFG_CUDA(cudaFuncSetAttribute(k_wbwd_part_mr<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mr_part_smem(WS, sizeof(double))));
    RFG_CUDA(cudaFuncSetAttribute(k_wbwd_diag_mr<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mr_diag_smem(8)));
    RFG_CUDA(cudaFuncSetAttribute(k_wbwd_diag_mr<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mr_diag_smem(8)));
    RFG_CUDA(cudaFuncSetAttribute(k_wbwd<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wbwd_smem<float>(MAXR)));
}

void Engine::solve_device(double* X, int64_t nrhs, bool allow_graph) {
    if (nrhs <= 0 || plan_.n == 0) return;
    solve_set_attributes();
    // the sweep's workspace must exist before a capture. It is sized for up to four
    // right-hand sides, or for MAXR once a wider solve comes: a handle solved with one
    // right-hand side does not take (and grow the memory pool by) 32 columns of it
    if (ws_nrhs_ < std::min<int64_t>(nrhs, MAXR)) {
        const int64_t w = nrhs <= 4 ? 4 : MAXR;
        if (ws_nrhs_ > 0) {
            // the captured sweeps refer to the narrower buffers
            RFG_CUDA(cudaStreamSynchronize(stream_));
            for (auto& g : solve_graphs_) RFG_CUDA(cudaGraphExecDestroy(g.exec));
            solve_graphs_.clear();
            solve_seen_.clear();
            for (void* q : {(void*)vupd_, (void*)partial_, (void*)ybuf_, (void*)counters_}) {
                allocs_.erase(std::find(allocs_.begin(), allocs_.end(), q));
                dev_free(q, stream_);
            }
        }
        vupd_ = (double*)dalloc(std::max<int64_t>(plan_.vu_rows * w, 1) * sizeof(double));
        partial_ = (double*)dalloc(std::max<int64_t>(partial_rows() * w, 1) * sizeof(double));
        ybuf_ = (double*)dalloc(std::max<int64_t>(plan_.n * w, 1) * sizeof(double));
        counters_ = (int*)dalloc(ticket_words() * sizeof(int));
        RFG_CUDA(cudaMemsetAsync(counters_, 0, ticket_words() * sizeof(int), stream_));
        ws_nrhs_ = w;
    }
    if (chain_on(nrhs)) ensure_chain_inverse();
    if (use_graphs_ && nrhs <= MAXR) {
        cudaGraphExec_t ex = nullptr;
        for (auto& g : solve_graphs_)
            if (g.X == X && g.nrhs == nrhs) ex = g.exec;
        if (!ex) {
            // a sweep is captured the second time it runs on the same buffer and width; the
            // first run goes directly (a one-off solve does not pay for the capture)
            int64_t* uses = nullptr;
            for (auto& k : solve_seen_)
                if (k.first.first == X && k.first.second == nrhs) uses = &k.second;
            if (!uses) {
                solve_seen_.push_back({{X, nrhs}, 0});
                uses = &solve_seen_.back().second;
            }
            if (++*uses < 2 || !allow_graph) {
                if (prec_ == PREC_FP64)
                    solve_impl<double>(X, nrhs);
                else
                    solve_impl<float>(X, nrhs);
                return;
            }
        }
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

namespace {
int64_t round256(int64_t b) { return (b + 255) / 256 * 256; }
}  // namespace

bool Engine::chain_on(int64_t nrhs) const {
    return prec_ == PREC_MIXED && chain_inv_ != nullptr && nrhs >= 1 && nrhs <= PF_MAXR;
}

int64_t Engine::partial_rows() const {
    return std::max<int64_t>(2 * plan_.max_wpart, chain_inv_ ? plan_.chain_colpart : 0);
}

int64_t Engine::ticket_words() const {
    return std::max<int64_t>(plan_.max_nact, 1) + (chain_inv_ ? chain_flag_words(plan_) : 0);
}

// The chain blocks' inverses for the current factor: formed by the first sweep after each
// numeric phase (on the engine's stream, before that sweep's launches or graph).
void Engine::ensure_chain_inverse() {
    if (chain_inv_at_ == factor_calls_) return;
    launch_chain_inverse(chain_inv_, (const float*)panel_, linv_, dp_.fronts, dp_.chain_blk, dp_.chain_bfront,
                         plan_.chain_blocks, stream_);
    solve_launches++;
    chain_inv_at_ = factor_calls_;
}

void Engine::chain_check() {
    if (!chain_err_) return;
    int v = 0;
    RFG_CUDA(cudaMemcpyAsync(&v, chain_err_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaStreamSynchronize(stream_));
    if (v != 0) {
        RFG_CUDA(cudaMemsetAsync(chain_err_, 0, sizeof(int), stream_));
        throw CudaError("solve chain: a bounded wait gave up; the solutions since the last check are invalid");
    }
}

int64_t Engine::sweep_workspace_bytes(int64_t nrhs) const {
    const Plan& P = plan_;
    return round256(std::max<int64_t>(P.n * nrhs, 1) * 8) + round256(std::max<int64_t>(P.vu_rows * nrhs, 1) * 8) +
           round256(std::max<int64_t>(partial_rows() * nrhs, 1) * 8) + round256(ticket_words() * 4);
}

Engine::SweepWorkspace Engine::carve_sweep_workspace(void* base, int64_t nrhs) const {
    const Plan& P = plan_;
    char* p = (char*)base;
    SweepWorkspace ws;
    ws.y = (double*)p;
    p += round256(std::max<int64_t>(P.n * nrhs, 1) * 8);
    ws.v = (double*)p;
    p += round256(std::max<int64_t>(P.vu_rows * nrhs, 1) * 8);
    ws.partial = (double*)p;  // two blocks of partials per chunk on the prefetching path
    p += round256(std::max<int64_t>(partial_rows() * nrhs, 1) * 8);
    ws.tickets = (int*)p;
    return ws;
}

// The launches of solve_impl, on the workspace ws instead of the engine's own buffers.
template <typename T>
void Engine::solve_sweep_impl(double* X, int64_t nrhs_total, const SweepWorkspace& ws) {
    const Plan& P = plan_;
    int nrhs = (int)nrhs_total;
    RFG_CUDA(cudaMemsetAsync(ws.v, 0, std::max<int64_t>(P.vu_rows * nrhs, 1) * sizeof(double), stream_));
    RFG_CUDA(cudaMemsetAsync(ws.tickets, 0, ticket_words() * sizeof(int), stream_));
    int* chain = std::is_same<T, float>::value && chain_on(nrhs) ? ws.tickets + std::max<int64_t>(P.max_nact, 1) : nullptr;
    for (int64_t l = 0; l < P.nlevels; l++) {
        for (int r = 0; r < 2; r++) {
            const DXadd& x = P.xadd[2 * l + r];
            if (x.nblk == 0) continue;
            launch_chained(chained_sweep<T>(nrhs), k_vec_extend_add, (unsigned)x.nblk, 256, 0, stream_, X, ws.v, dp_.fronts,
                           (const int64_t*)(dp_.xadd_task + 4 * x.task_off), x.ntask, (const int32_t*)dp_.emap, nrhs);
        }
        forward_steps<T>(l, X, ws.y, ws.v, nrhs, chain);
    }
    launch_chained(chained_sweep<T>(nrhs), k_divide_d, (unsigned)grid_for(P.n * nrhs), 256, 0, stream_, ws.y, (const double*)d_, P.n, nrhs);
    for (int64_t l = P.nlevels - 1; l >= 0; l--) backward_steps<T>(l, ws.y, ws.v, nrhs, ws.partial, ws.tickets, chain);
    RFG_CUDA(cudaMemcpyAsync(X, ws.y, P.n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    RFG_CUDA(cudaGetLastError());
}

void Engine::solve_sweep_on(double* X, int64_t nrhs, const SweepWorkspace& ws) {
    if (nrhs <= 0 || plan_.n == 0) return;
    if (nrhs > MAXR) throw CudaError("solve_sweep_on: at most 32 right-hand sides per sweep");
    solve_set_attributes();
    if (chain_on(nrhs)) ensure_chain_inverse();
    if (prec_ == PREC_FP64)
        solve_sweep_impl<double>(X, nrhs, ws);
    else
        solve_sweep_impl<float>(X, nrhs, ws);
}

void* noalloc_scratch() {
    static std::mutex mu;
    static void* addr[64] = {};
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw CudaError("noalloc_scratch: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!addr[dev]) {
        void* ptr = nullptr;
        cudaError_t rc = cudaGetSymbolAddress((void**)&ptr, g_noalloc_scratch);
        if (rc != cudaSuccess || !ptr)
            throw CudaError(std::string("cudaGetSymbolAddress of the static solve scratch failed: ") +
                            cudaGetErrorString(rc));
        addr[dev] = ptr;
    }
    return addr[dev];
}

void Engine::set_segments(const std::vector<int64_t>& off) {
    if (off.size() < 2 || off.front() != 0 || off.back() != plan_.n) throw CudaError("set_segments: bad offsets");
    int64_t nseg = (int64_t)off.size() - 1;
    std::vector<int64_t> pre(nseg + 1, 0);
    for (int64_t g = 0; g < nseg; g++) {
        if (off[g + 1] < off[g]) throw CudaError("set_segments: offsets must not decrease");
        pre[g + 1] = pre[g] + (off[g + 1] - off[g] + SEG_ROWS - 1) / SEG_ROWS;
    }
    if (ref_red_ && (int64_t)seg_off_.size() != nseg + 1) {
        dev_free(ref_red_, stream_);
        ref_red_ = nullptr;
        ref_nrhs_ = 0;
        if (ref_r_) dev_free(ref_r_, stream_);
        if (ref_dx_) dev_free(ref_dx_, stream_);
        ref_r_ = ref_dx_ = nullptr;
    }
    seg_off_ = off;
    seg_blocks_ = pre[nseg];
    d_seg_off_ = (int64_t*)dalloc((nseg + 1) * sizeof(int64_t));
    d_seg_blk_ = (int64_t*)dalloc((nseg + 1) * sizeof(int64_t));
    RFG_CUDA(cudaMemcpyAsync(d_seg_off_, off.data(), (nseg + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    RFG_CUDA(cudaMemcpyAsync(d_seg_blk_, pre.data(), (nseg + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    RFG_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::build_matrix() {
    int64_t n = plan_.n, nseg = nseg_;
    if (nseg >= ((int64_t)1 << 32) || n >= ((int64_t)1 << 31)) throw CudaError("build_matrix: matrix too large");
    int64_t cnt = 2 * nseg;
    // the work buffers: the update arena when it is large enough (its update blocks are
    // dead once the numeric phase has run, and the next numeric phase rewrites them), so a
    // new handle's first solve allocates nothing of this size
    auto r256 = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t c1 = (size_t)std::max<int64_t>(cnt, 1);
    const size_t nr = (size_t)n + 2;  // rows 0..n (n: diagonal mirrors) and the total
    const size_t need = r256(c1 * 4) + 2 * r256(c1 * 8) + r256(nr * 8) + r256(nr * 4) +
                        r256((size_t)scan_tmp_elems((int64_t)nr) * 8);
    const size_t es = prec_ == PREC_FP64 ? sizeof(double) : sizeof(float);
    char* base = nullptr;
    const bool in_arena = (size_t)plan_.upd_elems * es >= need;
    base = in_arena ? (char*)upd_ : (char*)dev_alloc(need, stream_);
    char* p = base;
    int32_t* k0 = (int32_t*)p;
    p += r256(c1 * 4);
    uint64_t* v0 = (uint64_t*)p;
    p += r256(c1 * 8);
    uint64_t* v1 = (uint64_t*)p;
    p += r256(c1 * 8);
    int64_t* rp = (int64_t*)p;
    p += r256(nr * 8);
    int32_t* ticket = (int32_t*)p;
    p += r256(nr * 4);
    int64_t* stmp = (int64_t*)p;
    if (plan_.nfronts > 0)
        k_seg_entries<<<(unsigned)plan_.nfronts, 256, 0, stream_>>>(dp_.fronts, dp_.level_order, dp_.front_seg,
                                                                    dp_.seg_dst, dp_.rows, n, k0, v0);
    RFG_CUDA(cudaMemsetAsync(rp, 0, nr * 8, stream_));
    RFG_CUDA(cudaMemsetAsync(ticket, 0, nr * 4, stream_));
    if (cnt > 0) k_count_rows<<<grid_for(cnt), 256, 0, stream_>>>(k0, cnt, (unsigned long long*)rp);
    exclusive_scan_i64(rp, (int64_t)nr, stmp, stream_);
    if (cnt > 0) k_place_rows<<<grid_for(cnt), 256, 0, stream_>>>(k0, v0, cnt, rp, ticket, v1);
    // (column << 32 | segment) is distinct within a row: sorted rows do not depend on
    // the order in which the tickets were drawn
    sort_rows_u64(v1, rp, n, stream_);
    RFG_CUDA(cudaMemcpyAsync(a_rowptr_, rp, (n + 1) * sizeof(int64_t), cudaMemcpyDeviceToDevice, stream_));
    int64_t nnz = 0;
    RFG_CUDA(cudaMemcpyAsync(&nnz, rp + n, sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaStreamSynchronize(stream_));
    a_nnz_ = nnz;
    if (nnz > 0) k_split_entries<<<grid_for(nnz), 256, 0, stream_>>>(v1, nnz, a_col_, a_src_);
    if (!in_arena) dev_free(base, stream_);
    RFG_CUDA(cudaStreamSynchronize(stream_));
    matrix_built_ = true;
}

void Engine::matvec(const double* X, double* Y, int64_t nrhs) {
    const int64_t n = plan_.n;
    if (nrhs <= 1) {
        k_spmv<<<grid_for(n * 32, 256), 256, 0, stream_>>>(a_rowptr_, a_col_, a_val_, X, Y, n, (int)nrhs, nullptr);
        return;
    }
    int L = 1;
    while (L < nrhs && L < 32) L *= 2;
    k_spmm<<<grid_for(n * L, 256), 256, 0, stream_>>>(a_rowptr_, a_col_, a_val_, X, Y, n, (int)nrhs, L);
}

SolveStats Engine::solve_refined(double* X, const double* B, int64_t nrhs, double tol, int max_iter) {
    SolveStats st;
    int64_t n = plan_.n;
    if (n == 0 || nrhs == 0) return st;
    if (nrhs > MAXR) throw CudaError("solve_refined: at most 32 right-hand sides per call");
    HostTimer timer("solve_refined");
    // with RFG_HOST_TIMING set, each lap waits for the stream so that it times the device work
    auto lap = [&](const char* what) {
        if (!timer.on) return;
        RFG_CUDA(cudaStreamSynchronize(stream_));
        timer.lap(what);
    };
    if (!matrix_built_) build_matrix();
    lap("matrix");
    // the first refined solve of an engine runs its sweeps without capturing graphs
    const bool graphs = refined_calls_++ > 0;
    int64_t l0 = solve_launches;
    // the matrix values of the current factorization and ‖A‖∞
    k_gather_values<<<grid_for(a_nnz_), 256, 0, stream_>>>(a_val_, src_, a_src_, dp_.seg_ptr, dp_.seg_src, a_nnz_);
    if (seg_off_.empty()) set_segments({0, n});
    const int64_t nseg = (int64_t)seg_off_.size() - 1;
    // red: 5 values per (segment, right-hand side), then anorm per segment, then ‖A‖∞
    // and the two maxima of k_seg_eta
    const int64_t nred = 5 * nseg * MAXR + nseg + 3;
    if (ref_nrhs_ < nrhs) {
        if (ref_r_) dev_free(ref_r_, stream_);
        if (ref_dx_) dev_free(ref_dx_, stream_);
        if (ref_red_) dev_free(ref_red_, stream_);
        ref_r_ = (double*)dev_alloc(n * MAXR * sizeof(double), stream_);
        ref_dx_ = (double*)dev_alloc(n * MAXR * sizeof(double), stream_);
        ref_red_ = (double*)dev_alloc(nred * sizeof(double), stream_);
        ref_nrhs_ = MAXR;
    }
    double* seg_anorm = ref_red_ + 5 * nseg * MAXR;
    double* eta_out = seg_anorm + nseg + 1;
    RFG_CUDA(cudaMemsetAsync(ref_red_, 0, nred * sizeof(double), stream_));
    k_spmv<<<grid_for(n * 32, 256), 256, 0, stream_>>>(a_rowptr_, a_col_, a_val_, nullptr, nullptr, n, 0, ref_dx_);
    k_max_reduce<<<grid_for(n), 256, 0, stream_>>>(ref_dx_, n, seg_anorm + nseg);
    if (seg_blocks_ > 0)
        k_seg_max<<<(unsigned)seg_blocks_, 256, 0, stream_>>>(ref_dx_, d_seg_off_, d_seg_blk_, nseg, seg_anorm);
    RFG_CUDA(cudaMemcpyAsync(&anorm_, seg_anorm + nseg, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    if (X != B) RFG_CUDA(cudaMemcpyAsync(X, B, n * nrhs * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    lap("values, norms");
    solve_device(X, nrhs, graphs);
    lap("sweep");
    double eo[2] = {0.0, 0.0};
    for (int it = 0;; it++) {
        RFG_CUDA(cudaMemsetAsync(ref_red_, 0, 5 * nseg * nrhs * sizeof(double), stream_));
        matvec(X, ref_dx_, nrhs);
        if (seg_blocks_ > 0)
            k_residual_seg<<<(unsigned)seg_blocks_, 256, 0, stream_>>>(ref_r_, ref_dx_, B, X, d_seg_off_, d_seg_blk_,
                                                                      nseg, (int)nrhs, ref_red_);
        k_seg_eta<<<1, 256, 0, stream_>>>(ref_red_, seg_anorm, nseg, (int)nrhs, eta_out);
        solve_launches += 3;
        RFG_CUDA(cudaMemcpyAsync(eo, eta_out, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        RFG_CUDA(cudaStreamSynchronize(stream_));
        st.backward_error = eo[0];
        st.rel_residual = eo[1];
        st.iterations = it;
        lap("residual");
        if (eo[0] <= tol || it >= max_iter) break;
        solve_device(ref_r_, nrhs, graphs);
        k_axpy<<<grid_for(n * nrhs), 256, 0, stream_>>>(X, ref_r_, n * nrhs);
        solve_launches += 1;
        lap("sweep");
    }
    chain_check();
    st.launches = solve_launches - l0;
    return st;
}

}  // namespace rfg
