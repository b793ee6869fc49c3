// Solve chains (chain.h): the forward and backward sweeps of the levels with few fronts
// in one launch per level and direction.
//
// A level at the top of the tree has one to a few fronts of thousands of pivots. Stepped
// the usual way (solve.cu) each WS-wide block costs a launch for its diagonal block on one
// CTA and a launch for the rows below, and the GPU waits on the first. Here the level's
// work items are WS-wide diagonal blocks (and, forward, WS-row pieces of the later rows),
// each done by a cluster of four CTAs:
//   forward, block B of a front, CTA s owning the rows B·WS + 64s ... + 63:
//       x_s = X[rows] − Σ_{J < B} L[rows, J]·y_J   (tile J as soon as block J's flag is up)
//       x_B gathered from the cluster's CTAs (distributed shared memory),
//       y[rows] = inv(L_BB)[rows, :]·x_B, then the block's flag is raised;
//   forward, later rows: V[rows] −= Σ_J L[rows, J]·y_J over all blocks J;
//   backward, block B, CTA s owning the columns B·WS + 64s ... + 63:
//       z_s = Y[cols] − Σ_{r later} L[r, cols]·y_r − Σ_{J > B} L[J, cols]ᵀ·y_J,
//       y[cols] = inv(L_BB)[:, cols]ᵀ·z_B.
// The tiles of a block stream through a ring of four cp.async stages while the CTA waits
// for the flags; the dependency chain from block to block is one flag wait, the last
// tile, a cluster barrier and one product with the WS × WS inverse.
//
// Items are taken in the plan's order from a counter, by the first CTA of a cluster when
// its previous item is done. Every item depends only on items before it in that order and
// an item is only taken by a running cluster, so the launch progresses with any number of
// resident clusters. Waits are bounded: a wait that gives up sets *err, the CTA goes on
// with the values it finds, every later wait of the launch returns at once, and the host
// reports the error (Engine::chain_check).
#include <cooperative_groups.h>

#include <algorithm>
#include <mutex>

#include "chain.h"
#include "engine.h"
#include "tiles.cuh"

namespace cg = cooperative_groups;

namespace rfg {
namespace {

constexpr int CT = 256;             // threads per CTA
constexpr int CQ = WS / 4;          // rows (forward) or columns (backward) of a block per CTA
constexpr int CL = WS / CQ;         // CTAs per cluster: one block
constexpr int FQP = CQ + 16;        // pitch (floats) of a forward tile quarter: float4 rows without conflicts
constexpr int FLP = WS + 4;         // pitch (doubles) of the forward inverse rows
constexpr int BTP = CQ;             // pitch (floats) of a backward tile chunk
constexpr long CHAIN_SPIN = 1L << 22;  // polls of a flag (about a second) before a wait gives up

static_assert(CL == 4 && CT == 4 * CQ, "four CTAs of 256 threads per block");
static_assert(CQ == CHAIN_PIECE, "the later-row pieces of the plan are one CTA's rows or columns");

constexpr size_t fwd_smem(int R) {
    return (size_t)CQ * FLP * 8 + (size_t)4 * CQ * FQP * 4 + (size_t)WS * R * 8 + (size_t)CQ * R * 8;
}
constexpr size_t bwd_smem(int R) {
    return (size_t)WS * CQ * 8 + (size_t)4 * CQ * BTP * 4 + (size_t)4 * CQ * R * 8 + (size_t)WS * R * 8 +
           (size_t)CQ * R * 8;
}
constexpr size_t INV_SMEM = (size_t)2 * NB * (NB + 1) * sizeof(double);
static_assert(fwd_smem(4) <= 232448 && bwd_smem(4) <= 232448, "shared memory of a CTA");

__device__ __forceinline__ int ld_acquire(const int* p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed(const int* p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// One thread: waits until *flag >= target, at most CHAIN_SPIN polls.
__device__ void chain_wait(const int* flag, int target, int* err) {
    if (ld_acquire(flag) >= target) return;
    for (long it = 0; it < CHAIN_SPIN; it++) {
        if (ld_relaxed(err) != 0) return;
        __nanosleep(32);
        if (ld_acquire(flag) >= target) return;
    }
    atomicExch(err, 1);
}

// The CTA's writes before this call are visible to any thread that sees the flag count it.
__device__ __forceinline__ void chain_signal(int* flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(flag, 1);
    }
}

// cp.async of 8 bytes, global -> shared (the source written by an earlier launch)
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_wait_upto(int n) {
    if (n <= 0)
        cp_async_wait<0>();
    else if (n == 1)
        cp_async_wait<1>();
    else if (n == 2)
        cp_async_wait<2>();
    else
        cp_async_wait<3>();
}

// The cluster's next item: the first CTA takes it from the counter and writes it into the
// shared word of every CTA of the cluster.
__device__ __forceinline__ int64_t grab(cg::cluster_group& cluster, int64_t* s_item, int* counter) {
    if (cluster.block_rank() == 0 && threadIdx.x == 0) {
        const int64_t v = atomicAdd(counter, 1);
        for (int r = 0; r < CL; r++) *cluster.map_shared_rank(s_item, r) = v;
    }
    cluster.sync();
    return *s_item;
}

// Sum over the four lanes of a row (lanes 4i .. 4i+3); every lane gets the same value.
template <int R>
__device__ __forceinline__ void quad_sum(double (&a)[R]) {
#pragma unroll
    for (int r = 0; r < R; r++) {
        a[r] += __shfl_xor_sync(0xffffffffu, a[r], 1);
        a[r] += __shfl_xor_sync(0xffffffffu, a[r], 2);
    }
}

// Forward tiles: acc (thread (i, q): row i, columns 4(q + 4v) .. of each 64-column quarter)
// += Σ_{Q < nq} L[r0 + i, quarter Q]·y over the quarters of the blocks 0, 1, ...; quarter Q
// in ring slot Q & 3, three quarters in flight. yload(j) fills yb with y_j (all threads,
// starting with a barrier that ends the previous block's use of yb).
template <int R, typename YLoad>
__device__ __forceinline__ void fwd_tiles(double (&acc)[R], float* ring, double* yb, const float* prow, int64_t ldp,
                                          int64_t k, int nr, int nq, YLoad&& yload) {
    const int tid = threadIdx.x, i = tid >> 2, q = tid & 3;
    auto issue = [&](int Q) {
        const int64_t c0 = (int64_t)(Q >> 2) * WS + (Q & 3) * 64;
        const int ncol = (int)max((int64_t)0, min((int64_t)64, k - c0));
        if (ncol > 0 && nr > 0) cp_async_tile<float>(ring + (Q & 3) * CQ * FQP, FQP, prow + c0, ldp, nr, ncol, CQ, 64, CT);
        cp_async_commit();
    };
    for (int Q = 0; Q < min(3, nq); Q++) issue(Q);
    for (int Q = 0; Q < nq; Q++) {
        const int64_t j = Q >> 2;
        const int qq = Q & 3;
        if (qq == 0) yload(j);
        cp_wait_upto(min(2, nq - 1 - Q));
        __syncthreads();  // quarter Q and y_j visible; every thread is done with quarter Q − 1
        if (Q + 3 < nq) issue(Q + 3);
        if (j * WS + qq * 64 < k) {
            const float* Lt = ring + qq * CQ * FQP + i * FQP;
            const double* yq = yb + qq * 64 * R;
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const int c = 4 * (q + 4 * v);
                const float4 l = *reinterpret_cast<const float4*>(Lt + c);
#pragma unroll
                for (int r = 0; r < R; r++) {
                    acc[r] = fma((double)l.x, yq[c * R + r], acc[r]);
                    acc[r] = fma((double)l.y, yq[(c + 1) * R + r], acc[r]);
                    acc[r] = fma((double)l.z, yq[(c + 2) * R + r], acc[r]);
                    acc[r] = fma((double)l.w, yq[(c + 3) * R + r], acc[r]);
                }
            }
        }
    }
}

template <int R>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(CT, 1)
    k_chain_fwd(const double* __restrict__ X, double* __restrict__ Y, const float* __restrict__ panel,
                const double* __restrict__ cinv, const DFront* __restrict__ fr, const int64_t* __restrict__ chain_blk,
                const int64_t* __restrict__ items, int64_t nitems, int* __restrict__ flags, int* __restrict__ counter,
                int* __restrict__ err) {
    cg::cluster_group cluster = cg::this_cluster();
    const int s = (int)cluster.block_rank();
    extern __shared__ __align__(16) double sm[];
    double* Lv = sm;                                                   // [CQ][FLP]: inverse rows 64s ..
    float* ring = reinterpret_cast<float*>(sm + CQ * FLP);             // [4][CQ][FQP]: tile quarters
    double* yb = reinterpret_cast<double*>(ring + 4 * CQ * FQP);       // [WS][R]: y_J, then x_B
    double* xo = yb + WS * R;                                          // [CQ][R]: this CTA's rows of x_B
    __shared__ int64_t s_item;
    const int tid = threadIdx.x, i = tid >> 2, q = tid & 3;
    for (;;) {
        const int64_t it = grab(cluster, &s_item, counter);
        if (it >= nitems) break;
        const int64_t t = items[2 * it], b = items[2 * it + 1];
        const DFront f = fr[t];
        const int64_t cb0 = chain_blk[t];
        const int64_t r0 = b * WS + s * CQ;
        const int nr = (int)max((int64_t)0, min((int64_t)CQ, f.k - r0));
        const int cmax = CQ * (s + 1);  // inverse row 64s + i ends at the diagonal
        cp_async_tile<double>(Lv, FLP, cinv + ((cb0 + b) * WS + s * CQ) * (int64_t)WS, WS, CQ, cmax, CQ, cmax, CT);
        cp_async_commit();
        double acc[R];
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0.0;
        fwd_tiles<R>(acc, ring, yb, panel + f.poff + r0 * f.ldp, f.ldp, f.k, nr, 4 * (int)b, [&](int64_t j) {
            if (tid == 0) chain_wait(&flags[cb0 + j], CL, err);
            __syncthreads();
            const int wbj = (int)min((int64_t)WS, f.k - j * WS);
            const double* ys = Y + (f.start + j * WS) * R;
            for (int e = tid; e < WS * R; e += CT) yb[e] = e < wbj * R ? __ldcg(ys + e) : 0.0;
        });
        quad_sum<R>(acc);
        if (q == 0) {
#pragma unroll
            for (int r = 0; r < R; r++) xo[i * R + r] = i < nr ? X[(f.start + r0 + i) * R + r] - acc[r] : 0.0;
        }
        cluster.sync();
        for (int e = tid; e < WS * R; e += CT) {
            const int rk = e / (CQ * R);
            yb[e] = cluster.map_shared_rank(xo, rk)[e - rk * CQ * R];
        }
        cp_async_wait<0>();
        __syncthreads();
        double a[R];
#pragma unroll
        for (int r = 0; r < R; r++) a[r] = 0.0;
        for (int c = q; c < cmax; c += 4) {
            const double l = Lv[i * FLP + c];
#pragma unroll
            for (int r = 0; r < R; r++) a[r] = fma(l, yb[c * R + r], a[r]);
        }
        quad_sum<R>(a);
        if (q == 0 && i < nr) {
#pragma unroll
            for (int r = 0; r < R; r++) Y[(f.start + r0 + i) * R + r] = a[r];
        }
        chain_signal(&flags[cb0 + b]);
        cluster.sync();  // the cluster's x_B pieces may be overwritten after this
    }
}

// The later rows of a chain level's fronts after the level's chain: V[rows] −= L21·y over
// all the front's pivots, one CTA per CHAIN_PIECE rows.
template <int R>
__global__ void __launch_bounds__(CT) k_chain_rows(const double* __restrict__ Y, double* __restrict__ V,
                                                   const float* __restrict__ panel, const DFront* __restrict__ fr,
                                                   const int64_t* __restrict__ items) {
    extern __shared__ __align__(16) double sm[];
    float* ring = reinterpret_cast<float*>(sm);                   // [4][CQ][FQP]
    double* yb = reinterpret_cast<double*>(ring + 4 * CQ * FQP);  // [WS][R]
    const int tid = threadIdx.x, i = tid >> 2, q = tid & 3;
    const int64_t t = items[2 * blockIdx.x], c = items[2 * blockIdx.x + 1];
    const DFront f = fr[t];
    const int64_t r0 = f.k + c * CQ;
    const int nr = (int)min((int64_t)CQ, f.m - r0);
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = 0.0;
    fwd_tiles<R>(acc, ring, yb, panel + f.poff + r0 * f.ldp, f.ldp, f.k, nr, 4 * (int)((f.k + WS - 1) / WS),
                 [&](int64_t j) {
                     __syncthreads();
                     const int wbj = (int)min((int64_t)WS, f.k - j * WS);
                     const double* ys = Y + (f.start + j * WS) * R;
                     for (int e = tid; e < WS * R; e += CT) yb[e] = e < wbj * R ? ys[e] : 0.0;
                 });
    quad_sum<R>(acc);
    if (q == 0 && i < nr) {
        double* vt = V + (f.vuoff + c * CQ + i) * R;
#pragma unroll
        for (int r = 0; r < R; r++) vt[r] -= acc[r];
    }
}

// Backward chunks: acc (thread (c, g): column c, rows g, g + 4, ... of each 64-row chunk)
// += Σ_{h < nh} L[rows of chunk h, col0 + c]·y(rows); chunk h in ring slot h & 3, three in
// flight. rows_of(h, ra) gives the chunk's first row and row count; yload(h) runs before
// chunk h (all threads) and returns where the chunk's y values are in shared memory;
// issue_y(h) queues the chunk's y values with its tile (cp.async) when it can.
template <int R, typename Rows, typename YLoad, typename IssueY>
__device__ __forceinline__ void bwd_tiles(double (&acc)[R], float* ring, const float* pcol, int64_t ldp, int nc, int nh,
                                          Rows&& rows_of, YLoad&& yload, IssueY&& issue_y) {
    const int tid = threadIdx.x, c = tid & (CQ - 1), g = tid >> 6;
    auto issue = [&](int h) {
        int64_t ra;
        const int nrr = rows_of(h, ra);
        if (nrr > 0 && nc > 0)
            cp_async_tile<float>(ring + (h & 3) * CQ * BTP, BTP, pcol + ra * ldp, ldp, nrr, nc, CQ, CQ, CT);
        issue_y(h, ra, nrr);
        cp_async_commit();
    };
    for (int h = 0; h < min(3, nh); h++) issue(h);
    for (int h = 0; h < nh; h++) {
        int64_t ra;
        const int nrr = rows_of(h, ra);
        const double* yv = yload(h);
        cp_wait_upto(min(2, nh - 1 - h));
        __syncthreads();  // chunk h visible; every thread is done with chunk h − 1
        if (h + 3 < nh) issue(h + 3);
        if (nrr > 0) {
            const float* Lt = ring + (h & 3) * CQ * BTP + c;
#pragma unroll 4
            for (int u = 0; u < CQ / 4; u++) {
                const int rr = g + 4 * u;
                const double l = Lt[rr * BTP];
#pragma unroll
                for (int r = 0; r < R; r++) acc[r] = fma(l, yv[rr * R + r], acc[r]);
            }
        }
    }
}

// Σ over the four row groups of a column, in group order (threads tid < CQ get the total
// of column tid); red [4][CQ][R] in shared memory.
template <int R>
__device__ __forceinline__ void col_sum(double (&acc)[R], double* red) {
    const int tid = threadIdx.x, c = tid & (CQ - 1), g = tid >> 6;
#pragma unroll
    for (int r = 0; r < R; r++) red[(g * CQ + c) * R + r] = acc[r];
    __syncthreads();
    if (tid < CQ) {
#pragma unroll
        for (int r = 0; r < R; r++)
            acc[r] = ((red[c * R + r] + red[(CQ + c) * R + r]) + red[(2 * CQ + c) * R + r]) + red[(3 * CQ + c) * R + r];
    }
}

template <int R>
__global__ void __cluster_dims__(CL, 1, 1) __launch_bounds__(CT, 1)
    k_chain_bwd(double* __restrict__ Y, const float* __restrict__ panel, const double* __restrict__ cinv,
                const DFront* __restrict__ fr, const int64_t* __restrict__ chain_blk, const int64_t* __restrict__ items,
                int64_t nitems, int* __restrict__ flags, int* __restrict__ counter, int* __restrict__ err) {
    cg::cluster_group cluster = cg::this_cluster();
    const int s = (int)cluster.block_rank();
    extern __shared__ __align__(16) double sm[];
    double* Lc = sm;                                               // [WS][CQ]: rows 64s .. of inverse columns 64s ..
    float* ring = reinterpret_cast<float*>(sm + WS * CQ);          // [4][CQ][BTP]: tile chunks
    double* yp = reinterpret_cast<double*>(ring + 4 * CQ * BTP);   // [WS][R]: y of a later block; then z_B
    double* red = yp + WS * R;                                     // [4][CQ][R]
    double* zo = red + 4 * CQ * R;                                 // [CQ][R]: this CTA's columns of z_B
    __shared__ int64_t s_item;
    const int tid = threadIdx.x, c = tid & (CQ - 1), g = tid >> 6;
    for (;;) {
        const int64_t it = grab(cluster, &s_item, counter);
        if (it >= nitems) break;
        const int64_t t = items[2 * it], b = items[2 * it + 1];
        const DFront f = fr[t];
        const int64_t cb0 = chain_blk[t];
        const int64_t col0 = b * WS + s * CQ;
        const int nc = (int)max((int64_t)0, min((int64_t)CQ, f.k - col0));
        const int64_t nb = (f.k + WS - 1) / WS;
        const int ninv = WS - s * CQ;  // inverse column 64s + c starts at its diagonal row
        cp_async_tile<double>(Lc, CQ, cinv + ((cb0 + b) * WS + s * CQ) * (int64_t)WS + s * CQ, WS, ninv, CQ, ninv, CQ,
                              CT);
        cp_async_commit();
        double acc[R];
#pragma unroll
        for (int r = 0; r < R; r++) acc[r] = 0.0;
        // the chunks of blocks nb − 1, ..., b + 1, four per block
        bwd_tiles<R>(
            acc, ring, panel + f.poff + col0, f.ldp, nc, 4 * (int)(nb - 1 - b),
            [&](int h, int64_t& ra) -> int {
                ra = (nb - 1 - h / 4) * WS + (h & 3) * CQ;
                return (int)max((int64_t)0, min((int64_t)CQ, f.k - ra));
            },
            [&](int h) -> const double* {
                if ((h & 3) == 0) {
                    const int64_t bb = nb - 1 - h / 4;
                    if (tid == 0) chain_wait(&flags[cb0 + bb], CL, err);
                    __syncthreads();
                    const int wbb = (int)min((int64_t)WS, f.k - bb * WS);
                    const double* src = Y + (f.start + bb * WS) * R;
                    for (int e = tid; e < WS * R; e += CT) yp[e] = e < wbb * R ? __ldcg(src + e) : 0.0;
                }
                return yp + (h & 3) * CQ * R;
            },
            [](int, int64_t, int) {});
        col_sum<R>(acc, red);
        if (tid < CQ) {
#pragma unroll
            for (int r = 0; r < R; r++) zo[c * R + r] = c < nc ? Y[(f.start + col0 + c) * R + r] - acc[r] : 0.0;
        }
        cluster.sync();
        double* zf = yp;
        for (int e = tid; e < WS * R; e += CT) {
            const int rk = e / (CQ * R);
            zf[e] = cluster.map_shared_rank(zo, rk)[e - rk * CQ * R];
        }
        cp_async_wait<0>();
        __syncthreads();
        double a[R];
#pragma unroll
        for (int r = 0; r < R; r++) a[r] = 0.0;
        for (int rr = g; rr < ninv; rr += 4) {
            const double l = Lc[rr * CQ + c];
#pragma unroll
            for (int r = 0; r < R; r++) a[r] = fma(l, zf[(s * CQ + rr) * R + r], a[r]);
        }
        col_sum<R>(a, red);
        if (tid < nc) {
#pragma unroll
            for (int r = 0; r < R; r++) Y[(f.start + col0 + c) * R + r] = a[r];
        }
        chain_signal(&flags[cb0 + b]);
        cluster.sync();  // the cluster's z_B pieces may be overwritten after this
    }
}

// y of the later rows of a chain level's fronts into V (contiguous per front), before the
// level's backward: V[vuoff + i] = Y[rows[rows_off + i]], one CTA per CHAIN_PIECE rows.
__global__ void __launch_bounds__(CT) k_chain_gather(const double* __restrict__ Y, double* __restrict__ V,
                                                     const DFront* __restrict__ fr, const int64_t* __restrict__ rows,
                                                     const int64_t* __restrict__ items, int nrhs) {
    const int64_t t = items[2 * blockIdx.x], c = items[2 * blockIdx.x + 1];
    const DFront f = fr[t];
    const int64_t i0 = c * CQ;
    const int nr = (int)min((int64_t)CQ, f.u - i0);
    for (int e = threadIdx.x; e < nr * nrhs; e += CT) {
        const int ii = e / nrhs, r = e - ii * nrhs;
        V[(f.vuoff + i0 + ii) * nrhs + r] = Y[rows[f.rows_off + i0 + ii] * nrhs + r];
    }
}

// The later rows' part of a chain level's backward, before its chain: the partial sums
// L21ᵀ·y of the front's later rows (their y in V, from k_chain_gather), one CTA per
// CHAIN_PIECE pivot columns and group of rows (blockIdx.y of CHAIN_GROUPS), into
// part[(item · CHAIN_GROUPS + group) · CHAIN_PIECE + column]; k_chain_colsum subtracts them
// from z in group order.
template <int R>
__global__ void __launch_bounds__(CT) k_chain_cols(double* __restrict__ part, const double* __restrict__ V,
                                                   const float* __restrict__ panel, const DFront* __restrict__ fr,
                                                   const int64_t* __restrict__ items) {
    extern __shared__ __align__(16) double sm[];
    float* ring = reinterpret_cast<float*>(sm);                   // [4][CQ][BTP]
    double* ys = reinterpret_cast<double*>(ring + 4 * CQ * BTP);  // [4][CQ][R]: y of a chunk, by slot
    double* red = ys + 4 * CQ * R;                                // [4][CQ][R]
    const int tid = threadIdx.x, c = tid & (CQ - 1);
    const int64_t t = items[2 * blockIdx.x], cc = items[2 * blockIdx.x + 1];
    const DFront f = fr[t];
    const int64_t col0 = cc * CQ;
    const int nc = (int)min((int64_t)CQ, f.k - col0);
    const int nchunk = (int)((f.u + CQ - 1) / CQ), g = blockIdx.y;
    const int h0 = nchunk * g / CHAIN_GROUPS, h1 = nchunk * (g + 1) / CHAIN_GROUPS;
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; r++) acc[r] = 0.0;
    bwd_tiles<R>(
        acc, ring, panel + f.poff + col0, f.ldp, nc, h1 - h0,
        [&](int h, int64_t& ra) -> int {
            ra = f.k + (int64_t)(h0 + h) * CQ;
            return (int)min((int64_t)CQ, f.m - ra);
        },
        [&](int h) -> const double* { return ys + (h & 3) * CQ * R; },
        [&](int h, int64_t ra, int nrr) {
            if (tid < CQ * R) {
                const int rr = tid / R, r = tid - rr * R;
                double* dst = ys + ((h & 3) * CQ + rr) * R + r;
                if (rr < nrr)
                    cp_async8(dst, V + (f.vuoff + ra - f.k + rr) * R + r);
                else
                    *dst = 0.0;
            }
        });
    col_sum<R>(acc, red);
    if (tid < CQ) {
        double* out = part + (((int64_t)blockIdx.x * CHAIN_GROUPS + g) * CQ + c) * R;
#pragma unroll
        for (int r = 0; r < R; r++) out[r] = acc[r];
    }
}

// z[cols] −= the row groups' partial sums of k_chain_cols, added in group order.
__global__ void __launch_bounds__(CT) k_chain_colsum(double* __restrict__ Y, const double* __restrict__ part,
                                                     const DFront* __restrict__ fr, const int64_t* __restrict__ items,
                                                     int nrhs) {
    const int64_t t = items[2 * blockIdx.x], cc = items[2 * blockIdx.x + 1];
    const DFront f = fr[t];
    const int64_t col0 = cc * CQ;
    const int nc = (int)min((int64_t)CQ, f.k - col0);
    for (int e = threadIdx.x; e < nc * nrhs; e += CT) {
        const int c = e / nrhs, r = e - c * nrhs;
        double sum = 0.0;
        for (int g = 0; g < CHAIN_GROUPS; g++) sum += part[(((int64_t)blockIdx.x * CHAIN_GROUPS + g) * CQ + c) * nrhs + r];
        Y[(f.start + col0 + c) * nrhs + r] -= sum;
    }
}

// The inverse of a chain block's unit-lower diagonal block, by block columns of NB:
// M_jj = inv(L_jj) (from the factorization), M_ij = −inv(L_ii)·Σ_{j ≤ t < i} L_it·M_tj.
__global__ void __launch_bounds__(256) k_chain_inverse(double* __restrict__ cinv, const float* __restrict__ panel,
                                                       const double* __restrict__ linv, const DFront* __restrict__ fr,
                                                       const int64_t* __restrict__ chain_blk,
                                                       const int64_t* __restrict__ chain_bfront) {
    extern __shared__ __align__(16) double sm[];
    double(*A)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(sm);
    double(*B)[NB + 1] = A + NB;
    const int64_t cb = blockIdx.x, ft = chain_bfront[cb];
    const DFront f = fr[ft];
    const int64_t b = cb - chain_blk[ft], J0 = b * WS;
    const int wb = (int)min((int64_t)WS, f.k - J0), nbw = (wb + NB - 1) / NB;
    double* M = cinv + cb * (int64_t)WS * WS;
    const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
    for (int e = tid; e < WS * WS / 2; e += 256) reinterpret_cast<double2*>(M)[e] = make_double2(0.0, 0.0);
    __syncthreads();
    for (int j = 0; j < nbw; j++) {
        const double* li = linv + (f.blk_off + 4 * b + j) * (int64_t)(NB * NB);
        for (int e = tid; e < NB * NB; e += 256) M[(j * NB + e / NB) * WS + j * NB + e % NB] = li[e];
    }
    __syncthreads();
    auto gemm = [&](double (&acc)[4][4]) {
#pragma unroll 4
        for (int k = 0; k < NB; k++) {
            double av[4], bv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) av[u] = A[4 * ty + u][k];
#pragma unroll
            for (int v = 0; v < 4; v++) bv[v] = B[k][4 * tx + v];
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fma(av[u], bv[v], acc[u][v]);
        }
    };
    for (int j = 0; j + 1 < nbw; j++)
        for (int i = j + 1; i < nbw; i++) {
            double acc[4][4] = {};
            for (int tt = j; tt < i; tt++) {
                for (int e = tid; e < NB * NB; e += 256) {
                    const int r = e / NB, cc = e % NB, row = i * NB + r;
                    A[r][cc] = row < wb ? (double)panel[f.poff + (J0 + row) * f.ldp + J0 + tt * NB + cc] : 0.0;
                    B[r][cc] = __ldcg(&M[(tt * NB + r) * WS + j * NB + cc]);
                }
                __syncthreads();
                gemm(acc);
                __syncthreads();
            }
            // the sum becomes the right operand (B is free after the last product's barrier)
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) B[4 * ty + u][4 * tx + v] = acc[u][v];
            const double* li = linv + (f.blk_off + 4 * b + i) * (int64_t)(NB * NB);
            for (int e = tid; e < NB * NB; e += 256) A[e / NB][e % NB] = li[e];
            __syncthreads();
            double acc2[4][4] = {};
            gemm(acc2);
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) M[(i * NB + 4 * ty + u) * WS + j * NB + 4 * tx + v] = -acc2[u][v];
            __syncthreads();
        }
}

// per device: attributes set, the number of clusters that fit at once (forward, backward;
// by right-hand sides 1 .. 4)
struct ChainDev {
    bool done = false;
    int fwd[5] = {0, 0, 0, 0, 0}, bwd[5] = {0, 0, 0, 0, 0};
};

template <typename K>
int fit_clusters(K kern, size_t smem) {
    RFG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(CL * 64);
    cfg.blockDim = dim3(CT);
    cfg.dynamicSmemBytes = smem;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = CL;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    int n = 0;
    RFG_CUDA(cudaOccupancyMaxActiveClusters(&n, kern, &cfg));
    return n;
}

constexpr size_t rows_smem(int R) { return (size_t)4 * CQ * FQP * 4 + (size_t)WS * R * 8; }
constexpr size_t cols_smem(int R) { return (size_t)4 * CQ * BTP * 4 + (size_t)8 * CQ * R * 8; }

template <int R>
void set_piece_attrs() {
    RFG_CUDA(cudaFuncSetAttribute(k_chain_rows<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rows_smem(R)));
    RFG_CUDA(cudaFuncSetAttribute(k_chain_cols<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cols_smem(R)));
}

const ChainDev& chain_dev() {
    static std::mutex mu;
    static ChainDev devs[64];
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw CudaError("solve chain: device ordinal out of range");
    std::lock_guard<std::mutex> lock(mu);
    ChainDev& d = devs[dev];
    if (!d.done) {
        RFG_CUDA(cudaFuncSetAttribute(k_chain_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)INV_SMEM));
        d.fwd[1] = fit_clusters(k_chain_fwd<1>, fwd_smem(1));
        d.fwd[2] = fit_clusters(k_chain_fwd<2>, fwd_smem(2));
        d.fwd[3] = fit_clusters(k_chain_fwd<3>, fwd_smem(3));
        d.fwd[4] = fit_clusters(k_chain_fwd<4>, fwd_smem(4));
        d.bwd[1] = fit_clusters(k_chain_bwd<1>, bwd_smem(1));
        d.bwd[2] = fit_clusters(k_chain_bwd<2>, bwd_smem(2));
        d.bwd[3] = fit_clusters(k_chain_bwd<3>, bwd_smem(3));
        d.bwd[4] = fit_clusters(k_chain_bwd<4>, bwd_smem(4));
        set_piece_attrs<1>();
        set_piece_attrs<2>();
        set_piece_attrs<3>();
        set_piece_attrs<4>();
        d.done = true;
    }
    return d;
}

unsigned grid_for_items(int fit, int64_t nitems) {
    if (fit <= 0) throw CudaError("solve chain: no cluster of four CTAs fits on this device");
    return (unsigned)(std::min<int64_t>(fit, nitems) * CL);
}

void check_nrhs(int nrhs) {
    if (nrhs < 1 || nrhs > 4) throw CudaError("solve chain: 1 to 4 right-hand sides");
}

}  // namespace

void launch_chain_inverse(double* cinv, const float* panel, const double* linv, const DFront* fronts,
                          const int64_t* chain_blk, const int64_t* chain_bfront, int64_t nblocks, cudaStream_t st) {
    if (nblocks <= 0) return;
    chain_dev();
    k_chain_inverse<<<(unsigned)nblocks, 256, INV_SMEM, st>>>(cinv, panel, linv, fronts, chain_blk, chain_bfront);
    RFG_CUDA(cudaGetLastError());
}

// one of four instantiations by the number of right-hand sides
#define RFG_CHAIN_BY_R(nrhs, CALL) \
    do {                           \
        check_nrhs(nrhs);          \
        if ((nrhs) == 1) {         \
            constexpr int R = 1;   \
            CALL;                  \
        } else if ((nrhs) == 2) {  \
            constexpr int R = 2;   \
            CALL;                  \
        } else if ((nrhs) == 3) {  \
            constexpr int R = 3;   \
            CALL;                  \
        } else {                   \
            constexpr int R = 4;   \
            CALL;                  \
        }                          \
    } while (0)

void launch_chain_fwd(int nrhs, int64_t nitems, const double* X, double* Y, const float* panel, const double* cinv,
                      const DFront* fronts, const int64_t* chain_blk, const int64_t* items, int* flags, int* counter,
                      int* err, cudaStream_t st) {
    if (nitems <= 0) return;
    const ChainDev& d = chain_dev();
    RFG_CHAIN_BY_R(nrhs, (k_chain_fwd<R><<<grid_for_items(d.fwd[R], nitems), CT, fwd_smem(R), st>>>(
                              X, Y, panel, cinv, fronts, chain_blk, items, nitems, flags, counter, err)));
    RFG_CUDA(cudaGetLastError());
}

void launch_chain_rows(int nrhs, int64_t nitems, const double* Y, double* V, const float* panel, const DFront* fronts,
                       const int64_t* items, cudaStream_t st) {
    if (nitems <= 0) return;
    chain_dev();
    RFG_CHAIN_BY_R(nrhs, (k_chain_rows<R><<<(unsigned)nitems, CT, rows_smem(R), st>>>(Y, V, panel, fronts, items)));
    RFG_CUDA(cudaGetLastError());
}

void launch_chain_cols(int nrhs, int64_t ngather, const int64_t* gather_items, int64_t nitems, const int64_t* items,
                       double* Y, double* V, double* part, const float* panel, const DFront* fronts,
                       const int64_t* rows, cudaStream_t st) {
    if (nitems <= 0) return;
    chain_dev();
    check_nrhs(nrhs);
    if (ngather > 0) k_chain_gather<<<(unsigned)ngather, CT, 0, st>>>(Y, V, fronts, rows, gather_items, nrhs);
    RFG_CHAIN_BY_R(nrhs, (k_chain_cols<R><<<dim3((unsigned)nitems, CHAIN_GROUPS), CT, cols_smem(R), st>>>(
                              part, V, panel, fronts, items)));
    k_chain_colsum<<<(unsigned)nitems, CT, 0, st>>>(Y, part, fronts, items, nrhs);
    RFG_CUDA(cudaGetLastError());
}

void launch_chain_bwd(int nrhs, int64_t nitems, double* Y, const float* panel, const double* cinv,
                      const DFront* fronts, const int64_t* chain_blk, const int64_t* items, int* flags, int* counter,
                      int* err, cudaStream_t st) {
    if (nitems <= 0) return;
    const ChainDev& d = chain_dev();
    RFG_CHAIN_BY_R(nrhs, (k_chain_bwd<R><<<grid_for_items(d.bwd[R], nitems), CT, bwd_smem(R), st>>>(
                              Y, panel, cinv, fronts, chain_blk, items, nitems, flags, counter, err)));
    RFG_CUDA(cudaGetLastError());
}

#undef RFG_CHAIN_BY_R

}  // namespace rfg
