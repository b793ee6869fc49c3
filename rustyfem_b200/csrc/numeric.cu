// Numeric phase of the multifrontal LDLᵀ on the GPU (sm_100a).
//
// Level by level (see plan.h), each level of the elimination tree is
//   1. zero-filled (its panel range with one memset, its update blocks by kernel),
//   2. assembled: original entries stored into the panels (k_scatter), the
//      original diagonal captured for the pivot test (k_capture_diag), then the
//      children's update matrices added in child order (k_extend_add, one launch
//      per child rank, so no two CTAs add into the same entry),
//   3. factored in steps of NB pivots over all fronts of the level at once:
//        k_pivot_block  one CTA per front: blocked LDLᵀ of the NB×NB diagonal
//                       block in shared memory (FP64), with the reference's
//                       positive definite rule (src/sparse.rs:528-531), and the
//                       inverse of its unit-lower factor (for panels and solves);
//        k_panel        PR rows below the block per CTA, as a small GEMM with
//                       that inverse (FP64 tensor-core path): W = F·L⁻ᵀ,
//                       L = W·D⁻¹, plus the W and L operands of the Schur update
//                       in a scratch of NB-wide rows;
//        k_schur*       lower-triangular tiles of the trailing matrix,
//                       F −= W·Lᵀ (src/sparse.rs:559-573), written to the panel
//                       (pivot columns) or the update block (F22): in FP64 on the
//                       FP64 tensor-core path (mma.sync f64; k_schur_dmma64 for
//                       64-tiles, k_schur_dmma for the 128-tiles of large fronts),
//                       in the mixed path on tcgen05 (kernels_tc.cu) or, without
//                       tensor cores, on the CUDA cores (k_schur, k_schur_big).
// Storage T is double (FP64 path) or float (mixed path); pivot blocks are
// always factored in FP64 and the pivots D are kept in FP64.

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>

#include "engine.h"
#include "tc.cuh"
#include "tiles.cuh"

namespace rfg {

namespace {

// D = A·B + D on the FP64 tensor-core path for one 8×8×4 block (mma.sync m8n8k4 f64):
// lane l holds A[l / 4][l % 4], B[l % 4][l / 4] and D[l / 4][2·(l % 4) + {0, 1}].
__device__ __forceinline__ void dmma_884(double& c0, double& c1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

template <typename T>
__global__ void k_scatter(T* __restrict__ panel, const double* __restrict__ src, const int64_t* __restrict__ dst,
                          const int64_t* __restrict__ seg_ptr, const int64_t* __restrict__ seg_src, int64_t lo,
                          int64_t hi) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    for (int64_t i = lo + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < hi; i += (int64_t)gridDim.x * blockDim.x) {
        double s;
        if (seg_ptr) {
            s = 0.0;
            for (int64_t j = seg_ptr[i]; j < seg_ptr[i + 1]; j++) s += src[seg_src[j]];
        } else {
            s = src[seg_src[i]];
        }
        panel[dst[i]] = (T)s;
    }
}

template <typename T>
__global__ void k_capture_diag(const T* __restrict__ panel, double* __restrict__ adiag, const DFront* __restrict__ fr,
                               const int64_t* __restrict__ order, int64_t lo) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    const DFront f = fr[order[lo + blockIdx.x]];
    for (int64_t i = threadIdx.x; i < f.k; i += blockDim.x) adiag[f.start + i] = (double)panel[f.poff + i * f.ldp + i];
}

// zero the lower triangle of the update blocks of a level: warp w of block (i, y) clears
// rows 8y + w, 8y + w + 8·gridDim.y, ... of front order[lo + i], its lanes in 16-byte stores
// along the row (rows are 16-byte aligned and ldu ≥ ⌈u⌉₈, so rounding a row's length up
// stays inside the row); gridDim.y follows the level's largest update block
template <typename T>
__global__ void k_zero_update(T* __restrict__ upd, const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                              int64_t lo) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
    constexpr int VEC = 16 / (int)sizeof(T);
    const DFront f = fr[order[lo + blockIdx.x]];
    const V z{};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int64_t x = (int64_t)blockIdx.y * 8 + warp; x < f.u; x += (int64_t)gridDim.y * 8) {
        V* row = reinterpret_cast<V*>(upd + f.uoff + x * f.ldu);
        for (int64_t y = lane; y * VEC <= x; y += 32) row[y] = z;
    }
}

// F_parent[emap[x], emap[y]] += U_child[x, y] for y <= x, one launch per child rank. The
// child's lower triangle is cut into XT × XT tiles (tile rows by tile columns, row-major
// over the lower triangle), one warp per tile and eight tiles per CTA: lane l takes column
// Y0 + l of the tile's rows (the child row read as one 128-byte segment, the parent's
// column index once per tile, the parent rows of the tile's rows shuffled from one load),
// eight rows in flight before any store; no per-row pointers are held, so four CTAs fit
// on an SM. Child and parent
// never overlap, and no two lanes of a launch touch one entry.
template <typename T>
__global__ void __launch_bounds__(256, 4) k_extend_add(T* __restrict__ panel, T* __restrict__ upd,
                                                    const DFront* __restrict__ fr, const int64_t* __restrict__ child,
                                                    const int64_t* __restrict__ pre, int64_t nchild,
                                                    const int32_t* __restrict__ emap, int64_t* __restrict__ status) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    int64_t b = blockIdx.x;
    int64_t i = find_slot_warp(pre, nchild, b);
    int64_t c = child[i];
    int64_t chunk = b - pre[i];
    const DFront fc = fr[c];
    const DFront fp = fr[fc.parent];
    if (status[c] != -1) {
        if (chunk == 0 && threadIdx.x == 0) status[fc.parent] = -2;  // an ancestor of a failed front
        return;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t nt = (fc.u + XT - 1) / XT;
    const int64_t lt = chunk * 8 + warp;
    if (lt >= nt * (nt + 1) / 2) return;
    int64_t ti = (int64_t)((sqrt(8.0 * (double)lt + 1.0) - 1.0) * 0.5);
    while (ti * (ti + 1) / 2 > lt) ti--;
    while ((ti + 1) * (ti + 2) / 2 <= lt) ti++;
    const int64_t tj = lt - ti * (ti + 1) / 2;
    const int32_t* em = emap + fc.emap_off;
    const int64_t y = tj * XT + lane;
    const int64_t py = y < fc.u ? em[y] : -1;
    const int64_t X0 = ti * XT, X1 = min(fc.u, X0 + XT);
    // the parent rows of the tile's rows, one per lane, handed out by shuffles: the
    // parent's loads do not wait for a load of the map
    const int32_t emx = X0 + lane < X1 ? em[X0 + lane] : 0;
    // this lane's parent column: in a panel row (column py) or in an update-block row
    // (column py − k); a parent row px starts at pcol + (px − pshift)·pld
    const bool in_panel = py < fp.k;
    T* const pcol = in_panel ? panel + fp.poff + py : upd + fp.uoff + (py - fp.k);
    const int64_t pld = in_panel ? fp.ldp : fp.ldu, pshift = in_panel ? 0 : fp.k;
    const T* ucol = upd + fc.uoff + y;
    constexpr int U = 8;
    for (int64_t x0 = X0; x0 < X1; x0 += U) {
        T v[U], old[U];
        uint32_t okm = 0;  // bit u: row x0 + u is added by this lane
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t x = x0 + u;
            const bool ok = x < X1 && py >= 0 && y <= x;
            okm |= (uint32_t)ok << u;
            v[u] = ok ? ucol[x * fc.ldu] : T(0);
        }
        // the parent row offsets are shuffled again for the loads and for the stores
        // instead of being held in registers across them
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t px = __shfl_sync(0xffffffffu, emx, (int)(x0 + u - X0) & (XT - 1));
            old[u] = (okm >> u) & 1u ? pcol[(px - pshift) * pld] : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            const int64_t px = __shfl_sync(0xffffffffu, emx, (int)(x0 + u - X0) & (XT - 1));
            if ((okm >> u) & 1u) pcol[(px - pshift) * pld] = old[u] + v[u];
        }
    }
}

// LDLᵀ of the NB×NB diagonal block [j0, j1) of each active front in FP64 shared memory,
// with the inverse of its unit lower factor (stored as a full NB×NB block, identity
// beyond jb) for the panels and the solves. One CTA of PBT threads per front.
//
// The block is factored in four sub-panels of SB = 16 pivots. A sub-panel is factored
// by at most three warps with one row per lane (lanes 0..15 the diagonal sub-block, which
// every such warp computes, lanes 16..31 sixteen rows below it); within a warp the pivot
// column is passed through shared memory, so the 16 pivots take no CTA barrier. The
// sub-panel's rank-16 update of the trailing block is split: its update of the next
// sub-panel's columns (look-ahead) is applied by all threads right away, the rest by
// warps 3..7 while the next sub-panel is factored, together with the inverse of the
// finished diagonal sub-block and the block row of the inverse below it:
//     X_pp = L_pp⁻¹,   X[p, :p] = −X_pp·(L[p, :p]·X[:p, :p]).
// This is the factorization of the reference's diagonal block (row by row there,
// src/sparse.rs:516-537) with the same sums taken in another order; the pivot test
// (src/sparse.rs:528-531) runs on every pivot in order and stops the front at the first
// failure, recording that equation.
constexpr int PBT = 256;  // threads of the pivot-block kernel
constexpr int SB = 16;    // pivots per sub-panel

// X_pp = L_pp⁻¹ of the SB×SB diagonal sub-block at cp, one column c per lane:
// x_r = −Σ_{q<r} L[r][q]·x_q; lanes c ≥ SB store nothing.
__device__ __forceinline__ void pb_diag_inverse(const double (*A)[NB + 1], double (*X)[NB + 1], int cp, int c) {
    double xv[SB];
#pragma unroll
    for (int r = 0; r < SB; r++) xv[r] = (r == c) ? 1.0 : 0.0;
#pragma unroll
    for (int r = 1; r < SB; r++) {
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int q = 0; q < r; q++) {
            const double lq = A[cp + r][cp + q];
            if (q & 1)
                s1 -= lq * xv[q];
            else
                s0 -= lq * xv[q];
        }
        if (r > c) xv[r] = s0 + s1;
    }
    if (c < SB) {
#pragma unroll
        for (int r = 0; r < SB; r++)
            if (r >= c) X[cp + r][cp + c] = xv[r];
    }
}

// Work of warps 3..7 (160 threads) for the finished sub-panel p while sub-panel p+1 is
// factored: warp 3 inverts the diagonal sub-block; warps 4..7 apply the rest of the
// sub-panel's trailing update (rows/cols from cp + 2·SB, when a later sub-panel needs it)
// and Y = −L[p, :p]·X[:p, :p] (X is lower triangular, zero above the diagonal); then all
// five form X[p, :p] = X_pp·Y.
__device__ __forceinline__ void pb_group(double (*A)[NB + 1], double (*X)[NB + 1], const double (*Wq)[SB + 1],
                                         double (*Y)[NB - SB + 1], int p, bool rest) {
    const int gt = threadIdx.x - 96;
    const int cp = p * SB;
    if (gt < 32) {
        pb_diag_inverse(A, X, cp, gt);
    } else {
        const int g4 = gt - 32;  // 0..127
        if (rest) {
            const int base = cp + 2 * SB, T = NB - base;
            const int ty = g4 >> 3, tx = g4 & 7;
            if (T == 32) {
                double acc[2][4];
#pragma unroll
                for (int i = 0; i < 2; i++)
#pragma unroll
                    for (int k = 0; k < 4; k++) acc[i][k] = A[base + ty + 16 * i][base + tx + 8 * k];
#pragma unroll 4
                for (int q = 0; q < SB; q++) {
                    double w[2], lv[4];
#pragma unroll
                    for (int i = 0; i < 2; i++) w[i] = Wq[base + ty + 16 * i][q];
#pragma unroll
                    for (int k = 0; k < 4; k++) lv[k] = A[base + tx + 8 * k][cp + q];
#pragma unroll
                    for (int i = 0; i < 2; i++)
#pragma unroll
                        for (int k = 0; k < 4; k++) acc[i][k] -= w[i] * lv[k];
                }
#pragma unroll
                for (int i = 0; i < 2; i++)
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        if (ty + 16 * i >= tx + 8 * k) A[base + ty + 16 * i][base + tx + 8 * k] = acc[i][k];
            } else if (T == 16) {
                double acc[2];
#pragma unroll
                for (int k = 0; k < 2; k++) acc[k] = A[base + ty][base + tx + 8 * k];
#pragma unroll 4
                for (int q = 0; q < SB; q++) {
                    const double w = Wq[base + ty][q];
#pragma unroll
                    for (int k = 0; k < 2; k++) acc[k] -= w * A[base + tx + 8 * k][cp + q];
                }
#pragma unroll
                for (int k = 0; k < 2; k++)
                    if (ty >= tx + 8 * k) A[base + ty][base + tx + 8 * k] = acc[k];
            }
        }
        if (p > 0) {
            const int rr = g4 & 15, cg = g4 >> 4;  // columns cg + 8m
            double acc[6][2];
#pragma unroll
            for (int m = 0; m < 6; m++) acc[m][0] = acc[m][1] = 0.0;
            for (int q = 0; q < cp; q += 2) {
                const double l0 = A[cp + rr][q], l1 = A[cp + rr][q + 1];
#pragma unroll
                for (int m = 0; m < 6; m++)
                    if (8 * m < cp) {
                        acc[m][0] -= l0 * X[q][cg + 8 * m];
                        acc[m][1] -= l1 * X[q + 1][cg + 8 * m];
                    }
            }
#pragma unroll
            for (int m = 0; m < 6; m++)
                if (8 * m < cp) Y[rr][cg + 8 * m] = acc[m][0] + acc[m][1];
        }
    }
    asm volatile("bar.sync 1, 160;" ::: "memory");  // warps 3..7 only
    if (p > 0) {
        for (int idx = gt; idx < SB * cp; idx += 160) {
            const int rr = idx & 15, c = idx >> 4;
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int q = 0; q < SB; q += 2) {
                s0 += X[cp + rr][cp + q] * Y[q][c];
                s1 += X[cp + rr][cp + q + 1] * Y[q + 1][c];
            }
            X[cp + rr][c] = s0 + s1;
        }
    }
}

// The last sub-panel's block row of the inverse, with the whole CTA: warp 0 the diagonal
// sub-block, warps 2..7 Y (four columns cg + 12m each), then X[p, :p] = X_pp·Y.
__device__ __forceinline__ void pb_final(const double (*A)[NB + 1], double (*X)[NB + 1], double (*Y)[NB - SB + 1],
                                         int p) {
    const int cp = p * SB;
    if (threadIdx.x < 32) {
        pb_diag_inverse(A, X, cp, threadIdx.x);
    } else if (threadIdx.x >= 64 && p > 0) {
        const int g = threadIdx.x - 64, rr = g & 15, cg = g >> 4;
        double acc[4] = {0.0, 0.0, 0.0, 0.0};
        for (int q = 0; q < cp; q++) {
            const double l = A[cp + rr][q];
#pragma unroll
            for (int m = 0; m < 4; m++)
                if (12 * m < cp) acc[m] -= l * X[q][cg + 12 * m];
        }
#pragma unroll
        for (int m = 0; m < 4; m++)
            if (cg + 12 * m < cp) Y[rr][cg + 12 * m] = acc[m];
    }
    __syncthreads();
    if (p > 0) {
        for (int idx = threadIdx.x; idx < SB * cp; idx += PBT) {
            const int rr = idx & 15, c = idx >> 4;
            double s0 = 0.0, s1 = 0.0;
#pragma unroll
            for (int q = 0; q < SB; q += 2) {
                s0 += X[cp + rr][cp + q] * Y[q][c];
                s1 += X[cp + rr][cp + q + 1] * Y[q + 1][c];
            }
            X[cp + rr][c] = s0 + s1;
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(PBT, 2) k_pivot_block(T* __restrict__ panel, double* __restrict__ d,
                                                        const double* __restrict__ adiag,
                                                        const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                        int64_t fr_off, int64_t s, int64_t* __restrict__ status,
                                                        double* __restrict__ linv) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    extern __shared__ double pb_smem[];
    double(*A)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(pb_smem);
    double(*X)[NB + 1] = reinterpret_cast<double(*)[NB + 1]>(pb_smem + NB * (NB + 1));
    __shared__ double Wp[2][NB][SB + 1];        // unscaled W = L·D of the last two sub-panels
    __shared__ double Y[SB][NB - SB + 1];       // a block row of the inverse before X_pp
    __shared__ __align__(16) double colbuf[3][2][SB];  // pivot column of the sub-panel warps
    __shared__ double orig[NB];
    __shared__ int failed;
    const int64_t t = order[fr_off + blockIdx.x];
    if (status[t] != -1) return;
    const DFront f = fr[t];
    const int64_t j0 = s * NB;
    const int jb = (int)min((int64_t)NB, f.k - j0);
    T* blk = panel + f.poff + j0 * f.ldp + j0;
    {
        // each thread loads EPT consecutive entries of one row (all issued before any
        // store); rows beyond jb get a unit diagonal so the sub-panels need no bounds
        constexpr int EPT = NB * NB / PBT, TPR = NB / EPT;
        const int r = threadIdx.x / TPR, c0 = (threadIdx.x % TPR) * EPT;
        T v[EPT];
#pragma unroll
        for (int e = 0; e < EPT; e++) {
            const int c = c0 + e;
            v[e] = (r < jb && c <= r) ? blk[(int64_t)r * f.ldp + c] : T(0);
        }
#pragma unroll
        for (int e = 0; e < EPT; e++) {
            const int c = c0 + e;
            A[r][c] = (r >= jb && c == r) ? 1.0 : (double)v[e];
            X[r][c] = (r == c) ? 1.0 : 0.0;
        }
    }
    for (int p = threadIdx.x; p < jb; p += blockDim.x) orig[p] = adiag[f.start + j0 + p];
    if (threadIdx.x == 0) failed = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nsub = (jb + SB - 1) / SB;
    for (int b = 0; b < nsub; b++) {
        const int c0 = b * SB;
        const int nbelow = NB - c0 - SB;
        const int nw = nbelow > 0 ? (nbelow + 15) / 16 : 1;
        if (warp < nw) {
            const bool dlane = lane < SB;
            const int r = dlane ? c0 + lane : c0 + SB + warp * 16 + (lane - 16);
            const bool live = r < NB;
            double(*Wb)[SB + 1] = Wp[b & 1];
            double a[SB];  // row r, columns c0 .. c0+SB−1
#pragma unroll
            for (int c = 0; c < SB; c++) a[c] = live ? A[r][c0 + c] : 0.0;
#pragma unroll
            for (int jj = 0; jj < SB; jj++) {
                // column jj of the diagonal sub-block (final after pivot jj−1) to every
                // lane; two buffers by parity, so one __syncwarp per pivot suffices
                double* cb = colbuf[warp][jj & 1];
                if (dlane && lane >= jj) cb[lane] = a[jj];
                __syncwarp();
                double acj[SB];
#pragma unroll
                for (int c = jj & ~1; c < SB; c += 2) {
                    const double2 v = *reinterpret_cast<const double2*>(cb + c);
                    acj[c] = v.x;
                    acj[c + 1] = v.y;
                }
                const double piv = acj[jj];
                const int j = c0 + jj;
                if (j < jb && (!(orig[j] > 0.0) || !(piv > 1e-12 * orig[j]))) {
                    if (warp == 0 && lane == 0) {
                        failed = 1;
                        status[t] = f.start + j0 + j;
                    }
                    break;
                }
                if (warp == 0 && lane == jj && j < jb) d[f.start + j0 + j] = piv;
                const double l = a[jj] * recip_newton(piv);  // piv > 0, tested above
                if (!dlane || lane > jj) {
#pragma unroll
                    for (int c = jj + 1; c < SB; c++) a[c] -= l * acj[c];
                    if (live) Wb[r][jj] = a[jj];
                    a[jj] = l;
                }
            }
            if (live && (!dlane || warp == 0)) {
#pragma unroll
                for (int c = 0; c < SB; c++)
                    if (!dlane || c <= lane) A[r][c0 + c] = a[c];
            }
        } else if (warp >= 3 && b > 0) {
            pb_group(A, X, Wp[(b - 1) & 1], Y, b - 1, b + 1 < nsub);
        }
        __syncthreads();
        if (failed) return;
        if (b + 1 < nsub) {
            // look-ahead: this sub-panel's update of the next sub-panel's columns
            const int cn = c0 + SB, R = NB - cn;
            const int cc = threadIdx.x & 15, rg = threadIdx.x >> 4;
            const int c = cn + cc;
            const double(*Wb)[SB + 1] = Wp[b & 1];
            double lv[SB];
#pragma unroll
            for (int q = 0; q < SB; q++) lv[q] = A[c][c0 + q];
#pragma unroll
            for (int i = 0; i < 3; i++) {
                const int r = cn + rg + 16 * i;
                if (16 * i < R && r >= c) {
                    double s0 = A[r][c], s1 = 0.0;
#pragma unroll
                    for (int q = 0; q < SB; q += 2) {
                        s0 -= Wb[r][q] * lv[q];
                        s1 -= Wb[r][q + 1] * lv[q + 1];
                    }
                    A[r][c] = s0 + s1;
                }
            }
        }
        __syncthreads();
    }
    pb_final(A, X, Y, nsub - 1);
    __syncthreads();
    {
        constexpr int EPT = NB * NB / PBT, TPR = NB / EPT;
        const int r = threadIdx.x / TPR, c0 = (threadIdx.x % TPR) * EPT;
        if (r < jb)
#pragma unroll
            for (int e = 0; e < EPT; e++) {
                const int c = c0 + e;
                if (c <= r) blk[(int64_t)r * f.ldp + c] = (T)A[r][c];
            }
    }
    double* out = linv + (f.blk_off + s) * (int64_t)(NB * NB);
    for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) out[idx] = X[idx / NB][idx % NB];
}

// Panel of one step as a small GEMM against the inverse of the diagonal block stored by
// k_pivot_block: for the PR rows r in [j1, m) of a CTA,
//     W[r, :] = F[r, j0:j1]·L_bb⁻ᵀ,   L[r, :] = W[r, :]·D⁻¹
// (the forward substitution w ← w·L⁻ᵀ of src/sparse.rs:547-558, applied as a product).
// L goes to the panel; W and L to the outer block's scratch (front row r is scratch
// row pre_scr[i] + r − J0, columns j0 − J0 ..); in the tensor-core path also their TF32
// head and tail. 256 threads; the products run on the FP64 tensor-core path (8 warps of
// 32 rows × 32 columns, mma.sync m8n8k4 f64) from shared tiles with a row pitch of
// PNP = NB + 4 doubles (the fragment loads, 8 rows × 4 columns per warp, hit distinct
// banks in each half-warp); FP64 arithmetic in both precisions.
constexpr int PNP = NB + 4;
constexpr size_t PANEL_SMEM = (PR + NB) * PNP * sizeof(double) + NB * sizeof(double) +
                              NB * sizeof(double) + PR * sizeof(float);  // + FP16 split: D^(1/2) (FP32), row scales
constexpr size_t PANEL_SMEM_D = PANEL_SMEM + NB * PNP * sizeof(double);  // FP64: + L_bb

// acc[a][c] (+)= ±A·Bᵀ for the warp's 32×32 outputs (rows 32·wm + 8a + g, columns
// 32·wn + 8c + 2q + {0, 1}), A = [PR][PNP] and B = [NB][PNP] in shared memory, over the
// columns [0, 4·ksteps) of both.
template <bool NEG>
__device__ __forceinline__ void panel_mma(double (&acc)[4][4][2], const double* A, const double* B, int ksteps,
                                          int wm, int wn, int g, int q) {
    const double* a0 = A + (wm * 32 + g) * PNP + q;
    const double* b0 = B + (wn * 32 + g) * PNP + q;
#pragma unroll 4
    for (int k = 0; k < 4 * ksteps; k += 4) {
        double fa[4], fb[4];
#pragma unroll
        for (int a = 0; a < 4; a++) fa[a] = NEG ? -a0[a * 8 * PNP + k] : a0[a * 8 * PNP + k];
#pragma unroll
        for (int c = 0; c < 4; c++) fb[c] = b0[c * 8 * PNP + k];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 4; c++) dmma_884(acc[a][c][0], acc[a][c][1], fa[a], fb[c]);
    }
}

// The warp's accumulators into the shared tile (columns >= jb as zero).
__device__ __forceinline__ void panel_store(double* Fs, const double (&acc)[4][4][2], int jb, int wm, int wn, int g,
                                            int q) {
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++)
#pragma unroll
            for (int e = 0; e < 2; e++) {
                const int col = wn * 32 + c * 8 + 2 * q + e;
                Fs[(wm * 32 + a * 8 + g) * PNP + col] = col < jb ? acc[a][c][e] : 0.0;
            }
}

// FP16 split of the tensor-core update: the power-of-two scale of a row of U = L·D^(1/2)
// from the row's diagonal a_rr in the original matrix. Every Schur complement of a
// positive definite matrix has its diagonal below the original one and U[r, p]² is at
// most the diagonal of row r in the Schur complement that eliminates p, so
// |U[r, p]| ≤ a_rr^(1/2) and the scaled row stays below 2^12, far inside the FP16 range
// (65504). 0 for a diagonal that is not positive and finite.
__device__ __forceinline__ float u16_row_scale(double arr) {
    if (!(arr > 0.0) || !(arr < INFINITY)) return 0.f;
    int e;
    frexp(sqrt(arr), &e);  // sqrt(a_rr) < 2^e
    return (float)ldexp(1.0, 12 - e);
}

// Rows of a panel CTA after its loads: W = F·L_bb⁻ᵀ over the jb pivots (FP64 panels add
// one refinement step against L_bb), L = W·D⁻¹, stores: L into the panel, and as the
// plan's mode says, W and L rows in the storage precision (PANEL_SCR) and the split
// operands of the tensor cores (PANEL_SPLIT): the TF32 heads and tails of W and L (whi
// non-null) or the FP16 head and tail of U·s_r = L·D^(1/2)·s_r (uhi non-null; usq the
// step's D^(1/2) in FP32, rsc the rows' scales s_r, powers of two). U is formed in FP32 from L
// as stored (one FP64 → FP32 conversion per entry for L and U together: the conversions, not
// the products, bound these stores). A scaled U entry outside the FP16 range sets *err = 21.
template <typename T, typename S>
__device__ __forceinline__ void panel_rows(T* __restrict__ panel, const DFront& f, double* Fs, const double* Li,
                                           const double* dinv, double* pnl_smem, int64_t r0, int nr, int jb,
                                           int64_t j0, int64_t J0, int64_t scr0, S* __restrict__ scr_w,
                                           S* __restrict__ scr_l, float* __restrict__ whi, float* __restrict__ wlo,
                                           float* __restrict__ lhi, float* __restrict__ llo, bool scr,
                                           __half* __restrict__ uhi, __half* __restrict__ ulo, const float* usq,
                                           const float* rsc, int* __restrict__ err) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int wm = warp & 3, wn = warp >> 2;
    const bool busy = wm * 32 < nr;  // warps whose rows are all past the chunk's end idle
    const int ksteps = (jb + 3) / 4;
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c][0] = acc[a][c][1] = 0.0;
    if constexpr (sizeof(T) == sizeof(double)) {
        // FP64 panels: one refinement step against the triangular system itself,
        // R = F − W·L_bbᵀ, W += R·L⁻ᵀ, so that W matches forward substitution to
        // rounding even when the product with the explicit inverse loses digits
        double* Lb = pnl_smem + (PR + NB) * PNP + NB;
        const T* blk = panel + f.poff + j0 * f.ldp + j0;
        for (int idx = threadIdx.x; idx < NB * NB; idx += blockDim.x) {
            const int p = idx / NB, c = idx - p * NB;
            Lb[p * PNP + c] = (p < jb && c < p) ? (double)blk[(int64_t)p * f.ldp + c] : (p == c ? 1.0 : 0.0);
        }
        double rv[4][4][2];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 4; c++)
#pragma unroll
                for (int e = 0; e < 2; e++) rv[a][c][e] = Fs[(wm * 32 + a * 8 + g) * PNP + wn * 32 + c * 8 + 2 * q + e];
        if (busy) panel_mma<false>(acc, Fs, Li, ksteps, wm, wn, g, q);
        __syncthreads();  // every warp has read F (and Lb is in)
        panel_store(Fs, acc, jb, wm, wn, g, q);
        __syncthreads();
        if (busy) panel_mma<true>(rv, Fs, Lb, ksteps, wm, wn, g, q);
        __syncthreads();
        panel_store(Fs, rv, jb, wm, wn, g, q);
        __syncthreads();
        if (busy) panel_mma<false>(acc, Fs, Li, ksteps, wm, wn, g, q);
    } else {
        if (busy) panel_mma<false>(acc, Fs, Li, ksteps, wm, wn, g, q);
    }
    __syncthreads();
    panel_store(Fs, acc, jb, wm, wn, g, q);
    __syncthreads();
    // stores: 16 consecutive columns per half-warp row
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
#pragma unroll
    for (int a = 0; a < PR / 16; a++) {
        const int rr = ty + 16 * a;
        if (rr >= nr) continue;
        const int64_t r = r0 + rr;
        const int64_t so = (scr0 + (r - J0)) * NBO + (j0 - J0);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int p = tx + 16 * c;
            const double w = Fs[rr * PNP + p], l = w * dinv[p];
            const T lt = (T)l;
            if (p < jb) panel[f.poff + r * f.ldp + j0 + p] = lt;
            if (scr) {
                scr_w[so + p] = (S)w;
                scr_l[so + p] = (S)l;
            }
            if (whi) {
                float wf = (float)w, lf = (float)l;
                float wh = tc::to_tf32(wf), lh = tc::to_tf32(lf);
                whi[so + p] = wh;
                wlo[so + p] = tc::to_tf32(wf - wh);
                lhi[so + p] = lh;
                llo[so + p] = tc::to_tf32(lf - lh);
            }
            if (uhi) {
                const float u = (float)lt * usq[p] * rsc[rr];
                const __half h = __float2half_rn(u);
                uhi[so + p] = h;
                ulo[so + p] = __float2half_rn(u - __half2float(h));
                if (!(fabsf(u) < 65504.f)) atomicExch(err, 21);
            }
        }
    }
}

template <typename T, typename S>
__global__ void __launch_bounds__(256) k_panel(T* __restrict__ panel, const double* __restrict__ d,
                                               const double* __restrict__ linv, const DFront* __restrict__ fr,
                                               const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                               const int64_t* __restrict__ pre_panel, const int64_t* __restrict__ pre_scr,
                                               int64_t s, S* __restrict__ scr_w, S* __restrict__ scr_l,
                                               const int64_t* __restrict__ status, float* __restrict__ whi,
                                               float* __restrict__ wlo, float* __restrict__ lhi, float* __restrict__ llo,
                                               const uint8_t* __restrict__ mode, const int64_t* __restrict__ rows,
                                               const double* __restrict__ adiag0, __half* __restrict__ uhi,
                                               __half* __restrict__ ulo, float* __restrict__ uscale,
                                               int* __restrict__ err) {
    extern __shared__ double pnl_smem[];
    double* Fs = pnl_smem;                // [PR][PNP]
    double* Li = pnl_smem + PR * PNP;     // [NB][PNP]
    double* dinv = pnl_smem + (PR + NB) * PNP;
    int64_t b = blockIdx.x;
    int64_t i = find_slot_warp(pre_panel, nact, b);
    int64_t chunk = b - pre_panel[i];
    int64_t t = order[fr_off + i];
    const DFront f = fr[t];
    int64_t j0 = s * NB;
    int jb = (int)min((int64_t)NB, f.k - j0);
    int64_t j1 = j0 + jb;
    int64_t J0 = (s / KO) * NBO;
    int64_t r0 = j1 + chunk * PR;
    int nr = (int)min((int64_t)PR, f.m - r0);
    // the chunk's rows of the step's columns are final once the update kernel before the
    // pivot kernel has completed, which the pivot kernel waited for before it let this
    // kernel start (programmatic launch): they are loaded while the pivot block is factored
    load_tile_p<T, PR, 256, PNP>(Fs, panel + f.poff + r0 * f.ldp + j0, f.ldp, nr, jb);
    // the scratch rows and the split operands only where an update reads them
    const uint8_t md = mode[i];
    if (!(md & PANEL_SPLIT)) {
        whi = nullptr;
        uhi = nullptr;
    }
    float* usq = reinterpret_cast<float*>(pnl_smem + (PR + NB) * PNP + NB);
    float* rsc = reinterpret_cast<float*>(pnl_smem + (PR + NB) * PNP + 2 * NB);
    if (sizeof(T) == sizeof(float) && uhi) {
        // the rows' scales from their original diagonal (known since the assembly), also
        // kept per scratch row for the tensor-core epilogue: while the pivot block runs
        const int64_t sr0 = pre_scr[i] + (r0 - J0);
        for (int rr = threadIdx.x; rr < nr; rr += blockDim.x) {
            const int64_t r = r0 + rr;
            const int64_t q = r < f.k ? f.start + r : rows[f.rows_off + r - f.k];
            const float sc = u16_row_scale(adiag0[q]);
            if (sc == 0.f) atomicExch(err, 21);
            uscale[sr0 + rr] = sc;
            rsc[rr] = sc;
        }
    }
    pdl_wait();
    pdl_launch_dependents();
    if (status[t] != -1) return;
    load_linv_p<256, PNP>(Li, linv + (f.blk_off + s) * (int64_t)(NB * NB));
    for (int p = threadIdx.x; p < NB; p += blockDim.x) dinv[p] = p < jb ? 1.0 / d[f.start + j0 + p] : 0.0;
    if (sizeof(T) == sizeof(float) && uhi)
        for (int p = threadIdx.x; p < NB; p += blockDim.x) usq[p] = p < jb ? (float)sqrt(d[f.start + j0 + p]) : 0.f;
    __syncthreads();
    panel_rows<T, S>(panel, f, Fs, Li, dinv, pnl_smem, r0, nr, jb, j0, J0, pre_scr[i], scr_w, scr_l, whi, wlo, lhi,
                     llo, (md & PANEL_SCR) != 0, uhi, ulo, usq, rsc, err);
}

// Tile lt of a step's update on the UT×UT grid, with the pivots it applies (kofs, klen:
// offset and count in the outer block's scratch rows):
//   inner (OUTER = false): rows [j1, m), columns [j1, J1e), the step's pivots [j0, j1);
//   outer (OUTER = true):  rows [J1e, m), columns [J1e, k) (panel) and [k, m) (update
//                          block), the outer block's pivots [J0, J1e).
// The panel part's lower-triangular tiles come first (column by column, rows from the
// diagonal tile down), then the lower triangle of the update block.
struct SmallTile {
    int64_t row0, col0, col_end, kofs, klen;
    bool in_panel;
};
template <bool OUTER>
__device__ __forceinline__ SmallTile small_tile(const DFront& f, int64_t s, int64_t lt) {
    const int64_t j0 = s * NB;
    const int64_t j1 = min(j0 + NB, f.k);
    const int64_t J0 = (s / KO) * NBO;
    const int64_t J1e = min(J0 + NBO, f.k);
    const int64_t rbase = OUTER ? J1e : j1;
    const int64_t pcol_end = OUTER ? f.k : J1e;
    SmallTile b;
    b.kofs = OUTER ? 0 : j0 - J0;
    b.klen = OUTER ? J1e - J0 : j1 - j0;
    const int64_t R = f.m - rbase;
    const int64_t nrt = (R + UT - 1) / UT, ncp = (pcol_end - rbase + UT - 1) / UT;
    const int64_t cntP = ncp * nrt - ncp * (ncp - 1) / 2;
    if (lt < cntP) {
        int64_t tj = 0, cnt = nrt;
        while (lt >= cnt) {
            lt -= cnt;
            tj++;
            cnt = nrt - tj;
        }
        b.row0 = rbase + (tj + lt) * UT;
        b.col0 = rbase + tj * UT;
        b.col_end = pcol_end;
        b.in_panel = true;
    } else {
        const int64_t idx = lt - cntP;
        int64_t ti = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
        while (ti * (ti + 1) / 2 > idx) ti--;
        while ((ti + 1) * (ti + 2) / 2 <= idx) ti++;
        const int64_t tj = idx - ti * (ti + 1) / 2;
        b.row0 = f.k + ti * UT;
        b.col0 = f.k + tj * UT;
        b.col_end = f.m;
        b.in_panel = false;
    }
    return b;
}

// Schur update F[r, c] −= Σ_p W[r, p]·L[c, p] for c <= r on the tiles of small_tile, tile
// UT×UT, 256 threads with 4×4 outputs each, K in chunks of NB through shared memory.
template <typename T, typename S, bool OUTER>
__global__ void __launch_bounds__(256) k_schur(T* __restrict__ panel, T* __restrict__ upd, const DFront* __restrict__ fr,
                                               const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                               const int64_t* __restrict__ pre_tiles, const int64_t* __restrict__ pre_scr,
                                               int64_t s, const S* __restrict__ scr_w, const S* __restrict__ scr_l,
                                               const int64_t* __restrict__ status) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S* As = reinterpret_cast<S*>(smem_raw);  // [NB][UT + 1]
    S* Bs = As + NB * (UT + 1);
    int64_t b = blockIdx.x;
    int64_t i = find_slot_warp(pre_tiles, nact, b);
    int64_t lt = b - pre_tiles[i];
    int64_t t = order[fr_off + i];
    if (status[t] != -1) return;
    const DFront f = fr[t];
    const int64_t J0 = (s / KO) * NBO;
    const SmallTile st = small_tile<OUTER>(f, s, lt);
    const int64_t row0 = st.row0, col0 = st.col0, col_end = st.col_end, kofs = st.kofs, klen = st.klen;
    const bool in_panel = st.in_panel;
    // scratch row of front row r: pre_scr[i] + r − J0
    const S* wbase = scr_w + (pre_scr[i] - J0) * NBO + kofs;
    const S* lbase = scr_l + (pre_scr[i] - J0) * NBO + kofs;
    int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    S acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c] = (S)0;
    for (int64_t k0 = 0; k0 < klen; k0 += NB) {
        int kc = (int)min((int64_t)NB, klen - k0);
        if (k0 > 0) __syncthreads();
        for (int idx = threadIdx.x; idx < UT * NB; idx += blockDim.x) {
            int rr = idx / NB, kk = idx - rr * NB;
            int64_t r = row0 + rr, c = col0 + rr;
            bool kin = kk < kc;
            As[kk * (UT + 1) + rr] = (kin && r < f.m) ? wbase[r * NBO + k0 + kk] : (S)0;
            Bs[kk * (UT + 1) + rr] = (kin && c < col_end) ? lbase[c * NBO + k0 + kk] : (S)0;
        }
        __syncthreads();
#pragma unroll 8
        for (int kk = 0; kk < NB; kk++) {
            S av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; a++) av[a] = As[kk * (UT + 1) + ty + 16 * a];
#pragma unroll
            for (int c = 0; c < 4; c++) bv[c] = Bs[kk * (UT + 1) + tx + 16 * c];
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) acc[a][c] = fma(av[a], bv[c], acc[a][c]);
        }
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
        int64_t r = row0 + ty + 16 * a;
        if (r >= f.m) continue;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            int64_t cc = col0 + tx + 16 * c;
            if (cc >= col_end || cc > r) continue;
            if (in_panel)
                panel[f.poff + r * f.ldp + cc] -= (T)acc[a][c];
            else
                upd[f.uoff + (r - f.k) * f.ldu + (cc - f.k)] -= (T)acc[a][c];
        }
    }
}

constexpr size_t PB_SMEM = 2 * NB * (NB + 1) * sizeof(double);

// Outer update of large fronts on the CUDA cores: 128×128 tiles (the tile grid of the
// tensor-core kernel), 256 threads with 8×8 outputs each, K in chunks of 16 through
// a two-stage shared-memory ring.
constexpr int BT = 128, BK = 16;
template <typename S>
constexpr size_t big_smem() {
    return 2 * 2 * BK * (BT + 1) * sizeof(S);
}

// Tile lt of an outer update on the 128×128 grid: first the lower-triangular tiles of the
// panel columns [J1e, k) (column by column, rows from the diagonal tile down), then the
// lower triangle of the update block [k, m)².
struct BigTile {
    int64_t row0, col0, col_end;
    bool in_panel;
};
__device__ __forceinline__ BigTile big_tile(const DFront& f, int64_t J1e, int64_t lt) {
    const int64_t R = f.m - J1e;
    const int64_t nrt = (R + BT - 1) / BT, ncp = (f.k - J1e + BT - 1) / BT;
    const int64_t cntP = ncp * nrt - ncp * (ncp - 1) / 2;
    BigTile b;
    if (lt < cntP) {
        int64_t tj = 0, cnt = nrt;
        while (lt >= cnt) {
            lt -= cnt;
            tj++;
            cnt = nrt - tj;
        }
        b.row0 = J1e + (tj + lt) * BT;
        b.col0 = J1e + tj * BT;
        b.col_end = f.k;
        b.in_panel = true;
    } else {
        const int64_t idx = lt - cntP;
        int64_t ti = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
        while (ti * (ti + 1) / 2 > idx) ti--;
        while ((ti + 1) * (ti + 2) / 2 <= idx) ti++;
        const int64_t tj = idx - ti * (ti + 1) / 2;
        b.row0 = f.k + ti * BT;
        b.col0 = f.k + tj * BT;
        b.col_end = f.m;
        b.in_panel = false;
    }
    return b;
}

template <typename T, typename S>
__global__ void __launch_bounds__(256) k_schur_big(T* __restrict__ panel, T* __restrict__ upd, const DFront* __restrict__ fr,
                                                   const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                                   const int64_t* __restrict__ pre_tiles,
                                                   const int64_t* __restrict__ pre_scr, int64_t s,
                                                   const S* __restrict__ scr_w, const S* __restrict__ scr_l,
                                                   const int64_t* __restrict__ status) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    S* sbuf = reinterpret_cast<S*>(smem_raw);  // [2 stages][A|B][BK][BT + 1]
    int64_t b = blockIdx.x;
    int64_t i = find_slot_warp(pre_tiles, nact, b);
    int64_t lt = b - pre_tiles[i];
    int64_t t = order[fr_off + i];
    if (status[t] != -1) return;
    const DFront f = fr[t];
    int64_t J0 = (s / KO) * NBO;
    int64_t J1e = min(J0 + NBO, f.k);
    int64_t klen = J1e - J0;
    const BigTile bt = big_tile(f, J1e, lt);
    const int64_t row0 = bt.row0, col0 = bt.col0, col_end = bt.col_end;
    const bool in_panel = bt.in_panel;
    const S* wbase = scr_w + (pre_scr[i] - J0) * NBO;
    const S* lbase = scr_l + (pre_scr[i] - J0) * NBO;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    // loader: asynchronous copies (cp.async, zero-filled outside the tile) of 128 rows ×
    // BK pivots of W and of L into one stage; consecutive threads take consecutive pivots
    auto load = [&](int stage, int64_t k0) {
        S* As = sbuf + stage * 2 * BK * (BT + 1);
        S* Bs = As + BK * (BT + 1);
        for (int idx = threadIdx.x; idx < BT * BK; idx += 256) {
            int rr = idx / BK, kk = idx - rr * BK;
            int64_t r = row0 + rr, c = col0 + rr;
            bool kin = k0 + kk < klen;
            bool ra = kin && r < f.m, rb = kin && c < col_end;
            const S* ga = ra ? wbase + r * NBO + k0 + kk : wbase;
            const S* gb = rb ? lbase + c * NBO + k0 + kk : lbase;
            uint32_t sa = (uint32_t)__cvta_generic_to_shared(As + kk * (BT + 1) + rr);
            uint32_t sb = (uint32_t)__cvta_generic_to_shared(Bs + kk * (BT + 1) + rr);
            asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(sa), "l"(ga), "n"(sizeof(S)),
                         "r"(ra ? (int)sizeof(S) : 0)
                         : "memory");
            asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;" ::"r"(sb), "l"(gb), "n"(sizeof(S)),
                         "r"(rb ? (int)sizeof(S) : 0)
                         : "memory");
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    S acc[8][8];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int c = 0; c < 8; c++) acc[a][c] = (S)0;
    int nk = (int)((klen + BK - 1) / BK);
    load(0, 0);
    for (int kc = 0; kc < nk; kc++) {
        if (kc + 1 < nk) {
            load((kc + 1) & 1, (int64_t)(kc + 1) * BK);
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        }
        __syncthreads();
        const S* As = sbuf + (kc & 1) * 2 * BK * (BT + 1);
        const S* Bs = As + BK * (BT + 1);
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            S av[8], bv[8];
#pragma unroll
            for (int a = 0; a < 8; a++) av[a] = As[kk * (BT + 1) + ty + 16 * a];
#pragma unroll
            for (int c = 0; c < 8; c++) bv[c] = Bs[kk * (BT + 1) + tx + 16 * c];
#pragma unroll
            for (int a = 0; a < 8; a++)
#pragma unroll
                for (int c = 0; c < 8; c++) acc[a][c] = fma(av[a], bv[c], acc[a][c]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int a = 0; a < 8; a++) {
        int64_t r = row0 + ty + 16 * a;
        if (r >= f.m) continue;
#pragma unroll
        for (int c = 0; c < 8; c++) {
            int64_t cc = col0 + tx + 16 * c;
            if (cc >= col_end || cc > r) continue;
            if (in_panel)
                panel[f.poff + r * f.ldp + cc] -= (T)acc[a][c];
            else
                upd[f.uoff + (r - f.k) * f.ldu + (cc - f.k)] -= (T)acc[a][c];
        }
    }
}

// Outer update of large fronts in FP64 on the tensor cores' FP64 path (mma.sync m8n8k4
// f64, one instruction per 8×8×4 block). Two CTAs per 128×128 tile of k_schur_big's grid,
// one per 64-column half, and two CTAs per SM, so that one CTA's start (the front lookup)
// and read-modify-write epilogue overlap the other's MMAs. 4 warps of 64×32 outputs; K in
// chunks of 16 through a three-stage cp.async ring of padded rows (W and L copied
// row-major, pivots contiguous as in the scratch, pitch 20 doubles: the fragment loads,
// 8 rows × 4 pivots per warp, hit distinct banks in each half-warp). Each warp loads the
// fragments of the next 4-pivot step before it issues the MMAs of the current one.
constexpr int DM_BK = 16, DM_PITCH = 20, DM_STAGES = 3, DM_TN = 64, DM_THREADS = 128;
constexpr int DM_STAGE = (BT + DM_TN) * DM_PITCH;  // doubles per stage: W rows, then L rows
constexpr size_t DM_SMEM = (size_t)DM_STAGES * DM_STAGE * sizeof(double);

// Start of front row r in the output of an outer-update tile, indexed by front column:
// the panel row (columns < k) or the update-block row (columns >= k).
__device__ __forceinline__ double* out_row(double* panel, double* upd, const DFront& f, bool in_panel, int64_t r) {
    return in_panel ? panel + f.poff + r * f.ldp : upd + f.uoff + (r - f.k) * f.ldu - f.k;
}

__global__ void __launch_bounds__(DM_THREADS, 2)
    k_schur_dmma(double* __restrict__ panel, double* __restrict__ upd, const DFront* __restrict__ fr,
                 const int64_t* __restrict__ order, int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre_tiles,
                 const int64_t* __restrict__ pre_scr, int64_t s, const double* __restrict__ scr_w,
                 const double* __restrict__ scr_l, const int64_t* __restrict__ status) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sbuf = reinterpret_cast<double*>(smem_raw);  // [stage][BT W rows | DM_TN L rows][DM_PITCH]
    const int64_t b = blockIdx.x >> 1;
    const int half = blockIdx.x & 1;
    const int64_t i = find_slot_warp(pre_tiles, nact, b);
    const int64_t t = order[fr_off + i];
    if (status[t] != -1) return;
    const DFront f = fr[t];
    const int64_t J0 = (s / KO) * NBO;
    const int64_t J1e = min(J0 + NBO, f.k);
    const int klen = (int)(J1e - J0);
    const BigTile bt = big_tile(f, J1e, b - pre_tiles[i]);
    const int64_t col0 = bt.col0 + half * DM_TN;
    if (col0 >= bt.col_end) return;
    // scratch row of front row r: pre_scr[i] + r − J0
    const double* wrow = scr_w + (pre_scr[i] - J0 + bt.row0) * NBO;
    const double* lrow = scr_l + (pre_scr[i] - J0 + col0) * NBO;
    const int nra = (int)min((int64_t)BT, f.m - bt.row0);
    const int nrb = (int)min((int64_t)DM_TN, bt.col_end - col0);
    const int nk = (klen + DM_BK - 1) / DM_BK;
    {
        // L2 prefetch of this CTA's output rows (in range only), read back at the end
        const int64_t r = bt.row0 + threadIdx.x;
        const int64_t cend = r < f.m ? min(bt.col_end, min(col0 + DM_TN, r + 1)) : col0;
        if (cend > col0) {
            const double* rowp = out_row(panel, upd, f, bt.in_panel, r);
            for (int64_t c = col0; c < cend; c += 16) asm volatile("prefetch.global.L2 [%0];" ::"l"(rowp + c));
            asm volatile("prefetch.global.L2 [%0];" ::"l"(rowp + cend - 1));
        }
    }
    auto load = [&](int kc) {
        double* st = sbuf + (kc % DM_STAGES) * DM_STAGE;
        const int k0 = kc * DM_BK;
        cp_async_tile(st, DM_PITCH, wrow + k0, NBO, nra, klen - k0, BT, DM_BK, DM_THREADS);
        cp_async_tile(st + BT * DM_PITCH, DM_PITCH, lrow + k0, NBO, nrb, klen - k0, DM_TN, DM_BK, DM_THREADS);
    };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;  // warp tile rows [64·wm, +64), columns [32·wn, +32)
    const int aoff = (wm * 64 + g) * DM_PITCH + q, boff = (BT + wn * 32 + g) * DM_PITCH + q;
    auto frag = [&](double* fa, double* fb, int kc, int kk) {
        const double* st = sbuf + (kc % DM_STAGES) * DM_STAGE + kk;
#pragma unroll
        for (int a = 0; a < 8; a++) fa[a] = st[aoff + a * 8 * DM_PITCH];
#pragma unroll
        for (int c = 0; c < 4; c++) fb[c] = st[boff + c * 8 * DM_PITCH];
    };
    double acc[8][4][2];
#pragma unroll
    for (int a = 0; a < 8; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c][0] = acc[a][c][1] = 0.0;
    double fa[2][8], fb[2][4];
    load(0);
    cp_async_commit();
    if (nk > 1) load(1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (nk > 2) load(2);
    cp_async_commit();
    frag(fa[0], fb[0], 0, 0);
    for (int kc = 0; kc < nk; kc++) {
#pragma unroll
        for (int j = 0; j < DM_BK / 4; j++) {
            const int cur = j & 1, nxt = cur ^ 1;
            if (j + 1 < DM_BK / 4) {
                frag(fa[nxt], fb[nxt], kc, (j + 1) * 4);
            } else if (kc + 1 < nk) {
                // chunk kc + 1 is in once at most one group is pending; after the barrier no
                // warp reads chunk kc's stage any more, so chunk kc + 3 may replace it
                cp_async_wait<1>();
                __syncthreads();
                if (kc + 3 < nk) load(kc + 3);
                cp_async_commit();
                frag(fa[nxt], fb[nxt], kc + 1, 0);
            }
#pragma unroll
            for (int a = 0; a < 8; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) dmma_884(acc[a][c][0], acc[a][c][1], fa[cur][a], fb[cur][c]);
        }
    }
    cp_async_wait<0>();
    // accumulator (a, c, e): row 64·wm + 8a + g, column 32·wn + 8c + 2q + e; F −= W·Lᵀ on the
    // lower triangle, two columns per 16-byte access where the pair is aligned and in range.
    // Two batches of 16 pairs: all loads of a batch are in flight before its first store.
#pragma unroll
    for (int h = 0; h < 2; h++) {
        double2 v[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int64_t r = bt.row0 + wm * 64 + (h * 4 + a) * 8 + g;
            const int64_t cend = r < f.m ? min(bt.col_end, r + 1) : 0;
            const double* rowp = r < f.m ? out_row(panel, upd, f, bt.in_panel, r) : panel;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int64_t cc = col0 + wn * 32 + c * 8 + 2 * q;
                const double* p = rowp + cc;
                if (cc + 1 < cend && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
                    v[a][c] = *reinterpret_cast<const double2*>(p);
                } else {
                    v[a][c].x = cc < cend ? p[0] : 0.0;
                    v[a][c].y = cc + 1 < cend ? p[1] : 0.0;
                }
            }
        }
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int64_t r = bt.row0 + wm * 64 + (h * 4 + a) * 8 + g;
            if (r >= f.m) continue;
            const int64_t cend = min(bt.col_end, r + 1);
            double* rowp = out_row(panel, upd, f, bt.in_panel, r);
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int64_t cc = col0 + wn * 32 + c * 8 + 2 * q;
                double* p = rowp + cc;
                const double x = v[a][c].x - acc[h * 4 + a][c][0], y = v[a][c].y - acc[h * 4 + a][c][1];
                if (cc + 1 < cend && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
                    *reinterpret_cast<double2*>(p) = make_double2(x, y);
                } else {
                    if (cc < cend) p[0] = x;
                    if (cc + 1 < cend) p[1] = y;
                }
            }
        }
    }
}

// The FP64 updates on the UT×UT grid of k_schur (inner updates, and outer updates of small
// fronts) on the FP64 tensor-core path: 128 threads, 4 warps of 32×32 outputs, K in chunks
// of 16 through a three-stage cp.async ring (the ring, pitch and fragment pipelining of
// k_schur_dmma), two or more CTAs per SM.
constexpr int D64_STAGE = 2 * UT * DM_PITCH;  // doubles per stage: W rows, then L rows
constexpr size_t D64_SMEM = (size_t)DM_STAGES * D64_STAGE * sizeof(double);

template <bool OUTER>
__global__ void __launch_bounds__(128, 2) k_schur_dmma64(double* __restrict__ panel, double* __restrict__ upd,
                                                      const DFront* __restrict__ fr,
                                                      const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                                      const int64_t* __restrict__ pre_tiles,
                                                      const int64_t* __restrict__ pre_scr, int64_t s,
                                                      const double* __restrict__ scr_w,
                                                      const double* __restrict__ scr_l,
                                                      const int64_t* __restrict__ status) {
    pdl_wait();  // wait first: a dependent launched early may then read our inputs
    pdl_launch_dependents();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double* sbuf = reinterpret_cast<double*>(smem_raw);  // [stage][UT W rows | UT L rows][DM_PITCH]
    const int64_t b = blockIdx.x;
    const int64_t i = find_slot_warp(pre_tiles, nact, b);
    const int64_t t = order[fr_off + i];
    if (status[t] != -1) return;
    const DFront f = fr[t];
    const int64_t J0 = (s / KO) * NBO;
    const SmallTile tl = small_tile<OUTER>(f, s, b - pre_tiles[i]);
    // scratch row of front row r: pre_scr[i] + r − J0; the tile's pivots start at kofs
    const double* wrow = scr_w + (pre_scr[i] - J0 + tl.row0) * NBO + tl.kofs;
    const double* lrow = scr_l + (pre_scr[i] - J0 + tl.col0) * NBO + tl.kofs;
    const int klen = (int)tl.klen;
    const int nra = (int)min((int64_t)UT, f.m - tl.row0);
    const int nrb = (int)min((int64_t)UT, tl.col_end - tl.col0);
    const int nk = (klen + DM_BK - 1) / DM_BK;
    auto load = [&](int kc) {
        double* st = sbuf + (kc % DM_STAGES) * D64_STAGE;
        const int k0 = kc * DM_BK;
        cp_async_tile(st, DM_PITCH, wrow + k0, NBO, nra, klen - k0, UT, DM_BK, 128);
        cp_async_tile(st + UT * DM_PITCH, DM_PITCH, lrow + k0, NBO, nrb, klen - k0, UT, DM_BK, 128);
    };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int wm = warp & 1, wn = warp >> 1;  // warp tile rows [32·wm, +32), columns [32·wn, +32)
    const int aoff = (wm * 32 + g) * DM_PITCH + q, boff = (UT + wn * 32 + g) * DM_PITCH + q;
    auto frag = [&](double* fa, double* fb, int kc, int kk) {
        const double* st = sbuf + (kc % DM_STAGES) * D64_STAGE + kk;
#pragma unroll
        for (int a = 0; a < 4; a++) fa[a] = st[aoff + a * 8 * DM_PITCH];
#pragma unroll
        for (int c = 0; c < 4; c++) fb[c] = st[boff + c * 8 * DM_PITCH];
    };
    double acc[4][4][2];
#pragma unroll
    for (int a = 0; a < 4; a++)
#pragma unroll
        for (int c = 0; c < 4; c++) acc[a][c][0] = acc[a][c][1] = 0.0;
    double fa[2][4], fb[2][4];
    load(0);
    cp_async_commit();
    if (nk > 1) load(1);
    cp_async_commit();
    cp_async_wait<1>();
    __syncthreads();
    if (nk > 2) load(2);
    cp_async_commit();
    frag(fa[0], fb[0], 0, 0);
    for (int kc = 0; kc < nk; kc++) {
#pragma unroll
        for (int j = 0; j < DM_BK / 4; j++) {
            const int cur = j & 1, nxt = cur ^ 1;
            if (j + 1 < DM_BK / 4) {
                frag(fa[nxt], fb[nxt], kc, (j + 1) * 4);
            } else if (kc + 1 < nk) {
                cp_async_wait<1>();
                __syncthreads();
                if (kc + 3 < nk) load(kc + 3);
                cp_async_commit();
                frag(fa[nxt], fb[nxt], kc + 1, 0);
            }
#pragma unroll
            for (int a = 0; a < 4; a++)
#pragma unroll
                for (int c = 0; c < 4; c++) dmma_884(acc[a][c][0], acc[a][c][1], fa[cur][a], fb[cur][c]);
        }
    }
    cp_async_wait<0>();
    // accumulator (a, c, e): row 32·wm + 8a + g, column 32·wn + 8c + 2q + e; all loads of
    // the tile's pairs are in flight before the first store
    double2 v[4][4];
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int64_t r = tl.row0 + wm * 32 + a * 8 + g;
        const int64_t cend = r < f.m ? min(tl.col_end, r + 1) : 0;
        const double* rowp = r < f.m ? out_row(panel, upd, f, tl.in_panel, r) : panel;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int64_t cc = tl.col0 + wn * 32 + c * 8 + 2 * q;
            const double* p = rowp + cc;
            if (cc + 1 < cend && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
                v[a][c] = *reinterpret_cast<const double2*>(p);
            } else {
                v[a][c].x = cc < cend ? p[0] : 0.0;
                v[a][c].y = cc + 1 < cend ? p[1] : 0.0;
            }
        }
    }
#pragma unroll
    for (int a = 0; a < 4; a++) {
        const int64_t r = tl.row0 + wm * 32 + a * 8 + g;
        if (r >= f.m) continue;
        const int64_t cend = min(tl.col_end, r + 1);
        double* rowp = out_row(panel, upd, f, tl.in_panel, r);
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int64_t cc = tl.col0 + wn * 32 + c * 8 + 2 * q;
            double* p = rowp + cc;
            const double x = v[a][c].x - acc[a][c][0], y = v[a][c].y - acc[a][c][1];
            if (cc + 1 < cend && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
                *reinterpret_cast<double2*>(p) = make_double2(x, y);
            } else {
                if (cc < cend) p[0] = x;
                if (cc + 1 < cend) p[1] = y;
            }
        }
    }
}

// Scatter of the caller's entries built on the device, one warp per internal column,
// the columns in level order (lcol: the column, lfront: its front). Entry p of the
// caller's column c = owner[q] is an original entry of the factorization when its
// internal row eq[row] is at least q (the positive definite factorization reads the
// internal lower triangle, ffi/src/lib.rs:216-224). k_map_count counts them per column
// and flags (bit 0) a column whose rows are not strictly increasing; k_map_fill, given
// the prefix sums of the counts, writes each entry's panel offset and source index in
// the caller's order (the order of the host lists of scatter_from_caller). A row that
// the front does not hold sets bit 1 and is sent to the column's diagonal entry.
__global__ void k_map_count(const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices,
                            const int64_t* __restrict__ eq, const int64_t* __restrict__ owner,
                            const int32_t* __restrict__ lcol, int64_t ncols, int64_t* __restrict__ cnt,
                            int* __restrict__ flag, int64_t* __restrict__ diag_src) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= ncols) return;
    const int64_t q = lcol[i], c = owner[q];
    const int64_t p0 = indptr[c], p1 = indptr[c + 1];
    int64_t z = 0;
    bool bad = false;
    for (int64_t p = p0 + lane; p < p1; p += 32) {
        const int64_t r = indices[p];
        z += eq[r] >= q ? 1 : 0;
        if (p > p0 && indices[p - 1] >= r) bad = true;
        if (r == c) diag_src[q] = p;  // rows are distinct when no column is flagged
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(0xffffffffu, z, o);
    if (__any_sync(0xffffffffu, bad) && lane == 0) atomicOr(flag, 1);
    if (lane == 0) cnt[i] = z;
}

__global__ void k_map_fill(const int64_t* __restrict__ indptr, const int64_t* __restrict__ indices,
                           const int64_t* __restrict__ eq, const int64_t* __restrict__ owner,
                           const int32_t* __restrict__ lcol, const int32_t* __restrict__ lfront,
                           const DFront* __restrict__ fr, const int64_t* __restrict__ rows, int64_t ncols,
                           const int64_t* __restrict__ off, int64_t* __restrict__ dst, int64_t* __restrict__ src,
                           int* __restrict__ flag) {
    const int lane = threadIdx.x & 31;
    const int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (i >= ncols) return;
    const int64_t q = lcol[i], c = owner[q];
    const DFront f = fr[lfront[i]];
    const int64_t p0 = indptr[c], p1 = indptr[c + 1];
    const int64_t colo = q - f.start;
    int64_t base = off[i];
    for (int64_t pb = p0; pb < p1; pb += 32) {
        const int64_t p = pb + lane;
        bool keep = false;
        int64_t lr = colo;
        if (p < p1) {
            const int64_t qr = eq[indices[p]];
            keep = qr >= q;
            if (keep) {
                if (qr < f.start + f.k) {
                    lr = qr - f.start;
                } else {
                    const int64_t* rw = rows + f.rows_off;
                    int64_t lo = 0, hi = f.u;
                    while (lo < hi) {
                        const int64_t mid = (lo + hi) >> 1;
                        if (rw[mid] < qr)
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    if (lo < f.u && rw[lo] == qr) {
                        lr = f.k + lo;
                    } else {
                        atomicOr(flag, 2);
                        lr = colo;
                    }
                }
            }
        }
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (keep) {
            const int64_t o = base + __popc(m & ((1u << lane) - 1u));
            dst[o] = f.poff + lr * f.ldp + colo;
            src[o] = p;
        }
        base += __popc(m);
    }
}

// the original diagonal of every equation (FP16 split scales): the value of the caller's
// diagonal entry of its column, or 0 where that entry is not known
__global__ void k_orig_diag(const double* __restrict__ src, const int64_t* __restrict__ diag_src, int64_t n,
                            double* __restrict__ out) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = diag_src[q];
        out[q] = p >= 0 ? src[p] : 0.0;
    }
}

__global__ void k_gather_i64(const int64_t* __restrict__ a, const int64_t* __restrict__ idx, int64_t n,
                             int64_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = a[idx[i]];
}

template <typename T>
struct ScrType {
    using type = T;
};

}  // namespace

// ---------------------------------------------------------------------------
// Engine
// ---------------------------------------------------------------------------
void* Engine::dalloc(size_t bytes) {
    void* p = dev_alloc(bytes, stream_);
    allocs_.push_back(p);
    return p;
}

template <typename V, typename A>
static V* upload(const std::vector<V, A>& v, cudaStream_t st, std::vector<void*>& allocs, int64_t& bytes_total) {
    V* p = nullptr;
    bytes_total += (int64_t)(v.size() * sizeof(V));
    size_t bytes = std::max<size_t>(v.size() * sizeof(V), 256);
    p = (V*)dev_alloc(bytes, st);
    allocs.push_back(p);
    if (!v.empty()) host_upload(p, v.data(), v.size() * sizeof(V), st);
    return p;
}

void Engine::upload_plan() {
    auto up = [&](const auto& v) { return upload(v, stream_, allocs_, plan_bytes_); };
    dp_.fronts = up(plan_.fronts);
    dp_.level_order = up(plan_.level_order);
    dp_.pre_panel = up(plan_.pre_panel);
    dp_.pre_inner = up(plan_.pre_inner);
    dp_.pre_inner_tc = up(plan_.pre_inner_tc);
    dp_.pre_wrows = up(plan_.pre_wrows);
    dp_.pre_wpart = up(plan_.pre_wpart);
    dp_.pre_outer = up(plan_.pre_outer);
    dp_.pre_outer_tc = up(plan_.pre_outer_tc);
    dp_.pre_outer_tc2 = up(plan_.pre_outer_tc2);
    dp_.pre_scr = up(plan_.pre_scr);
    dp_.panel_mode = up(plan_.panel_mode);
    dp_.outer_mode = up(plan_.outer_mode);
    dp_.xadd_child = up(plan_.xadd_child);
    dp_.xadd_task = up(plan_.xadd_task);
    dp_.xadd_fpre = up(plan_.xadd_fpre);
    dp_.rows = up(plan_.rows);
    dp_.emap = up(plan_.emap);
    dp_.chain_blk = up(plan_.chain_blk);
    dp_.chain_bfront = up(plan_.chain_bfront);
    dp_.chain_fwd = up(plan_.chain_fwd);
    dp_.chain_bwd = up(plan_.chain_bwd);
    dp_.chain_rows = up(plan_.chain_rows);
    dp_.chain_cols = up(plan_.chain_cols);
    level_poff_.assign(plan_.nlevels + 1, plan_.panel_elems);
    for (int64_t l = 0; l < plan_.nlevels; l++)
        if (plan_.level_off[l + 1] > plan_.level_off[l]) level_poff_[l] = plan_.fronts[plan_.level_order[plan_.level_off[l]]].poff;
    for (int64_t l = plan_.nlevels - 1; l >= 0; l--)
        if (plan_.level_off[l + 1] == plan_.level_off[l]) level_poff_[l] = level_poff_[l + 1];
}

// The host scatter lists on the device; the host copies of the per-entry lists are
// released (only the level and front offsets stay on the host).
void Engine::upload_scatter() {
    auto up = [&](const auto& v) { return upload(v, stream_, allocs_, plan_bytes_); };
    nseg_ = (int64_t)scatter_.dst.size();
    dp_.seg_dst = up(scatter_.dst);
    bool single = (int64_t)scatter_.src.size() == (int64_t)scatter_.dst.size();
    dp_.seg_ptr = single ? nullptr : up(scatter_.seg_ptr);
    dp_.seg_src = up(scatter_.src);
    dp_.front_seg = up(scatter_.front_seg);
    SegVec().swap(scatter_.dst);
    SegVec().swap(scatter_.src);
    std::vector<int64_t>().swap(scatter_.seg_ptr);
}

void Engine::build_scatter_device(const CallerPattern& cp) {
    const Plan& P = plan_;
    const std::vector<int64_t>& eq = *cp.eq;
    const int64_t N = cp.ncaller, nnz = N > 0 ? cp.indptr[N] : 0, n = P.n;
    // the internal columns in level order and their fronts; the position of each front's
    // first column
    std::vector<int32_t> lcol(std::max<int64_t>(n, 1)), lfront(std::max<int64_t>(n, 1));
    std::vector<int64_t> fpos(P.nfronts + 1, 0);
    {
        int64_t o = 0;
        for (int64_t j = 0; j < P.nfronts; j++) {
            const int64_t t = P.level_order[j];
            const DFront& d = P.fronts[t];
            fpos[j] = o;
            for (int64_t q = d.start; q < d.start + d.k; q++) {
                lcol[o] = (int32_t)q;
                lfront[o] = (int32_t)t;
                o++;
            }
        }
        fpos[P.nfronts] = o;
        if (o != n) throw CudaError("build_scatter_device: the fronts do not cover the equations");
    }
    std::vector<int64_t> owner(std::max<int64_t>(n, 1), 0);
    for (int64_t i = 0; i < N; i++)
        if (eq[i] >= 0) owner[eq[i]] = i;
    // work buffers: the update arena when it is large enough (unused before the first
    // numeric phase)
    auto r256 = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t nc1 = (size_t)n + 1;
    const size_t nind = cp.indices_dev ? 1 : (size_t)std::max<int64_t>(nnz, 1);
    const size_t need = r256(nind * 8) + r256(((size_t)N + 1) * 8) +
                        r256((size_t)std::max<int64_t>(N, 1) * 8) + r256(nc1 * 8) + 2 * r256(nc1 * 4) +
                        r256(nc1 * 8) + r256((size_t)scan_tmp_elems((int64_t)nc1) * 8) +
                        r256(((size_t)P.nfronts + 1) * 8) + r256(4) + 256;
    const size_t es = prec_ == PREC_FP64 ? sizeof(double) : sizeof(float);
    const bool in_arena = (size_t)P.upd_elems * es >= need;
    char* base = in_arena ? (char*)upd_ : (char*)dev_alloc(need, stream_);
    char* w = base;
    auto carve = [&](size_t bytes) {
        char* r = w;
        w += r256(bytes);
        return r;
    };
    int64_t* d_ind = (int64_t*)carve(nind * 8);
    int64_t* d_ptr = (int64_t*)carve(((size_t)N + 1) * 8);
    int64_t* d_eq = (int64_t*)carve((size_t)std::max<int64_t>(N, 1) * 8);
    int64_t* d_owner = (int64_t*)carve(nc1 * 8);
    int32_t* d_lcol = (int32_t*)carve(nc1 * 4);
    int32_t* d_lfront = (int32_t*)carve(nc1 * 4);
    int64_t* d_off = (int64_t*)carve(nc1 * 8);
    int64_t* d_stmp = (int64_t*)carve((size_t)scan_tmp_elems((int64_t)nc1) * 8);
    int64_t* d_fpos = (int64_t*)carve(((size_t)P.nfronts + 1) * 8);
    int* d_flag = (int*)carve(4);
    if ((size_t)(w - base) > need) throw CudaError("build_scatter_device: work buffer layout");
    const int64_t* ind = d_ind;
    if (cp.indices_dev) {
        ind = cp.indices_dev;
        if (cp.wait_indices) cp.wait_indices((void*)stream_);
    } else if (nnz > 0) {
        host_upload(d_ind, cp.indices, (size_t)nnz * 8, stream_);
    }
    host_upload(d_ptr, cp.indptr, ((size_t)N + 1) * 8, stream_);
    if (N > 0) host_upload(d_eq, eq.data(), (size_t)N * 8, stream_);
    host_upload(d_owner, owner.data(), (size_t)n * 8, stream_);
    host_upload(d_lcol, lcol.data(), (size_t)n * 4, stream_);
    host_upload(d_lfront, lfront.data(), (size_t)n * 4, stream_);
    host_upload(d_fpos, fpos.data(), ((size_t)P.nfronts + 1) * 8, stream_);
    RFG_CUDA(cudaMemsetAsync(d_flag, 0, 4, stream_));
    RFG_CUDA(cudaMemsetAsync(d_off + n, 0, 8, stream_));
    const unsigned wblocks = (unsigned)std::max<int64_t>(1, (n * 32 + 255) / 256);
    diag_src_ = (int64_t*)dalloc((size_t)std::max<int64_t>(n, 1) * 8);
    RFG_CUDA(cudaMemsetAsync(diag_src_, 0xff, (size_t)std::max<int64_t>(n, 1) * 8, stream_));
    if (n > 0)
        k_map_count<<<wblocks, 256, 0, stream_>>>(d_ptr, ind, d_eq, d_owner, d_lcol, n, d_off, d_flag, diag_src_);
    exclusive_scan_i64(d_off, (int64_t)nc1, d_stmp, stream_);
    int64_t total = 0;
    int flag = 0;
    RFG_CUDA(cudaMemcpyAsync(&total, d_off + n, 8, cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaMemcpyAsync(&flag, d_flag, 4, cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaStreamSynchronize(stream_));
    plan_bytes_ += (int64_t)((cp.indices_dev ? 0 : (size_t)nnz * 8) + ((size_t)N + 1) * 8 + (size_t)N * 8 +
                             (size_t)n * 16 + ((size_t)P.nfronts + 1) * 8);
    if (flag & 1) {
        // a column with unsorted or repeated rows: the host lists (duplicates summed); the
        // diagonal sources are not known, so the tensor cores keep the TF32 split
        diag_src_ = nullptr;
        if (!in_arena) dev_free(base, stream_);
        scatter_ = scatter_from_caller(P, *cp.sym, N, cp.indptr, cp.indices, eq);
        upload_scatter();
        return;
    }
    nseg_ = total;
    dp_.seg_dst = (int64_t*)dalloc((size_t)std::max<int64_t>(total, 1) * 8);
    dp_.seg_src = (int64_t*)dalloc((size_t)std::max<int64_t>(total, 1) * 8);
    dp_.seg_ptr = nullptr;
    dp_.front_seg = (int64_t*)dalloc(((size_t)P.nfronts + 1) * 8);
    if (n > 0)
        k_map_fill<<<wblocks, 256, 0, stream_>>>(d_ptr, ind, d_eq, d_owner, d_lcol, d_lfront, dp_.fronts, dp_.rows,
                                                 n, d_off, dp_.seg_dst, dp_.seg_src, d_flag);
    k_gather_i64<<<(unsigned)((P.nfronts + 256) / 256), 256, 0, stream_>>>(d_off, d_fpos, P.nfronts + 1,
                                                                           dp_.front_seg);
    RFG_CUDA(cudaGetLastError());
    scatter_.front_seg.assign(P.nfronts + 1, 0);
    RFG_CUDA(cudaMemcpyAsync(scatter_.front_seg.data(), dp_.front_seg, ((size_t)P.nfronts + 1) * 8,
                             cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaMemcpyAsync(&flag, d_flag, 4, cudaMemcpyDeviceToHost, stream_));
    if (!in_arena) dev_free(base, stream_);
    RFG_CUDA(cudaStreamSynchronize(stream_));
    if (flag & 2) throw CudaError("build_scatter_device: an entry's row is not in its front (symbolic mismatch)");
    scatter_.level_seg.assign(P.nlevels + 1, 0);
    for (int64_t l = 0; l <= P.nlevels; l++) scatter_.level_seg[l] = scatter_.front_seg[P.level_off[l]];
}

Engine::Engine(Plan&& plan, Scatter&& scatter, int64_t nsrc, Precision prec, bool use_tc)
    : plan_(std::move(plan)), scatter_(std::move(scatter)), nsrc_(nsrc), prec_(prec),
      use_tc_(use_tc && prec == PREC_MIXED) {
    RFG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    RFG_CUDA(cudaEventCreate(&ev0_));
    RFG_CUDA(cudaEventCreate(&ev1_));
    upload_plan();
    upload_scatter();
    init(use_tc);
}

Engine::Engine(Plan&& plan, const CallerPattern& pattern, int64_t nsrc, Precision prec, bool use_tc)
    : plan_(std::move(plan)), nsrc_(nsrc), prec_(prec), use_tc_(use_tc && prec == PREC_MIXED) {
    RFG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    RFG_CUDA(cudaEventCreate(&ev0_));
    RFG_CUDA(cudaEventCreate(&ev1_));
    upload_plan();
    // the arenas first: the pattern is mapped in the (still unused) update arena
    size_t es = prec_ == PREC_FP64 ? sizeof(double) : sizeof(float);
    panel_ = dalloc(plan_.panel_elems * es);
    upd_ = dalloc(plan_.upd_elems * es);
    build_scatter_device(pattern);
    init(use_tc);
}

void Engine::init(bool) {
    set_attributes();
    size_t es = prec_ == PREC_FP64 ? sizeof(double) : sizeof(float);
    if (!panel_) panel_ = dalloc(plan_.panel_elems * es);
    if (!upd_) upd_ = dalloc(plan_.upd_elems * es);
    scr_w_ = dalloc(std::max<int64_t>(plan_.max_scr_rows, 1) * NBO * es);
    scr_l_ = dalloc(std::max<int64_t>(plan_.max_scr_rows, 1) * NBO * es);
    d_ = (double*)dalloc(std::max<int64_t>(plan_.n, 1) * sizeof(double));
    linv_ = (double*)dalloc(std::max<int64_t>(plan_.nblocks, 1) * NB * NB * sizeof(double));
    if (prec_ == PREC_MIXED && plan_.chain_blocks > 0) {
        chain_inv_ = (double*)dalloc(plan_.chain_blocks * (int64_t)WS * WS * sizeof(double));
        chain_err_ = (int*)dalloc(sizeof(int));
        RFG_CUDA(cudaMemsetAsync(chain_err_, 0, sizeof(int), stream_));
    }
    adiag_ = (double*)dalloc(std::max<int64_t>(plan_.n, 1) * sizeof(double));
    status_ = (int64_t*)dalloc(std::max<int64_t>(plan_.nfronts, 1) * sizeof(int64_t));
    src_ = (double*)dalloc(std::max<int64_t>(nsrc_, 1) * sizeof(double));
    {
        // the FP64 matrix of the refinement (CSR in the internal numbering, built by the
        // first refined solve), sized for every scattered entry and its mirror
        const int64_t cap = std::max<int64_t>(2 * nseg_, 1);
        a_rowptr_ = (int64_t*)dalloc((plan_.n + 1) * sizeof(int64_t));
        a_col_ = (int64_t*)dalloc(cap * sizeof(int64_t));
        a_src_ = (int64_t*)dalloc(cap * sizeof(int64_t));
        a_val_ = (double*)dalloc(cap * sizeof(double));
    }
    if (use_tc_) {
        // the split operands in two buffers, alternating with the parity of the outer block
        // (a block's operands stay readable while the next block's panels are written)
        size_t sz = 2 * std::max<int64_t>(plan_.max_scr_rows, 1) * NBO * sizeof(float);
        scr_whi_ = dalloc(sz);
        scr_wlo_ = dalloc(sz);
        scr_lhi_ = dalloc(sz);
        scr_llo_ = dalloc(sz);
        RFG_CUDA(cudaMemsetAsync(scr_whi_, 0, sz, stream_));
        RFG_CUDA(cudaMemsetAsync(scr_wlo_, 0, sz, stream_));
        RFG_CUDA(cudaMemsetAsync(scr_lhi_, 0, sz, stream_));
        RFG_CUDA(cudaMemsetAsync(scr_llo_, 0, sz, stream_));
        const size_t hz = 2 * std::max<int64_t>(plan_.max_scr_rows, 1) * NBO * 2;
        scr_uhi_ = dalloc(hz);
        scr_ulo_ = dalloc(hz);
        scr_uscale_ = dalloc(std::max<int64_t>(plan_.max_scr_rows, 1) * sizeof(float));
        RFG_CUDA(cudaMemsetAsync(scr_uhi_, 0, hz, stream_));
        RFG_CUDA(cudaMemsetAsync(scr_ulo_, 0, hz, stream_));
        RFG_CUDA(cudaMemsetAsync(scr_uscale_, 0, std::max<int64_t>(plan_.max_scr_rows, 1) * sizeof(float), stream_));
        adiag0_ = (double*)dalloc(std::max<int64_t>(plan_.n, 1) * sizeof(double));
        setup_tc();
    }
    RFG_CUDA(cudaStreamSynchronize(stream_));
}

void Engine::set_attributes() {
    RFG_CUDA(cudaFuncSetAttribute(k_schur_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DM_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_dmma64<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D64_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_dmma64<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)D64_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_big<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)big_smem<float>()));
    RFG_CUDA(cudaFuncSetAttribute(k_panel<double, double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PANEL_SMEM_D));
    RFG_CUDA(cudaFuncSetAttribute(k_panel<float, float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PANEL_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_pivot_block<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_pivot_block<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PB_SMEM));
    const size_t s32 = 2 * NB * (UT + 1) * sizeof(float);
    RFG_CUDA(cudaFuncSetAttribute(k_schur<float, float, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s32));
    RFG_CUDA(cudaFuncSetAttribute(k_schur<float, float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)s32));
}

int Engine::tc_error() const {
    if (!tc_err_) return 0;
    int e = 0;
    RFG_CUDA(cudaMemcpy(&e, tc_err_, sizeof(int), cudaMemcpyDeviceToHost));
    return e;
}

Engine::~Engine() {
    if (stream_) cudaStreamSynchronize(stream_);
    for (cudaGraphExec_t& g : factor_graph_)
        if (g) cudaGraphExecDestroy(g);
    for (auto& g : solve_graphs_) cudaGraphExecDestroy(g.exec);
    for (cudaEvent_t e : prof_ev_) cudaEventDestroy(e);
    for (void* p : allocs_) dev_free(p, stream_);
    for (void* p : {(void*)ref_r_, (void*)ref_dx_, (void*)ref_red_}) dev_free(p, stream_);
    if (stream_) cudaStreamSynchronize(stream_);
    if (ev0_) cudaEventDestroy(ev0_);
    if (ev1_) cudaEventDestroy(ev1_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Engine::pivots_to_host(double* out) const {
    RFG_CUDA(cudaMemcpyAsync(out, d_, plan_.n * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaStreamSynchronize(stream_));
}

template <typename T>
void Engine::factor_impl() {
    using S = typename ScrType<T>::type;
    T* panel = (T*)panel_;
    T* upd = (T*)upd_;
    S* sw = (S*)scr_w_;
    S* sl = (S*)scr_l_;
    const Plan& P = plan_;
    int64_t launches = 0;
    size_t schur_smem = 2 * NB * (UT + 1) * sizeof(S);
    int64_t nprof = 0;
    prof_phase_.clear();
    // PROF_SKIP: the interval before a 128-tile outer update at profiling level 2 (not counted)
    constexpr int PROF_SKIP = 7;
    auto mark = [&](int phase) {
        // an event after each launch; the time since the previous event goes to its phase
        // (level 2: only the events around the 128-tile outer updates)
        if (!profile_) return;
        if (profile_ == 2 && phase != 6 && phase != PROF_SKIP) return;
        if (profile_ == 1 && phase == PROF_SKIP) return;
        if (prof_ev_.size() <= prof_phase_.size() + 1) {
            cudaEvent_t e;
            RFG_CUDA(cudaEventCreate(&e));
            prof_ev_.push_back(e);
        }
        // external: under stream capture the record becomes an event-record node of the graph
        RFG_CUDA(cudaEventRecordWithFlags(prof_ev_[prof_phase_.size() + 1], stream_, cudaEventRecordExternal));
        prof_phase_.push_back(phase);
    };
    if (profile_) {
        if (prof_ev_.empty()) {
            cudaEvent_t e;
            RFG_CUDA(cudaEventCreate(&e));
            prof_ev_.push_back(e);
        }
        RFG_CUDA(cudaEventRecordWithFlags(prof_ev_[0], stream_, cudaEventRecordExternal));
    }
    RFG_CUDA(cudaMemsetAsync(status_, 0xff, std::max<int64_t>(P.nfronts, 1) * sizeof(int64_t), stream_));
    RFG_CUDA(cudaMemsetAsync(d_, 0, std::max<int64_t>(P.n, 1) * sizeof(double), stream_));
    if (h16_ && P.n > 0) {
        // RFG_TC_H16_FALLBACK_TEST: no diagonal, so that every row reports an invalid scale
        // and the engine takes its TF32 fallback (tests of that path)
        const bool fail_test = getenv("RFG_TC_H16_FALLBACK_TEST") != nullptr;
        if (fail_test) {
            RFG_CUDA(cudaMemsetAsync(adiag0_, 0, P.n * sizeof(double), stream_));
        } else {
            k_orig_diag<<<(unsigned)std::min<int64_t>((P.n + 255) / 256, 148 * 8), 256, 0, stream_>>>(
                (const double*)src_, (const int64_t*)diag_src_, P.n, adiag0_);
            launches++;
        }
    }
    for (int64_t l = 0; l < P.nlevels; l++) {
        int64_t lo = P.level_off[l], nl = P.level_off[l + 1] - lo;
        if (nl == 0) continue;
        int64_t pbytes = (level_poff_[l + 1] - level_poff_[l]) * sizeof(T);
        if (pbytes > 0) RFG_CUDA(cudaMemsetAsync(panel + level_poff_[l], 0, pbytes, stream_));
        int64_t maxu = 0;
        for (int64_t i = lo; i < lo + nl; i++) maxu = std::max(maxu, P.fronts[P.level_order[i]].u);
        const unsigned zy = (unsigned)std::min<int64_t>(256, std::max<int64_t>(1, (maxu + 31) / 32));
        launch_pdl(true, k_zero_update<T>, dim3((unsigned)nl, zy), dim3(256), 0, stream_, upd,
                   (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, lo);
        mark(0);
        int64_t s0 = scatter_.level_seg[l], s1 = scatter_.level_seg[l + 1];
        if (s1 > s0) {
            int64_t nb = std::min<int64_t>((s1 - s0 + 255) / 256, 148 * 16);
            launch_pdl(true, k_scatter<T>, dim3((unsigned)nb), dim3(256), 0, stream_, panel, (const double*)src_,
                       (const int64_t*)dp_.seg_dst, (const int64_t*)dp_.seg_ptr, (const int64_t*)dp_.seg_src, s0, s1);
            launches++;
            mark(0);
        }
        launch_pdl(true, k_capture_diag<T>, dim3((unsigned)nl), dim3(128), 0, stream_, (const T*)panel, adiag_,
                   (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, lo);
        launches += 2;
        mark(0);
        for (int r = 0; r < 2; r++) {
            const DXadd& x = P.xadd[2 * l + r];
            if (x.fnblk == 0) continue;
            launch_pdl(true, k_extend_add<T>, dim3((unsigned)x.fnblk), dim3(256), 0, stream_, panel, upd,
                       (const DFront*)dp_.fronts, (const int64_t*)(dp_.xadd_child + x.off),
                       (const int64_t*)(dp_.xadd_fpre + x.fpre_off), x.nchild, (const int32_t*)dp_.emap, status_);
            launches++;
            mark(1);
        }
        for (int64_t si = P.step_off[l]; si < P.step_off[l + 1]; si++) {
            const DStep& st = P.steps[si];
            launch_pdl(true, k_pivot_block<T>, dim3((unsigned)st.nact), dim3(PBT), PB_SMEM, stream_, panel, d_,
                       (const double*)adiag_, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                       st.s, status_, linv_);
            launches++;
            mark(2);
            if (st.n_panel > 0) {
                // this outer block's buffer of the split operands
                const int64_t so = use_tc_ ? ((st.s / KO) & 1) * std::max<int64_t>(plan_.max_scr_rows, 1) * NBO : 0;
                launch_pdl(true, k_panel<T, S>, dim3((unsigned)st.n_panel), dim3(256),
                           sizeof(T) == 8 ? PANEL_SMEM_D : PANEL_SMEM, stream_, panel, (const double*)d_,
                           (const double*)linv_, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                           st.nact, (const int64_t*)(dp_.pre_panel + st.pre_off),
                           (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, sw, sl, (const int64_t*)status_,
                           h16_ ? (float*)nullptr : (float*)scr_whi_ + so, (float*)scr_wlo_ + so,
                           (float*)scr_lhi_ + so, (float*)scr_llo_ + so,
                           (const uint8_t*)(dp_.panel_mode + st.pre_off), (const int64_t*)dp_.rows,
                           (const double*)adiag0_, h16_ ? (__half*)scr_uhi_ + so : (__half*)nullptr,
                           (__half*)scr_ulo_ + so, (float*)scr_uscale_,
                           tc_err_);
                launches++;
                mark(3);
            }
            if (st.n_inner > 0) {
                if constexpr (sizeof(T) == 8)
                    launch_pdl(true, k_schur_dmma64<false>, dim3((unsigned)st.n_inner), dim3(128), D64_SMEM, stream_,
                               panel, upd, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                               st.nact, (const int64_t*)(dp_.pre_inner + st.pre_off),
                               (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const double*)sw, (const double*)sl,
                               (const int64_t*)status_);
                else
                    launch_pdl(true, k_schur<T, S, false>, dim3((unsigned)st.n_inner), dim3(256), schur_smem, stream_,
                               panel, upd, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                               st.nact, (const int64_t*)(dp_.pre_inner + st.pre_off),
                               (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const S*)sw, (const S*)sl,
                               (const int64_t*)status_);
                launches++;
                mark(4);
            }
            if (st.n_inner_tc > 0 && use_tc_) {
                launch_schur_tc_inner(st);
                launches++;
                mark(4);
            }
            if (st.n_outer + st.n_outer_tc > 0) {
                if (st.n_outer > 0) {
                    if constexpr (sizeof(T) == 8)
                        launch_pdl(true, k_schur_dmma64<true>, dim3((unsigned)st.n_outer), dim3(128), D64_SMEM,
                                   stream_, panel, upd, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order,
                                   st.fr_off, st.nact, (const int64_t*)(dp_.pre_outer + st.pre_off),
                                   (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const double*)sw,
                                   (const double*)sl, (const int64_t*)status_);
                    else
                        launch_pdl(true, k_schur<T, S, true>, dim3((unsigned)st.n_outer), dim3(256), schur_smem,
                                   stream_, panel, upd, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order,
                                   st.fr_off, st.nact, (const int64_t*)(dp_.pre_outer + st.pre_off),
                                   (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const S*)sw, (const S*)sl,
                                   (const int64_t*)status_);
                    launches++;
                    mark(5);
                }
                if (st.n_outer_tc > 0) {
                    mark(PROF_SKIP);
                    if (use_tc_) {
                        launch_schur_tc(st);
                    } else if constexpr (sizeof(T) == 8) {
                        launch_pdl(true, k_schur_dmma, dim3((unsigned)(2 * st.n_outer_tc)), dim3(DM_THREADS), DM_SMEM, stream_,
                                   panel, upd, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                                   st.nact, (const int64_t*)(dp_.pre_outer_tc + st.pre_off),
                                   (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const double*)sw,
                                   (const double*)sl, (const int64_t*)status_);
                    } else {
                        launch_pdl(true, k_schur_big<T, S>, dim3((unsigned)st.n_outer_tc), dim3(256), big_smem<S>(),
                                   stream_, panel, upd, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order,
                                   st.fr_off, st.nact, (const int64_t*)(dp_.pre_outer_tc + st.pre_off),
                                   (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const S*)sw, (const S*)sl,
                                   (const int64_t*)status_);
                    }
                    launches++;
                    mark(6);
                    nprof += profile_ ? 1 : 0;
                }
            }
        }
    }
    RFG_CUDA(cudaGetLastError());
    last_factor.launches = launches;
    last_factor.schur_launches = nprof;
}

int64_t Engine::factor(const double* src, bool on_device) {
    if (nsrc_ > 0) {
        if (on_device)
            RFG_CUDA(cudaMemcpyAsync(src_, src, nsrc_ * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        else
            host_upload(src_, src, nsrc_ * sizeof(double), stream_);
    }
    RFG_CUDA(cudaEventRecord(ev0_, stream_));
    // The first numeric phase of an engine is launched directly: a handle that is factored
    // once (and freed) would not win back the cost of capturing and instantiating the
    // graph. Later calls capture it once and replay it.
    const bool direct = factor_calls_++ == 0 && !factor_graph_[profile_];
    if (use_graphs_ && !direct) {
        // with profiling on, the phase events are recorded by event nodes of the graph
        cudaGraphExec_t& ex = factor_graph_[profile_];
        if (!ex) {
            cudaGraph_t g;
            RFG_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
            if (prec_ == PREC_FP64)
                factor_impl<double>();
            else
                factor_impl<float>();
            RFG_CUDA(cudaStreamEndCapture(stream_, &g));
            RFG_CUDA(cudaGraphInstantiate(&ex, g, 0));
            RFG_CUDA(cudaGraphDestroy(g));
            prof_phase_graph_[profile_] = prof_phase_;
        }
        prof_phase_ = prof_phase_graph_[profile_];
        RFG_CUDA(cudaGraphLaunch(ex, stream_));
    } else if (prec_ == PREC_FP64) {
        factor_impl<double>();
    } else {
        factor_impl<float>();
    }
    RFG_CUDA(cudaEventRecord(ev1_, stream_));
    std::vector<int64_t> st(plan_.nfronts);
    if (plan_.nfronts > 0)
        RFG_CUDA(cudaMemcpyAsync(st.data(), status_, plan_.nfronts * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
    int tc_err = 0;
    if (tc_err_) RFG_CUDA(cudaMemcpyAsync(&tc_err, tc_err_, sizeof(int), cudaMemcpyDeviceToHost, stream_));
    RFG_CUDA(cudaStreamSynchronize(stream_));
    if (tc_err == 21 && h16_) {
        // a row of the FP16 split left its range (a front whose diagonal no longer bounds
        // its rows, e.g. after heavy cancellation): this engine factors with the TF32 split
        h16_ = false;
        RFG_CUDA(cudaMemsetAsync(tc_err_, 0, sizeof(int), stream_));
        for (cudaGraphExec_t& g : factor_graph_)
            if (g) {
                RFG_CUDA(cudaGraphExecDestroy(g));
                g = nullptr;
            }
        return factor(src, on_device);
    }
    if (tc_err)
        throw CudaError("tensor-core Schur update: a bounded wait gave up (code " + std::to_string(tc_err) +
                        "); the factor is invalid");
    float ms = 0.f;
    RFG_CUDA(cudaEventElapsedTime(&ms, ev0_, ev1_));
    last_factor.t_factor_ms = ms;
    last_factor.schur_ms = 0.0;
    last_factor.schur_flops = plan_.outer_big_flops;
    last_factor.schur_entries = plan_.outer_big_entries;
    last_factor.schur_opvals = plan_.outer_big_opvals;
    last_factor.h2d_bytes = on_device ? 0 : nsrc_ * (int64_t)sizeof(double);
    for (double& v : last_factor.phase_ms) v = 0.0;
    for (size_t i = 0; i < prof_phase_.size(); i++) {
        float e = 0.f;
        RFG_CUDA(cudaEventElapsedTime(&e, prof_ev_[i], prof_ev_[i + 1]));
        if (prof_phase_[i] < 7) last_factor.phase_ms[prof_phase_[i]] += e;
    }
    last_factor.schur_ms = last_factor.phase_ms[6];
    // the first failing front in postorder among those whose subtree was factored
    for (int64_t t = 0; t < plan_.nfronts; t++)
        if (st[t] >= 0) return st[t];
    return -1;
}

}  // namespace rfg
