// Unsymmetric multifrontal LU on the GPU (see lu.h). Compiled with -fmad=false:
// products and sums are rounded one by one, as in the reference.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <stdexcept>

#include "engine.h"
#include "lu.h"
#include "plan.h"

namespace rfg {

namespace {

constexpr double ZERO_TOL = 1e-12;  // src/sparse/indef.rs:29 (used by src/sparse/lu.rs:19)
constexpr int LKB = 64;             // src/sparse/lu.rs:23
constexpr int ET = 512;             // threads of the elimination CTA

struct LFrontDesc {
    double* F;          // m × m row-major, both triangles
    int64_t m, kf, k, start, u;
    int64_t* fs;        // kf variables, permuted by the elimination
    int64_t* gidx;      // rows of L21 / columns of U12: fs[npiv..kf] then the front's rows
    int64_t* rperm;     // root: row permutation of the partial-pivoting block (kf − npiv entries)
    int64_t nchild;
    int64_t child[2];
    const int64_t* cmap[2];  // local index in this front of each row of the child's update matrix
    int64_t npiv;       // out: pivots taken by the threshold pivoting
    int64_t nroot;      // out: size of the root's partial-pivoting block (0 elsewhere)
    int64_t err;        // out: equation at which the root is singular, or −1
    int32_t root;
    int32_t done;       // no further block of this front
    int64_t p, width;   // next pivot, width of the next block
    int64_t blk_p0, blk_npb, blk_b1;  // the last block: first pivot, pivots taken, end
};

__device__ __forceinline__ double block_max(double v, double* red) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < ET / 32; i++) r = fmax(r, red[i]);
    return r;
}

// the largest value (strictly greater wins, so the first index among equal maxima)
__device__ __forceinline__ void block_argmax(double v, int64_t idx, double* redv, int64_t* redi, double* outv,
                                             int64_t* outi) {
    for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int64_t oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
        }
    }
    const int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) {
        redv[w] = v;
        redi[w] = idx;
    }
    __syncthreads();
    double bv = redv[0];
    int64_t bi = redi[0];
    for (int i = 1; i < ET / 32; i++)
        if (redv[i] > bv || (redv[i] == bv && redi[i] < bi)) {
            bv = redv[i];
            bi = redi[i];
        }
    *outv = bv;
    *outi = bi;
}

// symmetric swap of p and q (src/sparse/lu.rs:272-283): rows, then columns, then the variables
__device__ void swap_pq(double* F, int64_t m, int64_t* fs, int64_t p, int64_t q) {
    if (p == q) return;
    for (int64_t c = threadIdx.x; c < m; c += ET) {
        const double t = F[p * m + c];
        F[p * m + c] = F[q * m + c];
        F[q * m + c] = t;
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < m; i += ET) {
        const double t = F[i * m + p];
        F[i * m + p] = F[i * m + q];
        F[i * m + q] = t;
    }
    if (threadIdx.x == 0) {
        const int64_t t = fs[p];
        fs[p] = fs[q];
        fs[q] = t;
    }
    __syncthreads();
}

// Assembly of a level on all SMs (src/sparse/lu.rs:176-200), the fronts zeroed before: the
// original entries of the fronts' own columns (every position receives at most one, from the
// lower triangle or its transposed upper partner), then each child slot's update matrices in
// its own launch, so that a position shared by both children sums child 0 before child 1.
__global__ void k_lu_asm_orig(double* __restrict__ Fbuf, const int64_t* __restrict__ dst,
                              const int64_t* __restrict__ dst_t, const int64_t* __restrict__ src, int64_t nent,
                              const double* __restrict__ lval, const double* __restrict__ uval) {
    for (int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; z < nent; z += (int64_t)gridDim.x * blockDim.x) {
        Fbuf[dst[z]] += lval[src[z]];
        if (dst_t[z] >= 0) Fbuf[dst_t[z]] += uval[src[z]];
    }
}

// one warp per row of child slot ci's update matrix; cpre: prefix of those rows over the level
__global__ void __launch_bounds__(256) k_lu_asm_child(const LFrontDesc* __restrict__ desc,
                                                      const int64_t* __restrict__ ids, int64_t nl,
                                                      const int64_t* __restrict__ cpre, int ci) {
    const int lane = threadIdx.x & 31;
    const int64_t total = cpre[nl];
    for (int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); w < total; w += (int64_t)gridDim.x * 8) {
        int64_t lo = 0, hi = nl;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (cpre[mid] <= w)
                lo = mid;
            else
                hi = mid;
        }
        const LFrontDesc& f = desc[ids[lo]];
        const LFrontDesc& c = desc[f.child[ci]];
        const int64_t x = w - cpre[lo];
        const int64_t nr = c.m - c.npiv;
        const int64_t* map = f.cmap[ci];
        double* row = f.F + map[x] * f.m;
        const double* src = c.F + (c.npiv + x) * c.m + c.npiv;
        for (int64_t y = lane; y < nr; y += 32) row[map[y]] += src[y];
    }
}

constexpr int LCMAX = 1024;           // block columns whose maxima are kept in shared memory
constexpr int LSMEM_VEC_MAX = 12288;  // multipliers kept in shared memory up to this many rows

// Column maxima of the block's candidate columns j = c0 + x (x < ncols) over the rows
// i ∈ [r0, m), i ≠ j, into cmax (8 row lanes × 64 columns per pass). With lc non-null the
// same pass first applies the elimination of pivot p to those columns (F[i][j] −= l_i·u_j,
// rows with l_i = 0 untouched: src/sparse/lu.rs:318-328) and takes the maxima of the new
// values.
__device__ void lu_cols_pass(double* F, int64_t m, int64_t r0, int64_t c0, int64_t ncols, const double* lc,
                             const double* uc, int64_t p, double* cmax, double* red8) {
    const int cl = threadIdx.x & 63, rl = threadIdx.x >> 6;
    for (int64_t x0 = 0; x0 < ncols; x0 += 64) {
        const int64_t x = x0 + cl;
        double mx = 0.0;
        if (x < ncols) {
            const int64_t j = c0 + x;
            const double ux = lc ? uc[x] : 0.0;
            int64_t i = r0 + rl;
            // UR rows in flight per thread: the loads first, then the updates
            constexpr int UR = 8;
            for (; i + (UR - 1) * (ET / 64) < m; i += UR * (ET / 64)) {
                double v[UR];
#pragma unroll
                for (int u = 0; u < UR; u++) v[u] = F[(i + u * (ET / 64)) * m + j];
#pragma unroll
                for (int u = 0; u < UR; u++) {
                    const int64_t ii = i + u * (ET / 64);
                    if (lc) {
                        const double li = lc[ii - p - 1];
                        if (li != 0.0) {
                            v[u] -= li * ux;
                            F[ii * m + j] = v[u];
                        }
                    }
                    if (ii != j) mx = fmax(mx, fabs(v[u]));
                }
            }
            for (; i < m; i += ET / 64) {
                double v = F[i * m + j];
                if (lc) {
                    const double li = lc[i - p - 1];
                    if (li != 0.0) {
                        v -= li * ux;
                        F[i * m + j] = v;
                    }
                }
                if (i != j) mx = fmax(mx, fabs(v));
            }
        }
        red8[rl * 64 + cl] = mx;
        __syncthreads();
        if (rl == 0 && x < ncols && x < LCMAX) {
            double r = red8[cl];
            for (int q = 1; q < ET / 64; q++) r = fmax(r, red8[q * 64 + cl]);
            cmax[x] = r;
        }
        __syncthreads();
    }
}

// The end of a block round (src/sparse/lu.rs:351-357): the width for the next block, and
// at the root, once no candidate passes, the partial-pivoting LU of the rest S = F[p.., p..]
// (:210-222, :246-270: first maximum of the column, the same singularity test) in place; the
// row swaps stay inside S, the computed L21/U12 keep their rows. Then the front's state. One
// CTA (ET threads).
__device__ void lu_block_finish(LFrontDesc* desc, int64_t id, const LFrontDesc& f, const double* scale, int64_t p0,
                                int64_t p, int64_t b1, int64_t width, double* lcol, double* red, int64_t* redi) {
    double* F = f.F;
    const int64_t m = f.m, kf = f.kf;
    int64_t* fs = f.fs;
    int64_t err = -1, nroot = 0;
    const int64_t npb = p - p0;
    bool done = p >= kf;
    if (npb == 0) {
        if (b1 == kf) {
            done = true;
            if (p < kf && f.root) {
                const int64_t r = kf - p;
                int64_t* perm = f.rperm;
                for (int64_t i = threadIdx.x; i < r; i += ET) perm[i] = i;
                __syncthreads();
                for (int64_t q = 0; q < r; q++) {
                    double v = 0.0;
                    int64_t vi = INT64_MAX;
                    for (int64_t i = q + threadIdx.x; i < r; i += ET) {
                        const double a = fabs(F[(p + i) * m + p + q]);
                        if (a > v) {
                            v = a;
                            vi = i;
                        }
                    }
                    double big;
                    int64_t bi;
                    block_argmax(v, vi, red, redi, &big, &bi);
                    if (!(big > ZERO_TOL * scale[fs[p + q]])) {
                        err = fs[p + q];
                        break;
                    }
                    if (bi != q) {
                        for (int64_t c = threadIdx.x; c < r; c += ET) {
                            const double t = F[(p + q) * m + p + c];
                            F[(p + q) * m + p + c] = F[(p + bi) * m + p + c];
                            F[(p + bi) * m + p + c] = t;
                        }
                        if (threadIdx.x == 0) {
                            const int64_t t = perm[q];
                            perm[q] = perm[bi];
                            perm[bi] = t;
                        }
                        __syncthreads();
                    }
                    const double dq = F[(p + q) * m + p + q];
                    for (int64_t i = q + 1 + threadIdx.x; i < r; i += ET) {
                        const double l = F[(p + i) * m + p + q] / dq;
                        F[(p + i) * m + p + q] = l;
                        lcol[i] = l;
                    }
                    __syncthreads();
                    const int64_t w = r - q - 1;
                    for (int64_t z = threadIdx.x; z < w * w; z += ET) {
                        const int64_t i = q + 1 + z / w, c = q + 1 + z % w;
                        const double l = lcol[i];
                        if (l != 0.0) F[(p + i) * m + p + c] -= l * F[(p + q) * m + p + c];
                    }
                    __syncthreads();
                }
                nroot = r;
            }
        } else {
            width *= 2;
        }
    } else {
        width = LKB;
    }
    if (threadIdx.x == 0) {
        desc[id].p = p;
        desc[id].width = width;
        desc[id].done = done ? 1 : 0;
        desc[id].blk_p0 = p0;
        desc[id].blk_npb = npb;
        desc[id].blk_b1 = b1;
        desc[id].npiv = p;
        desc[id].nroot = nroot;
        desc[id].err = err;
    }
}

// One block of the threshold pivoting of one front on one CTA (src/sparse/lu.rs:292-330):
// for each position p of the block [p0, b1), the first candidate j in [p, b1) with
// |a_jj| > ZERO_TOL·scale and |a_jj| >= u·max_{i >= p, i ≠ j} |a_ij|, swapped to p and
// eliminated with the eager update of the block's columns of every row (the rest of the rows
// inside the block: k_lu_rowblock). The column maxima of the candidates come out of the
// previous elimination's update pass (one pass over the block's columns per pivot). A block
// that takes no pivot doubles the width (:351-357). The state stays in the descriptor
// between rounds.
__device__ void lu_block_cta(LFrontDesc* desc, int64_t id, const double* scale, double thr, double* urow,
                             double* lcol, double* cmax, double* red8, double* red, int64_t* redi, int64_t* s_pick) {
    const LFrontDesc f = desc[id];
    double* F = f.F;
    const int64_t m = f.m, kf = f.kf;
    int64_t* fs = f.fs;
    int64_t p = f.p;
    const int64_t width = f.width;
    const int64_t p0 = p;
    const int64_t b1 = min(p + width, kf);
    // maxima of the candidate columns [p, b1) over the rows [p, m) before the first pivot
    lu_cols_pass(F, m, p, p, b1 - p, nullptr, nullptr, p, cmax, red8);
    while (p < b1) {
        if (threadIdx.x == 0) *s_pick = -1;
        for (int64_t j = p; j < b1; j++) {
            const double ajj = fabs(F[j * m + j]);
            if (!(ajj > ZERO_TOL * scale[fs[j]])) continue;
            double g;
            if (j - p < LCMAX) {
                g = cmax[j - p];
            } else {
                g = 0.0;
                for (int64_t i = p + threadIdx.x; i < m; i += ET)
                    if (i != j) g = fmax(g, fabs(F[i * m + j]));
                g = block_max(g, red);
            }
            if (ajj >= thr * g) {
                if (threadIdx.x == 0) *s_pick = j;
                break;
            }
        }
        __syncthreads();
        const int64_t j = *s_pick;
        __syncthreads();
        if (j < 0) break;
        swap_pq(F, m, fs, p, j);
        const double dp = F[p * m + p];
        const int64_t wshort = b1 - p - 1;
        for (int64_t x = threadIdx.x; x < wshort; x += ET) urow[x] = F[p * m + p + 1 + x];
        for (int64_t i = p + 1 + threadIdx.x; i < m; i += ET) {
            const double li = F[i * m + p] / dp;
            F[i * m + p] = li;
            lcol[i - p - 1] = li;
        }
        __syncthreads();
        // the block's columns of every row below p, with the maxima of the next candidates; the
        // columns beyond the block of the rows inside it follow in k_lu_rowblock, once the
        // block's pivots are known (the same products and differences, in the same order)
        lu_cols_pass(F, m, p + 1, p + 1, wshort, lcol, urow, p, cmax, red8);
        p += 1;
    }
    __syncthreads();
    lu_block_finish(desc, id, f, scale, p0, p, b1, width, lcol, red, redi);
}

// one CTA per front (the level's smaller fronts)
__global__ void __launch_bounds__(ET) k_lu_block(LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                                 const double* __restrict__ scale, double thr,
                                                 double* __restrict__ wbuf, int64_t wstride) {
    extern __shared__ double lsm[];
    __shared__ double red[ET / 32];
    __shared__ int64_t redi[ET / 32];
    __shared__ int64_t s_pick;
    __shared__ double cmax[LCMAX];
    __shared__ double red8[ET];
    const int64_t id = ids[blockIdx.x];
    if (desc[id].done) {
        if (threadIdx.x == 0) desc[id].blk_npb = 0;
        return;
    }
    // the pivot row's block columns and the multipliers: shared memory when they fit
    double* urow = wstride <= LSMEM_VEC_MAX ? lsm : wbuf + blockIdx.x * 2 * wstride;
    double* lcol = urow + wstride;
    lu_block_cta(desc, id, scale, thr, urow, lcol, cmax, red8, red, redi, &s_pick);
}

// The same block on a cluster of LCS CTAs for the level's large fronts: each CTA owns a
// slice of the rows; per pivot the candidates' column maxima are combined from the CTAs'
// partial maxima (distributed shared memory), every CTA takes the same decision, the row
// swap is split over the CTAs by columns and the column swap by rows, and each CTA eliminates
// its own rows (the same products and differences per entry as on one CTA). Blocks wider
// than LPW candidates, and the root's partial pivoting, run on the cluster's first CTA.
constexpr int LCS = 8;     // CTAs per cluster
constexpr int LPW = 64;    // candidates per block handled by the whole cluster
__global__ void __cluster_dims__(LCS, 1, 1) __launch_bounds__(ET)
    k_lu_block_cl(LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, const double* __restrict__ scale,
                  double thr, double* __restrict__ wbuf, int64_t wstride) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ double red[ET / 32];
    __shared__ int64_t redi[ET / 32];
    __shared__ int64_t s_pick;
    __shared__ double cmax[LCMAX];
    __shared__ double part[LPW];  // this CTA's maxima of the candidates over its rows
    __shared__ double red8[ET];
    __shared__ double urow[LPW];
    const int rank = (int)cluster.block_rank();
    const int64_t slot = blockIdx.x / LCS;
    const int64_t id = ids[slot];
    double* wb = wbuf + slot * 2 * wstride;
    if (desc[id].done) {
        if (rank == 0 && threadIdx.x == 0) desc[id].blk_npb = 0;
        return;  // the whole cluster returns: no distributed shared memory was touched
    }
    const LFrontDesc f = desc[id];
    const int64_t m = f.m, kf = f.kf;
    const int64_t p0 = f.p;
    const int64_t b1 = min(p0 + f.width, kf);
    if (b1 - p0 > LPW) {
        // a block that has grown past LPW candidates: on one CTA (uses no cluster barrier)
        if (rank == 0) lu_block_cta(desc, id, scale, thr, wb, wb + wstride, cmax, red8, red, redi, &s_pick);
        return;
    }
    double* F = f.F;
    int64_t* fs = f.fs;
    double* lcol = wb + wstride;  // multipliers of rows p+1.. (each CTA writes its own rows)
    // rows of this CTA: [lo, hi) of the panel rows [p0, m); columns swaps cover all rows [0, m)
    const int64_t S = (m - p0 + LCS - 1) / LCS;
    const int64_t lo = min(p0 + rank * S, m), hi = min(lo + S, m);
    const int64_t SA = (m + LCS - 1) / LCS;
    const int64_t alo = min(rank * SA, m), ahi = min(alo + SA, m);
    const int64_t CW = (m + LCS - 1) / LCS;  // columns of the row swap per CTA
    const int64_t clo = min(rank * CW, m), chi = min(clo + CW, m);
    const int cl = threadIdx.x & 63, rl = threadIdx.x >> 6;
    // partial maxima of the columns c0 + x (x < ncols) over this CTA's rows i >= r0, i ≠ column
    auto partial_pass = [&](int64_t r0, int64_t c0, int64_t ncols, bool elim, int64_t p) {
        double mx = 0.0;
        const int64_t x = cl;
        if (x < ncols) {
            const int64_t j = c0 + x;
            const double ux = elim ? urow[x] : 0.0;
            for (int64_t i = max(lo, r0) + rl; i < hi; i += ET / 64) {
                double v = F[i * m + j];
                if (elim) {
                    const double li = lcol[i - p - 1];
                    if (li != 0.0) {
                        v -= li * ux;
                        F[i * m + j] = v;
                    }
                }
                if (i != j) mx = fmax(mx, fabs(v));
            }
        }
        red8[rl * 64 + cl] = mx;
        __syncthreads();
        if (rl == 0) {
            double r = red8[cl];
            for (int q = 1; q < ET / 64; q++) r = fmax(r, red8[q * 64 + cl]);
            part[cl] = r;
        }
        __syncthreads();
    };
    int64_t p = p0;
    partial_pass(p, p, b1 - p, false, p);
    cluster.sync();
    while (p < b1) {
        // the candidates' maxima: the largest of the CTAs' partial maxima
        if (threadIdx.x < b1 - p) {
            double g = 0.0;
            for (int r = 0; r < LCS; r++) g = fmax(g, cluster.map_shared_rank(part, r)[threadIdx.x]);
            cmax[threadIdx.x] = g;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            s_pick = -1;
            for (int64_t j = p; j < b1; j++) {
                const double ajj = fabs(F[j * m + j]);
                if (!(ajj > ZERO_TOL * scale[fs[j]])) continue;
                if (ajj >= thr * cmax[j - p]) {
                    s_pick = j;
                    break;
                }
            }
        }
        __syncthreads();
        const int64_t j = s_pick;
        // every CTA has read the partial maxima before any of them is overwritten
        cluster.sync();
        if (j < 0) break;
        if (j != p) {
            // rows p and j, this CTA's share of the columns; then columns p and j of its rows
            for (int64_t c = clo + threadIdx.x; c < chi; c += ET) {
                const double t = F[p * m + c];
                F[p * m + c] = F[j * m + c];
                F[j * m + c] = t;
            }
            cluster.sync();
            for (int64_t i = alo + threadIdx.x; i < ahi; i += ET) {
                const double t = F[i * m + p];
                F[i * m + p] = F[i * m + j];
                F[i * m + j] = t;
            }
            if (rank == 0 && threadIdx.x == 0) {
                const int64_t t = fs[p];
                fs[p] = fs[j];
                fs[j] = t;
            }
            cluster.sync();
        }
        const double dp = F[p * m + p];
        const int64_t wshort = b1 - p - 1;
        if (threadIdx.x < wshort) urow[threadIdx.x] = F[p * m + p + 1 + threadIdx.x];
        for (int64_t i = max(lo, p + 1) + threadIdx.x; i < hi; i += ET) {
            const double li = F[i * m + p] / dp;
            F[i * m + p] = li;
            lcol[i - p - 1] = li;
        }
        __syncthreads();
        partial_pass(p + 1, p + 1, wshort, true, p);
        // the pivot row is read by every CTA before the next swap may change it
        cluster.sync();
        p += 1;
    }
    // no CTA leaves while another may still read its partial maxima
    cluster.sync();
    if (rank == 0) lu_block_finish(desc, id, f, scale, p0, p, b1, f.width, lcol, red, redi);
}

// tiles of the trailing update of each front's last block (64×64 tiles of [b1, m)²; none
// when the block took no pivot or nothing trails it): their prefix over the level's
// fronts, and the number of fronts not yet done
constexpr int LTT = 64;
constexpr int LRB = 128;  // columns per CTA of the row-block update
__device__ __forceinline__ int64_t cta_scan(int64_t v, int64_t* wsum, int64_t* total) {
    // inclusive scan of v over the CTA; *total = the CTA's sum
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int64_t inc = v;
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) wsum[w] = inc;
    __syncthreads();
    int64_t woff = 0, tot = 0;
    for (int q = 0; q < (int)(blockDim.x >> 5); q++) {
        if (q < w) woff += wsum[q];
        tot += wsum[q];
    }
    __syncthreads();
    *total = tot;
    return woff + inc;
}

// per front of the level, for its last block: the 64×64 tiles of the trailing update ([b1, m)²)
// and the 128-column tiles of the row-block update ([b1, m) columns of the block's rows); none
// when the block took no pivot or nothing trails it. Their prefixes over the level's fronts,
// and the number of fronts not yet done.
__global__ void __launch_bounds__(1024) k_lu_tiles(const LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                                   int64_t nl, int64_t* __restrict__ tpre, int64_t* __restrict__ rpre,
                                                   int64_t* __restrict__ nactive) {
    __shared__ int64_t wsum[32];
    __shared__ int64_t carry_t, carry_r, active;
    if (threadIdx.x == 0) {
        carry_t = 0;
        carry_r = 0;
        active = 0;
        tpre[0] = 0;
        rpre[0] = 0;
    }
    __syncthreads();
    for (int64_t c0 = 0; c0 < nl; c0 += blockDim.x) {
        const int64_t ii = c0 + threadIdx.x;
        int64_t v = 0, vr = 0;
        if (ii < nl) {
            const LFrontDesc& f = desc[ids[ii]];
            if (f.blk_npb > 0 && f.blk_b1 < f.m) {
                const int64_t T = (f.m - f.blk_b1 + LTT - 1) / LTT;
                v = T * T;
                if (f.blk_b1 - f.blk_p0 > 1) vr = (f.m - f.blk_b1 + LRB - 1) / LRB;
            }
            if (!f.done) atomicAdd((unsigned long long*)&active, 1ull);
        }
        int64_t tt, tr;
        const int64_t it = cta_scan(v, wsum, &tt);
        const int64_t ir = cta_scan(vr, wsum, &tr);
        if (ii < nl) {
            tpre[ii + 1] = carry_t + it;
            rpre[ii + 1] = carry_r + ir;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            carry_t += tt;
            carry_r += tr;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *nactive = active;
}

// The columns beyond the block of the rows inside it (src/sparse/lu.rs:318-328, deferred to
// the end of the block): F[i][c] −= F[i][q]·F[q][c] for the block's rows i, every column
// c >= b1 and the block's pivots q < i in order — for each (i, c) the reference's sequence
// of products and differences, row q final before row i uses it. One thread per column,
// 128 columns per CTA, the block's multipliers in shared memory.
constexpr int LRB_MAXW = 64;
constexpr size_t LRB_SMEM = (size_t)LRB_MAXW * LRB * sizeof(double);
__global__ void __launch_bounds__(LRB) k_lu_rowblock(const LFrontDesc* __restrict__ desc,
                                                    const int64_t* __restrict__ ids, int64_t nl,
                                                    const int64_t* __restrict__ rpre) {
    __shared__ double Lb[LRB_MAXW][LRB_MAXW + 1];
    extern __shared__ double Cs[];  // [LRB_MAXW][LRB]: the tile's columns of the block's rows
    const int64_t total = rpre[nl];
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        int64_t lo = 0, hi = nl;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (rpre[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        const LFrontDesc& fr = desc[ids[lo]];
        double* F = fr.F;
        const int64_t m = fr.m, b1 = fr.blk_b1, p0 = fr.blk_p0, pe = p0 + fr.blk_npb;
        const int64_t c = b1 + (t - rpre[lo]) * LRB + threadIdx.x;
        const int64_t nb = b1 - p0;  // rows of the block
        if (nb <= LRB_MAXW) {
            // the usual block: its multipliers and the tile's columns of its rows in shared memory
            const int64_t npb = pe - p0;
            __syncthreads();
            for (int z = threadIdx.x; z < LRB_MAXW * LRB_MAXW; z += LRB) {
                const int a = z / LRB_MAXW, b = z % LRB_MAXW;
                Lb[a][b] = (a < nb && b < npb) ? F[(p0 + a) * m + p0 + b] : 0.0;
            }
            const int64_t cbase = b1 + (t - rpre[lo]) * LRB;
            for (int z = threadIdx.x; z < nb * LRB; z += LRB) {
                const int a = z / LRB, x = z % LRB;
                if (cbase + x < m) Cs[a * LRB + x] = F[(p0 + a) * m + cbase + x];
            }
            __syncthreads();
            if (c < m) {
                for (int a = 1; a < nb; a++) {
                    const int qend = (int)min((int64_t)a, npb);
                    double v = Cs[a * LRB + threadIdx.x];
                    for (int b = 0; b < qend; b++) {
                        const double l = Lb[a][b];
                        if (l != 0.0) v -= l * Cs[b * LRB + threadIdx.x];
                    }
                    Cs[a * LRB + threadIdx.x] = v;
                }
            }
            __syncthreads();
            for (int z = threadIdx.x; z < nb * LRB; z += LRB) {
                const int a = z / LRB, x = z % LRB;
                if (a > 0 && cbase + x < m) F[(p0 + a) * m + cbase + x] = Cs[a * LRB + x];
            }
            continue;
        }
        // multipliers of the block's rows, in chunks of LRB_MAXW rows (a doubled block is wider)
        for (int64_t i0 = 0; i0 < nb; i0 += LRB_MAXW) {
            // rows i in [p0 + i0, p0 + i0 + LRB_MAXW) depend on every earlier row of the block:
            // the chunks run in order, each row once
            for (int64_t q0 = 0; q0 < min(i0 + LRB_MAXW, pe - p0); q0 += LRB_MAXW) {
                __syncthreads();
                for (int z = threadIdx.x; z < LRB_MAXW * LRB_MAXW; z += LRB) {
                    const int a = z / LRB_MAXW, b = z % LRB_MAXW;
                    const int64_t i = p0 + i0 + a, q = p0 + q0 + b;
                    Lb[a][b] = (i < b1 && q < pe) ? F[i * m + q] : 0.0;
                }
                __syncthreads();
                if (c < m) {
                    for (int a = 0; a < LRB_MAXW; a++) {
                        const int64_t i = p0 + i0 + a;
                        if (i >= b1) break;
                        const int64_t qend = min(i, pe);  // pivots before row i
                        if (p0 + q0 >= qend) continue;
                        double v = F[i * m + c];
                        for (int b = 0; b < LRB_MAXW; b++) {
                            const int64_t q = p0 + q0 + b;
                            if (q >= qend) break;
                            const double l = Lb[a][b];
                            if (l != 0.0) v -= l * F[q * m + c];
                        }
                        F[i * m + c] = v;
                    }
                }
            }
        }
        __syncthreads();
    }
}

// F[x][y] −= Σ_q L[x][q]·U[q][y] for b1 <= x, y < m over the block's pivots q in order,
// one fused multiply-add chain per entry from 0 (src/sparse/lu.rs:331-350 through
// src/sparse.rs:329-343). 64×64 tiles, 256 threads with 4×4 entries each, K in chunks of
// 64 through shared memory; CTAs walk the level's tiles.
constexpr int LTK = 64;
constexpr size_t LTRAIL_SMEM = 2 * LTT * (LTK + 1) * sizeof(double);
__global__ void __launch_bounds__(256) k_lu_trailing(const LFrontDesc* __restrict__ desc,
                                                     const int64_t* __restrict__ ids, int64_t nl,
                                                     const int64_t* __restrict__ tpre) {
    extern __shared__ double lts[];
    double* Ls = lts;                    // [LTT][LTK + 1]: L of the tile's rows
    double* Us = lts + LTT * (LTK + 1);  // [LTT][LTK + 1]: U of the tile's columns (transposed)
    const int64_t total = tpre[nl];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    for (int64_t t = blockIdx.x; t < total; t += gridDim.x) {
        int64_t lo = 0, hi = nl;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (tpre[mid] <= t)
                lo = mid;
            else
                hi = mid;
        }
        const LFrontDesc& fr = desc[ids[lo]];
        double* F = fr.F;
        const int64_t m = fr.m, b1 = fr.blk_b1, p0 = fr.blk_p0, npb = fr.blk_npb;
        const int64_t T = (m - b1 + LTT - 1) / LTT;
        const int64_t lt = t - tpre[lo];
        const int64_t x0 = b1 + (lt / T) * LTT, y0 = b1 + (lt % T) * LTT;
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][c] = 0.0;
        for (int64_t k0 = 0; k0 < npb; k0 += LTK) {
            const int kc = (int)min((int64_t)LTK, npb - k0);
            __syncthreads();
            for (int z = threadIdx.x; z < LTT * LTK; z += 256) {
                const int r = z / LTK, q = z % LTK;
                double lv = 0.0;
                if (q < kc && x0 + r < m) lv = F[(x0 + r) * m + p0 + k0 + q];
                Ls[r * (LTK + 1) + q] = lv;
            }
            for (int z = threadIdx.x; z < LTT * LTK; z += 256) {
                const int q = z / LTT, c = z % LTT;
                double uv = 0.0;
                if (q < kc && y0 + c < m) uv = F[(p0 + k0 + q) * m + y0 + c];
                Us[c * (LTK + 1) + q] = uv;
            }
            __syncthreads();
            for (int q = 0; q < kc; q++) {
                double lr[4], uc[4];
#pragma unroll
                for (int a = 0; a < 4; a++) lr[a] = Ls[(ty + 16 * a) * (LTK + 1) + q];
#pragma unroll
                for (int c = 0; c < 4; c++) uc[c] = Us[(tx + 16 * c) * (LTK + 1) + q];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[a][c] = fma(lr[a], uc[c], acc[a][c]);
            }
        }
        __syncthreads();
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int64_t x = x0 + ty + 16 * a;
            if (x >= m) continue;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int64_t y = y0 + tx + 16 * c;
                if (y < m) F[x * m + y] -= acc[a][c];
            }
        }
    }
}

// ---- solve (src/sparse/lu.rs:364-402): forward up the levels, backward down ----
__global__ void __launch_bounds__(ET) k_lu_fwd(const LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                               double* X, int nrhs, double* __restrict__ xbuf, int64_t xstride) {
    const LFrontDesc f = desc[ids[blockIdx.x]];
    const int64_t k = f.npiv, nr = f.m - k, m = f.m;
    double* xp = xbuf + blockIdx.x * xstride;
    for (int j = 0; j < nrhs; j++) {
        for (int64_t i = threadIdx.x; i < k; i += ET) xp[i] = X[f.fs[i] * nrhs + j];
        __syncthreads();
        // unit lower triangle of the pivot block, by columns
        for (int64_t i = 0; i < k; i++) {
            const double xi = xp[i];
            for (int64_t q = i + 1 + threadIdx.x; q < k; q += ET) xp[q] -= f.F[q * m + i] * xi;
            __syncthreads();
        }
        for (int64_t r = threadIdx.x; r < nr; r += ET) {
            const double* l = f.F + (k + r) * m;
            double t = 0.0;
            for (int64_t q = 0; q < k; q++) t += l[q] * xp[q];
            atomicAdd(&X[f.gidx[r] * nrhs + j], -t);
        }
        for (int64_t i = threadIdx.x; i < k; i += ET) X[f.fs[i] * nrhs + j] = xp[i];
        __syncthreads();
        if (f.nroot > 0) {
            // the root's partial-pivoting block: rows in the order of its permutation
            const int64_t r = f.nroot;
            for (int64_t i = threadIdx.x; i < r; i += ET) xp[i] = X[f.fs[k + f.rperm[i]] * nrhs + j];
            __syncthreads();
            for (int64_t i = 0; i < r; i++) {
                const double xi = xp[i];
                for (int64_t q = i + 1 + threadIdx.x; q < r; q += ET) xp[q] -= f.F[(k + q) * m + k + i] * xi;
                __syncthreads();
            }
            for (int64_t i = threadIdx.x; i < r; i += ET) X[f.fs[k + i] * nrhs + j] = xp[i];
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(ET) k_lu_bwd(const LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                               double* X, int nrhs, double* __restrict__ xbuf, int64_t xstride) {
    __shared__ double s_xi;
    const LFrontDesc f = desc[ids[blockIdx.x]];
    const int64_t k = f.npiv, nr = f.m - k, m = f.m;
    double* xp = xbuf + blockIdx.x * xstride;
    for (int j = 0; j < nrhs; j++) {
        if (f.nroot > 0) {
            // the root's partial-pivoting block first (the reverse of the forward order)
            const int64_t r = f.nroot;
            for (int64_t i = threadIdx.x; i < r; i += ET) xp[i] = X[f.fs[k + i] * nrhs + j];
            __syncthreads();
            for (int64_t i = r - 1; i >= 0; i--) {
                if (threadIdx.x == 0) {
                    s_xi = xp[i] / f.F[(k + i) * m + k + i];
                    xp[i] = s_xi;
                }
                __syncthreads();
                const double xi = s_xi;
                for (int64_t q = threadIdx.x; q < i; q += ET) xp[q] -= f.F[(k + q) * m + k + i] * xi;
                __syncthreads();
            }
            for (int64_t i = threadIdx.x; i < r; i += ET) X[f.fs[k + i] * nrhs + j] = xp[i];
            __syncthreads();
        }
        for (int64_t i = threadIdx.x; i < k; i += ET) {
            double v = X[f.fs[i] * nrhs + j];
            const double* u = f.F + i * m + k;
            for (int64_t r = 0; r < nr; r++) v -= u[r] * X[f.gidx[r] * nrhs + j];
            xp[i] = v;
        }
        __syncthreads();
        for (int64_t i = k - 1; i >= 0; i--) {
            if (threadIdx.x == 0) {
                s_xi = xp[i] / f.F[i * m + i];
                xp[i] = s_xi;
            }
            __syncthreads();
            const double xi = s_xi;
            for (int64_t q = threadIdx.x; q < i; q += ET) xp[q] -= f.F[q * m + i] * xi;
            __syncthreads();
        }
        for (int64_t i = threadIdx.x; i < k; i += ET) X[f.fs[i] * nrhs + j] = xp[i];
        __syncthreads();
    }
}

// The level's results for the host in one copy: pivots taken, root block size and error.
__global__ void k_lu_results(const LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, int64_t nl,
                             int64_t* __restrict__ out) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < nl; ii += (int64_t)gridDim.x * blockDim.x) {
        const LFrontDesc& f = desc[ids[ii]];
        out[3 * ii] = f.npiv;
        out[3 * ii + 1] = f.nroot;
        out[3 * ii + 2] = f.err;
    }
}

// the rows of L21 / columns of U12 of the level's fronts (gbuf + goff[ii])
__global__ void k_lu_set_gidx(LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, int64_t nl,
                              int64_t* __restrict__ gbuf, const int64_t* __restrict__ goff) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < nl; ii += (int64_t)gridDim.x * blockDim.x)
        desc[ids[ii]].gidx = gbuf + goff[ii];
}

// desc[ids[ii]] = stage[ii] for the level's fronts
__global__ void k_lu_place_desc(LFrontDesc* __restrict__ desc, const LFrontDesc* __restrict__ stage,
                                   const int64_t* __restrict__ ids, int64_t nl) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < nl; ii += (int64_t)gridDim.x * blockDim.x)
        desc[ids[ii]] = stage[ii];
}

}  // namespace

LuEngine::LuEngine(const Symbolic& S, const std::vector<int64_t>& colptr, const std::vector<int64_t>& rowidx,
                   double threshold)
    : S_(S), colptr_(colptr), rowidx_(rowidx), thr_(std::min(std::max(threshold, 1e-8), 1.0)) {
    RFG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    Plan P = build_plan(S, false);
    level_off_ = P.level_off;
    level_order_ = P.level_order;
    nlevels_ = P.nlevels;
    const int64_t nt = (int64_t)S.fronts.size();
    RFG_CUDA(cudaMalloc(&d_desc_, std::max<int64_t>(nt, 1) * sizeof(LFrontDesc)));
    RFG_CUDA(cudaMalloc(&d_lval_, std::max<size_t>(rowidx.size(), 1) * sizeof(double)));
    RFG_CUDA(cudaMalloc(&d_uval_, std::max<size_t>(rowidx.size(), 1) * sizeof(double)));
    RFG_CUDA(cudaMalloc(&d_scale_, std::max<int64_t>(S.n, 1) * sizeof(double)));
    int64_t maxl = 1;
    for (int64_t l = 0; l < nlevels_; l++) maxl = std::max(maxl, level_off_[l + 1] - level_off_[l]);
    RFG_CUDA(cudaMalloc(&d_tpre_, (maxl + 1) * sizeof(int64_t)));
    RFG_CUDA(cudaMalloc(&d_rpre_, (maxl + 1) * sizeof(int64_t)));
    RFG_CUDA(cudaMalloc(&d_active_, sizeof(int64_t)));
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    RFG_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    RFG_CUDA(cudaFuncSetAttribute(k_lu_trailing, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LTRAIL_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_lu_rowblock, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LRB_SMEM));
    // fronts of at least this many rows run their block rounds on a cluster (RFG_LU_CLUSTER_ROWS)
    if (const char* e = getenv("RFG_LU_CLUSTER_ROWS")) cluster_rows_ = std::max<int64_t>(1, atoll(e));
    RFG_CUDA(cudaFuncSetAttribute(k_lu_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * LSMEM_VEC_MAX * sizeof(double))));
}

void LuEngine::release_fronts() {
    // the per-level buffers come from the library's stream-ordered pool (no device-wide sync)
    for (void* p : front_bufs_) dev_free(p, stream_);
    for (void* p : level_bufs_) dev_free(p, stream_);
    front_bufs_.clear();
    level_bufs_.clear();
}

LuEngine::~LuEngine() {
    if (stream_) cudaStreamSynchronize(stream_);
    release_fronts();
    cudaFree(d_desc_);
    cudaFree(d_lval_);
    cudaFree(d_uval_);
    cudaFree(d_scale_);
    cudaFree(d_tpre_);
    cudaFree(d_rpre_);
    cudaFree(d_active_);
    if (stream_) cudaStreamDestroy(stream_);
}

int64_t LuEngine::factor(const double* lval, const double* uval) {
    auto t0 = std::chrono::steady_clock::now();
    release_fronts();
    const Symbolic& S = S_;
    const int64_t nt = (int64_t)S.fronts.size(), n = S.n;
    stats_ = LuStats{};
    // Full::scale (src/sparse/lu.rs:72-88): the largest magnitude in each row and column,
    // the diagonal counted once
    std::vector<double> scale(n, 0.0);
    for (int t = 0; t < 2; t++) {
        const double* v = t ? uval : lval;
        for (int64_t c = 0; c < n; c++)
            for (int64_t p = colptr_[c]; p < colptr_[c + 1]; p++) {
                const int64_t r = rowidx_[p];
                if (t && r == c) continue;
                const double a = std::fabs(v[p]);
                scale[c] = std::fmax(scale[c], a);
                scale[r] = std::fmax(scale[r], a);
            }
    }
    if (!rowidx_.empty()) {
        RFG_CUDA(cudaMemcpyAsync(d_lval_, lval, rowidx_.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
        RFG_CUDA(cudaMemcpyAsync(d_uval_, uval, rowidx_.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
    }
    if (n > 0) RFG_CUDA(cudaMemcpyAsync(d_scale_, scale.data(), n * sizeof(double), cudaMemcpyHostToDevice, stream_));
    std::vector<LFrontDesc> desc(nt);
    std::vector<std::vector<int64_t>> fs(nt), gidx(nt);
    npiv_.assign(nt, 0);
    kf_.assign(nt, 0);
    m_.assign(nt, 0);
    std::vector<int64_t> nroot(nt, 0);
    std::vector<int64_t> pos(n, -1);
    int64_t launches = 0;
    int64_t err = -1;
    for (int64_t l = 0; l < nlevels_ && err < 0; l++) {
        const int64_t lo = level_off_[l], hi = level_off_[l + 1], nl = hi - lo;
        // fully summed sets (own pivots, then the children's delayed variables in child
        // order: src/sparse/lu.rs:155-169), sizes and maps
        std::vector<int64_t> orig_dst, orig_dst_t, orig_src, cmap,
            ids(level_order_.begin() + lo, level_order_.begin() + hi);
        std::vector<int64_t> cmap_off(2 * nl, 0), cpre(2 * (nl + 1), 0);
        int64_t fbytes = 0, vbytes = 0;
        for (int64_t ii = 0; ii < nl; ii++) {
            const int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            auto& Fs = fs[t];
            Fs.clear();
            for (int64_t g = sf.start; g < sf.start + sf.k; g++) Fs.push_back(g);
            for (int64_t c = 0; c < sf.nchild; c++) {
                const int64_t ch = S.children[sf.child_off + c];
                for (int64_t x = npiv_[ch]; x < kf_[ch]; x++) Fs.push_back(fs[ch][x]);
            }
            kf_[t] = (int64_t)Fs.size();
            m_[t] = kf_[t] + sf.u;
            stats_.delayed += kf_[t] - sf.k;
            fbytes += m_[t] * m_[t];
            vbytes += kf_[t];
            for (int64_t i = 0; i < kf_[t]; i++) pos[Fs[i]] = i;
            for (int64_t x = 0; x < sf.u; x++) pos[S.rows[sf.rows_off + x]] = kf_[t] + x;
            // positions within the level's front buffer (this front starts at fbytes − m²)
            const int64_t fo_t = fbytes - m_[t] * m_[t];
            for (int64_t c = 0; c < sf.k; c++)
                for (int64_t p = colptr_[sf.start + c]; p < colptr_[sf.start + c + 1]; p++) {
                    const int64_t lr = pos[rowidx_[p]];
                    orig_dst.push_back(fo_t + lr * m_[t] + c);
                    orig_dst_t.push_back(lr != c ? fo_t + c * m_[t] + lr : -1);
                    orig_src.push_back(p);
                }
            for (int64_t c = 0; c < 2; c++) {
                int64_t nr = 0;
                if (c < sf.nchild) {
                    const int64_t ch = S.children[sf.child_off + c];
                    cmap_off[2 * ii + c] = (int64_t)cmap.size();
                    for (int64_t g : gidx[ch]) cmap.push_back(pos[g]);
                    nr = (int64_t)gidx[ch].size();
                }
                cpre[c * (nl + 1) + ii + 1] = cpre[c * (nl + 1) + ii] + nr;
            }
        }
        double* Fbuf = nullptr;
        int64_t* ibuf = nullptr;
        int64_t* mbuf = nullptr;
        Fbuf = (decltype(Fbuf))dev_alloc(std::max<int64_t>(fbytes, 1) * sizeof(double), stream_);
        // fs and the root permutations: 2 × kf per front
        ibuf = (decltype(ibuf))dev_alloc(std::max<int64_t>(2 * vbytes, 1) * sizeof(int64_t), stream_);
        const size_t nmap = 3 * orig_dst.size() + cmap.size() + cpre.size() + 2 * nl;
        mbuf = (decltype(mbuf))dev_alloc(std::max<size_t>(nmap, 1) * sizeof(int64_t), stream_);
        front_bufs_.push_back(Fbuf);
        front_bufs_.push_back(ibuf);
        level_bufs_.push_back(mbuf);
        std::vector<int64_t> ibuf_h;
        int64_t fo = 0, vo = 0;
        const int64_t no = (int64_t)orig_dst.size();
        for (int64_t ii = 0; ii < nl; ii++) {
            const int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            LFrontDesc& D = desc[t];
            D = LFrontDesc{};
            D.F = Fbuf + fo;
            D.m = m_[t];
            D.kf = kf_[t];
            D.k = sf.k;
            D.start = sf.start;
            D.u = sf.u;
            D.fs = ibuf + vo;
            D.rperm = ibuf + vbytes + vo;
            D.nchild = sf.nchild;
            for (int64_t c = 0; c < sf.nchild; c++) {
                D.child[c] = S.children[sf.child_off + c];
                D.cmap[c] = mbuf + 3 * no + cmap_off[2 * ii + c];
            }
            D.npiv = 0;
            D.nroot = 0;
            D.err = -1;
            D.root = sf.parent < 0;
            D.done = 0;
            D.p = 0;
            D.width = LKB;
            ibuf_h.insert(ibuf_h.end(), fs[t].begin(), fs[t].end());
            fo += m_[t] * m_[t];
            vo += kf_[t];
        }
        std::vector<int64_t> mh(orig_dst);
        mh.insert(mh.end(), orig_dst_t.begin(), orig_dst_t.end());
        mh.insert(mh.end(), orig_src.begin(), orig_src.end());
        mh.insert(mh.end(), cmap.begin(), cmap.end());
        const int64_t cpre_off = (int64_t)mh.size();
        mh.insert(mh.end(), cpre.begin(), cpre.end());
        const int64_t ids_off = (int64_t)mh.size();
        mh.insert(mh.end(), ids.begin(), ids.end());
        // the level's fronts by size: the block rounds of the large ones run on clusters
        std::vector<int64_t> ids_small, ids_big;
        for (int64_t t : ids) (m_[t] >= cluster_rows_ ? ids_big : ids_small).push_back(t);
        const int64_t small_off = (int64_t)mh.size();
        mh.insert(mh.end(), ids_small.begin(), ids_small.end());
        const int64_t big_off = (int64_t)mh.size();
        mh.insert(mh.end(), ids_big.begin(), ids_big.end());
        const int64_t nsmall = (int64_t)ids_small.size(), nbig = (int64_t)ids_big.size();
        RFG_CUDA(cudaMemcpyAsync(mbuf, mh.data(), mh.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        if (!ibuf_h.empty())
            RFG_CUDA(cudaMemcpyAsync(ibuf, ibuf_h.data(), ibuf_h.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                     stream_));
        {
            // the level's descriptors in one copy, then into their places
            std::vector<LFrontDesc> stage(nl);
            for (int64_t ii = 0; ii < nl; ii++) stage[ii] = desc[ids[ii]];
            LFrontDesc* dstage = (LFrontDesc*)dev_alloc(nl * sizeof(LFrontDesc), stream_);
            level_bufs_.push_back(dstage);
            RFG_CUDA(cudaMemcpyAsync(dstage, stage.data(), nl * sizeof(LFrontDesc), cudaMemcpyHostToDevice, stream_));
            k_lu_place_desc<<<(unsigned)std::min<int64_t>((nl + 127) / 128, 1024), 128, 0, stream_>>>(
                (LFrontDesc*)d_desc_, dstage, mbuf + ids_off, nl);
        }
        // per CTA: the pivot row (m − p − 1 values) and the multipliers (m − p − 1)
        double* wbuf = nullptr;
        int64_t wstride = LKB;
        for (int64_t ii = 0; ii < nl; ii++) wstride = std::max(wstride, m_[ids[ii]]);
        wbuf = (decltype(wbuf))dev_alloc(nl * 2 * wstride * sizeof(double), stream_);
        level_bufs_.push_back(wbuf);
        const size_t block_smem = wstride <= LSMEM_VEC_MAX ? 2 * wstride * sizeof(double) : 0;
        RFG_CUDA(cudaMemsetAsync(Fbuf, 0, std::max<int64_t>(fbytes, 1) * sizeof(double), stream_));
        if (no > 0)
            k_lu_asm_orig<<<(unsigned)std::min<int64_t>((no + 255) / 256, num_sms_ * 8), 256, 0, stream_>>>(
                Fbuf, mbuf, mbuf + no, mbuf + 2 * no, no, d_lval_, d_uval_);
        for (int ci = 0; ci < 2; ci++) {
            const int64_t rows = cpre[ci * (nl + 1) + nl];
            if (rows > 0)
                k_lu_asm_child<<<(unsigned)std::min<int64_t>((rows + 7) / 8, num_sms_ * 8), 256, 0, stream_>>>(
                    (LFrontDesc*)d_desc_, mbuf + ids_off, nl, mbuf + cpre_off + ci * (nl + 1), ci);
        }
        launches += 4;
        {
            const unsigned tgrid = (unsigned)(num_sms_ * 4);
            int64_t round = 0, active = 1;
            while (active > 0) {
                if (nsmall > 0)
                    k_lu_block<<<(unsigned)nsmall, ET, block_smem, stream_>>>((LFrontDesc*)d_desc_, mbuf + small_off,
                                                                             d_scale_, thr_, wbuf, wstride);
                if (nbig > 0)
                    k_lu_block_cl<<<(unsigned)(nbig * LCS), ET, 0, stream_>>>(
                        (LFrontDesc*)d_desc_, mbuf + big_off, d_scale_, thr_, wbuf + nsmall * 2 * wstride, wstride);
                k_lu_tiles<<<1, 1024, 0, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, nl, d_tpre_, d_rpre_,
                                                    d_active_);
                k_lu_rowblock<<<tgrid, LRB, LRB_SMEM, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, nl, d_rpre_);
                k_lu_trailing<<<tgrid, 256, LTRAIL_SMEM, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, nl,
                                                                   d_tpre_);
                launches += 4;
                round++;
                if (round <= 2 || round == 4 || round % 8 == 0) {
                    RFG_CUDA(cudaMemcpyAsync(&active, d_active_, sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
                    RFG_CUDA(cudaStreamSynchronize(stream_));
                }
            }
        }
        RFG_CUDA(cudaGetLastError());
        int64_t* rbuf = (int64_t*)dev_alloc(std::max<int64_t>(3 * nl, 1) * sizeof(int64_t), stream_);
        level_bufs_.push_back(rbuf);
        k_lu_results<<<(unsigned)std::min<int64_t>((nl + 255) / 256, 1024), 256, 0, stream_>>>(
            (LFrontDesc*)d_desc_, mbuf + ids_off, nl, rbuf);
        std::vector<int64_t> out(3 * nl);
        RFG_CUDA(cudaMemcpyAsync(out.data(), rbuf, 3 * nl * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
        if (!ibuf_h.empty())
            RFG_CUDA(cudaMemcpyAsync(ibuf_h.data(), ibuf, vbytes * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
        RFG_CUDA(cudaStreamSynchronize(stream_));
        vo = 0;
        for (int64_t ii = 0; ii < nl; ii++) {
            const int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            npiv_[t] = out[3 * ii];
            nroot[t] = out[3 * ii + 1];
            if (out[3 * ii + 2] >= 0 && err < 0) err = out[3 * ii + 2];
            fs[t].assign(ibuf_h.begin() + vo, ibuf_h.begin() + vo + kf_[t]);
            vo += kf_[t];
            gidx[t].assign(fs[t].begin() + npiv_[t], fs[t].end());
            for (int64_t x = 0; x < sf.u; x++) gidx[t].push_back(S.rows[sf.rows_off + x]);
            desc[t].npiv = npiv_[t];
            desc[t].nroot = nroot[t];
        }
        std::vector<int64_t> gh, goff(nl);
        for (int64_t ii = 0; ii < nl; ii++) {
            goff[ii] = (int64_t)gh.size();
            gh.insert(gh.end(), gidx[ids[ii]].begin(), gidx[ids[ii]].end());
        }
        int64_t* gbuf = nullptr;
        gbuf = (decltype(gbuf))dev_alloc((gh.size() + nl + 1) * sizeof(int64_t), stream_);
        front_bufs_.push_back(gbuf);
        std::vector<int64_t> gup(gh);
        gup.insert(gup.end(), goff.begin(), goff.end());
        RFG_CUDA(cudaMemcpyAsync(gbuf, gup.data(), gup.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        k_lu_set_gidx<<<(unsigned)std::min<int64_t>((nl + 255) / 256, 1024), 256, 0, stream_>>>(
            (LFrontDesc*)d_desc_, mbuf + ids_off, nl, gbuf, gbuf + gh.size());
        for (int64_t ii = 0; ii < nl; ii++) desc[ids[ii]].gidx = gbuf + goff[ii];
        RFG_CUDA(cudaStreamSynchronize(stream_));
    }
    stats_.launches = launches;
    if (err >= 0) return err;
    for (int64_t t = 0; t < nt; t++) {
        const int64_t k = npiv_[t], nr = m_[t] - k;
        stats_.factor_size += k * k + 2 * k * nr + nroot[t] * nroot[t];
    }
    stats_.t_factor_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return -1;
}

void LuEngine::solve_device(double* X, int64_t nrhs) {
    const int64_t nt = (int64_t)S_.fronts.size();
    if (nt == 0 || nrhs <= 0) return;
    int64_t maxl = 0, xstride = 1;
    for (int64_t l = 0; l < nlevels_; l++) maxl = std::max(maxl, level_off_[l + 1] - level_off_[l]);
    for (int64_t t = 0; t < nt; t++) xstride = std::max(xstride, kf_[t]);
    double* xbuf = nullptr;
    int64_t* dids = nullptr;
    RFG_CUDA(cudaMallocAsync((void**)&xbuf, maxl * xstride * sizeof(double), stream_));
    RFG_CUDA(cudaMallocAsync((void**)&dids, nt * sizeof(int64_t), stream_));
    RFG_CUDA(cudaMemcpyAsync(dids, level_order_.data(), nt * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    for (int64_t l = 0; l < nlevels_; l++) {
        const int64_t lo = level_off_[l], nl = level_off_[l + 1] - lo;
        k_lu_fwd<<<(unsigned)nl, ET, 0, stream_>>>((LFrontDesc*)d_desc_, dids + lo, X, (int)nrhs, xbuf, xstride);
    }
    for (int64_t l = nlevels_ - 1; l >= 0; l--) {
        const int64_t lo = level_off_[l], nl = level_off_[l + 1] - lo;
        k_lu_bwd<<<(unsigned)nl, ET, 0, stream_>>>((LFrontDesc*)d_desc_, dids + lo, X, (int)nrhs, xbuf, xstride);
    }
    RFG_CUDA(cudaGetLastError());
    RFG_CUDA(cudaFreeAsync(xbuf, stream_));
    RFG_CUDA(cudaFreeAsync(dids, stream_));
}

}  // namespace rfg
