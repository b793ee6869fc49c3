// Unsymmetric multifrontal LU on the GPU (see lu.h). Compiled with -fmad=false:
// products and sums are rounded one by one, as in the reference.

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
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
    const int64_t* orig_dst;    // (i·m + j) of each lower entry of the front's own columns
    const int64_t* orig_dst_t;  // its transposed position (c·m + i), −1 on the diagonal
    int64_t orig_src0;  // first entry of the front's columns in the lower CSC
    int64_t norig;
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

__global__ void __launch_bounds__(ET) k_lu_assemble(LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                                    const double* __restrict__ lval, const double* __restrict__ uval) {
    const LFrontDesc f = desc[ids[blockIdx.x]];
    const int64_t mm = f.m * f.m;
    for (int64_t z = threadIdx.x; z < mm; z += ET) f.F[z] = 0.0;
    __syncthreads();
    // src/sparse/lu.rs:180-190: every position receives at most one original value
    for (int64_t z = threadIdx.x; z < f.norig; z += ET) {
        f.F[f.orig_dst[z]] += lval[f.orig_src0 + z];
        if (f.orig_dst_t[z] >= 0) f.F[f.orig_dst_t[z]] += uval[f.orig_src0 + z];
    }
    __syncthreads();
    // :191-200: the children's update matrices, one child after the other
    for (int ci = 0; ci < f.nchild; ci++) {
        const LFrontDesc c = desc[f.child[ci]];
        const int64_t nr = c.m - c.npiv;
        const int64_t* map = f.cmap[ci];
        for (int64_t z = threadIdx.x; z < nr * nr; z += ET) {
            const int64_t x = z / nr, y = z - x * nr;
            f.F[map[x] * f.m + map[y]] += c.F[(c.npiv + x) * c.m + c.npiv + y];
        }
        __syncthreads();
    }
}

// One block of the threshold pivoting of one front per CTA (src/sparse/lu.rs:292-330):
// for each position p of the block [p0, b1), the first candidate j in [p, b1) with
// |a_jj| > ZERO_TOL·scale and |a_jj| >= u·max_{i >= p, i ≠ j} |a_ij|, swapped to p and
// eliminated with the eager update of the block's columns of every row and the whole row
// of the rows inside the block. A block that takes no pivot doubles the width (:351-357);
// when the last block takes none the front is done, and the root factors the rest with
// partial pivoting (:210-222, :246-270). The state stays in the descriptor between rounds.
__global__ void __launch_bounds__(ET) k_lu_block(LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                                 const double* __restrict__ scale, double thr,
                                                 double* __restrict__ wbuf, int64_t wstride) {
    __shared__ double red[ET / 32];
    __shared__ int64_t redi[ET / 32];
    __shared__ int64_t s_pick;
    const int64_t id = ids[blockIdx.x];
    const LFrontDesc f = desc[id];
    if (f.done) {
        if (threadIdx.x == 0) desc[id].blk_npb = 0;
        return;
    }
    double* F = f.F;
    const int64_t m = f.m, kf = f.kf;
    int64_t* fs = f.fs;
    double* urow = wbuf + blockIdx.x * 2 * wstride;  // wstride >= m
    double* lcol = urow + wstride;
    int64_t p = f.p, width = f.width;
    int64_t err = -1, nroot = 0;
    const int64_t p0 = p;
    const int64_t b1 = min(p + width, kf);
    while (p < b1) {
        if (threadIdx.x == 0) s_pick = -1;
        for (int64_t j = p; j < b1; j++) {
            const double ajj = fabs(F[j * m + j]);
            if (!(ajj > ZERO_TOL * scale[fs[j]])) continue;
            double g = 0.0;
            for (int64_t i = p + threadIdx.x; i < m; i += ET)
                if (i != j) g = fmax(g, fabs(F[i * m + j]));
            g = block_max(g, red);
            if (ajj >= thr * g) {
                if (threadIdx.x == 0) s_pick = j;
                break;
            }
        }
        __syncthreads();
        const int64_t j = s_pick;
        __syncthreads();
        if (j < 0) break;
        swap_pq(F, m, fs, p, j);
        const double dp = F[p * m + p];
        const int64_t wfull = m - p - 1, wshort = b1 - p - 1;
        for (int64_t x = threadIdx.x; x < wfull; x += ET) urow[x] = F[p * m + p + 1 + x];
        for (int64_t i = p + 1 + threadIdx.x; i < m; i += ET) {
            const double li = F[i * m + p] / dp;
            F[i * m + p] = li;
            lcol[i - p - 1] = li;
        }
        __syncthreads();
        // rows inside the block: the whole row; rows below it: the block's columns
        const int64_t nin = wshort;  // rows p+1 .. b1-1
        const int64_t tot = nin * wfull + (m - b1) * wshort;
        for (int64_t z = threadIdx.x; z < tot; z += ET) {
            int64_t i, x;
            if (z < nin * wfull) {
                i = p + 1 + z / wfull;
                x = z % wfull;
            } else {
                const int64_t z2 = z - nin * wfull;
                i = b1 + z2 / wshort;
                x = z2 % wshort;
            }
            const double li = lcol[i - p - 1];
            if (li != 0.0) F[i * m + p + 1 + x] -= li * urow[x];
        }
        __syncthreads();
        p += 1;
    }
    __syncthreads();
    const int64_t npb = p - p0;
    bool done = p >= kf;
    if (npb == 0) {
        if (b1 == kf) {
            done = true;
            if (p < kf && f.root) {
                // partial pivoting on the rest S = F[p.., p..] of the root (no later rows); the
                // row swaps stay inside S, the computed L21/U12 keep their rows
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

// tiles of the trailing update of each front's last block (64×64 tiles of [b1, m)²; none
// when the block took no pivot or nothing trails it): their prefix over the level's
// fronts, and the number of fronts not yet done
constexpr int LTT = 64;
__global__ void __launch_bounds__(1024) k_lu_tiles(const LFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                                   int64_t nl, int64_t* __restrict__ tpre, int64_t* __restrict__ nactive) {
    __shared__ int64_t wsum[32];
    __shared__ int64_t carry, active;
    if (threadIdx.x == 0) {
        carry = 0;
        active = 0;
        tpre[0] = 0;
    }
    __syncthreads();
    for (int64_t c0 = 0; c0 < nl; c0 += blockDim.x) {
        const int64_t ii = c0 + threadIdx.x;
        int64_t v = 0;
        if (ii < nl) {
            const LFrontDesc& f = desc[ids[ii]];
            if (f.blk_npb > 0 && f.blk_b1 < f.m) {
                const int64_t T = (f.m - f.blk_b1 + LTT - 1) / LTT;
                v = T * T;
            }
            if (!f.done) atomicAdd((unsigned long long*)&active, 1ull);
        }
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        int64_t inc = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) wsum[w] = inc;
        __syncthreads();
        int64_t woff = 0;
        for (int q = 0; q < w; q++) woff += wsum[q];
        if (ii < nl) tpre[ii + 1] = carry + woff + inc;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry += woff + inc;
        __syncthreads();
    }
    if (threadIdx.x == 0) *nactive = active;
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
    RFG_CUDA(cudaMalloc(&d_active_, sizeof(int64_t)));
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    RFG_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    RFG_CUDA(cudaFuncSetAttribute(k_lu_trailing, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LTRAIL_SMEM));
}

void LuEngine::release_fronts() {
    for (void* p : front_bufs_) cudaFree(p);
    for (void* p : level_bufs_) cudaFree(p);
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
        std::vector<int64_t> orig_dst, orig_dst_t, cmap, ids(level_order_.begin() + lo, level_order_.begin() + hi);
        std::vector<int64_t> cmap_off(2 * nl, 0), orig_off(nl, 0);
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
            orig_off[ii] = (int64_t)orig_dst.size();
            for (int64_t c = 0; c < sf.k; c++)
                for (int64_t p = colptr_[sf.start + c]; p < colptr_[sf.start + c + 1]; p++) {
                    const int64_t lr = pos[rowidx_[p]];
                    orig_dst.push_back(lr * m_[t] + c);
                    orig_dst_t.push_back(lr != c ? c * m_[t] + lr : -1);
                }
            for (int64_t c = 0; c < sf.nchild; c++) {
                const int64_t ch = S.children[sf.child_off + c];
                cmap_off[2 * ii + c] = (int64_t)cmap.size();
                for (int64_t g : gidx[ch]) cmap.push_back(pos[g]);
            }
        }
        double* Fbuf = nullptr;
        int64_t* ibuf = nullptr;
        int64_t* mbuf = nullptr;
        RFG_CUDA(cudaMalloc(&Fbuf, std::max<int64_t>(fbytes, 1) * sizeof(double)));
        // fs and the root permutations: 2 × kf per front
        RFG_CUDA(cudaMalloc(&ibuf, std::max<int64_t>(2 * vbytes, 1) * sizeof(int64_t)));
        const size_t nmap = 2 * orig_dst.size() + cmap.size() + nl;
        RFG_CUDA(cudaMalloc(&mbuf, std::max<size_t>(nmap, 1) * sizeof(int64_t)));
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
            D.orig_dst = mbuf + orig_off[ii];
            D.orig_dst_t = mbuf + no + orig_off[ii];
            D.orig_src0 = colptr_[sf.start];
            D.norig = colptr_[sf.start + sf.k] - colptr_[sf.start];
            D.nchild = sf.nchild;
            for (int64_t c = 0; c < sf.nchild; c++) {
                D.child[c] = S.children[sf.child_off + c];
                D.cmap[c] = mbuf + 2 * no + cmap_off[2 * ii + c];
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
        mh.insert(mh.end(), cmap.begin(), cmap.end());
        const int64_t ids_off = (int64_t)mh.size();
        mh.insert(mh.end(), ids.begin(), ids.end());
        RFG_CUDA(cudaMemcpyAsync(mbuf, mh.data(), mh.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        if (!ibuf_h.empty())
            RFG_CUDA(cudaMemcpyAsync(ibuf, ibuf_h.data(), ibuf_h.size() * sizeof(int64_t), cudaMemcpyHostToDevice,
                                     stream_));
        for (int64_t ii = 0; ii < nl; ii++) {
            const int64_t t = ids[ii];
            RFG_CUDA(cudaMemcpyAsync((LFrontDesc*)d_desc_ + t, &desc[t], sizeof(LFrontDesc), cudaMemcpyHostToDevice,
                                     stream_));
        }
        // per CTA: the pivot row (m − p − 1 values) and the multipliers (m − p − 1)
        double* wbuf = nullptr;
        int64_t wstride = LKB;
        for (int64_t ii = 0; ii < nl; ii++) wstride = std::max(wstride, m_[ids[ii]]);
        RFG_CUDA(cudaMalloc(&wbuf, nl * 2 * wstride * sizeof(double)));
        level_bufs_.push_back(wbuf);
        k_lu_assemble<<<(unsigned)nl, ET, 0, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, d_lval_, d_uval_);
        launches++;
        {
            const unsigned tgrid = (unsigned)(num_sms_ * 4);
            int64_t round = 0, active = 1;
            while (active > 0) {
                k_lu_block<<<(unsigned)nl, ET, 0, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, d_scale_, thr_,
                                                            wbuf, wstride);
                k_lu_tiles<<<1, 1024, 0, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, nl, d_tpre_, d_active_);
                k_lu_trailing<<<tgrid, 256, LTRAIL_SMEM, stream_>>>((LFrontDesc*)d_desc_, mbuf + ids_off, nl,
                                                                   d_tpre_);
                launches += 3;
                round++;
                if (round <= 2 || round == 4 || round % 8 == 0) {
                    RFG_CUDA(cudaMemcpyAsync(&active, d_active_, sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
                    RFG_CUDA(cudaStreamSynchronize(stream_));
                }
            }
        }
        RFG_CUDA(cudaGetLastError());
        std::vector<LFrontDesc> out(nl);
        for (int64_t ii = 0; ii < nl; ii++)
            RFG_CUDA(cudaMemcpyAsync(&out[ii], (LFrontDesc*)d_desc_ + ids[ii], sizeof(LFrontDesc),
                                     cudaMemcpyDeviceToHost, stream_));
        if (!ibuf_h.empty())
            RFG_CUDA(cudaMemcpyAsync(ibuf_h.data(), ibuf, vbytes * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
        RFG_CUDA(cudaStreamSynchronize(stream_));
        vo = 0;
        for (int64_t ii = 0; ii < nl; ii++) {
            const int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            npiv_[t] = out[ii].npiv;
            nroot[t] = out[ii].nroot;
            if (out[ii].err >= 0 && err < 0) err = out[ii].err;
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
        RFG_CUDA(cudaMalloc(&gbuf, std::max<size_t>(gh.size(), 1) * sizeof(int64_t)));
        front_bufs_.push_back(gbuf);
        if (!gh.empty())
            RFG_CUDA(cudaMemcpyAsync(gbuf, gh.data(), gh.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        for (int64_t ii = 0; ii < nl; ii++) {
            const int64_t t = ids[ii];
            desc[t].gidx = gbuf + goff[ii];
            RFG_CUDA(cudaMemcpyAsync(&((LFrontDesc*)d_desc_ + t)->gidx, &desc[t].gidx, sizeof(int64_t*),
                                     cudaMemcpyHostToDevice, stream_));
        }
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
