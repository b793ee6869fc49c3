// Symmetric indefinite multifrontal LDLᵀ on the GPU (see indef.h). Compiled with
// -fmad=false: products and sums are rounded one by one, as in the reference.

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <stdexcept>

#include "engine.h"
#include "indef.h"
#include "plan.h"

namespace rfg {

namespace {

constexpr double THRESHOLD = 0.01;            // src/sparse/indef.rs:27
constexpr double ZERO_TOL = 1e-12;            // :29
constexpr double ALPHA = 0.6403882032022079;  // :31
constexpr int IKB = 64;                       // :33
constexpr int ET = 512;                       // threads of the elimination CTA

struct IFrontDesc {
    double* F;          // m × m row-major (lower triangle + fully summed block in both triangles)
    int64_t m, kf, k, start, u;
    int64_t* fs;        // kf equations of the fully summed variables, permuted by the elimination
    double* d;
    double* e;
    int8_t* kind;       // 1 = 1×1, 2 = first of a 2×2 block, 0 = second of a 2×2 block
    int64_t* gidx;      // equations of the rows of L21 (fs[npiv..kf] then the front's rows)
    int64_t nchild;
    int64_t child[2];
    const int64_t* cmap[2];   // local index in this front of each row of the child's L21
    int64_t npiv;       // out
    int64_t err;        // out: equation at which the root is singular, or -1
    int32_t root;
    // elimination state between the block rounds of the level loop
    int32_t done;       // no further block of this front
    int64_t p, width;   // next pivot, width of the next block
    int64_t blk_p0, blk_npb, blk_b1;  // the last block: first pivot, pivots taken, end
};

__device__ __forceinline__ double block_max(double v, double* red) {
    // max over the CTA (ET threads); red has ET/32 slots
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    int w = threadIdx.x >> 5;
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[w] = v;
    __syncthreads();
    double r = red[0];
    for (int i = 1; i < ET / 32; i++) r = fmax(r, red[i]);
    return r;
}

// argmax of |value| with the smallest index among equal maxima (strictly-greater scan)
__device__ __forceinline__ void block_argmax(double v, int64_t idx, double* redv, int64_t* redi, double* outv,
                                             int64_t* outi) {
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, v, o);
        int64_t oi = __shfl_xor_sync(0xffffffffu, idx, o);
        if (ov > v || (ov == v && oi < idx)) {
            v = ov;
            idx = oi;
        }
    }
    int w = threadIdx.x >> 5;
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

// max |F(i, j)| for i in [p, m), i ∉ {j, x} (src/sparse/indef.rs:277-285)
__device__ double colmax(const double* F, int64_t m, int64_t p, int64_t j, int64_t x, double* red) {
    double g = 0.0;
    for (int64_t i = p + threadIdx.x; i < m; i += ET)
        if (i != j && i != x) g = fmax(g, fabs(F[i * m + j]));
    return block_max(g, red);
}

// symmetric swap of p and q (src/sparse/indef.rs:262-273): rows p and q over the
// columns c < climit, then columns p and q over all rows. The reference swaps the rows
// over all kf fully summed columns; here the lower triangle is kept everywhere and the
// upper triangle only inside the current block's diagonal square [p0, climit), the part
// that the pivot search reads, so the rows are swapped up to the block's end: the lower
// triangle and the square come out as in the reference (data movement only).
__device__ void swap_pq(double* F, int64_t m, int64_t climit, int64_t* fs, int64_t p, int64_t q) {
    if (p == q) return;
    for (int64_t c = threadIdx.x; c < climit; c += ET) {
        double t = F[p * m + c];
        F[p * m + c] = F[q * m + c];
        F[q * m + c] = t;
    }
    __syncthreads();
    for (int64_t i = threadIdx.x; i < m; i += ET) {
        double t = F[i * m + p];
        F[i * m + p] = F[i * m + q];
        F[i * m + q] = t;
    }
    if (threadIdx.x == 0) {
        int64_t t = fs[p];
        fs[p] = fs[q];
        fs[q] = t;
    }
    __syncthreads();
}

constexpr int ICMAX = 1024;            // block columns whose maxima are kept in shared memory
constexpr int ISMEM_VEC_MAX = 10240;   // multipliers kept in shared memory up to this many rows

// Maxima of the candidate columns: per column j = c0 + x the largest |F[i][j]| over the rows
// i >= r0, i ≠ j (v1, at row i1) and the largest over the rows other than i1 (v2), so that
// the maximum without one more row r is v2 if r = i1 and v1 otherwise (the colmax of
// indef.rs:277-285 with the 2×2 test's exclusion, :309-312).
struct ColMax {
    double* v1;
    int64_t* i1;
    double* v2;
    double* sv1;  // [ET]: per thread, for the reduction over the 8 row lanes
    int64_t* si1;
    double* sv2;
};

__device__ __forceinline__ void top2_add(double a, int64_t i, double& v1, int64_t& i1, double& v2) {
    if (a > v1) {
        v2 = v1;
        v1 = a;
        i1 = i;
    } else if (a > v2) {
        v2 = a;
    }
}

// One pass over the columns c0 + x (x < ncols) of the rows [r0, m), 64 columns × 8 rows at a
// time (coalesced rows): with K = 1 the 1×1 elimination F[i][c] −= l_i·w[x] (rows with l_i = 0
// untouched; l_i = lc0[i − loff]), with K = 2 the 2×2 one F[i][c] −= l0_i·w0[x] + l1_i·w1[x]
// (indef.rs:375-411), K = 0 reads only; then the maxima of the new values (cm non-null).
template <int K>
__device__ void indef_cols_pass(double* F, int64_t m, int64_t r0, int64_t rend, int64_t c0, int64_t ncols,
                                const double* lc0, const double* lc1, int64_t loff, const double* w0, const double* w1,
                                const ColMax* cm) {
    const int cl = threadIdx.x & 63, rl = threadIdx.x >> 6;
    for (int64_t x0 = 0; x0 < ncols; x0 += 64) {
        const int64_t x = x0 + cl;
        double v1 = 0.0, v2 = 0.0;
        int64_t i1 = -1;
        if (x < ncols) {
            const int64_t j = c0 + x;
            const double u0 = K >= 1 ? w0[x] : 0.0, u1 = K == 2 ? w1[x] : 0.0;
            int64_t i = r0 + rl;
            // UR rows in flight per thread: the loads first, then the updates
            constexpr int UR = 8;
            for (; i + (UR - 1) * (ET / 64) < rend; i += UR * (ET / 64)) {
                double v[UR];
#pragma unroll
                for (int u = 0; u < UR; u++) v[u] = F[(i + u * (ET / 64)) * m + j];
#pragma unroll
                for (int u = 0; u < UR; u++) {
                    const int64_t ii = i + u * (ET / 64);
                    if (K == 1) {
                        const double li = lc0[ii - loff];
                        if (li != 0.0) {
                            v[u] -= li * u0;
                            F[ii * m + j] = v[u];
                        }
                    } else if (K == 2) {
                        const double l0 = lc0[ii - loff], l1 = lc1[ii - loff];
                        if (l0 != 0.0 || l1 != 0.0) {
                            v[u] -= l0 * u0 + l1 * u1;
                            F[ii * m + j] = v[u];
                        }
                    }
                    if (cm && ii != j) top2_add(fabs(v[u]), ii, v1, i1, v2);
                }
            }
            for (; i < rend; i += ET / 64) {
                double v = F[i * m + j];
                if (K == 1) {
                    const double li = lc0[i - loff];
                    if (li != 0.0) {
                        v -= li * u0;
                        F[i * m + j] = v;
                    }
                } else if (K == 2) {
                    const double l0 = lc0[i - loff], l1 = lc1[i - loff];
                    if (l0 != 0.0 || l1 != 0.0) {
                        v -= l0 * u0 + l1 * u1;
                        F[i * m + j] = v;
                    }
                }
                if (cm && i != j) top2_add(fabs(v), i, v1, i1, v2);
            }
        }
        if (cm) {
            cm->sv1[threadIdx.x] = v1;
            cm->si1[threadIdx.x] = i1;
            cm->sv2[threadIdx.x] = v2;
            __syncthreads();
            if (rl == 0 && x < ncols && x < ICMAX) {
                double a1 = cm->sv1[cl], a2 = cm->sv2[cl];
                int64_t b1 = cm->si1[cl];
                for (int q = 1; q < ET / 64; q++) {
                    const double o1 = cm->sv1[q * 64 + cl], o2 = cm->sv2[q * 64 + cl];
                    const int64_t oi = cm->si1[q * 64 + cl];
                    if (o1 > a1) {
                        a2 = fmax(a1, fmax(a2, o2));
                        a1 = o1;
                        b1 = oi;
                    } else {
                        a2 = fmax(a2, fmax(o1, o2));
                    }
                }
                cm->v1[x] = a1;
                cm->i1[x] = b1;
                cm->v2[x] = a2;
            }
            __syncthreads();
        }
    }
}

// 1×1 elimination of p with the eager update of the columns (p, bend) of all rows
// (indef.rs:375-389): the multipliers first (lc), then one pass over those columns, which
// also yields the next candidates' maxima (cm non-null).
__device__ double elim1(double* F, int64_t m, int64_t p, int64_t bend, double* w, double* lc, const ColMax* cm) {
    const double dp = F[p * m + p];
    const int nw = (int)(bend - p - 1);
    for (int x = threadIdx.x; x < nw; x += ET) w[x] = F[(p + 1 + x) * m + p];
    __syncthreads();
    for (int64_t i = p + 1 + threadIdx.x; i < m; i += ET) {
        const double li = F[i * m + p] / dp;
        lc[i - p - 1] = li;
        F[i * m + p] = li;
    }
    __syncthreads();
    indef_cols_pass<1>(F, m, p + 1, m, p + 1, nw, lc, nullptr, p + 1, w, nullptr, cm);
    __syncthreads();
    return dp;
}

// 2×2 elimination of (p, p+1) (indef.rs:392-411), in the same two phases
__device__ void elim2(double* F, int64_t m, int64_t p, int64_t bend, double* w0, double* w1, double* lc0, double* lc1,
                      double* a_out, double* b_out, double* c_out, const ColMax* cm) {
    const double a = F[p * m + p], b = F[(p + 1) * m + p], c = F[(p + 1) * m + p + 1];
    const double det = a * c - b * b;
    const int nw = (int)(bend - p - 2);
    for (int x = threadIdx.x; x < nw; x += ET) {
        w0[x] = F[(p + 2 + x) * m + p];
        w1[x] = F[(p + 2 + x) * m + p + 1];
    }
    __syncthreads();
    for (int64_t i = p + 2 + threadIdx.x; i < m; i += ET) {
        const double x0 = F[i * m + p], x1 = F[i * m + p + 1];
        const double l0 = (x0 * c - x1 * b) / det;
        const double l1 = (x1 * a - x0 * b) / det;
        lc0[i - p - 2] = l0;
        lc1[i - p - 2] = l1;
        F[i * m + p] = l0;
        F[i * m + p + 1] = l1;
    }
    __syncthreads();
    indef_cols_pass<2>(F, m, p + 2, m, p + 2, nw, lc0, lc1, p + 2, w0, w1, cm);
    __syncthreads();
    *a_out = a;
    *b_out = b;
    *c_out = c;
}

// F[x][y] −= (L·D)[x]·L[y]ᵀ for b1 <= y <= x < m with the pivots [p0, p0 + npb)
// (indef.rs:504-532); every entry is one fused multiply-add chain over the pivots
// starting from 0, as the reference's micro-kernel computes it.
__device__ void trailing_update(double* F, int64_t m, int64_t p0, int64_t npb, int64_t b1, const double* d,
                                const double* e, const int8_t* kind) {
    int64_t rows = m - b1;
    int64_t total = rows * (rows + 1) / 2;
    for (int64_t z = threadIdx.x; z < total; z += ET) {
        int64_t x = (int64_t)((sqrt(8.0 * (double)z + 1.0) - 1.0) * 0.5);
        while (x * (x + 1) / 2 > z) x--;
        while ((x + 1) * (x + 2) / 2 <= z) x++;
        int64_t y = z - x * (x + 1) / 2;
        const double* fx = F + (b1 + x) * m + p0;
        const double* fy = F + (b1 + y) * m + p0;
        double acc = 0.0;
        int64_t q = 0;
        while (q < npb) {
            if (kind[q] == 2) {
                double l0 = fx[q], l1 = fx[q + 1];
                double w0 = l0 * d[q] + l1 * e[q];
                double w1 = l0 * e[q] + l1 * d[q + 1];
                acc = fma(w0, fy[q], acc);
                acc = fma(w1, fy[q + 1], acc);
                q += 2;
            } else {
                acc = fma(fx[q] * d[q], fy[q], acc);
                q += 1;
            }
        }
        F[(b1 + x) * m + b1 + y] -= acc;
    }
    __syncthreads();
}

// Assembly of a level on all SMs (indef.rs:173-210), the fronts zeroed before: the original
// entries of the fronts' own columns (lower triangle, one value per position), then each child
// slot's update matrices in its own launch (a position shared by both children sums child 0
// before child 1), then the fully summed block mirrored into its upper triangle.
__global__ void k_indef_asm_orig(double* __restrict__ Fbuf, const int64_t* __restrict__ dst,
                                 const int64_t* __restrict__ src, int64_t nent, const double* __restrict__ val) {
    for (int64_t z = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; z < nent; z += (int64_t)gridDim.x * blockDim.x)
        Fbuf[dst[z]] += val[src[z]];
}

__device__ __forceinline__ int64_t find_front(const int64_t* __restrict__ pre, int64_t nl, int64_t w) {
    int64_t lo = 0, hi = nl;
    while (hi - lo > 1) {
        const int64_t mid = (lo + hi) >> 1;
        if (pre[mid] <= w)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// one warp per row x of child slot ci's update matrix (its lower triangle y <= x)
__global__ void __launch_bounds__(256) k_indef_asm_child(const IFrontDesc* __restrict__ desc,
                                                         const int64_t* __restrict__ ids, int64_t nl,
                                                         const int64_t* __restrict__ cpre, int ci) {
    const int lane = threadIdx.x & 31;
    const int64_t total = cpre[nl];
    for (int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); w < total; w += (int64_t)gridDim.x * 8) {
        const int64_t ii = find_front(cpre, nl, w);
        const IFrontDesc& f = desc[ids[ii]];
        const IFrontDesc& c = desc[f.child[ci]];
        const int64_t x = w - cpre[ii];
        const int64_t* map = f.cmap[ci];
        const double* urow = c.F + (c.npiv + x) * c.m + c.npiv;
        const int64_t mx = map[x];
        for (int64_t y = lane; y <= x; y += 32) {
            int64_t a = mx, b = map[y];
            if (a < b) {
                const int64_t t = a;
                a = b;
                b = t;
            }
            f.F[a * f.m + b] += urow[y];
        }
    }
}

// one warp per row i of the fully summed block: F[j][i] = F[i][j] for j < i
__global__ void __launch_bounds__(256) k_indef_mirror(const IFrontDesc* __restrict__ desc,
                                                      const int64_t* __restrict__ ids, int64_t nl,
                                                      const int64_t* __restrict__ kpre) {
    const int lane = threadIdx.x & 31;
    const int64_t total = kpre[nl];
    for (int64_t w = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5); w < total; w += (int64_t)gridDim.x * 8) {
        const int64_t ii = find_front(kpre, nl, w);
        const IFrontDesc& f = desc[ids[ii]];
        const int64_t i = w - kpre[ii];
        for (int64_t j = lane; j < i; j += 32) f.F[j * f.m + i] = f.F[i * f.m + j];
    }
}

// upper triangle of the diagonal square [p0, b1) from its lower triangle (the part of the
// reference's mirror, src/sparse/indef.rs:458-463, that the next pivot search reads)
__device__ void mirror_square(double* F, int64_t m, int64_t p0, int64_t b1) {
    const int64_t w = b1 - p0;
    for (int64_t z = threadIdx.x; z < w * w; z += ET) {
        const int64_t i = p0 + z / w, j = p0 + z % w;
        if (j < i) F[j * m + i] = F[i * m + j];
    }
    __syncthreads();
}

// The end of a block round (indef.rs:465-498): the width for the next block, and at the root,
// once no candidate passes, Bunch–Kaufman on its whole remaining fully summed block; then the
// front's state. One CTA (ET threads).
__device__ void indef_block_finish(IFrontDesc* desc, int64_t id, IFrontDesc& f, const double* scale, int64_t p0,
                                   int64_t p, int64_t b1, int64_t width, double* w0, double* w1, double* lc0,
                                   double* lc1, double* red, int64_t* redi) {
    double* F = f.F;
    const int64_t m = f.m, kf = f.kf;
    int64_t* fs = f.fs;
    int64_t err = -1;
    const int64_t npb = p - p0;
    bool done = p >= kf;
    if (npb == 0) {
        if (b1 == kf) {
            done = true;
            if (p < kf && f.root) {
                // Bunch–Kaufman on the rest of the root (indef.rs:326-372, 474-498), with the
                // whole remaining fully summed block in both triangles
                mirror_square(F, m, p, kf);
                while (p < kf) {
                    double big;
                    int64_t lin;
                    {
                        double v = -1.0;
                        int64_t vi = INT64_MAX;
                        int64_t n2 = kf - p;
                        for (int64_t z = threadIdx.x; z < n2 * n2; z += ET) {
                            int64_t jj = p + z / n2, ii = p + z % n2;  // (j outer, i inner) order
                            if (ii < jj) continue;
                            double a = fabs(F[ii * m + jj]);
                            int64_t key = z;
                            if (a > v || (a == v && key < vi)) {
                                v = a;
                                vi = key;
                            }
                        }
                        block_argmax(v, vi, red, redi, &big, &lin);
                    }
                    int64_t n2 = kf - p;
                    int64_t bj = p + lin / n2, bi = p + lin % n2;
                    int64_t kind = 0, j = 0, r = 0;
                    auto one = [&](int64_t jj) -> bool {
                        if (fabs(F[jj * m + jj]) > ZERO_TOL * scale[fs[jj]]) {
                            kind = 1;
                            j = jj;
                            return true;
                        }
                        err = fs[jj];
                        return false;
                    };
                    if (!(big > ZERO_TOL * fmax(scale[fs[bj]], scale[fs[bi]]))) {
                        err = fs[bj];
                    } else if (bi == bj) {
                        one(bj);
                    } else {
                        int64_t jj = bj, rr = bi;
                        double lam = big;
                        double ajj = fabs(F[jj * m + jj]);
                        if (ajj >= ALPHA * lam) {
                            one(jj);
                        } else {
                            double sg = 0.0;
                            for (int64_t i = p + threadIdx.x; i < kf; i += ET)
                                if (i != rr) sg = fmax(sg, fabs(i >= rr ? F[i * m + rr] : F[rr * m + i]));
                            double sig = block_max(sg, red);
                            if (ajj * sig >= ALPHA * lam * lam) {
                                one(jj);
                            } else if (fabs(F[rr * m + rr]) >= ALPHA * sig) {
                                one(rr);
                            } else {
                                double a = F[jj * m + jj], b = F[rr * m + jj], c = F[rr * m + rr];
                                double det = a * c - b * b;
                                if (!(fabs(det) > ZERO_TOL * scale[fs[jj]] * scale[fs[rr]])) {
                                    err = fs[jj];
                                } else {
                                    kind = 2;
                                    j = jj;
                                    r = rr;
                                }
                            }
                        }
                    }
                    __syncthreads();
                    if (kind == 0) break;
                    if (kind == 1) {
                        swap_pq(F, m, kf, fs, p, j);
                        double dp = elim1(F, m, p, kf, w0, lc0, nullptr);
                        if (threadIdx.x == 0) {
                            f.d[p] = dp;
                            f.e[p] = 0.0;
                            f.kind[p] = 1;
                        }
                        p += 1;
                    } else {
                        int64_t rr = (r == p) ? j : r;
                        swap_pq(F, m, kf, fs, p, j);
                        swap_pq(F, m, kf, fs, p + 1, rr);
                        double a, b, c;
                        elim2(F, m, p, kf, w0, w1, lc0, lc1, &a, &b, &c, nullptr);
                        if (threadIdx.x == 0) {
                            f.d[p] = a;
                            f.d[p + 1] = c;
                            f.e[p] = b;
                            f.e[p + 1] = 0.0;
                            f.kind[p] = 2;
                            f.kind[p + 1] = 0;
                        }
                        p += 2;
                    }
                    __syncthreads();
                }
            }
        } else {
            width *= 2;
        }
    } else {
        width = IKB;
    }
    if (threadIdx.x == 0) {
        desc[id].p = p;
        desc[id].width = width;
        desc[id].done = done ? 1 : 0;
        desc[id].blk_p0 = p0;
        desc[id].blk_npb = npb;
        desc[id].blk_b1 = b1;
        desc[id].npiv = p;
        desc[id].err = err;
    }
}

// One block of the threshold pivoting of one front (indef.rs:416-500) on one CTA: the pivot
// search over [p, b1) with b1 = p + width, symmetric swaps, 1×1 / 2×2 eliminations with
// the eager update of the block's columns. The trailing update of the block's pivots runs
// afterwards on all SMs (k_indef_trailing). A block that takes no pivot doubles the width
// (:465-472); when the last block takes none the front is done, and the root finishes its
// fully summed block by Bunch–Kaufman (:326-372, :474-498). The state (p, width, done,
// the last block) stays in the descriptor between rounds.
__device__ void indef_block_cta(IFrontDesc* desc, int64_t id, const double* scale, double thr, double* w0,
                                double* w1, double* lc0, double* lc1, const ColMax& cmx, double* red, int64_t* redi,
                                int64_t* s_kind_p, int64_t* s_j_p, int64_t* s_r_p) {
    IFrontDesc f = desc[id];
    double* F = f.F;
    const int64_t m = f.m, kf = f.kf;
    int64_t* fs = f.fs;
    double* cv1 = cmx.v1;
    double* cv2 = cmx.v2;
    int64_t* ci1 = cmx.i1;
    int64_t& s_kind = *s_kind_p;
    int64_t& s_j = *s_j_p;
    int64_t& s_r = *s_r_p;
    int64_t p = f.p, width = f.width;
    const int64_t p0 = p;
    const int64_t b1 = min(p + width, kf);
    mirror_square(F, m, p0, b1);
    // maxima of the candidate columns [p, b1) over the rows [p, m) before the first pivot; each
    // elimination's update pass then gives those of the next position
    indef_cols_pass<0>(F, m, p, m, p, b1 - p, nullptr, nullptr, 0, nullptr, nullptr, &cmx);
    // the largest |F[i][j]| over the rows i >= p, i ∉ {j, x} (colmax, indef.rs:277-285)
    auto cmax_of = [&](int64_t j, int64_t x) -> double {
        const int64_t c = j - p;
        if (c < ICMAX) return (x >= 0 && ci1[c] == x) ? cv2[c] : cv1[c];
        return colmax(F, m, p, j, x, red);
    };
    while (p < b1) {
        // choose (indef.rs:288-323)
        if (threadIdx.x == 0) s_kind = 0;
        for (int64_t j = p; j < b1; j++) {
            double ajj = F[j * m + j];
            double sj = scale[fs[j]];
            double gj = cmax_of(j, -1);
            if (fabs(ajj) > ZERO_TOL * sj && fabs(ajj) >= thr * gj) {
                if (threadIdx.x == 0) {
                    s_kind = 1;
                    s_j = j;
                }
                break;
            }
            double best;
            int64_t r;
            double v = 0.0;
            int64_t vi = INT64_MAX;
            for (int64_t i = p + threadIdx.x; i < b1; i += ET) {
                if (i == j) continue;
                double a = fabs(F[i * m + j]);
                if (a > v) {
                    v = a;
                    vi = i;
                }
            }
            block_argmax(v, vi, red, redi, &best, &r);
            if (!(best > 0.0)) continue;
            double a = ajj, b = F[r * m + j], c = F[r * m + r];
            double det = a * c - b * b;
            double sr = scale[fs[r]];
            if (!(fabs(det) > ZERO_TOL * sj * sr)) continue;
            double gj2 = cmax_of(j, r);
            double gr2 = cmax_of(r, j);
            double ad = fabs(det);
            if ((fabs(c) * gj2 + fabs(b) * gr2) / ad <= 1.0 / thr && (fabs(b) * gj2 + fabs(a) * gr2) / ad <= 1.0 / thr) {
                if (threadIdx.x == 0) {
                    s_kind = 2;
                    s_j = j;
                    s_r = r;
                }
                break;
            }
        }
        __syncthreads();
        int64_t kind = s_kind, j = s_j, r = s_r;
        __syncthreads();
        if (kind == 1) {
            swap_pq(F, m, b1, fs, p, j);
            double dp = elim1(F, m, p, b1, w0, lc0, &cmx);
            if (threadIdx.x == 0) {
                f.d[p] = dp;
                f.e[p] = 0.0;
                f.kind[p] = 1;
            }
            p += 1;
        } else if (kind == 2) {
            int64_t rr = (r == p) ? j : r;
            swap_pq(F, m, b1, fs, p, j);
            swap_pq(F, m, b1, fs, p + 1, rr);
            double a, b, c;
            elim2(F, m, p, b1, w0, w1, lc0, lc1, &a, &b, &c, &cmx);
            if (threadIdx.x == 0) {
                f.d[p] = a;
                f.d[p + 1] = c;
                f.e[p] = b;
                f.e[p + 1] = 0.0;
                f.kind[p] = 2;
                f.kind[p + 1] = 0;
            }
            p += 2;
        } else {
            break;
        }
        __syncthreads();
    }
    __syncthreads();
    indef_block_finish(desc, id, f, scale, p0, p, b1, width, w0, w1, lc0, lc1, red, redi);
}

// one CTA per front (the level's smaller fronts)
__global__ void __launch_bounds__(ET) k_indef_block(IFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids,
                                                    const double* __restrict__ scale, double thr,
                                                    double* __restrict__ wbuf, int64_t wstride) {
    extern __shared__ double ism[];
    __shared__ double red[ET / 32];
    __shared__ int64_t redi[ET / 32];
    __shared__ int64_t s_kind, s_j, s_r;
    __shared__ double cv1[ICMAX], cv2[ICMAX];
    __shared__ int64_t ci1[ICMAX];
    __shared__ double sv1[ET], sv2[ET];
    __shared__ int64_t si1[ET];
    const int64_t id = ids[blockIdx.x];
    if (desc[id].done) {
        if (threadIdx.x == 0) desc[id].blk_npb = 0;
        return;
    }
    double* w0 = wbuf + blockIdx.x * 4 * wstride;  // wstride >= m: the eager-update rows and the
    double* w1 = w0 + wstride;                      // multipliers of the 1×1 / 2×2 eliminations
    double* lc0 = wstride <= ISMEM_VEC_MAX ? ism : w1 + wstride;  // (shared memory when they fit)
    double* lc1 = lc0 + wstride;
    const ColMax cmx{cv1, ci1, cv2, sv1, si1, sv2};
    indef_block_cta(desc, id, scale, thr, w0, w1, lc0, lc1, cmx, red, redi, &s_kind, &s_j, &s_r);
}

// The same block on a cluster of ICS CTAs for the level's large fronts: each CTA owns a slice
// of the rows; per pivot the candidates' column maxima (top two per column) are combined from
// the CTAs' partial maxima (distributed shared memory), one warp of every CTA takes the same
// decision (indef.rs:288-323), the row swaps are split over the CTAs by columns and the
// column swaps by rows, and each CTA eliminates its own rows (the same products and
// differences per entry as on one CTA). Blocks wider than IPW candidates, and the root's
// Bunch–Kaufman phase, run on the cluster's first CTA.
constexpr int ICS = 8;   // CTAs per cluster
constexpr int IPW = 64;  // candidates per block handled by the whole cluster
__global__ void __cluster_dims__(ICS, 1, 1) __launch_bounds__(ET)
    k_indef_block_cl(IFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, const double* __restrict__ scale,
                     double thr, double* __restrict__ wbuf, int64_t wstride) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ double red[ET / 32];
    __shared__ int64_t redi[ET / 32];
    __shared__ int64_t s_kind, s_j, s_r;
    __shared__ double cv1[ICMAX], cv2[ICMAX];
    __shared__ int64_t ci1[ICMAX];
    __shared__ double sv1[ET], sv2[ET];
    __shared__ int64_t si1[ET];
    __shared__ double pv1[IPW], pv2[IPW];  // this CTA's partial maxima of the candidates
    __shared__ int64_t pi1[IPW];
    __shared__ double w0s[IPW], w1s[IPW];
    const int rank = (int)cluster.block_rank();
    const int64_t slot = blockIdx.x / ICS;
    const int64_t id = ids[slot];
    double* wb = wbuf + slot * 4 * wstride;
    if (desc[id].done) {
        if (rank == 0 && threadIdx.x == 0) desc[id].blk_npb = 0;
        return;  // the whole cluster returns: no distributed shared memory was touched
    }
    IFrontDesc f = desc[id];
    const int64_t m = f.m, kf = f.kf;
    const int64_t p0 = f.p;
    const int64_t b1 = min(p0 + f.width, kf);
    const ColMax cmx{cv1, ci1, cv2, sv1, si1, sv2};
    if (b1 - p0 > IPW) {
        // a block that has grown past IPW candidates: on one CTA (uses no cluster barrier)
        if (rank == 0)
            indef_block_cta(desc, id, scale, thr, wb, wb + wstride, wb + 2 * wstride, wb + 3 * wstride, cmx, red, redi,
                            &s_kind, &s_j, &s_r);
        return;
    }
    double* F = f.F;
    int64_t* fs = f.fs;
    double* lc0 = wb + 2 * wstride;  // multipliers of this CTA's rows (written after a cluster barrier)
    double* lc1 = wb + 3 * wstride;
    const int64_t S = (m - p0 + ICS - 1) / ICS;
    const int64_t lo = min(p0 + rank * S, m), hi = min(lo + S, m);
    const int64_t SA = (m + ICS - 1) / ICS;
    const int64_t alo = min(rank * SA, m), ahi = min(alo + SA, m);
    const int64_t CW = (b1 + ICS - 1) / ICS;  // columns [0, b1) of the row swaps per CTA
    const int64_t clo = min(rank * CW, b1), chi = min(clo + CW, b1);
    const ColMax pcm{pv1, pi1, pv2, sv1, si1, sv2};
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // swap_pq over the cluster: rows a and b over the columns [0, b1), then columns a and b
    auto cswap = [&](int64_t a, int64_t b) {
        if (a == b) return;
        for (int64_t c = clo + threadIdx.x; c < chi; c += ET) {
            const double t = F[a * m + c];
            F[a * m + c] = F[b * m + c];
            F[b * m + c] = t;
        }
        cluster.sync();
        for (int64_t i = alo + threadIdx.x; i < ahi; i += ET) {
            const double t = F[i * m + a];
            F[i * m + a] = F[i * m + b];
            F[i * m + b] = t;
        }
        if (rank == 0 && threadIdx.x == 0) {
            const int64_t t = fs[a];
            fs[a] = fs[b];
            fs[b] = t;
        }
        cluster.sync();
    };
    if (rank == 0) mirror_square(F, m, p0, b1);
    cluster.sync();
    int64_t p = p0;
    indef_cols_pass<0>(F, m, max(lo, p), hi, p, b1 - p, nullptr, nullptr, 0, nullptr, nullptr, &pcm);
    cluster.sync();
    while (p < b1) {
        // the candidates' maxima: the CTAs' partial top two merged
        if (threadIdx.x < b1 - p) {
            const int x = threadIdx.x;
            double a1 = 0.0, a2 = 0.0;
            int64_t ai = -1;
            for (int r = 0; r < ICS; r++) {
                const double o1 = cluster.map_shared_rank(pv1, r)[x], o2 = cluster.map_shared_rank(pv2, r)[x];
                const int64_t oi = cluster.map_shared_rank(pi1, r)[x];
                if (o1 > a1) {
                    a2 = fmax(a1, fmax(a2, o2));
                    a1 = o1;
                    ai = oi;
                } else {
                    a2 = fmax(a2, fmax(o1, o2));
                }
            }
            cv1[x] = a1;
            ci1[x] = ai;
            cv2[x] = a2;
        }
        __syncthreads();
        // choose (indef.rs:288-323), by one warp of every CTA
        if (warp == 0) {
            int64_t kind = 0, jj = 0, rr = 0;
            for (int64_t j = p; j < b1; j++) {
                const double ajj = F[j * m + j];
                const double sj = scale[fs[j]];
                const double gj = cv1[j - p];
                if (fabs(ajj) > ZERO_TOL * sj && fabs(ajj) >= thr * gj) {
                    kind = 1;
                    jj = j;
                    break;
                }
                double v = 0.0;
                int64_t vi = INT64_MAX;
                for (int64_t i = p + lane; i < b1; i += 32) {
                    if (i == j) continue;
                    const double a = fabs(F[i * m + j]);
                    if (a > v) {
                        v = a;
                        vi = i;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const double ov = __shfl_xor_sync(0xffffffffu, v, o);
                    const int64_t oi = __shfl_xor_sync(0xffffffffu, vi, o);
                    if (ov > v || (ov == v && oi < vi)) {
                        v = ov;
                        vi = oi;
                    }
                }
                const double best = v;
                const int64_t r = vi;
                if (!(best > 0.0)) continue;
                const double a = ajj, b = F[r * m + j], c = F[r * m + r];
                const double det = a * c - b * b;
                const double sr = scale[fs[r]];
                if (!(fabs(det) > ZERO_TOL * sj * sr)) continue;
                const double gj2 = ci1[j - p] == r ? cv2[j - p] : cv1[j - p];
                const double gr2 = ci1[r - p] == j ? cv2[r - p] : cv1[r - p];
                const double ad = fabs(det);
                if ((fabs(c) * gj2 + fabs(b) * gr2) / ad <= 1.0 / thr &&
                    (fabs(b) * gj2 + fabs(a) * gr2) / ad <= 1.0 / thr) {
                    kind = 2;
                    jj = j;
                    rr = r;
                    break;
                }
            }
            if (lane == 0) {
                s_kind = kind;
                s_j = jj;
                s_r = rr;
            }
        }
        __syncthreads();
        const int64_t kind = s_kind, j = s_j, r = s_r;
        // every CTA has read the partial maxima and the candidates before anything changes
        cluster.sync();
        if (kind == 0) break;
        if (kind == 1) {
            cswap(p, j);
            const double dp = F[p * m + p];
            const int64_t nw = b1 - p - 1;
            if (threadIdx.x < nw) w0s[threadIdx.x] = F[(p + 1 + threadIdx.x) * m + p];
            for (int64_t i = max(lo, p + 1) + threadIdx.x; i < hi; i += ET) lc0[i - p - 1] = F[i * m + p] / dp;
            __syncthreads();
            indef_cols_pass<1>(F, m, max(lo, p + 1), hi, p + 1, nw, lc0, nullptr, p + 1, w0s, nullptr, &pcm);
            // every CTA has read column p before the multipliers replace it
            cluster.sync();
            for (int64_t i = max(lo, p + 1) + threadIdx.x; i < hi; i += ET) F[i * m + p] = lc0[i - p - 1];
            if (rank == 0 && threadIdx.x == 0) {
                f.d[p] = dp;
                f.e[p] = 0.0;
                f.kind[p] = 1;
            }
            p += 1;
        } else {
            const int64_t r2 = (r == p) ? j : r;
            cswap(p, j);
            cswap(p + 1, r2);
            const double a = F[p * m + p], b = F[(p + 1) * m + p], c = F[(p + 1) * m + p + 1];
            const double det = a * c - b * b;
            const int64_t nw = b1 - p - 2;
            if (threadIdx.x < nw) {
                w0s[threadIdx.x] = F[(p + 2 + threadIdx.x) * m + p];
                w1s[threadIdx.x] = F[(p + 2 + threadIdx.x) * m + p + 1];
            }
            for (int64_t i = max(lo, p + 2) + threadIdx.x; i < hi; i += ET) {
                const double x0 = F[i * m + p], x1 = F[i * m + p + 1];
                lc0[i - p - 2] = (x0 * c - x1 * b) / det;
                lc1[i - p - 2] = (x1 * a - x0 * b) / det;
            }
            __syncthreads();
            indef_cols_pass<2>(F, m, max(lo, p + 2), hi, p + 2, nw, lc0, lc1, p + 2, w0s, w1s, &pcm);
            cluster.sync();
            for (int64_t i = max(lo, p + 2) + threadIdx.x; i < hi; i += ET) {
                F[i * m + p] = lc0[i - p - 2];
                F[i * m + p + 1] = lc1[i - p - 2];
            }
            if (rank == 0 && threadIdx.x == 0) {
                f.d[p] = a;
                f.d[p + 1] = c;
                f.e[p] = b;
                f.e[p + 1] = 0.0;
                f.kind[p] = 2;
                f.kind[p + 1] = 0;
            }
            p += 2;
        }
    }
    // no CTA leaves while another may still read its partial maxima; the multipliers are in place
    cluster.sync();
    if (rank == 0)
        indef_block_finish(desc, id, f, scale, p0, p, b1, f.width, wb, wb + wstride, wb + 2 * wstride,
                           wb + 3 * wstride, red, redi);
}

// tiles of the trailing update of each front's last block (64×64 tiles of the lower
// triangle of [b1, m)²; none when the block took no pivot or nothing trails it): their
// prefix over the level's fronts, and the number of fronts not yet done
constexpr int ITT = 64;
__global__ void __launch_bounds__(1024) k_indef_tiles(const IFrontDesc* __restrict__ desc,
                                                      const int64_t* __restrict__ ids, int64_t nl,
                                                      int64_t* __restrict__ tpre, int64_t* __restrict__ nactive) {
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
            const IFrontDesc& f = desc[ids[ii]];
            if (f.blk_npb > 0 && f.blk_b1 < f.m) {
                const int64_t T = (f.m - f.blk_b1 + ITT - 1) / ITT;
                v = T * (T + 1) / 2;
            }
            if (!f.done) atomicAdd((unsigned long long*)&active, 1ull);
        }
        // inclusive scan of v over the CTA
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

// Trailing update of the last block of each front of the level (indef.rs:504-532):
// F[x][y] −= Σ_q W[x][q]·L[y][q] for b1 <= y <= x < m over the block's pivots q, with
// W = L·D taking 2×2 blocks into account (:512-522). Each entry is one fused
// multiply-add chain over the pivots in order, starting from 0, as the reference's
// micro-kernel computes it. 64×64 tiles of the lower triangle, 256 threads with 4×4
// entries each, K in chunks of 64 through shared memory; CTAs walk the level's tiles.
constexpr int ITK = 64;
constexpr size_t ITRAIL_SMEM = 2 * ITT * (ITK + 1) * sizeof(double);
__global__ void __launch_bounds__(256) k_indef_trailing(const IFrontDesc* __restrict__ desc,
                                                        const int64_t* __restrict__ ids, int64_t nl,
                                                        const int64_t* __restrict__ tpre) {
    extern __shared__ double its[];
    double* Ws = its;                    // [ITT][ITK + 1]: W of the tile's rows
    double* Ls = its + ITT * (ITK + 1);  // [ITT][ITK + 1]: L of the tile's columns
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
        const IFrontDesc& fr = desc[ids[lo]];
        const double* F0 = fr.F;
        double* F = fr.F;
        const int64_t m = fr.m, b1 = fr.blk_b1, p0 = fr.blk_p0, npb = fr.blk_npb;
        const double* d = fr.d + p0;
        const double* e = fr.e + p0;
        const int8_t* kind = fr.kind + p0;
        int64_t lt = t - tpre[lo];
        const int64_t T = (m - b1 + ITT - 1) / ITT;
        int64_t tc = 0, cnt = T;
        while (lt >= cnt) {
            lt -= cnt;
            tc++;
            cnt = T - tc;
        }
        const int64_t tr = tc + lt;
        const int64_t x0 = b1 + tr * ITT, y0 = b1 + tc * ITT;
        double acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; a++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[a][c] = 0.0;
        for (int64_t k0 = 0; k0 < npb; k0 += ITK) {
            const int kc = (int)min((int64_t)ITK, npb - k0);
            __syncthreads();
            for (int z = threadIdx.x; z < ITT * ITK; z += 256) {
                const int r = z / ITK, q = z % ITK;
                double wv = 0.0, lv = 0.0;
                if (q < kc) {
                    const int64_t qq = k0 + q;
                    const int64_t x = x0 + r, y = y0 + r;
                    if (x < m) {
                        const double* fx = F0 + x * m + p0;
                        if (kind[qq] == 2) {
                            wv = fx[qq] * d[qq] + fx[qq + 1] * e[qq];
                        } else if (kind[qq] == 0) {
                            wv = fx[qq - 1] * e[qq - 1] + fx[qq] * d[qq];
                        } else {
                            wv = fx[qq] * d[qq];
                        }
                    }
                    if (y < m) lv = F0[y * m + p0 + qq];
                }
                Ws[r * (ITK + 1) + q] = wv;
                Ls[r * (ITK + 1) + q] = lv;
            }
            __syncthreads();
            for (int q = 0; q < kc; q++) {
                double wr[4], lc[4];
#pragma unroll
                for (int a = 0; a < 4; a++) wr[a] = Ws[(ty + 16 * a) * (ITK + 1) + q];
#pragma unroll
                for (int c = 0; c < 4; c++) lc[c] = Ls[(tx + 16 * c) * (ITK + 1) + q];
#pragma unroll
                for (int a = 0; a < 4; a++)
#pragma unroll
                    for (int c = 0; c < 4; c++) acc[a][c] = fma(wr[a], lc[c], acc[a][c]);
            }
        }
#pragma unroll
        for (int a = 0; a < 4; a++) {
            const int64_t x = x0 + ty + 16 * a;
            if (x >= m) continue;
#pragma unroll
            for (int c = 0; c < 4; c++) {
                const int64_t y = y0 + tx + 16 * c;
                if (y <= x) F[x * m + y] -= acc[a][c];
            }
        }
    }
}

// ---- solve: forward (levels up), diagonal, backward (levels down) ----
__global__ void k_indef_fwd(const IFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, double* X, int nrhs,
                            double* __restrict__ xbuf, int64_t xstride) {
    __shared__ double red[ET / 32];
    const IFrontDesc f = desc[ids[blockIdx.x]];
    int64_t k = f.npiv;
    double* xp = xbuf + blockIdx.x * xstride;
    for (int j = 0; j < nrhs; j++) {
        for (int64_t i = threadIdx.x; i < k; i += ET) xp[i] = X[f.fs[i] * nrhs + j];
        __syncthreads();
        for (int64_t i = 1; i < k; i++) {
            double sacc = 0.0;
            for (int64_t q = threadIdx.x; q < i; q += ET)
                if (!(f.kind[i] == 0 && q == i - 1)) sacc += f.F[i * f.m + q] * xp[q];
            for (int o = 16; o > 0; o >>= 1) sacc += __shfl_xor_sync(0xffffffffu, sacc, o);
            __syncthreads();
            if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sacc;
            __syncthreads();
            if (threadIdx.x == 0) {
                double t = 0.0;
                for (int w = 0; w < ET / 32; w++) t += red[w];
                xp[i] -= t;
            }
            __syncthreads();
        }
        int64_t nr = f.m - k;
        for (int64_t r = threadIdx.x; r < nr; r += ET) {
            const double* l = f.F + (k + r) * f.m;
            double t = 0.0;
            for (int64_t q = 0; q < k; q++) t += l[q] * xp[q];
            atomicAdd(&X[f.gidx[r] * nrhs + j], -t);
        }
        for (int64_t i = threadIdx.x; i < k; i += ET) X[f.fs[i] * nrhs + j] = xp[i];
        __syncthreads();
    }
}

__global__ void k_indef_diag(const IFrontDesc* __restrict__ desc, int64_t nfronts, double* X, int nrhs) {
    for (int64_t t = blockIdx.x; t < nfronts; t += gridDim.x) {
        const IFrontDesc f = desc[t];
        for (int64_t i = threadIdx.x; i < f.npiv; i += blockDim.x) {
            if (f.kind[i] == 0) continue;
            for (int j = 0; j < nrhs; j++) {
                if (f.kind[i] == 2) {
                    double a = f.d[i], b = f.e[i], c = f.d[i + 1];
                    double det = a * c - b * b;
                    int64_t g0 = f.fs[i], g1 = f.fs[i + 1];
                    double y0 = X[g0 * nrhs + j], y1 = X[g1 * nrhs + j];
                    X[g0 * nrhs + j] = (c * y0 - b * y1) / det;
                    X[g1 * nrhs + j] = (a * y1 - b * y0) / det;
                } else {
                    X[f.fs[i] * nrhs + j] /= f.d[i];
                }
            }
        }
    }
}

__global__ void k_indef_bwd(const IFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, double* X, int nrhs,
                            double* __restrict__ xbuf, int64_t xstride) {
    const IFrontDesc f = desc[ids[blockIdx.x]];
    int64_t k = f.npiv, nr = f.m - k;
    double* xp = xbuf + blockIdx.x * xstride;
    for (int j = 0; j < nrhs; j++) {
        for (int64_t p = threadIdx.x; p < k; p += ET) {
            double v = X[f.fs[p] * nrhs + j];
            for (int64_t r = 0; r < nr; r++) v -= f.F[(k + r) * f.m + p] * X[f.gidx[r] * nrhs + j];
            xp[p] = v;
        }
        __syncthreads();
        for (int64_t i = k - 1; i >= 0; i--) {
            double xi = xp[i];
            for (int64_t q = threadIdx.x; q < i; q += ET)
                if (!(f.kind[i] == 0 && q == i - 1)) xp[q] -= f.F[i * f.m + q] * xi;
            __syncthreads();
        }
        for (int64_t i = threadIdx.x; i < k; i += ET) X[f.fs[i] * nrhs + j] = xp[i];
        __syncthreads();
    }
}

// The level's results for the host in one copy: pivots taken and error per front.
__global__ void k_indef_results(const IFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, int64_t nl,
                                int64_t* __restrict__ out) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < nl; ii += (int64_t)gridDim.x * blockDim.x) {
        const IFrontDesc& f = desc[ids[ii]];
        out[2 * ii] = f.npiv;
        out[2 * ii + 1] = f.err;
    }
}

// the rows of L21 of the level's fronts (gbuf + goff[ii])
__global__ void k_indef_set_gidx(IFrontDesc* __restrict__ desc, const int64_t* __restrict__ ids, int64_t nl,
                                 int64_t* __restrict__ gbuf, const int64_t* __restrict__ goff) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < nl; ii += (int64_t)gridDim.x * blockDim.x)
        desc[ids[ii]].gidx = gbuf + goff[ii];
}

// desc[ids[ii]] = stage[ii] for the level's fronts
__global__ void k_indef_place_desc(IFrontDesc* __restrict__ desc, const IFrontDesc* __restrict__ stage,
                                   const int64_t* __restrict__ ids, int64_t nl) {
    for (int64_t ii = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; ii < nl; ii += (int64_t)gridDim.x * blockDim.x)
        desc[ids[ii]] = stage[ii];
}

}  // namespace

IndefEngine::IndefEngine(const Symbolic& S, const std::vector<int64_t>& colptr, const std::vector<int64_t>& rowidx,
                         double threshold)
    : S_(S), colptr_(colptr), rowidx_(rowidx), thr_(std::min(std::max(threshold, 1e-8), 0.5)) {
    RFG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    Plan P = build_plan(S, false);
    level_off_ = P.level_off;
    level_order_ = P.level_order;
    nlevels_ = P.nlevels;
    int64_t nt = (int64_t)S.fronts.size();
    RFG_CUDA(cudaMalloc(&d_desc_, std::max<int64_t>(nt, 1) * sizeof(IFrontDesc)));
    RFG_CUDA(cudaMalloc(&d_val_, std::max<size_t>(rowidx.size(), 1) * sizeof(double)));
    RFG_CUDA(cudaMalloc(&d_scale_, std::max<int64_t>(S.n, 1) * sizeof(double)));
    int64_t maxl = 1;
    for (int64_t l = 0; l < nlevels_; l++) maxl = std::max(maxl, level_off_[l + 1] - level_off_[l]);
    RFG_CUDA(cudaMalloc(&d_tpre_, (maxl + 1) * sizeof(int64_t)));
    RFG_CUDA(cudaMalloc(&d_active_, sizeof(int64_t)));
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    RFG_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    RFG_CUDA(cudaFuncSetAttribute(k_indef_trailing, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ITRAIL_SMEM));
    // fronts of at least this many rows run their block rounds on a cluster (RFG_INDEF_CLUSTER_ROWS)
    if (const char* e = getenv("RFG_INDEF_CLUSTER_ROWS")) cluster_rows_ = std::max<int64_t>(1, atoll(e));
    RFG_CUDA(cudaFuncSetAttribute(k_indef_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(2 * ISMEM_VEC_MAX * sizeof(double))));
}

void IndefEngine::release_fronts() {
    // the per-level buffers come from the library's stream-ordered pool (no device-wide sync)
    for (void* p : front_bufs_) dev_free(p, stream_);
    for (void* p : level_bufs_) dev_free(p, stream_);
    front_bufs_.clear();
    level_bufs_.clear();
}

IndefEngine::~IndefEngine() {
    if (stream_) cudaStreamSynchronize(stream_);
    release_fronts();
    cudaFree(d_desc_);
    cudaFree(d_val_);
    cudaFree(d_scale_);
    cudaFree(d_tpre_);
    cudaFree(d_active_);
    if (stream_) cudaStreamDestroy(stream_);
}

int64_t IndefEngine::factor(const double* val) {
    auto t0 = std::chrono::steady_clock::now();
    release_fronts();
    const Symbolic& S = S_;
    int64_t nt = (int64_t)S.fronts.size(), n = S.n;
    stats_ = IndefStats{};
    // column_scale (indef.rs:98-108)
    std::vector<double> scale(n, 0.0);
    for (int64_t c = 0; c < n; c++)
        for (int64_t p = colptr_[c]; p < colptr_[c + 1]; p++) {
            double v = std::fabs(val[p]);
            scale[c] = std::fmax(scale[c], v);
            scale[rowidx_[p]] = std::fmax(scale[rowidx_[p]], v);
        }
    if (!rowidx_.empty())
        RFG_CUDA(cudaMemcpyAsync(d_val_, val, rowidx_.size() * sizeof(double), cudaMemcpyHostToDevice, stream_));
    if (n > 0) RFG_CUDA(cudaMemcpyAsync(d_scale_, scale.data(), n * sizeof(double), cudaMemcpyHostToDevice, stream_));
    std::vector<IFrontDesc> desc(nt);
    std::vector<std::vector<int64_t>> fs(nt), gidx(nt);
    npiv_.assign(nt, 0);
    kf_.assign(nt, 0);
    m_.assign(nt, 0);
    lvl_d_.clear();
    lvl_kind_.clear();
    front_lvl_.assign(nt, 0);
    front_vo_.assign(nt, 0);
    front_vb_.assign(nt, 0);
    std::vector<int64_t> pos(n, -1);
    int64_t launches = 0;
    int64_t err = -1;
    for (int64_t l = 0; l < nlevels_ && err < 0; l++) {
        int64_t lo = level_off_[l], hi = level_off_[l + 1], nl = hi - lo;
        // sizes, fully summed sets and maps (indef.rs:173-199)
        std::vector<int64_t> orig_dst, orig_src, cmap, ids(level_order_.begin() + lo, level_order_.begin() + hi);
        std::vector<int64_t> cmap_off(2 * nl, 0), cpre(2 * (nl + 1), 0), kpre(nl + 1, 0);
        int64_t fbytes = 0, vbytes = 0;
        for (int64_t ii = 0; ii < nl; ii++) {
            int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            auto& F = fs[t];
            F.clear();
            for (int64_t g = sf.start; g < sf.start + sf.k; g++) F.push_back(g);
            for (int64_t c = 0; c < sf.nchild; c++) {
                int64_t ch = S.children[sf.child_off + c];
                for (int64_t x = npiv_[ch]; x < kf_[ch]; x++) F.push_back(fs[ch][x]);
            }
            kf_[t] = (int64_t)F.size();
            m_[t] = kf_[t] + sf.u;
            stats_.delayed += kf_[t] - sf.k;
            fbytes += m_[t] * m_[t];
            vbytes += kf_[t];
            // local index: own pivots, delayed variables, later rows
            for (int64_t i = 0; i < kf_[t]; i++) pos[F[i]] = i;
            for (int64_t x = 0; x < sf.u; x++) pos[S.rows[sf.rows_off + x]] = kf_[t] + x;
            // positions within the level's front buffer (this front starts at fbytes − m²)
            const int64_t fo_t = fbytes - m_[t] * m_[t];
            for (int64_t c = 0; c < sf.k; c++)
                for (int64_t p = colptr_[sf.start + c]; p < colptr_[sf.start + c + 1]; p++) {
                    orig_dst.push_back(fo_t + pos[rowidx_[p]] * m_[t] + c);
                    orig_src.push_back(p);
                }
            for (int64_t c = 0; c < 2; c++) {
                int64_t nr = 0;
                if (c < sf.nchild) {
                    int64_t ch = S.children[sf.child_off + c];
                    cmap_off[2 * ii + c] = (int64_t)cmap.size();
                    for (int64_t g : gidx[ch]) cmap.push_back(pos[g]);
                    nr = (int64_t)gidx[ch].size();
                }
                cpre[c * (nl + 1) + ii + 1] = cpre[c * (nl + 1) + ii] + nr;
            }
            kpre[ii + 1] = kpre[ii] + kf_[t];
        }
        // device buffers of the level: fronts, fs, d, e, kind, maps
        double* Fbuf = nullptr;
        int64_t* ibuf = nullptr;
        double* debuf = nullptr;
        int8_t* kbuf = nullptr;
        int64_t* mbuf = nullptr;
        Fbuf = (decltype(Fbuf))dev_alloc(std::max<int64_t>(fbytes, 1) * sizeof(double), stream_);
        ibuf = (decltype(ibuf))dev_alloc(std::max<int64_t>(vbytes + nl, 1) * sizeof(int64_t), stream_);
        debuf = (decltype(debuf))dev_alloc(std::max<int64_t>(2 * vbytes, 1) * sizeof(double), stream_);
        kbuf = (decltype(kbuf))dev_alloc(std::max<int64_t>(vbytes, 1), stream_);
        const int64_t no = (int64_t)orig_dst.size();
        mbuf = (decltype(mbuf))dev_alloc(
            std::max<size_t>(2 * orig_dst.size() + cmap.size() + cpre.size() + kpre.size() + 2 * nl, 1) * sizeof(int64_t),
            stream_);
        front_bufs_.push_back(Fbuf);
        front_bufs_.push_back(ibuf);
        front_bufs_.push_back(debuf);
        front_bufs_.push_back(kbuf);
        level_bufs_.push_back(mbuf);
        std::vector<int64_t> ibuf_h;
        int64_t fo = 0, vo = 0;
        for (int64_t ii = 0; ii < nl; ii++) {
            int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            IFrontDesc& D = desc[t];
            D = IFrontDesc{};
            D.F = Fbuf + fo;
            D.m = m_[t];
            D.kf = kf_[t];
            D.k = sf.k;
            D.start = sf.start;
            D.u = sf.u;
            D.fs = ibuf + vo;
            D.d = debuf + vo;
            D.e = debuf + vbytes + vo;
            D.kind = kbuf + vo;
            D.nchild = sf.nchild;
            for (int64_t c = 0; c < sf.nchild; c++) {
                D.child[c] = S.children[sf.child_off + c];
                D.cmap[c] = mbuf + 2 * no + cmap_off[2 * ii + c];
            }
            D.npiv = 0;
            D.err = -1;
            D.root = sf.parent < 0;
            D.done = 0;
            D.p = 0;
            D.width = IKB;
            ibuf_h.insert(ibuf_h.end(), fs[t].begin(), fs[t].end());
            fo += m_[t] * m_[t];
            vo += kf_[t];
        }
        std::vector<int64_t> mh(orig_dst);
        mh.insert(mh.end(), orig_src.begin(), orig_src.end());
        mh.insert(mh.end(), cmap.begin(), cmap.end());
        const int64_t cpre_off = (int64_t)mh.size();
        mh.insert(mh.end(), cpre.begin(), cpre.end());
        const int64_t kpre_off = (int64_t)mh.size();
        mh.insert(mh.end(), kpre.begin(), kpre.end());
        int64_t ids_off = (int64_t)mh.size();
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
            RFG_CUDA(cudaMemcpyAsync(ibuf, ibuf_h.data(), ibuf_h.size() * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
        {
            // the level's descriptors in one copy, then into their places
            std::vector<IFrontDesc> stage(nl);
            for (int64_t ii = 0; ii < nl; ii++) stage[ii] = desc[ids[ii]];
            IFrontDesc* dstage = (IFrontDesc*)dev_alloc(nl * sizeof(IFrontDesc), stream_);
            level_bufs_.push_back(dstage);
            RFG_CUDA(cudaMemcpyAsync(dstage, stage.data(), nl * sizeof(IFrontDesc), cudaMemcpyHostToDevice, stream_));
            k_indef_place_desc<<<(unsigned)std::min<int64_t>((nl + 127) / 128, 1024), 128, 0, stream_>>>(
                (IFrontDesc*)d_desc_, dstage, mbuf + ids_off, nl);
        }
        double* wbuf = nullptr;
        int64_t wstride = IKB;
        for (int64_t ii = 0; ii < nl; ii++) wstride = std::max(wstride, m_[ids[ii]]);
        wbuf = (decltype(wbuf))dev_alloc(nl * 4 * wstride * sizeof(double), stream_);
        const size_t block_smem = wstride <= ISMEM_VEC_MAX ? 2 * wstride * sizeof(double) : 0;
        level_bufs_.push_back(wbuf);
        RFG_CUDA(cudaMemsetAsync(Fbuf, 0, std::max<int64_t>(fbytes, 1) * sizeof(double), stream_));
        if (no > 0)
            k_indef_asm_orig<<<(unsigned)std::min<int64_t>((no + 255) / 256, num_sms_ * 8), 256, 0, stream_>>>(
                Fbuf, mbuf, mbuf + no, no, d_val_);
        for (int ci = 0; ci < 2; ci++) {
            const int64_t rows = cpre[ci * (nl + 1) + nl];
            if (rows > 0)
                k_indef_asm_child<<<(unsigned)std::min<int64_t>((rows + 7) / 8, num_sms_ * 8), 256, 0, stream_>>>(
                    (IFrontDesc*)d_desc_, mbuf + ids_off, nl, mbuf + cpre_off + ci * (nl + 1), ci);
        }
        if (kpre[nl] > 0)
            k_indef_mirror<<<(unsigned)std::min<int64_t>((kpre[nl] + 7) / 8, num_sms_ * 8), 256, 0, stream_>>>(
                (IFrontDesc*)d_desc_, mbuf + ids_off, nl, mbuf + kpre_off);
        launches += 5;
        // block rounds: pivot search and eager updates of one block per front (one CTA
        // each), then the trailing updates of those blocks on all SMs, until every front
        // of the level is done (checked after rounds 1, 2, 4, 8 and then every 8)
        {
            const unsigned tgrid = (unsigned)(num_sms_ * 4);
            int64_t round = 0, active = 1;
            while (active > 0) {
if (nsmall > 0)
                    k_indef_block<<<(unsigned)nsmall, ET, block_smem, stream_>>>(
                        (IFrontDesc*)d_desc_, mbuf + small_off, d_scale_, thr_, wbuf, wstride);
                if (nbig > 0)
                    k_indef_block_cl<<<(unsigned)(nbig * ICS), ET, 0, stream_>>>(
                        (IFrontDesc*)d_desc_, mbuf + big_off, d_scale_, thr_, wbuf + nsmall * 4 * wstride, wstride);
                k_indef_tiles<<<1, 1024, 0, stream_>>>((IFrontDesc*)d_desc_, mbuf + ids_off, nl, d_tpre_,
                                                      d_active_);
                k_indef_trailing<<<tgrid, 256, ITRAIL_SMEM, stream_>>>((IFrontDesc*)d_desc_, mbuf + ids_off, nl,
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
        // results of the level: pivots eliminated, the permuted fully summed sets, and D
        // (one copy each)
        int64_t* rbuf = (int64_t*)dev_alloc(std::max<int64_t>(2 * nl, 1) * sizeof(int64_t), stream_);
        level_bufs_.push_back(rbuf);
        k_indef_results<<<(unsigned)std::min<int64_t>((nl + 255) / 256, 1024), 256, 0, stream_>>>(
            (IFrontDesc*)d_desc_, mbuf + ids_off, nl, rbuf);
        std::vector<int64_t> out(2 * nl);
        RFG_CUDA(cudaMemcpyAsync(out.data(), rbuf, 2 * nl * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
        if (!ibuf_h.empty())
            RFG_CUDA(cudaMemcpyAsync(ibuf_h.data(), ibuf, ibuf_h.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, stream_));
        lvl_d_.emplace_back(2 * vbytes);
        lvl_kind_.emplace_back(vbytes);
        if (vbytes > 0) {
            RFG_CUDA(cudaMemcpyAsync(lvl_d_.back().data(), debuf, 2 * vbytes * sizeof(double), cudaMemcpyDeviceToHost,
                                     stream_));
            RFG_CUDA(cudaMemcpyAsync(lvl_kind_.back().data(), kbuf, vbytes, cudaMemcpyDeviceToHost, stream_));
        }
        RFG_CUDA(cudaStreamSynchronize(stream_));
        vo = 0;
        for (int64_t ii = 0; ii < nl; ii++) {
            int64_t t = ids[ii];
            const SymFront& sf = S.fronts[t];
            npiv_[t] = out[2 * ii];
            const int64_t e_ii = out[2 * ii + 1];
            if (e_ii >= 0 && err < 0) err = e_ii;
            front_lvl_[t] = (int64_t)lvl_d_.size() - 1;
            front_vo_[t] = vo;
            front_vb_[t] = vbytes;
            fs[t].assign(ibuf_h.begin() + vo, ibuf_h.begin() + vo + kf_[t]);
            vo += kf_[t];
            gidx[t].assign(fs[t].begin() + npiv_[t], fs[t].end());
            for (int64_t x = 0; x < sf.u; x++) gidx[t].push_back(S.rows[sf.rows_off + x]);
            desc[t].npiv = npiv_[t];
        }
        // rows of L21 per front, for the parent's maps and the solve
        std::vector<int64_t> gh;
        std::vector<int64_t> goff(nl);
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
        k_indef_set_gidx<<<(unsigned)std::min<int64_t>((nl + 255) / 256, 1024), 256, 0, stream_>>>(
            (IFrontDesc*)d_desc_, mbuf + ids_off, nl, gbuf, gbuf + gh.size());
        for (int64_t ii = 0; ii < nl; ii++) desc[ids[ii]].gidx = gbuf + goff[ii];
        RFG_CUDA(cudaStreamSynchronize(stream_));
    }
    if (err >= 0) {
        stats_.launches = launches;
        return err;
    }
    // inertia and statistics (indef.rs:125-155)
    for (int64_t t = 0; t < nt; t++) {
        int64_t k = npiv_[t];
        // D and the pivot kinds of front t, from its level's host copy
        const double* d = lvl_d_[front_lvl_[t]].data() + front_vo_[t];
        const double* e = lvl_d_[front_lvl_[t]].data() + front_vb_[t] + front_vo_[t];
        const int8_t* kind = lvl_kind_[front_lvl_[t]].data() + front_vo_[t];
        int64_t i = 0;
        while (i < k) {
            if (kind[i] == 2) {
                stats_.two_by_two++;
                double a = d[i], b = e[i], c = d[i + 1];
                double det = a * c - b * b;
                if (det < 0.0) {
                    stats_.neg++;
                    stats_.pos++;
                } else if (a + c < 0.0) {
                    stats_.neg += 2;
                } else {
                    stats_.pos += 2;
                }
                i += 2;
            } else {
                if (d[i] < 0.0)
                    stats_.neg++;
                else if (d[i] > 0.0)
                    stats_.pos++;
                else
                    stats_.zero++;
                i += 1;
            }
        }
        stats_.factor_size += k * (k > 0 ? k - 1 : 0) / 2 + (m_[t] - k) * k;
    }
    stats_.launches = launches;
    stats_.t_factor_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return -1;
}

void IndefEngine::solve_device(double* X, int64_t nrhs) {
    int64_t nt = (int64_t)S_.fronts.size();
    if (nt == 0 || nrhs <= 0) return;
    int64_t maxl = 0, xstride = 1;
    for (int64_t l = 0; l < nlevels_; l++) maxl = std::max(maxl, level_off_[l + 1] - level_off_[l]);
    for (int64_t t = 0; t < nt; t++) xstride = std::max(xstride, npiv_[t]);
    double* xbuf = nullptr;
    int64_t* dids = nullptr;
    RFG_CUDA(cudaMallocAsync((void**)&xbuf, maxl * xstride * sizeof(double), stream_));
    RFG_CUDA(cudaMallocAsync((void**)&dids, nt * sizeof(int64_t), stream_));
    RFG_CUDA(cudaMemcpyAsync(dids, level_order_.data(), nt * sizeof(int64_t), cudaMemcpyHostToDevice, stream_));
    for (int64_t l = 0; l < nlevels_; l++) {
        int64_t lo = level_off_[l], nl = level_off_[l + 1] - lo;
        k_indef_fwd<<<(unsigned)nl, ET, 0, stream_>>>((IFrontDesc*)d_desc_, dids + lo, X, (int)nrhs, xbuf, xstride);
    }
    k_indef_diag<<<148, 256, 0, stream_>>>((IFrontDesc*)d_desc_, nt, X, (int)nrhs);
    for (int64_t l = nlevels_ - 1; l >= 0; l--) {
        int64_t lo = level_off_[l], nl = level_off_[l + 1] - lo;
        k_indef_bwd<<<(unsigned)nl, ET, 0, stream_>>>((IFrontDesc*)d_desc_, dids + lo, X, (int)nrhs, xbuf, xstride);
    }
    RFG_CUDA(cudaGetLastError());
    RFG_CUDA(cudaFreeAsync(xbuf, stream_));
    RFG_CUDA(cudaFreeAsync(dids, stream_));
}

}  // namespace rfg
