// Tile loads shared by the panel and solve kernels: global -> shared memory staging
// with many 16-byte loads in flight per thread.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <type_traits>

#include "plan.h"

namespace rfg {

// Loads the ROWS × NB tile src[rr·ld + c] (rr < nr, c < jb; zero elsewhere) into the
// shared tile dst (element type D) with NT threads. Each thread issues its 16-byte loads in
// batches of up to 16 before storing any, so a CTA keeps hundreds of loads in flight
// instead of waiting for one load per element (rows are 16-byte aligned: panel offsets
// are multiples of 32 elements, row strides multiples of 8, j0 a multiple of 64).
// Rows of dst are P elements apart (P = NB + 1 for the [NB + 1] tiles).
template <typename T, int ROWS, int NT, int P, typename D>
__device__ __forceinline__ void load_tile_p(D* dst, const T* __restrict__ src, int64_t ld, int nr, int jb) {
    constexpr int VEC = 16 / (int)sizeof(T);
    constexpr int PER_ROW = NB / VEC;
    constexpr int PER_THREAD = ROWS * PER_ROW / NT;
    constexpr int BATCH = PER_THREAD < 16 ? PER_THREAD : 16;
    static_assert((ROWS * PER_ROW) % NT == 0 && PER_THREAD % BATCH == 0, "tile split");
    using V = typename std::conditional<sizeof(T) == 4, float4, double2>::type;
#pragma unroll 1
    for (int b0 = 0; b0 < PER_THREAD; b0 += BATCH) {
        T v[BATCH][VEC];
#pragma unroll
        for (int u = 0; u < BATCH; u++) {
            int idx = (b0 + u) * NT + (int)threadIdx.x;
            int rr = idx / PER_ROW, c = (idx - rr * PER_ROW) * VEC;
            const T* q = src + (int64_t)rr * ld + c;
            if (rr < nr && c + VEC <= jb) {
                *reinterpret_cast<V*>(&v[u][0]) = __ldg(reinterpret_cast<const V*>(q));
            } else {
#pragma unroll
                for (int e = 0; e < VEC; e++) v[u][e] = (rr < nr && c + e < jb) ? q[e] : T(0);
            }
        }
#pragma unroll
        for (int u = 0; u < BATCH; u++) {
            int idx = (b0 + u) * NT + (int)threadIdx.x;
            int rr = idx / PER_ROW, c = (idx - rr * PER_ROW) * VEC;
#pragma unroll
            for (int e = 0; e < VEC; e++) dst[rr * P + c + e] = (D)v[u][e];
        }
    }
}
template <typename T, int ROWS, int NT, typename D>
__device__ __forceinline__ void load_tile(D (*dst)[NB + 1], const T* __restrict__ src, int64_t ld, int nr, int jb) {
    load_tile_p<T, ROWS, NT, NB + 1>(&dst[0][0], src, ld, nr, jb);
}

// The NB × NB inverse diagonal block (contiguous, 16-byte aligned) into dst, NT threads.
template <int NT, int P>
__device__ __forceinline__ void load_linv_p(double* dst, const double* __restrict__ src) {
    constexpr int PER_THREAD = NB * NB / 2 / NT;
    constexpr int BATCH = PER_THREAD < 16 ? PER_THREAD : 16;
    static_assert(PER_THREAD % BATCH == 0, "block split");
    const double2* s2 = reinterpret_cast<const double2*>(src);
#pragma unroll 1
    for (int b0 = 0; b0 < PER_THREAD; b0 += BATCH) {
        double2 v[BATCH];
#pragma unroll
        for (int u = 0; u < BATCH; u++) v[u] = __ldg(&s2[(b0 + u) * NT + threadIdx.x]);
#pragma unroll
        for (int u = 0; u < BATCH; u++) {
            int e = 2 * ((b0 + u) * NT + (int)threadIdx.x);
            dst[(e / NB) * P + e % NB] = v[u].x;
            dst[(e / NB) * P + e % NB + 1] = v[u].y;
        }
    }
}
template <int NT>
__device__ __forceinline__ void load_linv(double (*dst)[NB + 1], const double* __restrict__ src) {
    load_linv_p<NT, NB + 1>(&dst[0][0], src);
}

// 1/p for a positive normal p: Newton–Raphson iteration on f(r) = 1/r − p,
// r ← r + r·(1 − p·r), from the hardware's approximate reciprocal (rcp.approx.ftz.f64, a
// relative error near 2^-23); each step squares the relative error, so two steps leave the
// rounding of the last fused multiply-add: within one unit in the last place of 1/p. Several
// times shorter as a dependency chain than the IEEE division 1.0 / p.
__device__ __forceinline__ double recip_newton(double p) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(p));
    double e = fma(-p, r, 1.0);
    r = fma(r, e, r);
    e = fma(-p, r, 1.0);
    return fma(r, e, r);
}

// Programmatic dependent launch (PDL): a kernel launched with the programmatic
// stream-serialization attribute may start while its predecessor in the stream still
// runs. pdl_wait() blocks until the predecessor grid has completed and its memory is
// visible (it returns at once for a kernel launched without the attribute), so a kernel
// reads or writes nothing that its predecessors produce or consume before it;
// pdl_launch_dependents() lets the next kernel start once every CTA of this grid has
// issued it.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// cp.async of 16 bytes global -> shared (cached in L2 only), src_bytes ∈ [0, 16] read and
// the rest of the 16 bytes zero-filled; both addresses 16-byte aligned.
__device__ __forceinline__ void cp_async16(void* dst, const void* src, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// cp.async of the tile src[rr·ld + c] (rr < nr, c < ncol) into dst[rr·pitch + c] for
// rr < rows, c < cols, zero-filled outside (cols a multiple of 16 bytes, pitch·sizeof(T)
// a multiple of 16 bytes, src rows 16-byte aligned). Threads [0, nt) issue the copies.
template <typename T>
__device__ __forceinline__ void cp_async_tile(T* dst, int pitch, const T* src, int64_t ld, int nr, int ncol, int rows,
                                              int cols, int nt) {
    constexpr int VEC = 16 / (int)sizeof(T);
    const int per_row = cols / VEC;
    // (row, chunk) of this thread's first copy, then advanced by nt chunks without division
    int rr = (int)threadIdx.x / per_row, cc = (int)threadIdx.x - rr * per_row;
    const int dr = nt / per_row, dc = nt - dr * per_row;
    for (; rr < rows; rr += dr) {
        const int c = cc * VEC;
        int bytes = 0;
        const T* s = src;
        if (rr < nr && c < ncol) {
            bytes = min(VEC, ncol - c) * (int)sizeof(T);
            s = src + (int64_t)rr * ld + c;
        }
        cp_async16(dst + (int64_t)rr * pitch + c, s, bytes);
        cc += dc;
        if (cc >= per_row) {
            cc -= per_row;
            rr++;
        }
    }
}

// cp.async of n contiguous 16-byte chunks (both ends 16-byte aligned), threads [0, nt).
__device__ __forceinline__ void cp_async_flat(void* dst, const void* src, int n, int nt) {
    for (int i = threadIdx.x; i < n; i += nt)
        cp_async16(static_cast<char*>(dst) + 16 * (size_t)i, static_cast<const char*>(src) + 16 * (size_t)i, 16);
}
// Index i of the segment that holds item b: pre[i] <= b < pre[i+1], i in [0, n) (pre
// nondecreasing, pre[0] = 0, pre[n] > b). Warp-cooperative: every round the 32 lanes
// probe 32 evenly spaced entries and the ballot narrows the range 32-fold, so a launch
// over thousands of segments pays ~3 dependent loads per CTA instead of ~13. Must be
// called by all 32 lanes of a warp with the same b.
__device__ __forceinline__ int64_t find_slot_warp(const int64_t* __restrict__ pre, int64_t n, int64_t b) {
    const int lane = threadIdx.x & 31;
    int64_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const int64_t step = (hi - lo + 31) / 32;
        const int64_t idx = lo + lane * step;
        const bool ok = idx < hi && pre[idx] <= b;
        const unsigned m = __ballot_sync(0xffffffffu, ok);
        const int k = 31 - __clz(m);  // lane 0 probes lo, where pre[lo] <= b
        lo += k * step;
        hi = min(hi, lo + step);
    }
    return lo;
}

}  // namespace rfg
