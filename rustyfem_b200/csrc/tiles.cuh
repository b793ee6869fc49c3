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
template <typename T, int ROWS, int NT, typename D>
__device__ __forceinline__ void load_tile(D (*dst)[NB + 1], const T* __restrict__ src, int64_t ld, int nr, int jb) {
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
            for (int e = 0; e < VEC; e++) dst[rr][c + e] = (D)v[u][e];
        }
    }
}

// The NB × NB inverse diagonal block (contiguous, 16-byte aligned) into dst, NT threads.
template <int NT>
__device__ __forceinline__ void load_linv(double (*dst)[NB + 1], const double* __restrict__ src) {
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
            dst[e / NB][e % NB] = v[u].x;
            dst[e / NB][e % NB + 1] = v[u].y;
        }
    }
}

}  // namespace rfg
