// Small device utilities shared by the set-up kernels: an exclusive prefix sum of
// 64-bit counts (block scans, then the block totals scanned the same way, then the
// totals added back) and a per-row sort of 64-bit keys.

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <mutex>

#include "engine.h"
#include "tiles.cuh"

namespace rfg {

namespace {

constexpr int SCAN_THREADS = 256;
constexpr int SCAN_PER_THREAD = 8;
constexpr int64_t SCAN_BLOCK = SCAN_THREADS * SCAN_PER_THREAD;

// Exclusive scan of d[blk·2048, …) in place; the block's total goes to sums[blk].
__global__ void __launch_bounds__(SCAN_THREADS) k_scan_blocks(int64_t* __restrict__ d, int64_t n,
                                                              int64_t* __restrict__ sums) {
    __shared__ int64_t warp_tot[SCAN_THREADS / 32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_BLOCK + (int64_t)threadIdx.x * SCAN_PER_THREAD;
    int64_t v[SCAN_PER_THREAD];
    int64_t run = 0;
#pragma unroll
    for (int i = 0; i < SCAN_PER_THREAD; i++) {
        const int64_t x = base + i < n ? d[base + i] : 0;
        v[i] = run;
        run += x;
    }
    // inclusive scan of the thread totals within the warp, then across warps
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int64_t inc = run;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int64_t y = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) warp_tot[warp] = inc;
    __syncthreads();
    int64_t woff = 0;
    for (int w = 0; w < warp; w++) woff += warp_tot[w];
    const int64_t toff = woff + inc - run;
#pragma unroll
    for (int i = 0; i < SCAN_PER_THREAD; i++)
        if (base + i < n) d[base + i] = v[i] + toff;
    if (threadIdx.x == SCAN_THREADS - 1) sums[blockIdx.x] = toff + run;
}

__global__ void k_scan_add(int64_t* __restrict__ d, int64_t n, const int64_t* __restrict__ sums) {
    const int64_t add = sums[blockIdx.x];
    const int64_t b0 = (int64_t)blockIdx.x * SCAN_BLOCK;
    for (int64_t i = b0 + threadIdx.x; i < min(n, b0 + SCAN_BLOCK); i += blockDim.x) d[i] += add;
}

// Rows [rp[r], rp[r+1]) of key sorted ascending, one warp per row, bitonic in shared
// memory for rows of at most ROWSORT_MAX keys; longer rows are sorted by lane 0 (shell
// sort in global memory, deterministic). Keys must be distinct within a row for the
// result not to depend on the input order.
constexpr int ROWSORT_MAX = 1024;
constexpr int ROWSORT_WARPS = 8;

__global__ void __launch_bounds__(ROWSORT_WARPS * 32) k_sort_rows(uint64_t* __restrict__ key,
                                                                 const int64_t* __restrict__ rp, int64_t nrows) {
    extern __shared__ uint64_t rs_smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t r = (int64_t)blockIdx.x * ROWSORT_WARPS + warp;
    if (r >= nrows) return;
    uint64_t* a = rs_smem + (size_t)warp * ROWSORT_MAX;
    const int64_t b = rp[r], len = rp[r + 1] - b;
    if (len < 2) return;
    if (len > ROWSORT_MAX) {
        if (lane == 0) {
            uint64_t* k = key + b;
            for (int64_t gap = len / 2; gap > 0; gap /= 2)
                for (int64_t i = gap; i < len; i++) {
                    const uint64_t t = k[i];
                    int64_t j = i;
                    for (; j >= gap && k[j - gap] > t; j -= gap) k[j] = k[j - gap];
                    k[j] = t;
                }
        }
        return;
    }
    int P = 2;
    while (P < len) P <<= 1;
    for (int i = lane; i < P; i += 32) a[i] = i < len ? key[b + i] : ~0ull;
    __syncwarp();
    for (int k = 2; k <= P; k <<= 1)
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = lane; i < P; i += 32) {
                const int l = i ^ j;
                if (l > i) {
                    const bool up = (i & k) == 0;
                    const uint64_t x = a[i], y = a[l];
                    if ((x > y) == up) {
                        a[i] = y;
                        a[l] = x;
                    }
                }
            }
            __syncwarp();
        }
    for (int i = lane; i < len; i += 32) key[b + i] = a[i];
}

}  // namespace

int64_t scan_tmp_elems(int64_t n) {
    int64_t t = 0;
    while (n > 1) {
        n = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
        t += n;
    }
    return t + 1;
}

void exclusive_scan_i64(int64_t* d, int64_t n, int64_t* tmp, cudaStream_t st) {
    if (n <= 0) return;
    const int64_t nb = (n + SCAN_BLOCK - 1) / SCAN_BLOCK;
    k_scan_blocks<<<(unsigned)nb, SCAN_THREADS, 0, st>>>(d, n, tmp);
    RFG_CUDA(cudaGetLastError());
    if (nb == 1) return;
    exclusive_scan_i64(tmp, nb, tmp + nb, st);
    k_scan_add<<<(unsigned)nb, SCAN_THREADS, 0, st>>>(d, n, tmp);
    RFG_CUDA(cudaGetLastError());
}

void sort_rows_u64(uint64_t* key, const int64_t* rp, int64_t nrows, cudaStream_t st) {
    if (nrows <= 0) return;
    static std::mutex mu;
    static bool attr[64] = {};
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw CudaError("sort_rows_u64: device ordinal out of range");
    const size_t smem = (size_t)ROWSORT_WARPS * ROWSORT_MAX * sizeof(uint64_t);
    {
        std::lock_guard<std::mutex> lock(mu);
        if (!attr[dev]) {
            RFG_CUDA(cudaFuncSetAttribute(k_sort_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            attr[dev] = true;
        }
    }
    const int64_t nb = (nrows + ROWSORT_WARPS - 1) / ROWSORT_WARPS;
    k_sort_rows<<<(unsigned)nb, ROWSORT_WARPS * 32, smem, st>>>(key, rp, nrows);
    RFG_CUDA(cudaGetLastError());
}

namespace {
__global__ void k_selftest_reciprocal(const double* __restrict__ x, double* __restrict__ r, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        r[i] = recip_newton(x[i]);
}
}  // namespace

}  // namespace rfg

// The pivot blocks' reciprocal (recip_newton) on the current device for n host values
// x > 0, into r: lets a test compare it with the correctly rounded 1/x.
extern "C" int32_t rfg_selftest_reciprocal(const double* x, double* r, size_t n) {
    using namespace rfg;
    if (n == 0) return 0;
    double* d = nullptr;
    if (cudaMalloc(&d, 2 * n * sizeof(double)) != cudaSuccess) return -1;
    bool ok = cudaMemcpy(d, x, n * sizeof(double), cudaMemcpyHostToDevice) == cudaSuccess;
    if (ok) {
        k_selftest_reciprocal<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256>>>(d, d + n, (int64_t)n);
        ok = cudaGetLastError() == cudaSuccess &&
             cudaMemcpy(r, d + n, n * sizeof(double), cudaMemcpyDeviceToHost) == cudaSuccess;
    }
    cudaFree(d);
    return ok ? 0 : -1;
}
