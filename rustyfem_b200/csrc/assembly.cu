// Assembly of K on the GPU (see assembly.h). Compiled with -fmad=false: every product
// and sum of the element matrix and of the assembly is rounded separately, in the
// reference's order, so that the values equal the reference's bit for bit.

#include "assembly.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

#include "engine.h"

namespace rfg {

namespace {

// position of row r in rows[lo, hi) (sorted), or -1 when r is not there
__device__ __forceinline__ int64_t find_row(const int64_t* __restrict__ rows, int64_t lo, int64_t hi, int64_t r) {
    const int64_t end = hi;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (rows[mid] < r)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < end && rows[lo] == r) ? lo : -1;
}

// The entry (ia, ib) of element pair (e, a, b), ia >= ib, or -1 (no equation or not a lower
// pair); -2 when the entry is missing in the pattern.
__device__ __forceinline__ int64_t pair_entry(const int64_t* __restrict__ edof, const int64_t* __restrict__ colptr,
                                              const int64_t* __restrict__ rowidx, int64_t nd, int64_t t, int64_t* ia,
                                              int64_t* ib) {
    const int64_t e = t / (nd * nd), ab = t - e * nd * nd;
    const int64_t a = ab / nd, b = ab - a * nd;
    *ia = edof[e * nd + a];
    *ib = edof[e * nd + b];
    if (*ia < 0 || *ib < 0 || *ia < *ib) return -1;
    const int64_t p = find_row(rowidx, colptr[*ib], colptr[*ib + 1], *ia);
    return p < 0 ? -2 : p;
}

__global__ void k_asm_count(const int64_t* __restrict__ edof, const int64_t* __restrict__ colptr,
                            const int64_t* __restrict__ rowidx, int64_t nd, int64_t total,
                            unsigned long long* __restrict__ cnt, long long* __restrict__ bad) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t ia, ib;
        const int64_t p = pair_entry(edof, colptr, rowidx, nd, t, &ia, &ib);
        if (p >= 0) {
            atomicAdd(&cnt[p], 1ull);
        } else if (p == -2) {
            // the first pair (in enumeration order) that misses the pattern
            atomicMin(&bad[0], (long long)t);
        }
    }
}

__global__ void k_asm_fill(const int64_t* __restrict__ edof, const int64_t* __restrict__ colptr,
                           const int64_t* __restrict__ rowidx, int64_t nd, int64_t total,
                           unsigned long long* __restrict__ cursor, uint64_t* __restrict__ key) {
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t ia, ib;
        const int64_t p = pair_entry(edof, colptr, rowidx, nd, t, &ia, &ib);
        if (p >= 0) key[atomicAdd(&cursor[p], 1ull)] = (uint64_t)t;
    }
}

// K[p] = Σ over the entry's contributions in (element, a, b) order of ½(ke[a,b] + ke[b,a]),
// zero terms skipped, from 0 (SystemMatrix::zero then add: src/fem/assembly.rs:402-409)
__global__ void k_asm_gather(const int64_t* __restrict__ start, const uint64_t* __restrict__ key,
                             const double* __restrict__ ke, int64_t nd, int64_t nnz, double* __restrict__ val) {
    for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < nnz; p += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int64_t q = start[p]; q < start[p + 1]; q++) {
            const int64_t t = (int64_t)key[q];
            const int64_t e = t / (nd * nd), ab = t - e * nd * nd;
            const int64_t a = ab / nd, b = ab - a * nd;
            const double v = 0.5 * (ke[t] + ke[e * nd * nd + b * nd + a]);
            if (v != 0.0) s += v;
        }
        val[p] = s;
    }
}

constexpr int KE_THREADS = 192;

// One C3D8 element per CTA: src/elements/continuum3d.rs:39-84 (shape derivatives,
// Jacobian, 2×2×2 Gauss points, ξ fastest), src/elements/common.rs:48-70 (inv3),
// :142-200 (B and the volumetric B-bar), src/materials/elastic.rs:57-70 (D) and
// src/elements/common.rs:264-289 (K += Bᵀ D B w per point, zero terms skipped).
// Each sum runs in the reference's order from +0.
__global__ void __launch_bounds__(KE_THREADS) k_ke_hex8(const double* __restrict__ xyz, const int64_t* __restrict__ conn,
                                                        const double* __restrict__ emod, double nu, int64_t nelem,
                                                        double* __restrict__ ke, long long* __restrict__ bad) {
    constexpr int ND = 24, NS = 6;
    __shared__ double sx[24];
    __shared__ double sdn[8][3][8];
    __shared__ double sji[8][3][3];
    __shared__ double sw[8];
    __shared__ double sB[8][NS * ND];
    __shared__ double sdb[8][NS * ND];
    __shared__ double savg[ND];
    __shared__ double sD[NS * NS];
    __shared__ int sbad;
    const int t = threadIdx.x;
    for (int64_t e = blockIdx.x; e < nelem; e += gridDim.x) {
        if (t < 24) sx[t] = xyz[conn[e * 8 + t / 3] * 3 + t % 3];
        if (t == 0) sbad = 0;
        if (t < NS * NS) {
            const double E = emod[e];
            const double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
            const double mu = E / (2.0 * (1.0 + nu));
            const int i = t / NS, j = t % NS;
            double d = 0.0;
            if (i < 3 && j < 3)
                d = i == j ? lam + 2.0 * mu : lam;
            else if (i == j)
                d = mu;
            sD[t] = d;
        }
        if (t < 64) {
            const int q = t >> 3, i = t & 7;
            const double g = 0.5773502691896258;
            const double p0 = (q & 1) ? g : -g, p1 = (q & 2) ? g : -g, p2 = (q & 4) ? g : -g;
            const double n0 = (i == 1 || i == 2 || i == 5 || i == 6) ? 1.0 : -1.0;
            const double n1 = (i == 2 || i == 3 || i == 6 || i == 7) ? 1.0 : -1.0;
            const double n2 = i >= 4 ? 1.0 : -1.0;
            const double f0 = 1.0 + p0 * n0, f1 = 1.0 + p1 * n1, f2 = 1.0 + p2 * n2;
            sdn[q][0][i] = 0.125 * n0 * f1 * f2;
            sdn[q][1][i] = 0.125 * n1 * f0 * f2;
            sdn[q][2][i] = 0.125 * n2 * f0 * f1;
        }
        for (int k = t; k < 8 * NS * ND; k += KE_THREADS) (&sB[0][0])[k] = 0.0;
        __syncthreads();
        if (t < 8) {
            // Jacobian and its inverse at point t
            const int q = t;
            double J[3][3];
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    double s = 0.0;
                    for (int i = 0; i < 8; i++) s += sdn[q][r][i] * sx[i * 3 + c];
                    J[r][c] = s;
                }
            const double det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                               J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                               J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
            const double id = 1.0 / det;
            sji[q][0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) * id;
            sji[q][0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) * id;
            sji[q][0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) * id;
            sji[q][1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) * id;
            sji[q][1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) * id;
            sji[q][1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) * id;
            sji[q][2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) * id;
            sji[q][2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) * id;
            sji[q][2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) * id;
            sw[q] = det * 1.0;
            if (det <= 0.0) sbad = 1;
        }
        __syncthreads();
        if (sbad) {
            if (t == 0) atomicMin(bad, (long long)e);
            __syncthreads();
            continue;
        }
        if (t < 64) {
            // dN/dx at point q for node i, into the B matrix
            const int q = t >> 3, i = t & 7;
            double d[3];
            for (int c = 0; c < 3; c++) {
                double s = 0.0;
                for (int r = 0; r < 3; r++) s += sji[q][c][r] * sdn[q][r][i];
                d[c] = s;
            }
            double* b = sB[q];
            const int c = 3 * i;
            b[c] = d[0];
            b[ND + c + 1] = d[1];
            b[2 * ND + c + 2] = d[2];
            b[3 * ND + c] = d[1];
            b[3 * ND + c + 1] = d[0];
            b[4 * ND + c] = d[2];
            b[4 * ND + c + 2] = d[0];
            b[5 * ND + c + 1] = d[2];
            b[5 * ND + c + 2] = d[1];
        }
        __syncthreads();
        if (t < ND) {
            // volume-averaged dilatation of column t
            double wsum = 0.0;
            for (int q = 0; q < 8; q++) wsum += sw[q];
            double s = 0.0;
            for (int q = 0; q < 8; q++) s += sw[q] * (sB[q][t] + sB[q][ND + t] + sB[q][2 * ND + t]);
            savg[t] = s / wsum;
        }
        __syncthreads();
        {
            // B-bar: column c of point q gets (avg − vol)/3 on its three normal rows
            const int q = t / ND, c = t % ND;
            double* b = sB[q];
            const double corr = (savg[c] - (b[c] + b[ND + c] + b[2 * ND + c])) / 3.0;
            for (int r = 0; r < 3; r++) b[r * ND + c] += corr;
        }
        __syncthreads();
        for (int k = t; k < 8 * NS * ND; k += KE_THREADS) {
            // D·B at point q
            const int q = k / (NS * ND), rc = k % (NS * ND), r = rc / ND, c = rc % ND;
            double s = 0.0;
            for (int m = 0; m < NS; m++) {
                const double drm = sD[r * NS + m];
                if (drm != 0.0) s += drm * sB[q][m * ND + c];
            }
            sdb[q][rc] = s;
        }
        __syncthreads();
        for (int k = t; k < ND * ND; k += KE_THREADS) {
            const int i = k / ND, j = k % ND;
            double s = 0.0;
            for (int q = 0; q < 8; q++)
                for (int r = 0; r < NS; r++) {
                    const double bri = sB[q][r * ND + i] * sw[q];
                    if (bri != 0.0) s += bri * sdb[q][r * ND + j];
                }
            ke[e * ND * ND + k] = s;
        }
        __syncthreads();
    }
}
static_assert(KE_THREADS == 8 * 24, "one thread per (point, column) in the B-bar step");

template <typename T>
T* dmalloc(size_t count) {
    void* p = nullptr;
    RFG_CUDA(cudaMalloc(&p, std::max<size_t>(count, 1) * sizeof(T)));
    return (T*)p;
}

int grid_for(int64_t work, int threads) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t g = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(g, (int64_t)sms * 16));
}

}  // namespace

Assembler::Assembler(int64_t n, const int64_t* colptr, const int64_t* rowidx, int64_t nelem, int64_t nd,
                     const int64_t* edof, cudaStream_t st)
    : n_(n), nnz_(colptr[n]), nelem_(nelem), nd_(nd), st_(st) {
    for (int i = 0; i < 3; i++) RFG_CUDA(cudaEventCreate(&ev_[i]));
    int64_t* d_colptr = dmalloc<int64_t>(n + 1);
    int64_t* d_rowidx = dmalloc<int64_t>(nnz_);
    int64_t* d_edof = dmalloc<int64_t>(nelem * nd);
    long long* d_bad = dmalloc<long long>(1);
    int64_t* d_cursor = nullptr;
    int64_t* d_tmp = nullptr;
    auto release = [&] {
        cudaFree(d_colptr);
        cudaFree(d_rowidx);
        cudaFree(d_edof);
        cudaFree(d_bad);
        cudaFree(d_cursor);
        cudaFree(d_tmp);
    };
    try {
        RFG_CUDA(cudaMemcpyAsync(d_colptr, colptr, (n + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
        if (nnz_ > 0)
            RFG_CUDA(cudaMemcpyAsync(d_rowidx, rowidx, nnz_ * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
        if (nelem * nd > 0)
            RFG_CUDA(cudaMemcpyAsync(d_edof, edof, nelem * nd * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
        const long long none = (long long)(((unsigned long long)1 << 63) - 1);
        RFG_CUDA(cudaMemcpyAsync(d_bad, &none, sizeof(long long), cudaMemcpyHostToDevice, st_));
        d_start_ = dmalloc<int64_t>(nnz_ + 1);
        RFG_CUDA(cudaMemsetAsync(d_start_, 0, (nnz_ + 1) * sizeof(int64_t), st_));
        const int64_t total = nelem * nd * nd;
        if (total > 0)
            k_asm_count<<<grid_for(total, 256), 256, 0, st_>>>(d_edof, d_colptr, d_rowidx, nd, total,
                                                              (unsigned long long*)d_start_, d_bad);
        RFG_CUDA(cudaGetLastError());
        long long bad = 0;
        RFG_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof(long long), cudaMemcpyDeviceToHost, st_));
        RFG_CUDA(cudaStreamSynchronize(st_));
        if (bad != none) {
            const int64_t e = bad / (nd * nd), ab = bad % (nd * nd);
            const int64_t ia = edof[e * nd + ab / nd], ib = edof[e * nd + ab % nd];
            throw CudaError("entry (" + std::to_string(ia) + ", " + std::to_string(ib) +
                            ") missing in the pattern (element " + std::to_string(e) + ")");
        }
        d_tmp = dmalloc<int64_t>(scan_tmp_elems(nnz_ + 1));
        exclusive_scan_i64(d_start_, nnz_ + 1, d_tmp, st_);
        RFG_CUDA(cudaMemcpyAsync(&ncontrib_, d_start_ + nnz_, sizeof(int64_t), cudaMemcpyDeviceToHost, st_));
        RFG_CUDA(cudaStreamSynchronize(st_));
        d_key_ = dmalloc<uint64_t>(ncontrib_);
        d_cursor = dmalloc<int64_t>(nnz_);
        if (nnz_ > 0)
            RFG_CUDA(cudaMemcpyAsync(d_cursor, d_start_, nnz_ * sizeof(int64_t), cudaMemcpyDeviceToDevice, st_));
        if (total > 0)
            k_asm_fill<<<grid_for(total, 256), 256, 0, st_>>>(d_edof, d_colptr, d_rowidx, nd, total,
                                                             (unsigned long long*)d_cursor, d_key_);
        RFG_CUDA(cudaGetLastError());
        if (nnz_ > 0) sort_rows_u64(d_key_, d_start_, nnz_, st_);
        RFG_CUDA(cudaStreamSynchronize(st_));
    } catch (...) {
        release();
        cudaFree(d_start_);
        cudaFree(d_key_);
        for (auto& ev : ev_)
            if (ev) cudaEventDestroy(ev);
        throw;
    }
    release();
}

Assembler::~Assembler() {
    cudaStreamSynchronize(st_);
    cudaFree(d_start_);
    cudaFree(d_key_);
    cudaFree(d_ke_);
    cudaFree(d_xyz_);
    cudaFree(d_conn_);
    cudaFree(d_emod_);
    cudaFree(d_bad_);
    for (auto& ev : ev_)
        if (ev) cudaEventDestroy(ev);
}

void Assembler::ensure_ke() {
    if (!d_ke_) d_ke_ = dmalloc<double>(nelem_ * nd_ * nd_);
}

void Assembler::assemble(const double* ke, bool ke_on_device, double* val) {
    const double* src = ke;
    if (!ke_on_device) {
        ensure_ke();
        if (nelem_ * nd_ * nd_ > 0) host_upload(d_ke_, ke, nelem_ * nd_ * nd_ * sizeof(double), st_);
        src = d_ke_;
    }
    RFG_CUDA(cudaEventRecord(ev_[1], st_));
    if (nnz_ > 0) k_asm_gather<<<grid_for(nnz_, 256), 256, 0, st_>>>(d_start_, d_key_, src, nd_, nnz_, val);
    RFG_CUDA(cudaGetLastError());
    RFG_CUDA(cudaEventRecord(ev_[2], st_));
    RFG_CUDA(cudaEventSynchronize(ev_[2]));
    float ms = 0.f;
    RFG_CUDA(cudaEventElapsedTime(&ms, ev_[1], ev_[2]));
    gather_ms_ = ms;
}

int64_t Assembler::hex8(int64_t nn, const double* xyz, const int64_t* conn, const double* emod, double nu,
                        double* val) {
    if (nd_ != 24) throw CudaError("C3D8 assembly needs 24 DOFs per element (prepared with " + std::to_string(nd_) + ")");
    for (int64_t i = 0; i < nelem_ * 8; i++)
        if (conn[i] < 0 || conn[i] >= nn) throw CudaError("element node id out of range");
    ensure_ke();
    if (nn > nn_cap_) {
        cudaFree(d_xyz_);
        d_xyz_ = dmalloc<double>(nn * 3);
        nn_cap_ = nn;
    }
    if (!d_conn_) d_conn_ = dmalloc<int64_t>(nelem_ * 8);
    if (!d_emod_) d_emod_ = dmalloc<double>(nelem_);
    if (!d_bad_) d_bad_ = dmalloc<long long>(1);
    RFG_CUDA(cudaMemcpyAsync(d_xyz_, xyz, nn * 3 * sizeof(double), cudaMemcpyHostToDevice, st_));
    RFG_CUDA(cudaMemcpyAsync(d_conn_, conn, nelem_ * 8 * sizeof(int64_t), cudaMemcpyHostToDevice, st_));
    RFG_CUDA(cudaMemcpyAsync(d_emod_, emod, nelem_ * sizeof(double), cudaMemcpyHostToDevice, st_));
    const long long none = (long long)(((unsigned long long)1 << 63) - 1);
    RFG_CUDA(cudaMemcpyAsync(d_bad_, &none, sizeof(long long), cudaMemcpyHostToDevice, st_));
    RFG_CUDA(cudaEventRecord(ev_[0], st_));
    if (nelem_ > 0)
        k_ke_hex8<<<(unsigned)std::min<int64_t>(nelem_, 148 * 64), KE_THREADS, 0, st_>>>(
            d_xyz_, d_conn_, d_emod_, nu, nelem_, d_ke_, d_bad_);
    RFG_CUDA(cudaGetLastError());
    RFG_CUDA(cudaEventRecord(ev_[1], st_));
    long long bad = 0;
    RFG_CUDA(cudaMemcpyAsync(&bad, d_bad_, sizeof(long long), cudaMemcpyDeviceToHost, st_));
    RFG_CUDA(cudaStreamSynchronize(st_));
    float ms = 0.f;
    RFG_CUDA(cudaEventElapsedTime(&ms, ev_[0], ev_[1]));
    element_ms_ = ms;
    if (bad != none) return (int64_t)bad;
    assemble(d_ke_, true, val);
    return -1;
}

}  // namespace rfg
