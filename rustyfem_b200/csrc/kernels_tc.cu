// Tensor-core Schur update of large fronts (mixed precision path), sm_100a.
//
// One CTA computes one 128×128 tile of the trailing matrix of a front,
//     F[r, c] −= Σ_p W[r, p]·L[c, p],   p over the outer block's pivots (K ≤ 256),
// with FP32 accuracy from the TF32 tensor cores by splitting each operand into a
// TF32 head and a TF32 tail (x = hi + lo, both written by the panel kernel):
//     W·Lᵀ ≈ W_hi·L_hiᵀ + W_hi·L_loᵀ + W_lo·L_hiᵀ   (three kind::tf32 MMAs per K step).
// Operand tiles (128 rows × 32 K, 128-byte swizzle) are loaded by TMA into a
// two-stage shared-memory ring; thread 0 produces, thread 32 issues tcgen05.mma
// with the accumulator in TMEM (128 lanes × 128 columns, A negated so that the
// accumulator is −W·Lᵀ); the four warps read the accumulator back with
// tcgen05.ld, write it in the 128-byte swizzle layout into shared memory, and
// TMA adds it into the front (cp.reduce.async.bulk.tensor .add) — the tile of F
// is never read by the SMs. No multicast: every CTA loads its own tiles.
// Writes of the upper triangle of diagonal tiles land in entries that nothing
// reads (the strict upper triangle of the panel and of the update block).
//
// FP16 variant of the persistent kernel (H16, the default). With U = L·D^(1/2) the
// update is F −= U·Uᵀ, both operands rows of one matrix. The panel kernel writes each
// row of U scaled by a power of two s_r chosen from the row's current diagonal at the
// start of the outer block (|U[r, p]| ≤ F_rr^(1/2) for a positive definite front, so
// |U·s_r| < 2^12) and split into an FP16 head and tail. The tile is
//     −U_hi·U_hiᵀ − U_hi·U_loᵀ − U_lo·U_hiᵀ  (three kind::f16 MMAs per K step of 16),
// about 2⁻²² relative per product as with the TF32 split, at twice the tensor rate and
// half the operand bytes; the epilogue multiplies the accumulator by 1/(s_r·s_c) before
// the reduce-add. A row whose scaled entries would leave the FP16 range is reported
// (code 21) and the engine factors again with the TF32 split.

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "engine.h"
#include "tc.cuh"
#include "tiles.cuh"

namespace rfg {

namespace {

constexpr int TCM = 128;  // tile rows (TMEM lanes)
constexpr int TCN = 128;  // tile columns (TMEM columns)
constexpr int TCK = 32;   // K per stage: one 128-byte swizzle atom of FP32
constexpr int NSTAGE = 2;
constexpr int OP_BYTES = TCM * TCK * 4;       // 16 KB per operand tile
constexpr int STAGE_BYTES = 4 * OP_BYTES;     // W_hi, W_lo, L_hi, L_lo
constexpr int TC_SMEM = NSTAGE * STAGE_BYTES + 1024 + 256;

__device__ __forceinline__ int64_t find_slot_tc(const int64_t* pre, int64_t n, int64_t b) {
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

__global__ void __launch_bounds__(128, 1)
    k_schur_tc(const __grid_constant__ TcMaps maps, const CUtensorMap* __restrict__ cmaps, const DFront* __restrict__ fr,
               const int64_t* __restrict__ order, int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre_tiles,
               const int64_t* __restrict__ pre_scr, int64_t s, const int64_t* __restrict__ status, int* __restrict__ err) {
    extern __shared__ unsigned char smem_raw[];
    uint8_t* base = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint64_t* full = (uint64_t*)(base + NSTAGE * STAGE_BYTES);
    uint64_t* empty = full + NSTAGE;
    uint64_t* done = empty + NSTAGE;
    uint32_t* tmem_slot = (uint32_t*)(done + 1);

    int64_t b = blockIdx.x;
    int64_t i = find_slot_tc(pre_tiles, nact, b);
    int64_t lt = b - pre_tiles[i];
    int64_t t = order[fr_off + i];
    if (status[t] != -1) return;
    const DFront f = fr[t];
    int64_t J0 = (s / KO) * NBO;
    int64_t J1e = min(J0 + NBO, f.k);
    int64_t klen = J1e - J0;
    int64_t R = f.m - J1e;
    int64_t nrt = (R + TCM - 1) / TCM, ncp = (f.k - J1e + TCN - 1) / TCN;
    int64_t cntP = ncp * nrt - ncp * (ncp - 1) / 2;
    int64_t row0, col0;
    bool in_panel;
    if (lt < cntP) {
        int64_t tj = 0, cnt = nrt;
        while (lt >= cnt) {
            lt -= cnt;
            tj++;
            cnt = nrt - tj;
        }
        row0 = J1e + (tj + lt) * TCM;
        col0 = J1e + tj * TCN;
        in_panel = true;
    } else {
        int64_t idx = lt - cntP;
        int64_t ti = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
        while (ti * (ti + 1) / 2 > idx) ti--;
        while ((ti + 1) * (ti + 2) / 2 <= idx) ti++;
        int64_t tj = idx - ti * (ti + 1) / 2;
        row0 = f.k + ti * TCM;
        col0 = f.k + tj * TCN;
        in_panel = false;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) {
        tc::tmem_alloc(tmem_slot, TCN);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 32) {
        for (int q = 0; q < NSTAGE; q++) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        tc::mbar_init(done, 1);
        tc::fence_barrier_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    const int nk = (int)((klen + TCK - 1) / TCK);
    const int srowA = (int)(pre_scr[i] + (row0 - J0));
    const int srowB = (int)(pre_scr[i] + (col0 - J0));
    if (threadIdx.x == 0) {
        // producer: TMA loads of the four operand tiles per K chunk
        for (int kc = 0; kc < nk; kc++) {
            int st = kc % NSTAGE;
            if (kc >= NSTAGE && !tc::mbar_wait(&empty[st], ((kc / NSTAGE) - 1) & 1, err, 1)) break;
            uint8_t* sb = base + st * STAGE_BYTES;
            tc::mbar_expect_tx(&full[st], STAGE_BYTES);
            int x = kc * TCK;
            const int par = (int)((s / KO) & 1);
            tc::tma_load_2d(sb, &maps.whi[par], x, srowA, &full[st]);
            tc::tma_load_2d(sb + OP_BYTES, &maps.wlo[par], x, srowA, &full[st]);
            tc::tma_load_2d(sb + 2 * OP_BYTES, &maps.lhi[par], x, srowB, &full[st]);
            tc::tma_load_2d(sb + 3 * OP_BYTES, &maps.llo[par], x, srowB, &full[st]);
        }
    } else if (threadIdx.x == 32) {
        // MMA issuer
        constexpr uint32_t idesc = tc::idesc_tf32(TCM, TCN, true);
        for (int kc = 0; kc < nk; kc++) {
            int st = kc % NSTAGE;
            if (!tc::mbar_wait(&full[st], (kc / NSTAGE) & 1, err, 2)) break;
            tc::tc_fence_after();
            uint32_t sb = tc::smem_u32(base + st * STAGE_BYTES);
#pragma unroll
            for (int ks = 0; ks < TCK / 8; ks++) {
                uint32_t off = ks * 32;
                uint64_t ahi = tc::sw128_desc(sb + off), alo = tc::sw128_desc(sb + OP_BYTES + off);
                uint64_t bhi = tc::sw128_desc(sb + 2 * OP_BYTES + off), blo = tc::sw128_desc(sb + 3 * OP_BYTES + off);
                tc::mma_tf32(tmem, ahi, bhi, idesc, (kc | ks) != 0);
                tc::mma_tf32(tmem, ahi, blo, idesc, 1);
                tc::mma_tf32(tmem, alo, bhi, idesc, 1);
            }
            tc::mma_commit(&empty[st]);
        }
        tc::mma_commit(done);
    }
    __syncwarp();
    bool ok = tc::mbar_wait(done, 0, err, 3);
    tc::tc_fence_after();
    // epilogue: TMEM -> registers -> shared (128-byte swizzle boxes of 128 rows × 32 columns)
    const int rl = warp * 32 + lane;
#pragma unroll 1
    for (int cb = 0; cb < TCN / 32; cb++) {
        uint32_t v[32];
        tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + cb * 32, v);
        tc::tmem_wait_ld();
        uint8_t* rowp = base + cb * (TCM * 128) + rl * 128;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint4 q = make_uint4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
            *reinterpret_cast<uint4*>(rowp + ((j ^ (rl & 7)) * 16)) = q;
        }
    }
    tc::fence_proxy_async_smem();
    tc::tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && ok) {
        const CUtensorMap* cm = &cmaps[2 * t + (in_panel ? 0 : 1)];
        int64_t cbase = in_panel ? 0 : f.k;
        int64_t width = in_panel ? f.k : f.u;
        for (int cb = 0; cb < TCN / 32; cb++) {
            int64_t x = (col0 - cbase) + cb * 32;
            if (x >= width) break;
            tc::tma_reduce_add_2d(cm, (int)x, (int)(row0 - cbase), base + cb * (TCM * 128));
        }
        tc::bulk_commit();
        tc::bulk_wait0();
    }
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, TCN);
}

// ---------------------------------------------------------------------------
// Persistent variant: one CTA per SM walks the step's tiles (tile = blockIdx.x +
// i·gridDim.x). Warp 0 produces (TMA into a 3-stage ring), warp 1 issues the MMAs
// into one of two TMEM accumulators, warps 2-5 drain the other accumulator (TMEM →
// registers → 128-byte-swizzle box → TMA reduce-add into the front) while the next
// tile is multiplied. mbarriers: full/empty per stage, tmem_full/tmem_empty per
// accumulator; every wait is bounded.
// ---------------------------------------------------------------------------
// Tile 128 × TN: TN = 128 for the inner updates (at most NBO − NB columns), TN = 256 for the
// outer updates, where a row block of W is multiplied against 256 columns of L per load
// (a quarter less operand traffic per flop than two 128-wide tiles, half the MMAs).
// The stage layout in bytes is the same for both kinds: a 128-byte operand row holds 32
// TF32 or 64 FP16 values of K.
template <int TN>
struct PsLayout {
    static constexpr int OPA = TCM * TCK * 4;          // one W (U) operand tile (hi or lo)
    static constexpr int OPB = TN * TCK * 4;           // one L (U) operand tile
    static constexpr int STAGE = 2 * OPA + 2 * OPB;    // A_hi, A_lo, B_hi, B_lo
    static constexpr int STAGES = TN == 128 ? 3 : 2;
    static constexpr int BOX = TCM * 32 * 4;           // 16 KB epilogue box (128 rows × 32 columns)
    static constexpr int CSCALE = TN * 4;              // FP16 kind: the tile's column scales
    static constexpr int SMEM = STAGES * STAGE + 2 * BOX + CSCALE + 1024 + 256;
};
static_assert(PsLayout<256>::SMEM <= 232448, "shared memory of the 128x256 tile kernel");
constexpr int PS_STAGES = PsLayout<128>::STAGES;
constexpr int PS_BOX = PsLayout<128>::BOX;
constexpr int PS_SMEM = PsLayout<128>::SMEM;
constexpr int PS_THREADS = 192;

struct TileInfo {
    int64_t t, row0, col0, klen, J0;
    int64_t k0;    // first scratch column of the K range (relative to J0)
    int64_t xmax;  // columns at or beyond this (map coordinates) are not written
    int64_t i;     // slot of the front in the step
    int64_t klen0; // two-block pass: the first klen0 values of K are the previous block's pivots
                   // (its scratch buffer and layout), the rest this block's
    bool in_panel;
};

__device__ __forceinline__ TileInfo decode_tile(const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre_tiles,
                                                int64_t s, int64_t b, DFront* fout, uint8_t mode) {
    TileInfo ti;
    int64_t i = find_slot_tc(pre_tiles, nact, b);
    int64_t lt = b - pre_tiles[i];
    ti.i = i;
    ti.t = order[fr_off + i];
    const DFront f = fr[ti.t];
    *fout = f;
    int64_t J0 = (s / KO) * NBO;
    int64_t J1e = min(J0 + NBO, f.k);
    ti.J0 = J0;
    ti.klen0 = mode == OUT_PAIR ? NBO : 0;
    ti.klen = J1e - J0 + ti.klen0;
    ti.k0 = 0;
    int64_t R = f.m - J1e;
    // a strip pass covers the next block's columns only (no update-block part)
    const int64_t W = mode == OUT_STRIP ? min((int64_t)NBO, f.k - J1e) : f.k - J1e;
    int64_t nrt = (R + TCM - 1) / TCM, ncp = (W + TCN - 1) / TCN;
    int64_t cntP = ncp * nrt - ncp * (ncp - 1) / 2;
    if (lt < cntP) {
        int64_t tj = 0, cnt = nrt;
        while (lt >= cnt) {
            lt -= cnt;
            tj++;
            cnt = nrt - tj;
        }
        ti.row0 = J1e + (tj + lt) * TCM;
        ti.col0 = J1e + tj * TCN;
        ti.in_panel = true;
        ti.xmax = J1e + W;
    } else {
        int64_t idx = lt - cntP;
        int64_t r = (int64_t)((sqrt(8.0 * (double)idx + 1.0) - 1.0) * 0.5);
        while (r * (r + 1) / 2 > idx) r--;
        while ((r + 1) * (r + 2) / 2 <= idx) r++;
        int64_t tj = idx - r * (r + 1) / 2;
        ti.row0 = f.k + r * TCM;
        ti.col0 = f.k + tj * TCN;
        ti.in_panel = false;
        ti.xmax = f.u;
    }
    return ti;
}

// Inner update of step s: rows [j1, m) × columns [j1, J1e) of the front's panel with
// K = the step's NB pivots (scratch columns j0 − J0 ..); 128×128 tiles (tj ≤ tr),
// column tile by column tile; columns at or beyond J1e are not written.
__device__ __forceinline__ TileInfo decode_tile_inner(const DFront* __restrict__ fr,
                                                      const int64_t* __restrict__ order, int64_t fr_off,
                                                      int64_t nact, const int64_t* __restrict__ pre_tiles,
                                                      int64_t s, int64_t b, DFront* fout) {
    TileInfo ti;
    int64_t i = find_slot_tc(pre_tiles, nact, b);
    int64_t lt = b - pre_tiles[i];
    ti.i = i;
    ti.t = order[fr_off + i];
    const DFront f = fr[ti.t];
    *fout = f;
    const int64_t j0 = s * NB, j1 = min(j0 + NB, f.k);
    const int64_t J0 = (s / KO) * NBO, J1e = min(J0 + NBO, f.k);
    ti.J0 = J0;
    ti.k0 = j0 - J0;
    ti.klen = j1 - j0;
    ti.klen0 = 0;
    const int64_t nrt = (f.m - j1 + TCM - 1) / TCM;
    int64_t tj = 0, cnt = nrt;
    while (lt >= cnt) {
        lt -= cnt;
        tj++;
        cnt = nrt - tj;
    }
    ti.row0 = j1 + (tj + lt) * TCM;
    ti.col0 = j1 + tj * TCN;
    ti.in_panel = true;
    ti.xmax = J1e;
    return ti;
}

// Outer update in 128×256 tiles: the panel columns [J1e, k) in column tiles of 256, each
// with its row tiles from its diagonal to m, then the update block [k, m)² the same way.
// Columns beyond the region (the last column tile of the panel, or beyond u) and the
// strict upper part of the tiles on the diagonal are computed and not written (beyond the
// map) or written into entries that nothing reads.
__device__ __forceinline__ TileInfo decode_tile_wide(const DFront* __restrict__ fr, const int64_t* __restrict__ order,
                                                     int64_t fr_off, int64_t nact, const int64_t* __restrict__ pre_tiles,
                                                     int64_t s, int64_t b, DFront* fout, uint8_t mode) {
    TileInfo ti;
    int64_t i = find_slot_tc(pre_tiles, nact, b);
    int64_t lt = b - pre_tiles[i];
    ti.i = i;
    ti.t = order[fr_off + i];
    const DFront f = fr[ti.t];
    *fout = f;
    const int64_t J0 = (s / KO) * NBO, J1e = min(J0 + NBO, f.k);
    ti.J0 = J0;
    ti.klen0 = mode == OUT_PAIR ? NBO : 0;
    ti.klen = J1e - J0 + ti.klen0;
    ti.k0 = 0;
    // a strip pass covers the next block's columns only (one column tile, no update block)
    const int64_t R = f.m - J1e, W = mode == OUT_STRIP ? min((int64_t)NBO, f.k - J1e) : f.k - J1e;
    const int64_t nr = (R + TCM - 1) / TCM, nc = (W + 255) / 256;
    const int64_t cntP = nc * nr - nc * (nc - 1);
    int64_t base, nrr;
    if (lt < cntP) {
        base = J1e;
        nrr = nr;
        ti.in_panel = true;
        ti.xmax = J1e + W;
    } else {
        lt -= cntP;
        base = f.k;
        nrr = (f.u + TCM - 1) / TCM;
        ti.in_panel = false;
        ti.xmax = f.u;
    }
    int64_t tj = 0, cnt = nrr;
    while (lt >= cnt) {
        lt -= cnt;
        tj++;
        cnt = nrr - 2 * tj;
    }
    ti.col0 = base + tj * 256;
    ti.row0 = ti.col0 + lt * TCM;
    return ti;
}

template <int TN>
__device__ __forceinline__ TileInfo decode_any(bool inner, const DFront* __restrict__ fr,
                                               const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                                               const int64_t* __restrict__ pre_tiles, int64_t s, int64_t b,
                                               DFront* fout, const uint8_t* __restrict__ omode) {
    if (inner) return decode_tile_inner(fr, order, fr_off, nact, pre_tiles, s, b, fout);
    // the front's kind of outer update at this step (full, strip or the pair's second pass)
    const int64_t i = find_slot_tc(pre_tiles, nact, b);
    const uint8_t mode = omode ? omode[i] : OUT_FULL;
    return TN == 256 ? decode_tile_wide(fr, order, fr_off, nact, pre_tiles, s, b, fout, mode)
                     : decode_tile(fr, order, fr_off, nact, pre_tiles, s, b, fout, mode);
}

template <int TN, bool H16>
__global__ void __launch_bounds__(PS_THREADS, 1)
    k_schur_tc_persistent(const __grid_constant__ TcMaps maps, const CUtensorMap* __restrict__ cmaps,
                          const DFront* __restrict__ fr, const int64_t* __restrict__ order, int64_t fr_off, int64_t nact,
                          const int64_t* __restrict__ pre_tiles, int64_t ntiles, const int64_t* __restrict__ pre_scr,
                          int64_t s, const int64_t* __restrict__ status, int* __restrict__ err, int inner,
                          const float* __restrict__ uscale, int64_t scale_rows, const uint8_t* __restrict__ omode,
                          const int64_t* __restrict__ pre_scr_prev) {
    using L = PsLayout<TN>;
    constexpr int KC = H16 ? 64 : TCK;  // K per stage
    extern __shared__ unsigned char smem_raw[];
    uint8_t* base = (uint8_t*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    uint8_t* boxes = base + L::STAGES * L::STAGE;
    float* cinv = (float*)(boxes + 2 * L::BOX);  // H16: 1/s_c of the tile's columns
    uint64_t* full = (uint64_t*)(boxes + 2 * L::BOX + L::CSCALE);
    uint64_t* empty = full + L::STAGES;
    uint64_t* tfull = empty + L::STAGES;
    uint64_t* tempty = tfull + 2;
    uint32_t* tmem_slot = (uint32_t*)(tempty + 2);
    volatile uint32_t* eflag = tmem_slot + 1;  // epilogue: the accumulator wait succeeded
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 1) {
        tc::tmem_alloc(tmem_slot, 2 * TN);
        tc::tmem_relinquish();
    }
    if (threadIdx.x == 0) {
        for (int q = 0; q < L::STAGES; q++) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        for (int a = 0; a < 2; a++) {
            tc::mbar_init(&tfull[a], 1);
            tc::mbar_init(&tempty[a], 4);
        }
        tc::fence_barrier_init();
    }
    tc::tc_fence_before();
    __syncthreads();
    tc::tc_fence_after();
    // the set-up above overlaps the previous kernel (programmatic launch); the operands and
    // the front are touched only after it has completed
    pdl_wait();
    pdl_launch_dependents();
    const uint32_t tmem = *tmem_slot;
    bool ok = true;
    if (warp == 0) {
        if (lane == 0) {
            int64_t g = 0;  // chunk counter over all tiles of this CTA
            for (int64_t b = blockIdx.x; b < ntiles && ok; b += gridDim.x) {
                DFront f;
                TileInfo ti = decode_any<TN>(inner != 0, fr, order, fr_off, nact, pre_tiles, s, b, &f, omode);
                if (status[ti.t] != -1) continue;
                const int par = (int)((s / KO) & 1);
                // this block's rows in its scratch layout, and for the second pass of a pair the
                // previous block's (the other buffer)
                const int srowA = (int)(pre_scr[ti.i] + (ti.row0 - ti.J0));
                const int srowB = (int)(pre_scr[ti.i] + (ti.col0 - ti.J0));
                const int srowA0 = ti.klen0 ? (int)(pre_scr_prev[ti.i] + (ti.row0 - (ti.J0 - NBO))) : 0;
                const int srowB0 = ti.klen0 ? (int)(pre_scr_prev[ti.i] + (ti.col0 - (ti.J0 - NBO))) : 0;
                const int nk = (int)((ti.klen + KC - 1) / KC);
                for (int kc = 0; kc < nk; kc++, g++) {
                    int st = (int)(g % L::STAGES);
                    if (g >= L::STAGES && !tc::mbar_wait(&empty[st], (uint32_t)(((g / L::STAGES) - 1) & 1), err, 11)) {
                        ok = false;
                        break;
                    }
                    uint8_t* sb = base + st * L::STAGE;
                    tc::mbar_expect_tx(&full[st], L::STAGE);
                    const bool prev = kc * KC < ti.klen0;
                    const int p = prev ? par ^ 1 : par;
                    const int x = prev ? kc * KC : (int)ti.k0 + (kc * KC - (int)ti.klen0);
                    const int ya = prev ? srowA0 : srowA, yb = prev ? srowB0 : srowB;
                    if constexpr (H16) {
                        tc::tma_load_2d(sb, &maps.uhi[p], x, ya, &full[st]);
                        tc::tma_load_2d(sb + L::OPA, &maps.ulo[p], x, ya, &full[st]);
                        tc::tma_load_2d(sb + 2 * L::OPA, TN == 256 ? &maps.uhi2[p] : &maps.uhi[p], x, yb, &full[st]);
                        tc::tma_load_2d(sb + 2 * L::OPA + L::OPB, TN == 256 ? &maps.ulo2[p] : &maps.ulo[p], x, yb,
                                        &full[st]);
                    } else {
                        tc::tma_load_2d(sb, &maps.whi[p], x, ya, &full[st]);
                        tc::tma_load_2d(sb + L::OPA, &maps.wlo[p], x, ya, &full[st]);
                        tc::tma_load_2d(sb + 2 * L::OPA, TN == 256 ? &maps.lhi2[p] : &maps.lhi[p], x, yb, &full[st]);
                        tc::tma_load_2d(sb + 2 * L::OPA + L::OPB, TN == 256 ? &maps.llo2[p] : &maps.llo[p], x, yb,
                                        &full[st]);
                    }
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            constexpr uint32_t idesc = H16 ? tc::idesc_f16(TCM, TN, true) : tc::idesc_tf32(TCM, TN, true);
            int64_t g = 0, tl = 0;
            for (int64_t b = blockIdx.x; b < ntiles && ok; b += gridDim.x) {
                DFront f;
                TileInfo ti = decode_any<TN>(inner != 0, fr, order, fr_off, nact, pre_tiles, s, b, &f, omode);
                if (status[ti.t] != -1) continue;
                const int a = (int)(tl & 1);
                if (tl >= 2 && !tc::mbar_wait(&tempty[a], (uint32_t)(((tl >> 1) - 1) & 1), err, 12)) {
                    ok = false;
                    break;
                }
                tc::tc_fence_after();
                const uint32_t acc = tmem + a * TN;
                const int nk = (int)((ti.klen + KC - 1) / KC);
                for (int kc = 0; kc < nk; kc++, g++) {
                    int st = (int)(g % L::STAGES);
                    if (!tc::mbar_wait(&full[st], (uint32_t)((g / L::STAGES) & 1), err, 13)) {
                        ok = false;
                        break;
                    }
                    tc::tc_fence_after();
                    uint32_t sb = tc::smem_u32(base + st * L::STAGE);
                    // four MMA K steps per 128-byte row: 8 TF32 or 16 FP16 values, 32 bytes each
#pragma unroll
                    for (int ks = 0; ks < 4; ks++) {
                        uint32_t off = ks * 32;
                        uint64_t ahi = tc::sw128_desc(sb + off), alo = tc::sw128_desc(sb + L::OPA + off);
                        uint64_t bhi = tc::sw128_desc(sb + 2 * L::OPA + off),
                                 blo = tc::sw128_desc(sb + 2 * L::OPA + L::OPB + off);
                        if constexpr (H16) {
                            tc::mma_f16(acc, ahi, bhi, idesc, (kc | ks) != 0);
                            tc::mma_f16(acc, ahi, blo, idesc, 1);
                            tc::mma_f16(acc, alo, bhi, idesc, 1);
                        } else {
                            tc::mma_tf32(acc, ahi, bhi, idesc, (kc | ks) != 0);
                            tc::mma_tf32(acc, ahi, blo, idesc, 1);
                            tc::mma_tf32(acc, alo, bhi, idesc, 1);
                        }
                    }
                    tc::mma_commit(&empty[st]);
                }
                tc::mma_commit(&tfull[a]);
                tl++;
            }
        }
    } else {
        // epilogue warps 2..5: TMEM lane quarter (warp % 4)
        const int q = warp & 3;
        const int et = threadIdx.x - 64;  // 0..127
        const int rl = q * 32 + lane;     // tile row of this thread
        int64_t tl = 0, nbox = 0;
        for (int64_t b = blockIdx.x; b < ntiles; b += gridDim.x) {
            DFront f;
            TileInfo ti = decode_any<TN>(inner != 0, fr, order, fr_off, nact, pre_tiles, s, b, &f, omode);
            if (status[ti.t] != -1) continue;
            const int a = (int)(tl & 1);
            // one thread waits (bounded) and tells the other 127 through shared memory, so
            // that all epilogue threads take the same branch at every named barrier
            if (et == 0) *eflag = tc::mbar_wait(&tfull[a], (uint32_t)((tl >> 1) & 1), err, 14) ? 1u : 0u;
            tc::named_barrier(1, 128);
            if (*eflag == 0) break;
            tc::tc_fence_after();
            float rinv = 1.f;
            if constexpr (H16) {
                // the scales of the tile's rows and columns (rows past the scratch belong to
                // tiles' padding, whose results are not written)
                const int64_t srA = pre_scr[ti.i] + (ti.row0 - ti.J0), srB = pre_scr[ti.i] + (ti.col0 - ti.J0);
                // a row's scale depends on the row alone (its original diagonal), so the two
                // blocks of a pair share it: this block's scratch layout gives it
                const int64_t ra = srA + rl;
                rinv = ra < scale_rows ? 1.f / uscale[ra] : 0.f;
                for (int c = et; c < TN; c += 128) cinv[c] = srB + c < scale_rows ? 1.f / uscale[srB + c] : 0.f;
                tc::named_barrier(1, 128);
            }
            const CUtensorMap* cm = &cmaps[2 * ti.t + (ti.in_panel ? 0 : 1)];
            const int64_t cbase = ti.in_panel ? 0 : f.k;
            const int64_t width = ti.xmax;
            for (int cb = 0; cb < TN / 32; cb++, nbox++) {
                uint32_t v[32];
                tc::tmem_ld32(tmem + a * TN + ((uint32_t)(q * 32) << 16) + cb * 32, v);
                tc::tmem_wait_ld();
                if (cb == TN / 32 - 1) {
                    // the accumulator is drained: the MMA warp may reuse it
                    tc::tc_fence_before();
                    __syncwarp();
                    if (lane == 0) tc::mbar_arrive(&tempty[a]);
                }
                uint8_t* box = boxes + (nbox & 1) * L::BOX;
                if (et == 0) tc::bulk_wait_read1();  // the reduce issued from this box two boxes ago
                tc::named_barrier(1, 128);
                uint8_t* rowp = box + rl * 128;
                if constexpr (H16) {
#pragma unroll
                    for (int j = 0; j < 32; j++)
                        v[j] = __float_as_uint(__uint_as_float(v[j]) * rinv * cinv[cb * 32 + j]);
                }
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    uint4 qv = make_uint4(v[4 * j], v[4 * j + 1], v[4 * j + 2], v[4 * j + 3]);
                    *reinterpret_cast<uint4*>(rowp + ((j ^ (rl & 7)) * 16)) = qv;
                }
                tc::fence_proxy_async_smem();
                tc::named_barrier(1, 128);
                if (et == 0) {
                    int64_t x = (ti.col0 - cbase) + cb * 32;
                    if (x < width) tc::tma_reduce_add_2d(cm, (int)x, (int)(ti.row0 - cbase), box);
                    tc::bulk_commit();
                }
            }
            tl++;
        }
        if (et == 0) tc::bulk_wait0();
    }
    tc::tc_fence_before();
    __syncthreads();
    if (warp == 1) tc::tmem_dealloc(tmem, 2 * TN);
}

typedef CUresult (*EncodeFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                             const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                             CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        RFG_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
        if (!p || q != cudaDriverEntryPointSuccess) throw CudaError("cuTensorMapEncodeTiled is not available");
        fn = (EncodeFn)p;
    }
    return fn;
}

// 2D tensor map: width × height elements, row stride ld elements, 128-byte swizzle, box
// of one 128-byte row (32 FP32 or 64 FP16 values) × box_rows
CUtensorMap make_map(const void* ptr, int64_t width, int64_t height, int64_t ld, int box_rows = 128,
                     bool fp16 = false) {
    CUtensorMap m;
    const int es_bytes = fp16 ? 2 : 4;
    cuuint64_t dims[2] = {(cuuint64_t)width, (cuuint64_t)height};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * es_bytes)};
    cuuint32_t box[2] = {(cuuint32_t)(128 / es_bytes), (cuuint32_t)box_rows};
    cuuint32_t es[2] = {1, 1};
    CUresult r = encode_fn()(&m, fp16 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT16 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2,
                             (void*)ptr, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
    return m;
}

}  // namespace

int tc_smem_bytes() { return TC_SMEM; }

void Engine::setup_tc() {
    // operand maps over the split scratch arrays, and one panel / update map per front
    // (two buffers of rows × NBO each, by the parity of the outer block)
    int64_t rows = std::max<int64_t>(plan_.max_scr_rows, 1);
    for (int p = 0; p < 2; p++) {
        const int64_t o = p * rows * NBO;
        tc_maps_.whi[p] = make_map((const float*)scr_whi_ + o, NBO, rows, NBO);
        tc_maps_.wlo[p] = make_map((const float*)scr_wlo_ + o, NBO, rows, NBO);
        tc_maps_.lhi[p] = make_map((const float*)scr_lhi_ + o, NBO, rows, NBO);
        tc_maps_.llo[p] = make_map((const float*)scr_llo_ + o, NBO, rows, NBO);
        tc_maps_.lhi2[p] = make_map((const float*)scr_lhi_ + o, NBO, rows, NBO, TC_WIDE);
        tc_maps_.llo2[p] = make_map((const float*)scr_llo_ + o, NBO, rows, NBO, TC_WIDE);
        tc_maps_.uhi[p] = make_map((const uint16_t*)scr_uhi_ + o, NBO, rows, NBO, 128, true);
        tc_maps_.ulo[p] = make_map((const uint16_t*)scr_ulo_ + o, NBO, rows, NBO, 128, true);
        tc_maps_.uhi2[p] = make_map((const uint16_t*)scr_uhi_ + o, NBO, rows, NBO, TC_WIDE, true);
        tc_maps_.ulo2[p] = make_map((const uint16_t*)scr_ulo_ + o, NBO, rows, NBO, TC_WIDE, true);
    }
    std::vector<CUtensorMap> cm(2 * std::max<int64_t>(plan_.nfronts, 1));
    memset(cm.data(), 0, cm.size() * sizeof(CUtensorMap));
    for (int64_t t = 0; t < plan_.nfronts; t++) {
        const DFront& d = plan_.fronts[t];
        const bool outer = plan_.front_tc[t] != 0, inner = plan_.front_tc_inner[t] != 0;
        if (!outer && !inner) continue;
        // outer updates have panel tiles only when k > NBO (J1e = k otherwise) and update
        // tiles only when u >= 128; inner updates always write the panel
        if ((outer && d.k > NBO) || inner) cm[2 * t] = make_map((const float*)panel_ + d.poff, d.k, d.m, d.ldp);
        if (outer && d.u >= TC_TILE) cm[2 * t + 1] = make_map((const float*)upd_ + d.uoff, d.u, d.u, d.ldu);
    }
    d_cmaps_ = (CUtensorMap*)dalloc(cm.size() * sizeof(CUtensorMap));
    RFG_CUDA(cudaMemcpyAsync(d_cmaps_, cm.data(), cm.size() * sizeof(CUtensorMap), cudaMemcpyHostToDevice, stream_));
    tc_err_ = (int*)dalloc(sizeof(int));
    RFG_CUDA(cudaMemsetAsync(tc_err_, 0, sizeof(int), stream_));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_tc_persistent<128, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  PsLayout<128>::SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_tc_persistent<256, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  PsLayout<256>::SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_tc_persistent<128, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  PsLayout<128>::SMEM));
    RFG_CUDA(cudaFuncSetAttribute(k_schur_tc_persistent<256, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  PsLayout<256>::SMEM));
    int dev = 0;
    RFG_CUDA(cudaGetDevice(&dev));
    RFG_CUDA(cudaDeviceGetAttribute(&num_sms_, cudaDevAttrMultiProcessorCount, dev));
    const char* e = getenv("RFG_TC_PERSISTENT");
    tc_persistent_ = !(e && e[0] == '0');
    // the FP16 split (default) or the TF32 split (RFG_TC_KIND=tf32, and after an FP16
    // range overflow); the one-tile-per-CTA kernel is TF32 only
    const char* k = getenv("RFG_TC_KIND");
    h16_ = tc_persistent_ && diag_src_ != nullptr && !(k && std::string(k) == "tf32");
}

void Engine::launch_schur_tc(const DStep& st) {
    if (tc_persistent_ && plan_.outer_tn == 128) {
        // 128×128 tiles (the autotuner's other tile shape)
        int64_t grid = std::min<int64_t>(st.n_outer_tc, num_sms_);
        launch_pdl(true, h16_ ? k_schur_tc_persistent<128, true> : k_schur_tc_persistent<128, false>,
                   dim3((unsigned)grid), dim3(PS_THREADS), PsLayout<128>::SMEM, stream_, tc_maps_,
                   (const CUtensorMap*)d_cmaps_, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                   st.nact, (const int64_t*)(dp_.pre_outer_tc + st.pre_off), st.n_outer_tc,
                   (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const int64_t*)status_, tc_err_, 0,
                   (const float*)scr_uscale_, plan_.max_scr_rows, (const uint8_t*)(dp_.outer_mode + st.pre_off),
                   (const int64_t*)(dp_.pre_scr + st.scr_off_prev));
        return;
    }
    if (tc_persistent_) {
        int64_t grid = std::min<int64_t>(st.n_outer_tc2, num_sms_);
        launch_pdl(true, h16_ ? k_schur_tc_persistent<256, true> : k_schur_tc_persistent<256, false>,
                   dim3((unsigned)grid), dim3(PS_THREADS), PsLayout<256>::SMEM, stream_, tc_maps_,
                   (const CUtensorMap*)d_cmaps_, (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off,
                   st.nact, (const int64_t*)(dp_.pre_outer_tc2 + st.pre_off), st.n_outer_tc2,
                   (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const int64_t*)status_, tc_err_, 0,
                   (const float*)scr_uscale_, plan_.max_scr_rows, (const uint8_t*)(dp_.outer_mode + st.pre_off),
                   (const int64_t*)(dp_.pre_scr + st.scr_off_prev));
        return;
    }
    k_schur_tc<<<(unsigned)st.n_outer_tc, 128, TC_SMEM, stream_>>>(tc_maps_, d_cmaps_, dp_.fronts, dp_.level_order,
                                                                    st.fr_off, st.nact, dp_.pre_outer_tc + st.pre_off,
                                                                    dp_.pre_scr + st.scr_off, st.s, status_, tc_err_);
}

void Engine::launch_schur_tc_inner(const DStep& st) {
    int64_t grid = std::min<int64_t>(st.n_inner_tc, num_sms_);
    launch_pdl(true, h16_ ? k_schur_tc_persistent<128, true> : k_schur_tc_persistent<128, false>, dim3((unsigned)grid),
               dim3(PS_THREADS), PsLayout<128>::SMEM, stream_, tc_maps_, (const CUtensorMap*)d_cmaps_,
               (const DFront*)dp_.fronts, (const int64_t*)dp_.level_order, st.fr_off, st.nact,
               (const int64_t*)(dp_.pre_inner_tc + st.pre_off), st.n_inner_tc,
               (const int64_t*)(dp_.pre_scr + st.scr_off), st.s, (const int64_t*)status_, tc_err_, 1,
               (const float*)scr_uscale_, plan_.max_scr_rows, (const uint8_t*)nullptr, (const int64_t*)nullptr);
}

}  // namespace rfg
