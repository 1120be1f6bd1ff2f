// skm_table_tc.cuh -- the two GEMM-shaped kernels of the phase-table path on the 5th-generation
// tensor cores: tcgen05.mma kind::tf32 with FP32 accumulators in TMEM, FP32-accurate through a
// hi/lo split of both operands (x = hi + lo, hi = x truncated to tf32).
//
// Rows of both GEMMs are (component, cell) pairs, component-major: row = comp * ct + c with
// ct = 128 / D cells per tile (42 in 3-D, 64 in 2-D), so one M = 128 MMA serves all components.
//
//   transform  D[row][n] = sum_t A[row][t] B[n][t]  over taps t (K), phases n (N)
//              A = im2col of w*alpha over a brick of cells, staged per tile as hi/lo planes,
//              B = [T_hi ; T_lo]: n < np is the tf32 part of T[phase n][t], n >= np the rest;
//              per K step  A_hi x [B_hi ; B_lo]  (N = 2 np)  and  A_lo x B_hi  (N = np), so
//              u[row][p] = D[row][p] + D[row][np + p] = A_hi B_hi + A_lo B_hi + A_hi B_lo.
//   contrib    D[row][tap] = sum_p G[row][p] T[p][tap],  G = (a f + b m + c) grad M per texel;
//              per K step  G_hi T_hi + G_hi T_lo + G_lo T_hi  (N = taps padded to 16).
//
// One CTA per SM, persistent over tiles, warp-specialized: 8 producer warps build the A operand
// of each K chunk in a ring of shared-memory stages (full/empty mbarriers), one thread issues the
// MMAs of a chunk as soon as its stage is full and commits them to the stage's empty barrier, and
// 4 epilogue warps drain the finished accumulator of a tile from TMEM (two accumulators, so the
// MMAs of the next tile run meanwhile).  The transform's control points of the next brick arrive
// by one tiled TMA load while the producers build the current one.  Operands use the K-major
// 128-byte-swizzled canonical layout (32 K elements per 128-byte row, 8-row atoms of 1024 bytes,
// K blocks of 32 one after the other), which the tensor cores read at full rate.
// Every mbarrier wait is bounded; a wait that gives up sets *err and a CTA-wide abort flag that
// ends the other roles' waits, the MMA thread waits (bounded) for its MMAs in flight, and the
// CTA frees its TMEM and returns.
#pragma once

#include <algorithm>
#include <cstring>
#include <vector>

#include "skm_table.cuh"
#include "skm_tc.cuh"
#include "skm_warp_tma.cuh"

namespace skm {

constexpr int kTcEpiWarps = 4;                                   // warps 0-3: TMEM -> global
constexpr int kTcMmaWarp = 4;                                    // warp 4: TMEM owner, lane 0 issues
constexpr int kTcProdWarps = 8;                                  // contrib producers
constexpr int kTcProdThreads = kTcProdWarps * 32;
constexpr int kTcProdBase = (kTcEpiWarps + 1) * 32;              // first producer thread
constexpr int kTrProdWarps = 8;                                  // transform producers: warps 5.., a
constexpr int kTrProdThreads = kTrProdWarps * 32;                // K slice of one TMEM lane quarter each
constexpr int kTrSlices = kTrProdWarps / 4;                      // K slices of a 32-column block
constexpr int kTrCols = 32 / kTrSlices;                          // columns per producer warp and K block
constexpr int kTrTmaWarp = kTcProdBase / 32 + kTrProdWarps;   // transform: issues the region loads
constexpr int kTcThreads = kTcProdBase + kTrProdThreads + 32;
constexpr int kTcStages = 4;                                     // mbarrier slots (stages <= 4)
constexpr int kTcKBlock = 32;                                    // K elements per 128-byte swizzle row
constexpr int kTcRows = 128;
constexpr int kTcProdBar = 1;                                    // named barrier of all producers
constexpr int kTrEpiBar = 2;                                     // transform: named barrier of the epilogue
constexpr int kTcGroupBar = 2;                                   // + group: named barriers of the groups
constexpr int kTcGroupThreads = kTcProdThreads / 2;              // contrib: two producer groups
// contrib: 8 epilogue warps (two per TMEM lane quarter, alternate 16-column chunks), then the
// MMA warp, then the producers
constexpr int kConEpiWarps = 8;
constexpr int kConMmaWarp = kConEpiWarps;
constexpr int kConProdBase = (kConEpiWarps + 1) * 32;
constexpr int kConLoadWarp = kConProdBase / 32 + kTcProdWarps;  // contrib: issues the record loads
constexpr int kConThreads = kConProdBase + kTcProdThreads + 32;     // 576
static_assert((kTrProdWarps == 8 || kTrProdWarps == 16) && (kTcEpiWarps + 1) % 4 == 1,
              "transform producers: (lane quarter, K slice) pairs");
constexpr int kTcRegionBufs = 3;                                 // transform region buffers (at most)
constexpr int kTcNumBars = 2 * kTcStages + 6 + 2 * kTcRegionBufs;
constexpr int kTcMaxRegion = 4096;                               // staged control points per brick
constexpr size_t kTcSmemMax = 227 * 1024;

struct TcDev {
    int ct;                  // transform: cells per tile (rows per component)
    int ctc;                 // contrib: cells per tile (3-D: 32, so that a lane quarter is one
                             // component's 32 consecutive cells and its stores are whole lines)
    // transform
    int bx, by, bz;          // brick of cells per tile
    int tiles[3];
    int rx, ry, rz;          // control-point region of a brick
    int rxp, ryp, rzb;       // its staged box: x covers the origin's rounding down to a multiple of 4,
                             // y and z padding place the rows on distinct shared-memory banks
    int rps;                 // floats per staged plane (rxp ryp rzb)
    int rbuf;                // floats per region buffer (D planes, 128-byte aligned)
    int nrb;                 // region buffers (2 or 3: loads run that many tiles ahead, minus one)
    int nus;                 // output staging buffers (0: the epilogue stores u directly)
    int ustr;                // floats per staged output row (np + 4: rows 4 banks apart)
    int ustage;              // floats per staging buffer (D brick rows, 128-byte aligned)
    int pairs_x;             // tap pairs per x row: ceil(nt0 / 2)
    int npairs;              // tap pairs (two x-neighbouring taps, the second virtual when nt0 is odd)
                             // with a nonzero table column
    int kp;                  // 4 * ceil(npairs / 2) padded to 32 (K): k = 4 u + j, unit u = pairs 2u, 2u + 1
    int np;                  // phases padded to 16 (half of N)
    int ns_tr;               // A stages in TMEM (one 32-tap K block each: 32 hi + 32 lo columns)
    int tr_stride, tr_cols;  // TMEM columns per accumulator, allocated columns
    int tr_abase;            // first TMEM column of the A stages
    const float *btr;        // 2 np rows x kp, K-major 128-byte swizzled
    // contrib
    const int2 *pairoff;     // [kp / 4]: region offsets (tx + rxp (ty + ryp tz)) of a unit's two pairs
    int kpc;                 // phases padded to 32 (K)
    int nct;                 // contrib taps: the box taps with a nonzero table column
    int npc;                 // nct padded to 16 (N)
    int ns_con;              // shared-memory stages (one 32-phase K block each)
    int nrr;                 // record ring slots (tiled loads of a chunk's records; 0: direct loads)
    int rslot, rfix;         // bytes per ring slot, offset of the fixed-image values in a slot
    int con_stride, con_cols;
    const float *bcon;       // npc rows x kpc, K-major 128-byte swizzled: hi, then lo
    unsigned *err;           // sticky failure word of the bounded waits (read and reset by the host)
    unsigned long long wait_ns;  // contrib: limit of one bounded wait (2 s; shortened by the wait drill)
    int drill;               // contrib: CTA 0's first producer group withholds its first stage from the
                             // MMA thread, whose wait for it then runs out (skm_evaluator_wait_drill)
    // contrib with brick partials (3-D): tiles are bricks of kBrick cells loaded by 5-D / 4-D tiled
    // loads, the epilogue scatters each cell's tap columns into its brick's control-point patch
    int fused;               // 1: brick partials (the launch chooses), 0: the Contrib array
    int nbrick[3];           // bricks per axis
    int pxp, pyp, pzp, pv;   // patch extent per axis, floats per component patch
    const int *cpoff;        // [nct]: patch offset (ox + px (oy + py oz)) of contrib tap k
    float *partial;          // [brick][comp][pv]
};

constexpr int kBrickX = 4, kBrickY = 4, kBrickZ = 2;   // contrib brick (32 cells: one lane quarter)
constexpr int kConEpiBar = 4;                          // contrib: named barrier of the epilogue warps

// mbarriers of one CTA: full[s] producers -> MMA (kTcProdThreads arrivals), empty[s] MMA ->
// producers (commit), acc_full[b] MMA -> epilogue (commit), acc_empty[b] epilogue -> MMA
// (kTcEpiWarps * 32 arrivals), drain (final commit of the MMA thread), table and region[b]
// (transaction counts of the bulk copies), region_empty[b] producers -> region loads (one arrival)
struct TcBars {
    uint64_t *full, *empty, *acc_full, *acc_empty, *drain, *table, *region, *region_empty;
    __device__ explicit TcBars(uint64_t *b)
        : full(b), empty(b + kTcStages), acc_full(b + 2 * kTcStages), acc_empty(b + 2 * kTcStages + 2),
          drain(b + 2 * kTcStages + 4), table(b + 2 * kTcStages + 5), region(b + 2 * kTcStages + 6),
          region_empty(b + 2 * kTcStages + 6 + kTcRegionBufs)
    {
    }
    __device__ void init(int full_count, int epi_threads = kTcEpiWarps * 32) const
    {
        for (int s = 0; s < kTcStages; ++s) {     // stages beyond the kernel's count stay unused
            tc::mbar_init(&full[s], full_count);
            tc::mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            tc::mbar_init(&acc_full[b], 1);
            tc::mbar_init(&acc_empty[b], epi_threads);
        }
        tc::mbar_init(drain, 1);
        tc::mbar_init(table, 1);
        for (int b = 0; b < kTcRegionBufs; ++b) {
            tc::mbar_init(&region[b], 1);
            tc::mbar_init(&region_empty[b], 1);
        }
        tc::fence_mbarrier_init();
    }
};

__device__ __forceinline__ void tc_fail(volatile int *abort, unsigned *err)
{
    *abort = 1;
    atomicOr(err, 1u);
}

__device__ __forceinline__ void split4(const float *v, float4 &h, float4 &l)
{
    float hx, lx, hy, ly, hz, lz, hw, lw;
    tc::split_tf32(v[0], hx, lx);
    tc::split_tf32(v[1], hy, ly);
    tc::split_tf32(v[2], hz, lz);
    tc::split_tf32(v[3], hw, lw);
    h = make_float4(hx, hy, hz, hw);
    l = make_float4(lx, ly, lz, lw);
}

__device__ __forceinline__ void cp_async16(void *dst, const void *src, bool valid)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(tc::smem_addr(dst)), "l"(src),
                 "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Teardown shared by both kernels: the MMA thread waits (bounded) until its MMAs have retired,
// then the MMA warp frees the TMEM after every role has left its loop.
__device__ __forceinline__ void tc_teardown(const TcBars &B, uint32_t tmem, uint32_t cols, int mma_warp = kTcMmaWarp)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == mma_warp && lane == 0) {
        tc::commit(B.drain);
        tc::mbar_wait(B.drain, 0);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == mma_warp) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tmem, cols);
    }
}

// Shared-memory carve-up, in bytes from a 1024-byte-aligned base (the swizzle atoms need it):
// A stages first (each [hi | lo], 128 rows x 32 K elements = 16 KB per half), then the table.
constexpr int kTcStageBytes = 2 * kTcRows * kTcKBlock * 4;

// Transform: the table, then nrb region buffers, each one tiled load of the weighted control-point
// planes (RegionPlanes) over a brick's region: [D][rzb][ryp][rxp] floats; then nus output staging
// buffers, each the tile's u as [D][bz][by][bx][ustr] floats for one tiled store.
struct TcTransformLayout {
    int b, reg, pairoff, ust, bars, total_bytes;
    __host__ __device__ explicit TcTransformLayout(const TcDev &C)
    {
        b = 0;                                         // the table (A stages live in TMEM)
        reg = (b + C.kp * 2 * C.np * 4 + 127) / 128 * 128;   // [nrb][rbuf] floats, 128-byte aligned
        pairoff = reg + C.nrb * 4 * C.rbuf;            // [kp / 4] int2: region offsets of a unit's pairs
        ust = (pairoff + 8 * (C.kp / 4) + 127) / 128 * 128;  // [nus][ustage] floats
        bars = (ust + C.nus * 4 * C.ustage + 15) / 16 * 16;
        total_bytes = bars + 8 * kTcNumBars + 8 + 1024;   // + alignment slack of the base
    }
};

// tiled store of a 5-D box from shared memory (bulk group of the issuing thread; no multicast)
__device__ __forceinline__ void tma_store_5d(const CUtensorMap *map, const void *src, int c0, int c1, int c2, int c3,
                                             int c4)
{
    asm volatile("cp.async.bulk.tensor.5d.global.shared::cta.bulk_group [%0, {%2, %3, %4, %5, %6}], [%1];"
                 :: "l"(map), "r"(tc::smem_addr(src)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4) : "memory");
}

__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int x, int y, int z, int w,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
        :: "r"(tc::smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(w), "r"(tc::smem_addr(bar)) : "memory");
}

// Contrib: A stages, the table (hi, lo), then nrr ring slots, each a chunk's records (cell c, phase
// p of the chunk: 128-byte rows c * 4 + p / 8, their 16-byte pieces swizzled by the row index, as
// the tiled load's 128-byte swizzle writes them) and fixed-image values ([cell][32] floats).
struct TcContribLayout {
    int a, bhi, blo, rr, patch, poff, bars, total_bytes;
    // fused: patches of the two epilogue halves for every component, and the taps' patch offsets
    __host__ __device__ TcContribLayout(const TcDev &C, bool fused)
    {
        a = 0;
        bhi = a + C.ns_con * kTcStageBytes;
        blo = bhi + C.kpc * C.npc * 4;
        rr = (blo + C.kpc * C.npc * 4 + 1023) / 1024 * 1024;
        patch = rr + C.nrr * C.rslot;
        poff = patch + (fused ? 2 * 3 * C.pv * 4 : 0);
        bars = (poff + (fused ? C.npc * 4 : 0) + 15) / 16 * 16;
        total_bytes = bars + 8 * kTcNumBars + 8 + 1024;
    }
};

__device__ __forceinline__ unsigned char *tc_aligned_smem(float4 *dyn)
{
    const uint32_t a = tc::smem_addr(dyn);
    return reinterpret_cast<unsigned char *>(dyn) + (((a + 1023u) & ~1023u) - a);
}

// ------------------------------------------------------------------------------------------------
// u(q, p) = sum_t T[p][t] (w alpha)[q + t] on the tensor cores; u planar [comp][cell][phase].
// The region of each brick comes by one tiled TMA load (no multicast) of the weighted
// control-point planes, into a ring of nrb buffers so that the loads run ahead of the bricks; the
// A operand (im2col of the region, split into tf32 hi / lo in registers) goes from registers
// straight into TMEM stages (tcgen05.st) and the MMAs read it there, so shared memory carries only
// the region reads and the table reads of the tensor cores.
__global__ void __launch_bounds__(kTcThreads, 1) table_transform_tc_kernel(EvalParams P, TableDev T, TcDev C,
                                                                           const __grid_constant__ CUtensorMap rmap,
                                                                           const __grid_constant__ CUtensorMap umap)
{
    extern __shared__ float4 tc_smem4[];
    unsigned char *sm = tc_aligned_smem(tc_smem4);
    const TcTransformLayout L(C);
    float *Bs = reinterpret_cast<float *>(sm + L.b);
    float *Rg = reinterpret_cast<float *>(sm + L.reg);
    int2 *pairoff = reinterpret_cast<int2 *>(sm + L.pairoff);
    uint64_t *barmem = reinterpret_cast<uint64_t *>(sm + L.bars);
    const TcBars B(barmem);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(barmem + kTcNumBars);
    volatile int *abort = reinterpret_cast<volatile int *>(tmem_holder + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Kp = C.kp, Np = C.np, N2 = 2 * C.np, NS = C.ns_tr;
    const int D = T.D;
    const int ntiles = C.tiles[0] * C.tiles[1] * C.tiles[2];
    const int nchunk = Kp / kTcKBlock;
    const int brick = C.bx * C.by * C.bz;
    const uint32_t table_bytes = (uint32_t)(Kp * N2 * 4);
    const int NB = C.nrb;
    const uint32_t region_bytes = (uint32_t)(D * C.rps * 4);
    const int mine = (int)blockIdx.x < ntiles ? (ntiles - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x : 0;
    // the tiled load of the region of the CTA's k-th tile into buffer k % NB (one thread); x
    // rounds down to a multiple of 4 (the load's alignment rule), the producers index from the
    // remainder
    auto issue_region = [&](int k) {
        const int tile = blockIdx.x + k * gridDim.x;
        const int t0 = tile % C.tiles[0], t12 = tile / C.tiles[0];
        const int jx = T.qmin[0] + t0 * C.bx + T.tlo[0];
        const int jy = T.qmin[1] + (t12 % C.tiles[1]) * C.by + T.tlo[1];
        const int jz = T.qmin[2] + (t12 / C.tiles[1]) * C.bz + T.tlo[2];
        tc::mbar_expect_tx(&B.region[k % NB], region_bytes);
        tma_load_4d(Rg + (k % NB) * C.rbuf, &rmap, jx & ~3, jy, jz, 0, &B.region[k % NB]);
    };

    // the load-issuing thread sets up the barriers and starts the table and the first regions at
    // once, while the others allocate TMEM and stage the pair offsets
    if (warp == kTrTmaWarp && lane == 0) {
        B.init(kTrProdThreads);
        *abort = 0;
        tc::mbar_expect_tx(B.table, table_bytes);            // the table: one bulk copy
        tc::bulk_g2s(Bs, C.btr, table_bytes, B.table);
        for (int k = 0; k < NB && k < mine; ++k) issue_region(k);
    }
    if (warp == kTcMmaWarp) tc::tmem_alloc(tmem_holder, (uint32_t)C.tr_cols);
    // unit u of the K axis = tap pairs 2u and 2u + 1 (pairs: x-neighbouring taps of one x row)
    for (int u = tid; u < Kp / 4; u += kTcThreads) pairoff[u] = C.pairoff[u];
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_holder;

    if (warp == kTrTmaWarp) {
        // ---------------- region loads (one thread), NB tiles ahead ----------------
        if (lane == 0) {
            int k = NB;
            for (; k < mine; ++k) {
                // buffer k % NB is free once every producer has left tile k - NB
                if (!tc::mbar_wait(&B.region_empty[k % NB], (k / NB - 1) & 1, abort)) {
                    tc_fail(abort, C.err);
                    break;
                }
                issue_region(k);
            }
            // the last load into each buffer lands before the CTA leaves (bounded): a failed
            // CTA may leave loads nobody waits for
            const int issued = k < mine ? k : mine;
            for (int j = issued > NB ? issued - NB : 0; j < issued; ++j) tc::mbar_wait(&B.region[j % NB], (j / NB) & 1);
        }
        __syncwarp();
    } else if (warp >= kTcEpiWarps + 1) {
        // ---------------- producers: region -> split im2col hi/lo stages in TMEM ----------------
        // A warp writes the TMEM lanes of its quarter (warp % 4): thread = row r, and slice h of
        // each 32-column K block (kTrCols / 4 units of 4 columns), hi and lo.
        const int q = warp & 3, h = (warp - (kTcEpiWarps + 1)) >> 2;
        const int pt = tid - kTcProdBase;
        const int r = 32 * q + lane;
        const int comp = r / C.ct, c = r - comp * C.ct;
        const bool row_exists = comp < D && c < brick;
        const int cx = c % C.bx, cy = (c / C.bx) % C.by, cz = c / (C.bx * C.by);
        // rows without a cell read real region data; the epilogue never stores them
        const int rowbase = row_exists ? cx + C.rxp * (cy + C.ryp * cz) : 0;
        const int cbase = row_exists ? comp * C.rps : 0;
        const uint32_t lane_addr = (uint32_t)(32 * q) << 16;
        // control-point index of a tile's region origin
        auto region_origin = [&](int tile, int *j0) {
            const int t0 = tile % C.tiles[0], t12 = tile / C.tiles[0];
            j0[0] = T.qmin[0] + t0 * C.bx + T.tlo[0];
            j0[1] = T.qmin[1] + (t12 % C.tiles[1]) * C.by + T.tlo[1];
            j0[2] = T.qmin[2] + (t12 / C.tiles[1]) * C.bz + T.tlo[2];
        };
        int s = 0;
        uint32_t phase = 0;                                  // parity of stage s's current use
        unsigned g = 0;
        bool failed = false;
        for (int it = 0;; ++it) {
            const int tile = blockIdx.x + it * gridDim.x;
            if (tile >= ntiles) break;
            {
                const bool ok = tc::mbar_wait(&B.region[it % NB], (it / NB) & 1, abort);
                if (__any_sync(0xffffffffu, !ok)) {
                    if (lane == 0) tc_fail(abort, C.err);
                    failed = true;
                }
            }
            int j0[3];
            region_origin(tile, j0);
            const float *R = Rg + (it % NB) * C.rbuf + cbase + rowbase + (j0[0] & 3);
            for (int kc = 0; kc < nchunk; ++kc, ++g) {
                // a failed wait skips the rest of the tile (warp-uniform: tcgen05.st is warp-wide);
                // the decision is made uniform across the producers at the tile's end
                if (!failed && g >= (unsigned)NS) {
                    const bool ok = tc::mbar_wait(&B.empty[s], phase ^ 1u, abort);
                    if (__any_sync(0xffffffffu, !ok)) {
                        if (lane == 0) tc_fail(abort, C.err);
                        failed = true;
                    }
                }
                if (!failed) {
                    tc::fence_after_sync();
                    float vh[kTrCols], vl[kTrCols];
                    const int2 *po = pairoff + kc * (kTcKBlock / 4) + (kTrCols / 4) * h;
#pragma unroll
                    for (int u = 0; u < kTrCols / 4; ++u) {
                        const int2 o = po[u];
                        tc::split_tf32(R[o.x], vh[4 * u], vl[4 * u]);
                        tc::split_tf32(R[o.x + 1], vh[4 * u + 1], vl[4 * u + 1]);
                        tc::split_tf32(R[o.y], vh[4 * u + 2], vl[4 * u + 2]);
                        tc::split_tf32(R[o.y + 1], vh[4 * u + 3], vl[4 * u + 3]);
                    }
                    const uint32_t col = (uint32_t)(C.tr_abase + 2 * kTcKBlock * s + kTrCols * h);
                    if (kTrCols == 16) {
                        tc::tmem_st16(tmem + lane_addr + col, vh);
                        tc::tmem_st16(tmem + lane_addr + col + kTcKBlock, vl);
                    } else {
                        tc::tmem_st8(tmem + lane_addr + col, vh);
                        tc::tmem_st8(tmem + lane_addr + col + kTcKBlock, vl);
                    }
                    tc::tmem_wait_st();
                    tc::fence_before_sync();
                    tc::mbar_arrive(&B.full[s]);
                }
                if (++s == NS) {
                    s = 0;
                    phase ^= 1u;
                }
            }
            // every producer has finished the tile (and read its region buffer for the last time)
            if (tc::bar_or(kTcProdBar, kTrProdThreads, failed)) break;
            if (pt == 0) tc::mbar_arrive(&B.region_empty[it % NB]);
        }
    } else if (warp == kTcMmaWarp) {
        // ---------------- MMA issue (one thread) ----------------
        if (lane == 0) {
            const uint32_t idesc_cat = tc::idesc_tf32(kTcRows, N2), idesc_hi = tc::idesc_tf32(kTcRows, Np);
            const uint32_t b_base = tc::smem_addr(Bs);
            bool ok = tc::mbar_wait(B.table, 0, abort);      // the table has landed
            if (!ok) tc_fail(abort, C.err);
            int s = 0;
            uint32_t phase = 0;
            for (int it = 0; ok; ++it) {
                const int tile = blockIdx.x + it * gridDim.x;
                if (tile >= ntiles) break;
                const int b = it & 1;
                if (it >= 2 && !tc::mbar_wait(&B.acc_empty[b], ((it >> 1) + 1) & 1, abort)) {
                    tc_fail(abort, C.err);
                    break;
                }
                tc::fence_after_sync();
                bool failed = false;
                for (int kc = 0; kc < nchunk; ++kc) {
                    if (!tc::mbar_wait(&B.full[s], phase, abort)) {
                        tc_fail(abort, C.err);
                        failed = true;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t dacc = tmem + (uint32_t)(b * C.tr_stride);
                    const uint32_t ahi = tmem + (uint32_t)(C.tr_abase + 2 * kTcKBlock * s);
                    const uint32_t alo = ahi + (uint32_t)kTcKBlock;
                    const uint32_t bk = b_base + (uint32_t)kc * (uint32_t)N2 * 128u;   // K block kc of the table
#pragma unroll
                    for (int ks = 0; ks < kTcKBlock / 8; ++ks) {
                        const uint64_t db = tc::smem_desc_sw128(bk + 32u * ks);
                        tc::mma_tf32_tmem_a(dacc, ahi + 8u * ks, db, idesc_cat, (kc | ks) != 0);
                        tc::mma_tf32_tmem_a(dacc, alo + 8u * ks, db, idesc_hi, 1);
                    }
                    tc::commit(&B.empty[s]);
                    if (++s == NS) {
                        s = 0;
                        phase ^= 1u;
                    }
                }
                if (failed) break;
                tc::commit(&B.acc_full[b]);
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: TMEM -> u (lane quarter = warp) ----------------
        // Staged (nus > 0): the rows go to a shared-memory tile that one tiled store writes to u
        // (cells past the grid's end fall outside the tensor and are not written), so that the
        // output leaves as whole lines instead of one 16-byte piece per row and instruction.
        const long long plane = T.ncell * T.nph;
        const int r = warp * 32 + lane;
        const int comp = r / C.ct, c = r - comp * C.ct;
        const int cx = c % C.bx, cy = (c / C.bx) % C.by, cz = c / (C.bx * C.by);
        const bool row_ok = comp < D && c < brick;
        float *ust = reinterpret_cast<float *>(sm + L.ust);
        const int NU = C.nus;
        for (int it = 0;; ++it) {
            const int tile = blockIdx.x + it * gridDim.x;
            if (tile >= ntiles) break;
            const int b = it & 1;
            const int sb = NU > 0 ? it % NU : 0;
            // the staging buffer's previous store (NU tiles ago) has read it
            if (NU > 0 && tid == 0) {
                if (NU > 1) tc::bulk_wait_read<1>();
                else tc::bulk_wait_read<0>();
            }
            // warp-uniform decision (tcgen05.ld below is a warp-wide instruction), made uniform
            // across the epilogue warps when they share barriers
            const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(&B.acc_full[b], (it >> 1) & 1, abort));
            if (NU > 0 ? tc::bar_or(kTrEpiBar, kTcEpiWarps * 32, !ok) : !ok) {
                if (lane == 0 && !ok) tc_fail(abort, C.err);
                break;
            }
            tc::fence_after_sync();
            const int t0 = tile % C.tiles[0], t1 = (tile / C.tiles[0]) % C.tiles[1], t2 = tile / (C.tiles[0] * C.tiles[1]);
            const uint32_t tb = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * C.tr_stride);
            if (NU > 0) {
                float *dst = ust + sb * C.ustage + (comp * brick + c) * C.ustr;
                for (int j = 0; j < (Np >> 4); ++j) {
                    float vh[16], vl[16];
                    tc::tmem_ld16(tb + (uint32_t)(16 * j), vh);
                    tc::tmem_ld16(tb + (uint32_t)(Np + 16 * j), vl);
                    if (row_ok)
#pragma unroll
                        for (int v = 0; v < 4; ++v)
                            reinterpret_cast<float4 *>(dst + 16 * j)[v] =
                                make_float4(vh[4 * v] + vl[4 * v], vh[4 * v + 1] + vl[4 * v + 1],
                                            vh[4 * v + 2] + vl[4 * v + 2], vh[4 * v + 3] + vl[4 * v + 3]);
                }
                tc::fence_before_sync();
                tc::mbar_arrive(&B.acc_empty[b]);            // the accumulator is free again
                tc::fence_proxy_async_smem();
                tc::bar_sync(kTrEpiBar, kTcEpiWarps * 32);
                if (tid == 0) {
                    tma_store_5d(&umap, ust + sb * C.ustage, 0, t0 * C.bx, t1 * C.by, t2 * C.bz, 0);
                    tc::bulk_commit();
                }
                continue;
            }
            const int qx = t0 * C.bx + cx, qy = t1 * C.by + cy, qz = t2 * C.bz + cz;
            const bool valid = row_ok && qx < T.nq[0] && qy < T.nq[1] && qz < T.nq[2];
            const long long cell = (long long)qx + (long long)T.nq[0] * (qy + (long long)T.nq[1] * qz);
            for (int j = 0; j < (Np >> 4); ++j) {
                float vh[16], vl[16];
                tc::tmem_ld16(tb + (uint32_t)(16 * j), vh);
                tc::tmem_ld16(tb + (uint32_t)(Np + 16 * j), vl);
                if (valid) {
                    float *dst = T.ucp + (long long)comp * plane + cell * T.nph + 16 * j;
                    if (16 * j + 16 <= T.nph && (T.nph & 3) == 0) {
#pragma unroll
                        for (int v = 0; v < 4; ++v)
                            reinterpret_cast<float4 *>(dst)[v] =
                                make_float4(vh[4 * v] + vl[4 * v], vh[4 * v + 1] + vl[4 * v + 1],
                                            vh[4 * v + 2] + vl[4 * v + 2], vh[4 * v + 3] + vl[4 * v + 3]);
                    } else {
                        for (int v = 0; v < 16; ++v)
                            if (16 * j + v < T.nph) dst[v] = vh[v] + vl[v];
                    }
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&B.acc_empty[b]);
        }
        if (NU > 0 && tid == 0) tc::bulk_wait_all();          // the stores complete before the CTA leaves
    }
    // the table copy has completed before the teardown frees nothing in shared memory it writes:
    // the MMA thread waited for it, or (no tile) wait here (bounded)
    if (tid == 0 && (int)blockIdx.x >= ntiles) tc::mbar_wait(B.table, 0, abort);
    tc_teardown(B, tmem, (uint32_t)C.tr_cols);
}

// ------------------------------------------------------------------------------------------------
// Contrib[comp][t][cell] = sum_p T[p][t] g(cell, p) on the tensor cores
__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
        :: "r"(tc::smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(tc::smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void tma_load_5d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3, int c4,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.5d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5, %6}], [%7];"
        :: "r"(tc::smem_addr(dst)), "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(c4), "r"(tc::smem_addr(bar))
        : "memory");
}

// FUSED (3-D, tiled record loads): a tile is a brick of kBrickX x kBrickY x kBrickZ cells (row c =
// x + 4 y + 16 z of its lane quarter), loaded by 5-D / 4-D tiled loads (cells past the grid read
// as zeros), and the epilogue scatters each cell's tap columns into the brick's control-point
// patch in shared memory -- one tap after the other, the lanes of a tap on distinct control
// points, so every patch entry sums in a fixed order without atomics -- then writes the patch
// (the two column halves added) as the brick's partial.  Otherwise Contrib[comp][tap][cell].
template <bool FUSED>
__global__ void __launch_bounds__(kConThreads, 1) table_contrib_tc_kernel(TableDev T, TcDev C,
                                                                        const double *__restrict__ stats,
                                                                        const __grid_constant__ CUtensorMap recmap,
                                                                        const __grid_constant__ CUtensorMap fixmap)
{
    extern __shared__ float4 tc_smem4[];
    unsigned char *sm = tc_aligned_smem(tc_smem4);
    const TcContribLayout L(C, FUSED);
    unsigned char *As = sm + L.a;
    float *Bhi = reinterpret_cast<float *>(sm + L.bhi), *Blo = reinterpret_cast<float *>(sm + L.blo);
    uint64_t *barmem = reinterpret_cast<uint64_t *>(sm + L.bars);
    const TcBars B(barmem);
    uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(barmem + kTcNumBars);
    volatile int *abort = reinterpret_cast<volatile int *>(tmem_holder + 1);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int Kp = C.kpc, Np = C.npc, ct = C.ctc, NS = C.ns_con;
    const int D = T.D, nph = T.nph;
    const long long ntiles = FUSED ? (long long)C.nbrick[0] * C.nbrick[1] * C.nbrick[2] : (T.ncell + ct - 1) / ct;
    const int nchunk = Kp / kTcKBlock;

    if (FUSED) {                                            // zeroed patches, the taps' patch offsets
        float *patch = reinterpret_cast<float *>(sm + L.patch);
        for (int i = tid; i < 2 * 3 * C.pv; i += kConThreads) patch[i] = 0.f;
        int *poff = reinterpret_cast<int *>(sm + L.poff);
        for (int k = tid; k < C.nct; k += kConThreads) poff[k] = C.cpoff[k];
    }
    if (tid == 0) {
        B.init(kTcGroupThreads, kConEpiWarps * 32);
        *abort = 0;
        // the table (hi, then lo): one bulk copy, waited for by the MMA thread
        tc::mbar_expect_tx(B.table, (uint32_t)(2 * Kp * Np * 4));
        tc::bulk_g2s(Bhi, C.bcon, (uint32_t)(2 * Kp * Np * 4), B.table);
    }
    if (warp == kConMmaWarp) tc::tmem_alloc(tmem_holder, (uint32_t)C.con_cols);
    // rows past D * ct never receive data: zero their 128-byte rows once in every stage half
    const int pad_rows = kTcRows - D * ct;
    for (int i = tid; i < NS * 2 * pad_rows * 8; i += kConThreads) {
        const int half = i / (pad_rows * 8), r = D * ct + (i / 8) % pad_rows, c16 = i & 7;
        *reinterpret_cast<float4 *>(As + half * (kTcStageBytes / 2) + (r >> 3) * 1024 + (r & 7) * 128 + c16 * 16) =
            make_float4(0.f, 0.f, 0.f, 0.f);
    }
    tc::fence_proxy_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = *tmem_holder;
    unsigned char *Rr = sm + L.rr;
    const int NR = C.nrr;

    if (warp == kConLoadWarp) {
        // ---------------- record loads (one thread), NR chunks ahead ----------------
        if (lane == 0 && NR > 0) {
            const long long mine = (long long)blockIdx.x < ntiles ? (ntiles - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
            const long long nch = mine * nchunk;
            const uint32_t bytes = (uint32_t)(ct * 32 * 20);
            long long g = 0;
            for (; g < nch; ++g) {
                const int slot = (int)(g % NR);
                // slot g % NR is free once its producer group has left chunk g - NR
                if (g >= NR && !tc::mbar_wait(&B.region_empty[slot], (uint32_t)((g / NR - 1) & 1), abort, C.wait_ns)) {
                    tc_fail(abort, C.err);
                    break;
                }
                const long long tile = blockIdx.x + (g / nchunk) * gridDim.x;
                const int kc = (int)(g % nchunk);
                unsigned char *dst = Rr + slot * C.rslot;
                tc::mbar_expect_tx(&B.region[slot], bytes);
                if (FUSED) {
                    const int bx = (int)(tile % C.nbrick[0]) * kBrickX;
                    const int by = (int)((tile / C.nbrick[0]) % C.nbrick[1]) * kBrickY;
                    const int bz = (int)(tile / ((long long)C.nbrick[0] * C.nbrick[1])) * kBrickZ;
                    tma_load_5d(dst, &recmap, 0, kc * 4, bx, by, bz, &B.region[slot]);
                    tma_load_4d(dst + C.rfix, &fixmap, kc * kTcKBlock, bx, by, bz, &B.region[slot]);
                } else {
                    tma_load_3d(reinterpret_cast<float *>(dst), &recmap, 0, kc * 4, (int)(tile * ct), &B.region[slot]);
                    tma_load_2d(dst + C.rfix, &fixmap, kc * kTcKBlock, (int)(tile * ct), &B.region[slot]);
                }
            }
            // the last load into each slot lands before the CTA leaves (bounded)
            for (long long j = g > NR ? g - NR : 0; j < g; ++j)
                tc::mbar_wait(&B.region[j % NR], (uint32_t)((j / NR) & 1));
        }
        __syncwarp();
    } else if (warp >= kConEpiWarps + 1) {
        // ---------------- producers: g = (a f + b m + c) grad M, hi/lo stages ----------------
        // Two groups of 4 warps take alternate K chunks, so that one group's global loads are in
        // flight while the other converts and stores.  Item = (cell c, 4 phases); 8 consecutive lanes
        // take the 32 phases of one cell, so a warp's record loads cover 4 contiguous 512-byte runs.
        const int pt = tid - kConProdBase;
        const int grp = pt / kTcGroupThreads, gt = pt - grp * kTcGroupThreads;
        const float cf = (float)stats[S_COEF_F], cm = (float)stats[S_COEF_M], cc = (float)stats[S_COEF_C];
        const int nitems = ct * (kTcKBlock / 4);
        constexpr int kMaxItems = 3;                        // ceil(42 * 8 / 128); 2-D: 64 * 8 / 128 = 4
        const bool vec = (nph & 3) == 0;
        bool failed = false;
        for (unsigned g = grp;; g += 2) {
            const long long tile = blockIdx.x + (long long)(g / nchunk) * gridDim.x;
            if (tile >= ntiles) break;
            const int kc = (int)(g % nchunk);
            const long long cell0 = tile * ct;
            const int s = (int)(g % NS);
            bool ok = true;
            if (g >= (unsigned)NS) ok = tc::mbar_wait(&B.empty[s], ((g / NS) + 1) & 1, abort, C.wait_ns);
            if (NR > 0 && ok) ok = tc::mbar_wait(&B.region[g % NR], (g / NR) & 1, abort, C.wait_ns);   // the records
            if (tc::bar_or(kTcGroupBar + grp, kTcGroupThreads, !ok)) {
                if (gt == 0) tc_fail(abort, C.err);
                failed = true;
                break;
            }
            unsigned char *Ahi = As + s * kTcStageBytes, *Alo = Ahi + kTcStageBytes / 2;
            const int k0 = kc * kTcKBlock;
            const unsigned char *slot = Rr + (NR > 0 ? (int)(g % NR) * C.rslot : 0);
            const float *fsm = reinterpret_cast<const float *>(slot + C.rfix);
            for (int base = 0; base < nitems; base += kMaxItems * kTcGroupThreads) {
                float4 rr[kMaxItems][4], ff[kMaxItems];
#pragma unroll
                for (int u = 0; u < kMaxItems; ++u) {           // all loads first
                    const int i = base + gt + u * kTcGroupThreads;
                    const int c = i >> 3, jg = i & 7;
                    const long long cell = cell0 + c;
                    const int p0 = k0 + 4 * jg;
                    if (NR > 0) {                                // from the ring slot (zeros past the data)
                        const bool in = i < nitems;
#pragma unroll
                        for (int e = 0; e < 4; ++e) {
                            const int row = 4 * c + ((4 * jg + e) >> 3), piece = ((4 * jg + e) & 7) ^ (row & 7);
                            rr[u][e] = in ? *reinterpret_cast<const float4 *>(slot + row * 128 + piece * 16)
                                          : make_float4(0.f, 0.f, 0.f, 0.f);
                        }
                        ff[u] = in ? *reinterpret_cast<const float4 *>(fsm + c * kTcKBlock + 4 * jg)
                                   : make_float4(0.f, 0.f, 0.f, 0.f);
                        continue;
                    }
                    const bool in = i < nitems && cell < T.ncell;
#pragma unroll
                    for (int e = 0; e < 4; ++e)
                        rr[u][e] = (in && p0 + e < nph) ? T.rec[cell * nph + p0 + e] : make_float4(0.f, 0.f, 0.f, 0.f);
                    if (in && vec && p0 < nph) {
                        ff[u] = *reinterpret_cast<const float4 *>(T.fixcp + cell * nph + p0);
                    } else {
                        float f4[4];
#pragma unroll
                        for (int e = 0; e < 4; ++e) f4[e] = (in && p0 + e < nph) ? T.fixcp[cell * nph + p0 + e] : 0.f;
                        ff[u] = make_float4(f4[0], f4[1], f4[2], f4[3]);
                    }
                }
#pragma unroll
                for (int u = 0; u < kMaxItems; ++u) {
                    const int i = base + gt + u * kTcGroupThreads;
                    if (i >= nitems) break;
                    const int c = i >> 3, jg = i & 7;
                    const float fv[4] = {ff[u].x, ff[u].y, ff[u].z, ff[u].w};
                    float gv[3][4];
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const float coef = fmaf(cf, fv[e], fmaf(cm, rr[u][e].w, cc));
                        gv[0][e] = coef * rr[u][e].x;
                        gv[1][e] = coef * rr[u][e].y;
                        gv[2][e] = coef * rr[u][e].z;
                    }
#pragma unroll
                    for (int comp = 0; comp < 3; ++comp) {
                        if (comp < D) {
                            float4 h, l;
                            split4(gv[comp], h, l);
                            const uint32_t off = tc::sw128_offset(comp * ct + c, 4 * jg, kTcRows);
                            *reinterpret_cast<float4 *>(Ahi + off) = h;
                            *reinterpret_cast<float4 *>(Alo + off) = l;
                        }
                    }
                }
            }
            if (NR > 0) {                                        // the group has read the slot
                tc::bar_sync(kTcGroupBar + grp, kTcGroupThreads);
                if (gt == 0) tc::mbar_arrive(&B.region_empty[g % NR]);
            }
            tc::fence_proxy_async();
            // the wait drill: CTA 0 withholds stage 0 of its first chunk (no MMA, no copy depends on
            // it), so the MMA thread's first wait runs out and every role leaves through its error path
            if (!(C.drill && blockIdx.x == 0 && g == 0)) tc::mbar_arrive(&B.full[s]);
        }
    } else if (warp == kConMmaWarp) {
        // ---------------- MMA issue (one thread) ----------------
        if (lane == 0) {
            const uint32_t idesc = tc::idesc_tf32(kTcRows, Np);
            const uint32_t a_base = tc::smem_addr(As), bh_base = tc::smem_addr(Bhi), bl_base = tc::smem_addr(Blo);
            unsigned g = 0;
            const bool table_ok = tc::mbar_wait(B.table, 0, abort);   // the table has landed
            if (!table_ok) tc_fail(abort, C.err);
            for (int it = 0; table_ok; ++it) {
                const long long tile = blockIdx.x + (long long)it * gridDim.x;
                if (tile >= ntiles) break;
                const int b = it & 1;
                if (it >= 2 && !tc::mbar_wait(&B.acc_empty[b], ((it >> 1) + 1) & 1, abort, C.wait_ns)) {
                    tc_fail(abort, C.err);
                    break;
                }
                tc::fence_after_sync();
                bool failed = false;
                for (int kc = 0; kc < nchunk; ++kc, ++g) {
                    const int s = (int)(g % NS);
                    if (!tc::mbar_wait(&B.full[s], (g / NS) & 1, abort, C.wait_ns)) {
                        tc_fail(abort, C.err);
                        failed = true;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t dacc = tmem + (uint32_t)(b * C.con_stride);
                    const uint32_t ahi = a_base + (uint32_t)(s * kTcStageBytes);
                    const uint32_t alo = ahi + (uint32_t)(kTcStageBytes / 2);
                    const uint32_t bo = (uint32_t)kc * (uint32_t)Np * 128u;             // K block kc of the table
#pragma unroll
                    for (int ks = 0; ks < kTcKBlock / 8; ++ks) {
                        const uint64_t dah = tc::smem_desc_sw128(ahi + 32u * ks);
                        const uint64_t dal = tc::smem_desc_sw128(alo + 32u * ks);
                        const uint64_t dbh = tc::smem_desc_sw128(bh_base + bo + 32u * ks);
                        const uint64_t dbl = tc::smem_desc_sw128(bl_base + bo + 32u * ks);
                        tc::mma_tf32(dacc, dah, dbh, idesc, (kc | ks) != 0);
                        tc::mma_tf32(dacc, dah, dbl, idesc, 1);
                        tc::mma_tf32(dacc, dal, dbh, idesc, 1);
                    }
                    tc::commit(&B.empty[s]);
                }
                if (failed) break;
                tc::commit(&B.acc_full[b]);
            }
        }
        __syncwarp();
    } else if (FUSED) {
        // ---------------- epilogue: TMEM -> brick patch -> partial ----------------
        // warp w reads lane quarter w % 4 (component w % 4, brick cell = lane); warps w and w + 4
        // take alternate 32-column blocks into their own patch, added when the brick is written
        const int quarter = warp & 3, half = warp >> 2;
        const int comp = quarter;
        const int cbase = (lane & 3) + C.pxp * (((lane >> 2) & 3) + C.pyp * (lane >> 4));
        float *patch = reinterpret_cast<float *>(sm + L.patch);
        const int *poff = reinterpret_cast<const int *>(sm + L.poff);
        float *mine = patch + (half * 3 + (comp < 3 ? comp : 0)) * C.pv + cbase;
        const int nv = D * C.pv;
        for (int it = 0;; ++it) {
            const long long tile = blockIdx.x + (long long)it * gridDim.x;
            if (tile >= ntiles) break;
            const int b = it & 1;
            // every epilogue warp leaves together (the named barriers below need all of them)
            const bool ok = __all_sync(0xffffffffu, tc::mbar_wait(&B.acc_full[b], (it >> 1) & 1, abort, C.wait_ns));
            if (tc::bar_or(kConEpiBar, kConEpiWarps * 32, !ok)) {
                if (!ok && lane == 0) tc_fail(abort, C.err);
                break;
            }
            tc::fence_after_sync();
            if (comp < D) {                                  // warp-uniform: tcgen05.ld is warp-wide
                const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * C.con_stride);
                for (int j = half; 32 * j < Np; j += kConEpiWarps / 4) {
                    float v[32];
                    if (32 * j + 32 <= Np) {
                        tc::tmem_ld32(tb + (uint32_t)(32 * j), v);
                    } else {
                        tc::tmem_ld16(tb + (uint32_t)(32 * j), v);
#pragma unroll
                        for (int e = 16; e < 32; ++e) v[e] = 0.f;
                    }
                    const int ne = C.nct - 32 * j;
#pragma unroll
                    for (int e = 0; e < 32; ++e) {
                        if (e < ne) mine[poff[32 * j + e]] += v[e];
                        __syncwarp();                        // tap e's adds before tap e + 1's
                    }
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&B.acc_empty[b]);                // the accumulator is read
            tc::bar_sync(kConEpiBar, kConEpiWarps * 32);     // both halves have scattered
            float *out = C.partial + tile * (long long)nv;
            for (int i = tid; i < nv; i += kConEpiWarps * 32) {
                const int cc = i / C.pv, pi = i - cc * C.pv;
                float *p0 = patch + cc * C.pv + pi, *p1 = patch + (3 + cc) * C.pv + pi;
                out[i] = *p0 + *p1;
                *p0 = 0.f;
                *p1 = 0.f;
            }
            tc::bar_sync(kConEpiBar, kConEpiWarps * 32);     // zeroed before the next brick's adds
        }
    } else {
        // ---------------- epilogue: TMEM -> Contrib ----------------
        // warp w reads TMEM lane quarter w % 4; warps w and w + 4 take alternate 16-column chunks
        const int quarter = warp & 3, half = warp >> 2;
        const int r = quarter * 32 + lane;
        const int comp = r / ct, c = r - comp * ct;
        const int ncell = (int)T.ncell;
        for (int it = 0;; ++it) {
            const long long tile = blockIdx.x + (long long)it * gridDim.x;
            if (tile >= ntiles) break;
            const int b = it & 1;
            // warp-uniform decision: tcgen05.ld below is a warp-wide instruction
            if (!__all_sync(0xffffffffu, tc::mbar_wait(&B.acc_full[b], (it >> 1) & 1, abort, C.wait_ns))) {
                if (lane == 0) tc_fail(abort, C.err);
                break;
            }
            tc::fence_after_sync();
            const int cell = (int)(tile * ct) + c;
            const bool valid = comp < D && cell < ncell;
            const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(b * C.con_stride);
            // 32-column blocks (one TMEM load and wait each), the two warps of a quarter alternating;
            // N is a multiple of 16, so the last block may hold 16 columns
            for (int j = half; 32 * j < Np; j += kConEpiWarps / 4) {
                float v[32];
                if (32 * j + 32 <= Np) {
                    tc::tmem_ld32(tb + (uint32_t)(32 * j), v);
                } else {
                    tc::tmem_ld16(tb + (uint32_t)(32 * j), v);
#pragma unroll
                    for (int e = 16; e < 32; ++e) v[e] = 0.f;
                }
                if (valid) {
                    float *dst = T.contrib + (comp * C.nct + 32 * j) * ncell + cell;
#pragma unroll
                    for (int e = 0; e < 32; ++e)
                        if (32 * j + e < C.nct) dst[e * ncell] = v[e];
                }
            }
            tc::fence_before_sync();
            tc::mbar_arrive(&B.acc_empty[b]);
        }
    }
    // the table copy lands before the CTA leaves (the MMA thread waited for it, or: no tile)
    if (tid == 0 && blockIdx.x >= ntiles) tc::mbar_wait(B.table, 0, abort);
    tc_teardown(B, tmem, (uint32_t)C.con_cols, kConMmaWarp);
}

// ------------------------------------------------------------------------------------------------
// host side

// tf32 part of x (round to nearest, ties away from zero, as cvt.rna.tf32.f32)
inline float tf32_hi_host(float x)
{
    uint32_t u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) == 0x7f800000u) return x;
    u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
}

inline uint32_t pow2_at_least(uint32_t v)
{
    uint32_t p = 32;
    while (p < v) p <<= 1;
    return p;
}

struct TcPlan {
    bool enabled = false;
    TcDev dev{};
    RegionPlanes rp{};               // weighted control-point planes (written by the packing kernels)
    CUtensorMap rmap{};              // tiled loads of a brick's region from rp
    CUtensorMap umap{};              // tiled stores of a tile's u (when dev.nus > 0)
    CUtensorMap recmap{}, fixmap{};  // contrib: tiled loads of a chunk's records and fixed values (dev.nrr > 0)
    float *d_btr = nullptr, *d_bcon = nullptr;
    int2 *d_pairoff = nullptr;
    int *d_ctap = nullptr;           // contrib tap k -> box tap
    unsigned *d_err = nullptr;
    int transform_blocks = 0, contrib_blocks = 0;
    size_t transform_smem = 0, contrib_smem = 0;
    WarpTmaPlan wt;                  // the warp kernel with TMA-staged coefficients (3-D)
    // contrib with brick partials (3-D): its tiled loads by bricks, the partials, the launch
    bool fused = false;              // planned
    bool fused_on = false;           // selected (skm_evaluator_path request 3 turns it on)
    CUtensorMap recmap5{}, fixmap4{};
    int *d_cpoff = nullptr;
    float *d_partial = nullptr;
    size_t contrib_smem_fused = 0;
    int contrib_blocks_fused = 0;
};

// Shared-memory wavefronts of the producers' region loads (4-byte loads of rows r = 32 q + lane,
// two per tap pair) for a staged box pitch: the distinct words on the busiest bank, averaged over
// the four x remainders of the region origin.  Host-side, to choose the box padding.
inline double region_bank_cost(const TcDev &C, int D, const std::vector<int> &pairs, const int *nt, int rxp, int ryp,
                               int rzb)
{
    const int rps = rxp * ryp * rzb, brick = C.bx * C.by * C.bz;
    int rowoff[128];
    long long total = 0;
    for (int r = 0; r < 128; ++r) {
        const int comp = r / C.ct, c = r % C.ct;
        const bool ex = comp < D && c < brick;
        rowoff[r] = ex ? comp * rps + c % C.bx + rxp * ((c / C.bx) % C.by + ryp * (c / (C.bx * C.by))) : 0;
    }
    for (int xs = 0; xs < 4; ++xs)
        for (int q = 0; q < 4; ++q)
            for (int t0 : pairs)
                for (int t1 = 0; t1 < 2; ++t1) {
                    const int tx = t0 % nt[0] + t1, ty = (t0 / nt[0]) % nt[1], tz = t0 / (nt[0] * nt[1]);
                    const int off = xs + tx + rxp * (ty + ryp * tz);
                    int w[32], cnt[32] = {0};
                    for (int l = 0; l < 32; ++l) w[l] = rowoff[32 * q + l] + off;
                    std::sort(w, w + 32);
                    for (int i = 0; i < 32; ++i)
                        if (i == 0 || w[i] != w[i - 1]) ++cnt[w[i] % 32];
                    total += *std::max_element(cnt, cnt + 32);
                }
    return (double)total / (16.0 * std::max<size_t>(1, pairs.size()));
}

// Decides whether the tensor-core kernels apply to a table plan and builds their operand
// tables.  ncp: control-point grid size per axis.  Returns 0 (tc.enabled says whether they
// apply) or 2 on a CUDA error.
inline int table_tc_plan(TcPlan &tc, TablePlan &pl, const int *ncp, cudaStream_t stream)
{
    tc.enabled = false;
    const TableDev &T = pl.dev;
    const std::vector<float> &tgemm = pl.h_tgemm;
    TcDev &C = tc.dev;
    C = TcDev{};
    if (T.D != 2 && T.D != 3) return 0;
    C.ct = kTcRows / T.D;
    C.ctc = T.D == 3 ? 32 : kTcRows / T.D;
    C.np = (T.nph + 15) / 16 * 16;
    // transform K axis: x-neighbouring tap pairs (the second tap of a row's last pair is virtual
    // when nt0 is odd), two pairs per 16-byte unit
    // taps whose table column is zero for every phase contribute nothing: both GEMMs skip them
    std::vector<char> nz((size_t)T.ntap, 0);
    for (int t = 0; t < T.ntap; ++t)
        for (int p = 0; p < T.nph && !nz[(size_t)t]; ++p) nz[(size_t)t] = tgemm[(size_t)p * T.ntap_pad + t] != 0.f;
    std::vector<int> ctap;                                   // contrib taps, box order
    for (int t = 0; t < T.ntap; ++t)
        if (nz[(size_t)t]) ctap.push_back(t);
    if (ctap.empty()) return 0;
    C.pairs_x = (T.nt[0] + 1) / 2;
    std::vector<int> pairs;                                  // box index of a pair's first tap
    for (int tz = 0; tz < T.nt[2]; ++tz)
        for (int ty = 0; ty < T.nt[1]; ++ty)
            for (int px = 0; px < C.pairs_x; ++px) {
                const int t0 = 2 * px + T.nt[0] * (ty + T.nt[1] * tz);
                const bool second = 2 * px + 1 < T.nt[0];
                if (nz[(size_t)t0] || (second && nz[(size_t)t0 + 1])) pairs.push_back(t0);
            }
    C.npairs = (int)pairs.size();
    C.kp = (4 * ((C.npairs + 1) / 2) + kTcKBlock - 1) / kTcKBlock * kTcKBlock;
    C.nct = (int)ctap.size();
    C.npc = (C.nct + 15) / 16 * 16;
    C.kpc = (T.nph + kTcKBlock - 1) / kTcKBlock * kTcKBlock;
    if (2 * C.np > 256 || C.npc > 256) return 0;
    const int xpad = 2 * C.pairs_x - T.nt[0];                    // virtual column of odd tap rows
    // brick of at most ct cells with the fewest tiles (then the smallest staged region), whose
    // transform layout fits the shared memory with two stages
    long long best_tiles = -1, best_rv = 0;
    for (int bz = 1; bz <= std::min(C.ct, T.nq[2]); ++bz)
        for (int by = 1; by <= std::min(C.ct / bz, T.nq[1]); ++by)
            for (int bx = 1; bx <= std::min(C.ct / (bz * by), T.nq[0]); ++bx) {
                const long long tiles = (long long)((T.nq[0] + bx - 1) / bx) * ((T.nq[1] + by - 1) / by) *
                                        ((T.nq[2] + bz - 1) / bz);
                const int rx = bx + T.nt[0] - 1 + xpad, ry = by + T.nt[1] - 1, rz = bz + T.nt[2] - 1;
                const long long rv = (long long)rx * ry * rz;
                if (rv > kTcMaxRegion) continue;
                TcDev probe = C;
                probe.rps = (rx + 3 + 3) / 4 * 4 * ry * rz;
                probe.rbuf = (T.D * probe.rps + 31) / 32 * 32;
                probe.nrb = 2;
                if ((size_t)TcTransformLayout(probe).total_bytes > kTcSmemMax) continue;
                if (best_tiles < 0 || tiles < best_tiles || (tiles == best_tiles && rv < best_rv)) {
                    best_tiles = tiles;
                    best_rv = rv;
                    C.bx = bx;
                    C.by = by;
                    C.bz = bz;
                }
            }
    if (best_tiles <= 0 || best_tiles > (1LL << 30)) return 0;
    C.tiles[0] = (T.nq[0] + C.bx - 1) / C.bx;
    C.tiles[1] = (T.nq[1] + C.by - 1) / C.by;
    C.tiles[2] = (T.nq[2] + C.bz - 1) / C.bz;
    C.rx = C.bx + T.nt[0] - 1 + xpad;
    C.ry = C.by + T.nt[1] - 1;
    C.rz = C.bz + T.nt[2] - 1;
    if (C.rx * C.ry * C.rz > kTcMaxRegion) return 0;
    // staged box: x covers the region from an origin rounded down to a multiple of 4; among the
    // paddings that fit with two buffers, the one with the fewest shared-memory wavefronts (then
    // the smallest); a third buffer when it fits too
    {
        const int rxp0 = (C.rx + 3 + 3) / 4 * 4;
        double best = -1.0;
        for (int rxp = rxp0; rxp <= rxp0 + 4; rxp += 4)
            for (int ryp = C.ry; ryp <= C.ry + 2; ++ryp)
                for (int rzb = C.rz; rzb <= C.rz + (T.D == 3 ? 1 : 0); ++rzb) {
                    if (rxp > 256 || ryp > 256 || rzb > 256) continue;
                    TcDev probe = C;
                    probe.rps = rxp * ryp * rzb;
                    probe.rbuf = (T.D * probe.rps + 31) / 32 * 32;
                    probe.nrb = 2;
                    if ((size_t)TcTransformLayout(probe).total_bytes > kTcSmemMax) continue;
                    const double cost = region_bank_cost(C, T.D, pairs, T.nt, rxp, ryp, rzb);
                    if (best < 0.0 || cost < best - 1e-9 || (cost < best + 1e-9 && probe.rps < C.rps)) {
                        best = cost;
                        C.rxp = rxp;
                        C.ryp = ryp;
                        C.rzb = rzb;
                        C.rps = probe.rps;
                        C.rbuf = probe.rbuf;
                    }
                }
        if (best < 0.0) return 0;
        // output staging: two buffers, else one, else none (direct stores); then a third region
        // buffer when it fits too.  The tiled store needs u's rows (nph floats) 16-byte aligned.
        C.nrb = 2;
        C.ustr = C.np + 4;
        C.ustage = (T.D * C.bx * C.by * C.bz * C.ustr + 31) / 32 * 32;
        C.nus = (T.nph % 4 == 0 && C.ustr <= 256) ? 2 : 0;
        while (C.nus > 0 && (size_t)TcTransformLayout(C).total_bytes > kTcSmemMax) --C.nus;
        C.nrb = kTcRegionBufs;
        if ((size_t)TcTransformLayout(C).total_bytes > kTcSmemMax) C.nrb = 2;
    }
    C.tr_stride = (int)pow2_at_least(2 * C.np);
    C.tr_abase = 2 * C.tr_stride;                            // then the A stages: 64 columns each
    C.tr_cols = 512;
    C.ns_tr = std::min(kTcStages, (C.tr_cols - C.tr_abase) / (2 * kTcKBlock));
    if (C.ns_tr < 2) return 0;
    C.con_stride = (int)pow2_at_least(C.npc);
    C.con_cols = 2 * C.con_stride;
    if (C.tr_cols > 512 || C.con_cols > 512) return 0;
    // contrib: two A stages and a ring of three (else two) record slots when they fit and the
    // records allow tiled loads (a chunk's 32 phases as four 128-byte rows per cell); else as many
    // stages (up to 3, at least 2) as the shared memory holds and direct record loads
    C.nrr = 0;
    C.rfix = (512 * C.ctc + 127) / 128 * 128;
    C.rslot = (C.rfix + 128 * C.ctc + 1023) / 1024 * 1024;
    if (T.nph % 8 == 0 && C.ctc <= 256) {
        C.ns_con = 2;
        for (C.nrr = 3; C.nrr >= 2 && (size_t)TcContribLayout(C, false).total_bytes > kTcSmemMax; --C.nrr) {
        }
        if (C.nrr < 2) C.nrr = 0;
    }
    if (C.nrr == 0)
        for (C.ns_con = 3; C.ns_con > 2 && (size_t)TcContribLayout(C, false).total_bytes > kTcSmemMax; --C.ns_con) {
        }
    tc.transform_smem = (size_t)TcTransformLayout(C).total_bytes;
    tc.contrib_smem = (size_t)TcContribLayout(C, false).total_bytes;
    // both kernels must hold one CTA per SM alone (their TMEM allocations assume it)
    if (tc.transform_smem > kTcSmemMax || tc.contrib_smem > kTcSmemMax) return 0;
    if (tc.transform_smem < kTcSmemMax / 2 + 1024) tc.transform_smem = kTcSmemMax / 2 + 1024;
    if (tc.contrib_smem < kTcSmemMax / 2 + 1024) tc.contrib_smem = kTcSmemMax / 2 + 1024;

    // B operands, K-major 128-byte swizzled (float index of element (row, k))
    auto kmaj = [](int row, int k, int rows) { return (size_t)tc::sw128_offset(row, k & ~3, rows) / 4 + (k & 3); };
    std::vector<float> btr((size_t)C.kp * 2 * C.np, 0.f);
    std::vector<float> bcon((size_t)2 * C.kpc * C.npc, 0.f);
    const size_t lo_off = (size_t)C.kpc * C.npc;
    for (int p = 0; p < T.nph; ++p)
        for (int k = 0; k < C.nct; ++k) {
            const float v = tgemm[(size_t)p * T.ntap_pad + ctap[(size_t)k]];
            const float hi = tf32_hi_host(v), lo = v - hi;
            bcon[kmaj(k, p, C.npc)] = hi;
            bcon[lo_off + kmaj(k, p, C.npc)] = lo;
        }
    // transform table in the pair order of the K axis: k = 4 u + j is tap t0 + (j & 1) of pair
    // 2 u + (j >> 1) (t0 its first box tap); virtual taps and padding stay zero
    std::vector<int2> pairoff((size_t)C.kp / 4, int2{0, 0});
    auto region_off = [&](int t) {
        return t % T.nt[0] + C.rxp * ((t / T.nt[0]) % T.nt[1] + C.ryp * (t / (T.nt[0] * T.nt[1])));
    };
    for (int u = 0; u < C.kp / 4; ++u) {
        pairoff[(size_t)u].x = 2 * u < C.npairs ? region_off(pairs[(size_t)(2 * u)]) : 0;
        pairoff[(size_t)u].y = 2 * u + 1 < C.npairs ? region_off(pairs[(size_t)(2 * u + 1)]) : 0;
    }
    for (int k = 0; k < C.kp; ++k) {
        const int pi = 2 * (k / 4) + ((k & 3) >> 1);
        if (pi >= C.npairs) continue;
        const int t0 = pairs[(size_t)pi];
        if (t0 % T.nt[0] + (k & 1) >= T.nt[0]) continue;
        const int t = t0 + (k & 1);
        for (int p = 0; p < T.nph; ++p) {
            const float v = tgemm[(size_t)p * T.ntap_pad + t];
            const float hi = tf32_hi_host(v), lo = v - hi;
            btr[kmaj(p, k, 2 * C.np)] = hi;
            btr[kmaj(C.np + p, k, 2 * C.np)] = lo;
        }
    }
    if (pool_malloc((void **)&tc.d_btr, btr.size() * sizeof(float)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&tc.d_bcon, bcon.size() * sizeof(float)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&tc.d_err, sizeof(unsigned)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&tc.d_pairoff, pairoff.size() * sizeof(int2)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&tc.d_ctap, ctap.size() * sizeof(int)) != cudaSuccess) return 2;
    if (cudaMemcpyAsync(tc.d_pairoff, pairoff.data(), pairoff.size() * sizeof(int2), cudaMemcpyHostToDevice,
                        stream) != cudaSuccess ||
        cudaMemcpyAsync(tc.d_ctap, ctap.data(), ctap.size() * sizeof(int), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess)
        return 2;
    if (cudaMemcpyAsync(tc.d_btr, btr.data(), btr.size() * sizeof(float), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaMemcpyAsync(tc.d_bcon, bcon.data(), bcon.size() * sizeof(float), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess ||
        cudaMemsetAsync(tc.d_err, 0, sizeof(unsigned), stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return 2;
    C.btr = tc.d_btr;
    C.bcon = tc.d_bcon;
    C.pairoff = tc.d_pairoff;
    C.err = tc.d_err;
    C.wait_ns = tc::kTcWaitNs;
    C.drill = 0;
    pl.dev.tc_err = tc.d_err;

    // weighted control-point planes and the tiled load of a brick's region from them
    {
        const int n0 = ncp[0], n1 = ncp[1], n2 = T.D == 3 ? ncp[2] : 1;
        const int nxp = (n0 + 3) / 4 * 4;
        const long long plane = (long long)nxp * n1 * n2;
        if (pool_malloc((void **)&tc.rp.p, sizeof(float) * T.D * plane) != cudaSuccess) return 2;
        if (cudaMemsetAsync(tc.rp.p, 0, sizeof(float) * T.D * plane, stream) != cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return 2;
        tc.rp.n0 = n0;
        tc.rp.nxp = nxp;
        tc.rp.D = T.D;
        tc.rp.plane = plane;
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult qr{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) != cudaSuccess || !fn ||
            qr != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return 0;
        }
        const cuuint64_t gdim[4] = {(cuuint64_t)nxp, (cuuint64_t)n1, (cuuint64_t)n2, (cuuint64_t)T.D};
        const cuuint64_t gstride[3] = {(cuuint64_t)nxp * 4, (cuuint64_t)nxp * n1 * 4, (cuuint64_t)plane * 4};
        const cuuint32_t bdim[4] = {(cuuint32_t)C.rxp, (cuuint32_t)C.ryp, (cuuint32_t)C.rzb, (cuuint32_t)T.D};
        const cuuint32_t estride[4] = {1, 1, 1, 1};
        if (reinterpret_cast<PfnTensorMapEncodeTiled>(fn)(
                &tc.rmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, tc.rp.p, gdim, gstride, bdim, estride,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
            return 0;
        // u as [D][nq2][nq1][nq0][nph]; the box's rows are ustr >= nph floats long, the columns
        // past nph (and cells past the grid) lie outside the tensor and are not stored
        if (C.nus > 0) {
            const cuuint64_t ud[5] = {(cuuint64_t)T.nph, (cuuint64_t)T.nq[0], (cuuint64_t)T.nq[1], (cuuint64_t)T.nq[2],
                                      (cuuint64_t)T.D};
            const cuuint64_t us[4] = {(cuuint64_t)T.nph * 4, (cuuint64_t)T.nph * T.nq[0] * 4,
                                      (cuuint64_t)T.nph * T.nq[0] * T.nq[1] * 4, (cuuint64_t)T.ncell * T.nph * 4};
            const cuuint32_t ub[5] = {(cuuint32_t)C.ustr, (cuuint32_t)C.bx, (cuuint32_t)C.by, (cuuint32_t)C.bz,
                                      (cuuint32_t)T.D};
            const cuuint32_t ue[5] = {1, 1, 1, 1, 1};
            if (reinterpret_cast<PfnTensorMapEncodeTiled>(fn)(
                    &tc.umap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, T.ucp, ud, us, ub, ue, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                C.nus = 0;                                   // direct stores
        }
        // contrib's records as [cell][nph / 8][32 floats] (128-byte rows, swizzled in shared
        // memory) and fixed values as [cell][nph]; a failed encoding keeps the direct loads
        if (C.nrr > 0) {
            const cuuint64_t rd[3] = {32, (cuuint64_t)(T.nph / 8), (cuuint64_t)T.ncell};
            const cuuint64_t rs[2] = {128, (cuuint64_t)T.nph * 16};
            const cuuint32_t rb[3] = {32, 4, (cuuint32_t)C.ctc};
            const cuuint64_t fd[2] = {(cuuint64_t)T.nph, (cuuint64_t)T.ncell};
            const cuuint64_t fs[1] = {(cuuint64_t)T.nph * 4};
            const cuuint32_t fb[2] = {(cuuint32_t)kTcKBlock, (cuuint32_t)C.ctc};
            const cuuint32_t e1[3] = {1, 1, 1};
            auto enc = reinterpret_cast<PfnTensorMapEncodeTiled>(fn);
            if (enc(&tc.recmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, (void *)T.rec, rd, rs, rb, e1,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
                enc(&tc.fixmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void *)T.fixcp, fd, fs, fb, e1,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS) {
                C.nrr = 0;
                for (C.ns_con = 3; C.ns_con > 2 && (size_t)TcContribLayout(C, false).total_bytes > kTcSmemMax; --C.ns_con) {
                }
            }
        }
    }

    // brick partials (3-D, tiled record loads, a brick of 32 cells = one lane quarter): records as
    // [cell z][cell y][cell x][nph / 8][32 floats] and fixed values as [z][y][x][nph], boxes of one
    // brick; the patches of both epilogue halves and the taps' patch offsets in shared memory
    if (C.nrr > 0 && T.D == 3 && C.ctc == kBrickX * kBrickY * kBrickZ) {
        const int bdim[3] = {kBrickX, kBrickY, kBrickZ};
        for (int d = 0; d < 3; ++d) C.nbrick[d] = (T.nq[d] + bdim[d] - 1) / bdim[d];
        C.pxp = kBrickX + T.nt[0] - 1;
        C.pyp = kBrickY + T.nt[1] - 1;
        C.pzp = kBrickZ + T.nt[2] - 1;
        C.pv = C.pxp * C.pyp * C.pzp;
        const size_t fsmem = (size_t)TcContribLayout(C, true).total_bytes;
        void *fn = nullptr;
        cudaDriverEntryPointQueryResult qr{};
        bool ok = fsmem <= kTcSmemMax &&
                  cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &qr) == cudaSuccess && fn &&
                  qr == cudaDriverEntryPointSuccess;
        if (!ok) cudaGetLastError();
        if (ok) {
            const cuuint64_t row = (cuuint64_t)T.nph * 16, frow = (cuuint64_t)T.nph * 4;
            const cuuint64_t rd[5] = {32, (cuuint64_t)(T.nph / 8), (cuuint64_t)T.nq[0], (cuuint64_t)T.nq[1],
                                      (cuuint64_t)T.nq[2]};
            const cuuint64_t rs[4] = {128, row, row * T.nq[0], row * T.nq[0] * T.nq[1]};
            const cuuint32_t rb[5] = {32, 4, kBrickX, kBrickY, kBrickZ};
            const cuuint64_t fd[4] = {(cuuint64_t)T.nph, (cuuint64_t)T.nq[0], (cuuint64_t)T.nq[1], (cuuint64_t)T.nq[2]};
            const cuuint64_t fs[3] = {frow, frow * T.nq[0], frow * T.nq[0] * T.nq[1]};
            const cuuint32_t fb[4] = {(cuuint32_t)kTcKBlock, kBrickX, kBrickY, kBrickZ};
            const cuuint32_t e1[5] = {1, 1, 1, 1, 1};
            auto enc = reinterpret_cast<PfnTensorMapEncodeTiled>(fn);
            ok = enc(&tc.recmap5, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 5, (void *)T.rec, rd, rs, rb, e1,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS &&
                 enc(&tc.fixmap4, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)T.fixcp, fd, fs, fb, e1,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
        }
        if (ok) {
            std::vector<int> cpoff((size_t)C.nct);
            for (int k = 0; k < C.nct; ++k) {
                const int i = ctap[(size_t)k];
                cpoff[(size_t)k] = i % T.nt[0] + C.pxp * ((i / T.nt[0]) % T.nt[1] + C.pyp * (i / (T.nt[0] * T.nt[1])));
            }
            const long long nbr = (long long)C.nbrick[0] * C.nbrick[1] * C.nbrick[2];
            if (pool_malloc((void **)&tc.d_cpoff, cpoff.size() * sizeof(int)) != cudaSuccess ||
                pool_malloc((void **)&tc.d_partial, (size_t)nbr * T.D * C.pv * sizeof(float)) != cudaSuccess ||
                cudaMemcpyAsync(tc.d_cpoff, cpoff.data(), cpoff.size() * sizeof(int), cudaMemcpyHostToDevice, stream) !=
                    cudaSuccess ||
                cudaStreamSynchronize(stream) != cudaSuccess)
                return 2;
            C.cpoff = tc.d_cpoff;
            C.partial = tc.d_partial;
            tc.contrib_smem_fused = std::max(fsmem, kTcSmemMax / 2 + 1024);
            tc.fused = true;
        }
    }

    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 2;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 2;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (cudaFuncSetAttribute(table_transform_tc_kernel, a, (int)tc.transform_smem) != cudaSuccess) return 2;
    if (cudaFuncSetAttribute(table_contrib_tc_kernel<false>, a, (int)tc.contrib_smem) != cudaSuccess) return 2;
    if (tc.fused) {
        int occ_f = 0;
        if (cudaFuncSetAttribute(table_contrib_tc_kernel<true>, a, (int)tc.contrib_smem_fused) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_f, table_contrib_tc_kernel<true>, kConThreads,
                                                          tc.contrib_smem_fused) != cudaSuccess)
            return 2;
        const long long nbr = (long long)C.nbrick[0] * C.nbrick[1] * C.nbrick[2];
        tc.contrib_blocks_fused = (int)std::max<long long>(1, std::min<long long>(nbr, sms));
        if (occ_f < 1) tc.fused = false;
    }
    // both kernels must be launchable with their block sizes and shared memory (else: CUDA cores)
    int occ_t = 0, occ_c = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_t, table_transform_tc_kernel, kTcThreads,
                                                      tc.transform_smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ_c, table_contrib_tc_kernel<false>, kConThreads,
                                                      tc.contrib_smem) != cudaSuccess)
        return 2;
    if (occ_t < 1 || occ_c < 1) return 0;
    const long long ttiles = (long long)C.tiles[0] * C.tiles[1] * C.tiles[2];
    const long long ctiles = (T.ncell + C.ctc - 1) / C.ctc;
    tc.transform_blocks = (int)std::max<long long>(1, std::min<long long>(ttiles, sms));
    tc.contrib_blocks = (int)std::max<long long>(1, std::min<long long>(ctiles, sms));
    tc.enabled = true;
    return 0;
}

inline int table_transform_tc(const TcPlan &tc, const TablePlan &pl, const EvalParams &P, cudaStream_t s)
{
    table_transform_tc_kernel<<<tc.transform_blocks, kTcThreads, tc.transform_smem, s>>>(P, pl.dev, tc.dev, tc.rmap,
                                                                                         tc.umap);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

inline bool tc_bricks(const TcPlan &tc) { return tc.fused && tc.fused_on; }

inline int table_contrib_tc(const TcPlan &tc, const TablePlan &pl, const double *stats, cudaStream_t s)
{
    if (tc_bricks(tc))
        table_contrib_tc_kernel<true><<<tc.contrib_blocks_fused, kConThreads, tc.contrib_smem_fused, s>>>(
            pl.dev, tc.dev, stats, tc.recmap5, tc.fixmap4);
    else
        table_contrib_tc_kernel<false><<<tc.contrib_blocks, kConThreads, tc.contrib_smem, s>>>(pl.dev, tc.dev, stats,
                                                                                              tc.recmap, tc.fixmap);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

// ------------------------------------------------------------------------------------------------
// launch sequences of the table path (tc: tensor-core GEMMs, or NULL for the CUDA-core ones)

template <int HL, int NCZ>
inline int table_transform_launch(TablePlan &pl, const EvalParams &P, cudaStream_t s)
{
    table_transform_kernel<HL, NCZ><<<pl.transform_blocks, 256, table_value_smem(pl), s>>>(P, pl.dev);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

// value pass of the table path: transform, then warp + statistics; writes its own partials
// (pl.d_part, pl.dev.value_blocks blocks)
inline int table_value(TablePlan &pl, const TcPlan *tc, const EvalParams &P, int D, int metric, double *stats,
                       unsigned *counter, cudaStream_t s, cudaEvent_t mid = nullptr)
{
    int rc;
    if (tc && tc->enabled) {
        rc = table_transform_tc(*tc, pl, P, s);
    } else if (pl.big) {                                     // coarse levels: tables in global memory
        const size_t smem = table_big_transform_smem(pl.dev);
        const int nb = pl.transform_blocks;
        if (D == 3) {
            if (pl.big_pb == 4) table_transform_big_kernel<3, 4><<<nb, 256, smem, s>>>(P, pl.dev);
            else if (pl.big_pb == 2) table_transform_big_kernel<3, 2><<<nb, 256, smem, s>>>(P, pl.dev);
            else table_transform_big_kernel<3, 1><<<nb, 256, smem, s>>>(P, pl.dev);
        } else {
            if (pl.big_pb == 4) table_transform_big_kernel<2, 4><<<nb, 256, smem, s>>>(P, pl.dev);
            else if (pl.big_pb == 2) table_transform_big_kernel<2, 2><<<nb, 256, smem, s>>>(P, pl.dev);
            else table_transform_big_kernel<2, 1><<<nb, 256, smem, s>>>(P, pl.dev);
        }
        rc = cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
    } else if (D == 3) {
        switch (pl.hl) {
        case 1: rc = table_transform_launch<1, 4>(pl, P, s); break;
        case 2: rc = table_transform_launch<2, 4>(pl, P, s); break;
        case 4: rc = table_transform_launch<4, 4>(pl, P, s); break;
        default: rc = table_transform_launch<8, 4>(pl, P, s); break;
        }
    } else {
        rc = table_transform_launch<1, 1>(pl, P, s);
    }
    if (rc) return rc;
    if (mid && cudaEventRecord(mid, s) != cudaSuccess) return 2;
    if (D == 3 && tc && tc->enabled && tc->wt.enabled)
        table_warp_tma_kernel<<<tc->wt.blocks, 256, tc->wt.smem, s>>>(P, pl.dev, tc->wt.dev, tc->wt.map, metric, stats,
                                                                     counter);
    else if (D == 3)
        table_warp_kernel<3><<<pl.dev.value_blocks, 256, 0, s>>>(P, pl.dev, metric, stats, counter);
    else
        table_warp_kernel<2><<<pl.dev.value_blocks, 256, 0, s>>>(P, pl.dev, metric, stats, counter);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

inline int table_derivative(TablePlan &pl, const TcPlan *tc, const EvalParams &P, const DerivParams &Q, int D,
                            int gather_blocks, cudaStream_t s, cudaEvent_t mid = nullptr)
{
    TableDev G = pl.dev;                                     // the gather reads the contrib layout
    const bool bricks = tc && tc->enabled && tc_bricks(*tc);
    if (tc && tc->enabled) {
        if (table_contrib_tc(*tc, pl, Q.stats, s)) return 2;
        G.gtap = tc->d_ctap;                                 // nonzero taps only
        G.ngtap = tc->dev.nct;
        if (bricks) {
            const TcDev &C = tc->dev;
            G.bp.partial = C.partial;
            G.bp.b[0] = kBrickX;
            G.bp.b[1] = kBrickY;
            G.bp.b[2] = kBrickZ;
            for (int d = 0; d < 3; ++d) G.bp.nb[d] = C.nbrick[d];
            G.bp.px = C.pxp;
            G.bp.py = C.pyp;
            G.bp.pv = C.pv;
        }
    } else if (pl.big) {
        table_contrib_big_kernel<<<pl.contrib_blocks, 256, 0, s>>>(pl.dev, Q.stats);
        if (pl.dev.big_splits > 1) table_contrib_big_reduce<<<592, 256, 0, s>>>(pl.dev);
        if (cudaPeekAtLastError() != cudaSuccess) return 2;
    } else {
        const size_t smem = table_contrib_smem(pl.dev);
        table_contrib_kernel<<<pl.contrib_blocks, kTabContribThreads, smem, s>>>(pl.dev, Q.stats);
        if (cudaPeekAtLastError() != cudaSuccess) return 2;
    }
    if (mid && cudaEventRecord(mid, s) != cudaSuccess) return 2;
    if (D == 3 && bricks)
        table_gather_kernel<3, true><<<gather_blocks, kGatherThreads, 0, s>>>(P, G, Q);
    else if (D == 3)
        table_gather_launch<3>(P, G, Q, gather_blocks, s);
    else
        table_gather_launch<2>(P, G, Q, gather_blocks, s);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

inline int table_derivative_gather_only(TablePlan &pl, const EvalParams &P, const DerivParams &Q, int D,
                                        int gather_blocks, cudaStream_t s)
{
    if (D == 3)
        table_gather_launch<3>(P, pl.dev, Q, gather_blocks, s);
    else
        table_gather_launch<2>(P, pl.dev, Q, gather_blocks, s);
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 2;
}

inline void table_tc_free(TcPlan &tc)
{
    if (tc.d_btr) pool_release(tc.d_btr);
    if (tc.d_bcon) pool_release(tc.d_bcon);
    if (tc.d_err) pool_release(tc.d_err);
    if (tc.d_pairoff) pool_release(tc.d_pairoff);
    if (tc.rp.p) pool_release(tc.rp.p);
    warp_tma_free(tc.wt);
    if (tc.d_ctap) pool_release(tc.d_ctap);
    if (tc.d_cpoff) pool_release(tc.d_cpoff);
    if (tc.d_partial) pool_release(tc.d_partial);
    tc = TcPlan{};
}

}  // namespace skm
