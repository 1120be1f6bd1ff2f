// skm_warp_tma.cuh -- the table path's warp kernel with the moving image's coefficients staged in
// shared memory by TMA (3-D, volumes).
//
// Same work and the same arithmetic as table_warp_kernel<3> (B-spline value and gradient of the
// moving image at x + u(x), NCC/MSE statistics, the (grad M, m) record per texel), reorganised
// for locality: a CTA takes a brick of cells (up to 64 cells, 256 texels per pass) and
// first loads the coefficient box that the brick's stencils can reach -- the brick's extent in
// moving-image index space plus kWtMargin voxels of displacement on every side -- with one
// cp.async.bulk.tensor.3d load (no multicast) into one of two buffers, so the next brick's load
// runs while this one is evaluated.  The two buffers form a full/empty mbarrier pipeline with no
// block-wide barrier per brick: a warp starts its next brick once that brick's box has landed, and
// the next load into a buffer is issued once every warp has released it.  A texel whose stencil
// leaves the box (displacement beyond the margin) reads the global row-expanded copy instead, so
// results do not depend on the margin.  The stencil sums run on packed FP32 pairs
// (bspline_sum3_x2).  Each mbarrier wait is bounded; a wait that gives up sets the evaluator's
// sticky fault word (the result then reports SKM_ERR_TIMEOUT) and the warp skips its later bricks.
#pragma once

#include <cuda.h>

namespace skm {

constexpr int kWtBoxX = 28, kWtBoxY = 17, kWtBoxZ = 17;          // staged box (floats), x multiple of 4
constexpr int kWtMargin = 3;                                     // voxels of displacement inside the box
constexpr int kWtBoxFloats = kWtBoxX * kWtBoxY * kWtBoxZ;
constexpr int kWtBufFloats = (kWtBoxFloats + 31) / 32 * 32;      // 128-byte aligned buffers
constexpr uint32_t kWtBoxBytes = kWtBoxFloats * 4;
constexpr int kWtMaxCells = 64;                                  // cells per brick
constexpr int kWtMaxPhase = 512;                                 // phases (the table path allows 8^3)

struct WarpTma {
    int bc[3];               // brick in cells
    int nb[3];               // bricks per axis
    double a[3], b[3];       // moving-image index of fixed voxel x: a x + b (no displacement)
    int xlo[3];              // lowest voxel offset of a cell's texels: x = h q + xlo .. h q + xlo + h - 1
    int lanes4x8;            // h = 4 and a 4 x 2 x 2-cell brick: a warp takes 4 x 8 voxels of one z
};

__device__ __forceinline__ void tma_load_3d(float *dst, const CUtensorMap *map, int x, int y, int z,
                                            uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        :: "r"(tc::smem_addr(dst)), "l"(map), "r"(x), "r"(y), "r"(z), "r"(tc::smem_addr(bar)) : "memory");
}

__global__ void __launch_bounds__(256, 3) table_warp_tma_kernel(EvalParams P, TableDev T, WarpTma W,
                                                                const __grid_constant__ CUtensorMap map,
                                                                int metric, double *stats, unsigned *counter)
{
    constexpr int D = 3;
    extern __shared__ float4 wt_smem4[];
    // [2][kWtBufFloats] boxes (128-byte aligned for the TMA), then phx[nph] (voxel offset of phase
    // p: x = h q + phx[p]) and cellxyz[cells of a brick]
    unsigned char *wsm = reinterpret_cast<unsigned char *>(wt_smem4);
    wsm += (128u - (tc::smem_addr(wsm) & 127u)) & 127u;
    float *wbuf = reinterpret_cast<float *>(wsm);
    int4 *phx = reinterpret_cast<int4 *>(wbuf + 2 * kWtBufFloats);
    int4 *cellxyz = phx + T.nph;
    // full[b]: the box of buffer b has landed (TMA transaction count); empty[b]: every warp is done
    // reading buffer b (one arrival per warp), so the next load may overwrite it
    __shared__ __align__(8) uint64_t full[2], empty[2];
    __shared__ int r0s[2][3];                                       // box origin of each buffer
    __shared__ double sh[NQ * 32];
    const int tid = threadIdx.x, lane = tid & 31;
    const int nph = T.nph;
    const int ncb = W.bc[0] * W.bc[1] * W.bc[2];
    const int nbr = W.nb[0] * W.nb[1] * W.nb[2];
    if (tid == 0) {
        tc::mbar_init(&full[0], 1);
        tc::mbar_init(&full[1], 1);
        tc::mbar_init(&empty[0], blockDim.x / 32);
        tc::mbar_init(&empty[1], blockDim.x / 32);
        tc::fence_mbarrier_init();
    }
    for (int c = tid; c < ncb; c += blockDim.x)
        cellxyz[c] = make_int4(c % W.bc[0], (c / W.bc[0]) % W.bc[1], c / (W.bc[0] * W.bc[1]), 0);
    for (int p = tid; p < nph; p += blockDim.x) {
        const int pyz = p / T.h[0], pz = pyz / T.h[1];
        const int ph[3] = {p - pyz * T.h[0], pyz - pz * T.h[1], pz};
        int xo[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) xo[d] = T.h[d] * (T.qmin[d] - T.qoff[d][ph[d]]) + ph[d];
        phx[p] = make_int4(xo[0], xo[1], xo[2], 0);
    }
    __syncthreads();

    // box origin of a brick: its lowest texel mapped to moving-image index space, minus the
    // margin (x rounded down to 4 floats, the TMA alignment of the innermost coordinate)
    auto issue = [&](int brick, int buf) {
        const int bq[3] = {brick % W.nb[0], (brick / W.nb[0]) % W.nb[1], brick / (W.nb[0] * W.nb[1])};
        int r0[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int x = T.h[d] * (T.qmin[d] + bq[d] * W.bc[d]) + W.xlo[d];
            r0[d] = (int)floor(W.a[d] * x + W.b[d]) - kWtMargin;
        }
        r0[0] = (r0[0] >= 0) ? (r0[0] & ~3) : -((-r0[0] + 3) & ~3);
        r0s[buf][0] = r0[0];
        r0s[buf][1] = r0[1];
        r0s[buf][2] = r0[2];
        tc::mbar_expect_tx(&full[buf], kWtBoxBytes);               // arrival (release): r0s visible
        tma_load_3d(wbuf + buf * kWtBufFloats, &map, r0[0], r0[1], r0[2], &full[buf]);
    };

    float vf[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) vf[k] = 0.f;
    const int fn[3] = {P.fixed.n[0], P.fixed.n[1], P.fixed.n[2]};
    const int plane = (int)(T.ncell * T.nph);
    // Thread 0 issues the loads: brick it + 1 into buffer (it + 1) & 1 once every warp has released
    // that buffer (brick it - 1).  No block-wide barrier inside the loop: a warp moves on to its next
    // brick as soon as that brick's box has landed, whatever the other warps are doing.  Every wait
    // is bounded; a thread whose wait gives up records the fault and stops working (its warp's later
    // bricks are skipped, the result reports SKM_ERR_TIMEOUT).
    int issued = 0, waited0 = 0;                                    // thread 0's load bookkeeping
    if (tid == 0 && (int)blockIdx.x < nbr) {
        issue(blockIdx.x, 0);
        issued = 1;
    }
    int it = 0;
    for (int brick = blockIdx.x; brick < nbr; brick += gridDim.x, ++it) {
        const int buf = it & 1;
        const int next = brick + gridDim.x;
        bool ok = true;
        if (tid == 0 && next < nbr) {
            // buffer buf ^ 1 held brick it - 1 (use (it - 1) >> 1 of that buffer); warp 0's own
            // arrival for it came at the end of the previous iteration
            if (it == 0 || tc::mbar_wait(&empty[buf ^ 1], (uint32_t)(((it - 1) >> 1) & 1))) {
                issue(next, buf ^ 1);
                ++issued;
            } else {
                ok = false;
            }
        }
        if (ok) ok = tc::mbar_wait(&full[buf], (uint32_t)((it >> 1) & 1));
        if (tid == 0 && ok) ++waited0;
        // the decision to stop is the warp's (its lanes then leave the loop together)
        if (__any_sync(0xffffffffu, !ok)) {
            if (lane == 0 && T.tc_err) atomicOr(T.tc_err, 2u);
            break;
        }
        {
            const float *box = wbuf + buf * kWtBufFloats;
            const int r0[3] = {r0s[buf][0], r0s[buf][1], r0s[buf][2]};
            const int bq[3] = {brick % W.nb[0], (brick / W.nb[0]) % W.nb[1], brick / (W.nb[0] * W.nb[1])};
            for (int t = tid; t < ncb * nph; t += blockDim.x) {
                int cl, p;
                if (W.lanes4x8) {
                    // lanes = 4 x-neighbours x 8 y-neighbours of one z: with the box's row stride of
                    // 28 floats (-4 modulo 32 banks) a stencil tap of the warp hits 32 distinct banks
                    const int w = t >> 5;
                    const int xi = lane & 3, yi = lane >> 2, cx = w & 3, vz = w >> 2;
                    cl = cx + 4 * ((yi >> 2) + 2 * (vz >> 2));
                    p = xi + 4 * (yi & 3) + 16 * (vz & 3);
                } else {
                    cl = (int)T.div_nph.div((uint32_t)t);
                    p = t - cl * nph;
                }
                const int4 cxyz = cellxyz[cl];
                const int cc[3] = {bq[0] * W.bc[0] + cxyz.x, bq[1] * W.bc[1] + cxyz.y, bq[2] * W.bc[2] + cxyz.z};
                if (cc[0] >= T.nq[0] || cc[1] >= T.nq[1] || cc[2] >= T.nq[2]) continue;
                const int cell = cc[0] + T.nq[0] * (cc[1] + T.nq[1] * cc[2]);
                const int i = cell * nph + p;
                const int4 xo = phx[p];
                const int x[3] = {T.h[0] * cc[0] + xo.x, T.h[1] * cc[1] + xo.y, T.h[2] * cc[2] + xo.z};
                float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
                if (x[0] >= 0 && x[0] < fn[0] && x[1] >= 0 && x[1] < fn[1] && x[2] >= 0 && x[2] < fn[2]) {
                    const float u[3] = {T.ucp[i], T.ucp[i + plane], T.ucp[i + 2 * plane]};
                    const float f = T.fixcp[i];
                    double fi[3] = {(double)x[0], (double)x[1], (double)x[2]}, pp[3], mp[3], ml[3];
                    to_global<D>(P.fixed, fi, pp);
#pragma unroll
                    for (int d = 0; d < D; ++d) mp[d] = pp[d];
                    if (P.has_df) {
                        const long long di = nearest_index<D>(P.df, pp);
                        if (di >= 0) {
                            const float4 dv = P.dfd[di];
                            mp[0] += dv.x;
                            mp[1] += dv.y;
                            mp[2] += dv.z;
                        }
                    }
                    mp[0] += (double)u[0];
                    mp[1] += (double)u[1];
                    mp[2] += (double)u[2];
                    to_local<D>(P.mov, mp, ml);
                    if (bspline_inside<D>(P.mov, ml)) {
                        float m, g[3];
                        int ii[3];
                        float Wt[4][3], dW[4][3];
                        bspline_weights<D>(ml, ii, Wt, dW);
                        const int j0 = ii[0] - r0[0], j1 = ii[1] - r0[1], j2 = ii[2] - r0[2];
                        if (j0 >= 0 && j0 + 4 <= kWtBoxX && j1 >= 0 && j1 + 4 <= kWtBoxY && j2 >= 0 &&
                            j2 + 4 <= kWtBoxZ) {
                            const float *bb = box + j0 + kWtBoxX * (j1 + kWtBoxY * j2);
                            bspline_sum3_x2(
                                [&](int y, int z) {
                                    const float *rr = bb + kWtBoxX * (y + kWtBoxY * z);
                                    return make_float4(rr[0], rr[1], rr[2], rr[3]);
                                },
                                Wt, dW, P.mov, m, g);
                        } else {                                    // beyond the margin: global rows
                            const int sy = (int)P.mov.st[1], sz = (int)P.mov.st[2];
                            const float4 *base = P.coeffs4 + (ii[0] + ii[1] * sy + ii[2] * sz);
                            bspline_sum3_x2([&](int y, int z) { return __ldg(base + (y * sy + z * sz)); }, Wt,
                                            dW, P.mov, m, g);
                        }
                        vf[Q_COUNT] += 1.f;
                        vf[Q_D2] += (m - f) * (m - f);
                        vf[Q_SF] += f;
                        vf[Q_SM] += m;
                        vf[Q_SFF] += f * f;
                        vf[Q_SMM] += m * m;
                        vf[Q_SFM] += f * m;
                        rec = make_float4(g[0], g[1], g[2], m);
                    }
                }
                T.rec[i] = rec;
            }
        }
        __syncwarp();
        if (lane == 0) tc::mbar_arrive(&empty[buf]);                // this warp is done with buffer buf
    }
    // every issued load must land before the CTA leaves (after a failure some were never waited
    // for): thread 0 waits for the rest, bounded
    if (tid == 0)
        for (; waited0 < issued; ++waited0)
            if (!tc::mbar_wait(&full[waited0 & 1], (uint32_t)((waited0 >> 1) & 1))) break;
    __syncthreads();
    double v[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = (double)vf[k];
    block_sum<NQ>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) T.part[(long long)k * gridDim.x + blockIdx.x] = v[k];
    if (last_block_arrived(counter)) {                     // fused statistics, fixed order
        double w[NQ];
        sum_partials<NQ>(T.part, gridDim.x, w, sh);
        if (threadIdx.x == 0) stats_finalize(w, metric, stats);
    }
}

// ------------------------------------------------------------------------------------------------
// host side

struct WarpTmaPlan {
    bool enabled = false;
    WarpTma dev{};
    CUtensorMap map{};
    float *d_coefp = nullptr;        // coefficients with rows padded to a multiple of 4 floats
    int blocks = 0;
    size_t smem = 0;
};

typedef CUresult (*PfnTensorMapEncodeTiled)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                            const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                            const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                            CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// Plans the staged warp kernel for a 3-D table plan whose operands allow it; returns 0
// (wt.enabled says whether it applies) or 2 on a CUDA error.  d_coeffs: the padded coefficient
// volume (float, moving size + 3 per axis) on the device.
inline int warp_tma_plan(WarpTmaPlan &wt, const TablePlan &pl, const EvalParams &P, const float *d_coeffs,
                         cudaStream_t stream)
{
    wt.enabled = false;
    const TableDev &T = pl.dev;
    if (T.D != 3 || !T.tc_err || T.nph > kWtMaxPhase) return 0;
    WarpTma &W = wt.dev;
    // moving index of fixed voxel x (no displacement): (fo + fs x - mo) / ms
    for (int d = 0; d < 3; ++d) {
        W.a[d] = P.fixed.s[d] * P.mov.inv[d];
        W.b[d] = (P.fixed.o[d] - P.mov.o[d]) * P.mov.inv[d];
        if (!(W.a[d] > 0.0) || W.a[d] > 4.0) return 0;
        int lo = 1 << 30;
        for (int ph = 0; ph < T.h[d]; ++ph) lo = std::min(lo, ph - T.h[d] * T.qoff[d][ph]);
        int hi = -(1 << 30);
        for (int ph = 0; ph < T.h[d]; ++ph) hi = std::max(hi, ph - T.h[d] * T.qoff[d][ph]);
        if (hi - lo != T.h[d] - 1) return 0;                  // a cell's texels form one run per axis
        W.xlo[d] = lo;
    }
    // the largest brick (cells per axis) whose box holds its stencils with the margin
    const int box[3] = {kWtBoxX - 3, kWtBoxY, kWtBoxZ};       // x: the origin rounds down by up to 3
    for (int d = 0; d < 3; ++d) {
        int bc = 0;
        for (int c = 1; c <= T.nq[d]; ++c) {
            const double span = W.a[d] * (T.h[d] * c - 1);
            if ((int)ceil(span) + 1 + 2 * kWtMargin + 3 <= box[d]) bc = c;
        }
        if (bc < 1) return 0;
        W.bc[d] = bc;
    }
    while (W.bc[0] * W.bc[1] * W.bc[2] > kWtMaxCells) {
        if (W.bc[0] >= W.bc[1] && W.bc[0] >= W.bc[2]) --W.bc[0];
        else if (W.bc[1] >= W.bc[2]) --W.bc[1];
        else --W.bc[2];
    }
    for (int d = 0; d < 3; ++d) W.nb[d] = (T.nq[d] + W.bc[d] - 1) / W.bc[d];
    static_assert(kWtBoxX % 32 == 28, "the 4 x 8 lane layout relies on a row stride of -4 banks");
    W.lanes4x8 = T.h[0] == 4 && T.h[1] == 4 && T.h[2] == 4 && W.bc[0] == 4 && W.bc[1] == 2 && W.bc[2] == 2;
    const long long nbr = (long long)W.nb[0] * W.nb[1] * W.nb[2];

    // tensor map over a row-pitched copy (global strides must be multiples of 16 bytes)
    const int PX = P.mov.n[0], PY = P.mov.n[1], PZ = P.mov.n[2];
    const int pitch = (PX + 3) / 4 * 4;
    const size_t npad = (size_t)pitch * PY * PZ;
    if (pool_malloc((void **)&wt.d_coefp, npad * sizeof(float)) != cudaSuccess) return 2;
    if (cudaMemsetAsync(wt.d_coefp, 0, npad * sizeof(float), stream) != cudaSuccess ||
        cudaMemcpy2DAsync(wt.d_coefp, (size_t)pitch * 4, d_coeffs, (size_t)PX * 4, (size_t)PX * 4, (size_t)PY * PZ,
                          cudaMemcpyDeviceToDevice, stream) != cudaSuccess ||
        cudaStreamSynchronize(stream) != cudaSuccess)
        return 2;
    void *fn = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess || !fn ||
        q != cudaDriverEntryPointSuccess) {
        cudaGetLastError();
        return 0;
    }
    const cuuint64_t gdim[3] = {(cuuint64_t)PX, (cuuint64_t)PY, (cuuint64_t)PZ};
    const cuuint64_t gstride[2] = {(cuuint64_t)pitch * 4, (cuuint64_t)pitch * PY * 4};
    const cuuint32_t bdim[3] = {kWtBoxX, kWtBoxY, kWtBoxZ};
    const cuuint32_t estride[3] = {1, 1, 1};
    if (reinterpret_cast<PfnTensorMapEncodeTiled>(fn)(
            &wt.map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, wt.d_coefp, gdim, gstride, bdim, estride,
            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
            CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return 0;
    wt.smem = (size_t)2 * kWtBufFloats * sizeof(float) + 128 +
              sizeof(int4) * (size_t)(T.nph + W.bc[0] * W.bc[1] * W.bc[2]);
    if (cudaFuncSetAttribute(table_warp_tma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)wt.smem) !=
        cudaSuccess)
        return 2;
    int occ = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, table_warp_tma_kernel, 256, wt.smem) != cudaSuccess)
        return 2;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 2;
    if (occ < 1) return 0;
    // the statistics partials are sized for value_blocks
    wt.blocks = (int)std::max<long long>(1, std::min<long long>({nbr, (long long)sms * occ, (long long)T.value_blocks}));
    wt.enabled = true;
    return 0;
}

inline void warp_tma_free(WarpTmaPlan &wt)
{
    if (wt.d_coefp) pool_release(wt.d_coefp);
    wt = WarpTmaPlan{};
}

}  // namespace skm
