// skm_batch.cuh -- many registration pairs of uneven sizes in ONE persistent kernel per optimizer
// iteration (included by skm_capi.cu, after the evaluator and the optimizer).
//
// The reference evaluates one pair per GpuKernelEvaluator (include/cuda/GpuEvaluator.cu:30-91) and
// one call per optimizer iteration (GpuEvaluator.cu:361-714).  Here every pair of a batch runs the
// phase-table formulation (skm_table.cuh: stationary kernel, control spacing an integer multiple of
// the voxel spacing, every voxel sampled), and one iteration of ALL pairs is one launch of
// batch_iteration_kernel, captured once in a CUDA graph and replayed.  Its phases, separated by a
// bounded grid barrier:
//   PACK       (pair, 256 control points)  planar parameters -> (alpha, w) floats
//   TRANSFORM  (pair, brick of cells)      u = sum_t T[p][t] (w alpha)[q + t]       (CUDA cores)
//   WARP       (pair, chunk of texels)     B-spline warp, (grad M, m) records, FP64 statistics partials
//   STATS      (pair)                      statistics in a fixed order -> derivative coefficients
//   CONTRIB    (pair, 32 cells)            Contrib[t][cell] = sum_p T[p][t] g(cell, p) over the taps
//                                          with a nonzero table column
//   GATHER     (pair, 32 control points)   derivative = w sum_t Contrib[t][j - t], RKHS/RD/PG,
//                                          L1/L2/L2,1, sign, optimizer step, value partials
//   FINISH     (pair)                      result vector, adaptive time, best value
// Work items of a phase are handed out by a device work queue (one atomic head per phase) in pair
// order, so the pairs of uneven sizes balance over the persistent CTAs and consecutive items of a
// CTA mostly share the pair's tables.  Every sum is taken in a fixed order (per-item partials,
// summed by one CTA per pair), so results do not depend on which CTA took which item.
//
// The grid barrier is bounded (2 s of %globaltimer): a CTA that gives up sets the batch's sticky
// error word and leaves; the CTAs still waiting see the word and leave too, and the host reports
// SKM_ERR_TIMEOUT.  The launch asks for cooperative scheduling (all CTAs resident), with the grid
// no larger than the resident capacity the occupancy calculator reports.
#pragma once

namespace {

constexpr int kBatchThreads = 256;
constexpr unsigned long long kBatchWaitNs = 2000000000ull;   // bounded grid barrier: 2 s

enum { BP_PACK = 0, BP_TRANSFORM, BP_WARP, BP_STATS, BP_CONTRIB, BP_GATHER, BP_FINISH, BP_N };

// One pair of the batch as the kernel sees it (copied to shared memory when a CTA changes pairs).
struct BatchPair {
    EvalParams P;            // images, geometry, kernel; P.cpd = the packed (alpha, w) floats
    TableDev T;              // phase tables and the pair's intermediates (u, records, Contrib);
                             // T.tgemm / T.ntap_pad / T.gtap / T.ngtap: the compact contrib taps
    DerivParams Q;           // weights, metric-level terms, statistics, derivative, partials, step
    int metric;
    const double *cpw;       // control-point weights
    double *vpart;           // [NQ][warp items]: statistics partials
    int items[BP_N];         // work items of this pair per phase
};

struct BatchCtl {            // device control words of one batch
    unsigned queue[BP_N];    // work-queue heads, reset at the end of every launch
    unsigned bar_count, bar_gen;
    unsigned err;            // sticky: a barrier wait gave up
};

struct BatchDev {
    const BatchPair *pairs;
    const int *first;        // [BP_N][npairs + 1]: first global item of each pair, per phase
    int npairs;
    int total[BP_N];
    BatchCtl *ctl;
    int step_on;             // 1: optimizer iteration (derivative + step); 0: one evaluation
    int warp_chunk;          // texels per WARP item (multiple of kBatchThreads and of the phase count)
};

__device__ __forceinline__ unsigned long long batch_clock_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// Bounded grid barrier (all CTAs of the launch).  Returns false when this CTA must leave: its wait
// gave up or another CTA's did.
__device__ bool batch_barrier(BatchCtl *ctl)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        volatile unsigned *gen = &ctl->bar_gen;
        volatile unsigned *err = &ctl->err;
        const unsigned g = *gen;
        __threadfence();
        if (atomicAdd(&ctl->bar_count, 1u) == gridDim.x - 1) {
            ctl->bar_count = 0u;              // nobody arrives again before the generation moves on
            __threadfence();
            atomicAdd(&ctl->bar_gen, 1u);
        } else {
            const unsigned long long t0 = batch_clock_ns();
            while (*gen == g) {
                if (*err) {
                    ok = 0;
                    break;
                }
                if (batch_clock_ns() - t0 > kBatchWaitNs) {
                    atomicOr(&ctl->err, 1u);
                    ok = 0;
                    break;
                }
                __nanosleep(100);
            }
        }
        if (*err) ok = 0;
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

__device__ __forceinline__ int batch_find_pair(const int *first, int npairs, int item)
{
    int lo = 0, hi = npairs;                  // first[lo] <= item < first[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(first + mid) <= item) lo = mid;
        else hi = mid;
    }
    return lo;
}

// ---- PACK --------------------------------------------------------------------------------------
__device__ __forceinline__ void bt_pack(const BatchPair &B, int item)
{
    const long long C = B.P.C;
    const long long i = (long long)item * kBatchThreads + threadIdx.x;
    if (i >= C) return;
    const double *pos = B.Q.step.pos;
    float4 r;
    r.x = (float)pos[i];
    r.y = (float)pos[i + C];
    r.z = (float)pos[i + 2 * C];
    r.w = (float)B.cpw[i];
    const_cast<float4 *>(B.P.cpd)[i] = r;
}

// ---- TRANSFORM (the CUDA-core table transform of skm_table.cuh, one brick per item) ------------
// tf: the pair's [tap][(px, py)][pz] table in shared memory; A: the brick's weighted control points.
template <int HL, int NCZ>
__device__ __forceinline__ void bt_transform(const BatchPair &B, int tile, float4 *A, const float *tf)
{
    const EvalParams &P = B.P;
    const TableDev &T = B.T;
    const int nphxy = T.h[0] * T.h[1];
    const int ncell_blk = kBatchThreads / nphxy;
    const int ax = T.tile_x + T.nt[0] - 1, ay = T.tile_y + T.nt[1] - 1, az = NCZ + T.nt[2] - 1;
    const int pxy = threadIdx.x % nphxy, cl = threadIdx.x / nphxy;
    const int px = pxy % T.h[0], py = pxy / T.h[0];
    const int cx = cl % T.tile_x, cy = cl / T.tile_x;
    const int tx0 = (tile % T.tiles_x) * T.tile_x;
    const int ty0 = ((tile / T.tiles_x) % T.tiles_y) * T.tile_y;
    const int tz0 = (tile / (T.tiles_x * T.tiles_y)) * NCZ;
    const int q0[3] = {T.qmin[0] + tx0, T.qmin[1] + ty0, T.qmin[2] + tz0};
    for (int i = threadIdx.x; i < ax * ay * az; i += kBatchThreads) {
        const int x = i % ax, y = (i / ax) % ay, z = i / (ax * ay);
        const int j[3] = {q0[0] + T.tlo[0] + x, q0[1] + T.tlo[1] + y, q0[2] + T.tlo[2] + z};
        float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
        if (j[0] >= 0 && j[0] < P.cp.n[0] && j[1] >= 0 && j[1] < P.cp.n[1] && j[2] >= 0 && j[2] < P.cp.n[2]) {
            const float4 c = __ldcg(P.cpd + j[0] + P.cp.st[1] * j[1] + P.cp.st[2] * j[2]);
            a = make_float4(c.w * c.x, c.w * c.y, c.w * c.z, 0.f);
        }
        A[i] = a;
    }
    __syncthreads();
    if (cl >= ncell_blk || tx0 + cx >= T.nq[0] || ty0 + cy >= T.nq[1]) return;
    float acc[NCZ][HL][3];
#pragma unroll
    for (int c = 0; c < NCZ; ++c)
#pragma unroll
        for (int k = 0; k < HL; ++k) acc[c][k][0] = acc[c][k][1] = acc[c][k][2] = 0.f;
    const int nt0 = T.nt[0], plane = ax * ay;
    int tap = 0;
    for (int tz = 0; tz < T.nt[2]; ++tz)
        for (int ty = 0; ty < T.nt[1]; ++ty) {
            const float4 *arow = A + (cx + ax * (cy + ty) + plane * tz);
            const float *trow = tf + (tap * nphxy + pxy) * HL;
#pragma unroll 3
            for (int tx = 0; tx < nt0; ++tx) {
                float tv[HL];
                if (HL == 4) {
                    const float4 t4 = *reinterpret_cast<const float4 *>(trow + tx * nphxy * HL);
                    tv[0] = t4.x; tv[1] = t4.y; tv[2] = t4.z; tv[3] = t4.w;
                } else {
#pragma unroll
                    for (int k = 0; k < HL; ++k) tv[k] = trow[tx * nphxy * HL + k];
                }
#pragma unroll
                for (int c = 0; c < NCZ; ++c) {
                    const float4 a = arow[tx + plane * c];
#pragma unroll
                    for (int k = 0; k < HL; ++k) {
                        acc[c][k][0] = fmaf(tv[k], a.x, acc[c][k][0]);
                        acc[c][k][1] = fmaf(tv[k], a.y, acc[c][k][1]);
                        acc[c][k][2] = fmaf(tv[k], a.z, acc[c][k][2]);
                    }
                }
            }
            tap += nt0;
        }
    const long long uplane = T.ncell * T.nph;
#pragma unroll
    for (int c = 0; c < NCZ; ++c) {
        if (tz0 + c >= T.nq[2]) break;
        const long long cell =
            (long long)(tx0 + cx) + (long long)T.nq[0] * ((ty0 + cy) + (long long)T.nq[1] * (tz0 + c));
#pragma unroll
        for (int k = 0; k < HL; ++k) {
            const long long i = cell * T.nph + px + T.h[0] * (py + T.h[1] * k);
            T.ucp[i] = acc[c][k][0];
            T.ucp[i + uplane] = acc[c][k][1];
            T.ucp[i + 2 * uplane] = acc[c][k][2];
        }
    }
}

// ---- WARP: per texel of one chunk (cell-phase order) ------------------------------------------
__device__ __forceinline__ void bt_warp(const BatchPair &B, int item, int chunk, double *sh)
{
    const EvalParams &P = B.P;
    const TableDev &T = B.T;
    float vf[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) vf[k] = 0.f;
    const int total = (int)(T.ncell * T.nph);
    const int base = item * chunk, end = min(base + chunk, total);
    const int i0 = base + threadIdx.x;
    // chunk and the block size are multiples of the phase count: one phase per thread
    const int p_fix = i0 % T.nph;
    int xo[3];
    {
        const int pyz = p_fix / T.h[0], pz = pyz / T.h[1];
        const int ph[3] = {p_fix - pyz * T.h[0], pyz - pz * T.h[1], pz};
#pragma unroll
        for (int d = 0; d < 3; ++d) xo[d] = T.h[d] * (T.qmin[d] - T.qoff[d][ph[d]]) + ph[d];
    }
    const long long uplane = (long long)total;
    for (int i = i0; i < end; i += kBatchThreads) {
        const int cell = (int)T.div_nph.div((uint32_t)i);
        const int cyz = (int)T.div_nq0.div((uint32_t)cell), cz = (int)T.div_nq01.div((uint32_t)cell);
        const int cc[3] = {cell - cyz * T.nq[0], cyz - cz * T.nq[1], cz};
        int x[3];
        bool ok = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x[d] = T.h[d] * cc[d] + xo[d];
            if (x[d] < 0 || x[d] >= P.fixed.n[d]) ok = false;
        }
        float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ok) {
            const float u0 = __ldcg(T.ucp + i), u1 = __ldcg(T.ucp + i + uplane), u2 = __ldcg(T.ucp + i + 2 * uplane);
            const float f = __ldg(T.fixcp + i);
            double fi[3] = {(double)x[0], (double)x[1], (double)x[2]}, p[3], ml[3];
            to_global<3>(P.fixed, fi, p);
            p[0] += (double)u0;
            p[1] += (double)u1;
            p[2] += (double)u2;
            to_local<3>(P.mov, p, ml);
            if (bspline_inside<3>(P.mov, ml)) {
                float m, g[3] = {0.f, 0.f, 0.f};
                bspline_derivs4<3>(P.coeffs4, P.mov, ml, m, g);
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
    double v[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = (double)vf[k];
    block_sum<NQ>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) B.vpart[(long long)k * B.items[BP_WARP] + item] = v[k];
}

// ---- STATS / FINISH (one CTA per pair, fixed order) ----------------------------------------------
__device__ __forceinline__ void bt_stats(const BatchPair &B, double *sh)
{
    double w[NQ];
    sum_partials<NQ>(B.vpart, B.items[BP_WARP], w, sh);
    if (threadIdx.x == 0) stats_finalize(w, B.metric, const_cast<double *>(B.Q.stats));
}

__device__ __forceinline__ void bt_finish(const BatchPair &B, int step_on, double *sh)
{
    const DerivParams &Q = B.Q;
    double w[NR], wsp[1] = {0.0};
    sum_partials<NR>(Q.rpart, B.items[BP_GATHER], w, sh);
    if (step_on) sum_partials<1>(Q.step.sp_part, B.items[BP_GATHER], wsp, sh);
    if (threadIdx.x == 0) {
        result_finalize(Q.stats, w, Q.reg_rkhs, Q.reg_rd, Q.reg_pg, Q.reg_l1, Q.reg_l21, Q.reg_l2, Q.out, nullptr);
        if (step_on) opt_finish(Q.step, wsp[0], opt_learning_rate(Q.step, Q.step.scal[T_TIME]), Q.out);
    }
}

// ---- CONTRIB (the CUDA-core contrib GEMM of skm_table.cuh over the compact taps) --------------
// G: [kTabCells][nph + 1] float4; tg: the pair's compact [nph][ntap_pad] table.
__device__ __forceinline__ void bt_contrib(const BatchPair &B, int tile, float4 *G, const float *tg)
{
    const TableDev &T = B.T;
    const int nph = T.nph, ntp = T.ntap_pad, gst = nph + 1;
    const double *st = B.Q.stats;
    const float cf = (float)__ldcg(st + S_COEF_F), cm = (float)__ldcg(st + S_COEF_M), cc = (float)__ldcg(st + S_COEF_C);
    const long long c0 = (long long)tile * kTabCells;
    for (int i = threadIdx.x; i < kTabCells * nph; i += kBatchThreads) {
        const int c = i / nph, p = i % nph;
        float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
        if (c0 + c < T.ncell) {
            const long long idx = (c0 + c) * nph + p;
            const float4 r = __ldcg(T.rec + idx);
            const float coef = fmaf(cf, __ldg(T.fixcp + idx), fmaf(cm, r.w, cc));
            g = make_float4(coef * r.x, coef * r.y, coef * r.z, 0.f);
        }
        G[c * gst + p] = g;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = kBatchThreads >> 5;
    const int nchunk = ntp / kTabTapChunk;
    const long long cell = c0 + lane;
    const int ntap = T.ngtap;
    for (int ch = warp; ch < nchunk; ch += nwarps) {
        float acc[kTabTapChunk][3];
#pragma unroll
        for (int k = 0; k < kTabTapChunk; ++k) acc[k][0] = acc[k][1] = acc[k][2] = 0.f;
        const float *trow = tg + ch * kTabTapChunk;
        const float4 *grow = G + lane * gst;
#pragma unroll 4
        for (int p = 0; p < nph; ++p) {
            const float4 g = grow[p];
            const float4 ta = *reinterpret_cast<const float4 *>(trow + p * ntp);
            const float4 tb = *reinterpret_cast<const float4 *>(trow + p * ntp + 4);
            const float4 tc = *reinterpret_cast<const float4 *>(trow + p * ntp + 8);
            const float tv[12] = {ta.x, ta.y, ta.z, ta.w, tb.x, tb.y, tb.z, tb.w, tc.x, tc.y, tc.z, tc.w};
#pragma unroll
            for (int k = 0; k < kTabTapChunk; ++k) {
                acc[k][0] = fmaf(tv[k], g.x, acc[k][0]);
                acc[k][1] = fmaf(tv[k], g.y, acc[k][1]);
                acc[k][2] = fmaf(tv[k], g.z, acc[k][2]);
            }
        }
        if (cell < T.ncell) {
#pragma unroll
            for (int k = 0; k < kTabTapChunk; ++k) {
                const int tap = ch * kTabTapChunk + k;
                if (tap < ntap) {
#pragma unroll
                    for (int d = 0; d < 3; ++d) T.contrib[((long long)d * ntap + tap) * T.ncell + cell] = acc[k][d];
                }
            }
        }
    }
}

// ---- GATHER (the table gather of skm_table.cuh, one block of 32 control points per item) ------
struct BatchGatherSmem {
    float *sacc;             // [kGatherGroups][3][32]
    float *sreg;             // [kGatherGroups][9][32]
    double *sval;            // [kGatherGroups][3][32]
    double *ssp;             // [3]
    float *kcp;              // [1024] nonzero kernel values between control points ...
    int *kcpo;               // [1024] ... and their packed offsets
    int4 *tapoff;            // [kTabMaxTap^3] control-point offset of each compact tap
};

__device__ __forceinline__ void bt_gather(const BatchPair &B, int item, const BatchGatherSmem &S)
{
    constexpr int D = 3;
    const EvalParams &P = B.P;
    const TableDev &T = B.T;
    const DerivParams &Q = B.Q;
    const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const long long j_lin = (long long)item * 32 + lane;
    const bool active = j_lin < P.C;
    int j[3] = {0, 0, 0};
    if (active) cell_of<D>(P.cp.n, j_lin, j);
    const float4 cj = active ? __ldcg(P.cpd + j_lin) : make_float4(0.f, 0.f, 0.f, 0.f);
    const int sd = grp;
    const bool stepper = Q.step.on && active && sd < D;
    double st_g = 0.0, st_b = 0.0, st_x = 0.0, st_t = 0.0, st_p = 0.0;
    if (stepper) {
        st_g = Q.step.tmp[j_lin + sd * P.C];
        st_b = Q.step.base[j_lin + sd * P.C];
        st_x = Q.step.pos[j_lin + sd * P.C];
        st_t = Q.step.scal[T_TIME];
        st_p = Q.step.scal[T_PENDING];
    }
    float acc[3] = {0.f, 0.f, 0.f};
    if (active) {
        constexpr int kU = 20;
        const int ntap = T.ngtap, ncell = (int)T.ncell;
        const float *c0p = T.contrib, *c1p = T.contrib + ntap * ncell, *c2p = T.contrib + 2 * ntap * ncell;
        for (int base = grp; base < ntap; base += kGatherGroups * kU) {
            float v[kU][3];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int tap = base + u * kGatherGroups;
                const int4 o = S.tapoff[min(tap, ntap - 1)];
                const int qx = j[0] - o.x, qy = j[1] - o.y, qz = j[2] - o.z;
                const bool in = tap < ntap && (unsigned)qx < (unsigned)T.nq[0] && (unsigned)qy < (unsigned)T.nq[1] &&
                                (unsigned)qz < (unsigned)T.nq[2];
                const int c = in ? tap * ncell + (qz * T.nq[1] + qy) * T.nq[0] + qx : 0;
                v[u][0] = in ? __ldcg(c0p + c) : 0.f;
                v[u][1] = in ? __ldcg(c1p + c) : 0.f;
                v[u][2] = in ? __ldcg(c2p + c) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                acc[0] += v[u][0];
                acc[1] += v[u][1];
                acc[2] += v[u][2];
            }
        }
    }
    double pc[3] = {0.0, 0.0, 0.0};
    if (grp < D && active)
#pragma unroll
        for (int d = 0; d < D; ++d) pc[d] = Q.params[j_lin + d * P.C];
    float drk[3] = {0.f, 0.f, 0.f}, drd[3] = {0.f, 0.f, 0.f}, dpg[3] = {0.f, 0.f, 0.f};
    double vr = 0.0, vd = 0.0, vp = 0.0;
    const bool rkhs = Q.reg_rkhs > 0.0, rd = Q.reg_rd > 0.0, pg = Q.reg_pg > 0.0;
    if (active && (rkhs || rd || pg)) {
        const float wj = cj.w;
        const float cjv[3] = {cj.x, cj.y, cj.z};
        const float pgs = (float)Q.pg_scaling;
        for (int o = grp; o < T.nkcp; o += kGatherGroups) {
            const float k = S.kcp[o];
            const int pk = S.kcpo[o];
            const int ii[3] = {j[0] + (pk & 1023) - 512, j[1] + ((pk >> 10) & 1023) - 512, j[2] + (pk >> 20) - 512};
            if ((unsigned)ii[0] >= (unsigned)P.cp.n[0] || (unsigned)ii[1] >= (unsigned)P.cp.n[1] ||
                (unsigned)ii[2] >= (unsigned)P.cp.n[2])
                continue;
            const float4 ci4 = __ldcg(P.cpd + lin_of<D>(P.cp, ii));
            const float ci[3] = {ci4.x, ci4.y, ci4.z};
            const float kw = k * wj;
            if (rkhs) {                                        // Regularizers.cu:68-73
                float dot = 0.f;
#pragma unroll
                for (int d = 0; d < D; ++d) dot = fmaf(cjv[d], ci[d], dot);
                vr += (double)(kw * dot);
#pragma unroll
                for (int d = 0; d < D; ++d) drk[d] = fmaf(2.0f * kw, ci[d], drk[d]);
            }
            if (rd) {                                          // Regularizers.cu:141-144
                float l2 = 0.f;
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    const float e = cjv[d] - ci[d];
                    l2 = fmaf(e, e, l2);
                }
                vd += (double)(kw * l2);
#pragma unroll
                for (int d = 0; d < D; ++d) drd[d] = fmaf(4.0f * kw, cjv[d] - ci[d], drd[d]);
            }
            if (pg) {                                          // Regularizers.cu:218-237
                const float cr0 = ci[1] * cjv[2] - ci[2] * cjv[1];
                const float cr1 = ci[2] * cjv[0] - ci[0] * cjv[2];
                const float cr2 = ci[0] * cjv[1] - ci[1] * cjv[0];
                const double n2 = (double)cr0 * cr0 + (double)cr1 * cr1 + (double)cr2 * cr2;
                const double sc = (double)pgs;
                vp += (double)kw * sc * sc / 2.0 * log(1.0 + n2 / sc);
                const float den = 2.0f * ((float)n2 / pgs + 1.0f);
                const float dp0 = 2.0f * ci[2] * (ci[2] * cjv[0] - ci[0] * cjv[2]) - 2.0f * ci[1] * (ci[0] * cjv[1] - ci[1] * cjv[0]);
                const float dp1 = 2.0f * ci[0] * (ci[0] * cjv[1] - ci[1] * cjv[0]) - 2.0f * ci[2] * (ci[1] * cjv[2] - ci[2] * cjv[1]);
                const float dp2 = 2.0f * ci[1] * (ci[1] * cjv[2] - ci[2] * cjv[1]) - 2.0f * ci[0] * (ci[2] * cjv[0] - ci[0] * cjv[2]);
                dpg[0] = fmaf(2.0f * kw, pgs * dp0 / den, dpg[0]);
                dpg[1] = fmaf(2.0f * kw, pgs * dp1 / den, dpg[1]);
                dpg[2] = fmaf(2.0f * kw, pgs * dp2 / den, dpg[2]);
            }
        }
    }
    float *sacc = S.sacc, *sreg = S.sreg;
    double *sval = S.sval;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sacc[(grp * 3 + d) * 32 + lane] = acc[d];
        sreg[(grp * 9 + d) * 32 + lane] = drk[d];
        sreg[(grp * 9 + 3 + d) * 32 + lane] = drd[d];
        sreg[(grp * 9 + 6 + d) * 32 + lane] = dpg[d];
    }
    sval[(grp * 3 + 0) * 32 + lane] = vr;
    sval[(grp * 3 + 1) * 32 + lane] = vd;
    sval[(grp * 3 + 2) * 32 + lane] = vp;
    __syncthreads();
    double val[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) val[k] = 0.0;
    double sp = 0.0;
    if (grp < D && active) {
        const int d = grp;
        float a = 0.f, rk = 0.f, rdd = 0.f, rp = 0.f;
        for (int g = 0; g < kGatherGroups; ++g) {              // fixed combination order
            a += sacc[(g * 3 + d) * 32 + lane];
            rk += sreg[(g * 9 + d) * 32 + lane];
            rdd += sreg[(g * 9 + 3 + d) * 32 + lane];
            rp += sreg[(g * 9 + 6 + d) * 32 + lane];
            if (d == 0) {
                val[R_RKHS] += sval[(g * 3 + 0) * 32 + lane];
                val[R_RD] += sval[(g * 3 + 1) * 32 + lane];
                val[R_PG] += sval[(g * 3 + 2) * 32 + lane];
            }
        }
        const double *st = Q.stats;
        double pn2 = 0.0;
#pragma unroll
        for (int e = 0; e < D; ++e) pn2 += pc[e] * pc[e];
        const double pnorm = sqrt(pn2);
        double g;
        if (Q.metric == 1)
            g = __ldcg(st + S_DENOM) != 0.0 ? (double)cj.w * (double)a : 0.0;
        else
            g = (double)cj.w * (double)a;
        if (rkhs) g += (double)rk * Q.reg_rkhs;
        if (rd) g += (double)rdd * Q.reg_rd;
        if (pg) g += (double)rp * Q.reg_pg;
        const double par = pc[d];
        if (Q.reg_l1 > 0.0) {                                  // metric hxx:447-466
            const double w = Q.reg_l1;
            if (fabs(par) > 0.0) g += w * (par < 0.0 ? -1.0 : 1.0);
            else if (g < -w) g += w;
            else if (g > w) g -= w;
            else g = 0.0;
        }
        if (Q.reg_l2 > 0.0) g += Q.reg_l2 * 2.0 * par;          // hxx:482-485
        if (Q.reg_l21 > 0.0) {                                 // hxx:504-521
            const double w = Q.reg_l21;
            if (pnorm > 0.0) g += w * par / pnorm;
            else if (g < -w) g += w;
            else if (g > w) g -= w;
            else g = 0.0;
        }
        if (Q.negate) g = -g;
        Q.deriv[j_lin + d * P.C] = g;
        if (stepper)
            sp = opt_update(Q.step, j_lin + d * P.C, g, opt_learning_rate(Q.step, st_t), st_p != 0.0, st_g, st_b, st_x);
        if (d == 0) {
            double l1 = 0.0;
#pragma unroll
            for (int e = 0; e < D; ++e) l1 += fabs(pc[e]);
            val[R_L1] = Q.reg_l1 > 0.0 ? l1 : 0.0;
            val[R_L2] = Q.reg_l2 > 0.0 ? pn2 : 0.0;
            val[R_L21] = Q.reg_l21 > 0.0 ? pnorm : 0.0;
        }
    }
    const int nitems = B.items[BP_GATHER];
    if (grp == 0) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            const double sum = warp_sum(val[k]);
            if (lane == 0) Q.rpart[(long long)k * nitems + item] = sum;
        }
    }
    if (Q.step.on) {
        if (grp < D) {
            sp = warp_sum(sp);
            if (lane == 0) S.ssp[grp] = sp;
        }
        __syncthreads();
        if (threadIdx.x == 0) Q.step.sp_part[item] = S.ssp[0] + S.ssp[1] + S.ssp[2];
    }
}

// Shared-memory carve-up of the batch kernel (dynamic part), in bytes.
struct BatchSmem {
    int table, region, g, gather, total;
};

template <int HL, int NCZ>
// 128 registers a thread, so that two CTAs fit on an SM (the autotuner picks 1 or 2 per SM)
__global__ void __launch_bounds__(kBatchThreads, 2) batch_iteration_kernel(BatchDev B)
{
    extern __shared__ float4 bsm4[];
    __shared__ __align__(16) unsigned char sp_raw[sizeof(BatchPair)];   // the current pair's descriptor
    BatchPair &sp = *reinterpret_cast<BatchPair *>(sp_raw);
    __shared__ int s_item, s_pair;
    __shared__ double sh[NQ * 32];
    unsigned char *bsm = reinterpret_cast<unsigned char *>(bsm4);
    for (int ph = 0; ph < BP_N; ++ph) {
        if (ph > 0 && !batch_barrier(B.ctl)) return;
        const int *first = B.first + ph * (B.npairs + 1);
        int loaded = -1;                     // pair whose tables this CTA holds for this phase
        for (;;) {
            if (threadIdx.x == 0) {
                const int item = (int)atomicAdd(&B.ctl->queue[ph], 1u);
                s_item = item;
                s_pair = item < B.total[ph] ? batch_find_pair(first, B.npairs, item) : -1;
            }
            __syncthreads();
            const int item = s_item, pair = s_pair;
            if (pair < 0) break;
            const int local = item - __ldg(first + pair);
            if (pair != loaded) {            // the pair's descriptor (and, per phase, its tables)
                __syncthreads();
                const int *src = reinterpret_cast<const int *>(B.pairs + pair);
                int *dst = reinterpret_cast<int *>(&sp);
                for (int i = threadIdx.x; i < (int)(sizeof(BatchPair) / sizeof(int)); i += kBatchThreads)
                    dst[i] = __ldg(src + i);
                __syncthreads();
                if (threadIdx.x == 0 && !B.step_on) sp.Q.step.on = 0;      // evaluation only: no step
                if (ph == BP_TRANSFORM) {
                    float *tf = reinterpret_cast<float *>(bsm);
                    const int n = sp.T.ntap * sp.T.nph;
                    for (int i = threadIdx.x; i < n; i += kBatchThreads) tf[i] = __ldg(sp.T.tfwd + i);
                } else if (ph == BP_CONTRIB) {
                    float *tg = reinterpret_cast<float *>(bsm);
                    const int n = sp.T.nph * sp.T.ntap_pad;
                    for (int i = threadIdx.x; i < n; i += kBatchThreads) tg[i] = __ldg(sp.T.tgemm + i);
                } else if (ph == BP_GATHER) {
                    float *kcp = reinterpret_cast<float *>(bsm);
                    int *kcpo = reinterpret_cast<int *>(bsm + 4096);
                    int4 *tapoff = reinterpret_cast<int4 *>(bsm + 8192);
                    for (int i = threadIdx.x; i < sp.T.nkcp; i += kBatchThreads) {
                        kcp[i] = __ldg(sp.T.kcp + i);
                        kcpo[i] = __ldg(sp.T.kcpo + i);
                    }
                    const TableDev &T = sp.T;
                    for (int k = threadIdx.x; k < T.ngtap; k += kBatchThreads) {
                        const int i = __ldg(T.gtap + k);
                        tapoff[k] = make_int4(T.tlo[0] + T.qmin[0] + i % T.nt[0],
                                              T.tlo[1] + T.qmin[1] + (i / T.nt[0]) % T.nt[1],
                                              T.tlo[2] + T.qmin[2] + i / (T.nt[0] * T.nt[1]), 0);
                    }
                }
                loaded = pair;
            }
            __syncthreads();
            switch (ph) {
            case BP_PACK: bt_pack(sp, local); break;
            case BP_TRANSFORM: {
                const int tbytes = (sp.T.ntap * sp.T.nph * 4 + 127) / 128 * 128;
                bt_transform<HL, NCZ>(sp, local, reinterpret_cast<float4 *>(bsm + tbytes),
                                      reinterpret_cast<const float *>(bsm));
                break;
            }
            case BP_WARP: bt_warp(sp, local, B.warp_chunk, sh); break;
            case BP_STATS: bt_stats(sp, sh); break;
            case BP_CONTRIB: {
                const int tbytes = (sp.T.nph * sp.T.ntap_pad * 4 + 127) / 128 * 128;
                bt_contrib(sp, local, reinterpret_cast<float4 *>(bsm + tbytes), reinterpret_cast<const float *>(bsm));
                break;
            }
            case BP_GATHER: {
                BatchGatherSmem S;
                const int t0 = 8192 + kTabMaxTap * kTabMaxTap * kTabMaxTap * 16;
                S.kcp = reinterpret_cast<float *>(bsm);
                S.kcpo = reinterpret_cast<int *>(bsm + 4096);
                S.tapoff = reinterpret_cast<int4 *>(bsm + 8192);
                S.sval = reinterpret_cast<double *>(bsm + t0);
                S.sacc = reinterpret_cast<float *>(bsm + t0 + kGatherGroups * 3 * 32 * 8);
                S.sreg = S.sacc + kGatherGroups * 3 * 32;
                S.ssp = reinterpret_cast<double *>(S.sreg + kGatherGroups * 9 * 32);
                bt_gather(sp, local, S);
                break;
            }
            default: bt_finish(sp, B.step_on, sh); break;
            }
            __syncthreads();
        }
    }
    // every CTA has left the last phase: reset the queue heads for the next launch
    if (!batch_barrier(B.ctl)) return;
    if (blockIdx.x == 0 && threadIdx.x < BP_N) B.ctl->queue[threadIdx.x] = 0u;
}

// bytes of dynamic shared memory the kernel needs for the given pairs and transform shape
inline size_t batch_smem_bytes(const std::vector<BatchPair> &pairs, int ncz)
{
    size_t m = 8192 + (size_t)kTabMaxTap * kTabMaxTap * kTabMaxTap * 16 + kGatherGroups * 3 * 32 * 8 +
               kGatherGroups * 12 * 32 * 4 + 64;
    for (const BatchPair &b : pairs) {
        const TableDev &T = b.T;
        const size_t tbytes = ((size_t)T.ntap * T.nph * 4 + 127) / 128 * 128;
        const size_t region = (size_t)(T.tile_x + T.nt[0] - 1) * (T.tile_y + T.nt[1] - 1) * (ncz + T.nt[2] - 1) * 16;
        m = std::max(m, tbytes + region);
        const size_t cbytes = ((size_t)T.nph * T.ntap_pad * 4 + 127) / 128 * 128;
        m = std::max(m, cbytes + (size_t)kTabCells * (T.nph + 1) * 16);
    }
    return m;
}

}  // namespace

// ------------------------------------------------------------------------------------------------
// host side

struct skm_batch {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::vector<skm_evaluator *> ev;           // one evaluator per pair: images, tables, intermediates
    std::vector<BatchPair> hp;
    std::vector<skm_optimizer_desc> od;
    std::vector<long long> nparam;
    std::vector<int> first;                    // [BP_N][n + 1]
    std::vector<void *> bufs;                  // device buffers owned by the batch
    BatchDev dev{};
    BatchPair *d_pairs = nullptr;
    int *d_first = nullptr;
    BatchCtl *d_ctl = nullptr;
    int hl = 4, ncz = 4, tile_x = 4, tile_y = 4, warp_chunk = 1024, ctas_per_sm = 1, grid = 0;
    size_t smem = 0;
    cudaGraphExec_t g_step = nullptr, g_eval = nullptr;
    double tuned_ms = 0.0;
    int candidates = 0;
    int iteration = 0;

    ~skm_batch()
    {
        cudaSetDevice(device);
        cudaDeviceSynchronize();
        if (g_step) cudaGraphExecDestroy(g_step);
        if (g_eval) cudaGraphExecDestroy(g_eval);
        for (void *b : bufs)
            if (b) pool_release(b);
        cudaStreamSynchronize(0);
        for (skm_evaluator *e : ev) delete e;
        if (stream) cudaStreamDestroy(stream);
    }
};

template <typename T>
static int batch_alloc(skm_batch *b, T **p, size_t n)
{
    if (dalloc(p, n)) return SKM_ERR_CUDA;
    b->bufs.push_back(*p);
    return SKM_OK;
}

template <int HL, int NCZ>
static cudaError_t batch_launch_t(const skm_batch *b, const BatchDev &dev, cudaStream_t s)
{
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(b->grid);
    cfg.blockDim = dim3(kBatchThreads);
    cfg.dynamicSmemBytes = b->smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, batch_iteration_kernel<HL, NCZ>, dev);
}

template <int HL, int NCZ>
static cudaError_t batch_prepare_t(skm_batch *b, int *max_blocks)
{
    cudaError_t e = cudaFuncSetAttribute(batch_iteration_kernel<HL, NCZ>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)b->smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(max_blocks, batch_iteration_kernel<HL, NCZ>, kBatchThreads,
                                                         b->smem);
}

static cudaError_t batch_dispatch(skm_batch *b, bool prepare, int *max_blocks, const BatchDev *dev, cudaStream_t s)
{
    const int key = b->hl * 10 + b->ncz;
    switch (key) {
    case 42: return prepare ? batch_prepare_t<4, 2>(b, max_blocks) : batch_launch_t<4, 2>(b, *dev, s);
    case 44: return prepare ? batch_prepare_t<4, 4>(b, max_blocks) : batch_launch_t<4, 4>(b, *dev, s);
    case 22: return prepare ? batch_prepare_t<2, 2>(b, max_blocks) : batch_launch_t<2, 2>(b, *dev, s);
    default: return prepare ? batch_prepare_t<2, 4>(b, max_blocks) : batch_launch_t<2, 4>(b, *dev, s);
    }
}

// Applies one shape (transform tile, cells per thread along z, texels per warp item, CTAs per
// SM): item counts, first-item tables, shared memory, grid.  Returns SKM_ERR_UNSUPPORTED when the
// shape does not fit.
static int batch_apply_shape(skm_batch *b, int tile_x, int tile_y, int ncz, int warp_chunk, int ctas_per_sm)
{
    const int n = (int)b->hp.size();
    b->tile_x = tile_x;
    b->tile_y = tile_y;
    b->ncz = ncz;
    b->warp_chunk = warp_chunk;
    for (BatchPair &p : b->hp) {
        TableDev &T = p.T;
        T.tile_x = tile_x;
        T.tile_y = tile_y;
        T.tiles_x = (T.nq[0] + tile_x - 1) / tile_x;
        T.tiles_y = (T.nq[1] + tile_y - 1) / tile_y;
        T.tiles_z = (T.nq[2] + ncz - 1) / ncz;
        p.items[BP_PACK] = (int)((p.P.C + kBatchThreads - 1) / kBatchThreads);
        p.items[BP_TRANSFORM] = T.tiles_x * T.tiles_y * T.tiles_z;
        p.items[BP_WARP] = (int)((T.ncell * T.nph + warp_chunk - 1) / warp_chunk);
        p.items[BP_STATS] = 1;
        p.items[BP_CONTRIB] = (int)((T.ncell + kTabCells - 1) / kTabCells);
        p.items[BP_GATHER] = (int)((p.P.C + 31) / 32);
        p.items[BP_FINISH] = 1;
    }
    b->first.assign((size_t)BP_N * (n + 1), 0);
    for (int ph = 0; ph < BP_N; ++ph) {
        long long acc = 0;
        for (int i = 0; i < n; ++i) {
            b->first[(size_t)ph * (n + 1) + i] = (int)acc;
            acc += b->hp[i].items[ph];
        }
        if (acc >= (1LL << 30)) return fail(SKM_ERR_UNSUPPORTED, "batch: too many work items");
        b->first[(size_t)ph * (n + 1) + n] = (int)acc;
        b->dev.total[ph] = (int)acc;
    }
    b->smem = batch_smem_bytes(b->hp, ncz);
    if (b->smem > 220 * 1024) return fail(SKM_ERR_UNSUPPORTED, "batch: %zu bytes of shared memory", b->smem);
    int max_blocks = 0, sms = 0;
    cudaError_t e = batch_dispatch(b, true, &max_blocks, nullptr, nullptr);
    if (e != cudaSuccess) return fail(SKM_ERR_CUDA, "batch kernel attributes: %s", cudaGetErrorString(e));
    SKM_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
    if (max_blocks < 1) return fail(SKM_ERR_UNSUPPORTED, "batch kernel does not fit on an SM");
    b->ctas_per_sm = std::min(ctas_per_sm, max_blocks);
    b->grid = b->ctas_per_sm * sms;
    SKM_CUDA(cudaMemcpyAsync(b->d_pairs, b->hp.data(), sizeof(BatchPair) * n, cudaMemcpyHostToDevice, b->stream));
    SKM_CUDA(cudaMemcpyAsync(b->d_first, b->first.data(), sizeof(int) * b->first.size(), cudaMemcpyHostToDevice,
                             b->stream));
    SKM_CUDA(cudaStreamSynchronize(b->stream));
    return SKM_OK;
}

static int batch_check_ctl(skm_batch *b)
{
    BatchCtl c{};
    SKM_CUDA(cudaMemcpyAsync(&c, b->d_ctl, sizeof c, cudaMemcpyDeviceToHost, b->stream));
    SKM_CUDA(cudaStreamSynchronize(b->stream));
    if (c.err) {
        SKM_CUDA(cudaMemsetAsync(b->d_ctl, 0, sizeof(BatchCtl), b->stream));
        SKM_CUDA(cudaStreamSynchronize(b->stream));
        return fail(SKM_ERR_TIMEOUT, "batch: a grid barrier wait gave up; results discarded");
    }
    return SKM_OK;
}

static int batch_launch(skm_batch *b, int step_on)
{
    BatchDev d = b->dev;
    d.step_on = step_on;
    d.warp_chunk = b->warp_chunk;
    cudaError_t e = batch_dispatch(b, false, nullptr, &d, b->stream);
    if (e != cudaSuccess) return fail(SKM_ERR_CUDA, "batch launch: %s", cudaGetErrorString(e));
    return SKM_OK;
}

static int batch_capture(skm_batch *b, int step_on, cudaGraphExec_t *exec)
{
    if (*exec) cudaGraphExecDestroy(*exec);
    *exec = nullptr;
    SKM_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    int r = batch_launch(b, step_on);
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
    if (r) {
        if (g) cudaGraphDestroy(g);
        return r;
    }
    if (ce != cudaSuccess) return fail(SKM_ERR_CUDA, "batch graph capture: %s", cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(exec, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        *exec = nullptr;
        return fail(SKM_ERR_CUDA, "batch graph instantiation: %s", cudaGetErrorString(ie));
    }
    return SKM_OK;
}

// The project's autotuner: times each candidate shape on the batch itself (evaluation launches,
// CUDA events, median of three after one warm-up) and keeps the fastest.
static int batch_autotune(skm_batch *b, int nphxy)
{
    struct Shape {
        int tx, ty, ncz, chunk, ctas;
    };
    std::vector<Shape> cand;
    const int cells = kBatchThreads / nphxy;              // cells per transform row of threads
    std::vector<std::pair<int, int>> tiles;
    for (int tx = 1; tx <= cells; tx *= 2)
        if (cells % tx == 0 && tx <= 16 && cells / tx <= 16) tiles.push_back({tx, cells / tx});
    for (auto t : tiles)
        for (int ncz : {2, 4})
            for (int chunk : {1024, 4096})
                for (int ctas : {1, 2}) cand.push_back({t.first, t.second, ncz, chunk, ctas});
    cudaEvent_t e0, e1;
    SKM_CUDA(cudaEventCreate(&e0));
    SKM_CUDA(cudaEventCreate(&e1));
    double best = 1e30;
    Shape bs = cand.front();
    int tried = 0;
    for (const Shape &s : cand) {
        if (s.chunk % (b->hp[0].T.nph) != 0) continue;
        if (batch_apply_shape(b, s.tx, s.ty, s.ncz, s.chunk, s.ctas)) continue;
        if (s.ctas > b->ctas_per_sm) continue;                // duplicate of a smaller grid
        std::vector<float> t;
        for (int r = 0; r < 4; ++r) {
            SKM_CUDA(cudaEventRecord(e0, b->stream));
            int rc = batch_launch(b, 0);
            if (rc) return rc;
            SKM_CUDA(cudaEventRecord(e1, b->stream));
            SKM_CUDA(cudaEventSynchronize(e1));
            int c = batch_check_ctl(b);
            if (c) return c;
            float ms = 0.f;
            SKM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (r) t.push_back(ms);
        }
        std::sort(t.begin(), t.end());
        ++tried;
        if (t[1] < best) {
            best = t[1];
            bs = s;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!tried) return fail(SKM_ERR_UNSUPPORTED, "batch: no launch shape fits");
    b->tuned_ms = best;
    b->candidates = tried;
    return batch_apply_shape(b, bs.tx, bs.ty, bs.ncz, bs.chunk, bs.ctas);
}

extern "C" int skm_batch_create(int32_t npairs, const skm_batch_pair *pairs, skm_batch **out)
{
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (npairs < 1 || !pairs) return fail(SKM_ERR_INVALID, "a batch needs at least one pair");
    for (int i = 0; i < npairs; ++i) {
        const skm_batch_pair &q = pairs[i];
        if (!q.evaluator) return fail(SKM_ERR_INVALID, "pair %d: evaluator descriptor is NULL", i);
        int rc = validate_metric(&q.metric);
        if (rc) return rc;
        if (q.metric.metric != SKM_MSE && q.metric.metric != SKM_NCC)
            return fail(SKM_ERR_UNSUPPORTED, "pair %d: the batch runs MSE and NCC", i);
        if (q.evaluator->dimensions != 3) return fail(SKM_ERR_UNSUPPORTED, "pair %d: the batch runs 3-D pairs", i);
        if (!(q.optimizer.f_min != 0.0) || !(q.optimizer.omega != 0.0))
            return fail(SKM_ERR_INVALID, "pair %d: f_min and omega must be nonzero", i);
    }
    skm_batch *b = new skm_batch();
    int rc = [&]() -> int {
        SKM_CUDA(cudaGetDevice(&b->device));
        SKM_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        b->hp.resize(npairs);
        b->od.resize(npairs);
        b->nparam.resize(npairs);
        int nphxy = 0;
        for (int i = 0; i < npairs; ++i) {
            const skm_batch_pair &q = pairs[i];
            skm_evaluator *e = nullptr;
            int r = skm_evaluator_create(q.evaluator, &e);
            if (r) return r;
            b->ev.push_back(e);
            if (!e->table.enabled)
                return fail(SKM_ERR_UNSUPPORTED, "pair %d: the batch needs the phase-table path (stationary kernel, "
                                                 "control spacing an integer multiple of the voxel spacing, "
                                                 "subsample 1)", i);
            if (e->table.big)
                return fail(SKM_ERR_UNSUPPORTED, "pair %d: %d phases per cell; the batch takes at most %d", i,
                            e->table.dev.nph, kTabSmallPhases);
            const TableDev &T0 = e->table.dev;
            if (i == 0) {
                b->hl = T0.h[2];
                nphxy = T0.h[0] * T0.h[1];
            } else if (T0.h[2] != b->hl || T0.h[0] * T0.h[1] != nphxy) {
                return fail(SKM_ERR_UNSUPPORTED, "pair %d: every pair of a batch needs the same phase counts", i);
            }
            if (b->hl != 2 && b->hl != 4)
                return fail(SKM_ERR_UNSUPPORTED, "pair %d: the batch takes 2 or 4 phases along z (got %d)", i, b->hl);
            if (kBatchThreads % nphxy != 0 || T0.nph > kBatchThreads)
                return fail(SKM_ERR_UNSUPPORTED, "pair %d: phase counts do not divide the block", i);
            BatchPair &p = b->hp[i];
            p = BatchPair{};
            p.P = e->P;
            p.P.has_df = 0;
            p.T = T0;
            p.metric = q.metric.metric;
            const long long C = e->C, P = e->nparams;
            b->nparam[i] = P;
            b->od[i] = q.optimizer;
            // compact contrib taps: the box taps with a nonzero table column
            const std::vector<float> &tg = e->table.h_tgemm;
            std::vector<int> gtap;
            for (int t = 0; t < T0.ntap; ++t) {
                bool nz = false;
                for (int ph = 0; ph < T0.nph && !nz; ++ph) nz = tg[(size_t)ph * T0.ntap_pad + t] != 0.0f;
                if (nz) gtap.push_back(t);
            }
            if (gtap.empty()) gtap.push_back(0);
            const int nct = (int)gtap.size(), nct_pad = (nct + kTabTapChunk - 1) / kTabTapChunk * kTabTapChunk;
            std::vector<float> tgc((size_t)T0.nph * nct_pad, 0.f);
            for (int ph = 0; ph < T0.nph; ++ph)
                for (int k = 0; k < nct; ++k) tgc[(size_t)ph * nct_pad + k] = tg[(size_t)ph * T0.ntap_pad + gtap[k]];
            float *d_tgc = nullptr;
            int *d_gtap = nullptr;
            double *pos, *base, *tmp, *best, *cpw, *scal, *deriv, *out, *vpart, *rpart, *sppart;
            const int n_wp_max = (int)((T0.ncell * T0.nph + 1023) / 1024), n_ga = (int)((C + 31) / 32);
            if (batch_alloc(b, &d_tgc, tgc.size()) || batch_alloc(b, &d_gtap, gtap.size()) ||
                batch_alloc(b, &pos, P) || batch_alloc(b, &base, P) || batch_alloc(b, &tmp, P) ||
                batch_alloc(b, &best, P) || batch_alloc(b, &cpw, C) || batch_alloc(b, &scal, NT) ||
                batch_alloc(b, &deriv, P) || batch_alloc(b, &out, NO) || batch_alloc(b, &vpart, (size_t)NQ * n_wp_max) ||
                batch_alloc(b, &rpart, (size_t)NR * n_ga) || batch_alloc(b, &sppart, n_ga))
                return SKM_ERR_CUDA;
            SKM_CUDA(cudaMemcpyAsync(d_tgc, tgc.data(), tgc.size() * 4, cudaMemcpyHostToDevice, b->stream));
            SKM_CUDA(cudaMemcpyAsync(d_gtap, gtap.data(), gtap.size() * 4, cudaMemcpyHostToDevice, b->stream));
            std::vector<double> init(P, 0.0), w(C, 1.0);
            if (q.initial_parameters) std::memcpy(init.data(), q.initial_parameters, sizeof(double) * P);
            if (q.cpw) std::memcpy(w.data(), q.cpw, sizeof(double) * C);
            SKM_CUDA(cudaMemcpyAsync(pos, init.data(), sizeof(double) * P, cudaMemcpyHostToDevice, b->stream));
            SKM_CUDA(cudaMemcpyAsync(best, init.data(), sizeof(double) * P, cudaMemcpyHostToDevice, b->stream));
            SKM_CUDA(cudaMemcpyAsync(cpw, w.data(), sizeof(double) * C, cudaMemcpyHostToDevice, b->stream));
            SKM_CUDA(cudaMemsetAsync(base, 0, sizeof(double) * P, b->stream));
            SKM_CUDA(cudaMemsetAsync(tmp, 0, sizeof(double) * P, b->stream));
            SKM_CUDA(cudaMemsetAsync(deriv, 0, sizeof(double) * P, b->stream));
            const double s0[NT] = {0.0, 1.7976931348623157e308, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
            SKM_CUDA(cudaMemcpyAsync(scal, s0, sizeof s0, cudaMemcpyHostToDevice, b->stream));
            SKM_CUDA(cudaStreamSynchronize(b->stream));
            p.T.tgemm = d_tgc;
            p.T.ntap_pad = nct_pad;
            p.T.gtap = d_gtap;
            p.T.ngtap = nct;
            p.cpw = cpw;
            p.vpart = vpart;
            DerivParams &Q = p.Q;
            Q = DerivParams{};
            const skm_metric_desc &m = q.metric;
            Q.metric = m.metric;
            Q.with_metric = 1;
            Q.reg_rkhs = m.reg_rkhs;
            Q.reg_rd = m.reg_rd;
            Q.rd_scaling = m.reg_rd_scaling;
            Q.reg_pg = m.reg_pg;
            Q.pg_scaling = m.reg_pg_scaling;
            Q.reg_l1 = m.reg_l1;
            Q.reg_l21 = m.reg_l21;
            Q.reg_l2 = m.reg_l2;
            Q.negate = m.use_negative_gradient;
            Q.stats = e->d_stats;
            Q.params = pos;
            Q.deriv = deriv;
            Q.rpart = rpart;
            Q.out = out;
            Q.step.tmp = tmp;
            Q.step.base = base;
            Q.step.pos = pos;
            Q.step.best = best;
            Q.step.scal = scal;
            Q.step.sp_part = sppart;
            Q.step.on = 1;
            const skm_optimizer_desc &o = q.optimizer;
            Q.step.orthant = o.orthant_projection;
            Q.step.a = o.a;
            Q.step.A = o.A;
            Q.step.alpha = o.alpha;
            Q.step.f_max = o.f_max;
            Q.step.f_min = o.f_min;
            Q.step.omega = o.omega;
        }
        if (dalloc(&b->d_pairs, (size_t)npairs) || dalloc(&b->d_first, (size_t)BP_N * (npairs + 1)) ||
            dalloc(&b->d_ctl, 1))
            return SKM_ERR_CUDA;
        b->bufs.push_back(b->d_pairs);
        b->bufs.push_back(b->d_first);
        b->bufs.push_back(b->d_ctl);
        SKM_CUDA(cudaMemsetAsync(b->d_ctl, 0, sizeof(BatchCtl), b->stream));
        b->dev.pairs = b->d_pairs;
        b->dev.first = b->d_first;
        b->dev.npairs = npairs;
        b->dev.ctl = b->d_ctl;
        int r = batch_autotune(b, nphxy);
        if (r) return r;
        if ((r = batch_capture(b, 1, &b->g_step))) return r;
        if ((r = batch_capture(b, 0, &b->g_eval))) return r;
        // the autotuner's evaluation launches left the parameters untouched (no step)
        return SKM_OK;
    }();
    if (rc) {
        delete b;
        return rc;
    }
    *out = b;
    return SKM_OK;
}

extern "C" int skm_batch_destroy(skm_batch *b)
{
    delete b;
    return SKM_OK;
}

extern "C" int skm_batch_evaluate(skm_batch *b)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    SKM_CUDA(cudaSetDevice(b->device));
    SKM_CUDA(cudaGraphLaunch(b->g_eval, b->stream));
    return batch_check_ctl(b);
}

extern "C" int skm_batch_enqueue(skm_batch *b, int32_t iterations, void *stream_out)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    if (iterations < 0) return fail(SKM_ERR_INVALID, "iterations < 0");
    SKM_CUDA(cudaSetDevice(b->device));
    for (int i = 0; i < iterations; ++i) SKM_CUDA(cudaGraphLaunch(b->g_step, b->stream));
    b->iteration += iterations;
    if (stream_out) *static_cast<cudaStream_t *>(stream_out) = b->stream;
    return SKM_OK;
}

extern "C" int skm_batch_run(skm_batch *b, int32_t iterations)
{
    int rc = skm_batch_enqueue(b, iterations, nullptr);
    if (rc) return rc;
    return batch_check_ctl(b);
}

extern "C" int skm_batch_set_parameters(skm_batch *b, int32_t pair, const double *params, const double *cpw)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    if (pair < 0 || pair >= (int)b->hp.size()) return fail(SKM_ERR_INVALID, "pair %d out of range", pair);
    SKM_CUDA(cudaSetDevice(b->device));
    const BatchPair &p = b->hp[pair];
    if (params)
        SKM_CUDA(cudaMemcpyAsync(p.Q.step.pos, params, sizeof(double) * b->nparam[pair], cudaMemcpyHostToDevice,
                                 b->stream));
    if (cpw)
        SKM_CUDA(cudaMemcpyAsync(const_cast<double *>(p.cpw), cpw, sizeof(double) * p.P.C, cudaMemcpyHostToDevice,
                                 b->stream));
    SKM_CUDA(cudaStreamSynchronize(b->stream));
    return SKM_OK;
}

extern "C" int skm_batch_get_result(skm_batch *b, int32_t pair, skm_metric_values *values, double *derivative)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    if (pair < 0 || pair >= (int)b->hp.size()) return fail(SKM_ERR_INVALID, "pair %d out of range", pair);
    SKM_CUDA(cudaSetDevice(b->device));
    const BatchPair &p = b->hp[pair];
    double o[NO];
    SKM_CUDA(cudaMemcpyAsync(o, p.Q.out, sizeof o, cudaMemcpyDeviceToHost, b->stream));
    if (derivative)
        SKM_CUDA(cudaMemcpyAsync(derivative, p.Q.deriv, sizeof(double) * b->nparam[pair], cudaMemcpyDeviceToHost,
                                 b->stream));
    SKM_CUDA(cudaStreamSynchronize(b->stream));
    if (values) {
        values->value = o[O_VALUE];
        values->measure = o[O_MEASURE];
        values->reg_value = o[O_REG];
        values->reg_l1 = o[O_L1];
        values->reg_l21 = o[O_L21];
        values->reg_l2 = o[O_L2];
        values->reg_rkhs = o[O_RKHS];
        values->reg_rd = o[O_RD];
        values->reg_pg = o[O_PG];
        values->num_pixels_counted = (uint32_t)o[O_COUNT];
    }
    return SKM_OK;
}

extern "C" int skm_batch_get_parameters(skm_batch *b, int32_t pair, int32_t best, double *params)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    if (pair < 0 || pair >= (int)b->hp.size()) return fail(SKM_ERR_INVALID, "pair %d out of range", pair);
    if (!params) return fail(SKM_ERR_INVALID, "params is NULL");
    SKM_CUDA(cudaSetDevice(b->device));
    const OptStep &S = b->hp[pair].Q.step;
    const long long P = b->nparam[pair];
    if (best) {
        opt_best_pending_kernel<<<(int)std::min<long long>((P + 255) / 256, 1184), 256, 0, b->stream>>>(S.scal, S.pos,
                                                                                                       S.best, P);
        SKM_CHECK_LAUNCH();
    }
    SKM_CUDA(cudaMemcpyAsync(params, best ? S.best : S.pos, sizeof(double) * P, cudaMemcpyDeviceToHost, b->stream));
    SKM_CUDA(cudaStreamSynchronize(b->stream));
    return SKM_OK;
}

extern "C" int skm_batch_get_state(skm_batch *b, int32_t pair, skm_optimizer_state *out)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    if (pair < 0 || pair >= (int)b->hp.size()) return fail(SKM_ERR_INVALID, "pair %d out of range", pair);
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    SKM_CUDA(cudaSetDevice(b->device));
    double s[NT];
    SKM_CUDA(cudaMemcpyAsync(s, b->hp[pair].Q.step.scal, sizeof s, cudaMemcpyDeviceToHost, b->stream));
    SKM_CUDA(cudaStreamSynchronize(b->stream));
    out->iteration = (int32_t)s[T_ITER];
    out->current_time = s[T_TIME];
    out->learning_rate = s[T_LR];
    out->value = s[T_VALUE];
    out->best_value = s[T_BEST];
    out->scalar_product = s[T_SP];
    out->num_pixels_counted = (uint32_t)s[T_COUNT];
    return SKM_OK;
}

extern "C" int skm_batch_describe(skm_batch *b, skm_batch_info *out)
{
    if (!b) return fail(SKM_ERR_STATE, "batch is NULL");
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    skm_batch_info r{};
    r.pairs = (int32_t)b->hp.size();
    for (const BatchPair &p : b->hp) {
        r.fixed_texels += (int64_t)p.P.fixed.n[0] * p.P.fixed.n[1] * p.P.fixed.n[2];
        r.control_points += p.P.C;
    }
    r.grid = b->grid;
    r.ctas_per_sm = b->ctas_per_sm;
    r.transform_tile[0] = b->tile_x;
    r.transform_tile[1] = b->tile_y;
    r.transform_tile[2] = b->ncz;
    r.warp_chunk = b->warp_chunk;
    for (int ph = 0; ph < BP_N && ph < 8; ++ph) r.items[ph] = b->dev.total[ph];
    r.shared_memory = (int32_t)b->smem;
    r.tuned_ms = b->tuned_ms;
    r.candidates = b->candidates;
    *out = r;
    return SKM_OK;
}
