// skm_table.cuh -- phase-table fast path: stationary kernel on commensurate grids.
//
// When the control-point spacing is an integer multiple h_d of the fixed-image spacing and
// every texel is sampled, a texel x = h*a + p (phase p in [0,h)^D) lies at cp-index
// coordinate  q + phi(p)  with an integer cell q and a fractional offset phi that depends on
// the phase only.  The kernel value between texel (q, p) and control point q + t is then a
// table entry T[p][t] (stationary kernel, Kernel.h:96-103), and
//   forward:     u(q, p)   = sum_t T[p][t] * (w alpha)[q + t]          (a 3-D transposed convolution)
//   derivative:  d[j]      = w_j * sum_t sum_p T[p][t] * g(j - t, p)  (its adjoint)
// with g = (metric coefficient) * grad M per texel.  The sums run over exactly the control
// points inside the kernel support -- the same set the reference's truncated boxes visit for a
// stationary kernel (every point they add outside the support has k = 0).
//
// Kernels (one launch each):
//   table_transform_kernel  T x A register-blocked transform (4 z-phases of 2 cells per thread),
//                           u in cell-phase layout.
//   table_warp_kernel       per texel: B-spline warp + metric statistics; records (grad M, m) in
//                           cell-phase layout and per-block FP64 partials.
//   table_contrib_kernel    Contrib[t][cell] = sum_p T[p][t] g(cell, p): a register-blocked GEMM
//                           (taps x phases x cells) with T and the cells' g tile in shared memory.
//   table_gather_kernel     control-point-owned gather d[j] = w_j sum_t Contrib[t][j - t] (fixed
//                           order, no atomics) fused with RKHS/RD/PG (cp-offset kernel table),
//                           L1/L2/L2,1 and the sign flip; per-block FP64 partials of the values.
#pragma once

#include <cmath>
#include <vector>

#include "skm_kernels.cuh"

namespace skm {


constexpr int kTabMaxPhase = 16;     // phases per axis
constexpr int kTabSmallPhases = 256; // above this (or when the tables do not fit in shared memory) the
                                     // transform and the contrib GEMM run their large-phase kernels
constexpr int kTabBigCells = 8;      // cells per block of the large-phase kernels
constexpr int kTabMaxTap = 10;       // taps per axis
constexpr int kTabContribThreads = 288;   // 9 warps
constexpr int kTabCells = 32;        // cells per contrib block
constexpr int kTabTapChunk = 12;     // taps per thread in the contrib GEMM

// The contrib GEMM's output summed per brick of cells: every brick (bx x by x bz cells) adds its
// cells' tap contributions into the patch of control points they reach, (b + nt - 1) per axis,
// and writes that patch; the gather then sums, for each control point, the patches that hold it.
struct BrickPartials {
    const float *partial;   // [brick][comp][pz][py][px]; NULL: the Contrib array and tap gather
    int b[3];               // cells per brick
    int nb[3];              // bricks per axis (covering the cell grid)
    int px, py, pv;         // patch extent along x, y; floats per component patch
};

struct TableDev {
    int D;
    int h[3];            // phases per axis
    int nph;             // h0*h1*h2
    int tlo[3], nt[3];   // tap offsets t in [tlo, tlo + nt) per axis
    int ntap, ntap_pad;  // nt0*nt1*nt2, rounded up to kTabTapChunk
    int qmin[3], nq[3];  // cells covering the fixed image
    long long ncell;
    int qoff[3][kTabMaxPhase];   // cell of texel h*a + p is a + qoff[p]
    int clo[3], nc[3];           // control-point offsets of the regularizer box
    const float *tfwd;   // [tap][(px,py)][pz]; large-phase plans: [tap][phase]
    const float *tgemm;  // [phase][ntap_pad]
    const float *kcp;    // [nkcp]: nonzero kernel values between control points at an offset ...
    const int *kcpo;     // [nkcp]: ... and the offsets, (dx + 512) | (dy + 512) << 10 | (dz + 512) << 20
    int nkcp;            // offsets of the regularizer box with a nonzero kernel value, in box order
    float4 *rec;         // [cell][phase]: grad M, m
    float *ucp;          // [comp][cell][phase]: u = sum_t T w alpha (planes of ncell*nph)
    const float *fixcp;  // [cell][phase]: fixed image value (0 outside)
    float *contrib;      // [3][ngtap][ncell]
    const int *gtap;     // contrib tap k -> box tap index (NULL: identity, all ntap box taps)
    int ngtap;           // taps in the contrib layout
    double *part;        // [NQ][value blocks]
    float *bigpart;      // large-phase contrib: [big_splits][3][ntap][ncell] partial sums (big_splits > 1)
    int big_splits;      // phase splits of a cell group in the large-phase contrib (1: direct)
    unsigned *tc_err;    // failure word of the tensor-core kernels (NULL without them)
    BrickPartials bp;    // set for the gather when the contrib GEMM writes brick partials
    int value_blocks, tile_x, tile_y, tiles_x, tiles_y, tiles_z;
    FastDiv div_nph, div_nq0, div_nq01, div_h0, div_h01;   // index decomposition (ncell * nph < 2^31)
};

struct TablePlan {
    bool enabled = false;
    TableDev dev{};
    float *d_tfwd = nullptr, *d_tgemm = nullptr, *d_kcp = nullptr, *d_fixcp = nullptr, *d_contrib = nullptr;
    int *d_kcpo = nullptr;
    float4 *d_rec = nullptr;
    float *d_ucp = nullptr;
    double *d_part = nullptr;
    float *d_bigpart = nullptr;
    int hl = 1;          // z phases per thread in the transform kernel (template argument)
    int big_pb = 1;      // large-phase transform: phases per thread (template argument 1, 2 or 4)
    int ncz = 1;         // cells per thread along z in the transform kernel
    int transform_blocks = 0, contrib_blocks = 0;
    bool big = false;    // large-phase plan (coarse levels: control spacing 8 or 16 voxels): the
                         // tables stay in global memory / L2, table_transform_big_kernel and
                         // table_contrib_big_kernel replace the shared-memory-table kernels
    std::vector<float> h_tgemm;   // host copy of tgemm (operand tables of the tensor-core kernels)
};

// ------------------------------------------------------------------------------------------------
// value pass, part 1: u(q, p) = sum_t T[p][t] (w alpha)[q + t] for HL z-phases of NCZ cells
// (stacked along z) per thread.  Threads of a warp share the control-point values (2 cells) and
// read 16 different table rows, so every tap costs 3 shared-memory wavefronts per 12*NCZ FMAs.
template <int HL, int NCZ>
__global__ void __launch_bounds__(256, 2) table_transform_kernel(EvalParams P, TableDev T)
{
    extern __shared__ float4 smem4[];
    const int nphxy = T.h[0] * T.h[1];
    const int ncell_blk = blockDim.x / nphxy;
    const int ax = T.tile_x + T.nt[0] - 1, ay = T.tile_y + T.nt[1] - 1, az = NCZ + T.nt[2] - 1;
    float4 *A = smem4;
    float *tf = reinterpret_cast<float *>(smem4 + ax * ay * az);
    // the table once per block (16-byte loads), then the block walks its tiles
    const int tf_n4 = T.ntap * nphxy * HL / 4;
    for (int i = threadIdx.x; i < tf_n4; i += blockDim.x)
        reinterpret_cast<float4 *>(tf)[i] = __ldg(reinterpret_cast<const float4 *>(T.tfwd) + i);
    for (int i = tf_n4 * 4 + threadIdx.x; i < T.ntap * nphxy * HL; i += blockDim.x) tf[i] = T.tfwd[i];
    const int pxy = threadIdx.x % nphxy;
    const int cl = threadIdx.x / nphxy;
    const int px = pxy % T.h[0], py = pxy / T.h[0];
    const int cx = cl % T.tile_x, cy = cl / T.tile_x;
    const int ntiles = T.tiles_x * T.tiles_y * T.tiles_z;
    const int nt0 = T.nt[0];
    const int plane = ax * ay;
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int tx0 = (tile % T.tiles_x) * T.tile_x;
        const int ty0 = ((tile / T.tiles_x) % T.tiles_y) * T.tile_y;
        const int tz0 = (tile / (T.tiles_x * T.tiles_y)) * NCZ;
        const int q0[3] = {T.qmin[0] + tx0, T.qmin[1] + ty0, T.qmin[2] + tz0};
        __syncthreads();                                   // previous tile done with A
        for (int i = threadIdx.x; i < ax * ay * az; i += blockDim.x) {
            const int x = i % ax, y = (i / ax) % ay, z = i / (ax * ay);
            const int j[3] = {q0[0] + T.tlo[0] + x, q0[1] + T.tlo[1] + y, q0[2] + T.tlo[2] + z};
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
            if (j[0] >= 0 && j[0] < P.cp.n[0] && j[1] >= 0 && j[1] < P.cp.n[1] && j[2] >= 0 && j[2] < P.cp.n[2]) {
                const float4 c = __ldg(P.cpd + j[0] + P.cp.st[1] * j[1] + P.cp.st[2] * j[2]);
                a = make_float4(c.w * c.x, c.w * c.y, c.w * c.z, 0.f);
            }
            A[i] = a;
        }
        __syncthreads();
        if (cl >= ncell_blk || tx0 + cx >= T.nq[0] || ty0 + cy >= T.nq[1]) continue;
        float acc[NCZ][HL][3];
#pragma unroll
        for (int c = 0; c < NCZ; ++c)
#pragma unroll
            for (int k = 0; k < HL; ++k) acc[c][k][0] = acc[c][k][1] = acc[c][k][2] = 0.f;
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
#pragma unroll
        for (int c = 0; c < NCZ; ++c) {
            if (tz0 + c >= T.nq[2]) break;
            const long long cell =
                (long long)(tx0 + cx) + (long long)T.nq[0] * ((ty0 + cy) + (long long)T.nq[1] * (tz0 + c));
            const long long plane = T.ncell * T.nph;
#pragma unroll
            for (int k = 0; k < HL; ++k) {
                const long long i = cell * T.nph + px + T.h[0] * (py + T.h[1] * k);
                T.ucp[i] = acc[c][k][0];
                T.ucp[i + plane] = acc[c][k][1];
                if (T.D > 2) T.ucp[i + 2 * plane] = acc[c][k][2];
            }
        }
    }
}

// value pass, part 2: one thread per (cell, phase) texel -- displacement field, B-spline warp,
// metric statistics (FP64 block partials) and the (grad M, m) record, all in cell-phase order
// so that a warp covers a compact brick of texels.
template <int D>
__global__ void __launch_bounds__(256, 4) table_warp_kernel(EvalParams P, TableDev T, int metric, double *stats,
                                                         unsigned *counter)
{
    __shared__ double sh[NQ * 32];
    float vf[NQ];                 // per-thread partials over a few texels; block sums in double
#pragma unroll
    for (int k = 0; k < NQ; ++k) vf[k] = 0.f;
    const int total = (int)(T.ncell * T.nph);
    const int stride = gridDim.x * blockDim.x;
    // the grid stride is a multiple of the phase count (checked by the host): every texel of this
    // thread has the same phase, so its offsets are computed once
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int p_fix = i0 % T.nph;
    int ph[3], xo[3];
    {
        const int pyz = p_fix / T.h[0], pz = pyz / T.h[1];
        ph[0] = p_fix - pyz * T.h[0];
        ph[1] = pyz - pz * T.h[1];
        ph[2] = pz;
#pragma unroll
        for (int d = 0; d < 3; ++d) xo[d] = T.h[d] * (T.qmin[d] - T.qoff[d][ph[d]]) + ph[d];
    }
    const int fn[3] = {P.fixed.n[0], P.fixed.n[1], P.fixed.n[2]};
    const int hh[3] = {T.h[0], T.h[1], T.h[2]};
    const int nq0 = T.nq[0], nq1 = T.nq[1];
    const FastDiv dq0 = T.div_nq0, dq01 = T.div_nq01;
    const int nphv = T.nph;
    // u and the fixed value of the next texel are loaded one iteration ahead, so that their
    // latency overlaps the B-spline gathers of the current texel
    const int plane = total;
    float un[3] = {0.f, 0.f, 0.f}, fnx = 0.f;
    if (i0 < total) {
        un[0] = T.ucp[i0];
        un[1] = T.ucp[i0 + plane];
        if (D > 2) un[2] = T.ucp[i0 + 2 * plane];
        fnx = T.fixcp[i0];
    }
    for (int i = i0, cell = i0 / nphv; i < total; i += stride, cell += stride / nphv) {
        const float u[3] = {un[0], un[1], un[2]};
        const float f = fnx;
        if (i + stride < total) {
            un[0] = T.ucp[i + stride];
            un[1] = T.ucp[i + stride + plane];
            if (D > 2) un[2] = T.ucp[i + stride + 2 * plane];
            fnx = T.fixcp[i + stride];
        }
        const int cyz = (int)dq0.div((uint32_t)cell), cz = (int)dq01.div((uint32_t)cell);
        const int cc[3] = {cell - cyz * nq0, cyz - cz * nq1, cz};
        int x[3];
        bool ok = true;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            x[d] = hh[d] * cc[d] + xo[d];
            if (x[d] < 0 || x[d] >= fn[d]) ok = false;
        }
        float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ok) {
            double fi[3] = {(double)x[0], (double)x[1], (double)x[2]}, p[3], mp[3], ml[3];
            to_global<D>(P.fixed, fi, p);
#pragma unroll
            for (int d = 0; d < D; ++d) mp[d] = p[d];
            if (P.has_df) {
                const long long di = nearest_index<D>(P.df, p);
                if (di >= 0) {
                    const float4 dv = P.dfd[di];
                    mp[0] += dv.x;
                    if (D > 1) mp[1] += dv.y;
                    if (D > 2) mp[2] += dv.z;
                }
            }
            mp[0] += (double)u[0];
            if (D > 1) mp[1] += (double)u[1];
            if (D > 2) mp[2] += (double)u[2];
            to_local<D>(P.mov, mp, ml);
            if (bspline_inside<D>(P.mov, ml)) {
                float m, g[3] = {0.f, 0.f, 0.f};
                bspline_derivs4<D>(P.coeffs4, P.mov, ml, m, g);
                vf[Q_COUNT] += 1.f;
                vf[Q_D2] += (m - f) * (m - f);
                vf[Q_SF] += f;
                vf[Q_SM] += m;
                vf[Q_SFF] += f * f;
                vf[Q_SMM] += m * m;
                vf[Q_SFM] += f * m;
                rec = make_float4(g[0], g[1], D > 2 ? g[2] : 0.f, m);
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
        for (int k = 0; k < NQ; ++k) T.part[(long long)k * gridDim.x + blockIdx.x] = v[k];
    if (last_block_arrived(counter)) {                     // fused statistics, fixed order
        double w[NQ];
        sum_partials<NQ>(T.part, gridDim.x, w, sh);
        if (threadIdx.x == 0) stats_finalize(w, metric, stats);
    }
}

// ------------------------------------------------------------------------------------------------
// ------------------------------------------------------------------------------------------------
// Large-phase plans (coarse scale levels: control spacing 8 or 16 voxels, 512 or 4096 phases): the
// tables (up to 4096 x 216 floats) stay in global memory, where the L2 keeps them, and a block takes
// kTabBigCells cells at a time so that every table value it loads serves all of them.
//   transform: thread = phase, u(q, p) = sum_t T[t][p] (w alpha)[q + t] for the block's cells, the
//              cells' weighted control points in shared memory (table read [tap][phase]: coalesced)
//   contrib:   thread = tap, Contrib[t][q] = sum_p T[p][t] g(q, p) for the block's cells, g staged in
//              shared memory in chunks of kTabBigChunk phases (table read [phase][tap]: coalesced)
constexpr int kTabBigChunk = 128;

constexpr int kTabBigContribCells = 16;           // contrib: two halves of 8 cells, 2 taps per thread

// PB phases per thread (p, p + 256, ..): every staged control point a thread reads serves PB
// phases, every table value 8 cells, so a tap costs 8 shared loads and PB table loads for
// 24 PB multiply-adds
template <int D, int PB>
__global__ void __launch_bounds__(256) table_transform_big_kernel(EvalParams P, TableDev T)
{
    constexpr int CB = kTabBigCells;
    extern __shared__ float4 A[];                            // [CB][ntap] weighted control points
    const int ntap = T.ntap, nph = T.nph;
    const long long plane = T.ncell * T.nph;
    const long long ngroups = (T.ncell + CB - 1) / CB;
    const int span = blockDim.x * PB;
    const int npc = (nph + span - 1) / span;                 // phase chunks of one block's threads
    for (long long item = blockIdx.x; item < ngroups * npc; item += gridDim.x) {
        const long long grp = item / npc;
        const int pc = (int)(item - grp * npc);
        const long long c0 = grp * CB;
        __syncthreads();                                     // previous item done with A
        for (int i = threadIdx.x; i < CB * ntap; i += blockDim.x) {
            const int c = i / ntap, t = i - c * ntap;
            const long long cell = c0 + c;
            float4 a = make_float4(0.f, 0.f, 0.f, 0.f);
            if (cell < T.ncell) {
                const int cyz = (int)(cell / T.nq[0]), cz = cyz / T.nq[1];
                const int cc[3] = {(int)(cell - (long long)cyz * T.nq[0]), cyz - cz * T.nq[1], cz};
                const int tt[3] = {t % T.nt[0], (t / T.nt[0]) % T.nt[1], t / (T.nt[0] * T.nt[1])};
                int j[3];
                bool in = true;
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    j[d] = T.qmin[d] + cc[d] + T.tlo[d] + tt[d];
                    if (j[d] < 0 || j[d] >= P.cp.n[d]) in = false;
                }
                if (in) {
                    const float4 cp = __ldg(P.cpd + j[0] + P.cp.st[1] * j[1] + P.cp.st[2] * j[2]);
                    a = make_float4(cp.w * cp.x, cp.w * cp.y, cp.w * cp.z, 0.f);
                }
            }
            A[c * ntap + t] = a;
        }
        __syncthreads();
        const int p0 = pc * span + threadIdx.x;
        if (p0 < nph) {
            float acc[CB][3][PB];
#pragma unroll
            for (int c = 0; c < CB; ++c)
#pragma unroll
                for (int b = 0; b < PB; ++b) acc[c][0][b] = acc[c][1][b] = acc[c][2][b] = 0.f;
            const float *tp = T.tfwd + p0;
#pragma unroll 2
            for (int t = 0; t < ntap; ++t) {
                float k[PB];
#pragma unroll
                for (int b = 0; b < PB; ++b)
                    k[b] = p0 + b * (int)blockDim.x < nph ? __ldg(tp + (long long)t * nph + b * blockDim.x) : 0.f;
#pragma unroll
                for (int c = 0; c < CB; ++c) {
                    const float4 a = A[c * ntap + t];
#pragma unroll
                    for (int b = 0; b < PB; ++b) {
                        acc[c][0][b] = fmaf(k[b], a.x, acc[c][0][b]);
                        acc[c][1][b] = fmaf(k[b], a.y, acc[c][1][b]);
                        acc[c][2][b] = fmaf(k[b], a.z, acc[c][2][b]);
                    }
                }
            }
#pragma unroll
            for (int c = 0; c < CB; ++c) {
                if (c0 + c >= T.ncell) break;
#pragma unroll
                for (int b = 0; b < PB; ++b) {
                    const int p = p0 + b * blockDim.x;
                    if (p >= nph) break;
                    const long long i = (c0 + c) * nph + p;
                    T.ucp[i] = acc[c][0][b];
                    T.ucp[i + plane] = acc[c][1][b];
                    if (D > 2) T.ucp[i + 2 * plane] = acc[c][2][b];
                }
            }
        }
    }
}

// Thread = (half, tap pair): half h takes cells 8 h .. 8 h + 7 of the block's 16, taps t and
// t + 128 (ntap <= 256): every staged g a thread reads serves two taps
__global__ void __launch_bounds__(256) table_contrib_big_kernel(TableDev T, const double *__restrict__ stats)
{
    constexpr int CB = kTabBigContribCells, CH = CB / 2;
    __shared__ float4 G[CB][kTabBigChunk];
    const int nph = T.nph, ntap = T.ntap, ntp = T.ntap_pad;
    const float cf = (float)stats[S_COEF_F], cm = (float)stats[S_COEF_M], cc = (float)stats[S_COEF_C];
    const long long ngroups = (T.ncell + CB - 1) / CB;
    // the phases of a group may be split over T.big_splits items (few cells, many phases): each
    // writes partial sums that table_contrib_big_reduce adds in split order
    const int splits = T.big_splits;
    const int per = (nph + splits - 1) / splits;
    const int h = threadIdx.x >> 7, t0 = threadIdx.x & 127, t1 = t0 + 128;
    for (long long item = blockIdx.x; item < ngroups * splits; item += gridDim.x) {
        const long long grp = item / splits;
        const int sp = (int)(item - grp * splits);
        const long long c0 = grp * CB;
        float acc[CH][3][2];
#pragma unroll
        for (int c = 0; c < CH; ++c)
#pragma unroll
            for (int u = 0; u < 2; ++u) acc[c][0][u] = acc[c][1][u] = acc[c][2][u] = 0.f;
        const int pend = min(nph, (sp + 1) * per);
        for (int p0 = sp * per; p0 < pend; p0 += kTabBigChunk) {
            const int np = min(kTabBigChunk, pend - p0);
            __syncthreads();                                 // previous chunk done with G
            for (int i = threadIdx.x; i < CB * kTabBigChunk; i += blockDim.x) {
                const int c = i / kTabBigChunk, p = i - c * kTabBigChunk;
                float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
                if (c0 + c < T.ncell && p < np) {
                    const long long idx = (c0 + c) * nph + p0 + p;
                    const float4 r = T.rec[idx];
                    const float coef = fmaf(cf, T.fixcp[idx], fmaf(cm, r.w, cc));
                    g = make_float4(coef * r.x, coef * r.y, coef * r.z, 0.f);
                }
                G[c][p] = g;
            }
            __syncthreads();
            if (t0 < ntap) {
                const float *tp = T.tgemm + (long long)p0 * ntp;
                const bool two = t1 < ntap;
#pragma unroll 2
                for (int p = 0; p < np; ++p) {
                    const float k0 = __ldg(tp + (long long)p * ntp + t0);
                    const float k1 = two ? __ldg(tp + (long long)p * ntp + t1) : 0.f;
#pragma unroll
                    for (int c = 0; c < CH; ++c) {
                        const float4 g = G[h * CH + c][p];
                        acc[c][0][0] = fmaf(k0, g.x, acc[c][0][0]);
                        acc[c][1][0] = fmaf(k0, g.y, acc[c][1][0]);
                        acc[c][2][0] = fmaf(k0, g.z, acc[c][2][0]);
                        acc[c][0][1] = fmaf(k1, g.x, acc[c][0][1]);
                        acc[c][1][1] = fmaf(k1, g.y, acc[c][1][1]);
                        acc[c][2][1] = fmaf(k1, g.z, acc[c][2][1]);
                    }
                }
            }
        }
        float *dst = splits > 1 ? T.bigpart + (long long)sp * 3 * ntap * T.ncell : T.contrib;
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int t = u ? t1 : t0;
            if (t >= ntap) break;
#pragma unroll
            for (int c = 0; c < CH; ++c) {
                const long long cell = c0 + h * CH + c;
                if (cell >= T.ncell) break;
#pragma unroll
                for (int d = 0; d < 3; ++d) dst[((long long)d * ntap + t) * T.ncell + cell] = acc[c][d][u];
            }
        }
    }
}

// Contrib = sum of the big_splits partials, in split order
__global__ void table_contrib_big_reduce(TableDev T)
{
    const long long n = 3LL * T.ntap * T.ncell;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int sp = 0; sp < T.big_splits; ++sp) s += T.bigpart[(long long)sp * n + i];
        T.contrib[i] = s;
    }
}

// Contrib[t][cell] = sum_p T[p][t] * g(cell, p),  g = (a f + b m + c) grad M
__global__ void __launch_bounds__(kTabContribThreads) table_contrib_kernel(TableDev T, const double *__restrict__ stats)
{
    extern __shared__ float4 smem4[];
    const int nph = T.nph, ntp = T.ntap_pad;
    const int gst = nph + 1;                                  // padded row: lanes hit distinct banks
    float4 *G = smem4;                                        // [kTabCells][nph + 1]
    float *tg = reinterpret_cast<float *>(smem4 + kTabCells * gst);   // [nph][ntp]
    const float cf = (float)stats[S_COEF_F], cm = (float)stats[S_COEF_M], cc = (float)stats[S_COEF_C];
    for (int i = threadIdx.x; i < nph * ntp / 4; i += blockDim.x)
        reinterpret_cast<float4 *>(tg)[i] = __ldg(reinterpret_cast<const float4 *>(T.tgemm) + i);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int nchunk = ntp / kTabTapChunk;
    const long long ntiles = (T.ncell + kTabCells - 1) / kTabCells;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const long long c0 = tile * kTabCells;
        __syncthreads();                                      // previous tile done with G
        for (int i = threadIdx.x; i < kTabCells * nph; i += blockDim.x) {
            const int c = i / nph, p = i % nph;
            float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
            if (c0 + c < T.ncell) {
                const long long idx = (c0 + c) * nph + p;
                const float4 r = T.rec[idx];
                const float coef = fmaf(cf, T.fixcp[idx], fmaf(cm, r.w, cc));
                g = make_float4(coef * r.x, coef * r.y, coef * r.z, 0.f);
            }
            G[c * gst + p] = g;
        }
        __syncthreads();
        const long long cell = c0 + lane;
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
                    if (tap < T.ntap) {
#pragma unroll
                        for (int d = 0; d < 3; ++d)
                            T.contrib[((long long)d * T.ntap + tap) * T.ncell + cell] = acc[k][d];
                    }
                }
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// d[j] = w_j sum_t Contrib[t][j - t] + regularizers + metric-level terms.  A block owns 32
// consecutive control points; its 8 warps split the taps (and the regularizer offsets) so that
// every warp load reads 32 consecutive cells of one Contrib row; warp 0 then combines the 8
// partial sums in a fixed order -- deterministic, no atomics.
constexpr int kGatherGroups = 8;                    // warps per block, each over a share of the taps
constexpr int kGatherThreads = 32 * kGatherGroups;

__device__ __forceinline__ int floor_div(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }

// BP: the contributions come as brick partials (T.bp): control point j lies in the patch of every
// brick whose cells q = j - o reach it (o in the tap box), at patch coordinate j - o_min - brick
// origin; a warp takes every 8th of those bricks (at most 3 x 3 x 4), loads first, then sums in
// brick order.  Else the Contrib array, tap by tap.
template <int D, bool BP = false>
__global__ void __launch_bounds__(kGatherThreads, 3) table_gather_kernel(EvalParams P, TableDev T, DerivParams Q)
{
    __shared__ float sacc[kGatherGroups][3][32];
    __shared__ float sreg[kGatherGroups][9][32];
    __shared__ double sval[kGatherGroups][3][32];
    __shared__ float kcp_s[1024];
    __shared__ int kcpo_s[1024];
    __shared__ int4 tapoff[kTabMaxTap * kTabMaxTap * kTabMaxTap];   // (tx+tlo, ty+tlo, tz+tlo) per tap
    const int nkcp = T.nkcp;
    for (int i = threadIdx.x; i < nkcp; i += blockDim.x) {
        kcp_s[i] = T.kcp[i];
        kcpo_s[i] = T.kcpo[i];
    }
    for (int k = threadIdx.x; k < T.ngtap; k += blockDim.x) {
        const int i = T.gtap ? T.gtap[k] : k;
        tapoff[k] = make_int4(T.tlo[0] + T.qmin[0] + i % T.nt[0], T.tlo[1] + T.qmin[1] + (i / T.nt[0]) % T.nt[1],
                              T.tlo[2] + T.qmin[2] + i / (T.nt[0] * T.nt[1]), 0);
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const long long j_lin = (long long)blockIdx.x * 32 + lane;
    const bool active = j_lin < P.C;
    int j[3] = {0, 0, 0};
    if (active) cell_of<D>(P.cp.n, j_lin, j);
    const float4 cj = active ? P.cpd[j_lin] : make_float4(0.f, 0.f, 0.f, 0.f);
    // the fused optimizer step: warp d applies it to component d (after combining it, below); its
    // operands are loaded now so that their latency overlaps the sums
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
    if (BP && active && !Q.values_only) {
        const BrickPartials &F = T.bp;
        int blo[3], nbr[3], pj[3];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int qhi = j[d] - (T.tlo[d] + T.qmin[d]);      // cell reached through the lowest tap
            const int lo = max(floor_div(qhi - T.nt[d] + 1, F.b[d]), 0);
            const int hi = min(floor_div(qhi, F.b[d]), F.nb[d] - 1);
            blo[d] = lo;
            nbr[d] = max(hi - lo + 1, 0);
            pj[d] = qhi;
        }
        const int cnt = nbr[0] * nbr[1] * nbr[2];
        constexpr int kV = 5;                                 // 8 warps x 5 >= 3 x 3 x 4 bricks
        const long long cstride = F.pv;
        for (int base = grp; base < cnt; base += kGatherGroups * kV) {
            float v[kV][3];
#pragma unroll
            for (int u = 0; u < kV; ++u) {
                const int i = base + u * kGatherGroups;
                const bool in = i < cnt;
                const int ix = in ? i % nbr[0] : 0, iy = in ? (i / nbr[0]) % nbr[1] : 0,
                          iz = in ? i / (nbr[0] * nbr[1]) : 0;
                const int bx = blo[0] + ix, by = blo[1] + iy, bz = blo[2] + iz;
                const long long brick = ((long long)bz * F.nb[1] + by) * F.nb[0] + bx;
                const int pidx = (pj[0] - bx * F.b[0]) + F.px * ((pj[1] - by * F.b[1]) + F.py * (pj[2] - bz * F.b[2]));
                const float *src = F.partial + brick * D * cstride + pidx;
                v[u][0] = in ? __ldg(src) : 0.f;
                v[u][1] = in ? __ldg(src + cstride) : 0.f;
                v[u][2] = (in && D > 2) ? __ldg(src + 2 * cstride) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kV; ++u) {
                acc[0] += v[u][0];
                acc[1] += v[u][1];
                if (D > 2) acc[2] += v[u][2];
            }
        }
    } else if (active && !Q.values_only) {
        // groups of kU taps: all loads first (independent, predicated), then the sums in tap order
        // (20: one group covers the 160 taps of a 12-voxel support at 8 warps)
        constexpr int kU = 20;
        const int ntap = T.ngtap, ncell = (int)T.ncell;
        const float *c0p = T.contrib, *c1p = T.contrib + ntap * ncell, *c2p = T.contrib + 2 * ntap * ncell;
        for (int base = grp; base < ntap; base += kGatherGroups * kU) {
            float v[kU][3];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int tap = base + u * kGatherGroups;
                const int4 o = tapoff[min(tap, ntap - 1)];
                const int qx = j[0] - o.x, qy = j[1] - o.y, qz = j[2] - o.z;
                const bool in = tap < ntap && (unsigned)qx < (unsigned)T.nq[0] && (unsigned)qy < (unsigned)T.nq[1] &&
                                (unsigned)qz < (unsigned)T.nq[2];
                const int c = in ? tap * ncell + (qz * T.nq[1] + qy) * T.nq[0] + qx : 0;
                v[u][0] = in ? __ldg(c0p + c) : 0.f;
                v[u][1] = in ? __ldg(c1p + c) : 0.f;
                v[u][2] = (in && D > 2) ? __ldg(c2p + c) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                acc[0] += v[u][0];
                acc[1] += v[u][1];
                if (D > 2) acc[2] += v[u][2];
            }
        }
    }
    // the metric-level parameters for the combining warps 0..D-1, loaded now so that their latency
    // overlaps the regularizer loop
    double pc[3] = {0.0, 0.0, 0.0};
    if (Q.with_metric && grp < D && active)
#pragma unroll
        for (int d = 0; d < D; ++d) pc[d] = Q.params[j_lin + d * P.C];
    // regularizer parts over this group's share of the control-point offsets
    float drk[3] = {0.f, 0.f, 0.f}, drd[3] = {0.f, 0.f, 0.f}, dpg[3] = {0.f, 0.f, 0.f};
    double vr = 0.0, vd = 0.0, vp = 0.0;
    const bool rkhs = Q.reg_rkhs > 0.0, rd = Q.reg_rd > 0.0, pg = Q.reg_pg > 0.0;
    if (active && (rkhs || rd || pg)) {
        const float wj = cj.w;
        const float cjv[3] = {cj.x, cj.y, cj.z};
        const float pgs = (float)Q.pg_scaling;
        // kR offsets' neighbour loads issued first (independent, predicated), then their terms in
        // offset order -- the same order and sums as one offset at a time
        constexpr int kR = 4;
        for (int o0 = grp; o0 < nkcp; o0 += kGatherGroups * kR) {
            float4 cn[kR];
            float kk[kR];
            bool okk[kR];
#pragma unroll
            for (int u = 0; u < kR; ++u) {
                const int o = o0 + u * kGatherGroups;
                const int pk = o < nkcp ? kcpo_s[o] : (512 | (512 << 10) | (512 << 20));
                kk[u] = o < nkcp ? kcp_s[o] : 0.f;
                const int ii[3] = {j[0] + (pk & 1023) - 512, j[1] + ((pk >> 10) & 1023) - 512, j[2] + (pk >> 20) - 512};
                okk[u] = o < nkcp && (unsigned)ii[0] < (unsigned)P.cp.n[0] && (unsigned)ii[1] < (unsigned)P.cp.n[1] &&
                         (unsigned)ii[2] < (unsigned)P.cp.n[2];
                cn[u] = okk[u] ? __ldg(P.cpd + lin_of<D>(P.cp, ii)) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < kR; ++u) {
                if (!okk[u]) continue;
                const float k = kk[u];
                const float4 ci4 = cn[u];
                const float ci[3] = {ci4.x, ci4.y, ci4.z};
                const float kw = k * wj;
                // per-offset terms in FP32 (relative error ~1e-7), their sums in FP64
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
                if (pg) {
                    if (D == 3) {                                  // Regularizers.cu:218-237
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
                    } else {                                       // Regularizers.cu:447-459
                        const float v2d = ci[0] * cjv[1] - ci[1] * cjv[0];
                        const double v2 = (double)v2d * v2d;
                        const double sc = (double)pgs;
                        vp += (double)kw * sc * sc / 2.0 * log(1.0 + v2 / sc);
                        const float factor = (float)v2 / pgs + 1.0f;
                        dpg[0] = fmaf(2.0f * kw, -pgs * ci[1] * v2d / factor, dpg[0]);
                        dpg[1] = fmaf(2.0f * kw, pgs * ci[0] * v2d / factor, dpg[1]);
                    }
                }
            }
        }
    }
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        sacc[grp][d][lane] = acc[d];
        sreg[grp][d][lane] = drk[d];
        sreg[grp][3 + d][lane] = drd[d];
        sreg[grp][6 + d][lane] = dpg[d];
    }
    sval[grp][0][lane] = vr;
    sval[grp][1][lane] = vd;
    sval[grp][2][lane] = vp;
    __syncthreads();
    double val[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) val[k] = 0.0;
    __shared__ double ssp[3];
    // warp d < D combines component d (the groups' partials in a fixed order), adds the
    // metric-level terms, writes the derivative and applies the fused step; warp 0 also sums the
    // regularizer values
    double sp = 0.0;
    if (grp < D && active) {
        const int d = grp;
        float a = 0.f, rk = 0.f, rdd = 0.f, rp = 0.f;
        for (int g = 0; g < kGatherGroups; ++g) {           // fixed combination order
            a += sacc[g][d][lane];
            rk += sreg[g][d][lane];
            rdd += sreg[g][3 + d][lane];
            rp += sreg[g][6 + d][lane];
            if (d == 0) {
                val[R_RKHS] += sval[g][0][lane];
                val[R_RD] += sval[g][1][lane];
                val[R_PG] += sval[g][2][lane];
            }
        }
        const double *st = Q.stats;
        double pn2 = 0.0;
        if (Q.with_metric) {
#pragma unroll
            for (int e = 0; e < D; ++e) pn2 += pc[e] * pc[e];
        }
        const double pnorm = sqrt(pn2);
        double g;
        if (Q.metric == 1)
            g = st[S_DENOM] != 0.0 ? (double)cj.w * (double)a : 0.0;
        else
            g = (double)cj.w * (double)a;
        if (rkhs) g += (double)rk * Q.reg_rkhs;
        if (rd) g += (double)rdd * Q.reg_rd;
        if (pg) g += (double)rp * Q.reg_pg;
        if (Q.with_metric) {
            const double par = pc[d];
            if (Q.reg_l1 > 0.0) {                              // metric hxx:447-466
                const double w = Q.reg_l1;
                if (fabs(par) > 0.0) g += w * (par < 0.0 ? -1.0 : 1.0);
                else if (g < -w) g += w;
                else if (g > w) g -= w;
                else g = 0.0;
            }
            if (Q.reg_l2 > 0.0) g += Q.reg_l2 * 2.0 * par;      // hxx:482-485
            if (Q.reg_l21 > 0.0) {                             // hxx:504-521
                const double w = Q.reg_l21;
                if (pnorm > 0.0) g += w * par / pnorm;
                else if (g < -w) g += w;
                else if (g > w) g -= w;
                else g = 0.0;
            }
            if (Q.negate) g = -g;
        }
        Q.deriv[j_lin + d * P.C] = g;
        if (stepper)
            sp = opt_update(Q.step, j_lin + d * P.C, g, opt_learning_rate(Q.step, st_t), st_p != 0.0, st_g, st_b, st_x);
        if (d == 0 && Q.with_metric) {
            double l1 = 0.0;
#pragma unroll
            for (int e = 0; e < D; ++e) l1 += fabs(pc[e]);
            val[R_L1] = Q.reg_l1 > 0.0 ? l1 : 0.0;
            val[R_L2] = Q.reg_l2 > 0.0 ? pn2 : 0.0;
            val[R_L21] = Q.reg_l21 > 0.0 ? pnorm : 0.0;
        }
    }
    if (grp == 0) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            const double sum = warp_sum(val[k]);
            if (lane == 0) Q.rpart[(long long)k * gridDim.x + blockIdx.x] = sum;
        }
    }
    if (Q.step.on) {                                       // uniform over the grid
        if (grp < D) {
            sp = warp_sum(sp);
            if (lane == 0) ssp[grp] = sp;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int d = 0; d < D; ++d) b += ssp[d];
            Q.step.sp_part[blockIdx.x] = b;
        }
    }
    if (last_block_arrived(Q.counter)) {                   // fused result (and step scalars), fixed order
        __shared__ double shr[NR * 32];
        double w[NR], wsp[1] = {0.0};
        sum_partials<NR>(Q.rpart, gridDim.x, w, shr);
        if (Q.step.on) sum_partials<1>(Q.step.sp_part, gridDim.x, wsp, shr);
        if (threadIdx.x == 0) {
            result_finalize(Q.stats, w, Q.reg_rkhs, Q.reg_rd, Q.reg_pg, Q.reg_l1, Q.reg_l21, Q.reg_l2, Q.out,
                            T.tc_err);
            if (Q.step.on) opt_finish(Q.step, wsp[0], opt_learning_rate(Q.step, Q.step.scal[T_TIME]), Q.out);
        }
    }
}

// ------------------------------------------------------------------------------------------------
// The same gather (Contrib array, no brick partials) with its index work moved out of the loops:
// the block's prologue writes, per contrib tap, its cell offset (ox, oy, oz) and the linear offset
// k ncell - lin(o) of Contrib[k][j - o] relative to the control point's own cell index, and per
// regularizer offset (dx, dy, dz) its linear control-point offset; both lists are padded to whole
// rounds of the warps' unrolled loops with entries whose bounds test fails.  A tap then costs one
// shared-memory read, three index differences and their bounds test, and its three loads; an
// offset the same plus its terms.  GW warps split the taps and offsets (warp g takes every GW-th),
// each adds its loads in list order, and the warps' partials are combined in warp order: the sums
// are fixed for a given GW.  Shared memory is sized at launch (gather_rows_smem).
constexpr int kRowsTapUnroll = 20;     // taps whose loads a warp has in flight
constexpr int kRowsRegUnroll = 4;      // regularizer offsets whose loads a warp has in flight

inline size_t gather_rows_smem(int gw, int ntap, int nkcp)
{
    const int ntr = (ntap + gw * kRowsTapUnroll - 1) / (gw * kRowsTapUnroll) * (gw * kRowsTapUnroll);
    const int nkr = (nkcp + gw * kRowsRegUnroll - 1) / (gw * kRowsRegUnroll) * (gw * kRowsRegUnroll);
    return (size_t)gw * 3 * 32 * sizeof(double) + (size_t)(ntr + nkr) * sizeof(int4) + (size_t)nkr * sizeof(float) +
           (size_t)gw * 12 * 32 * sizeof(float);
}

template <int D, int GW>
__global__ void __launch_bounds__(GW * 32, 24 / GW) table_gather_rows_kernel(EvalParams P, TableDev T, DerivParams Q)
{
    constexpr int KU = kRowsTapUnroll, KR = kRowsRegUnroll;
    static_assert(GW >= 3, "warps 0..D-1 combine one component each");
    extern __shared__ double gr_smem[];
    const int ntap = Q.values_only ? 0 : T.ngtap;
    const int ntr = (ntap + GW * KU - 1) / (GW * KU) * (GW * KU);
    const int nkcp = T.nkcp;
    const int nkr = (nkcp + GW * KR - 1) / (GW * KR) * (GW * KR);
    double *sval = gr_smem;                                        // [GW][3][32]
    int4 *stap = reinterpret_cast<int4 *>(sval + GW * 3 * 32);     // [ntr] (ox, oy, oz, contrib offset)
    int4 *soff = stap + ntr;                                       // [nkr] (dx, dy, dz, linear offset)
    float *skv = reinterpret_cast<float *>(soff + nkr);            // [nkr] kernel values
    float *sacc = skv + nkr;                                       // [GW][3][32]
    float *sreg = sacc + GW * 3 * 32;                              // [GW][9][32]
    const int ncell = (int)T.ncell;
    for (int k = threadIdx.x; k < ntr; k += blockDim.x) {
        int4 o = make_int4(1 << 29, 1 << 29, 1 << 29, 0);         // padding: outside every cell range
        if (k < ntap) {
            const int i = T.gtap ? T.gtap[k] : k;
            o.x = T.tlo[0] + T.qmin[0] + i % T.nt[0];
            o.y = T.tlo[1] + T.qmin[1] + (i / T.nt[0]) % T.nt[1];
            o.z = T.tlo[2] + T.qmin[2] + i / (T.nt[0] * T.nt[1]);
            o.w = k * ncell - ((o.z * T.nq[1] + o.y) * T.nq[0] + o.x);
        }
        stap[k] = o;
    }
    const int st1 = (int)P.cp.st[1], st2 = (int)P.cp.st[2];
    for (int o = threadIdx.x; o < nkr; o += blockDim.x) {
        int4 d4 = make_int4(1 << 29, 0, 0, 0);                     // padding: outside the grid
        float kv = 0.f;
        if (o < nkcp) {
            const int pk = T.kcpo[o];
            d4.x = (pk & 1023) - 512;
            d4.y = ((pk >> 10) & 1023) - 512;
            d4.z = (pk >> 20) - 512;
            d4.w = d4.x + (D > 1 ? st1 * d4.y : 0) + (D > 2 ? st2 * d4.z : 0);
            kv = T.kcp[o];
        }
        soff[o] = d4;
        skv[o] = kv;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const int j_lin = blockIdx.x * 32 + lane;                      // C < 2^31 (checked at creation)
    const bool active = j_lin < P.C;
    int j[3] = {0, 0, 0};
    if (active) {
        j[0] = j_lin % P.cp.n[0];
        const int r = j_lin / P.cp.n[0];
        if (D > 1) j[1] = D > 2 ? r % P.cp.n[1] : r;
        if (D > 2) j[2] = r / P.cp.n[1];
    }
    const float4 cj = active ? P.cpd[j_lin] : make_float4(0.f, 0.f, 0.f, 0.f);
    // the fused optimizer step: warp d applies it to component d (after combining it, below); its
    // operands are loaded now so that their latency overlaps the sums
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
    if (active && ntap > 0) {
        const int jcell = (j[2] * T.nq[1] + j[1]) * T.nq[0] + j[0];
        const unsigned plane = (unsigned)ntap * (unsigned)ncell;  // floats between component planes
        for (int base = grp; base < ntr; base += GW * KU) {
            float v[KU][3];
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                const int4 o = stap[base + u * GW];
                const bool in = (unsigned)(j[0] - o.x) < (unsigned)T.nq[0] && (unsigned)(j[1] - o.y) < (unsigned)T.nq[1] &&
                                (unsigned)(j[2] - o.z) < (unsigned)T.nq[2];
                const unsigned c = (unsigned)(o.w + jcell);
                v[u][0] = in ? __ldg(T.contrib + c) : 0.f;
                v[u][1] = in ? __ldg(T.contrib + (c + plane)) : 0.f;
                v[u][2] = (in && D > 2) ? __ldg(T.contrib + (c + 2u * plane)) : 0.f;
            }
#pragma unroll
            for (int u = 0; u < KU; ++u) {
                acc[0] += v[u][0];
                acc[1] += v[u][1];
                if (D > 2) acc[2] += v[u][2];
            }
        }
    }
    double pc[3] = {0.0, 0.0, 0.0};
    if (Q.with_metric && grp < D && active)
#pragma unroll
        for (int d = 0; d < D; ++d) pc[d] = Q.params[j_lin + d * P.C];
    float drk[3] = {0.f, 0.f, 0.f}, drd[3] = {0.f, 0.f, 0.f}, dpg[3] = {0.f, 0.f, 0.f};
    double vr = 0.0, vd = 0.0, vp = 0.0;
    const bool rkhs = Q.reg_rkhs > 0.0, rd = Q.reg_rd > 0.0, pg = Q.reg_pg > 0.0;
    if (active && (rkhs || rd || pg)) {
        const float wj = cj.w;
        const float cjv[3] = {cj.x, cj.y, cj.z};
        const float pgs = (float)Q.pg_scaling;
        for (int o0 = grp; o0 < nkr; o0 += GW * KR) {
            float4 cn[KR];
            float kk[KR];
            bool okk[KR];
#pragma unroll
            for (int u = 0; u < KR; ++u) {
                const int o = o0 + u * GW;
                const int4 d4 = soff[o];
                kk[u] = skv[o];
                okk[u] = (unsigned)(j[0] + d4.x) < (unsigned)P.cp.n[0] && (unsigned)(j[1] + d4.y) < (unsigned)P.cp.n[1] &&
                         (unsigned)(j[2] + d4.z) < (unsigned)P.cp.n[2];
                cn[u] = okk[u] ? __ldg(P.cpd + (j_lin + d4.w)) : make_float4(0.f, 0.f, 0.f, 0.f);
            }
#pragma unroll
            for (int u = 0; u < KR; ++u) {
                if (!okk[u]) continue;
                const float k = kk[u];
                const float4 ci4 = cn[u];
                const float ci[3] = {ci4.x, ci4.y, ci4.z};
                const float kw = k * wj;
                // per-offset terms in FP32 (relative error ~1e-7), their sums in FP64
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
                if (pg) {
                    if (D == 3) {                                  // Regularizers.cu:218-237
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
                    } else {                                       // Regularizers.cu:447-459
                        const float v2d = ci[0] * cjv[1] - ci[1] * cjv[0];
                        const double v2 = (double)v2d * v2d;
                        const double sc = (double)pgs;
                        vp += (double)kw * sc * sc / 2.0 * log(1.0 + v2 / sc);
                        const float factor = (float)v2 / pgs + 1.0f;
                        dpg[0] = fmaf(2.0f * kw, -pgs * ci[1] * v2d / factor, dpg[0]);
                        dpg[1] = fmaf(2.0f * kw, pgs * ci[0] * v2d / factor, dpg[1]);
                    }
                }
            }
        }
    }
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
    __shared__ double ssp[3];
    double sp = 0.0;
    if (grp < D && active) {
        const int d = grp;
        float a = 0.f, rk = 0.f, rdd = 0.f, rp = 0.f;
        for (int g = 0; g < GW; ++g) {                          // fixed combination order
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
        if (Q.with_metric) {
#pragma unroll
            for (int e = 0; e < D; ++e) pn2 += pc[e] * pc[e];
        }
        const double pnorm = sqrt(pn2);
        double g;
        if (Q.metric == 1)
            g = st[S_DENOM] != 0.0 ? (double)cj.w * (double)a : 0.0;
        else
            g = (double)cj.w * (double)a;
        if (rkhs) g += (double)rk * Q.reg_rkhs;
        if (rd) g += (double)rdd * Q.reg_rd;
        if (pg) g += (double)rp * Q.reg_pg;
        if (Q.with_metric) {
            const double par = pc[d];
            if (Q.reg_l1 > 0.0) {                              // metric hxx:447-466
                const double w = Q.reg_l1;
                if (fabs(par) > 0.0) g += w * (par < 0.0 ? -1.0 : 1.0);
                else if (g < -w) g += w;
                else if (g > w) g -= w;
                else g = 0.0;
            }
            if (Q.reg_l2 > 0.0) g += Q.reg_l2 * 2.0 * par;      // hxx:482-485
            if (Q.reg_l21 > 0.0) {                             // hxx:504-521
                const double w = Q.reg_l21;
                if (pnorm > 0.0) g += w * par / pnorm;
                else if (g < -w) g += w;
                else if (g > w) g -= w;
                else g = 0.0;
            }
            if (Q.negate) g = -g;
        }
        Q.deriv[j_lin + d * P.C] = g;
        if (stepper)
            sp = opt_update(Q.step, j_lin + d * P.C, g, opt_learning_rate(Q.step, st_t), st_p != 0.0, st_g, st_b, st_x);
        if (d == 0 && Q.with_metric) {
            double l1 = 0.0;
#pragma unroll
            for (int e = 0; e < D; ++e) l1 += fabs(pc[e]);
            val[R_L1] = Q.reg_l1 > 0.0 ? l1 : 0.0;
            val[R_L2] = Q.reg_l2 > 0.0 ? pn2 : 0.0;
            val[R_L21] = Q.reg_l21 > 0.0 ? pnorm : 0.0;
        }
    }
    if (grp == 0) {
#pragma unroll
        for (int k = 0; k < NR; ++k) {
            const double sum = warp_sum(val[k]);
            if (lane == 0) Q.rpart[(long long)k * gridDim.x + blockIdx.x] = sum;
        }
    }
    if (Q.step.on) {                                       // uniform over the grid
        if (grp < D) {
            sp = warp_sum(sp);
            if (lane == 0) ssp[grp] = sp;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double b = 0.0;
            for (int d = 0; d < D; ++d) b += ssp[d];
            Q.step.sp_part[blockIdx.x] = b;
        }
    }
    if (last_block_arrived(Q.counter)) {                   // fused result (and step scalars), fixed order
        __shared__ double shr[NR * 32];
        double w[NR], wsp[1] = {0.0};
        sum_partials<NR>(Q.rpart, gridDim.x, w, shr);
        if (Q.step.on) sum_partials<1>(Q.step.sp_part, gridDim.x, wsp, shr);
        if (threadIdx.x == 0) {
            result_finalize(Q.stats, w, Q.reg_rkhs, Q.reg_rd, Q.reg_pg, Q.reg_l1, Q.reg_l21, Q.reg_l2, Q.out,
                            T.tc_err);
            if (Q.step.on) opt_finish(Q.step, wsp[0], opt_learning_rate(Q.step, Q.step.scal[T_TIME]), Q.out);
        }
    }
}

// Warps per 32 control points: 4 puts every block of the 128x128x96, 24,576-point grid on the GPU at
// once (768 blocks, 6 per SM); 8 was 4 us slower per launch on a B200 (two waves).
constexpr int kRowsWarps = 4;

// The gather over the Contrib array: the hoisted-index kernel when its tables fit in 48 KB of
// shared memory (no opt-in needed), else the kernel that indexes in its loops.
template <int D>
inline void table_gather_launch(const EvalParams &P, const TableDev &G, const DerivParams &Q, int blocks,
                                cudaStream_t s)
{
    const size_t smem = gather_rows_smem(kRowsWarps, Q.values_only ? 0 : G.ngtap, G.nkcp);
    if (smem <= 48 * 1024)
        table_gather_rows_kernel<D, kRowsWarps><<<blocks, kRowsWarps * 32, smem, s>>>(P, G, Q);
    else
        table_gather_kernel<D><<<blocks, kGatherThreads, 0, s>>>(P, G, Q);
}



// ------------------------------------------------------------------------------------------------
// host side

inline float wendland_host(double r, double sc4, double sc0)
{
    // the same float profile the device evaluates (k_stationary) on a double distance
    float rf = (float)r;
    float t4 = rf * (1.0f / (float)sc4), t0 = rf * (1.0f / (float)sc0);
    float f4 = fmaxf(0.0f, 1.0f - t4), f0 = fmaxf(0.0f, 1.0f - t0);
    float f2 = f4 * f4;
    return f2 * f2 * f2 * (3.0f + 18.0f * t4 + 35.0f * t4 * t4) * (1.0f / 3.0f) * (f0 * f0);
}

// Decides whether the table path applies and builds its tables.  Returns 0 (also when the
// path does not apply; plan.enabled says which) or a CUDA error code.
// fixed image in cell-phase layout: texel (x, y, z) -> cell q = x / h + qoff[x % h] - qmin per
// axis, phase p = x % h (x fastest); entries no texel reaches stay 0
static __global__ void table_fixcp_kernel(const float *__restrict__ fixed, int nx, int ny, int nz, TableDev T,
                                   float *__restrict__ out)
{
    const long long n = (long long)nx * ny * nz;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int c[3] = {(int)(i % nx), (int)((i / nx) % ny), (int)(i / ((long long)nx * ny))};
        long long cell = 0, mul = 1;
        int ph = 0, phmul = 1;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            const int p = c[d] % T.h[d];
            const int q = c[d] / T.h[d] + T.qoff[d][p] - T.qmin[d];
            cell += mul * q;
            mul *= T.nq[d];
            ph += phmul * p;
            phmul *= T.h[d];
        }
        out[cell * T.nph + ph] = fixed[i];
    }
}

inline int table_plan(TablePlan &pl, const EvalParams &P, int D, cudaStream_t stream)
{
    pl.enabled = false;
    if (P.K.kind != kStationary || P.sub != 1) return 0;
    TableDev &T = pl.dev;
    T = TableDev{};
    T.big_splits = 1;
    T.D = D;
    const double S = (double)P.K.support_min;
    double phi[3][kTabMaxPhase];
    for (int d = 0; d < 3; ++d) {
        if (d >= D) {
            T.h[d] = 1;
            T.qoff[d][0] = 0;
            phi[d][0] = 0.0;
            continue;
        }
        const double ratio = P.cp.s[d] / P.fixed.s[d];
        const int h = (int)llround(ratio);
        if (h < 1 || h > kTabMaxPhase || fabs(ratio - h) > 1e-9 * ratio) return 0;
        T.h[d] = h;
        // cell and fractional offset of every texel exactly as the device computes them
        int qo[kTabMaxPhase];
        bool seen[kTabMaxPhase] = {false};
        for (int x = 0; x < P.fixed.n[d]; ++x) {
            const double p = P.fixed.o[d] + P.fixed.s[d] * (double)x;
            const double ip = P.cp.inv[d] * (p - P.cp.o[d]);
            const double q = floor(ip);
            const int ph = x % h, a = x / h;
            const int off = (int)q - a;
            const double fr = ip - q;
            if (!seen[ph]) {
                seen[ph] = true;
                qo[ph] = off;
                phi[d][ph] = fr;
            } else if (qo[ph] != off || fabs(phi[d][ph] - fr) > 1e-9) {
                return 0;                        // phases do not repeat exactly
            }
        }
        for (int ph = 0; ph < h; ++ph) {
            if (!seen[ph]) {                    // image shorter than one cell: derive from phase 0 rule
                const double p = P.fixed.o[d] + P.fixed.s[d] * (double)ph;
                const double ip = P.cp.inv[d] * (p - P.cp.o[d]);
                qo[ph] = (int)floor(ip);
                phi[d][ph] = ip - floor(ip);
            }
            T.qoff[d][ph] = qo[ph];
        }
    }
    T.nph = T.h[0] * T.h[1] * T.h[2];
    if (T.nph > kTabMaxPhase * kTabMaxPhase * kTabMaxPhase) return 0;
    // tap range per axis: every t with |phi - t| * spacing < S for some phase
    for (int d = 0; d < 3; ++d) {
        if (d >= D) {
            T.tlo[d] = 0;
            T.nt[d] = 1;
            continue;
        }
        const double R = S / P.cp.s[d];
        int lo = 1 << 30, hi = -(1 << 30);
        for (int t = -(int)ceil(R) - 1; t <= (int)ceil(R) + 1; ++t)
            for (int ph = 0; ph < T.h[d]; ++ph)
                if (fabs(phi[d][ph] - t) < R) {
                    lo = std::min(lo, t);
                    hi = std::max(hi, t);
                }
        if (hi < lo) return 0;
        T.tlo[d] = lo;
        T.nt[d] = hi - lo + 1;
        if (T.nt[d] > kTabMaxTap) return 0;
    }
    T.ntap = T.nt[0] * T.nt[1] * T.nt[2];
    T.ntap_pad = ((T.ntap + kTabTapChunk - 1) / kTabTapChunk) * kTabTapChunk;
    T.gtap = nullptr;
    T.ngtap = T.ntap;
    // cells covering the fixed image
    long long ncell = 1;
    for (int d = 0; d < 3; ++d) {
        if (d >= D) {
            T.qmin[d] = 0;
            T.nq[d] = 1;
            continue;
        }
        int qmn = 1 << 30, qmx = -(1 << 30);
        for (int ph = 0; ph < T.h[d]; ++ph) {
            for (int x = ph; x < P.fixed.n[d]; x += T.h[d]) {
                const int q = x / T.h[d] + T.qoff[d][ph];
                qmn = std::min(qmn, q);
                qmx = std::max(qmx, q);
            }
        }
        T.qmin[d] = qmn;
        T.nq[d] = qmx - qmn + 1;
        ncell *= T.nq[d];
    }
    T.ncell = ncell;
    // regularizer box offsets: trunc(j - R + 1) .. trunc(j + R) for interior j (Regularizers.cu:52-53)
    for (int d = 0; d < 3; ++d) {
        if (d >= D) {
            T.clo[d] = 0;
            T.nc[d] = 1;
            continue;
        }
        // offsets of an interior control point j, evaluated with the reference's double
        // arithmetic trunc(j - R + 1) .. trunc(j + R) at a large j
        const double R = S / P.cp.s[d];
        const double jb = 4096.0;
        const int lo = (int)(jb - R + 1.0) - 4096;
        const int hi = (int)(jb + R) - 4096;
        T.clo[d] = lo;
        T.nc[d] = hi - lo + 1;
    }
    if (T.nc[0] * T.nc[1] * T.nc[2] > 1024) return 0;
    for (int d = 0; d < 3; ++d)
        if (T.clo[d] < -500 || T.clo[d] + T.nc[d] > 500) return 0;   // packed offsets of the gather
    // transform tiling: threads = (px,py) phases x cells; each thread HL z-phases of NCZ cells
    const int nphxy = T.h[0] * T.h[1];
    const int hl = T.h[2];
    const int ncz = D == 3 ? 4 : 1;
    // the shared-memory-table kernels need the tables in shared memory and (px, py) phases that
    // divide the block; otherwise (coarse levels) the large-phase kernels run
    {
        const size_t sv = (size_t)(2 + T.nt[0] - 1) * (2 + T.nt[1] - 1) * (ncz + T.nt[2] - 1) * sizeof(float4) +
                          (size_t)T.ntap * T.nph * sizeof(float);
        const size_t sc = (size_t)kTabCells * (T.nph + 1) * sizeof(float4) + (size_t)T.nph * T.ntap_pad * sizeof(float);
        pl.big = T.nph > kTabSmallPhases || !(hl == 1 || hl == 2 || hl == 4 || hl == 8) || 256 % nphxy != 0 ||
                 sv > 200 * 1024 || sc > 200 * 1024;
    }
    // large-phase kernels: one thread per tap in the contrib GEMM (256 threads), the cells' weighted
    // control points of the transform in at most 48 KB of shared memory
    if (pl.big && (T.ntap > 256 || (size_t)kTabBigCells * T.ntap * sizeof(float4) > 48 * 1024)) return 0;
    const int cells = pl.big ? 1 : 256 / nphxy;
    int tx = 1;
    while (tx * tx < cells) tx *= 2;
    T.tile_x = std::min(tx, cells);
    T.tile_y = cells / T.tile_x;
    T.tiles_x = (T.nq[0] + T.tile_x - 1) / T.tile_x;
    T.tiles_y = (T.nq[1] + T.tile_y - 1) / T.tile_y;
    T.tiles_z = (T.nq[2] + ncz - 1) / ncz;
    pl.transform_blocks = T.tiles_x * T.tiles_y * T.tiles_z;
    if (T.ncell * T.nph >= (1LL << 31) || (long long)D * T.ncell * T.nph >= (1LL << 31)) return 0;
    if (3LL * T.ntap * T.ncell >= (1LL << 31)) return 0;          // 32-bit contribution indices
    {
        // a grid stride that is a multiple of the phase count keeps every thread on one phase
        long long vb = std::min<long long>((T.ncell * T.nph + 255) / 256, 148LL * 8);
        int g = T.nph, b = 256;
        while (b) {
            const int t = g % b;
            g = b;
            b = t;
        }
        const long long m = T.nph / g;
        T.value_blocks = (int)std::max<long long>(m, (vb / m) * m);
    }
    T.div_nph = FastDiv((uint32_t)T.nph);
    T.div_nq0 = FastDiv((uint32_t)T.nq[0]);
    T.div_nq01 = FastDiv((uint32_t)(T.nq[0] * T.nq[1]));
    T.div_h0 = FastDiv((uint32_t)T.h[0]);
    T.div_h01 = FastDiv((uint32_t)(T.h[0] * T.h[1]));
    pl.hl = hl;
    pl.ncz = ncz;

    // tables (kernel evaluated on the exact double offset, float profile)
    std::vector<float> tfwd((size_t)T.ntap * nphxy * hl), tgemm((size_t)T.nph * T.ntap_pad, 0.f);
    std::vector<float> kcp((size_t)T.nc[0] * T.nc[1] * T.nc[2]);
    int tap = 0;
    for (int tz = 0; tz < T.nt[2]; ++tz)
        for (int ty = 0; ty < T.nt[1]; ++ty)
            for (int tx2 = 0; tx2 < T.nt[0]; ++tx2, ++tap) {
                const int t[3] = {T.tlo[0] + tx2, T.tlo[1] + ty, T.tlo[2] + tz};
                for (int pz = 0; pz < T.h[2]; ++pz)
                    for (int py = 0; py < T.h[1]; ++py)
                        for (int px = 0; px < T.h[0]; ++px) {
                            const int ph[3] = {px, py, pz};
                            double r2 = 0.0;
                            for (int d = 0; d < D; ++d) {
                                const double e = (phi[d][ph[d]] - (double)t[d]) * P.cp.s[d];
                                r2 += e * e;
                            }
                            const float k = wendland_host(sqrt(r2), P.K.sc4, P.K.sc0);
                            if (pl.big)   // [tap][phase]: the large-phase transform reads it coalesced
                                tfwd[(size_t)tap * T.nph + px + T.h[0] * (py + T.h[1] * pz)] = k;
                            else
                                tfwd[((size_t)tap * nphxy + px + T.h[0] * py) * hl + pz] = k;
                            tgemm[(size_t)(px + T.h[0] * (py + T.h[1] * pz)) * T.ntap_pad + tap] = k;
                        }
            }
    int o = 0;
    for (int oz = 0; oz < T.nc[2]; ++oz)
        for (int oy = 0; oy < T.nc[1]; ++oy)
            for (int ox = 0; ox < T.nc[0]; ++ox, ++o) {
                const int off[3] = {T.clo[0] + ox, T.clo[1] + oy, T.clo[2] + oz};
                double r2 = 0.0;
                for (int d = 0; d < D; ++d) {
                    const double e = (double)off[d] * P.cp.s[d];
                    r2 += e * e;
                }
                kcp[o] = wendland_host(sqrt(r2), P.K.sc4, P.K.sc0);
            }
    auto up = [&](float **dst, const std::vector<float> &src) -> bool {
        if (pool_malloc((void **)dst, std::max<size_t>(1, src.size()) * sizeof(float)) != cudaSuccess) return false;
        return cudaMemcpyAsync(*dst, src.data(), src.size() * sizeof(float), cudaMemcpyHostToDevice, stream) ==
               cudaSuccess;
    };
    pl.h_tgemm = tgemm;
    // nonzero entries of the regularizer box, in box order (the sums skip k = 0 terms anyway)
    std::vector<float> kcpv;
    std::vector<int> kcpo;
    for (int oz = 0, o = 0; oz < T.nc[2]; ++oz)
        for (int oy = 0; oy < T.nc[1]; ++oy)
            for (int ox = 0; ox < T.nc[0]; ++ox, ++o) {
                if (kcp[o] == 0.0f) continue;
                kcpv.push_back(kcp[o]);
                kcpo.push_back((T.clo[0] + ox + 512) | ((T.clo[1] + oy + 512) << 10) | ((T.clo[2] + oz + 512) << 20));
            }
    T.nkcp = (int)kcpv.size();
    if (pool_malloc((void **)&pl.d_kcpo, std::max<size_t>(1, kcpo.size()) * sizeof(int)) != cudaSuccess ||
        cudaMemcpyAsync(pl.d_kcpo, kcpo.data(), kcpo.size() * sizeof(int), cudaMemcpyHostToDevice, stream) !=
            cudaSuccess)
        return 2;
    if (!up(&pl.d_tfwd, tfwd) || !up(&pl.d_tgemm, tgemm) || !up(&pl.d_kcp, kcpv)) return 2;
    {   // the fixed image in cell-phase layout, from the evaluator's device copy
        const size_t nfix = (size_t)T.ncell * T.nph;
        const long long nt = (long long)P.fixed.n[0] * P.fixed.n[1] * P.fixed.n[2];
        if (pool_malloc((void **)&pl.d_fixcp, std::max<size_t>(1, nfix) * sizeof(float)) != cudaSuccess ||
            cudaMemsetAsync(pl.d_fixcp, 0, nfix * sizeof(float), stream) != cudaSuccess)
            return 2;
        table_fixcp_kernel<<<(int)std::min<long long>((nt + 255) / 256, 4096), 256, 0, stream>>>(
            P.fixed_data, P.fixed.n[0], P.fixed.n[1], P.fixed.n[2], T, pl.d_fixcp);
        if (cudaPeekAtLastError() != cudaSuccess) return 2;
    }
    if (pool_malloc((void **)&pl.d_rec, (size_t)T.ncell * T.nph * sizeof(float4)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&pl.d_ucp, (size_t)D * T.ncell * T.nph * sizeof(float)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&pl.d_contrib, (size_t)3 * T.ntap * T.ncell * sizeof(float)) != cudaSuccess) return 2;
    if (pool_malloc((void **)&pl.d_part, (size_t)NQ * T.value_blocks * sizeof(double)) != cudaSuccess) return 2;
    if (cudaStreamSynchronize(stream) != cudaSuccess) return 2;
    T.tfwd = pl.d_tfwd;
    T.tgemm = pl.d_tgemm;
    T.kcp = pl.d_kcp;
    T.kcpo = pl.d_kcpo;
    T.fixcp = pl.d_fixcp;
    T.rec = pl.d_rec;
    T.ucp = pl.d_ucp;
    T.contrib = pl.d_contrib;
    T.part = pl.d_part;
    // shared memory of the launches
    const size_t smem_value = (size_t)(T.tile_x + T.nt[0] - 1) * (T.tile_y + T.nt[1] - 1) * (ncz + T.nt[2] - 1) *
                                  sizeof(float4) + (size_t)T.ntap * nphxy * hl * sizeof(float);
    const size_t smem_contrib =
        (size_t)kTabCells * (T.nph + 1) * sizeof(float4) + (size_t)T.nph * T.ntap_pad * sizeof(float);
    if (!pl.big && (smem_value > 200 * 1024 || smem_contrib > 200 * 1024)) return 0;
    pl.enabled = true;
    return 0;
}

inline size_t table_big_transform_smem(const TableDev &T) { return (size_t)kTabBigCells * T.ntap * sizeof(float4); }

inline size_t table_value_smem(const TablePlan &pl)
{
    const TableDev &T = pl.dev;
    return (size_t)(T.tile_x + T.nt[0] - 1) * (T.tile_y + T.nt[1] - 1) * (pl.ncz + T.nt[2] - 1) * sizeof(float4) +
           (size_t)T.ntap * T.h[0] * T.h[1] * T.h[2] * sizeof(float);
}

inline size_t table_contrib_smem(const TableDev &T)
{
    return (size_t)kTabCells * (T.nph + 1) * sizeof(float4) + (size_t)T.nph * T.ntap_pad * sizeof(float);
}

// dynamic shared memory limits of the table kernels (set once, outside any stream capture)
inline int table_set_attributes(const TablePlan &pl)
{
    if (pl.big) return 0;                          // large-phase kernels: static / small dynamic shared memory
    const int sv = (int)table_value_smem(pl), sc = (int)table_contrib_smem(pl.dev);
    cudaError_t e = cudaSuccess;
    const cudaFuncAttribute a = cudaFuncAttributeMaxDynamicSharedMemorySize;
    if (pl.dev.D == 3) {
        if (pl.hl == 1) e = cudaFuncSetAttribute(table_transform_kernel<1, 4>, a, sv);
        else if (pl.hl == 2) e = cudaFuncSetAttribute(table_transform_kernel<2, 4>, a, sv);
        else if (pl.hl == 4) e = cudaFuncSetAttribute(table_transform_kernel<4, 4>, a, sv);
        else e = cudaFuncSetAttribute(table_transform_kernel<8, 4>, a, sv);
    } else {
        e = cudaFuncSetAttribute(table_transform_kernel<1, 1>, a, sv);
    }
    if (e != cudaSuccess) return 2;
    return cudaFuncSetAttribute(table_contrib_kernel, a, sc) == cudaSuccess ? 0 : 2;
}

// Persistent grid sizes: resident blocks per SM x SMs, capped by the work.
inline int table_size_grids(TablePlan &pl)
{
    int dev = 0, sms = 0, bt = 0, bc = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 2;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 2;
    if (pl.big) {                                  // items of kTabBigCells cells, grid-strided
        TableDev &T = pl.dev;
        const long long groups = (T.ncell + kTabBigCells - 1) / kTabBigCells;
        pl.big_pb = T.nph >= 512 ? 2 : 1;          // 2 phases per thread: 98 registers, 2 blocks per SM
        const long long titems = groups * ((T.nph + 256 * pl.big_pb - 1) / (256 * pl.big_pb));
        pl.transform_blocks = (int)std::max<long long>(1, std::min<long long>(titems, 8LL * sms));
        // few cell groups (the coarsest levels): split their phases so that every SM gets work
        const long long cgroups = (T.ncell + kTabBigContribCells - 1) / kTabBigContribCells;
        const int max_split = (T.nph + kTabBigChunk - 1) / kTabBigChunk;
        // as many splits as fill two waves of two blocks per SM without starting a third
        T.big_splits = (int)std::max<long long>(1, std::min<long long>(max_split, (4LL * sms) / cgroups));
        if (T.big_splits > 1 && !pl.d_bigpart) {
            if (pool_malloc((void **)&pl.d_bigpart, sizeof(float) * (size_t)T.big_splits * 3 * T.ntap * T.ncell) !=
                cudaSuccess)
                return 2;
        }
        T.bigpart = pl.d_bigpart;
        pl.contrib_blocks = (int)std::max<long long>(1, std::min<long long>(cgroups * T.big_splits, 8LL * sms));
        return 0;
    }
    cudaError_t e;
    const int sv = (int)table_value_smem(pl);
    if (pl.dev.D == 3) {
        if (pl.hl == 1) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, table_transform_kernel<1, 4>, 256, sv);
        else if (pl.hl == 2) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, table_transform_kernel<2, 4>, 256, sv);
        else if (pl.hl == 4) e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, table_transform_kernel<4, 4>, 256, sv);
        else e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, table_transform_kernel<8, 4>, 256, sv);
    } else {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bt, table_transform_kernel<1, 1>, 256, sv);
    }
    if (e != cudaSuccess) return 2;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bc, table_contrib_kernel, kTabContribThreads,
                                                      table_contrib_smem(pl.dev)) != cudaSuccess)
        return 2;
    const int ntiles = pl.dev.tiles_x * pl.dev.tiles_y * pl.dev.tiles_z;
    const long long ctiles = (pl.dev.ncell + kTabCells - 1) / kTabCells;
    pl.transform_blocks = std::max(1, std::min(ntiles, std::max(1, bt) * sms));
    pl.contrib_blocks = (int)std::max<long long>(1, std::min<long long>(ctiles, (long long)std::max(1, bc) * sms));
    return 0;
}

inline void table_free(TablePlan &pl)
{
    float *f[] = {pl.d_tfwd, pl.d_tgemm, pl.d_kcp, pl.d_fixcp, pl.d_contrib};
    if (pl.d_kcpo) pool_release(pl.d_kcpo);
    for (float *p : f)
        if (p) pool_release(p);
    if (pl.d_rec) pool_release(pl.d_rec);
    if (pl.d_ucp) pool_release(pl.d_ucp);
    if (pl.d_part) pool_release(pl.d_part);
    if (pl.d_bigpart) pool_release(pl.d_bigpart);
    pl = TablePlan{};
}

}  // namespace skm
