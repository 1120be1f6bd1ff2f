// skm_kernels.cuh -- the evaluation kernels (any kernel kind, 2-D/3-D, any subsampling).
//
// Work decomposition (B200): the value pass is one thread per sample that fuses the
// kernel-machine transform, the B-spline warp and the metric statistics and writes a
// per-sample (grad M, m) record plus per-block FP64 partial sums; the derivative is a
// control-point-owned gather with one warp per control point, lanes striding the
// control point's sample box and a fixed shuffle tree reducing the lanes -- no atomics,
// so results are bitwise reproducible.  The regularizers of the same control point run
// in the same warp and are added in the reference's order.
#pragma once

#include "skm_device.cuh"

namespace skm {

// per-block partial quantities of the value pass (laid out [quantity][block])
enum { Q_COUNT = 0, Q_D2, Q_SF, Q_SM, Q_SFF, Q_SMM, Q_SFM, Q_CC, NQ };
// per-block partial quantities of the derivative pass
enum { R_RKHS = 0, R_RD, R_PG, R_L1, R_L21, R_L2, NR };
// global statistics written by stats_kernel and read by the derivative pass
enum {
    S_COUNT = 0, S_MEASURE, S_COEF_F, S_COEF_M, S_COEF_C, S_MEAN_F, S_MEAN_M, S_DENOM, S_SFM, S_SMM,
    S_VALID, NS
};
// result vector written by result_kernel
enum {
    O_MEASURE = 0, O_RKHS, O_RD, O_PG, O_L1, O_L21, O_L2, O_REG, O_VALUE, O_COUNT, O_FAULT, NO
};

struct EvalParams {
    int sub, nbh;
    Geo fixed;         // fixed image
    Geo mov;           // B-spline coefficients (size+3 per axis), moving image origin/spacing
    Geo cp;            // control-point grid
    Geo df;            // previous-level displacement field
    int has_df;
    int ss[3];         // subsampled grid = size/subsample (GpuEvaluator.cu:44)
    long long Ns;      // number of samples
    long long C;       // control points
    const float *__restrict__ fixed_data;
    const float *__restrict__ coeffs;
    const float4 *__restrict__ coeffs4;  // row-expanded coefficients (c[i], c[i+1], c[i+2], c[i+3])
    const float4 *__restrict__ cpd;     // (alpha_x, alpha_y, alpha_z, w) per control point
    const float4 *__restrict__ dfd;     // displacement field, 4 floats per texel
    const uint32_t *__restrict__ shifts; // packed per-sample shift (8 bits per axis)
    KernelParams K;
};

// Device-resident optimizer scalars: adaptive time, best value, learning rate, <g, g_prev>,
// value, iteration, pixel count, and T_PENDING: the last step was taken from an improving
// evaluation, so its position (the current one) is the best one -- copied to `best` before the
// next step overwrites it, or when the best parameters are read.
enum { T_TIME = 0, T_BEST, T_LR, T_SP, T_VALUE, T_ITER, T_COUNT, T_PENDING, NT };

// The adaptive-step update of the optimizer (see skm_optimizer.cuh), when a derivative kernel
// applies it to the parameters it owns (on != 0).
struct OptStep {
    double *tmp, *base, *pos, *best, *scal;
    double *sp_part;                    // per-block <g, g_prev> partials
    int on, orthant;
    double a, A, alpha, f_max, f_min, omega;
};

// gamma(t) = a / (A + t + 1)^alpha  (itkAdaptiveStepsizeRegularStepGradientDescent...hxx:86-97)
__device__ __forceinline__ double opt_learning_rate(const OptStep &S, double t) { return S.a / pow(S.A + t + 1.0, S.alpha); }

// x = x_prev + gamma g with the orthant projection; the previous step's position becomes the best
// one first when that step came from an improving evaluation (pending).  gprev, b, x: tmp[j],
// base[j], pos[j] as loaded before the step.
__device__ __forceinline__ double opt_update(const OptStep &S, long long j, double g, double lr, bool pending,
                                            double gprev, double b, double x)
{
    const double sp = g * gprev;
    S.tmp[j] = g;
    if (pending) S.best[j] = x;
    double nx = b + g * lr;
    if (S.orthant && nx * b < 0.0) nx = 0.0;
    S.pos[j] = nx;
    S.base[j] = nx;
    return sp;
}

// the scalars after a step (one thread): t = max(0, t + f(-<g, g_prev>)), best value, counters
__device__ __forceinline__ void opt_finish(const OptStep &S, double sp, double lr, const double *out)
{
    double *scal = S.scal;
    const double t = scal[T_TIME];
    const double f = S.f_min + (S.f_max - S.f_min) / (1.0 - (S.f_max / S.f_min) * exp(sp / S.omega));
    scal[T_TIME] = fmax(0.0, t + f);
    const bool improving = out[O_VALUE] < scal[T_BEST];
    if (improving) scal[T_BEST] = out[O_VALUE];
    scal[T_PENDING] = improving ? 1.0 : 0.0;
    scal[T_LR] = lr;
    scal[T_SP] = sp;
    scal[T_VALUE] = out[O_VALUE];
    scal[T_ITER] += 1.0;
    scal[T_COUNT] = out[O_COUNT];
}

struct DerivParams {
    int metric;                 // 0 MSE, 1 NCC, 2 LCC
    int with_metric;            // 1: metric-level call (host regularizers + sign)
    double reg_rkhs, reg_rd, rd_scaling, reg_pg, pg_scaling;
    double reg_l1, reg_l21, reg_l2;
    int negate;
    const double *__restrict__ stats;
    const double *__restrict__ params;   // planar parameters (metric level), else null
    const float4 *__restrict__ samp;     // (grad M, m) per sample
    const float4 *__restrict__ dense;    // LCC: (grad M, m) per fixed texel
    const unsigned char *__restrict__ dense_in;
    const float4 *__restrict__ dense_sw; // LCC 3-D swapped-kernel field (non-stationary kinds)
    const unsigned char *__restrict__ dense_sw_in;
    const float4 *__restrict__ acache;   // LCC 3-D weight tensors: aniso_self_cache per listed texel
    const float *__restrict__ boxcoef;   // box-window LCC: coefficient per fixed texel (else null)
    double *__restrict__ deriv;          // planar output
    double *__restrict__ rpart;          // [NR][blocks]
    double *__restrict__ out;            // result vector (fused finalization)
    unsigned *counter;                   // ticket counter of the fused finalization
    int values_only;                     // table gather: regularizer values only (getValue)
    OptStep step;                        // table gather: the optimizer step fused (step.on)
};

// ---- sample positions ------------------------------------------------------------------------
template <int D>
__device__ __forceinline__ void cell_of(const int *n, long long t, int *c)
{
    c[0] = (int)(t % n[0]);
    c[1] = D > 1 ? (int)((t / n[0]) % n[1]) : 0;
    c[2] = D > 2 ? (int)(t / ((long long)n[0] * n[1])) : 0;
}

// samplePos = cell*subsample + shift (MSE.cu:171-174).  A shift equal to the subsample
// rate (a draw of exactly UINT_MAX) can place the last cell's sample outside the image,
// where the reference reads out of bounds; such a sample is treated as outside here.
template <int D>
__device__ __forceinline__ bool sample_pos(const EvalParams &P, long long t, int *sp)
{
    int c[3];
    cell_of<D>(P.ss, t, c);
    sp[0] = c[0]; sp[1] = c[1]; sp[2] = c[2];
    if (P.sub != 1) {
        uint32_t s = P.shifts[t];
#pragma unroll
        for (int d = 0; d < D; ++d) sp[d] = c[d] * P.sub + (int)((s >> (8 * d)) & 0xffu);
#pragma unroll
        for (int d = 0; d < D; ++d)
            if (sp[d] >= P.fixed.n[d]) return false;
    }
    return true;
}

template <int D>
__device__ __forceinline__ long long lin_of(const Geo &g, const int *i)
{
    long long r = i[0];
    if (D > 1) r += g.st[1] * i[1];
    if (D > 2) r += g.st[2] * i[2];
    return r;
}

// ---- forward transform -----------------------------------------------------------------------
// u += sum over the control-point box of w_i k(p, c_i) alpha_i (DisplacementField.cu:53-72).
// SWAP evaluates k(c_i, p) with p's kernel information (3-D LCC derivative, LCC.cu:429-442).
template <int D, int KIND, bool SWAP>
__device__ __forceinline__ void transform_add(const EvalParams &P, const double *p, const PInfo &pi, float *u)
{
    double ip[3];
    to_local<D>(P.cp, p, ip);
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    float base[3], hs[3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double sh = pi.support / P.cp.s[d];
        lo[d] = clampi((int)(ip[d] - sh + 1.0), 0, P.cp.n[d] - 1);
        hi[d] = clampi((int)(ip[d] + sh), 0, P.cp.n[d] - 1);
        base[d] = (float)(p[d] - (P.cp.o[d] + P.cp.s[d] * (double)lo[d]));
        hs[d] = (float)P.cp.s[d];
    }
    float ux = 0.f, uy = 0.f, uz = 0.f;
    for (int z = lo[2]; z <= hi[2]; ++z) {
        for (int y = lo[1]; y <= hi[1]; ++y) {
            long long row = (long long)z * P.cp.st[2] + (long long)y * P.cp.st[1];
            for (int x = lo[0]; x <= hi[0]; ++x) {
                float v[3];
                v[0] = base[0] - hs[0] * (float)(x - lo[0]);
                if (D > 1) v[1] = base[1] - hs[1] * (float)(y - lo[1]);
                if (D > 2) v[2] = base[2] - hs[2] * (float)(z - lo[2]);
                float k;
                if (KIND == kStationary) {
                    k = k_eval<KIND, D>(P.K, v, nullptr, pi);
                } else {
                    double q[3], qi[3] = {(double)x, (double)y, (double)z};
                    to_global<D>(P.cp, qi, q);
                    if (SWAP) {
                        // k(c_i, p) with sigma/cov taken at p for both ends
                        float vn[3];
#pragma unroll
                        for (int d = 0; d < D; ++d) vn[d] = -v[d];
                        k = k_eval<KIND, D>(P.K, vn, p, pi);
                    } else {
                        k = k_eval<KIND, D>(P.K, v, q, pi);
                    }
                }
                float4 c = __ldg(P.cpd + row + x);
                float wk = c.w * k;
                ux = fmaf(wk, c.x, ux);
                uy = fmaf(wk, c.y, uy);
                if (D > 2) uz = fmaf(wk, c.z, uz);
            }
        }
    }
    u[0] += ux;
    u[1] += uy;
    if (D > 2) u[2] += uz;
}

// moving-image point of fixed point p: p + DF(p) + u(p), returned in moving local coordinates.
template <int D, int KIND, bool SWAP>
__device__ __forceinline__ void moving_local(const EvalParams &P, const double *p, double *ml)
{
    double mp[3];
#pragma unroll
    for (int d = 0; d < D; ++d) mp[d] = p[d];
    if (P.has_df) {
        long long i = nearest_index<D>(P.df, p);
        if (i >= 0) {
            float4 v = P.dfd[i];
            mp[0] += v.x;
            if (D > 1) mp[1] += v.y;
            if (D > 2) mp[2] += v.z;
        }
    }
    PInfo pi;
    pinfo_at<KIND, D>(P.K, p, pi);
    float u[3] = {0.f, 0.f, 0.f};
    transform_add<D, KIND, SWAP>(P, p, pi, u);
#pragma unroll
    for (int d = 0; d < D; ++d) mp[d] += (double)u[d];
    to_local<D>(P.mov, mp, ml);
}

// ---- value pass ------------------------------------------------------------------------------
template <int D, int KIND>
__global__ void __launch_bounds__(256) value_kernel(EvalParams P, float4 *__restrict__ samp,
                                                    double *__restrict__ part)
{
    __shared__ double sh[NQ * 32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = 0.0;
    if (t < P.Ns) {
        int sp[3];
        float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
        if (sample_pos<D>(P, t, sp)) {
            double fi[3] = {(double)sp[0], (double)sp[1], (double)sp[2]}, p[3], ml[3];
            to_global<D>(P.fixed, fi, p);
            moving_local<D, KIND, false>(P, p, ml);
            if (bspline_inside<D>(P.mov, ml)) {
                float m, g[3] = {0.f, 0.f, 0.f};
                bspline_derivs4<D>(P.coeffs4, P.mov, ml, m, g);
                double f = (double)P.fixed_data[lin_of<D>(P.fixed, sp)];
                double md = (double)m;
                v[Q_COUNT] = 1.0;
                v[Q_D2] = (md - f) * (md - f);
                v[Q_SF] = f;
                v[Q_SM] = md;
                v[Q_SFF] = f * f;
                v[Q_SMM] = md * md;
                v[Q_SFM] = f * md;
                rec = make_float4(g[0], g[1], D > 2 ? g[2] : 0.f, m);
            }
        }
        samp[t] = rec;
    }
    block_sum<NQ>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) part[(long long)k * gridDim.x + blockIdx.x] = v[k];
}

// ---- statistics (GpuEvaluator.cu:449-571 host loops, on the device, FP64, fixed order) ------
// global statistics from the summed quantities (the host loops of GpuEvaluator.cu:449-571)
__device__ inline void stats_finalize(const double *v, int metric, double *__restrict__ stats)
{
    double n = v[Q_COUNT];
    double st[NS];
    for (int k = 0; k < NS; ++k) st[k] = 0.0;
    st[S_COUNT] = n;
    if (metric == 0) {
        st[S_MEASURE] = v[Q_D2] / n;                       // cu:462-470
        st[S_COEF_F] = -2.0 / n;                           // 2*(m-f)/n  (MSE.cu:291, cu:599-603)
        st[S_COEF_M] = 2.0 / n;
        st[S_COEF_C] = 0.0;
    } else if (metric == 1) {
        double sf = v[Q_SF], sm = v[Q_SM];
        double sff = v[Q_SFF] - sf * sf / n;               // cu:519-524
        double smm = v[Q_SMM] - sm * sm / n;
        double sfm = v[Q_SFM] - sf * sm / n;
        double denom = -1.0 * sqrt(sff * smm);
        st[S_MEASURE] = denom != 0.0 ? sfm / denom : 0.0;
        st[S_MEAN_F] = sf / n;
        st[S_MEAN_M] = sm / n;
        st[S_DENOM] = denom;
        st[S_SFM] = sfm;
        st[S_SMM] = smm;
        // (dF - (sfm/smm) dM)/denom with dF = sum (f - mf) w k gradM, dM = sum (m - mm) w k gradM
        // (NCC.cu:177-179, cu:624-633) == w sum k gradM (a f + b m + c)
        if (denom != 0.0) {
            double rho = sfm / smm;
            st[S_COEF_F] = 1.0 / denom;
            st[S_COEF_M] = -rho / denom;
            st[S_COEF_C] = (-st[S_MEAN_F] + rho * st[S_MEAN_M]) / denom;
        }
    } else {
        st[S_MEASURE] = v[Q_CC] / n;                       // cu:556-570
        st[S_COEF_C] = 1.0 / n;                            // derivatives /= pixelsCounted (cu:642-646)
    }
    st[S_VALID] = 1.0;
    for (int k = 0; k < NS; ++k) stats[k] = st[k];
}

// Sums the NV per-block partials [k][nblocks] with the whole block in a fixed order (L2 reads,
// bypassing L1 so that partials written by other blocks of the same launch are seen).  A thread
// issues kB of its partials of every value before adding them (in the order b = tid, tid + blockDim,
// ...), so the finishing block waits for one L2 latency per kB partials, not one per partial.
template <int NV>
__device__ __forceinline__ void sum_partials(const double *part, int nblocks, double *v, double *sh)
{
    constexpr int kB = 4;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = 0.0;
    for (int b0 = threadIdx.x; b0 < nblocks; b0 += kB * blockDim.x) {
        double x[NV][kB];
#pragma unroll
        for (int k = 0; k < NV; ++k)
#pragma unroll
            for (int u = 0; u < kB; ++u) {
                const int b = b0 + u * (int)blockDim.x;
                x[k][u] = b < nblocks ? __ldcg(part + (long long)k * nblocks + b) : 0.0;
            }
#pragma unroll
        for (int k = 0; k < NV; ++k)
#pragma unroll
            for (int u = 0; u < kB; ++u)
                if (b0 + u * (int)blockDim.x < nblocks) v[k] += x[k][u];
    }
    block_sum<NV>(v, sh);
}

// "Last block finalizes": every block has written its partials; the block that arrives last
// (atomic ticket) returns true, after which it may read all partials.  The ticket counter is
// reset by that block, so the pattern can repeat in the next launch (and in graph replays).
__device__ __forceinline__ bool last_block_arrived(unsigned *counter)
{
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        const unsigned ticket = atomicAdd(counter, 1u);
        last = (ticket == gridDim.x - 1);
        if (last) *counter = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

static __global__ void __launch_bounds__(1024) stats_kernel(const double *__restrict__ part, int nblocks, int metric,
                                                     double *__restrict__ stats)
{
    __shared__ double sh[NQ * 32];
    double v[NQ];
    sum_partials<NQ>(part, nblocks, v, sh);
    if (threadIdx.x == 0) stats_finalize(v, metric, stats);
}

// ---- derivative pass: warp per control point ------------------------------------------------
// Sample box of a control point (MSE.cu:255-263 / NCC.cu:138-146 for 3-D MSE/NCC;
// MSE.cu:273-280 and LCC.cu:236-244 / 722-729 for 2-D and LCC): truncation toward zero,
// clamped to the (subsampled) grid.
template <int D>
__device__ __forceinline__ void derivative_box(const EvalParams &P, bool wide, const double *ip, double support,
                                               int *lo, int *hi)
{
    lo[1] = hi[1] = lo[2] = hi[2] = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double sh = support / P.fixed.s[d];
        if (P.sub != 1) {
            double fs = (double)(float)P.sub;
            if (wide) {
                lo[d] = (int)((ip[d] - sh) / fs);
                hi[d] = (int)((ip[d] + sh) / fs + 1.0);
            } else {
                lo[d] = (int)((ip[d] - sh) / fs + 1.0);
                hi[d] = (int)((ip[d] + sh) / fs);
            }
            lo[d] = clampi(lo[d], 0, P.ss[d] - 1);
            hi[d] = clampi(hi[d], 0, P.ss[d] - 1);
        } else {
            if (wide) {
                lo[d] = (int)(ip[d] - sh);
                hi[d] = (int)(ip[d] + sh + 1.0);
            } else {
                lo[d] = (int)(ip[d] - sh + 1.0);
                hi[d] = (int)(ip[d] + sh);
            }
            lo[d] = clampi(lo[d], 0, P.fixed.n[d] - 1);
            hi[d] = clampi(hi[d], 0, P.fixed.n[d] - 1);
        }
    }
}

// Regularizers of control point j over its control-point box (GpuEvaluatorRegularizers.cu),
// lanes striding the box.  Values accumulate in double, gradients in float.
template <int D, int KIND>
__device__ __forceinline__ void regularizers_of(const EvalParams &P, const DerivParams &Q, const int *j,
                                                long long jl, const double *gp, const PInfo &pj, float4 cj, int lane,
                                                double *val, float *der_rkhs, float *der_rd, float *der_pg)
{
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double sh = pj.support / P.cp.s[d];
        lo[d] = clampi((int)((double)j[d] - sh + 1.0), 0, P.cp.n[d] - 1);
        hi[d] = clampi((int)((double)j[d] + sh), 0, P.cp.n[d] - 1);
    }
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
    const int total = nx * ny * nz;
    const float wj = cj.w;
    const float cjv[3] = {cj.x, cj.y, cj.z};
    const bool rkhs = Q.reg_rkhs > 0.0, rd = Q.reg_rd > 0.0, pg = Q.reg_pg > 0.0;
    const float pgs = (float)Q.pg_scaling;
    for (int t = lane; t < total; t += 32) {
        int x = lo[0] + t % nx;
        int y = lo[1] + (t / nx) % ny;
        int z = lo[2] + t / (nx * ny);
        int ii[3] = {x, y, z};
        float v[3];
#pragma unroll
        for (int d = 0; d < D; ++d) v[d] = -(float)P.cp.s[d] * (float)(ii[d] - j[d]);
        float k;
        if (KIND == kStationary) {
            k = k_eval<KIND, D>(P.K, v, nullptr, pj);
        } else {
            double qi[3] = {(double)x, (double)y, (double)z}, q[3];
            to_global<D>(P.cp, qi, q);
            k = k_eval<KIND, D>(P.K, v, q, pj);
        }
        if (k == 0.0f) continue;
        float4 ci4 = __ldg(P.cpd + lin_of<D>(P.cp, ii));
        float ci[3] = {ci4.x, ci4.y, ci4.z};
        float kw = k * wj;
        if (rkhs) {                                            // Regularizers.cu:68-73
            double dot = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) dot += (double)cjv[d] * (double)ci[d];
            val[R_RKHS] += (double)kw * dot;
#pragma unroll
            for (int d = 0; d < D; ++d) der_rkhs[d] = fmaf(2.0f * kw, ci[d], der_rkhs[d]);
        }
        if (rd) {                                              // Regularizers.cu:141-144
            double l2 = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double e = (double)cjv[d] - (double)ci[d];
                l2 += e * e;
            }
            val[R_RD] += l2 * (double)kw;
#pragma unroll
            for (int d = 0; d < D; ++d) der_rd[d] = fmaf(4.0f * kw, cjv[d] - ci[d], der_rd[d]);
        }
        if (pg) {
            if (D == 3) {                                      // Regularizers.cu:218-237
                float cr0 = ci[1] * cjv[2] - ci[2] * cjv[1];
                float cr1 = ci[2] * cjv[0] - ci[0] * cjv[2];
                float cr2 = ci[0] * cjv[1] - ci[1] * cjv[0];
                double n2 = (double)cr0 * cr0 + (double)cr1 * cr1 + (double)cr2 * cr2;
                double s = (double)pgs;
                val[R_PG] += (double)kw * s * s / 2.0 * log(1.0 + n2 / s);
                float den = 2.0f * ((float)n2 / pgs + 1.0f);
                float dp0 = 2.0f * ci[2] * (ci[2] * cjv[0] - ci[0] * cjv[2]) - 2.0f * ci[1] * (ci[0] * cjv[1] - ci[1] * cjv[0]);
                float dp1 = 2.0f * ci[0] * (ci[0] * cjv[1] - ci[1] * cjv[0]) - 2.0f * ci[2] * (ci[1] * cjv[2] - ci[2] * cjv[1]);
                float dp2 = 2.0f * ci[1] * (ci[1] * cjv[2] - ci[2] * cjv[1]) - 2.0f * ci[0] * (ci[2] * cjv[0] - ci[0] * cjv[2]);
                der_pg[0] = fmaf(2.0f * kw, pgs * dp0 / den, der_pg[0]);
                der_pg[1] = fmaf(2.0f * kw, pgs * dp1 / den, der_pg[1]);
                der_pg[2] = fmaf(2.0f * kw, pgs * dp2 / den, der_pg[2]);
            } else {                                           // Regularizers.cu:447-459
                float val2d = ci[0] * cjv[1] - ci[1] * cjv[0];
                double v2 = (double)val2d * val2d;
                double s = (double)pgs;
                val[R_PG] += (double)kw * s * s / 2.0 * log(1.0 + v2 / s);
                float factor = (float)v2 / pgs + 1.0f;
                der_pg[0] = fmaf(2.0f * kw, -pgs * ci[1] * val2d / factor, der_pg[0]);
                der_pg[1] = fmaf(2.0f * kw, pgs * ci[0] * val2d / factor, der_pg[1]);
            }
        }
    }
}

// LCC window statistics and derivative accumulators of one sample (LCC.cu:296-530).
template <int D, int KIND>
__device__ __forceinline__ void lcc_sample_derivative(const EvalParams &P, const DerivParams &Q, const double *gp,
                                                      const double *pt, float *der)
{
    PInfo ps;
    pinfo_at<KIND, D>(P.K, pt, ps);
    double fl[3];
    to_local<D>(P.fixed, pt, fl);
    int flo[3] = {0, 0, 0}, fhi[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double sh = ps.support / P.fixed.s[d];
        flo[d] = clampi((int)(fl[d] - sh + 1.0), 0, P.fixed.n[d] - 1);
        fhi[d] = clampi((int)(fl[d] + sh), 0, P.fixed.n[d] - 1);
    }
    const bool swapped = (D == 3 && KIND != kStationary);
    const float4 *dense = swapped ? Q.dense_sw : Q.dense;
    const unsigned char *dense_in = swapped ? Q.dense_sw_in : Q.dense_in;
    LccWindow W;
    double mkcka[3] = {0, 0, 0}, mkcmkcka[3] = {0, 0, 0}, fkcmka[3] = {0, 0, 0};
    for (int z = flo[2]; z <= fhi[2]; z += P.nbh)
        for (int y = flo[1]; y <= fhi[1]; y += P.nbh)
            for (int x = flo[0]; x <= fhi[0]; x += P.nbh) {
                int ni[3] = {x, y, z};
                double nf[3] = {(double)x, (double)y, (double)z}, q[3];
                to_global<D>(P.fixed, nf, q);
                // the tensor kind's kernel value comes from the texel's cached inverse and factor,
                // so only the support radius is looked up here
                constexpr bool cached = (D == 3 && KIND == kWeightTensor);
                PInfo pn;
                if (cached)
                    pn.support = support_at<KIND, D>(P.K, q);
                else
                    pinfo_at<KIND, D>(P.K, q, pn);
                // neighborhoodWeight with the neighbour's support passed as float (LCC.cu:28-35)
                double kwf = lcc_weight_base<D>(pt, q, (double)(float)pn.support);
                if (kwf <= 0.0) continue;
                double kw = __dmul_rn(kwf, kwf);
                long long nl = lin_of<D>(P.fixed, ni);
                if (!dense_in[nl]) continue;
                // ka = k(cp, n) with the neighbour's kernel information (LCC.cu:449-461)
                float v[3];
#pragma unroll
                for (int d = 0; d < D; ++d) v[d] = (float)(gp[d] - q[d]);
                float ka;
                if (cached)
                    ka = aniso_self_eval(P.K, v, Q.acache + 3 * nl);
                else
                    ka = k_eval<KIND, D>(P.K, v, q, pn);
                float4 rec = dense[nl];
                double mv = __dmul_rn((double)rec.w, kw);
                double fv = __dmul_rn(kw, (double)P.fixed_data[nl]);
                W.add(fv, mv);
                double g[3] = {rec.x, rec.y, rec.z};
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    double gk = g[d] * kw * (double)ka;
                    mkcmkcka[d] += mv * gk;
                    mkcka[d] += gk;
                    fkcmka[d] += fv * gk;
                }
            }
    if (W.n > 0) {
        double msf = W.msf(), msm = W.msm();
        double d1 = W.d1();
        double u = __dmul_rn(d1, W.d2());
        double vv = W.cross();
        if (fabs(u) > 1e-16) {
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double vd = 2.0 * vv * (fkcmka[d] - msf * mkcka[d]);
                double ud = 2.0 * d1 * (mkcmkcka[d] - msm * mkcka[d]);
                der[d] += (float)(-(vd * u - ud * (vv * vv)) / (u * u));
            }
        }
    }
}

// SPLIT = 1: one warp per control point (8 per block).  SPLIT = 8 (few control points, MSE/NCC):
// one block per control point, its 8 warps take interleaved z-planes of the support box and their
// sums are combined in warp order, so results stay deterministic.
template <int D, int KIND, int SPLIT = 1>
__global__ void __launch_bounds__(256) derivative_kernel(EvalParams P, DerivParams Q)
{
    __shared__ double shv[NR][8];
    __shared__ float sacc[8][3];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long j_lin = SPLIT > 1 ? (long long)blockIdx.x : (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    double val[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) val[k] = 0.0;
    if (j_lin < P.C) {
        int j[3];
        cell_of<D>(P.cp.n, j_lin, j);
        double jf[3] = {(double)j[0], (double)j[1], (double)j[2]}, gp[3], ip[3];
        to_global<D>(P.cp, jf, gp);
        const float4 cj = __ldg(P.cpd + j_lin);
        PInfo pj;
        pinfo_at<KIND, D>(P.K, gp, pj);
        float acc[3] = {0.f, 0.f, 0.f};
        const double *st = Q.stats;
        if (Q.metric != 2) {
            const bool wide = (D == 3);
            to_local<D>(P.fixed, gp, ip);
            int lo[3], hi[3];
            derivative_box<D>(P, wide, ip, pj.support, lo, hi);
            const float cf = (float)st[S_COEF_F], cm = (float)st[S_COEF_M], cc = (float)st[S_COEF_C];
            const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
            const int per_plane = nx * ny;
            const int sub = P.sub;
            // offsets relative to the first sample cell of the box
            int base_pos[3] = {lo[0] * sub, lo[1] * sub, lo[2] * sub};
            float base[3], hs[3];
#pragma unroll
            for (int d = 0; d < D; ++d) {
                base[d] = (float)(gp[d] - (P.fixed.o[d] + P.fixed.s[d] * (double)base_pos[d]));
                hs[d] = (float)P.fixed.s[d];
            }
            for (int zz = SPLIT > 1 ? wib : 0; zz < nz; zz += SPLIT) {
                const int z = lo[2] + zz;
                int x = lane % nx, y = lane / nx;              // lane position in the (y,x) plane
                for (int t = lane; t < per_plane; t += 32) {
                    const int cx = lo[0] + x, cy = lo[1] + y;
                    long long idx;
                    int pos[3] = {cx, cy, z};
                    if (sub != 1) {
                        idx = cx + (long long)P.ss[0] * (cy + (long long)P.ss[1] * z);
                        uint32_t s = __ldg(P.shifts + idx);
#pragma unroll
                        for (int d = 0; d < D; ++d) pos[d] = pos[d] * sub + (int)((s >> (8 * d)) & 0xffu);
                    } else {
                        idx = lin_of<D>(P.fixed, pos);
                    }
                    float4 rec = __ldg(Q.samp + idx);
                    if (rec.x != 0.f || rec.y != 0.f || rec.z != 0.f) {
                        float v[3];
                        v[0] = base[0] - hs[0] * (float)(pos[0] - base_pos[0]);
                        if (D > 1) v[1] = base[1] - hs[1] * (float)(pos[1] - base_pos[1]);
                        if (D > 2) v[2] = base[2] - hs[2] * (float)(pos[2] - base_pos[2]);
                        float k;
                        if (KIND == kStationary) {
                            k = k_eval<KIND, D>(P.K, v, nullptr, pj);
                        } else {
                            double pf[3] = {(double)pos[0], (double)pos[1], (double)pos[2]}, q[3];
                            to_global<D>(P.fixed, pf, q);
                            k = k_eval<KIND, D>(P.K, v, q, pj);
                        }
                        if (k != 0.0f) {
                            // box-window LCC: the texel's coefficient from its windows (times 1/count)
                            float coef;
                            if (Q.boxcoef) {
                                coef = cc * __ldg(Q.boxcoef + idx) * k;
                            } else {
                                const float f = __ldg(P.fixed_data + lin_of<D>(P.fixed, pos));
                                coef = fmaf(cf, f, fmaf(cm, rec.w, cc)) * k;
                            }
                            acc[0] = fmaf(coef, rec.x, acc[0]);
                            acc[1] = fmaf(coef, rec.y, acc[1]);
                            if (D > 2) acc[2] = fmaf(coef, rec.z, acc[2]);
                        }
                    }
                    x += 32;
                    while (x >= nx) { x -= nx; ++y; }
                }
            }
        } else if (SPLIT == 1) {
            // LCC: lanes over the samples of the box, each lane walks its sample's window
            to_local<D>(P.fixed, gp, ip);
            int lo[3], hi[3];
            derivative_box<D>(P, false, ip, pj.support, lo, hi);
            const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1, nz = hi[2] - lo[2] + 1;
            const int total = nx * ny * nz;
            for (int t = lane; t < total; t += 32) {
                int cell[3] = {lo[0] + t % nx, lo[1] + (t / nx) % ny, lo[2] + t / (nx * ny)};
                int pos[3] = {cell[0], cell[1], cell[2]};
                if (P.sub != 1) {
                    long long idx = cell[0] + (long long)P.ss[0] * (cell[1] + (long long)P.ss[1] * cell[2]);
                    uint32_t s = __ldg(P.shifts + idx);
#pragma unroll
                    for (int d = 0; d < D; ++d) pos[d] = cell[d] * P.sub + (int)((s >> (8 * d)) & 0xffu);
                }
                double pf[3] = {(double)pos[0], (double)pos[1], (double)pos[2]}, pt[3];
                to_global<D>(P.fixed, pf, pt);
                lcc_sample_derivative<D, KIND>(P, Q, gp, pt, acc);
            }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) acc[d] = warp_sum(acc[d]);
        if (SPLIT > 1) {                                   // the block's warps in a fixed order
            if (lane == 0)
#pragma unroll
                for (int d = 0; d < 3; ++d) sacc[wib][d] = acc[d];
            __syncthreads();
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                float t = 0.f;
                for (int w = 0; w < SPLIT; ++w) t += sacc[w][d];
                acc[d] = t;
            }
        }

        float drk[3] = {0.f, 0.f, 0.f}, drd[3] = {0.f, 0.f, 0.f}, dpg[3] = {0.f, 0.f, 0.f};
        if ((SPLIT == 1 || wib == 0) && (Q.reg_rkhs > 0.0 || Q.reg_rd > 0.0 || Q.reg_pg > 0.0)) {
            regularizers_of<D, KIND>(P, Q, j, j_lin, gp, pj, cj, lane, val, drk, drd, dpg);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                drk[d] = warp_sum(drk[d]);
                drd[d] = warp_sum(drd[d]);
                dpg[d] = warp_sum(dpg[d]);
            }
#pragma unroll
            for (int k = R_RKHS; k <= R_PG; ++k) val[k] = warp_sum(val[k]);
        }
        if (lane == 0 && (SPLIT == 1 || wib == 0)) {
            const double n = st[S_COUNT];
            double pc[3] = {0, 0, 0}, pn2 = 0.0;
            if (Q.with_metric) {
#pragma unroll
                for (int d = 0; d < D; ++d) {
                    pc[d] = Q.params[j_lin + d * P.C];
                    pn2 += pc[d] * pc[d];
                }
            }
            const double pnorm = sqrt(pn2);
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double g;
                if (Q.metric == 1)
                    g = st[S_DENOM] != 0.0 ? (double)cj.w * (double)acc[d] : 0.0;
                else if (Q.metric == 0 || Q.metric == 3)
                    g = (double)cj.w * (double)acc[d];
                else
                    g = (double)acc[d] / n;                    // LCC derivative omits w_i (LCC.cu:518)
                if (Q.reg_rkhs > 0.0) g += (double)drk[d] * Q.reg_rkhs;
                if (Q.reg_rd > 0.0) g += (double)drd[d] * Q.reg_rd;
                if (Q.reg_pg > 0.0) g += (double)dpg[d] * Q.reg_pg;
                if (Q.with_metric) {
                    const double par = pc[d];
                    if (Q.reg_l1 > 0.0) {                      // metric hxx:447-466
                        const double w = Q.reg_l1;
                        if (fabs(par) > 0.0) g += w * (par < 0.0 ? -1.0 : 1.0);
                        else if (g < -w) g += w;
                        else if (g > w) g -= w;
                        else g = 0.0;
                    }
                    if (Q.reg_l2 > 0.0) g += Q.reg_l2 * 2.0 * par;   // hxx:482-485
                    if (Q.reg_l21 > 0.0) {                     // hxx:504-521
                        const double w = Q.reg_l21;
                        if (pnorm > 0.0) g += w * par / pnorm;
                        else if (g < -w) g += w;
                        else if (g > w) g -= w;
                        else g = 0.0;
                    }
                    if (Q.negate) g = -g;
                }
                Q.deriv[j_lin + d * P.C] = g;
            }
            if (Q.with_metric) {
                double l1 = 0.0;
#pragma unroll
                for (int d = 0; d < D; ++d) l1 += fabs(pc[d]);
                // each term is computed only when its weight is positive (metric hxx:431,469,491)
                val[R_L1] = Q.reg_l1 > 0.0 ? l1 : 0.0;
                val[R_L2] = Q.reg_l2 > 0.0 ? pn2 : 0.0;
                val[R_L21] = Q.reg_l21 > 0.0 ? pnorm : 0.0;
            }
        }
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NR; ++k) shv[k][wib] = val[k];
    __syncthreads();
    if (threadIdx.x < NR) {
        double s = 0.0;
        const int nw = blockDim.x >> 5;
        for (int w = 0; w < nw; ++w) s += shv[threadIdx.x][w];
        Q.rpart[(long long)threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}

// Regularizer values only (getValue, GpuEvaluator.cu:300-353) over the control-point grid.
template <int D, int KIND>
__global__ void __launch_bounds__(256) regvalue_kernel(EvalParams P, DerivParams Q)
{
    __shared__ double shv[NR][8];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const long long j_lin = (long long)blockIdx.x * (blockDim.x >> 5) + wib;
    double val[NR];
#pragma unroll
    for (int k = 0; k < NR; ++k) val[k] = 0.0;
    if (j_lin < P.C) {
        int j[3];
        cell_of<D>(P.cp.n, j_lin, j);
        double jf[3] = {(double)j[0], (double)j[1], (double)j[2]}, gp[3];
        to_global<D>(P.cp, jf, gp);
        const float4 cj = __ldg(P.cpd + j_lin);
        PInfo pj;
        pinfo_at<KIND, D>(P.K, gp, pj);
        float drk[3] = {0.f, 0.f, 0.f}, drd[3] = {0.f, 0.f, 0.f}, dpg[3] = {0.f, 0.f, 0.f};
        regularizers_of<D, KIND>(P, Q, j, j_lin, gp, pj, cj, lane, val, drk, drd, dpg);
#pragma unroll
        for (int k = R_RKHS; k <= R_PG; ++k) val[k] = warp_sum(val[k]);
        if (lane == 0 && Q.with_metric) {
            double l1 = 0.0, n2 = 0.0;
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double par = Q.params[j_lin + d * P.C];
                l1 += fabs(par);
                n2 += par * par;
            }
            val[R_L1] = Q.reg_l1 > 0.0 ? l1 : 0.0;
            val[R_L2] = Q.reg_l2 > 0.0 ? n2 : 0.0;
            val[R_L21] = Q.reg_l21 > 0.0 ? sqrt(n2) : 0.0;
        }
    }
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NR; ++k) shv[k][wib] = val[k];
    __syncthreads();
    if (threadIdx.x < NR) {
        double s = 0.0;
        const int nw = blockDim.x >> 5;
        for (int w = 0; w < nw; ++w) s += shv[threadIdx.x][w];
        Q.rpart[(long long)threadIdx.x * gridDim.x + blockIdx.x] = s;
    }
}

// final scalars: measure, regularizer values, weighted sum (metric hxx:531-538, 572)
// fault: sticky failure word of the tensor-core kernels (NULL when none ran); copied to
// out[O_FAULT] so that the host sees it with the result.
__device__ inline void result_finalize(const double *stats, const double *v, double w_rkhs, double w_rd,
                                       double w_pg, double w_l1, double w_l21, double w_l2, double *__restrict__ out,
                                       const unsigned *fault = nullptr)
{
    double reg = 0.0;
    if (w_l1 > 0) reg += w_l1 * v[R_L1];
    if (w_l21 > 0) reg += w_l21 * v[R_L21];
    if (w_l2 > 0) reg += w_l2 * v[R_L2];
    if (w_rkhs > 0) reg += w_rkhs * v[R_RKHS];
    if (w_rd > 0) reg += w_rd * v[R_RD];
    if (w_pg > 0) reg += w_pg * v[R_PG];
    out[O_MEASURE] = stats[S_MEASURE];
    out[O_RKHS] = v[R_RKHS];
    out[O_RD] = v[R_RD];
    out[O_PG] = v[R_PG];
    out[O_L1] = v[R_L1];
    out[O_L21] = v[R_L21];
    out[O_L2] = v[R_L2];
    out[O_REG] = reg;
    out[O_VALUE] = stats[S_MEASURE] + reg;
    out[O_COUNT] = stats[S_COUNT];
    out[O_FAULT] = fault ? (double)*(const volatile unsigned *)fault : 0.0;
}

static __global__ void __launch_bounds__(256) result_kernel(const double *__restrict__ stats, const double *__restrict__ rpart,
                                                     int nblocks, double w_rkhs, double w_rd, double w_pg, double w_l1,
                                                     double w_l21, double w_l2, double *__restrict__ out,
                                                     const unsigned *fault)
{
    __shared__ double sh[NR * 32];
    double v[NR];
    if (rpart) {
        sum_partials<NR>(rpart, nblocks, v, sh);
    } else {
#pragma unroll
        for (int k = 0; k < NR; ++k) v[k] = 0.0;
    }
    if (threadIdx.x == 0) result_finalize(stats, v, w_rkhs, w_rd, w_pg, w_l1, w_l21, w_l2, out, fault);
}

// ---- LCC: dense fields and per-sample values --------------------------------------------------
// (grad M, m) and the inside flag at the fixed texels the LCC windows read: the neighbour
// transforms of the reference's LCC windows (LCC.cu:112-176) evaluated once per texel instead of
// once per window.
template <int D, int KIND, bool SWAP>
__device__ __forceinline__ void dense_texel(const EvalParams &P, long long t, float4 *__restrict__ dense,
                                            unsigned char *__restrict__ dense_in)
{
    int c[3];
    cell_of<D>(P.fixed.n, t, c);
    double fi[3] = {(double)c[0], (double)c[1], (double)c[2]}, p[3], ml[3];
    to_global<D>(P.fixed, fi, p);
    moving_local<D, KIND, SWAP>(P, p, ml);
    float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
    unsigned char in = 0;
    if (bspline_inside<D>(P.mov, ml)) {
        float m, g[3] = {0.f, 0.f, 0.f};
        bspline_derivs4<D>(P.coeffs4, P.mov, ml, m, g);
        rec = make_float4(g[0], g[1], D > 2 ? g[2] : 0.f, m);
        in = 1;
    }
    dense[t] = rec;
    dense_in[t] = in;
}

__device__ __forceinline__ void lcc_mark(unsigned *__restrict__ bits, int *__restrict__ list, int *__restrict__ count,
                                         long long i)
{
    const unsigned bit = 1u << (i & 31);
    if (!(atomicOr(bits + (i >> 5), bit) & bit)) list[atomicAdd(count, 1)] = (int)i;
}

// The texels that the value and derivative kernels read from the dense fields: each sample's own
// texel and every window point with a nonzero neighbourhood weight -- the same positions, bounds
// and weight test as lcc_value_kernel and lcc_sample_derivative (the derivative also walks the
// windows of samples whose shifted position lies past the image) -- listed once each.  With
// subsampled samples and strided windows this is a small part of the image (at 1.5 mm, sampling
// 32 and stride 48: ~10^4 of 10^7 texels).  The list's order does not matter: a listed texel
// writes only its own entry.
template <int D, int KIND>
__global__ void __launch_bounds__(256) lcc_mark_kernel(EvalParams P, unsigned *__restrict__ bits,
                                                       int *__restrict__ list, int *__restrict__ count)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.Ns) return;
    int c[3], sp[3];
    cell_of<D>(P.ss, t, c);
    bool inside = true;
#pragma unroll
    for (int d = 0; d < 3; ++d) sp[d] = c[d];
    if (P.sub != 1) {
        const uint32_t s = P.shifts[t];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            sp[d] = c[d] * P.sub + (int)((s >> (8 * d)) & 0xffu);
            if (sp[d] >= P.fixed.n[d]) inside = false;
        }
    }
    double fi[3] = {(double)sp[0], (double)sp[1], (double)sp[2]}, p[3];
    to_global<D>(P.fixed, fi, p);
    if (inside) lcc_mark(bits, list, count, lin_of<D>(P.fixed, sp));
    PInfo pi;
    pinfo_at<KIND, D>(P.K, p, pi);
    double fl[3];
    to_local<D>(P.fixed, p, fl);
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double shf = pi.support / P.fixed.s[d];
        lo[d] = clampi((int)(fl[d] - shf + 1.0), 0, P.fixed.n[d] - 1);
        hi[d] = clampi((int)(fl[d] + shf), 0, P.fixed.n[d] - 1);
    }
    for (int z = lo[2]; z <= hi[2]; z += P.nbh)
        for (int y = lo[1]; y <= hi[1]; y += P.nbh)
            for (int x = lo[0]; x <= hi[0]; x += P.nbh) {
                int ni[3] = {x, y, z};
                double nf[3] = {(double)x, (double)y, (double)z}, q[3];
                to_global<D>(P.fixed, nf, q);
                double sup;
                if (KIND == kStationary) {
                    sup = (double)P.K.support_min;
                } else {
                    PInfo pn;
                    pinfo_at<KIND, D>(P.K, q, pn);
                    sup = (double)(float)pn.support;
                }
                if (lcc_weight_base<D>(p, q, sup) <= 0.0) continue;
                lcc_mark(bits, list, count, lin_of<D>(P.fixed, ni));
            }
}

// the dense fields at the listed texels (grid-strided over the count the marking kernel wrote);
// acache (3-D weight tensors, swapped pass) also takes each listed texel's aniso_self_cache, which
// the derivative's window walk reads at the same texels
template <int D, int KIND, bool SWAP>
__global__ void __launch_bounds__(256) dense_list_kernel(EvalParams P, const int *__restrict__ list,
                                                         const int *__restrict__ count, float4 *__restrict__ dense,
                                                         unsigned char *__restrict__ dense_in,
                                                         float4 *__restrict__ acache = nullptr)
{
    const int n = *count;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int t = list[i];
        dense_texel<D, KIND, SWAP>(P, t, dense, dense_in);
        if (D == 3 && KIND == kWeightTensor && acache) {
            int c[3];
            cell_of<D>(P.fixed.n, t, c);
            double nf[3] = {(double)c[0], (double)c[1], (double)c[2]}, q[3];
            to_global<D>(P.fixed, nf, q);
            PInfo pn;
            pinfo_at<KIND, D>(P.K, q, pn);
            aniso_self_cache(pn.cov, acache + 3 * (long long)t);
        }
    }
}

// LCC value per sample (LCC.cu:38-204) from the dense fields.
template <int D, int KIND>
__global__ void __launch_bounds__(256) lcc_value_kernel(EvalParams P, const float4 *__restrict__ dense,
                                                        const unsigned char *__restrict__ dense_in,
                                                        double *__restrict__ part)
{
    __shared__ double sh[NQ * 32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = 0.0;
    if (t < P.Ns) {
        int sp[3];
        if (sample_pos<D>(P, t, sp)) {
            double fi[3] = {(double)sp[0], (double)sp[1], (double)sp[2]}, p[3];
            to_global<D>(P.fixed, fi, p);
            long long pl = lin_of<D>(P.fixed, sp);
            v[Q_COUNT] = dense_in[pl] ? 1.0 : 0.0;
            PInfo pi;
            pinfo_at<KIND, D>(P.K, p, pi);
            double fl[3];
            to_local<D>(P.fixed, p, fl);
            int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
#pragma unroll
            for (int d = 0; d < D; ++d) {
                double shf = pi.support / P.fixed.s[d];
                lo[d] = clampi((int)(fl[d] - shf + 1.0), 0, P.fixed.n[d] - 1);
                hi[d] = clampi((int)(fl[d] + shf), 0, P.fixed.n[d] - 1);
            }
            LccWindow W;
            for (int z = lo[2]; z <= hi[2]; z += P.nbh)
                for (int y = lo[1]; y <= hi[1]; y += P.nbh)
                    for (int x = lo[0]; x <= hi[0]; x += P.nbh) {
                        int ni[3] = {x, y, z};
                        double nf[3] = {(double)x, (double)y, (double)z}, q[3];
                        to_global<D>(P.fixed, nf, q);
                        double sup;
                        if (KIND == kStationary) {
                            sup = (double)P.K.support_min;
                        } else {
                            PInfo pn;
                            pinfo_at<KIND, D>(P.K, q, pn);
                            sup = (double)(float)pn.support;
                        }
                        double kwf = lcc_weight_base<D>(p, q, sup);
                        if (kwf <= 0.0) continue;
                        double kw = __dmul_rn(kwf, kwf);
                        long long nl = lin_of<D>(P.fixed, ni);
                        if (!dense_in[nl]) continue;
                        W.add(__dmul_rn(kw, (double)P.fixed_data[nl]), __dmul_rn((double)dense[nl].w, kw));
                    }
            v[Q_CC] = W.value();
        }
    }
    block_sum<NQ>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) part[(long long)k * gridDim.x + blockIdx.x] = v[k];
}

// ---- displacement field (DisplacementField.cu:24-127) -----------------------------------------
template <int D, int KIND>
__global__ void __launch_bounds__(256) displacement_kernel(EvalParams P, double *__restrict__ out)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long N = (long long)P.fixed.n[0] * P.fixed.n[1] * P.fixed.n[2];
    if (t >= N) return;
    int c[3];
    cell_of<D>(P.fixed.n, t, c);
    double fi[3] = {(double)c[0], (double)c[1], (double)c[2]}, p[3];
    to_global<D>(P.fixed, fi, p);
    double u[3] = {0.0, 0.0, 0.0};
    if (P.has_df) {
        long long i = nearest_index<D>(P.df, p);
        if (i >= 0) {
            float4 v = P.dfd[i];
            u[0] = v.x; u[1] = v.y; u[2] = v.z;
        }
    }
    PInfo pi;
    pinfo_at<KIND, D>(P.K, p, pi);
    float uf[3] = {0.f, 0.f, 0.f};
    transform_add<D, KIND, false>(P, p, pi, uf);
#pragma unroll
    for (int d = 0; d < D; ++d) out[t * D + d] = u[d] + (double)uf[d];
}

// ---- small helpers ----------------------------------------------------------------------------
// Weighted control points w alpha as planes for the tensor-core transform's tiled loads:
// [D][n2][n1][nxp] floats, one plane per component.  Rows are padded to nxp (a multiple of 4
// floats, the tiled loads' stride rule); the padding stays zero.  p == nullptr: not used.
struct RegionPlanes {
    float *p;
    int n0, nxp, D;
    long long plane;         // floats per plane
};

__device__ __forceinline__ void write_region_planes(const RegionPlanes &rp, long long i, const float4 &r)
{
    if (!rp.p) return;
    const long long yz = i / rp.n0;
    const int x = (int)(i - yz * rp.n0);
    const long long row = yz * rp.nxp;                 // yz = y + n1 z
    const float v[3] = {r.w * r.x, r.w * r.y, r.w * r.z};
    for (int k = 0; k < rp.D; ++k) {
        rp.p[k * rp.plane + row + x] = v[k];
    }
}

// pack AoS doubles (alpha) + weights into float4 records
static __global__ void pack_cp_aos(const double *__restrict__ cp, const double *__restrict__ cpw, long long C, int D,
                            float4 *__restrict__ out, RegionPlanes rp)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    float4 r;
    r.x = (float)cp[i * D];
    r.y = (float)cp[i * D + 1];
    r.z = D > 2 ? (float)cp[i * D + 2] : 0.f;
    r.w = (float)cpw[i];
    out[i] = r;
    write_region_planes(rp, i, r);
}

// pack planar parameters (metric level, itkTransformAdapter.hxx:202-236) + weights
static __global__ void pack_cp_planar(const double *__restrict__ params, const double *__restrict__ cpw, long long C, int D,
                               float4 *__restrict__ out, RegionPlanes rp)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    float4 r;
    r.x = (float)params[i];
    r.y = (float)params[i + C];
    r.z = D > 2 ? (float)params[i + 2 * C] : 0.f;
    r.w = (float)cpw[i];
    out[i] = r;
    write_region_planes(rp, i, r);
}

// pack_cp_planar reading the parameters from host memory the device maps (the pinned staging
// buffer), keeping a device copy of them in `copy`.
static __global__ void pack_cp_planar_copy(const double *__restrict__ params, const double *__restrict__ cpw,
                                           long long C, int D, float4 *__restrict__ out, double *__restrict__ copy,
                                           RegionPlanes rp)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C) return;
    const double px = params[i], py = params[i + C], pz = D > 2 ? params[i + 2 * C] : 0.0;
    copy[i] = px;
    copy[i + C] = py;
    if (D > 2) copy[i + 2 * C] = pz;
    const float4 r = make_float4((float)px, (float)py, (float)pz, (float)cpw[i]);
    out[i] = r;
    write_region_planes(rp, i, r);
}

// grid shifts of the PCG32 stream (GpuEvaluator.cu:107-118): texel t takes draws D*t..D*t+D-1
// counted from `state`; shift = int(nextI/double(UINT_MAX) * subsample).
static __global__ void shifts_kernel(unsigned long long state, RngJump J, long long Ns, int D, int sub,
                              uint32_t *__restrict__ shifts)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Ns) return;
    unsigned long long s = lcg_advance(state, (unsigned long long)t * D, J);
    uint32_t packed = 0;
    for (int d = 0; d < D; ++d) {
        unsigned out = pcg32_output(s);
        s = s * 6364136223846793005ULL + 1ULL;
        double f = (double)out / 4294967295.0;
        int sh = (int)(f * (double)sub);
        packed |= (uint32_t)sh << (8 * d);
    }
    shifts[t] = packed;
}

// ---- evaluator set-up on the device: the caller's double images become the kernels' float copies
static __global__ void to_float_kernel(const double *__restrict__ src, long long n, float *__restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = (float)src[i];
}

// row-expanded coefficients: c4[i] = (c[i], c[i + 1], c[i + 2], c[i + 3]), zeros past the end
static __global__ void expand_rows_kernel(const float *__restrict__ c, long long n, float4 *__restrict__ c4)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        c4[i] = make_float4(c[i], i + 1 < n ? c[i + 1] : 0.f, i + 2 < n ? c[i + 2] : 0.f, i + 3 < n ? c[i + 3] : 0.f);
}

// displacement field (D doubles per texel) as float4 (x, y, z, 0)
static __global__ void field_to_float4_kernel(const double *__restrict__ src, long long n, int D, float4 *__restrict__ dst)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        dst[i] = make_float4((float)src[i * D], (float)src[i * D + 1], D > 2 ? (float)src[i * D + 2] : 0.f, 0.f);
}

}  // namespace skm
