// skm_lccbox.cuh -- box-window local correlation: every texel is a window centre, its window the
// (2r+1)^D box around it (r = 2: 5^3) clipped at the image border, over the texels whose warped
// position is inside the moving image.  An extension beside the reference's LCC, whose windows are
// the kernel support weighted by (1 - (r/s)^10)^2 (include/cuda/GpuEvaluatorLCC.cu:28-35,94-191).
//
// Per counted centre x: cov = S_fm - S_f S_m / n, vf = S_ff - S_f^2 / n, vm = S_mm - S_m^2 / n,
// lcc_x = cov^2 / (vf vm), value = -(1/count) sum_x lcc_x.  d lcc_x / d m(y) = A_x (f(y) - mu_f(x))
// + B_x (m(y) - mu_m(x)) with A = 2 cov / (vf vm), B = -2 cov^2 / (vf vm^2), and the box is
// symmetric, so texel y's coefficient is a box sum over the centres around it:
//     c(y) = -(f(y) S_A(y) + m(y) S_B(y) - S_E(y)),   E = A mu_f + B mu_m,
// which the generic derivative kernel turns into d_j = w_j / count sum_y k(y, c_j) c(y) grad M(y).
//
// Both box sums are separable: 5-tap sums along x, then y, then z, one kernel per axis, all in FP64
// (the moments of CT-like intensities, ~1e3 with ~20 of noise, cancel in vf = S_ff - S_f^2 / n far
// beyond FP32; their products of FP32 values are exact in FP64).  A direct 5-tap sum per output costs
// two loads more than a prefix-sum difference and keeps every output's sum in one fixed order, with
// no long running sums.  A centre counts when both variances exceed 1e-12 of their raw second moments,
// so that flat windows are left out however their sums round.  Requires subsample 1 (every texel
// is a sample, and samples are texels in linear order).
#pragma once

#include "skm_kernels.cuh"

namespace skm {

constexpr int kBoxR = 2;                 // window half-width: 5^D texels
constexpr int kBoxMoments = 6;           // count, S_f, S_m, S_ff, S_mm, S_fm
constexpr double kBoxRelEps = 1e-12;

// (grad M, m) of every texel and whether its warped position is inside the moving image
template <int D, int KIND>
__global__ void __launch_bounds__(256) box_texel_kernel(EvalParams P, float4 *__restrict__ samp,
                                                        unsigned char *__restrict__ in)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < P.Ns;
         t += (long long)gridDim.x * blockDim.x) {
        int sp[3];
        float4 rec = make_float4(0.f, 0.f, 0.f, 0.f);
        unsigned char ok = 0;
        if (sample_pos<D>(P, t, sp)) {
            double fi[3] = {(double)sp[0], (double)sp[1], (double)sp[2]}, p[3], ml[3];
            to_global<D>(P.fixed, fi, p);
            moving_local<D, KIND, false>(P, p, ml);
            if (bspline_inside<D>(P.mov, ml)) {
                float m, g[3] = {0.f, 0.f, 0.f};
                bspline_derivs4<D>(P.coeffs4, P.mov, ml, m, g);
                rec = make_float4(g[0], g[1], D > 2 ? g[2] : 0.f, m);
                ok = 1;
            }
        }
        samp[t] = rec;
        in[t] = ok;
    }
}

// window moments, pass 1: 5-tap sums along x of (1, f, m, f^2, m^2, f m) over the inside texels;
// out planar [moment][texel]
__global__ void __launch_bounds__(256) box_moments_x_kernel(const float *__restrict__ fixed,
                                                            const float4 *__restrict__ samp,
                                                            const unsigned char *__restrict__ in, long long N, int nx,
                                                            double *__restrict__ out)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(t % nx);
        double s[kBoxMoments] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int o = -kBoxR; o <= kBoxR; ++o) {
            if (x + o < 0 || x + o >= nx) continue;
            const long long u = t + o;
            if (!in[u]) continue;
            const double f = (double)fixed[u], m = (double)samp[u].w;
            s[0] += 1.0;
            s[1] += f;
            s[2] += m;
            s[3] += f * f;
            s[4] += m * m;
            s[5] += f * m;
        }
#pragma unroll
        for (int k = 0; k < kBoxMoments; ++k) out[k * N + t] = s[k];
    }
}

// 5-tap sums of NF planar FP64 fields along one axis (texel stride `stride`, `n_axis` texels)
template <int NF>
__global__ void __launch_bounds__(256) box_axis_kernel(const double *__restrict__ src, double *__restrict__ dst,
                                                       long long N, long long stride, int n_axis)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        const int a = (int)((t / stride) % n_axis);
        double s[NF];
#pragma unroll
        for (int k = 0; k < NF; ++k) s[k] = 0.0;
#pragma unroll
        for (int o = -kBoxR; o <= kBoxR; ++o) {
            if (a + o < 0 || a + o >= n_axis) continue;
            const long long u = t + o * stride;
#pragma unroll
            for (int k = 0; k < NF; ++k) s[k] += src[k * N + u];
        }
#pragma unroll
        for (int k = 0; k < NF; ++k) dst[k * N + t] = s[k];
    }
}

// per centre: lcc, and the derivative factors A, B, E = A mu_f + B mu_m (zero where the centre does
// not count), planar into abe; per-block FP64 partials of the count and of -lcc (the statistics
// kernel's LCC slots), the sum over a block in a fixed order
__global__ void __launch_bounds__(256) box_centers_kernel(const double *__restrict__ mom,
                                                          const unsigned char *__restrict__ in, long long N,
                                                          double *__restrict__ abe, double *__restrict__ part)
{
    __shared__ double sh[NQ * 32];
    double v[NQ];
#pragma unroll
    for (int k = 0; k < NQ; ++k) v[k] = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        double A = 0.0, B = 0.0, E = 0.0;
        if (in[t]) {
            const double n = mom[t], sf = mom[N + t], sm = mom[2 * N + t];
            const double sff = mom[3 * N + t], smm = mom[4 * N + t], sfm = mom[5 * N + t];
            const double muf = sf / n, mum = sm / n;
            const double vf = sff - sf * muf, vm = smm - sm * mum, cov = sfm - sf * mum;
            if (vf > kBoxRelEps * sff && vm > kBoxRelEps * smm) {
                const double den = vf * vm;
                A = 2.0 * cov / den;
                B = -2.0 * cov * cov / (den * vm);
                E = A * muf + B * mum;
                v[Q_COUNT] += 1.0;
                v[Q_CC] -= cov * cov / den;
            }
        }
        abe[t] = A;
        abe[N + t] = B;
        abe[2 * N + t] = E;
    }
    block_sum<NQ>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < NQ; ++k) part[(long long)k * gridDim.x + blockIdx.x] = v[k];
}

// texel coefficient c(y) = -(f S_A + m S_B - S_E) from the box sums of A, B, E (0 outside)
__global__ void __launch_bounds__(256) box_coef_kernel(const double *__restrict__ sabe,
                                                       const float *__restrict__ fixed,
                                                       const float4 *__restrict__ samp,
                                                       const unsigned char *__restrict__ in, long long N,
                                                       float *__restrict__ coef)
{
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < N; t += (long long)gridDim.x * blockDim.x) {
        float c = 0.f;
        if (in[t]) {
            const double f = (double)fixed[t], m = (double)samp[t].w;
            c = (float)(-(f * sabe[t] + m * sabe[N + t] - sabe[2 * N + t]));
        }
        coef[t] = c;
    }
}

}  // namespace skm
