// skm_preprocess.cuh -- image preprocessing of the multi-scale driver on the GPU.
//
// GaussianSmoothing (include/itkUtils.h:139-150): a discrete Gaussian filter applied axis by
// axis.  Per axis the kernel is the discrete analogue of the Gaussian, T(n, t) = e^-t I_n(t)
// (I_n the modified Bessel function of the first kind, t = variance / spacing^2 when the image
// spacing is used), taken for n = 0, 1, 2, ... until the symmetric kernel holds 1 - maximum_error
// of the mass (or a term no longer changes the sum, or the half kernel exceeds the maximum
// width), then normalised to sum 1 -- the published construction of ITK's Gaussian operator,
// here with the Bessel values summed from their power series in double precision.  Borders
// repeat the edge voxel (zero-flux Neumann); sums in double.
//
// ThresholdImage + RescaleImage (include/itkUtils.h:45-110): every value is clamped to
// [smallest value above thresh_min, largest value below thresh_max] and the result mapped
// linearly so that its minimum and maximum become out_min and out_max.
#pragma once

#include <cfloat>
#include <cmath>
#include <vector>

namespace skm {

constexpr int kSmoothMaxRadius = 512;

// e^-t I_n(t) from the power series sum_k (t/2)^(2k+n) / (k! (k+n)!), all terms positive.
inline double scaled_bessel_i(int n, double t)
{
    const double h = 0.5 * t;
    double term = std::exp(-t);
    for (int j = 1; j <= n; ++j) term *= h / j;            // e^-t (t/2)^n / n!
    double sum = term;
    for (int k = 1; k < 100000; ++k) {
        term *= h * h / ((double)k * (double)(k + n));
        sum += term;
        if (term < sum * 1e-18) break;
    }
    return sum;
}

// Half kernel c[0..r] (c[0] the centre) of the discrete Gaussian of variance t (voxel units).
inline std::vector<double> gaussian_half_kernel(double t, double maximum_error, int maximum_width)
{
    std::vector<double> c;
    const double cap = 1.0 - maximum_error;
    c.push_back(scaled_bessel_i(0, t));
    double sum = c[0];
    c.push_back(scaled_bessel_i(1, t));
    sum += 2.0 * c[1];
    for (int i = 2; sum < cap; ++i) {
        c.push_back(scaled_bessel_i(i, t));
        sum += 2.0 * c[i];
        if (c[i] < sum * DBL_EPSILON) break;                  // no longer changes the sum
        if ((int)c.size() > maximum_width) break;
    }
    for (double &v : c) v /= sum;
    return c;
}

// One pass along `axis` of an X x Y x Z volume (x fastest): out = sum_k c[|k|] in[clamp(i + k)]
__global__ void smooth_axis_kernel(const double *__restrict__ in, double *__restrict__ out, int X, int Y, int Z,
                                   int axis, const double *__restrict__ c, int r)
{
    __shared__ double cs[kSmoothMaxRadius + 1];
    for (int k = threadIdx.x; k <= r; k += blockDim.x) cs[k] = c[k];
    __syncthreads();
    const long long n = (long long)X * Y * Z;
    const int len = axis == 0 ? X : (axis == 1 ? Y : Z);
    const long long stride = axis == 0 ? 1 : (axis == 1 ? (long long)X : (long long)X * Y);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long long)X * Y));
        const int p = axis == 0 ? x : (axis == 1 ? y : z);
        const long long base = i - (long long)p * stride;
        double s = cs[0] * in[i];
        for (int k = 1; k <= r; ++k) {
            const int lo = max(p - k, 0), hi = min(p + k, len - 1);
            s += cs[k] * (in[base + (long long)lo * stride] + in[base + (long long)hi * stride]);
        }
        out[i] = s;
    }
}

// min, max, largest value below tmax, smallest value above tmin: per-block partials, then one block
__global__ void range_kernel(const double *__restrict__ v, long long n, double tmin, double tmax,
                             double *__restrict__ part)
{
    __shared__ double sh[4][256];
    double mn = DBL_MAX, mx = -DBL_MAX, below = -DBL_MAX, above = DBL_MAX;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const double x = v[i];
        mn = fmin(mn, x);
        mx = fmax(mx, x);
        if (x < tmax) below = fmax(below, x);
        if (x > tmin) above = fmin(above, x);
    }
    sh[0][threadIdx.x] = mn;
    sh[1][threadIdx.x] = mx;
    sh[2][threadIdx.x] = below;
    sh[3][threadIdx.x] = above;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if ((int)threadIdx.x < s) {
            sh[0][threadIdx.x] = fmin(sh[0][threadIdx.x], sh[0][threadIdx.x + s]);
            sh[1][threadIdx.x] = fmax(sh[1][threadIdx.x], sh[1][threadIdx.x + s]);
            sh[2][threadIdx.x] = fmax(sh[2][threadIdx.x], sh[2][threadIdx.x + s]);
            sh[3][threadIdx.x] = fmin(sh[3][threadIdx.x], sh[3][threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int q = 0; q < 4; ++q) part[(long long)q * gridDim.x + blockIdx.x] = sh[q][0];
}

__global__ void range_finish_kernel(const double *__restrict__ part, int nblocks, double *__restrict__ out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double r[4] = {DBL_MAX, -DBL_MAX, -DBL_MAX, DBL_MAX};
    for (int b = 0; b < nblocks; ++b) {
        r[0] = fmin(r[0], part[b]);
        r[1] = fmax(r[1], part[nblocks + b]);
        r[2] = fmax(r[2], part[2 * nblocks + b]);
        r[3] = fmin(r[3], part[3 * nblocks + b]);
    }
    for (int q = 0; q < 4; ++q) out[q] = r[q];
}

__global__ void clamp_rescale_kernel(double *__restrict__ v, long long n, double lo, double hi, double scale,
                                     double shift)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        v[i] = fmin(fmax(v[i], lo), hi) * scale + shift;
}

}  // namespace skm
