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

__global__ void scale_kernel(const double *__restrict__ in, double *__restrict__ out, long long n, double w)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
        out[i] = in[i] * w;
}

// ---------------------------------------------------------------------------------------------
// Anisotropic covariance tensor (ComputeAnisotropicTensor, include/AnisotropicTensorUtils.h:37-371).
//
// Structure tensor components are stored as D(D+1)/2 planes of n texels, upper triangle row by
// row: 2-D xx, xy, yy; 3-D xx, xy, xz, yy, yz, zz.

__host__ __device__ constexpr int tensor_components(int D) { return D * (D + 1) / 2; }

template <int D>
__host__ __device__ constexpr int tensor_slot(int i, int j)
{
    return i <= j ? i * D - i * (i - 1) / 2 + (j - i) : j * D - j * (j - 1) / 2 + (i - j);
}

// Outer product of the image gradient (itk::GradientImageFilter: (f[i+1] - f[i-1]) / (2 spacing)
// per axis, an edge texel's missing neighbour replaced by the texel itself).
template <int D>
__global__ void gradient_outer_kernel(const double *__restrict__ f, int X, int Y, int Z, double hx, double hy,
                                      double hz, double *__restrict__ comp)
{
    const long long n = (long long)X * Y * Z;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        const int x = (int)(i % X), y = (int)((i / X) % Y), z = (int)(i / ((long long)X * Y));
        const long long sy = X, sz = (long long)X * Y;
        double g[3];
        g[0] = (f[i + (x < X - 1 ? 1 : 0)] - f[i - (x > 0 ? 1 : 0)]) / hx;
        g[1] = (f[i + (y < Y - 1 ? sy : 0)] - f[i - (y > 0 ? sy : 0)]) / hy;
        if (D == 3) g[2] = (f[i + (z < Z - 1 ? sz : 0)] - f[i - (z > 0 ? sz : 0)]) / hz;
#pragma unroll
        for (int a = 0; a < D; ++a)
#pragma unroll
            for (int b = a; b < D; ++b) comp[(long long)tensor_slot<D>(a, b) * n + i] = g[a] * g[b];
    }
}

// Cyclic Jacobi eigen decomposition of a symmetric D x D matrix (Golub & Van Loan, Matrix
// Computations, 4th ed., algorithms 8.5.1-8.5.3): a is overwritten, w[k] = a[k][k] at the end,
// column k of v the unit eigenvector of w[k].
template <int D>
__device__ void jacobi_eigen(double (&a)[3][3], double (&w)[3], double (&v)[3][3])
{
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) v[r][c] = r == c ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 32; ++sweep) {
        double off = 0.0, diag = 0.0;
#pragma unroll
        for (int p = 0; p < D; ++p) {
            diag += a[p][p] * a[p][p];
#pragma unroll
            for (int q = p + 1; q < D; ++q) off += a[p][q] * a[p][q];
        }
        if (off <= 1e-36 * diag || off == 0.0) break;
#pragma unroll
        for (int p = 0; p < D - 1; ++p)
#pragma unroll
            for (int q = p + 1; q < D; ++q) {
                const double apq = a[p][q];
                if (apq == 0.0) continue;
                // 2x2 symmetric Schur decomposition: tan of the angle that zeroes a[p][q]
                const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
                const double t = fabs(theta) > 1e150 ? 0.5 / theta
                                                     : copysign(1.0, theta) / (fabs(theta) + sqrt(theta * theta + 1.0));
                const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
                a[p][p] -= t * apq;
                a[q][q] += t * apq;
                a[p][q] = a[q][p] = 0.0;
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    if (r == p || r == q) continue;
                    const double arp = a[r][p], arq = a[r][q];
                    a[r][p] = a[p][r] = c * arp - s * arq;
                    a[r][q] = a[q][r] = s * arp + c * arq;
                }
#pragma unroll
                for (int r = 0; r < D; ++r) {
                    const double vp = v[r][p], vq = v[r][q];
                    v[r][p] = c * vp - s * vq;
                    v[r][q] = s * vp + c * vq;
                }
            }
    }
#pragma unroll
    for (int k = 0; k < D; ++k) w[k] = a[k][k];
}

template <int D>
__device__ __forceinline__ double row_norm(const double (&r)[3])
{
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) s += r[k] * r[k];
    return sqrt(s);
}

// Per texel: eigen system of the smoothed structure tensor ordered by magnitude with rows
// eigenvalue * eigenvector (include/itkSymmetricEigenDecompositionImageFilter.h), the direction
// weighting (AnisotropicTensorUtils.h:181-300) and the covariance U diag(column norms) U^T
// (:316-360).  tilt[i] = |main row| after the alignment weighting where the texel passed the
// 1e-8 test, else -DBL_MAX; bad counts texels whose covariance has a non-positive determinant.
template <int D>
__global__ void covariance_kernel(const double *__restrict__ comp, long long n, int alignment,
                                  double *__restrict__ cov, double *__restrict__ tilt, unsigned *__restrict__ bad)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double a[3][3] = {}, w[3] = {}, v[3][3];
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) a[r][c] = comp[(long long)tensor_slot<D>(r, c) * n + i];
        jacobi_eigen<D>(a, w, v);
        // order by |eigenvalue| ascending (stable), rows[k] = w * eigenvector
        int ord[3] = {0, 1, 2};
#pragma unroll
        for (int p = 1; p < D; ++p)
#pragma unroll
            for (int q = p; q > 0; --q)
                if (fabs(w[ord[q]]) < fabs(w[ord[q - 1]])) {
                    const int t = ord[q];
                    ord[q] = ord[q - 1];
                    ord[q - 1] = t;
                }
        double rows[3][3] = {}, mag[3];
        bool ok = true;
#pragma unroll
        for (int k = 0; k < D; ++k) {
#pragma unroll
            for (int c = 0; c < D; ++c) rows[k][c] = w[ord[k]] * v[c][ord[k]];
            mag[k] = row_norm<D>(rows[k]);
            ok = ok && mag[k] > 1e-8;
        }
        double M[3][3] = {};
        double rev = -DBL_MAX;
        if (ok) {
            double nrm[3] = {}, main[3] = {};
#pragma unroll
            for (int c = 0; c < D; ++c) {
                nrm[c] = rows[D - 1][c] / mag[D - 1];
                main[c] = rows[D - 1][c];
            }
            if (alignment >= 0 && alignment < D) {
                double cr;
                if (D == 2) {
                    const double m0 = alignment == 0 ? 1.0 : 0.0, m1 = alignment == 1 ? 1.0 : 0.0;
                    cr = fabs(nrm[0] * m1 - nrm[1] * m0);
                } else {
                    double m[3] = {0.0, 0.0, 0.0};
                    m[alignment] = 1.0;
                    const double c0 = nrm[1] * m[2] - nrm[2] * m[1], c1 = nrm[2] * m[0] - nrm[0] * m[2],
                                 c2 = nrm[0] * m[1] - nrm[1] * m[0];
                    cr = sqrt(c0 * c0 + c1 * c1 + c2 * c2);
                }
                double factor = cr + 1e-10;
                factor = factor * factor / sqrt((double)D);
#pragma unroll
                for (int c = 0; c < D; ++c) main[c] *= factor;
            }
            rev = row_norm<D>(main);
            const double p = pow(rev, 1.5);
            double out[3][3] = {};
#pragma unroll
            for (int c = 0; c < D; ++c) out[D - 1][c] = nrm[c] / (1.0 + p);
#pragma unroll
            for (int k = 0; k < D - 1; ++k)
#pragma unroll
                for (int c = 0; c < D; ++c) out[k][c] = rows[k][c] / mag[k] * (1.0 + p / (1.0 + p));
            // flipud().transpose(): M[r][c] = out[D - 1 - c][r]
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) M[r][c] = out[D - 1 - c][r];
        } else {
#pragma unroll
            for (int r = 0; r < D; ++r) M[r][r] = 1.0;
        }
        // covariance from the scaled eigenvectors (columns of M)
        double s[3], C[3][3] = {};
#pragma unroll
        for (int c = 0; c < D; ++c) {
            double q = 0.0;
#pragma unroll
            for (int r = 0; r < D; ++r) q += M[r][c] * M[r][c];
            s[c] = sqrt(q);
        }
        if (s[0] < 1e-8) {
#pragma unroll
            for (int r = 0; r < D; ++r) C[r][r] = 1.0;
        } else {
#pragma unroll
            for (int r = 0; r < D; ++r)
#pragma unroll
                for (int c = 0; c < D; ++c) {
                    double acc = 0.0;
#pragma unroll
                    for (int k = 0; k < D; ++k) acc += (M[r][k] / s[k]) * s[k] * (M[c][k] / s[k]);
                    C[r][c] = acc;
                }
        }
        const double det = D == 2 ? C[0][0] * C[1][1] - C[0][1] * C[1][0]
                                  : C[0][0] * (C[1][1] * C[2][2] - C[1][2] * C[2][1]) -
                                        C[0][1] * (C[1][0] * C[2][2] - C[1][2] * C[2][0]) +
                                        C[0][2] * (C[1][0] * C[2][1] - C[1][1] * C[2][0]);
        if (!(det > 0.0)) atomicAdd(bad, 1u);
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) cov[i * D * D + r * D + c] = C[r][c];
        tilt[i] = rev;
    }
}

// |largest eigenvalue| of each D x D tensor (vnl_symmetric_eigensystem's last eigenvalue, as
// itkTransformAdapter.hxx:352-358 compares it), and the determinant test of :348-350.
template <int D>
__global__ void max_eigenvalue_kernel(const double *__restrict__ tensor, long long n, double *__restrict__ out,
                                      unsigned *__restrict__ bad)
{
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        double a[3][3] = {}, w[3] = {}, v[3][3];
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < D; ++c) a[r][c] = tensor[i * D * D + r * D + c];
        const double det = D == 2 ? a[0][0] * a[1][1] - a[0][1] * a[1][0]
                                  : a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) -
                                        a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                                        a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
        if (!(det > 0.0)) atomicAdd(bad, 1u);
        // symmetrise the way the eigen solver reads the matrix (upper triangle)
#pragma unroll
        for (int r = 0; r < D; ++r)
#pragma unroll
            for (int c = 0; c < r; ++c) a[r][c] = a[c][r];
        jacobi_eigen<D>(a, w, v);
        double mx = w[0];
#pragma unroll
        for (int k = 1; k < D; ++k) mx = fmax(mx, w[k]);
        out[i] = fabs(mx);
    }
}

}  // namespace skm
