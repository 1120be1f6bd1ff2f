// skm_output.cuh -- result images of the registration application on the GPU.
//
// Warped image (src/SKMReg.cxx:484-488 with WarpImage, include/itkUtils.h:163-178, order 3; and the
// final resampling of src/SKMReg.cxx:504-522, order 1): out(i) = I(p_i + u_i), p_i the physical
// position of output texel i, u_i the displacement stored at that texel, I the moving image
// interpolated at p_i + u_i; positions whose continuous index lies outside [-0.5, size - 0.5) on
// any axis get the default value (ITK's IsInsideBuffer with centred pixel coordinates).
//   order 1: multilinear interpolation with the neighbour indices clamped to the image
//            (LinearInterpolateImageFunction's edge handling);
//   order 3: cubic B-spline interpolation of the prefiltered coefficients (the same recursive
//            prefilter as the moving image of the evaluator) with whole-sample mirrored indices
//            (BSplineInterpolateImageFunction: index floor(x) - 1 .. floor(x) + 2).
//
// Jacobian determinant (JacobianDeterminant, include/itkUtils.h:153-161, which SKMReg applies to
// the control-point image, src/SKMReg.cxx:471-472): det(I + du/dx) with
// du_i/dx_j = (u_i[x + e_j] - u_i[x - e_j]) / (2 spacing_j), an edge texel's missing neighbour
// replaced by the texel itself (DisplacementFieldJacobianDeterminantFilter with image spacing and
// its neighbourhood iterator's zero-flux boundary).
#pragma once

#include <cmath>

namespace skm {

struct OutGeo {
    double o[3], s[3];
    int n[3];
};

__device__ __forceinline__ int mirror_index(int k, int n)
{
    const int period = 2 * (n - 1);
    if (period <= 0) return 0;
    k %= period;
    if (k < 0) k += period;
    return k < n ? k : period - k;
}

template <int D, int ORDER>
__global__ void warp_kernel(const double *__restrict__ img, OutGeo gi, const double *__restrict__ field, OutGeo gf,
                            double fill, double *__restrict__ out)
{
    const long long n = (long long)gf.n[0] * gf.n[1] * (D == 3 ? gf.n[2] : 1);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        idx[0] = (int)(i % gf.n[0]);
        idx[1] = (int)((i / gf.n[0]) % gf.n[1]);
        idx[2] = D == 3 ? (int)(i / ((long long)gf.n[0] * gf.n[1])) : 0;
        double ci[3];
        bool inside = true;
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double p = gf.o[d] + gf.s[d] * idx[d] + field[i * D + d];
            ci[d] = (p - gi.o[d]) / gi.s[d];
            inside = inside && ci[d] >= -0.5 && ci[d] < gi.n[d] - 0.5;
        }
        if (!inside) {
            out[i] = fill;
            continue;
        }
        constexpr int K = ORDER == 1 ? 2 : 4;
        int ix[3][K];
        double w[3][K];
#pragma unroll
        for (int d = 0; d < D; ++d) {
            const double f = floor(ci[d]);
            const double t = ci[d] - f;
            const int b = (int)f;
            if (ORDER == 1) {
                ix[d][0] = min(max(b, 0), gi.n[d] - 1);
                ix[d][1] = min(max(b + 1, 0), gi.n[d] - 1);
                w[d][0] = 1.0 - t;
                w[d][1] = t;
            } else {
                // cubic B-spline weights of the four samples floor(x) - 1 .. floor(x) + 2
                const double s = 1.0 - t;
                w[d][0] = s * s * s / 6.0;
                w[d][1] = 2.0 / 3.0 - t * t + 0.5 * t * t * t;
                w[d][2] = 2.0 / 3.0 - s * s + 0.5 * s * s * s;
                w[d][3] = t * t * t / 6.0;
#pragma unroll
                for (int k = 0; k < 4; ++k) ix[d][k] = mirror_index(b - 1 + k, gi.n[d]);
            }
        }
        const long long sy = gi.n[0], sz = (long long)gi.n[0] * gi.n[1];
        double acc = 0.0;
        if (D == 3) {
#pragma unroll
            for (int c = 0; c < K; ++c) {
                double az = 0.0;
#pragma unroll
                for (int b = 0; b < K; ++b) {
                    const double *row = img + ix[2][c] * sz + ix[1][b] * sy;
                    double ax = 0.0;
#pragma unroll
                    for (int a = 0; a < K; ++a) ax += w[0][a] * row[ix[0][a]];
                    az += w[1][b] * ax;
                }
                acc += w[2][c] * az;
            }
        } else {
#pragma unroll
            for (int b = 0; b < K; ++b) {
                const double *row = img + ix[1][b] * sy;
                double ax = 0.0;
#pragma unroll
                for (int a = 0; a < K; ++a) ax += w[0][a] * row[ix[0][a]];
                acc += w[1][b] * ax;
            }
        }
        out[i] = acc;
    }
}

template <int D>
__global__ void jacobian_determinant_kernel(const double *__restrict__ u, OutGeo g, double *__restrict__ out)
{
    const long long n = (long long)g.n[0] * g.n[1] * (D == 3 ? g.n[2] : 1);
    const long long st[3] = {1, g.n[0], (long long)g.n[0] * g.n[1]};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
        int idx[3];
        idx[0] = (int)(i % g.n[0]);
        idx[1] = (int)((i / g.n[0]) % g.n[1]);
        idx[2] = D == 3 ? (int)(i / ((long long)g.n[0] * g.n[1])) : 0;
        double J[3][3];
#pragma unroll
        for (int j = 0; j < D; ++j) {
            const long long hi = i + (idx[j] < g.n[j] - 1 ? st[j] : 0);
            const long long lo = i - (idx[j] > 0 ? st[j] : 0);
#pragma unroll
            for (int c = 0; c < D; ++c)
                J[c][j] = (c == j ? 1.0 : 0.0) + (u[hi * D + c] - u[lo * D + c]) / (2.0 * g.s[j]);
        }
        out[i] = D == 2 ? J[0][0] * J[1][1] - J[0][1] * J[1][0]
                        : J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
                              J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
                              J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    }
}

}  // namespace skm
