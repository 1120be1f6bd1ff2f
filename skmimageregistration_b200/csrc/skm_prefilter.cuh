// skm_prefilter.cuh -- cubic B-spline prefilter on the GPU.
//
// BsplineImage::computeCoeffs (include/cuda/BsplineImage.h:37-108,174-221): each image
// line is filtered by the causal/anti-causal recursion with pole sqrt(3)-2 and mirror
// boundary initialisation, axis by axis in the reference's order, then the result is
// mirror-padded by one texel in front and two behind.  One thread owns one line; the
// recursion is sequential along the line, lines are independent.  Double precision,
// like the reference (Texel = ScalarType = double).
#pragma once

#include <cuda_runtime.h>

namespace skm {

__device__ inline double bs_initial_causal(const double *c, int len, long long st, double z)
{
    double zn = z, iz = 1.0 / z;
    double z2n = pow(z, (double)(len - 1));
    double sum = c[0] + z2n * c[(long long)(len - 1) * st];
    z2n *= z2n * iz;
    for (int n = 1; n < len - 1; n++) {
        sum += (zn + z2n) * c[(long long)n * st];
        zn *= z;
        z2n *= iz;
    }
    return sum / (1.0 - zn * zn);
}

__device__ inline void bs_convert_line(double *c, int len, long long st, double z)
{
    const double lambda = 2.0 - z - 1.0 / z;
    for (int n = 0; n < len; n++) c[(long long)n * st] *= lambda;
    c[0] = bs_initial_causal(c, len, st, z);
    for (int n = 1; n < len; n++) c[(long long)n * st] += z * c[(long long)(n - 1) * st];
    c[(long long)(len - 1) * st] =
        (z / (z * z - 1.0)) * (z * c[(long long)(len - 2) * st] + c[(long long)(len - 1) * st]);
    for (int n = len - 2; n >= 0; n--) c[(long long)n * st] = z * (c[(long long)(n + 1) * st] - c[(long long)n * st]);
}

// Filters all lines along `axis` of an X*Y*Z volume in place.
__global__ void bs_prefilter_axis(double *img, int X, int Y, int Z, int axis, double pole)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long XY = (long long)X * Y;
    if (axis == 2) {                      // lines along z, indexed by (x, y)
        if (t >= XY) return;
        bs_convert_line(img + t, Z, XY, pole);
    } else if (axis == 1) {               // lines along y, indexed by (x, z)
        if (t >= (long long)X * Z) return;
        long long x = t % X, z = t / X;
        bs_convert_line(img + x + z * XY, Y, X, pole);
    } else {                              // lines along x, indexed by (y, z)
        if (t >= (long long)Y * Z) return;
        bs_convert_line(img + t * X, X, 1, pole);
    }
}

// mirrorCoeffBorders (BsplineImage.h:72-108): padded index x -> W - |W - |x-1||.
__global__ void bs_mirror_pad(const double *src, int X, int Y, int Z, int D, double *dst)
{
    int PX = X + 3, PY = Y + 3, PZ = D == 3 ? Z + 3 : 1;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)PX * PY * PZ) return;
    int x = (int)(t % PX), y = (int)((t / PX) % PY), z = (int)(t / ((long long)PX * PY));
    int W = X - 1, H = Y - 1, Dp = Z - 1;
    int xi = W - abs(W - abs(x - 1));
    int yi = H - abs(H - abs(y - 1));
    int zi = D == 3 ? Dp - abs(Dp - abs(z - 1)) : 0;
    dst[t] = src[xi + (long long)X * (yi + (long long)zi * Y)];
}

}  // namespace skm
