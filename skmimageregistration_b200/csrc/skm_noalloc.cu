// skm_noalloc.cu -- metric value without any device allocation.
//
// Some callers cannot allocate device memory when they need a metric value: a host
// framework that owns the whole device memory budget and forbids third-party cudaMalloc,
// a real-time loop that must not hit the implicit device synchronisation cudaMalloc and
// cudaFree imply, or code that has pre-planned every buffer up front.  For them this file
// offers skm_value_noalloc: the caller passes device buffers for the inputs and the
// result, and the only other memory used is the fixed-size array below, which lives in
// the library image itself.
//
// Limits and rules (also stated at the declaration in include/skm_gpu.h):
//   * stationary kernel, subsampling 1, no displacement field, MSE or NCC;
//   * at most kNoAllocMaxSamples fixed-image texels (the scratch holds one partial-sum
//     record per 256-texel block); larger images are rejected with SKM_ERR_INVALID;
//   * the scratch is shared by every call on a device and keeps the last call's contents.
//     Each call writes every slot it later reads, so nothing has to start at zero, but two
//     calls that overlap on the GPU (different streams, no ordering) race on it;
//   * the first call on each device looks up the scratch's device address with
//     cudaGetSymbolAddress (once per device, under a lock); make that first call before
//     any stream capture.  The address is cached for the life of the process: after a
//     cudaDeviceReset (which unloads the module) the cached address is stale, so the entry
//     point must not be used across a reset;
//   * control_points must be 16-byte aligned (float4 loads), the images 4-byte and the
//     result 8-byte aligned; misaligned buffers are rejected with SKM_ERR_INVALID.
#include <cstdarg>
#include <cstdio>
#include <mutex>

#include "../../include/skm_gpu.h"
#include "skm_device.cuh"
#include "skm_kernels.cuh"

using namespace skm;

void skm_internal_set_error(const char *msg);   // skm_capi.cu: sets the skm_last_error() message

namespace {

constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocMaxBlocks = 8192;
constexpr long long kNoAllocMaxSamples = (long long)kNoAllocThreads * kNoAllocMaxBlocks;   // 2,097,152
constexpr int kNoAllocQ = 7;          // count, sum d^2, sf, sm, sff, smm, sfm
constexpr int kMaxDevices = 64;

// 7 * 8192 doubles = 458,752 bytes, held by every device that loads the library until exit.
static __device__ __align__(256) double g_value_scratch[kNoAllocQ * kNoAllocMaxBlocks];

std::mutex g_scratch_lock;
double *g_scratch_addr[kMaxDevices] = {nullptr};

int noalloc_fail(int code, const char *fmt, ...);

// Device address of g_value_scratch on the current device (looked up once per device).
int scratch_address(double **out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(SKM_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(SKM_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> g(g_scratch_lock);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_value_scratch);
        if (e != cudaSuccess)
            return noalloc_fail(SKM_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return SKM_OK;
}

Geo geo_of(const skm_geometry &g, int D, int pad)
{
    Geo r;
    for (int d = 0; d < 3; ++d) {
        if (d < D) {
            r.o[d] = g.origin[d];
            r.s[d] = g.spacing[d];
            r.inv[d] = 1.0 / g.spacing[d];
            r.n[d] = g.size[d] + pad;
        } else {
            r.o[d] = 0.0; r.s[d] = 1.0; r.inv[d] = 1.0; r.n[d] = 1;
        }
    }
    r.st[0] = 1;
    r.st[1] = r.n[0];
    r.st[2] = (long long)r.n[0] * r.n[1];
    return r;
}

// Value-only variant of value_kernel: no per-sample records, partial sums into the scratch.
template <int D>
__global__ void __launch_bounds__(kNoAllocThreads) value_noalloc_kernel(EvalParams P, double *__restrict__ scratch)
{
    __shared__ double sh[kNoAllocQ * 32];
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    double v[kNoAllocQ];
#pragma unroll
    for (int k = 0; k < kNoAllocQ; ++k) v[k] = 0.0;
    if (t < P.Ns) {
        int sp[3];
        cell_of<D>(P.ss, t, sp);
        double fi[3] = {(double)sp[0], (double)sp[1], (double)sp[2]}, p[3], ml[3];
        to_global<D>(P.fixed, fi, p);
        moving_local<D, kStationary, false>(P, p, ml);
        if (bspline_inside<D>(P.mov, ml)) {
            float m, g[3];
            bspline_derivs<D>(P.coeffs, P.mov, ml, m, g);
            double f = (double)P.fixed_data[lin_of<D>(P.fixed, sp)];
            double md = (double)m;
            v[0] = 1.0;
            v[1] = (md - f) * (md - f);
            v[2] = f;
            v[3] = md;
            v[4] = f * f;
            v[5] = md * md;
            v[6] = f * md;
        }
    }
    block_sum<kNoAllocQ>(v, sh);
    if (threadIdx.x == 0)
#pragma unroll
        for (int k = 0; k < kNoAllocQ; ++k) scratch[(long long)k * gridDim.x + blockIdx.x] = v[k];
}

// Reduces the block partials in a fixed order and writes {measure, pixels counted}.
__global__ void __launch_bounds__(1024) value_noalloc_finish(const double *__restrict__ scratch, int nblocks,
                                                             int metric, double *__restrict__ result)
{
    __shared__ double sh[kNoAllocQ * 32];
    double v[kNoAllocQ];
#pragma unroll
    for (int k = 0; k < kNoAllocQ; ++k) {
        double s = 0.0;
        for (int b = threadIdx.x; b < nblocks; b += blockDim.x) s += scratch[(long long)k * nblocks + b];
        v[k] = s;
    }
    block_sum<kNoAllocQ>(v, sh);
    if (threadIdx.x == 0) {
        double n = v[0], measure;
        if (metric == SKM_MSE) {
            measure = v[1] / n;
        } else {
            double sf = v[2], sm = v[3];
            double sff = v[4] - sf * sf / n, smm = v[5] - sm * sm / n, sfm = v[6] - sf * sm / n;
            double denom = -1.0 * sqrt(sff * smm);
            measure = denom != 0.0 ? sfm / denom : 0.0;
        }
        result[0] = measure;
        result[1] = n;
    }
}

// errors go to the library's skm_last_error() message
int noalloc_fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    skm_internal_set_error(buf);
    return code;
}

}  // namespace

extern "C" int skm_value_noalloc(int32_t dimensions, int32_t metric, const skm_geometry *fixed_geometry,
                                 const float *fixed_image, const skm_geometry *moving_geometry,
                                 const float *moving_coefficients, const skm_geometry *cp_geometry,
                                 const float *control_points, double sigma_c0, double sigma_c4, double *result,
                                 void *stream)
{
    const int D = dimensions;
    if (D != 2 && D != 3) return noalloc_fail(SKM_ERR_INVALID, "dimensions must be 2 or 3 (got %d)", D);
    if (metric != SKM_MSE && metric != SKM_NCC)
        return noalloc_fail(SKM_ERR_INVALID, "skm_value_noalloc supports MSE and NCC only (got %d)", metric);
    if (!fixed_geometry || !moving_geometry || !cp_geometry || !fixed_image || !moving_coefficients ||
        !control_points || !result)
        return noalloc_fail(SKM_ERR_INVALID, "NULL argument");
    if (!(sigma_c0 > 0.0) || !(sigma_c4 > 0.0)) return noalloc_fail(SKM_ERR_INVALID, "kernel parameters have to be positive");
    // the kernels read control points as float4 (16-byte loads), images as float, the result as
    // double: a misaligned buffer would fault on the device, so it is rejected here
    if (reinterpret_cast<uintptr_t>(control_points) % 16 != 0)
        return noalloc_fail(SKM_ERR_INVALID, "control_points must be 16-byte aligned (4 floats per control point)");
    if (reinterpret_cast<uintptr_t>(fixed_image) % alignof(float) != 0 ||
        reinterpret_cast<uintptr_t>(moving_coefficients) % alignof(float) != 0)
        return noalloc_fail(SKM_ERR_INVALID, "fixed_image and moving_coefficients must be 4-byte aligned");
    if (reinterpret_cast<uintptr_t>(result) % alignof(double) != 0)
        return noalloc_fail(SKM_ERR_INVALID, "result must be 8-byte aligned");
    long long N = 1;
    for (int d = 0; d < D; ++d) {
        if (fixed_geometry->size[d] < 1 || cp_geometry->size[d] < 1 || moving_geometry->size[d] < 2 ||
            !(fixed_geometry->spacing[d] > 0) || !(cp_geometry->spacing[d] > 0) || !(moving_geometry->spacing[d] > 0))
            return noalloc_fail(SKM_ERR_INVALID, "invalid geometry");
        N *= fixed_geometry->size[d];
    }
    if (N > kNoAllocMaxSamples)
        return noalloc_fail(SKM_ERR_INVALID,
                            "fixed image has %lld texels; skm_value_noalloc handles at most %lld (its scratch holds "
                            "%d block partials); use skm_get_value for larger images",
                            N, kNoAllocMaxSamples, kNoAllocMaxBlocks);
    double *scratch = nullptr;
    int rc = scratch_address(&scratch);
    if (rc) return rc;

    EvalParams P{};
    P.sub = 1;
    P.nbh = 1;
    P.fixed = geo_of(*fixed_geometry, D, 0);
    P.mov = geo_of(*moving_geometry, D, 3);
    P.cp = geo_of(*cp_geometry, D, 0);
    P.df = P.fixed;
    P.has_df = 0;
    for (int k = 0; k < 3; ++k) P.ss[k] = P.fixed.n[k];
    P.Ns = N;
    P.C = (long long)P.cp.n[0] * P.cp.n[1] * P.cp.n[2];
    P.fixed_data = fixed_image;
    P.coeffs = moving_coefficients;
    P.cpd = reinterpret_cast<const float4 *>(control_points);
    P.dfd = nullptr;
    P.shifts = nullptr;
    KernelParams &K = P.K;
    K.kind = kStationary;
    K.sc0 = (float)sigma_c0;
    K.sc4 = (float)sigma_c4;
    K.inv_sc0 = 1.0f / K.sc0;
    K.inv_sc4 = 1.0f / K.sc4;
    K.support_min = K.sc4 < K.sc0 ? K.sc4 : K.sc0;

    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int blocks = (int)((N + kNoAllocThreads - 1) / kNoAllocThreads);
    if (D == 3)
        value_noalloc_kernel<3><<<blocks, kNoAllocThreads, 0, s>>>(P, scratch);
    else
        value_noalloc_kernel<2><<<blocks, kNoAllocThreads, 0, s>>>(P, scratch);
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) return noalloc_fail(SKM_ERR_CUDA, "value launch: %s", cudaGetErrorString(e));
    value_noalloc_finish<<<1, 1024, 0, s>>>(scratch, blocks, metric, result);
    e = cudaPeekAtLastError();
    if (e != cudaSuccess) return noalloc_fail(SKM_ERR_CUDA, "finish launch: %s", cudaGetErrorString(e));
    return SKM_OK;
}
