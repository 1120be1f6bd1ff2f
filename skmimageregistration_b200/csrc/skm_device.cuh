// skm_device.cuh -- device-side building blocks of the SKM evaluation path on sm_100a.
//
// Geometry, the Wendland kernel family, the cubic B-spline sampler, the PCG32 grid
// shifts and deterministic block reductions.  Every formula restates a reference
// function (ChristophJud/SKMImageRegistration, include/cuda/...) cited at its
// definition; the arithmetic split is: positions and index boxes in double (they
// decide which control points / samples contribute, so they follow the reference's
// double arithmetic exactly), kernel values and sums over taps in float, global sums
// in double.
#pragma once

#include <cstdint>
#include <mutex>
#include <cuda_runtime.h>

namespace skm {

// Device buffers come from a stream-ordered memory pool private to this library (one per device,
// created on first use) whose release threshold keeps freed memory for reuse, so that evaluators
// created and destroyed level after level (the multi-scale driver) do not map and unmap their
// buffers every time.  The device's default pool, which the host application may use itself, is
// left untouched.  When the library's last live buffer on a device is freed, the pool is trimmed
// to kPoolKeepBytes (so that the next registration of a similar size does not map its buffers
// again) and the rest goes back to the driver; skm_release_memory() trims every pool to zero.
// pool_malloc and pool_free complete before returning (as cudaMalloc / cudaFree do), so no stream
// ordering leaks out of them.
constexpr int kPoolMaxDevices = 64;
constexpr size_t kPoolKeepBytes = (size_t)2 << 30;      // 2 GiB kept per device between uses


struct DevicePool {
    cudaMemPool_t pool = nullptr;
    long long live = 0;            // buffers of this library currently allocated from the pool
};

inline std::mutex &pool_lock()
{
    static std::mutex m;
    return m;
}

inline DevicePool *pool_table()
{
    static DevicePool t[kPoolMaxDevices];
    return t;
}

inline cudaError_t pool_malloc(void **p, size_t bytes)
{
    *p = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kPoolMaxDevices) return cudaErrorInvalidDevice;
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> g(pool_lock());
        DevicePool &dp = pool_table()[dev];
        if (!dp.pool) {
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = dev;
            e = cudaMemPoolCreate(&dp.pool, &props);
            if (e != cudaSuccess) {
                dp.pool = nullptr;
                return e;
            }
            uint64_t keep = UINT64_MAX;
            e = cudaMemPoolSetAttribute(dp.pool, cudaMemPoolAttrReleaseThreshold, &keep);
            if (e != cudaSuccess) return e;
        }
        pool = dp.pool;
        ++dp.live;
    }
    e = cudaMallocFromPoolAsync(p, bytes, pool, 0);
    if (e == cudaSuccess) e = cudaStreamSynchronize(0);
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> g(pool_lock());
        --pool_table()[dev].live;
    }
    return e;
}

// Frees without synchronising: the caller has made sure (one device synchronisation for many
// buffers) that no work still uses p.  Trims the pool when its last buffer goes.
inline cudaError_t pool_release(void *p)
{
    if (!p) return cudaSuccess;
    cudaPointerAttributes at{};
    cudaError_t e = cudaPointerGetAttributes(&at, p);
    if (e != cudaSuccess) return e;
    e = cudaFreeAsync(p, 0);
    if (e != cudaSuccess) return e;
    const int dev = at.device;
    if (dev >= 0 && dev < kPoolMaxDevices) {
        std::lock_guard<std::mutex> g(pool_lock());
        DevicePool &dp = pool_table()[dev];
        if (dp.live > 0 && --dp.live == 0 && dp.pool) {
            e = cudaStreamSynchronize(0);
            if (e != cudaSuccess) return e;
            e = cudaMemPoolTrimTo(dp.pool, kPoolKeepBytes);
        }
    }
    return e;
}

inline cudaError_t pool_free(void *p)
{
    if (!p) return cudaSuccess;
    cudaError_t e = cudaDeviceSynchronize();                 // as cudaFree: no work still uses p
    if (e != cudaSuccess) return e;
    e = pool_release(p);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(0);
}

// Trims the library's pool of every device to zero (nothing of the library may be alive on it).
inline cudaError_t pool_release_all()
{
    std::lock_guard<std::mutex> g(pool_lock());
    int cur = 0;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return e;
    for (int d = 0; d < kPoolMaxDevices; ++d) {
        DevicePool &dp = pool_table()[d];
        if (!dp.pool || dp.live != 0) continue;
        if ((e = cudaSetDevice(d)) != cudaSuccess) return e;
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
        if ((e = cudaMemPoolTrimTo(dp.pool, 0)) != cudaSuccess) return e;
    }
    return cudaSetDevice(cur);
}

constexpr int kMaxDim = 3;

// Division by a runtime constant d >= 1 for numerators below 2^31: q = (mulhi(n, m) + n) >> s with
// s = ceil(log2 d) and m = floor(2^32 (2^s - d) / d) + 1 (the sum cannot overflow for n < 2^31).
struct FastDiv {
    uint32_t d = 1, m = 1, s = 0;
    FastDiv() = default;
    __host__ explicit FastDiv(uint32_t dv) : d(dv)
    {
        s = 0;
        while ((1ull << s) < d) ++s;
        m = (uint32_t)((((uint64_t)1 << 32) * (((uint64_t)1 << s) - d)) / d + 1);
    }
    __device__ __forceinline__ uint32_t div(uint32_t n) const { return (__umulhi(n, m) + n) >> s; }
};

// ImageBase (include/cuda/ImageBase.h:40-100): physical = o + s*idx, local = inv*(p - o).
struct Geo {
    double o[3];
    double s[3];
    double inv[3];
    int n[3];
    long long st[3];
};

enum KernelKind : int { kStationary = 0, kWeightImage = 1, kWeightTensor = 2 };

// GKernel<float> (include/cuda/Kernel.h:134-209).
struct KernelParams {
    int kind;
    float sc0, sc4;          // sigma C0 / C4
    float inv_sc0, inv_sc4;
    float support_min;       // min(sigmaC4, sigmaC0) (float members, Kernel.h:158-161)
    float maxw;              // maximum weight (float member)
    float maxcov[9];         // maximum-eigenvalue covariance (MatF, float)
    const float *wimg;       // weight image (sigma per texel)
    Geo gw;
    const float *wten;       // covariance tensors, D*D floats per texel
    Geo gt;
    const double *wsup;      // support radius per weight-image / weight-tensor texel
    double sup_default;      // support radius outside that image
};

// Rounded as written (product, then sum; no contraction): global positions feed the truncated
// window and box bounds, which must not move by an ulp against the reference's arithmetic.
template <int D>
__device__ __forceinline__ void to_global(const Geo &g, const double *idx, double *p)
{
#pragma unroll
    for (int d = 0; d < D; ++d) p[d] = __dadd_rn(g.o[d], __dmul_rn(g.s[d], idx[d]));
}

// The product is rounded on its own: callers subtract a support half-width or add 0.5 and
// truncate, and a multiply-add fused across the inlined call would truncate inv*(p-o) - h + 1
// from just below an integer where the rounded product lands on it (window and box bounds one
// cell lower, and with a neighbourhood stride above 1 a different neighbour lattice).
template <int D>
__device__ __forceinline__ void to_local(const Geo &g, const double *p, double *l)
{
#pragma unroll
    for (int d = 0; d < D; ++d) l[d] = __dmul_rn(g.inv[d], __dsub_rn(p[d], g.o[d]));
}

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ImageNearest::atGlobal index (ImageNearest.h:69-84): int(local + 0.5), truncating.
template <int D>
__device__ __forceinline__ long long nearest_index(const Geo &g, const double *p)
{
    double l[3];
    to_local<D>(g, p, l);
    long long lin = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        int i = (int)(l[d] + 0.5);
        if (i < 0 || i >= g.n[d]) return -1;
        lin += g.st[d] * i;
    }
    return lin;
}

// ---------------------------------------------------------------------------------------------
// Wendland kernel family (Kernel.h:48-131), float like GKernel<float>.

__device__ __forceinline__ float wendland_c4(float r)
{
    float f = fmaxf(0.0f, 1.0f - r);
    float f2 = f * f;
    return f2 * f2 * f2 * (3.0f + 18.0f * r + 35.0f * r * r) * (1.0f / 3.0f);
}

__device__ __forceinline__ float wendland_c0(float r)
{
    float f = fmaxf(0.0f, 1.0f - r);
    return f * f;
}

// stationary C4*C0 product (Kernel.h:96-103); the C0 factor is always active (USE_WENDLAND_C0
// is tested with #ifdef and defined either way).
__device__ __forceinline__ float k_stationary(const KernelParams &K, float r)
{
    return wendland_c4(r * K.inv_sc4) * wendland_c0(r * K.inv_sc0);
}

template <int D>
__device__ __forceinline__ float det_m(const float *m)
{
    if (D == 2) return m[0] * m[3] - m[2] * m[1];
    return m[0] * m[4] * m[8] + m[3] * m[7] * m[2] + m[6] * m[1] * m[5] - m[0] * m[7] * m[5] -
           m[6] * m[4] * m[2] - m[3] * m[1] * m[8];
}

// v^T inv(M) v with the adjugate/determinant inverse of Mat.h:238-257.
template <int D>
__device__ __forceinline__ float quad_inv(const float *m, const float *v)
{
    float dt = det_m<D>(m);
    if (D == 2) {
        float a00 = m[3] / dt, a01 = -m[1] / dt, a10 = -m[2] / dt, a11 = m[0] / dt;
        float r0 = v[0] * a00 + v[1] * a10, r1 = v[0] * a01 + v[1] * a11;   // (v*inv)_i = sum_k v_k inv[k][i]
        return r0 * v[0] + r1 * v[1];
    }
#define M_(i, j) m[(i) * 3 + (j)]
    float a[9] = {M_(1, 1) * M_(2, 2) - M_(1, 2) * M_(2, 1), M_(0, 2) * M_(2, 1) - M_(0, 1) * M_(2, 2),
                  M_(0, 1) * M_(1, 2) - M_(0, 2) * M_(1, 1), M_(1, 2) * M_(2, 0) - M_(1, 0) * M_(2, 2),
                  M_(0, 0) * M_(2, 2) - M_(0, 2) * M_(2, 0), M_(0, 2) * M_(1, 0) - M_(0, 0) * M_(1, 2),
                  M_(1, 0) * M_(2, 1) - M_(1, 1) * M_(2, 0), M_(0, 1) * M_(2, 0) - M_(0, 0) * M_(2, 1),
                  M_(0, 0) * M_(1, 1) - M_(0, 1) * M_(1, 0)};
#undef M_
    float q = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float r = v[0] * (a[0 * 3 + i] / dt) + v[1] * (a[1 * 3 + i] / dt) + v[2] * (a[2 * 3 + i] / dt);
        q += r * v[i];
    }
    return q;
}

// Per-point information of GKernel::evaluate(p, q, [sigmaP | covP]) and its support radius.
struct PInfo {
    double support;
    float sigma;
    float cov[9];
};

template <int D>
__device__ __forceinline__ float sigma_at(const KernelParams &K, const double *p)
{
    long long i = nearest_index<D>(K.gw, p);
    return i >= 0 ? K.wimg[i] : 0.0f;     // ImageNearest default 0 (ImageNearest.h:41-45)
}

template <int D>
__device__ __forceinline__ void cov_at(const KernelParams &K, const double *p, float *c)
{
    long long i = nearest_index<D>(K.gt, p);
    if (i >= 0) {
#pragma unroll
        for (int e = 0; e < D * D; ++e) c[e] = K.wten[i * D * D + e];
    } else {                               // identity default (ImageNearest.h:47-51)
#pragma unroll
        for (int e = 0; e < D * D; ++e) c[e] = (e % (D + 1) == 0) ? 1.0f : 0.0f;
    }
}

// getRegionSupport overloads (Kernel.h:158-171).  The per-texel radii of the weight image and the
// weight tensors come from a table the host fills once (support_table in skm_capi.cu); outside the
// image the lookup default applies (sigma 0, identity covariance) and with it sup_default.
template <int KIND, int D>
__device__ __forceinline__ void pinfo_at(const KernelParams &K, const double *p, PInfo &pi)
{
    if (KIND == kWeightImage) {
        long long i = nearest_index<D>(K.gw, p);
        pi.sigma = i >= 0 ? K.wimg[i] : 0.0f;          // ImageNearest default 0 (ImageNearest.h:41-45)
        pi.support = i >= 0 ? K.wsup[i] : K.sup_default;
    } else if (KIND == kWeightTensor) {
        long long i = nearest_index<D>(K.gt, p);
        if (i >= 0) {
#pragma unroll
            for (int e = 0; e < D * D; ++e) pi.cov[e] = K.wten[i * D * D + e];
        } else {                                       // identity default (ImageNearest.h:47-51)
#pragma unroll
            for (int e = 0; e < D * D; ++e) pi.cov[e] = (e % (D + 1) == 0) ? 1.0f : 0.0f;
        }
        pi.support = i >= 0 ? K.wsup[i] : K.sup_default;
    } else {
        pi.support = (double)K.support_min;
    }
}

// getRegionSupport alone: pinfo_at's support radius without the sigma / covariance loads
template <int KIND, int D>
__device__ __forceinline__ double support_at(const KernelParams &K, const double *p)
{
    if (KIND == kWeightImage) {
        const long long i = nearest_index<D>(K.gw, p);
        return i >= 0 ? K.wsup[i] : K.sup_default;
    }
    if (KIND == kWeightTensor) {
        const long long i = nearest_index<D>(K.gt, p);
        return i >= 0 ? K.wsup[i] : K.sup_default;
    }
    return (double)K.support_min;
}

// The 3-D anisotropic kernel with one texel's covariance at both ends (the LCC derivative's
// k(c_i, n), LCC.cu:449-461): evaluateAnisotropic's factor F and the inverse of (covP + covQ) / 2
// (adjugate over determinant, as quad_inv forms it) depend on the texel alone, so they are
// computed once per texel, in the same expressions, and kept as three float4 (inverse row-major,
// then F).
__device__ __forceinline__ void aniso_self_cache(const float *c, float4 *out)
{
    float ms[9];
#pragma unroll
    for (int e = 0; e < 9; ++e) ms[e] = (c[e] + c[e]) * 0.5f;
    const float dt = det_m<3>(ms);
#define M_(i, j) ms[(i) * 3 + (j)]
    const float a[9] = {M_(1, 1) * M_(2, 2) - M_(1, 2) * M_(2, 1), M_(0, 2) * M_(2, 1) - M_(0, 1) * M_(2, 2),
                        M_(0, 1) * M_(1, 2) - M_(0, 2) * M_(1, 1), M_(1, 2) * M_(2, 0) - M_(1, 0) * M_(2, 2),
                        M_(0, 0) * M_(2, 2) - M_(0, 2) * M_(2, 0), M_(0, 2) * M_(1, 0) - M_(0, 0) * M_(1, 2),
                        M_(1, 0) * M_(2, 1) - M_(1, 1) * M_(2, 0), M_(0, 1) * M_(2, 0) - M_(0, 0) * M_(2, 1),
                        M_(0, 0) * M_(1, 1) - M_(0, 1) * M_(1, 0)};
#undef M_
    const float F = powf(det_m<3>(c), 0.25f) * powf(det_m<3>(c), 0.25f) * powf(det_m<3>(ms), -0.5f);
    out[0] = make_float4(a[0] / dt, a[1] / dt, a[2] / dt, a[3] / dt);
    out[1] = make_float4(a[4] / dt, a[5] / dt, a[6] / dt, a[7] / dt);
    out[2] = make_float4(a[8] / dt, F, 0.f, 0.f);
}

__device__ __forceinline__ float aniso_self_eval(const KernelParams &K, const float *v, const float4 *c)
{
    const float inv[9] = {c[0].x, c[0].y, c[0].z, c[0].w, c[1].x, c[1].y, c[1].z, c[1].w, c[2].x};
    float q = 0.0f;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float r = v[0] * inv[0 * 3 + i] + v[1] * inv[1 * 3 + i] + v[2] * inv[2 * 3 + i];
        q += r * v[i];
    }
    const float sqrtQ = sqrtf(q), F = c[2].y;
    return F * wendland_c4(sqrtQ * K.inv_sc4) * F * wendland_c0(sqrtQ * K.inv_sc0);
}

// GKernel::evaluate(p, q, p-side info) with v = p - q given in float and q's global
// position (needed for the sigma / covariance lookup at q).
template <int KIND, int D>
__device__ __forceinline__ float k_eval(const KernelParams &K, const float *v, const double *q, const PInfo &pi)
{
    if (KIND == kStationary) {
        float r2 = 0.0f;
#pragma unroll
        for (int d = 0; d < D; ++d) r2 = fmaf(v[d], v[d], r2);
        return k_stationary(K, sqrtf(r2));
    } else if (KIND == kWeightImage) {
        // evaluateNonStationary (Kernel.h:105-117): F^2 * C4(sqrtQ) * C0(sqrtQ)
        float sp = pi.sigma, sq = sigma_at<D>(K, q);
        float F = powf(fabsf(sp), 0.25f) * powf(fabsf(sq), 0.25f) * powf(fabsf((sp + sq) * 0.5f), -0.5f);
        float r2 = 0.0f;
#pragma unroll
        for (int d = 0; d < D; ++d) r2 = fmaf(v[d], v[d], r2);
        float sqrtQ = sqrtf(2.0f / (sp + sq)) * sqrtf(r2);
        return F * wendland_c4(sqrtQ * K.inv_sc4) * F * wendland_c0(sqrtQ * K.inv_sc0);
    } else {
        // evaluateAnisotropic (Kernel.h:119-131)
        float cq[9], ms[9];
        cov_at<D>(K, q, cq);
#pragma unroll
        for (int e = 0; e < D * D; ++e) ms[e] = (pi.cov[e] + cq[e]) * 0.5f;
        float sqrtQ = sqrtf(quad_inv<D>(ms, v));
        float F = powf(det_m<D>(pi.cov), 0.25f) * powf(det_m<D>(cq), 0.25f) * powf(det_m<D>(ms), -0.5f);
        return F * wendland_c4(sqrtQ * K.inv_sc4) * F * wendland_c0(sqrtQ * K.inv_sc0);
    }
}

// ---------------------------------------------------------------------------------------------
// cubic B-spline image (BsplineImage.h:110-144, 247-265, 285-296).  `mg` is the padded
// coefficient geometry (size+3 per axis), `l` the moving-image local coordinate in double.
template <int D>
__device__ __forceinline__ bool bspline_inside(const Geo &mg, const double *l)
{
#pragma unroll
    for (int d = 0; d < D; ++d)
        if (!(l[d] >= -0.5 && l[d] + 3.5 < (double)mg.n[d])) return false;   // NaN is outside too
    return true;
}

template <int D>
__device__ __forceinline__ void bspline_derivs(const float *__restrict__ c, const Geo &mg, const double *l,
                                               float &val, float *grad)
{
    int ii[3] = {0, 0, 0};
    float W[4][3], dW[4][3];
#pragma unroll
    for (int d = 0; d < D; ++d) {
        ii[d] = (int)l[d];                       // VecI(idx): truncation toward zero
        float w = (float)(l[d] - (double)ii[d]);
        float w3 = (1.0f / 6.0f) * w * w * w;
        float w0 = (1.0f / 6.0f) + 0.5f * w * (w - 1.0f) - w3;
        float w2 = w + w0 - 2.0f * w3;
        W[3][d] = w3; W[0][d] = w0; W[2][d] = w2; W[1][d] = 1.0f - w0 - w2 - w3;
        float d3 = 0.5f * w * w;
        float d0 = w - 0.5f - d3;
        float d2 = 1.0f + d0 - 2.0f * d3;
        dW[3][d] = d3; dW[0][d] = d0; dW[2][d] = d2; dW[1][d] = -d0 - d2 - d3;
    }
    if (D == 3) {
        float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
        const long long sy = mg.st[1], sz = mg.st[2];
        const float *base = c + ii[0] + ii[1] * sy + ii[2] * sz;
#pragma unroll
        for (int z = 0; z < 4; ++z) {
            float z0 = 0.f, z1 = 0.f, z3 = 0.f;
#pragma unroll
            for (int y = 0; y < 4; ++y) {
                const float *row = base + y * sy + z * sz;
                float a = __ldg(row), b = __ldg(row + 1), e = __ldg(row + 2), f = __ldg(row + 3);
                float dx = dW[0][0] * a + dW[1][0] * b + dW[2][0] * e + dW[3][0] * f;
                float vx = W[0][0] * a + W[1][0] * b + W[2][0] * e + W[3][0] * f;
                z0 += W[y][1] * dx;
                z1 += dW[y][1] * vx;
                z3 += W[y][1] * vx;
            }
            c0 += W[z][2] * z0;
            c1 += W[z][2] * z1;
            c2 += dW[z][2] * z3;
            c3 += W[z][2] * z3;
        }
        val = c3;
        grad[0] = c0 * (float)mg.inv[0];
        grad[1] = c1 * (float)mg.inv[1];
        grad[2] = c2 * (float)mg.inv[2];
    } else {
        float c0 = 0.f, c1 = 0.f, c2 = 0.f;
        const long long sy = mg.st[1];
        const float *base = c + ii[0] + ii[1] * sy;
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const float *row = base + y * sy;
            float a = __ldg(row), b = __ldg(row + 1), e = __ldg(row + 2), f = __ldg(row + 3);
            float dx = dW[0][0] * a + dW[1][0] * b + dW[2][0] * e + dW[3][0] * f;
            float vx = W[0][0] * a + W[1][0] * b + W[2][0] * e + W[3][0] * f;
            c0 += W[y][1] * dx;
            c1 += dW[y][1] * vx;
            c2 += W[y][1] * vx;
        }
        val = c2;
        grad[0] = c0 * (float)mg.inv[0];
        grad[1] = c1 * (float)mg.inv[1];
    }
}

// Cubic B-spline weights (value W and derivative dW) of the four stencil taps per axis at local
// coordinate l; ii = the stencil's first padded-grid index (VecI(idx): truncation toward zero).
template <int D>
__device__ __forceinline__ void bspline_weights(const double *l, int *ii, float (&W)[4][3], float (&dW)[4][3])
{
#pragma unroll
    for (int d = 0; d < D; ++d) {
        ii[d] = (int)l[d];
        float w = (float)(l[d] - (double)ii[d]);
        float w3 = (1.0f / 6.0f) * w * w * w;
        float w0 = (1.0f / 6.0f) + 0.5f * w * (w - 1.0f) - w3;
        float w2 = w + w0 - 2.0f * w3;
        W[3][d] = w3; W[0][d] = w0; W[2][d] = w2; W[1][d] = 1.0f - w0 - w2 - w3;
        float d3 = 0.5f * w * w;
        float d0 = w - 0.5f - d3;
        float d2 = 1.0f + d0 - 2.0f * d3;
        dW[3][d] = d3; dW[0][d] = d0; dW[2][d] = d2; dW[1][d] = -d0 - d2 - d3;
    }
}

// The 3-D stencil sum shared by the global-memory and the shared-memory versions: row(y, z)
// returns the four x coefficients of stencil row (y, z).
template <class Row>
__device__ __forceinline__ void bspline_sum3(const Row &row, const float (&W)[4][3], const float (&dW)[4][3],
                                             const Geo &mg, float &val, float *grad)
{
    float c0 = 0.f, c1 = 0.f, c2 = 0.f, c3 = 0.f;
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        float z0 = 0.f, z1 = 0.f, z3 = 0.f;
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const float4 r = row(y, z);
            float dx = dW[0][0] * r.x + dW[1][0] * r.y + dW[2][0] * r.z + dW[3][0] * r.w;
            float vx = W[0][0] * r.x + W[1][0] * r.y + W[2][0] * r.z + W[3][0] * r.w;
            z0 += W[y][1] * dx;
            z1 += dW[y][1] * vx;
            z3 += W[y][1] * vx;
        }
        c0 += W[z][2] * z0;
        c1 += W[z][2] * z1;
        c2 += dW[z][2] * z3;
        c3 += W[z][2] * z3;
    }
    val = c3;
    grad[0] = c0 * (float)mg.inv[0];
    grad[1] = c1 * (float)mg.inv[1];
    grad[2] = c2 * (float)mg.inv[2];
}

// The same stencil sum on packed FP32 pairs (sm_100 `fma.rn.f32x2`: one instruction, two
// round-to-nearest fused multiply-adds).  Rows y and y + 1 of a z slice travel together, so the
// x contractions of two rows, the y accumulations (even and odd y apart) and the z accumulations
// are all pair operations; the two halves are added at the end.  About 110 arithmetic
// instructions per stencil instead of 195; the sums group the rows differently from
// bspline_sum3, so results agree to FP32 rounding, not bitwise.
template <class Row>
__device__ __forceinline__ void bspline_sum3_x2(const Row &row, const float (&W)[4][3], const float (&dW)[4][3],
                                                const Geo &mg, float &val, float *grad)
{
    float2 bw[4], bd[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        bw[k] = make_float2(W[k][0], W[k][0]);
        bd[k] = make_float2(dW[k][0], dW[k][0]);
    }
    const float2 wy[2] = {make_float2(W[0][1], W[1][1]), make_float2(W[2][1], W[3][1])};
    const float2 dy[2] = {make_float2(dW[0][1], dW[1][1]), make_float2(dW[2][1], dW[3][1])};
    float2 c0 = make_float2(0.f, 0.f), c1 = c0, c2 = c0, c3 = c0;
#pragma unroll
    for (int z = 0; z < 4; ++z) {
        float2 z0 = make_float2(0.f, 0.f), z1 = z0, z3 = z0;
#pragma unroll
        for (int yp = 0; yp < 2; ++yp) {
            const float4 ra = row(2 * yp, z), rb = row(2 * yp + 1, z);
            const float2 px = make_float2(ra.x, rb.x), py = make_float2(ra.y, rb.y);
            const float2 pz = make_float2(ra.z, rb.z), pw = make_float2(ra.w, rb.w);
            float2 dx = __fmul2_rn(bd[0], px);
            dx = __ffma2_rn(bd[1], py, dx);
            dx = __ffma2_rn(bd[2], pz, dx);
            dx = __ffma2_rn(bd[3], pw, dx);
            float2 vx = __fmul2_rn(bw[0], px);
            vx = __ffma2_rn(bw[1], py, vx);
            vx = __ffma2_rn(bw[2], pz, vx);
            vx = __ffma2_rn(bw[3], pw, vx);
            z0 = __ffma2_rn(wy[yp], dx, z0);
            z1 = __ffma2_rn(dy[yp], vx, z1);
            z3 = __ffma2_rn(wy[yp], vx, z3);
        }
        const float2 wz = make_float2(W[z][2], W[z][2]), dz = make_float2(dW[z][2], dW[z][2]);
        c0 = __ffma2_rn(wz, z0, c0);
        c1 = __ffma2_rn(wz, z1, c1);
        c2 = __ffma2_rn(dz, z3, c2);
        c3 = __ffma2_rn(wz, z3, c3);
    }
    val = c3.x + c3.y;
    grad[0] = (c0.x + c0.y) * (float)mg.inv[0];
    grad[1] = (c1.x + c1.y) * (float)mg.inv[1];
    grad[2] = (c2.x + c2.y) * (float)mg.inv[2];
}

// Same as bspline_derivs, reading the coefficients from the row-expanded copy
// c4[i] = (c[i], c[i+1], c[i+2], c[i+3]): one aligned 16-byte load per stencil row.
template <int D>
__device__ __forceinline__ void bspline_derivs4(const float4 *__restrict__ c4, const Geo &mg, const double *l,
                                                float &val, float *grad)
{
    int ii[3] = {0, 0, 0};
    float W[4][3], dW[4][3];
    bspline_weights<D>(l, ii, W, dW);
    if (D == 3) {
        // 32-bit offsets: the coefficient volume holds fewer than 2^31 entries (checked at creation)
        const int sy = (int)mg.st[1], sz = (int)mg.st[2];
        const float4 *base = c4 + (ii[0] + ii[1] * sy + ii[2] * sz);
        bspline_sum3([&](int y, int z) { return __ldg(base + (y * sy + z * sz)); }, W, dW, mg, val, grad);
    } else {
        float c0 = 0.f, c1 = 0.f, c2 = 0.f;
        const int sy = (int)mg.st[1];
        const float4 *base = c4 + (ii[0] + ii[1] * sy);
#pragma unroll
        for (int y = 0; y < 4; ++y) {
            const float4 r = __ldg(base + y * sy);
            float dx = dW[0][0] * r.x + dW[1][0] * r.y + dW[2][0] * r.z + dW[3][0] * r.w;
            float vx = W[0][0] * r.x + W[1][0] * r.y + W[2][0] * r.z + W[3][0] * r.w;
            c0 += W[y][1] * dx;
            c1 += dW[y][1] * vx;
            c2 += W[y][1] * vx;
        }
        val = c2;
        grad[0] = c0 * (float)mg.inv[0];
        grad[1] = c1 * (float)mg.inv[1];
    }
}

// ---------------------------------------------------------------------------------------------
// PCG32 stream of UniformRng (UniformRng.h:28-46) with LCG jump-ahead so that every sample
// draws its own D values of the sequential stream in parallel.
struct RngJump {
    unsigned long long mul[64];   // a^(2^i)
    unsigned long long add[64];   // c*(a^(2^i)-1)/(a-1)
};

__device__ __forceinline__ unsigned long long lcg_advance(unsigned long long state, unsigned long long steps,
                                                          const RngJump &J)
{
    int i = 0;
    while (steps) {
        if (steps & 1ull) state = state * J.mul[i] + J.add[i];
        steps >>= 1;
        ++i;
    }
    return state;
}

__device__ __forceinline__ unsigned pcg32_output(unsigned long long old)
{
    unsigned xorshifted = (unsigned)(((old >> 18u) ^ old) >> 27u);
    unsigned rot = (unsigned)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((unsigned)(-(int)rot) & 31));
}

// ---------------------------------------------------------------------------------------------
// LCC window arithmetic (GpuEvaluatorLCC.cu:28-35, 152-191), every operation rounded as written.
// A window with one neighbour has sff = f*f, msf = f, so sff - 2*msf*sf + n*msf*msf is exactly 0
// when each product is rounded; a contracted multiply-add leaves the rounding error of f*f
// instead, which can pass the d1 > 0 && d2 > 0 test and turn into an arbitrary -cc^2/(d1*d2).
struct LccWindow {
    double sf = 0, sm = 0, sff = 0, smm = 0, sfm = 0;
    int n = 0;
    __device__ __forceinline__ void add(double fv, double mv)
    {
        sf = __dadd_rn(sf, fv);
        sm = __dadd_rn(sm, mv);
        sff = __dadd_rn(sff, __dmul_rn(fv, fv));
        smm = __dadd_rn(smm, __dmul_rn(mv, mv));
        sfm = __dadd_rn(sfm, __dmul_rn(fv, mv));
        ++n;
    }
    __device__ __forceinline__ double msf() const { return __ddiv_rn(sf, (double)n); }
    __device__ __forceinline__ double msm() const { return __ddiv_rn(sm, (double)n); }
    // s2 - 2*m*s + n*m*m
    __device__ __forceinline__ double centred(double s2, double s, double m) const
    {
        return __dadd_rn(__dsub_rn(s2, __dmul_rn(__dmul_rn(2.0, m), s)), __dmul_rn(__dmul_rn((double)n, m), m));
    }
    __device__ __forceinline__ double d1() const { return centred(sff, sf, msf()); }
    __device__ __forceinline__ double d2() const { return centred(smm, sm, msm()); }
    // sfm - msm*sf - msf*sm + n*msf*msm
    __device__ __forceinline__ double cross() const
    {
        double a = msf(), b = msm();
        return __dadd_rn(__dsub_rn(__dsub_rn(sfm, __dmul_rn(b, sf)), __dmul_rn(a, sm)),
                         __dmul_rn(__dmul_rn((double)n, a), b));
    }
    // the window's value: -cc^2 / (d1*d2) when both centred sums are positive, else 0
    __device__ __forceinline__ double value() const
    {
        if (n <= 0) return 0.0;
        double a = d1(), b = d2();
        if (!(a > 0 && b > 0)) return 0.0;
        double cc = cross();
        return __ddiv_rn(__dmul_rn(-cc, cc), __dmul_rn(a, b));
    }
};

// neighborhoodWeight(p, q, support, 10) (LCC.cu:28-35): (1 - (|p-q|/support)^10)^2, written as
// (r2/support^2)^5; returns a value <= 0 where the reference's weight is 0.  r2 and support^2
// are exact for grid positions and a float support, so the sign matches pow(|p-q|/support, 10).
template <int D>
__device__ __forceinline__ double lcc_weight_base(const double *p, const double *q, double support)
{
    double r2 = 0.0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
        double t = __dsub_rn(p[d], q[d]);
        r2 = __dadd_rn(r2, __dmul_rn(t, t));
    }
    double tt = __ddiv_rn(r2, __dmul_rn(support, support));
    double t2 = __dmul_rn(tt, tt);
    return __dsub_rn(1.0, __dmul_rn(__dmul_rn(t2, t2), tt));
}

// deterministic reductions (fixed shuffle tree, fixed block order)
template <typename T>
__device__ __forceinline__ T warp_sum(T v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Sum NV values over the block; result valid in thread 0.  `sh` holds NV*32 doubles.
template <int NV>
__device__ __forceinline__ void block_sum(double *v, double *sh)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] = warp_sum(v[k]);
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < NV; ++k) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < NV; ++k) {
            double x = lane < nw ? sh[k * 32 + lane] : 0.0;
            v[k] = warp_sum(x);
        }
    }
    __syncthreads();
}

}  // namespace skm
