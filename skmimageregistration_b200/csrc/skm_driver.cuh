// skm_driver.cuh -- preprocessing entry points and the multi-scale registration driver.
//
// skm_register restates the scale loop of the reference application (src/SKMReg.cxx:84-500):
// threshold + rescale both images (:85-90), then per scale level
//   smooth both images with the level's variance (:140-150),
//   prefilter the smoothed reference (moving) image into B-spline coefficients,
//   build the control-point grid with spacing min(sigma_C4, sigma_C0) / cp_spacing_scaler (:235-247,
//   itkTransformAdapter.hxx:246-308),
//   set up the evaluator (fixed = smoothed target, moving = smoothed reference) with the
//   displacement field of the previous levels as the frozen front transform (:127-136),
//   run the adaptive-step optimizer (a = initial step size, A = 20, alpha = 1, f_max = 1e7,
//   f_min = -1e6, omega = 1, best parameters; orthant projection when L1 or L2,1 is the only
//   regularizer) on the device (:392-442),
//   and evaluate the summed displacement field on the reference grid (:452-460).
// This file is included at the end of skm_capi.cu and uses its entry points.
#pragma once

#include <chrono>
#include <vector>

#include "skm_output.cuh"
#include "skm_preprocess.cuh"

namespace {

struct DevBuf {
    double *p = nullptr;
    ~DevBuf()
    {
        if (p) pool_free(p);
    }
};

int smooth_device(int D, const int *size, const double *spacing, double variance, int use_spacing,
                  double maximum_error, int maximum_width, double *d_img, double *d_tmp, cudaStream_t s)
{
    const int X = size[0], Y = D > 1 ? size[1] : 1, Z = D > 2 ? size[2] : 1;
    const long long n = (long long)X * Y * Z;
    double *src = d_img, *dst = d_tmp;
    for (int axis = 0; axis < D; ++axis) {
        const double sp = use_spacing ? spacing[axis] : 1.0;
        const std::vector<double> c = skm::gaussian_half_kernel(variance / (sp * sp), maximum_error, maximum_width);
        const int r = (int)c.size() - 1;
        if (r > skm::kSmoothMaxRadius) return fail(SKM_ERR_UNSUPPORTED, "smoothing kernel radius %d > %d", r,
                                                  skm::kSmoothMaxRadius);
        DevBuf dc;
        SKM_CUDA(pool_malloc((void **)&dc.p, c.size() * sizeof(double)));
        SKM_CUDA(cudaMemcpyAsync(dc.p, c.data(), c.size() * sizeof(double), cudaMemcpyHostToDevice, s));
        const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 16);
        skm::smooth_axis_kernel<<<blocks, 256, 0, s>>>(src, dst, X, Y, Z, axis, dc.p, r);
        SKM_CHECK_LAUNCH();
        SKM_CUDA(cudaStreamSynchronize(s));     // dc is freed at the end of this iteration
        std::swap(src, dst);
    }
    if (src != d_img) SKM_CUDA(cudaMemcpyAsync(d_img, src, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    return SKM_OK;
}

int threshold_rescale_device(long long n, int apply_threshold, double tmin, double tmax, double out_min,
                             double out_max, double *d_img, cudaStream_t s)
{
    const int blocks = (int)std::min<long long>((n + 255) / 256, 148LL * 4);
    DevBuf part, res;
    SKM_CUDA(pool_malloc((void **)&part.p, sizeof(double) * 4 * blocks));
    SKM_CUDA(pool_malloc((void **)&res.p, sizeof(double) * 4));
    skm::range_kernel<<<blocks, 256, 0, s>>>(d_img, n, tmin, tmax, part.p);
    SKM_CHECK_LAUNCH();
    skm::range_finish_kernel<<<1, 32, 0, s>>>(part.p, blocks, res.p);
    SKM_CHECK_LAUNCH();
    double r[4];
    SKM_CUDA(cudaMemcpyAsync(r, res.p, sizeof r, cudaMemcpyDeviceToHost, s));
    SKM_CUDA(cudaStreamSynchronize(s));
    double lo = r[0], hi = r[1];
    if (apply_threshold) {
        // largest value below tmax / smallest above tmin (itkUtils.h:50-62); none: nothing to keep
        if (r[2] == -DBL_MAX || r[3] == DBL_MAX || r[3] > r[2])
            return fail(SKM_ERR_INVALID, "no intensity inside the thresholds (%g, %g)", tmin, tmax);
        lo = r[3];
        hi = r[2];
    }
    // RescaleIntensityImageFilter: scale from the (thresholded) range, shift to out_min
    double scale;
    if (hi != lo) scale = (out_max - out_min) / (hi - lo);
    else if (hi != 0.0) scale = (out_max - out_min) / hi;
    else scale = 0.0;
    const double shift = out_min - lo * scale;
    skm::clamp_rescale_kernel<<<blocks, 256, 0, s>>>(d_img, n, lo, hi, scale, shift);
    SKM_CHECK_LAUNCH();
    return SKM_OK;
}

long long texel_count(int D, const int32_t *size)
{
    long long n = 1;
    for (int d = 0; d < D; ++d) n *= size[d];
    return n;
}

int grid_blocks(long long n, int per_sm)
{
    return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148LL * per_sm));
}

// largest value of d_v[0..n) (the max of range_kernel)
int device_max(const double *d_v, long long n, double *out, cudaStream_t s)
{
    const int blocks = grid_blocks(n, 4);
    DevBuf part, res;
    SKM_CUDA(pool_malloc((void **)&part.p, sizeof(double) * 4 * blocks));
    SKM_CUDA(pool_malloc((void **)&res.p, sizeof(double) * 4));
    skm::range_kernel<<<blocks, 256, 0, s>>>(d_v, n, 0.0, 0.0, part.p);
    SKM_CHECK_LAUNCH();
    skm::range_finish_kernel<<<1, 32, 0, s>>>(part.p, blocks, res.p);
    SKM_CHECK_LAUNCH();
    double r[4];
    SKM_CUDA(cudaMemcpyAsync(r, res.p, sizeof r, cudaMemcpyDeviceToHost, s));
    SKM_CUDA(cudaStreamSynchronize(s));
    *out = r[1];
    return SKM_OK;
}

// ComputeAnisotropicTensor (include/AnisotropicTensorUtils.h:37-371) with anisotropic_filtering
// false, the form src/SKMReg.cxx:271 and :284 call: d_img (n texels, unchanged) -> d_cov (n x D x D
// row-major) and the maximum tilt (largest |main row| after the alignment weighting over the texels
// that passed the 1e-8 test; -DBL_MAX when none did).
int anisotropic_tensor_device(int D, const int32_t *size, const double *spacing, const double *d_img, double sigma,
                              double weight, int alignment, double *d_cov, double *max_tilt, cudaStream_t s)
{
    const int X = size[0], Y = D > 1 ? size[1] : 1, Z = D > 2 ? size[2] : 1;
    const long long n = (long long)X * Y * Z;
    const int nc = skm::tensor_components(D);
    const int blocks = grid_blocks(n, 16);
    DevBuf f, tmp, comp, tilt;
    SKM_CUDA(pool_malloc((void **)&f.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&tmp.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&comp.p, nc * n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&tilt.p, n * sizeof(double)));
    unsigned *d_bad = nullptr;
    SKM_CUDA(pool_malloc((void **)&d_bad, sizeof(unsigned)));
    struct FreeBad {
        unsigned *p;
        ~FreeBad() { pool_free(p); }
    } free_bad{d_bad};
    SKM_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s));
    // weight * image, smoothed with variance sigma (:54-64)
    skm::scale_kernel<<<blocks, 256, 0, s>>>(d_img, f.p, n, weight);
    SKM_CHECK_LAUNCH();
    int rc = smooth_device(D, size, spacing, sigma, 1, 0.01, 64, f.p, tmp.p, s);
    if (rc) return rc;
    // gradient outer product (:65-103), every component smoothed with variance sigma / 4 (:106-155)
    if (D == 2)
        skm::gradient_outer_kernel<2><<<blocks, 256, 0, s>>>(f.p, X, Y, Z, 2.0 * spacing[0], 2.0 * spacing[1], 1.0,
                                                              comp.p);
    else
        skm::gradient_outer_kernel<3><<<blocks, 256, 0, s>>>(f.p, X, Y, Z, 2.0 * spacing[0], 2.0 * spacing[1],
                                                              2.0 * spacing[2], comp.p);
    SKM_CHECK_LAUNCH();
    for (int k = 0; k < nc; ++k)
        if ((rc = smooth_device(D, size, spacing, sigma / 4.0, 1, 0.01, 64, comp.p + k * n, tmp.p, s))) return rc;
    // eigen analysis, direction weighting and covariance (:160-371)
    if (D == 2)
        skm::covariance_kernel<2><<<blocks, 256, 0, s>>>(comp.p, n, alignment, d_cov, tilt.p, d_bad);
    else
        skm::covariance_kernel<3><<<blocks, 256, 0, s>>>(comp.p, n, alignment, d_cov, tilt.p, d_bad);
    SKM_CHECK_LAUNCH();
    unsigned bad = 0;
    SKM_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s));
    if ((rc = device_max(tilt.p, n, max_tilt, s))) return rc;
    if (bad) return fail(SKM_ERR_INVALID, "covariance tensor not positive definite at %u texels", bad);
    return SKM_OK;
}

// SetWeightingTensor with a negative tilt (itkTransformAdapter.hxx:341-361): the tensor whose
// largest eigenvalue has the largest magnitude (the first such texel), after the determinant test.
int max_eigenvalue_tensor(int D, long long n, const double *d_tensor, const double *h_tensor, double *maximum,
                          double *cov_out, cudaStream_t s)
{
    DevBuf ev;
    SKM_CUDA(pool_malloc((void **)&ev.p, n * sizeof(double)));
    unsigned *d_bad = nullptr;
    SKM_CUDA(pool_malloc((void **)&d_bad, sizeof(unsigned)));
    struct FreeBad {
        unsigned *p;
        ~FreeBad() { pool_free(p); }
    } free_bad{d_bad};
    SKM_CUDA(cudaMemsetAsync(d_bad, 0, sizeof(unsigned), s));
    const int blocks = grid_blocks(n, 16);
    if (D == 2) skm::max_eigenvalue_kernel<2><<<blocks, 256, 0, s>>>(d_tensor, n, ev.p, d_bad);
    else skm::max_eigenvalue_kernel<3><<<blocks, 256, 0, s>>>(d_tensor, n, ev.p, d_bad);
    SKM_CHECK_LAUNCH();
    std::vector<double> h((size_t)n);
    unsigned bad = 0;
    SKM_CUDA(cudaMemcpyAsync(h.data(), ev.p, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    SKM_CUDA(cudaMemcpyAsync(&bad, d_bad, sizeof bad, cudaMemcpyDeviceToHost, s));
    SKM_CUDA(cudaStreamSynchronize(s));
    if (bad) return fail(SKM_ERR_INVALID, "weighting tensors must be positive definite (%u texels are not)", bad);
    long long best = 0;
    double mx = -DBL_MAX;
    for (long long i = 0; i < n; ++i)
        if (h[(size_t)i] > mx) {
            mx = h[(size_t)i];
            best = i;
        }
    *maximum = mx;
    for (int k = 0; k < 9; ++k) cov_out[k] = 0.0;
    for (int r = 0; r < D; ++r)
        for (int c = 0; c < D; ++c) cov_out[r * D + c] = h_tensor[best * D * D + r * D + c];
    return SKM_OK;
}

struct HostStream {
    cudaStream_t s = nullptr;
    ~HostStream()
    {
        if (s) cudaStreamDestroy(s);
    }
};

}  // namespace

extern "C" int skm_gaussian_smooth(int32_t dimensions, const skm_geometry *geometry, double variance,
                                   int32_t use_image_spacing, double maximum_error, int32_t maximum_kernel_width,
                                   const double *src, double *dst)
{
    if (dimensions != 2 && dimensions != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (!geometry || !src || !dst) return fail(SKM_ERR_INVALID, "geometry / src / dst is NULL");
    if (!(variance >= 0.0) || !(maximum_error > 0.0 && maximum_error < 1.0) || maximum_kernel_width < 1)
        return fail(SKM_ERR_INVALID, "variance >= 0, 0 < maximum_error < 1 and maximum_kernel_width >= 1 required");
    for (int d = 0; d < dimensions; ++d)
        if (geometry->size[d] < 1 || (use_image_spacing && !(geometry->spacing[d] > 0.0)))
            return fail(SKM_ERR_INVALID, "size and spacing must be positive");
    const long long n = texel_count(dimensions, geometry->size);
    HostStream hs;
    SKM_CUDA(cudaStreamCreateWithFlags(&hs.s, cudaStreamNonBlocking));
    DevBuf a, b;
    SKM_CUDA(pool_malloc((void **)&a.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&b.p, n * sizeof(double)));
    SKM_CUDA(cudaMemcpyAsync(a.p, src, n * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    int rc = smooth_device(dimensions, geometry->size, geometry->spacing, variance, use_image_spacing, maximum_error,
                           maximum_kernel_width, a.p, b.p, hs.s);
    if (rc) return rc;
    SKM_CUDA(cudaMemcpyAsync(dst, a.p, n * sizeof(double), cudaMemcpyDeviceToHost, hs.s));
    SKM_CUDA(cudaStreamSynchronize(hs.s));
    return SKM_OK;
}

extern "C" int skm_threshold_rescale(int32_t dimensions, const int32_t *size, int32_t apply_threshold,
                                     double threshold_min, double threshold_max, double out_min, double out_max,
                                     const double *src, double *dst)
{
    if (dimensions != 2 && dimensions != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (!size || !src || !dst) return fail(SKM_ERR_INVALID, "size / src / dst is NULL");
    for (int d = 0; d < dimensions; ++d)
        if (size[d] < 1) return fail(SKM_ERR_INVALID, "size must be positive");
    const long long n = texel_count(dimensions, size);
    HostStream hs;
    SKM_CUDA(cudaStreamCreateWithFlags(&hs.s, cudaStreamNonBlocking));
    DevBuf a;
    SKM_CUDA(pool_malloc((void **)&a.p, n * sizeof(double)));
    SKM_CUDA(cudaMemcpyAsync(a.p, src, n * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    int rc = threshold_rescale_device(n, apply_threshold, threshold_min, threshold_max, out_min, out_max, a.p, hs.s);
    if (rc) return rc;
    SKM_CUDA(cudaMemcpyAsync(dst, a.p, n * sizeof(double), cudaMemcpyDeviceToHost, hs.s));
    SKM_CUDA(cudaStreamSynchronize(hs.s));
    return SKM_OK;
}

extern "C" int skm_anisotropic_tensor(int32_t dimensions, const skm_geometry *geometry, const double *image,
                                      double sigma, double weight, int32_t alignment_direction, double *covariance,
                                      double *maximum_tilt)
{
    if (dimensions != 2 && dimensions != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (!geometry || !image || !covariance) return fail(SKM_ERR_INVALID, "geometry / image / covariance is NULL");
    if (!(sigma >= 0.0) || !std::isfinite(sigma) || !std::isfinite(weight))
        return fail(SKM_ERR_INVALID, "sigma must be finite and >= 0, weight finite");
    for (int d = 0; d < dimensions; ++d)
        if (geometry->size[d] < 1 || !(geometry->spacing[d] > 0.0))
            return fail(SKM_ERR_INVALID, "size and spacing must be positive");
    const long long n = texel_count(dimensions, geometry->size);
    const long long nt = n * dimensions * dimensions;
    HostStream hs;
    SKM_CUDA(cudaStreamCreateWithFlags(&hs.s, cudaStreamNonBlocking));
    DevBuf img, cov;
    SKM_CUDA(pool_malloc((void **)&img.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&cov.p, nt * sizeof(double)));
    SKM_CUDA(cudaMemcpyAsync(img.p, image, n * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    double tilt = -DBL_MAX;
    int rc = anisotropic_tensor_device(dimensions, geometry->size, geometry->spacing, img.p, sigma, weight,
                                       alignment_direction, cov.p, &tilt, hs.s);
    if (rc) return rc;
    SKM_CUDA(cudaMemcpyAsync(covariance, cov.p, nt * sizeof(double), cudaMemcpyDeviceToHost, hs.s));
    SKM_CUDA(cudaStreamSynchronize(hs.s));
    if (maximum_tilt) *maximum_tilt = tilt;
    return SKM_OK;
}

namespace {

skm::OutGeo out_geo(int D, const skm_geometry &g)
{
    skm::OutGeo o{};
    for (int d = 0; d < 3; ++d) {
        o.o[d] = d < D ? g.origin[d] : 0.0;
        o.s[d] = d < D ? g.spacing[d] : 1.0;
        o.n[d] = d < D ? g.size[d] : 1;
    }
    return o;
}

bool out_geometry_ok(int D, const skm_geometry *g)
{
    if (!g) return false;
    for (int d = 0; d < D; ++d)
        if (g->size[d] < 1 || !(g->spacing[d] > 0.0) || !std::isfinite(g->origin[d])) return false;
    return true;
}

}  // namespace

extern "C" int skm_warp_image(int32_t dimensions, const skm_geometry *image_geometry, const double *image,
                              const skm_geometry *field_geometry, const double *field, int32_t order,
                              double default_value, double *out)
{
    if (dimensions != 2 && dimensions != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (!image || !field || !out) return fail(SKM_ERR_INVALID, "image / field / out is NULL");
    if (!out_geometry_ok(dimensions, image_geometry) || !out_geometry_ok(dimensions, field_geometry))
        return fail(SKM_ERR_INVALID, "invalid geometry (size < 1, spacing <= 0 or origin not finite)");
    if (order != 1 && order != 3) return fail(SKM_ERR_UNSUPPORTED, "interpolation order %d (1 or 3)", order);
    const int D = dimensions;
    if (order == 3)
        for (int d = 0; d < D; ++d)
            if (image_geometry->size[d] < 2)
                return fail(SKM_ERR_INVALID, "cubic interpolation needs at least 2 texels per axis");
    const long long ni = texel_count(D, image_geometry->size), nf = texel_count(D, field_geometry->size);
    HostStream hs;
    SKM_CUDA(cudaStreamCreateWithFlags(&hs.s, cudaStreamNonBlocking));
    DevBuf di, df, dout;
    SKM_CUDA(pool_malloc((void **)&di.p, ni * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&df.p, nf * D * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dout.p, nf * sizeof(double)));
    SKM_CUDA(cudaMemcpyAsync(di.p, image, ni * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    SKM_CUDA(cudaMemcpyAsync(df.p, field, nf * D * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    const skm::OutGeo gi = out_geo(D, *image_geometry), gf = out_geo(D, *field_geometry);
    if (order == 3) {
        // the evaluator's prefilter, in place, without the mirror padding
        const int X = gi.n[0], Y = gi.n[1], Z = gi.n[2];
        const double pole = std::sqrt(3.0) - 2.0;
        if (D == 3) {
            skm::bs_prefilter_axis<<<(int)(((long long)X * Y + 127) / 128), 128, 0, hs.s>>>(di.p, X, Y, Z, 2, pole);
            skm::bs_prefilter_axis<<<(int)(((long long)X * Z + 127) / 128), 128, 0, hs.s>>>(di.p, X, Y, Z, 1, pole);
            skm::bs_prefilter_axis<<<(int)(((long long)Y * Z + 127) / 128), 128, 0, hs.s>>>(di.p, X, Y, Z, 0, pole);
        } else {
            skm::bs_prefilter_axis<<<(Y + 127) / 128, 128, 0, hs.s>>>(di.p, X, Y, 1, 0, pole);
            skm::bs_prefilter_axis<<<(X + 127) / 128, 128, 0, hs.s>>>(di.p, X, Y, 1, 1, pole);
        }
        SKM_CHECK_LAUNCH();
    }
    const int blocks = grid_blocks(nf, 16);
    if (D == 2 && order == 1) skm::warp_kernel<2, 1><<<blocks, 256, 0, hs.s>>>(di.p, gi, df.p, gf, default_value, dout.p);
    if (D == 2 && order == 3) skm::warp_kernel<2, 3><<<blocks, 256, 0, hs.s>>>(di.p, gi, df.p, gf, default_value, dout.p);
    if (D == 3 && order == 1) skm::warp_kernel<3, 1><<<blocks, 256, 0, hs.s>>>(di.p, gi, df.p, gf, default_value, dout.p);
    if (D == 3 && order == 3) skm::warp_kernel<3, 3><<<blocks, 256, 0, hs.s>>>(di.p, gi, df.p, gf, default_value, dout.p);
    SKM_CHECK_LAUNCH();
    SKM_CUDA(cudaMemcpyAsync(out, dout.p, nf * sizeof(double), cudaMemcpyDeviceToHost, hs.s));
    SKM_CUDA(cudaStreamSynchronize(hs.s));
    return SKM_OK;
}

extern "C" int skm_jacobian_determinant(int32_t dimensions, const skm_geometry *geometry, const double *field,
                                        double *out)
{
    if (dimensions != 2 && dimensions != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (!field || !out) return fail(SKM_ERR_INVALID, "field / out is NULL");
    if (!out_geometry_ok(dimensions, geometry)) return fail(SKM_ERR_INVALID, "invalid geometry");
    const int D = dimensions;
    const long long n = texel_count(D, geometry->size);
    HostStream hs;
    SKM_CUDA(cudaStreamCreateWithFlags(&hs.s, cudaStreamNonBlocking));
    DevBuf du, dout;
    SKM_CUDA(pool_malloc((void **)&du.p, n * D * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dout.p, n * sizeof(double)));
    SKM_CUDA(cudaMemcpyAsync(du.p, field, n * D * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    const skm::OutGeo g = out_geo(D, *geometry);
    if (D == 2) skm::jacobian_determinant_kernel<2><<<grid_blocks(n, 16), 256, 0, hs.s>>>(du.p, g, dout.p);
    else skm::jacobian_determinant_kernel<3><<<grid_blocks(n, 16), 256, 0, hs.s>>>(du.p, g, dout.p);
    SKM_CHECK_LAUNCH();
    SKM_CUDA(cudaMemcpyAsync(out, dout.p, n * sizeof(double), cudaMemcpyDeviceToHost, hs.s));
    SKM_CUDA(cudaStreamSynchronize(hs.s));
    return SKM_OK;
}

namespace {

// ComputeControlPointImage (itkTransformAdapter.hxx:246-308): size ceil(extent / spacing), the grid
// centred on the image extent
void control_grid(int D, const skm_geometry &img, double spacing, skm_geometry &cp)
{
    cp = skm_geometry{};
    for (int d = 0; d < 3; ++d) {
        if (d >= D) {
            cp.origin[d] = 0.0;
            cp.spacing[d] = 1.0;
            cp.size[d] = 1;
            continue;
        }
        const double lower = img.origin[d], upper = img.origin[d] + (img.size[d] - 1) * img.spacing[d];
        const int n = (int)std::ceil(std::fabs((upper - lower) / spacing));
        const double cp_upper = img.origin[d] + (n - 1) * spacing;
        cp.size[d] = n;
        cp.spacing[d] = spacing;
        cp.origin[d] = img.origin[d] + std::fabs(upper - cp_upper) / 2.0;
    }
}

int check_register_desc(const skm_register_desc *r)
{
    if (!r) return fail(SKM_ERR_INVALID, "register descriptor is NULL");
    if (r->dimensions != 2 && r->dimensions != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (r->num_scales < 1 || r->num_scales > SKM_MAX_SCALES)
        return fail(SKM_ERR_INVALID, "num_scales must be in [1, %d]", SKM_MAX_SCALES);
    if (r->metric != SKM_MSE && r->metric != SKM_NCC && r->metric != SKM_LCC && r->metric != SKM_LCC_BOX)
        return fail(SKM_ERR_INVALID, "unknown metric %d", r->metric);
    for (int s = 0; s < r->num_scales; ++s) {
        if (!(r->sigma_c4[s] > 0.0) || !(r->sigma_c0[s] > 0.0))
            return fail(SKM_ERR_INVALID, "scale %d: sigma_C4 and sigma_C0 must be positive", s);
        if (r->sampling_rate[s] < 1 || r->neighborhood_sampling[s] < 1)
            return fail(SKM_ERR_INVALID, "scale %d: sampling rate and neighborhood sampling must be >= 1", s);
        if (r->num_function_evaluations[s] < 0 || !(r->smoothing_variance[s] >= 0.0))
            return fail(SKM_ERR_INVALID, "scale %d: negative iterations or smoothing variance", s);
    }
    return SKM_OK;
}

}  // namespace

extern "C" int skm_register(const skm_register_desc *r, const skm_geometry *geometry, const double *reference,
                            const double *target, double *displacement, skm_register_report *report)
{
    int rc;
    if ((rc = check_register_desc(r))) return rc;
    if (!geometry || !reference || !target || !displacement)
        return fail(SKM_ERR_INVALID, "geometry / reference / target / displacement is NULL");
    const int D = r->dimensions;
    for (int d = 0; d < D; ++d)
        if (geometry->size[d] < 4 || !(geometry->spacing[d] > 0.0))
            return fail(SKM_ERR_INVALID, "image size must be >= 4 and spacing positive along every axis");
    const long long n = texel_count(D, geometry->size);
    skm_register_report rep{};
    HostStream hs;
    SKM_CUDA(cudaStreamCreateWithFlags(&hs.s, cudaStreamNonBlocking));

    // preprocessing of both images (SKMReg.cxx:85-90)
    DevBuf dref, dtar, dtmp;
    SKM_CUDA(pool_malloc((void **)&dref.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dtar.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dtmp.p, n * sizeof(double)));
    SKM_CUDA(cudaMemcpyAsync(dref.p, reference, n * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    SKM_CUDA(cudaMemcpyAsync(dtar.p, target, n * sizeof(double), cudaMemcpyHostToDevice, hs.s));
    if ((rc = threshold_rescale_device(n, r->apply_threshold, r->threshold_min, r->threshold_max, 0.0, 1.0, dref.p,
                                       hs.s)))
        return rc;
    if ((rc = threshold_rescale_device(n, r->apply_threshold, r->threshold_min, r->threshold_max, 0.0, 1.0, dtar.p,
                                       hs.s)))
        return rc;

    // every level's images, coefficients and the summed field stay on the device: the smoothed
    // copies, the prefiltered reference and the field of the levels so far (past) go to the
    // evaluator and the optimizer as device pointers, and the next summed field (now) is written
    // on the device; the host sees the field only for the level callback and at the end
    long long ncoef = 1;
    for (int d = 0; d < D; ++d) ncoef *= geometry->size[d] + 3;
    const int GX = geometry->size[0], GY = D > 1 ? geometry->size[1] : 1, GZ = D > 2 ? geometry->size[2] : 1;
    DevBuf dref_s, dtar_s, dcoef, dpast, dnow;
    SKM_CUDA(pool_malloc((void **)&dref_s.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dtar_s.p, n * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dcoef.p, ncoef * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dpast.p, n * D * sizeof(double)));
    SKM_CUDA(pool_malloc((void **)&dnow.p, n * D * sizeof(double)));
    SKM_CUDA(cudaMemsetAsync(dpast.p, 0, n * D * sizeof(double), hs.s));
    std::vector<double> past_host;                  // the level callback's copy

    // kernel weighting (SKMReg.cxx:245-297): a weight image, or per level a covariance tensor built
    // from the guidance image / the smoothed target, or an external tensor where the weight is 0
    double max_weight_image = 0.0;
    if (r->weight_image)
        for (long long i = 0; i < n; ++i) max_weight_image = std::max(max_weight_image, r->weight_image[i]);
    bool any_tensor = false;
    for (int s = 0; s < r->num_scales; ++s) any_tensor = any_tensor || r->tensor_weights[s] > 0.0;
    DevBuf dguide, dcov, dext;
    std::vector<double> tensor;
    const long long nt = n * D * D;
    if (any_tensor) {
        SKM_CUDA(pool_malloc((void **)&dcov.p, nt * sizeof(double)));
        if (r->guidance_image) {
            SKM_CUDA(pool_malloc((void **)&dguide.p, n * sizeof(double)));
            SKM_CUDA(cudaMemcpyAsync(dguide.p, r->guidance_image, n * sizeof(double), cudaMemcpyHostToDevice, hs.s));
        }
        tensor.resize((size_t)nt);
    }
    double ext_maximum = 0.0, ext_cov[9] = {};
    bool ext_ready = false;

    // restart on a later level with the field of the levels before it (SKMReg.cxx:96-123)
    int first = 0;
    if (r->restart_at > 1 && r->restart_at <= r->num_scales && r->initial_displacement) {
        first = r->restart_at - 1;
        SKM_CUDA(cudaMemcpyAsync(dpast.p, r->initial_displacement, sizeof(double) * n * D, cudaMemcpyDefault, hs.s));
    }
    rep.first_level = first;

    for (int s = first; s < r->num_scales; ++s) {
        const auto t0 = std::chrono::steady_clock::now();
        // smoothed copies of both images (SKMReg.cxx:140-150), the reference prefiltered into its
        // B-spline coefficients (in place on a scratch copy)
        for (int which = 0; which < 2; ++which) {
            double *dst = which == 0 ? dref_s.p : dtar_s.p;
            SKM_CUDA(cudaMemcpyAsync(dst, which == 0 ? dref.p : dtar.p, n * sizeof(double), cudaMemcpyDeviceToDevice,
                                     hs.s));
            if (r->smoothing_variance[s] > 1e-5 &&
                (rc = smooth_device(D, geometry->size, geometry->spacing, r->smoothing_variance[s], 1, 0.01, 64,
                                    dst, dtmp.p, hs.s)))
                return rc;
        }
        SKM_CUDA(cudaMemcpyAsync(dtmp.p, dref_s.p, n * sizeof(double), cudaMemcpyDeviceToDevice, hs.s));
        if ((rc = bspline_coefficients_device(D, GX, GY, GZ, dtmp.p, dcoef.p, hs.s))) return rc;
        SKM_CUDA(cudaStreamSynchronize(hs.s));

        // control-point grid (SKMReg.cxx:235-247)
        // in float, as the reference computes it
        const float smin = std::min((float)r->sigma_c4[s], (float)r->sigma_c0[s]);
        const double cps = r->cp_spacing_scaler < 1.0 ? (double)(smin / 1.0f)
                                                      : (double)(smin / (float)r->cp_spacing_scaler);
        skm_geometry cpg;
        control_grid(D, *geometry, cps, cpg);
        const long long C = texel_count(D, cpg.size);
        std::vector<double> cpw((size_t)C, 1.0), params((size_t)C * D, 0.0), best((size_t)C * D);
        if (r->first_level_parameters && s == first) {             // learned warm start of the first level run
            if (r->first_level_parameter_count != C * D)
                return fail(SKM_ERR_INVALID, "first_level_parameters: %lld values, the level has %lld",
                            (long long)r->first_level_parameter_count, C * D);
            std::memcpy(params.data(), r->first_level_parameters, sizeof(double) * C * D);
        }

        skm_evaluator_desc ed{};
        ed.dimensions = D;
        ed.num_parameters = (int32_t)(C * D);
        ed.subsample = r->sampling_rate[s];
        ed.subsample_neighborhood = r->neighborhood_sampling[s];
        ed.sigma_c0 = r->sigma_c0[s];
        ed.sigma_c4 = r->sigma_c4[s];
        ed.use_weight_image = 0;
        ed.use_weight_tensor = 0;
        for (int d = 0; d < 3; ++d) {
            ed.weight_image_geometry.size[d] = 1;
            ed.weight_image_geometry.spacing[d] = 1.0;
            ed.weight_tensor_geometry.size[d] = 1;
            ed.weight_tensor_geometry.spacing[d] = 1.0;
        }
        // kernel weighting of this level (SKMReg.cxx:245-297)
        const double tw = r->tensor_weights[s];
        bool has_tensor = false;
        const double *tensor_ptr = nullptr;
        double tensor_weight = 1.0, tensor_cov[9] = {};
        for (int d = 0; d < D; ++d) tensor_cov[d * D + d] = 1.0;
        if (tw > 0.0) {
            // cases 3 and 4 (:269-286): tensor from the guidance image or the smoothed target with
            // sigma_C4 and this level's weight, alignment axis z.  SetWeightingTensor with the tilt
            // it returns (itkTransformAdapter.hxx:341-365): tilt >= 0 becomes the maximum weight and
            // the support covariance stays the identity; a negative tilt means no texel passed, every
            // tensor is the identity and so is the one with the largest eigenvalue (weight 1)
            double tilt = -DBL_MAX;
            if ((rc = anisotropic_tensor_device(D, geometry->size, geometry->spacing, dguide.p ? dguide.p : dtar_s.p,
                                                (double)(float)r->sigma_c4[s], tw, 2, dcov.p, &tilt, hs.s)))
                return rc;
            SKM_CUDA(cudaMemcpyAsync(tensor.data(), dcov.p, nt * sizeof(double), cudaMemcpyDeviceToHost, hs.s));
            SKM_CUDA(cudaStreamSynchronize(hs.s));
            has_tensor = true;
            tensor_ptr = tensor.data();
            tensor_weight = tilt >= 0.0 ? tilt : 1.0;
        } else if (tw == 0.0 && r->weight_tensor) {
            // case 2 (:259-268): external tensor with tilt -1: the tensor whose largest eigenvalue is
            // largest gives the support covariance and the maximum weight
            if (!ext_ready) {
                SKM_CUDA(pool_malloc((void **)&dext.p, nt * sizeof(double)));
                SKM_CUDA(cudaMemcpyAsync(dext.p, r->weight_tensor, nt * sizeof(double), cudaMemcpyHostToDevice,
                                         hs.s));
                if ((rc = max_eigenvalue_tensor(D, n, dext.p, r->weight_tensor, &ext_maximum, ext_cov, hs.s)))
                    return rc;
                ext_ready = true;
            }
            has_tensor = true;
            tensor_ptr = r->weight_tensor;
            tensor_weight = ext_maximum;
            for (int k = 0; k < 9; ++k) tensor_cov[k] = ext_cov[k];
        }
        if (r->weight_image) {
            // SetWeightingImage (itkTransformAdapter.hxx:312-331) sets the maximum weight, which a
            // later SetWeightingTensor overwrites; every kernel reads the weight image before any
            // tensor (GpuEvaluatorDisplacementField.cu:43-50), so the tensor itself goes unused
            ed.use_weight_image = 1;
            ed.maximum_weight = has_tensor ? tensor_weight : max_weight_image;
            ed.weight_image = r->weight_image;
            ed.weight_image_geometry = *geometry;
        } else if (has_tensor) {
            ed.use_weight_tensor = 1;
            ed.maximum_weight = tensor_weight;
            ed.weight_tensor = tensor_ptr;
            ed.weight_tensor_geometry = *geometry;
            for (int k = 0; k < 9; ++k) ed.maximum_eigenvalue_covariance[k] = tensor_cov[k];
        }
        ed.moving_coefficients = dcoef.p;                           // device memory, read in place
        ed.moving_geometry = *geometry;
        ed.fixed_image = dtar_s.p;
        ed.fixed_geometry = *geometry;
        ed.cp_geometry = cpg;
        ed.cpw_geometry = cpg;
        skm_evaluator *ev = nullptr;
        if ((rc = skm_evaluator_create(&ed, &ev))) return rc;

        skm_metric_desc md{};
        md.metric = r->metric;
        md.reg_l1 = r->reg_l1[s];
        md.reg_l21 = r->reg_l21[s];
        md.reg_l2 = r->reg_l2[s];
        md.reg_rkhs = r->reg_rkhs[s];
        md.reg_rd = r->reg_rd[s];
        md.reg_rd_scaling = r->reg_rd_scaling[s];
        md.reg_pg = r->reg_pg[s];
        md.reg_pg_scaling = r->reg_pg_scaling[s];
        md.use_negative_gradient = 1;
        md.do_resampling = 1;
        const bool only_l1 = md.reg_l1 > 0 && md.reg_l21 <= 0 && md.reg_l2 <= 0 && md.reg_rkhs <= 0 &&
                             md.reg_rd <= 0 && md.reg_pg <= 0;
        const bool only_l21 = md.reg_l1 <= 0 && md.reg_l21 > 0 && md.reg_l2 <= 0 && md.reg_rkhs <= 0 &&
                              md.reg_rd <= 0 && md.reg_pg <= 0;
        skm_optimizer_desc od{};
        od.a = r->initial_step_size[s];
        od.A = 20.0;
        od.alpha = 1.0;
        od.f_max = 1e7;
        od.f_min = -1e6;
        od.omega = 1.0;
        od.orthant_projection = (only_l1 || only_l21) ? 1 : 0;
        od.number_of_iterations = r->num_function_evaluations[s];
        od.return_best_parameters_and_value = 1;

        skm_field df{};
        df.data = s > 0 ? dpast.p : nullptr;
        df.geometry = *geometry;
        skm_optimizer *opt = nullptr;
        rc = skm_optimizer_create(ev, &od, &md, params.data(), cpw.data(), &df, &opt);
        skm_optimizer_state st{};
        const auto t_opt = std::chrono::steady_clock::now();
        if (!rc) rc = skm_optimizer_run(opt, r->num_function_evaluations[s]);
        rep.optimize_seconds[s] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t_opt).count();
        if (!rc) rc = skm_optimizer_get_parameters(opt, 1, best.data());
        if (!rc) rc = skm_optimizer_get_state(opt, &st);
        if (opt) skm_optimizer_destroy(opt);
        if (rc) {
            skm_evaluator_destroy(ev);
            return rc;
        }
        if (r->level_parameters) r->level_parameters(s, best.data(), C * D, r->level_user);
        // summed displacement field on the reference grid (SKMReg.cxx:452-460): planar -> AoS
        std::vector<double> cp_aos((size_t)C * D);
        for (long long i = 0; i < C; ++i)
            for (int d = 0; d < D; ++d) cp_aos[(size_t)(i * D + d)] = best[(size_t)(d * C + i)];
        rc = skm_evaluate_displacement_field(ev, cp_aos.data(), cpw.data(), &df, dnow.p);
        skm_evaluator_destroy(ev);
        if (rc) return rc;
        std::swap(dpast.p, dnow.p);
        rep.levels_done = s + 1;
        rep.best_value[s] = st.best_value;
        rep.iterations[s] = st.iteration;
        rep.control_points[s] = C;
        rep.seconds[s] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (r->level_done) {                                         // df-full-<s> (SKMReg.cxx:468)
            past_host.resize((size_t)n * D);
            SKM_CUDA(cudaMemcpy(past_host.data(), dpast.p, sizeof(double) * n * D, cudaMemcpyDeviceToHost));
            r->level_done(s, past_host.data(), r->level_user);
        }
    }
    SKM_CUDA(cudaMemcpy(displacement, dpast.p, sizeof(double) * n * D, cudaMemcpyDeviceToHost));
    if (report) *report = rep;
    return SKM_OK;
}
