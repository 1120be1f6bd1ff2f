/*
 * ref_host_kat.cpp -- host-side known-answer driver around the reference's own
 * __host__ __device__ math headers (include/cuda/{Kernel,BsplineImage,UniformRng,Mat}.h).
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles this file together with the
 * unmodified reference headers (include path -> the reference checkout) into
 * oracle/_ref/libskmref_host_d{2,3}.so.  The golden-vector script calls it to pin
 * the FP64 oracle to the reference's own arithmetic; nothing in the product links it.
 */
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <vector>

#include "CommonConfig.h"
#include "Vec.h"
#include "Mat.h"
#include "ImageNearest.h"
#include "BsplineImage.h"
#include "Kernel.h"
#include "UniformRng.h"

#include "../include/skm_gpu.h"

namespace {
constexpr int D = SpaceDimensions;
typedef Vec<ScalarType, D> VecT;
typedef Vec<int, D> VecIT;
typedef Mat<ScalarType, D> MatT;

VecT vec_of(const double *p)
{
    VecT v;
    for (int d = 0; d < D; ++d) v[d] = ScalarType(p[d]);
    return v;
}

VecIT veci_of(const int32_t *p)
{
    VecIT v;
    for (int d = 0; d < D; ++d) v[d] = p[d];
    return v;
}
}  // namespace

extern "C" int skmref_dimensions() { return D; }

/* BsplineImage::computeCoeffs (BsplineImage.h:209-221) */
extern "C" void skmref_bspline_coefficients(const int32_t *size, const double *image, double *coeffs)
{
    VecIT sz = veci_of(size);
    std::vector<ScalarType> src(sz.product());
    for (size_t i = 0; i < src.size(); ++i) src[i] = ScalarType(image[i]);
    BsplineImage<ScalarType, D> img(nullptr, VecT(0.0), VecT(1.0), sz);
    std::unique_ptr<ScalarType[]> out;
    img.computeCoeffs(src.data(), out);
    VecIT psz = sz + 3;
    for (int i = 0; i < psz.product(); ++i) coeffs[i] = double(out[i]);
}

/* BsplineImage::insideGlobal + derivsGlobal (BsplineImage.h:247-265,285-296) */
extern "C" void skmref_bspline_sample(const double *coeffs, const skm_geometry *g, int64_t n,
                                      const double *pts, int32_t *inside, double *vals, double *grads)
{
    VecIT sz = veci_of(g->size);
    std::vector<ScalarType> c((sz + 3).product());
    for (size_t i = 0; i < c.size(); ++i) c[i] = ScalarType(coeffs[i]);
    BsplineImage<ScalarType, D> img(c.data(), vec_of(g->origin), vec_of(g->spacing), sz);
    for (int64_t i = 0; i < n; ++i) {
        VecT p = vec_of(pts + i * D);
        ScalarType v = 0;
        VecT gr(0.0);
        inside[i] = img.insideLocal(img.toLocal(p)) ? 1 : 0;
        if (inside[i]) img.derivsGlobal(p, v, gr);
        vals[i] = double(v);
        for (int d = 0; d < D; ++d) grads[i * D + d] = double(gr[d]);
    }
}

/* GKernel<float>::evaluate (Kernel.h:173-186) with the descriptor's kernel kind. */
extern "C" void skmref_kernel_values(const skm_evaluator_desc *d, int64_t n, const double *p,
                                     const double *q, double *k)
{
    std::vector<ScalarType> wi;
    std::vector<MatT> wt;
    ImageNearest<ScalarType, D> wimg;
    ImageNearest<MatT, D> wten;
    if (d->use_weight_image) {
        VecIT sz = veci_of(d->weight_image_geometry.size);
        wi.resize(sz.product());
        for (size_t i = 0; i < wi.size(); ++i) wi[i] = ScalarType(d->weight_image[i]);
        wimg = ImageNearest<ScalarType, D>(wi.data(), vec_of(d->weight_image_geometry.origin),
                                           vec_of(d->weight_image_geometry.spacing), sz);
    }
    if (d->use_weight_tensor) {
        VecIT sz = veci_of(d->weight_tensor_geometry.size);
        wt.resize(sz.product());
        for (size_t i = 0; i < wt.size(); ++i)
            for (int e = 0; e < D * D; ++e) wt[i][e] = ScalarType(d->weight_tensor[i * D * D + e]);
        wten = ImageNearest<MatT, D>(wt.data(), vec_of(d->weight_tensor_geometry.origin),
                                     vec_of(d->weight_tensor_geometry.spacing), sz);
    }
    MatT maxcov;
    for (int e = 0; e < D * D; ++e) maxcov[e] = ScalarType(d->maximum_eigenvalue_covariance[e]);
    Kernel kern(ScalarType(d->sigma_c0), ScalarType(d->sigma_c4), d->use_weight_image != 0,
                ScalarType(d->maximum_weight), wimg, d->use_weight_tensor != 0, maxcov, wten);
    for (int64_t i = 0; i < n; ++i) {
        VecT a = vec_of(p + i * D), b = vec_of(q + i * D);
        ScalarType v;
        if (d->use_weight_image) v = kern.evaluate(a, b, kern.getSigmaAtPoint(a));
        else if (d->use_weight_tensor) v = kern.evaluate(a, b, kern.getCovarianceAtPoint(a));
        else v = kern.evaluate(a, b);
        k[i] = double(v);
    }
}

/* maxEigenValue (Mat.h:259-281) */
extern "C" double skmref_max_eigenvalue(const double *m)
{
    MatT a;
    for (int e = 0; e < D * D; ++e) a[e] = ScalarType(m[e]);
    return double(maxEigenValue(a));
}

/* UniformRng::nextI stream from the fixed seed (UniformRng.h:28-46). */
extern "C" void skmref_rng_stream(int64_t n, uint32_t *out)
{
    UniformRng rng;
    for (int64_t i = 0; i < n; ++i) out[i] = rng.nextI();
}

/* The grid shifts GpuEvaluator.cu:111-112 draws for n texels. */
extern "C" void skmref_grid_shifts(int64_t n, int subsample, int32_t *out)
{
    UniformRng rng;
    for (int64_t i = 0; i < n; ++i) {
        VecIT s = VecIT(rng.nextV<D>() * static_cast<ScalarType>(subsample));
        for (int d = 0; d < D; ++d) out[i * D + d] = s[d];
    }
}
