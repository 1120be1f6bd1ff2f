/*
 * ref_gpu_driver.cu -- C entry points around the reference's own CUDA evaluator
 * (include/cuda/GpuEvaluator.cu, unmodified) so that tests and the baseline
 * timing can run it on the same inputs as the product.
 *
 * TEST INFRASTRUCTURE ONLY.  oracle/Makefile compiles it with nvcc for sm_100a with
 * the reference's own flags (-use_fast_math, include/cuda/CMakeLists.txt:34-35) into
 * oracle/_ref/libskmref_gpu_<d|f><2|3>.so.  The one C++11 narrowing error of the
 * reference (GpuEvaluator.cu:356,713, int -> unsigned in a braced initialiser) is
 * downgraded with nvcc's -diag-suppress instead of patching the source.
 *
 * Safety: with subsample > 1 the reference can read the fixed image out of bounds
 * when a PCG32 draw equals UINT_MAX (UniformRng.h:43-46 gives shift == subsample).
 * The driver keeps a shadow copy of the generator and refuses a call whose draws
 * would contain such a value, so the reference never runs on such an input.
 */
#include "GpuEvaluator.cu"

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <vector>

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

struct RefHandle {
    std::vector<ScalarType> moving, fixed, wimg, cp, cpw, deriv, dfdata;
    std::vector<MatT> wten;
    std::unique_ptr<GpuKernelEvaluator> ev;
    UniformRng shadow;
    bool evaluated_once = false;
    int subsample = 1;
    int64_t nss = 0;
    int num_params = 0;
    const double *df_key = nullptr;
};

/* true if the next draws of the shadow generator are safe; advances it like the
 * reference does (GpuEvaluator.cu:107-115). */
bool advance_shadow(RefHandle *h, bool resample)
{
    if (h->subsample <= 1) return true;
    if (h->evaluated_once && !resample) return true;
    UniformRng probe = h->shadow;
    for (int64_t i = 0; i < h->nss * D; ++i)
        if (probe.nextI() == 0xFFFFFFFFu) return false;
    h->shadow = probe;
    h->evaluated_once = true;
    return true;
}

ImageNearest<VecT, D> field_of(RefHandle *h, const skm_field *df)
{
    if (!df || !df->data) return ImageNearest<VecT, D>();
    VecIT sz = veci_of(df->geometry.size);
    if (df->data != h->df_key) {          /* keep a stable converted copy per caller pointer */
        h->df_key = df->data;
        h->dfdata.assign(df->data, df->data + (size_t)sz.product() * D);
    }
    return ImageNearest<VecT, D>(reinterpret_cast<const VecT *>(h->dfdata.data()),
                                 vec_of(df->geometry.origin), vec_of(df->geometry.spacing), sz);
}

void load_params(RefHandle *h, const double *cp, const double *cpw)
{
    size_t C = (size_t)h->num_params / D;
    h->cp.assign(cp, cp + C * D);
    h->cpw.assign(cpw, cpw + C);
}
}  // namespace

extern "C" int skmref_dimensions() { return D; }
extern "C" int skmref_scalar_bytes() { return (int)sizeof(ScalarType); }

extern "C" int skmref_create(const skm_evaluator_desc *d, void **out)
{
    if (d->dimensions != D) return 1;
    RefHandle *h = new RefHandle();
    h->subsample = d->subsample;
    h->num_params = d->num_parameters;
    VecIT msz = veci_of(d->moving_geometry.size);
    h->moving.assign(d->moving_coefficients, d->moving_coefficients + (msz + 3).product());
    VecIT fsz = veci_of(d->fixed_geometry.size);
    h->fixed.assign(d->fixed_image, d->fixed_image + fsz.product());
    h->nss = (fsz / d->subsample).product();

    ImageNearest<ScalarType, D> wimg;
    ImageNearest<MatT, D> wten;
    if (d->use_weight_image) {
        VecIT sz = veci_of(d->weight_image_geometry.size);
        h->wimg.assign(d->weight_image, d->weight_image + sz.product());
        wimg = ImageNearest<ScalarType, D>(h->wimg.data(), vec_of(d->weight_image_geometry.origin),
                                           vec_of(d->weight_image_geometry.spacing), sz);
    } else {
        h->wimg.assign(1, ScalarType(0));
        wimg = ImageNearest<ScalarType, D>(h->wimg.data(), VecT(0.0), VecT(1.0), VecIT(1));
    }
    if (d->use_weight_tensor) {
        VecIT sz = veci_of(d->weight_tensor_geometry.size);
        h->wten.resize(sz.product());
        for (int i = 0; i < sz.product(); ++i)
            for (int e = 0; e < D * D; ++e) h->wten[i][e] = ScalarType(d->weight_tensor[(size_t)i * D * D + e]);
        wten = ImageNearest<MatT, D>(h->wten.data(), vec_of(d->weight_tensor_geometry.origin),
                                     vec_of(d->weight_tensor_geometry.spacing), sz);
    } else {
        h->wten.assign(1, MatT::identity());
        wten = ImageNearest<MatT, D>(h->wten.data(), VecT(0.0), VecT(1.0), VecIT(1));
    }
    MatT maxcov;
    for (int e = 0; e < D * D; ++e) maxcov[e] = ScalarType(d->maximum_eigenvalue_covariance[e]);
    Kernel kern(ScalarType(d->sigma_c0), ScalarType(d->sigma_c4), d->use_weight_image != 0,
                ScalarType(d->maximum_weight), wimg, d->use_weight_tensor != 0, maxcov, wten);

    BsplineImage<ScalarType, D> moving(h->moving.data(), vec_of(d->moving_geometry.origin),
                                       vec_of(d->moving_geometry.spacing), msz);
    ImageNearest<ScalarType, D> fixed(h->fixed.data(), vec_of(d->fixed_geometry.origin),
                                      vec_of(d->fixed_geometry.spacing), fsz);
    ImageNearest<VecT, D> cpimg(nullptr, vec_of(d->cp_geometry.origin), vec_of(d->cp_geometry.spacing),
                                veci_of(d->cp_geometry.size));
    ImageNearest<ScalarType, D> cpwimg(nullptr, vec_of(d->cpw_geometry.origin),
                                       vec_of(d->cpw_geometry.spacing), veci_of(d->cpw_geometry.size));
    h->ev.reset(new GpuKernelEvaluator(d->num_parameters, d->subsample, d->subsample_neighborhood, kern,
                                       moving, fixed, cpimg, cpwimg));
    *out = h;
    return 0;
}

extern "C" void skmref_destroy(void *p) { delete static_cast<RefHandle *>(p); }

extern "C" void skmref_set_regularizers(void *p, double rkhs, double rd, double rd_scaling, double pg,
                                        double pg_scaling)
{
    RefHandle *h = static_cast<RefHandle *>(p);
    h->ev->SetRegularizerRKHS(ScalarType(rkhs));
    h->ev->SetRegularizerRD(ScalarType(rd), ScalarType(rd_scaling));
    h->ev->SetRegularizerPG(ScalarType(pg), ScalarType(pg_scaling));
}

static GpuKernelEvaluator::MEASURE measure_of(int m)
{
    return m == SKM_NCC ? GpuKernelEvaluator::MEASURE::NCC
                        : (m == SKM_LCC ? GpuKernelEvaluator::MEASURE::LCC : GpuKernelEvaluator::MEASURE::MSE);
}

/* getValue / getValueAndDerivative; derivatives == NULL -> getValue.
 * Returns 2 (and runs nothing) if the draws would make the reference read out of bounds. */
extern "C" int skmref_evaluate(void *p, int metric, const double *cp, const double *cpw, const skm_field *df,
                               int do_resampling, double *derivatives, skm_result *out)
{
    RefHandle *h = static_cast<RefHandle *>(p);
    if (!advance_shadow(h, do_resampling != 0)) return 2;
    load_params(h, cp, cpw);
    ImageNearest<VecT, D> field = field_of(h, df);
    GpuKernelEvaluator::EvaluationResult r;
    if (derivatives) {
        h->deriv.assign(h->num_params, ScalarType(0));
        r = h->ev->getValueAndDerivative(measure_of(metric), reinterpret_cast<const VecT *>(h->cp.data()),
                                         h->cpw.data(), field, h->deriv.data(), do_resampling != 0);
        for (int i = 0; i < h->num_params; ++i) derivatives[i] = double(h->deriv[i]);
    } else {
        r = h->ev->getValue(measure_of(metric), reinterpret_cast<const VecT *>(h->cp.data()), h->cpw.data(), field,
                            do_resampling != 0);
    }
    out->measure = double(r.measure);
    out->reg_value_rkhs = double(r.reg_value_rkhs);
    out->reg_value_rd = double(r.reg_value_rd);
    out->reg_value_pg = double(r.reg_value_pg);
    out->num_pixels_counted = r.numPixelsCountedGpu;
    return 0;
}

extern "C" int skmref_displacement_field(void *p, const double *cp, const double *cpw, const skm_field *df,
                                         double *dst, int64_t n_texels)
{
    RefHandle *h = static_cast<RefHandle *>(p);
    load_params(h, cp, cpw);
    ImageNearest<VecT, D> field = field_of(h, df);
    std::vector<VecT> out((size_t)n_texels);
    h->ev->evaluateDisplacementField(reinterpret_cast<const VecT *>(h->cp.data()), h->cpw.data(), field, out.data());
    for (int64_t i = 0; i < n_texels; ++i)
        for (int d = 0; d < D; ++d) dst[i * D + d] = double(out[i][d]);
    return 0;
}
