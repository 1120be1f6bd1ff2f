/*
 * skm_gpu_evaluator.hpp -- header-only drop-in for the reference's include/cuda/GpuEvaluator.h.
 *
 * Defines `class GpuKernelEvaluator` with the constructor, member functions, nested types and
 * default arguments of the reference class (include/cuda/GpuEvaluator.h:69-179) and forwards
 * every call to the B200 C-ABI (skm_gpu.h, libskm_b200.so).  It is compiled inside the
 * reference's source tree: the boundary types it takes -- Vec, Mat, ImageNearest, BsplineImage,
 * GKernel (include/cuda/{Vec,Mat,ImageNearest,BsplineImage,Kernel}.h) and ScalarType /
 * SpaceDimensions (include/CommonConfig.h) -- are the reference's own headers, so
 * itkTransformAdapter.hxx, itkRegularizedImageToImageMetricv4.hxx and itkUtils.h compile against
 * it unchanged.  To switch, include this header where GpuEvaluator.h was included and link
 * libskm_b200.so instead of compiling GpuEvaluator.cu.
 *
 * Error behaviour follows the reference's cudaCheck (include/cuda/CudaUtils.h:25-31): the
 * message is printed and the process exits with -1.  Define SKM_SHIM_THROW to get a
 * std::runtime_error instead.
 */
#pragma once

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "CommonConfig.h"
#include "BsplineImage.h"
#include "ImageNearest.h"
#include "Kernel.h"
#include "Vec.h"
#include "Mat.h"

#include "skm_gpu.h"

namespace skm_shim {

// GKernel keeps its sigmas private and has no getters; the evaluator needs them.  Explicit
// template instantiation may name private members, which gives standard-conforming read access.
template <typename Tag, typename Tag::type M>
struct Member {
    friend typename Tag::type member_ptr(Tag) { return M; }
};
struct SigmaC0 { typedef float Kernel::*type; friend type member_ptr(SigmaC0); };
struct SigmaC4 { typedef float Kernel::*type; friend type member_ptr(SigmaC4); };
struct MaxWeight { typedef float Kernel::*type; friend type member_ptr(MaxWeight); };
struct MaxCov { typedef Mat<float, SpaceDimensions> Kernel::*type; friend type member_ptr(MaxCov); };
template struct Member<SigmaC0, &Kernel::_sigmaC0>;
template struct Member<SigmaC4, &Kernel::_sigmaC4>;
template struct Member<MaxWeight, &Kernel::_maximumWeight>;
template struct Member<MaxCov, &Kernel::_maximumEigenvalueCovariance>;

inline void check(int rc)
{
    if (rc == SKM_OK) return;
    std::string msg = std::string("skm evaluator error ") + std::to_string(rc) + ": " + skm_last_error();
#ifdef SKM_SHIM_THROW
    throw std::runtime_error(msg);
#else
    std::printf("%s\n", msg.c_str());
    std::exit(-1);
#endif
}

template <typename Image>
skm_geometry geometry(const Image &img, int pad = 0)
{
    skm_geometry g{};
    for (int d = 0; d < 3; ++d) {
        if (d < SpaceDimensions) {
            g.origin[d] = double(img.offset()[d]);
            g.spacing[d] = double(img.scale()[d]);
            g.size[d] = img.size()[d] - pad;
        } else {
            g.origin[d] = 0.0;
            g.spacing[d] = 1.0;
            g.size[d] = 1;
        }
    }
    return g;
}

template <typename T>
std::vector<double> to_double(const T *p, size_t n)
{
    std::vector<double> v(n);
    for (size_t i = 0; i < n; ++i) v[i] = double(p[i]);
    return v;
}

}  // namespace skm_shim

class GpuKernelEvaluator
{
    typedef Vec<ScalarType, SpaceDimensions> VecF;
    typedef Mat<ScalarType, SpaceDimensions> MatF;
    typedef Vec<int, SpaceDimensions> VecI;

    skm_evaluator *_ev = nullptr;
    int _numberOfParameters;
    size_t _numTexels;
    skm_geometry _fixedGeometry{};
    // double copies when ScalarType is float (the C-ABI takes double)
    std::vector<double> _cp, _cpw, _der, _df;
    const void *_dfKey = nullptr;

    skm_field field(const ImageNearest<VecF, SpaceDimensions> &df)
    {
        skm_field f{};
        f.data = nullptr;
        f.geometry = _fixedGeometry;
        if (!df.data()) return f;
        f.geometry = skm_shim::geometry(df);
        const size_t n = size_t(df.size().product()) * SpaceDimensions;
        if (sizeof(ScalarType) == sizeof(double)) {
            f.data = reinterpret_cast<const double *>(df.data());   // pointer identity kept for caching
        } else {
            if (_dfKey != df.data()) {                                 // re-convert only on a new field
                _df = skm_shim::to_double(reinterpret_cast<const ScalarType *>(df.data()), n);
                _dfKey = df.data();
            }
            f.data = _df.data();
        }
        return f;
    }

    const double *cps(const VecF *cpData)
    {
        if (sizeof(ScalarType) == sizeof(double)) return reinterpret_cast<const double *>(cpData);
        _cp = skm_shim::to_double(reinterpret_cast<const ScalarType *>(cpData), size_t(_numberOfParameters));
        return _cp.data();
    }

    const double *cpws(const ScalarType *cpwData)
    {
        if (sizeof(ScalarType) == sizeof(double)) return reinterpret_cast<const double *>(cpwData);
        _cpw = skm_shim::to_double(cpwData, size_t(_numberOfParameters / SpaceDimensions));
        return _cpw.data();
    }

public:
    struct EvaluationResult
    {
        ScalarType  measure;
        ScalarType  reg_value_rkhs;
        ScalarType  reg_value_rd;
        ScalarType  reg_value_pg;
        unsigned    numPixelsCountedGpu;
    };

    enum class MEASURE {MSE, NCC, LCC};

    GpuKernelEvaluator(int numParameters,
                       int subsample,
                       int subsampleNeighborhood,
                       Kernel kernel,
                       BsplineImage<ScalarType, SpaceDimensions> movingImage,
                       ImageNearest<ScalarType, SpaceDimensions> fixedImage,
                       ImageNearest<VecF, SpaceDimensions> cpImage,
                       ImageNearest<ScalarType, SpaceDimensions> cpwImage)
    : _numberOfParameters(numParameters),
      _numTexels(size_t(fixedImage.size().product()))
    {
        using namespace skm_shim;
        skm_evaluator_desc d{};
        d.dimensions = SpaceDimensions;
        d.num_parameters = numParameters;
        d.subsample = subsample;
        d.subsample_neighborhood = subsampleNeighborhood;
        d.sigma_c0 = double(kernel.*member_ptr(SigmaC0()));
        d.sigma_c4 = double(kernel.*member_ptr(SigmaC4()));
        d.maximum_weight = double(kernel.*member_ptr(MaxWeight()));
        const Mat<float, SpaceDimensions> mc = kernel.*member_ptr(MaxCov());
        for (int e = 0; e < SpaceDimensions * SpaceDimensions; ++e) d.maximum_eigenvalue_covariance[e] = double(mc[e]);
        std::vector<double> wimg, wten, mov, fix;
        d.use_weight_image = kernel.useWeightImage() ? 1 : 0;
        if (d.use_weight_image) {
            const auto &wi = kernel.wImage();
            wimg = to_double(wi.data(), size_t(wi.size().product()));
            d.weight_image = wimg.data();
            d.weight_image_geometry = geometry(wi);
        }
        d.use_weight_tensor = kernel.useWeightTensor() ? 1 : 0;
        if (d.use_weight_tensor) {
            const auto &wt = kernel.wTensor();
            const size_t n = size_t(wt.size().product()) * SpaceDimensions * SpaceDimensions;
            wten = to_double(reinterpret_cast<const ScalarType *>(wt.data()), n);
            d.weight_tensor = wten.data();
            d.weight_tensor_geometry = geometry(wt);
        }
        mov = to_double(movingImage.coeffs(), size_t(movingImage.size().product()));
        d.moving_coefficients = mov.data();
        d.moving_geometry = geometry(movingImage, 3);      // BsplineImage stores size+3
        fix = to_double(fixedImage.data(), _numTexels);
        d.fixed_image = fix.data();
        d.fixed_geometry = geometry(fixedImage);
        d.cp_geometry = geometry(cpImage);
        d.cpw_geometry = geometry(cpwImage);
        _fixedGeometry = d.fixed_geometry;
        check(skm_evaluator_create(&d, &_ev));
    }

    ~GpuKernelEvaluator() { skm_evaluator_destroy(_ev); }
    GpuKernelEvaluator(const GpuKernelEvaluator &) = delete;
    GpuKernelEvaluator &operator=(const GpuKernelEvaluator &) = delete;

    void SetRegularizerRKHS(ScalarType weight) { skm_shim::check(skm_set_regularizer_rkhs(_ev, double(weight))); }
    void SetRegularizerRD(ScalarType weight, ScalarType scaling = 1.0)
    {
        if (scaling <= 0.0) std::printf("Attention: scaling of regularizer must be strictly positive!\n");
        skm_shim::check(skm_set_regularizer_rd(_ev, double(weight), double(scaling)));
    }
    void SetRegularizerPG(ScalarType weight, ScalarType scaling = 1.0)
    {
        if (scaling <= 0.0) std::printf("Attention: scaling of regularizer must be strictly positive!\n");
        skm_shim::check(skm_set_regularizer_pg(_ev, double(weight), double(scaling)));
    }

    EvaluationResult getValue(MEASURE metric, const VecF *cpData, const ScalarType *cpwData,
                              ImageNearest<VecF, SpaceDimensions> displacementField, bool do_resampling = true)
    {
        skm_field f = field(displacementField);
        skm_result r{};
        skm_shim::check(skm_get_value(_ev, int32_t(metric), cps(cpData), cpws(cpwData), &f, do_resampling ? 1 : 0, &r));
        return EvaluationResult{ScalarType(r.measure), ScalarType(r.reg_value_rkhs), ScalarType(r.reg_value_rd),
                                ScalarType(r.reg_value_pg), r.num_pixels_counted};
    }

    EvaluationResult getValueAndDerivative(MEASURE metric, const VecF *cpData, const ScalarType *cpwData,
                                           ImageNearest<VecF, SpaceDimensions> displacementField,
                                           ScalarType *derivatives, bool do_resampling = true)
    {
        skm_field f = field(displacementField);
        skm_result r{};
        double *der = sizeof(ScalarType) == sizeof(double) ? reinterpret_cast<double *>(derivatives)
                                                           : (_der.resize(size_t(_numberOfParameters)), _der.data());
        skm_shim::check(skm_get_value_and_derivative(_ev, int32_t(metric), cps(cpData), cpws(cpwData), &f, der,
                                                     do_resampling ? 1 : 0, &r));
        if (sizeof(ScalarType) != sizeof(double))
            for (int i = 0; i < _numberOfParameters; ++i) derivatives[i] = ScalarType(der[i]);
        return EvaluationResult{ScalarType(r.measure), ScalarType(r.reg_value_rkhs), ScalarType(r.reg_value_rd),
                                ScalarType(r.reg_value_pg), r.num_pixels_counted};
    }

    void evaluateDisplacementField(const VecF *cpData, const ScalarType *cpwData,
                                   ImageNearest<VecF, SpaceDimensions> displacementField, VecF *dst)
    {
        skm_field f = field(displacementField);
        if (sizeof(ScalarType) == sizeof(double)) {
            skm_shim::check(skm_evaluate_displacement_field(_ev, cps(cpData), cpws(cpwData), &f,
                                                            reinterpret_cast<double *>(dst)));
        } else {
            std::vector<double> out(_numTexels * SpaceDimensions);
            skm_shim::check(skm_evaluate_displacement_field(_ev, cps(cpData), cpws(cpwData), &f, out.data()));
            ScalarType *o = reinterpret_cast<ScalarType *>(dst);
            for (size_t i = 0; i < out.size(); ++i) o[i] = ScalarType(out[i]);
        }
    }
};
