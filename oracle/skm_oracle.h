/*
 * skm_oracle.h -- FP64 CPU restatement of the reference SKM evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA product
 * is compared against; it is loaded by tests/, by __graft_entry__.smoke() and by
 * the CPU-baseline leg of bench.py, and by nothing else.  The product never links
 * or calls it.
 *
 * Every function follows one piece of the reference (ChristophJud/SKMImageRegistration)
 * and cites it by file:line.  Arithmetic is double throughout (the reference uses
 * a float kernel, GKernel<float>, and double elsewhere; see include/cuda/Kernel.h:209).
 * The descriptor structs are the ones of the product's C-ABI (include/skm_gpu.h)
 * so that tests feed byte-identical inputs to both.
 */
#ifndef SKM_ORACLE_H
#define SKM_ORACLE_H

#include <stdint.h>
#include "../include/skm_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_ctx ora_ctx;

/* Mirrors GpuKernelEvaluator's constructor (GpuEvaluator.cu:30-91).  Pointers in
 * desc are borrowed for the lifetime of the context. */
ora_ctx *ora_create(const skm_evaluator_desc *desc);
void     ora_destroy(ora_ctx *c);

/* SetRegularizerRKHS/RD/PG (GpuEvaluator.cu:786-831). */
void ora_set_regularizers(ora_ctx *c, double rkhs, double rd, double rd_scaling,
                          double pg, double pg_scaling);

/* getValue / getValueAndDerivative (GpuEvaluator.cu:94-357, 361-714).
 * derivatives == NULL -> value only.  Returns 0, or -1 if a sample read the fixed
 * image out of bounds (undefined behaviour in the reference). */
int ora_evaluate(ora_ctx *c, int metric, const double *cp, const double *cpw,
                 const skm_field *df, int do_resampling, double *derivatives,
                 skm_result *out);

/* evaluateDisplacementField (GpuEvaluator.cu:716-784, DisplacementField.cu:24-127). */
int ora_displacement_field(ora_ctx *c, const double *cp, const double *cpw,
                           const skm_field *df, double *dst);

/* RegularizedImageToImageMetricv4::GetValueAndDerivative
 * (itkRegularizedImageToImageMetricv4.hxx:316-573).  parameters/derivative planar. */
int ora_metric_evaluate(ora_ctx *c, const skm_metric_desc *m, const double *parameters,
                        const double *cpw, const skm_field *df, double *derivative,
                        skm_metric_values *out);

/* Adaptive-step gradient descent (itkAdaptiveStepGradientDescentOptimizerv4.hxx,
 * itkStandardGradientDescentOptimizerv4.hxx) in the ITK v4 loop.  Runs
 * `iterations` iterations from the optimizer state in *st / position (in, out),
 * writing the value of each evaluation to values[] (may be NULL). */
typedef struct ora_opt_state {
    int32_t iteration;
    double  current_time;
    double  learning_rate;
    double  scalar_product;
    double  best_value;
    double  last_value;
} ora_opt_state;
int ora_optimize(ora_ctx *c, const skm_optimizer_desc *o, const skm_metric_desc *m,
                 const double *cpw, const skm_field *df, int iterations,
                 double *position /* in/out, planar */, double *prev_neg_gradient /* in/out */,
                 double *base_position /* in/out: ITK m_PreviousGradient before the step */,
                 double *best_position /* out, may be NULL */,
                 ora_opt_state *st, double *values);

/* BsplineImage::computeCoeffs (BsplineImage.h:37-108,174-221). */
void ora_bspline_coefficients(int dimensions, const int32_t *size, const double *image,
                              double *coefficients);

/* BsplineImage::derivsGlobal + insideGlobal (BsplineImage.h:110-144,247-265,285-296)
 * at n points (D doubles each).  Returns inside flags, values and gradients. */
void ora_bspline_sample(int dimensions, const double *coefficients, const skm_geometry *g,
                        int64_t n, const double *points, int32_t *inside, double *values,
                        double *gradients);

/* GKernel::evaluate for n point pairs (Kernel.h:173-186); kind from the desc. */
void ora_kernel_values(const skm_evaluator_desc *desc, int64_t n, const double *p,
                       const double *q, double *k);

/* UniformRng (UniformRng.h:28-55) grid shifts as drawn by GpuEvaluator.cu:107-118:
 * n_texels * D ints, texel-major; *state advances. */
void ora_pcg32_shifts(uint64_t *state, int64_t n_texels, int dimensions, int subsample,
                      int32_t *shifts);
uint32_t ora_pcg32_next(uint64_t *state);

/* Shifts of the last evaluation (n_subsampled*D ints) or NULL when subsample == 1. */
const int32_t *ora_last_shifts(const ora_ctx *c);
int64_t        ora_num_subsampled(const ora_ctx *c);
void           ora_set_num_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
