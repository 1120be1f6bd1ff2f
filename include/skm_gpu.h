/*
 * skm_gpu.h -- C-ABI of the B200-native evaluation path of Sparse Kernel Machine
 * (SKM) image registration.
 *
 * The entry points replace the member functions of the reference's
 * `class GpuKernelEvaluator` (include/cuda/GpuEvaluator.h:69-179) one for one, plus
 * the host-side code that sits directly on top of it in the ITK glue
 * (regularizers L1/L2/L2,1 and the sign flip of
 * include/itkRegularizedImageToImageMetricv4.hxx:431-538, and the adaptive-step
 * optimizer of include/itkAdaptiveStepGradientDescentOptimizerv4.hxx:53-128).
 *
 * Conventions shared by every call
 *  - Plain pointers and sizes; no C++ or torch types cross this boundary.
 *  - Host buffers are borrowed for the duration of the call only (as in the
 *    reference, which copies them with cudaMemcpy on every call).
 *  - ScalarType is double (the reference default, SinglePrecisionType=0,
 *    include/CommonConfig.h:21-27).  Vector-valued images (control points,
 *    displacement fields) are arrays of structures: D doubles per texel.
 *  - Linear texel index is x-fastest: x + X*(y + Y*z) (include/cuda/ImageBase.h:40-49).
 *  - Parameters/derivatives are planar: value of axis d of control point i is at
 *    [d*C + i] (include/itkTransformAdapter.hxx:202-236).
 *  - Every call returns SKM_OK (0) or an error code; skm_last_error() returns the
 *    message of the last failure on the calling thread.  The reference instead
 *    prints and calls std::exit(-1) on CUDA errors (include/cuda/CudaUtils.h:25-31)
 *    and validates arguments in the ITK glue with itkExceptionMacro; both become
 *    return codes here.
 *  - All work runs on one CUDA stream owned by the evaluator, on the device that
 *    was current when the evaluator was created.  Calls return after the device
 *    work finished (the reference is synchronous too).
 *  - There is no CPU fallback: without a usable CUDA device every call that needs
 *    one fails with SKM_ERR_CUDA.
 */
#ifndef SKM_GPU_H
#define SKM_GPU_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SKM_ABI_VERSION 7

/* Status codes. */
#define SKM_OK              0
#define SKM_ERR_INVALID     1   /* argument rejected (reference: itkExceptionMacro) */
#define SKM_ERR_CUDA        2   /* CUDA runtime failure (reference: cudaCheck -> exit) */
#define SKM_ERR_UNSUPPORTED 3
#define SKM_ERR_NOMEM       4
#define SKM_ERR_STATE       5   /* call out of order (e.g. no evaluator) */
#define SKM_ERR_TIMEOUT     6   /* a bounded device-side wait gave up */

/* GpuKernelEvaluator::MEASURE (include/cuda/GpuEvaluator.h:160). */
#define SKM_MSE 0
#define SKM_NCC 1
#define SKM_LCC 2
/* Box-window local correlation: every texel a window centre, 5^D box window, separable window
 * sums.  No counterpart in the reference (its LCC windows are the kernel support weighted by
 * (1 - (r/s)^10)^2, include/cuda/GpuEvaluatorLCC.cu:28-35); requires subsample 1, any kernel kind,
 * runs on the generic kernels.  Value -(1/count) sum cov^2/(vf vm) over the centres whose window
 * variances exceed 1e-12 of their raw second moments; count = num_pixels_counted. */
#define SKM_LCC_BOX 3

/* ImageBase geometry (include/cuda/ImageBase.h:40-49): physical point of index i is
 * origin + spacing*i, no direction matrix.  For 2-D images entries [2] are ignored. */
typedef struct skm_geometry {
    double  origin[3];
    double  spacing[3];
    int32_t size[3];
} skm_geometry;

/* ImageNearest<VecF,D> used as the displacement field of earlier scale levels
 * (include/cuda/ImageNearest.h, GpuEvaluator.cu:120-126).  data == NULL means
 * "no field".  The device copy is cached by host pointer identity, exactly like
 * the reference (GpuEvaluator.cu:120-126): pass a different pointer to refresh it.
 * data may also be device memory of the evaluator's device (converted there, no copy to the
 * host). */
typedef struct skm_field {
    const double *data;        /* D doubles per texel, AoS (host or device memory) */
    skm_geometry  geometry;
} skm_field;

/* Constructor arguments of GpuKernelEvaluator (GpuEvaluator.h:147-154) together
 * with those of the kernel GKernel<float> (include/cuda/Kernel.h:134-146). */
typedef struct skm_evaluator_desc {
    int32_t dimensions;              /* 2 or 3 (reference: SpaceDimensions macro) */
    int32_t num_parameters;          /* C*D, C = number of control points */
    int32_t subsample;               /* fixed-grid subsampling rate, 1..100 */
    int32_t subsample_neighborhood;  /* LCC neighbourhood stride, 1..100 */

    /* kernel (Kernel.h:134-146) */
    double  sigma_c0;
    double  sigma_c4;
    int32_t use_weight_image;        /* non-stationary kernel from a sigma image */
    double  maximum_weight;          /* largest value of the weight image (or tilt) */
    const double *weight_image;      /* 1 double per texel, or NULL */
    skm_geometry  weight_image_geometry;
    int32_t use_weight_tensor;       /* anisotropic kernel from a covariance image */
    double  maximum_eigenvalue_covariance[9];  /* row-major DxD */
    const double *weight_tensor;     /* D*D doubles per texel, row-major, or NULL */
    skm_geometry  weight_tensor_geometry;

    /* moving image: cubic B-spline interpolation coefficients as produced by
     * BsplineImage::computeCoeffs (BsplineImage.h:209-221): (size+3) texels per
     * axis with a one-texel mirror offset.  moving_geometry.size is the size of
     * the image itself (the BsplineImage constructor adds the 3). */
    const double *moving_coefficients;     /* host or device memory (read in place on the device) */
    skm_geometry  moving_geometry;

    /* fixed image, 1 double per texel (host or device memory) */
    const double *fixed_image;
    skm_geometry  fixed_geometry;

    /* control-point grid and control-point weight grid (geometry only) */
    skm_geometry  cp_geometry;
    skm_geometry  cpw_geometry;
} skm_evaluator_desc;

/* GpuKernelEvaluator::EvaluationResult (GpuEvaluator.h:138-145).  Regularizer
 * values are unweighted, as in the reference. */
typedef struct skm_result {
    double   measure;
    double   reg_value_rkhs;
    double   reg_value_rd;
    double   reg_value_pg;
    uint32_t num_pixels_counted;
} skm_result;

typedef struct skm_evaluator skm_evaluator;

/* Message of the last failed call on this thread ("" if none). */
const char *skm_last_error(void);
int32_t     skm_abi_version(void);

/* Device memory (no counterpart in the reference, which calls cudaMalloc/cudaFree per buffer).
 * The library's buffers come from a stream-ordered pool of its own per device; when its last
 * buffer on a device is freed the pool keeps 2 GiB for the next evaluator or registration and
 * returns the rest to the driver.  This call returns everything the pools keep on devices where
 * none of the library's objects is alive. */
int         skm_release_memory(void);

/* GpuKernelEvaluator::GpuKernelEvaluator (GpuEvaluator.h:147-154, GpuEvaluator.cu:30-91).
 * Copies the images to device memory; all host pointers in desc are borrowed. */
int skm_evaluator_create(const skm_evaluator_desc *desc, skm_evaluator **out);
int skm_evaluator_destroy(skm_evaluator *ev);

/* Kernel path selection (no counterpart in the reference, which has one path).
 * request: -1 query only, 0 automatic (phase-table path where it applies, its two GEMMs on
 * the tensor cores where they fit), 1 generic kernels only, 2 phase-table path with its
 * GEMMs on the CUDA cores, 3 phase-table path on the tensor cores with the contrib GEMM summing
 * into per-brick control-point patches instead of the per-tap contribution array (3-D; same
 * sums in another order; slower on a B200 at 128x128x96, kept selectable).  *active (may be NULL) receives the path MSE/NCC calls take:
 * 1 generic, 2 phase table (stationary kernel, control spacing an integer multiple of
 * the fixed spacing, subsample 1), 3 phase table with tensor-core GEMMs (3xTF32, FP32
 * accuracy).  All paths compute the same sums. */
int skm_evaluator_path(skm_evaluator *ev, int32_t request, int32_t *active);

/* Work description of an evaluator (no counterpart in the reference): the kernel path and
 * the sizes that set the cost of one evaluation. */
typedef struct skm_evaluator_info {
    int32_t path;                     /* 1 generic, 2 phase table, 3 phase table on tensor cores */
    int32_t dimensions;
    int64_t fixed_texels;
    int64_t samples;                  /* fixed texels / subsample^D */
    int64_t control_points;
    int32_t table_phases;             /* texels per control-point cell (table path) */
    int32_t table_taps;               /* control points per cell in the kernel support */
    int32_t table_cells_per_axis[3];
    int64_t table_cells;
    int32_t table_regularizer_offsets;  /* control-point offsets with a nonzero kernel value */
    /* tensor-core GEMMs of the table path (zero when they do not apply): M = 128 rows of
     * (component, cell) per tile, N x K per MMA chain */
    int32_t tc_cells_per_tile;
    int32_t tc_brick[3];              /* cells per transform tile along x, y, z */
    int64_t tc_transform_tiles;
    int64_t tc_contrib_tiles;
    int32_t tc_transform_n;           /* 2 x phases padded to 16 (tf32 part and remainder of the table) */
    int32_t tc_transform_k;           /* tap pairs with a nonzero tap, 4 columns per two pairs, padded to 32 */
    int32_t tc_contrib_n;             /* taps with a nonzero table column, padded to 16 */
    int32_t tc_contrib_k;             /* phases padded to 32 */
    int32_t tc_contrib_taps;          /* taps with a nonzero table column (the contributions per cell) */
    int32_t warp_staged;              /* 1: the warp kernel stages coefficient boxes by TMA */
    int32_t tc_region_buffers;        /* transform: region buffers of the tiled-load ring */
    int32_t tc_u_staging;             /* transform: output staging buffers (0: direct stores of u) */
    int32_t tc_record_slots;          /* contrib: record ring slots (0: direct record loads) */
    int32_t tc_contrib_bricks;        /* 1: the contrib GEMM sums into per-brick control-point
                                         patches that the gather adds up (no per-tap array) */
} skm_evaluator_info;
int skm_evaluator_describe(skm_evaluator *ev, skm_evaluator_info *out);

/* Bounded-wait drill (no counterpart in the reference, whose kernels have no device-side waits).
 * Every mbarrier wait of the tensor-core kernels gives up after a bounded time, after which the
 * kernel waits (bounded) for its own copies and MMAs in flight, frees its tensor memory and
 * returns, and the call reports SKM_ERR_TIMEOUT with its results discarded.  armed != 0 makes the
 * next skm_get_value_and_derivative on this evaluator exercise that path: in the contrib GEMM,
 * the first block's first producer group withholds one shared-memory stage that nothing else
 * depends on, and the waits of that launch give up after 5 ms instead of 2 s.  The call then
 * returns SKM_ERR_TIMEOUT; the drill disarms itself and the evaluator stays usable.  Only on the
 * tensor-core table path (SKM_ERR_UNSUPPORTED otherwise); calls through skm_metric_evaluate or
 * the optimizer replay graphs captured without the drill and are unaffected. */
int skm_evaluator_wait_drill(skm_evaluator *ev, int32_t armed);

/* GpuKernelEvaluator::SetRegularizerRKHS/RD/PG (GpuEvaluator.h:156-158,
 * GpuEvaluator.cu:786-831).  weight <= 0 switches the term off. */
int skm_set_regularizer_rkhs(skm_evaluator *ev, double weight);
int skm_set_regularizer_rd  (skm_evaluator *ev, double weight, double scaling);
int skm_set_regularizer_pg  (skm_evaluator *ev, double weight, double scaling);

/* GpuKernelEvaluator::getValue (GpuEvaluator.h:162-166, GpuEvaluator.cu:94-357).
 * cp: C*D doubles (AoS), cpw: C doubles, df: previous-level field or NULL. */
int skm_get_value(skm_evaluator *ev, int32_t metric,
                  const double *cp, const double *cpw, const skm_field *df,
                  int32_t do_resampling, skm_result *out);

/* GpuKernelEvaluator::getValueAndDerivative (GpuEvaluator.h:168-173,
 * GpuEvaluator.cu:361-714).  derivatives: caller-allocated, C*D doubles, planar;
 * on return it holds the metric derivative plus the weighted RKHS/RD/PG
 * gradients, exactly what the reference writes there. */
int skm_get_value_and_derivative(skm_evaluator *ev, int32_t metric,
                                 const double *cp, const double *cpw, const skm_field *df,
                                 double *derivatives, int32_t do_resampling,
                                 skm_result *out);

/* GpuKernelEvaluator::evaluateDisplacementField (GpuEvaluator.h:175-178,
 * GpuEvaluator.cu:716-784): dst gets D doubles per fixed-image texel (dst may be device memory,
 * written in place). */
int skm_evaluate_displacement_field(skm_evaluator *ev,
                                    const double *cp, const double *cpw, const skm_field *df,
                                    double *dst);

/* ------------------------------------------------------------------------- */
/* Metric level: RegularizedImageToImageMetricv4::GetValue/GetValueAndDerivative
 * (include/itkRegularizedImageToImageMetricv4.hxx:148-213, 316-573).  Adds the
 * L1, L2,1 and L2 terms (hxx:431-526), the sign flip (hxx:528-529) and the
 * weighted sum of all terms (hxx:531-538) on the device. */
typedef struct skm_metric_desc {
    int32_t metric;            /* SKM_MSE / SKM_NCC / SKM_LCC / SKM_LCC_BOX */
    double  reg_l1;
    double  reg_l21;
    double  reg_l2;
    double  reg_rkhs;
    double  reg_rd;
    double  reg_rd_scaling;
    double  reg_pg;
    double  reg_pg_scaling;
    int32_t use_negative_gradient;   /* reference default: on (hxx:47) */
    int32_t do_resampling;           /* reference default: on (hxx:46) */
} skm_metric_desc;

/* The callback tuple of the reference metric (hxx:558-569) plus the total. */
typedef struct skm_metric_values {
    double   value;        /* measure + weighted sum of all regularizers */
    double   measure;
    double   reg_value;    /* weighted sum of all regularizers */
    double   reg_l1;
    double   reg_l21;
    double   reg_l2;
    double   reg_rkhs;
    double   reg_rd;
    double   reg_pg;
    uint32_t num_pixels_counted;
} skm_metric_values;

/* parameters/derivative: planar C*D doubles.  derivative may be NULL (value only). */
int skm_metric_evaluate(skm_evaluator *ev, const skm_metric_desc *metric,
                        const double *parameters, const double *cpw, const skm_field *df,
                        double *derivative, skm_metric_values *out);

/* ------------------------------------------------------------------------- */
/* Device-resident optimizer: AdaptiveStepGradientDescentOptimizerv4 over
 * StandardGradientDescentOptimizerv4 (include/itkAdaptiveStepGradientDescentOptimizerv4.hxx:53-128,
 * include/itkStandardGradientDescentOptimizerv4.hxx:83-166) driven by the ITK v4
 * gradient-descent loop (previous position, evaluate, step, keep best).  Parameters,
 * gradients and optimizer state stay in device memory; one iteration is one
 * metric evaluation plus one update, replayed from a CUDA graph. */
typedef struct skm_optimizer_desc {
    double  a;                  /* initial step size */
    double  A;                  /* reference: 20 (SKMReg.cxx:400) */
    double  alpha;              /* reference: 1 */
    double  f_max;              /* reference: 1e7 */
    double  f_min;              /* reference: -1e6 */
    double  omega;              /* reference: 1 */
    int32_t orthant_projection;
    int32_t number_of_iterations;
    int32_t return_best_parameters_and_value;
} skm_optimizer_desc;

typedef struct skm_optimizer_state {
    int32_t  iteration;        /* iterations done */
    double   current_time;     /* adaptive time t */
    double   learning_rate;    /* last step size */
    double   value;            /* metric value of the last evaluation */
    double   best_value;
    double   scalar_product;   /* <g, g_prev> of the last step */
    uint32_t num_pixels_counted;
} skm_optimizer_state;

typedef struct skm_optimizer skm_optimizer;

int skm_optimizer_create(skm_evaluator *ev, const skm_optimizer_desc *opt,
                         const skm_metric_desc *metric,
                         const double *initial_parameters, const double *cpw,
                         const skm_field *df, skm_optimizer **out);
/* Runs up to `iterations` more iterations (never past number_of_iterations). */
int skm_optimizer_run(skm_optimizer *o, int32_t iterations);
/* Enqueue up to `iterations` more iterations on the evaluator's stream without waiting;
 * if stream_out is not NULL it receives that cudaStream_t (for event timing). */
int skm_optimizer_enqueue(skm_optimizer *o, int32_t iterations, void *stream_out);
/* Runs up to `iterations` iterations outside the graph with CUDA events between the
 * phases; phase_ms[0..8] receives the mean milliseconds of: parameter packing, grid
 * shifts, transform (generic path: the whole value pass), warp + statistics, statistics,
 * contrib GEMM (table path), derivative gather + regularizers, result, optimizer update. */
int skm_optimizer_profile(skm_optimizer *o, int32_t iterations, double *phase_ms, int32_t nphase);
/* Number of kernel launches in one captured iteration. */
int skm_optimizer_graph_kernel_count(skm_optimizer *o, int32_t *count);
/* Current position, or the best one if best != 0 (ReturnBestParametersAndValue). */
int skm_optimizer_get_parameters(skm_optimizer *o, int32_t best, double *parameters);
int skm_optimizer_get_state(skm_optimizer *o, skm_optimizer_state *out);
int skm_optimizer_destroy(skm_optimizer *o);

/* ------------------------------------------------------------------------- */
/* BsplineImage::computeCoeffs (include/cuda/BsplineImage.h:37-108,174-221) on
 * the GPU: cubic B-spline prefilter (pole sqrt(3)-2, mirror boundaries) followed
 * by the one-texel mirror padding.  image: prod(size) doubles; coefficients:
 * prod(size+3) doubles. */
int skm_bspline_coefficients(int32_t dimensions, const int32_t *size,
                             const double *image, double *coefficients);

/* ------------------------------------------------------------------------- */
/* Preprocessing and the multi-scale driver.                                   */

/* GaussianSmoothing (include/itkUtils.h:139-150, ITK DiscreteGaussianImageFilter): discrete
 * Gaussian e^-t I_n(t) per axis, t = variance / spacing^2 when use_image_spacing, kernel grown
 * until it holds 1 - maximum_error of the mass (or half width > maximum_kernel_width), normalised,
 * edge voxels repeated.  Host buffers, x fastest.  The reference passes maximum_error 0.01 and
 * maximum_kernel_width 64. */
int skm_gaussian_smooth(int32_t dimensions, const skm_geometry *geometry, double variance,
                        int32_t use_image_spacing, double maximum_error, int32_t maximum_kernel_width,
                        const double *src, double *dst);

/* ThresholdImage + RescaleImage (include/itkUtils.h:45-110): with apply_threshold, clamp to
 * [smallest value > threshold_min, largest value < threshold_max]; then map the range linearly
 * onto [out_min, out_max].  SKM_ERR_INVALID when no value lies inside the thresholds. */
int skm_threshold_rescale(int32_t dimensions, const int32_t *size, int32_t apply_threshold,
                          double threshold_min, double threshold_max, double out_min, double out_max,
                          const double *src, double *dst);

#define SKM_MAX_SCALES 8

/* Configuration of src/SKMReg.cxx (defaults in include/ConfigUtils.h:29-62); per-scale arrays
 * hold num_scales entries (repeat the last one for "shorter lists", as CURRENT does). */
typedef struct skm_register_desc {
    int32_t dimensions;
    int32_t num_scales;
    int32_t metric;                   /* SKM_MSE / SKM_NCC / SKM_LCC / SKM_LCC_BOX */
    double  cp_spacing_scaler;        /* control spacing = min(sigma_C4, sigma_C0) / scaler (1 below 1) */
    int32_t apply_threshold;          /* intensity_thresholds given (2 entries) */
    double  threshold_min, threshold_max;
    double  sigma_c4[SKM_MAX_SCALES];
    double  sigma_c0[SKM_MAX_SCALES];
    double  smoothing_variance[SKM_MAX_SCALES];
    double  initial_step_size[SKM_MAX_SCALES];
    int32_t num_function_evaluations[SKM_MAX_SCALES];
    int32_t sampling_rate[SKM_MAX_SCALES];
    int32_t neighborhood_sampling[SKM_MAX_SCALES];
    double  reg_l1[SKM_MAX_SCALES], reg_l21[SKM_MAX_SCALES], reg_l2[SKM_MAX_SCALES];
    double  reg_rkhs[SKM_MAX_SCALES], reg_rd[SKM_MAX_SCALES], reg_rd_scaling[SKM_MAX_SCALES];
    double  reg_pg[SKM_MAX_SCALES], reg_pg_scaling[SKM_MAX_SCALES];
    /* kernel weighting (SKMReg.cxx:245-297; all images on the reference/target grid):
     * tensor_weights[s] > 0: covariance tensor of level s computed by skm_anisotropic_tensor from
     *   guidance_image (the reference's weight_tensor_filename read as an image, case 4) or, when
     *   that is NULL, from the level's smoothed target (case 3);
     * tensor_weights[s] == 0 and weight_tensor: that external tensor (case 2), N x D x D doubles;
     * weight_image (the reference's weight_filename): N doubles > 1e-8, read by the kernel before
     *   any tensor. */
    double  tensor_weights[SKM_MAX_SCALES];
    const double *guidance_image;
    const double *weight_tensor;
    const double *weight_image;
    /* restart (SKMReg's restart_at, src/SKMReg.cxx:96-123): with 1 < restart_at <= num_scales and
     * initial_displacement (N x D, the summed field after level restart_at - 1) the levels
     * restart_at..num_scales run on top of that field; otherwise every level runs from zero. */
    int32_t restart_at;
    const double *initial_displacement;
    /* optional: called after every level with the summed displacement field so far (N x D, valid
     * during the call) -- the df-full-<level> checkpoint SKMReg writes (src/SKMReg.cxx:468). */
    void (*level_done)(int32_t level, const double *displacement, void *user);
    void *level_user;
    /* learned warm start (no counterpart in the reference): planar C*D kernel weights alpha that the
     * first level run starts from instead of zeros (count must equal that level's C*D, else
     * SKM_ERR_INVALID); NULL = zeros.  With num_function_evaluations of that level 0 the weights are
     * used as they are. */
    const double *first_level_parameters;
    int64_t first_level_parameter_count;
    /* optional: called after every level with its best kernel weights (planar C*D, valid during the
     * call) -- the labels the warm-start network is trained on. */
    void (*level_parameters)(int32_t level, const double *parameters, int64_t count, void *user);
} skm_register_desc;

typedef struct skm_register_report {
    int32_t levels_done;              /* index of the last level run + 1 */
    int32_t first_level;              /* 0, or restart_at - 1 after a restart */
    int32_t iterations[SKM_MAX_SCALES];
    int64_t control_points[SKM_MAX_SCALES];
    double  best_value[SKM_MAX_SCALES];   /* metric value (+ regularizers) at the returned parameters */
    double  seconds[SKM_MAX_SCALES];
    double  optimize_seconds[SKM_MAX_SCALES];   /* of which the optimizer's iterations (the rest: set-up) */
} skm_register_report;

/* The scale loop of src/SKMReg.cxx:84-500 (skmreg): threshold + rescale, then per level
 * smoothing, B-spline prefilter, control-point grid, evaluator with the previous levels'
 * displacement field, device-resident adaptive-step optimizer, summed displacement field.
 * Reference (moving) and target (fixed) share `geometry` (the reference writes the field of the
 * target grid into a reference-sized image, GenerateDisplacementFieldGpu, itkUtils.h:181-253).
 * displacement: N x D doubles, x fastest, AoS. */
int skm_register(const skm_register_desc *desc, const skm_geometry *geometry, const double *reference,
                 const double *target, double *displacement, skm_register_report *report);

/* ComputeAnisotropicTensor (include/AnisotropicTensorUtils.h:37-371) with anisotropic_filtering
 * false, as src/SKMReg.cxx:271 and :284 call it: weight * image smoothed with variance sigma,
 * gradient outer product, each component smoothed with variance sigma / 4, eigen system ordered by
 * magnitude, main direction damped by its alignment with axis alignment_direction (0 x, 1 y,
 * 2 z; none when negative or >= dimensions), covariance U diag(s) U^T.  covariance: N x D x D
 * doubles, row-major per texel.  maximum_tilt (may be NULL): the largest damped main eigenvalue
 * over the texels whose eigenvalues all exceed 1e-8 in magnitude, -DBL_MAX when none do.
 * SKM_ERR_INVALID where a covariance is not positive definite (the reference prints and stops). */
int skm_anisotropic_tensor(int32_t dimensions, const skm_geometry *geometry, const double *image, double sigma,
                           double weight, int32_t alignment_direction, double *covariance, double *maximum_tilt);

/* Warped image: out(i) = I(p_i + u_i) on the field's grid (u: N x D doubles, AoS), I the image
 * interpolated with order 1 (multilinear, the final resampling of src/SKMReg.cxx:504-522) or
 * order 3 (cubic B-spline, WarpImage of include/itkUtils.h:163-178); default_value where the
 * continuous index leaves [-0.5, size - 0.5) on an axis. */
int skm_warp_image(int32_t dimensions, const skm_geometry *image_geometry, const double *image,
                   const skm_geometry *field_geometry, const double *field, int32_t order, double default_value,
                   double *out);

/* JacobianDeterminant (include/itkUtils.h:153-161): det(I + du/dx) per texel with central
 * differences over 2 spacing, edge texels repeated.  field: N x D doubles (AoS), out: N. */
int skm_jacobian_determinant(int32_t dimensions, const skm_geometry *geometry, const double *field, double *out);

/* ------------------------------------------------------------------------- */
/* Batched registration of many image pairs (no counterpart in the reference, which evaluates one
 * pair per GpuKernelEvaluator, include/cuda/GpuEvaluator.cu:30-91, and one call per optimizer
 * iteration, GpuEvaluator.cu:361-714, driven by the ITK v4 loop).
 *
 * Each pair has its own images, control-point grid, metric (MSE or NCC, with any of the
 * RKHS / RD / PG / L1 / L2 / L2,1 terms) and adaptive-step optimizer; pairs may differ in size.
 * One optimizer iteration of ALL pairs is one launch of one persistent kernel (captured in a CUDA
 * graph): its phases (pack, transform, warp + statistics, statistics, contribution GEMM, gather +
 * regularizers + step, result) are separated by bounded grid barriers, and the work items of each
 * phase (bricks of cells, chunks of texels, blocks of control points over all pairs) are handed out
 * by a device work queue.  The launch shape (transform brick, cells per thread along z, texels per
 * warp-phase item, blocks per SM) is chosen at creation by timing the candidates on the batch
 * itself.  Every pair must take the phase-table path (3-D, stationary kernel, control spacing an
 * integer multiple of the voxel spacing, subsample 1, no displacement field) with the same phase
 * counts (2 or 4 phases along z); SKM_ERR_UNSUPPORTED otherwise.  Results of each pair equal a
 * single-pair evaluation within FP32 rounding; sums are taken in a fixed order (deterministic). */
typedef struct skm_batch_pair {
    const skm_evaluator_desc *evaluator;  /* images and kernel of the pair (borrowed for the call) */
    skm_metric_desc    metric;
    skm_optimizer_desc optimizer;
    const double      *initial_parameters;  /* planar C*D, or NULL for zeros */
    const double      *cpw;                 /* C control-point weights, or NULL for ones */
} skm_batch_pair;

typedef struct skm_batch_info {
    int32_t pairs;
    int64_t fixed_texels;             /* sum over the pairs */
    int64_t control_points;
    int32_t grid;                     /* persistent CTAs */
    int32_t ctas_per_sm;
    int32_t transform_tile[3];        /* cells per transform brick along x, y; cells per thread along z */
    int32_t warp_chunk;               /* texels per warp-phase item */
    int32_t items[8];                 /* work items per phase over all pairs */
    int32_t shared_memory;            /* dynamic shared memory per CTA, bytes */
    double  tuned_ms;                 /* the chosen shape's time for one evaluation of the batch */
    int32_t candidates;               /* shapes the autotuner timed */
} skm_batch_info;

typedef struct skm_batch skm_batch;

int skm_batch_create(int32_t npairs, const skm_batch_pair *pairs, skm_batch **out);
int skm_batch_destroy(skm_batch *b);
/* One evaluation of every pair at its current parameters (value and derivative, no step). */
int skm_batch_evaluate(skm_batch *b);
/* `iterations` optimizer iterations of every pair (one graph launch each); run waits, enqueue does
 * not (stream_out, if not NULL, receives the batch's cudaStream_t for event timing). */
int skm_batch_run(skm_batch *b, int32_t iterations);
int skm_batch_enqueue(skm_batch *b, int32_t iterations, void *stream_out);
/* Replace a pair's position (planar C*D) and/or weights (C); NULL leaves either unchanged. */
int skm_batch_set_parameters(skm_batch *b, int32_t pair, const double *params, const double *cpw);
/* The pair's last evaluation: metric values and (negated, regularized) derivative, planar C*D. */
int skm_batch_get_result(skm_batch *b, int32_t pair, skm_metric_values *values, double *derivative);
int skm_batch_get_parameters(skm_batch *b, int32_t pair, int32_t best, double *params);
int skm_batch_get_state(skm_batch *b, int32_t pair, skm_optimizer_state *out);
int skm_batch_describe(skm_batch *b, skm_batch_info *out);

/* ------------------------------------------------------------------------- */
/* Metric value without any device allocation.  No counterpart in the reference.
 *
 * For callers that must not allocate device memory at evaluation time: frameworks that
 * own the whole device memory budget, real-time loops that cannot afford the implicit
 * device synchronisation of cudaMalloc/cudaFree, or code that plans every buffer up
 * front.  The caller passes device buffers for the inputs and for the result; the call
 * allocates nothing (no cudaMalloc, no allocating library routine) and only launches
 * kernels on `stream` (a cudaStream_t, NULL = default stream), returning without
 * waiting.  Intermediate partial sums live in one fixed array inside the library
 * (458,752 bytes, held by every device that loads the library until the process exits).
 *
 *   fixed_image          device, float, prod(fixed size) texels
 *   moving_coefficients  device, float, prod(moving size + 3) B-spline coefficients
 *   control_points       device, 4 floats per control point: alpha x, y, z (0 in 2-D), weight;
 *                        16-byte aligned (read as float4)
 *   result               device, 2 doubles: measure, number of pixels counted
 *
 * Misaligned buffers (control_points not 16-byte aligned, images not 4-byte, result not 8-byte
 * aligned) are rejected with SKM_ERR_INVALID before anything is launched.
 *
 * Same value as skm_get_value for a stationary kernel, subsample 1, no displacement
 * field, MSE or NCC.  Limit: at most 2,097,152 fixed-image texels; larger images are
 * rejected with SKM_ERR_INVALID.  Every call on a device shares the array and leaves its
 * contents behind (each call overwrites what it reads), so calls that overlap on the GPU
 * race.  The first call on each device looks up the array's device address; make that
 * first call before any stream capture.  The address is kept for the life of the process, so
 * do not call this entry point again after cudaDeviceReset (or after the device's primary
 * context was released and re-created).  Errors are reported through skm_last_error(). */
int skm_value_noalloc(int32_t dimensions, int32_t metric,
                      const skm_geometry *fixed_geometry, const float *fixed_image,
                      const skm_geometry *moving_geometry, const float *moving_coefficients,
                      const skm_geometry *cp_geometry, const float *control_points,
                      double sigma_c0, double sigma_c4, double *result, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SKM_GPU_H */
