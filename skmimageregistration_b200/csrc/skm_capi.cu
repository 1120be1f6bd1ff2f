// skm_capi.cu -- the evaluator object behind the C-ABI of include/skm_gpu.h.
//
// One evaluator owns every device buffer it needs (allocated once at creation, like
// GpuKernelEvaluator's constructor, GpuEvaluator.cu:30-91), one CUDA stream and pinned
// host staging buffers.  A call uploads the parameters, runs the launch sequence
//   [pack] -> [grid shifts] -> value pass -> statistics -> derivative+regularizers -> result
// on the stream and copies the scalars and the derivative back.  Every reduction is
// done on the device in a fixed order; no host loops over per-voxel arrays remain.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/skm_gpu.h"
#include "skm_device.cuh"
#include "skm_kernels.cuh"
#include "skm_lccbox.cuh"
#include "skm_prefilter.cuh"
#include "skm_table.cuh"
#include "skm_table_tc.cuh"

using namespace skm;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define SKM_CUDA(call)                                                                                 \
    do {                                                                                               \
        cudaError_t e_ = (call);                                                                       \
        if (e_ != cudaSuccess) return fail(SKM_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #call,    \
                                           cudaGetErrorString(e_));                                    \
    } while (0)

#define SKM_CHECK_LAUNCH() SKM_CUDA(cudaPeekAtLastError())

template <typename T>
int dalloc(T **p, size_t n)
{
    *p = nullptr;
    if (n == 0) n = 1;
    SKM_CUDA(pool_malloc((void **)p, n * sizeof(T)));
    return SKM_OK;
}

// a caller's pointer that is device memory (cudaMalloc, a memory pool, managed memory)
bool device_memory(const void *p)
{
    cudaPointerAttributes a{};
    if (!p || cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// doubles on the device: the caller's device memory as it is, or a host array copied into a
// buffer from the pool (released with this object, after the caller synchronised its stream)
struct StagedDoubles {
    const double *p = nullptr;
    double *own = nullptr;
    int stage(const double *src, long long n, cudaStream_t s)
    {
        if (device_memory(src)) {
            p = src;
            return SKM_OK;
        }
        if (dalloc(&own, n)) return SKM_ERR_CUDA;
        SKM_CUDA(cudaMemcpyAsync(own, src, n * sizeof(double), cudaMemcpyHostToDevice, s));
        p = own;
        return SKM_OK;
    }
    ~StagedDoubles()
    {
        if (own) pool_release(own);
    }
};

int grid_for(long long n) { return (int)std::max<long long>(1, std::min<long long>((n + 255) / 256, 148 * 16)); }

Geo make_geo(const skm_geometry &g, int D, int pad)
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

long long texels(const skm_geometry &g, int D)
{
    long long n = 1;
    for (int d = 0; d < D; ++d) n *= g.size[d];
    return n;
}

bool geometry_ok(const skm_geometry &g, int D)
{
    for (int d = 0; d < D; ++d)
        if (g.size[d] < 1 || !(g.spacing[d] > 0.0)) return false;
    return true;
}

void rng_jump_table(RngJump &J)
{
    unsigned long long m = 6364136223846793005ULL, a = 1ULL;   // PCG32 multiplier, increment (seq|1)
    for (int i = 0; i < 64; ++i) {
        J.mul[i] = m;
        J.add[i] = a;
        a = a * (m + 1ULL);
        m = m * m;
    }
}

unsigned long long rng_advance_host(unsigned long long s, unsigned long long steps, const RngJump &J)
{
    int i = 0;
    while (steps) {
        if (steps & 1ULL) s = s * J.mul[i] + J.add[i];
        steps >>= 1;
        ++i;
    }
    return s;
}

// maxEigenValue (Mat.h:259-281) with Type = float, evaluated as written (no multiply-add
// contraction on this host).  getRegionSupport(covP) (Kernel.h:168-171) adds the double tensor to
// the float member _maximumEigenvalueCovariance through Mat<float>::operator+ (Mat.h:108), so the
// sum, the eigenvalue, the division and the square root are all float.
float max_eig_f(const float *m, int D)
{
    if (D == 2) {
        float trace = m[0] + m[3];
        float det = m[0] * m[3] - m[2] * m[1];
        float disc = trace * trace - 4.0f * det;
        return 0.5f * (trace + std::sqrt(disc > 0.0f ? disc : 0.0f));
    }
    float triSq = m[1] * m[1] + m[2] * m[2] + m[5] * m[5];
    if (triSq == 0.0f) return std::max(m[0], std::max(m[4], m[8]));
    float q = (float)(1.0 / 3.0) * (m[0] + m[4] + m[8]);
    float pSq = 2.0f * triSq + (m[0] - q) * (m[0] - q) + (m[4] - q) * (m[4] - q) + (m[8] - q) * (m[8] - q);
    float p = std::sqrt(pSq * (float)(1.0 / 6.0));
    float b0 = m[0] - q, b4 = m[4] - q, b8 = m[8] - q;
    float det = b0 * b4 * b8 + m[3] * m[7] * m[2] + m[6] * m[1] * m[5] - b0 * m[7] * m[5] - m[6] * b4 * m[2] -
                m[3] * m[1] * b8;
    float r = det * (0.5f / (p * p * p));
    float phi = (float)(1.0 / 3.0) * std::acos(std::min(1.0f, std::max(-1.0f, r)));
    return q + 2.0f * p * std::cos(phi);
}

float tensor_support(const KernelParams &K, const double *cov, int D)
{
    float s[9];
    for (int e = 0; e < D * D; ++e) s[e] = K.maxcov[e] + (float)cov[e];
    return K.support_min / std::sqrt(2.0f / max_eig_f(s, D));
}

// Support radius per texel of the weight image (double: the float member _maximumWeight plus the
// double sigma, Kernel.h:163-166) or of the weight tensors (float, above), and the radius where
// the lookup falls outside the image (sigma 0 / identity covariance).  Radii decide the windows
// and boxes by truncation; with voxel-commensurate sigmas they sit on integer boundaries, so they
// are computed once here, exactly as the reference's expressions round them.
void support_table(const KernelParams &K, int D, const double *src, long long n, double *out, double *dflt)
{
    const bool tensor = K.kind == kWeightTensor;
    if (tensor) {
        double eye[9] = {0};
        for (int d = 0; d < D; ++d) eye[d * D + d] = 1.0;
        *dflt = (double)tensor_support(K, eye, D);
    } else {
        *dflt = (double)K.support_min / std::sqrt(2.0 / ((double)K.maxw + 0.0));
    }
    auto work = [&](long long b, long long e) {
        for (long long i = b; i < e; ++i)
            out[i] = tensor ? (double)tensor_support(K, src + i * D * D, D)
                            : (double)K.support_min / std::sqrt(2.0 / ((double)K.maxw + src[i]));
    };
    unsigned nt = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    if (n < (1LL << 16)) nt = 1;
    std::vector<std::thread> th;
    long long chunk = (n + nt - 1) / nt;
    for (unsigned t = 1; t < nt; ++t)
        th.emplace_back(work, std::min(n, t * chunk), std::min(n, (t + 1) * chunk));
    work(0, std::min(n, chunk));
    for (auto &x : th) x.join();
}

constexpr int kValueThreads = 256;
constexpr int kDerivThreads = 256;     // 8 warps = 8 control points per block
constexpr int kSplitBelowBlocks = 1024; // fewer derivative blocks than this: one block per control point
constexpr unsigned long long kDrillWaitNs = 5000000ull;   // bounded-wait limit during the wait drill: 5 ms

}  // namespace

struct skm_evaluator {
    int device = 0;
    int D = 3;
    cudaStream_t stream = nullptr;
    EvalParams P{};
    skm_geometry fixed_geo{}, cp_geo{};
    int nparams = 0;
    long long N = 0, Ns = 0, C = 0;
    int value_blocks = 0, deriv_blocks = 0, dense_blocks = 0, gather_blocks = 0;

    // device memory
    float *d_fixed = nullptr, *d_coeffs = nullptr, *d_wimg = nullptr, *d_wten = nullptr;
    double *d_wsup = nullptr;         // support radius per weight-image / weight-tensor texel
    float4 *d_coeffs4 = nullptr;
    float4 *d_cpd = nullptr, *d_df = nullptr, *d_samp = nullptr, *d_dense = nullptr, *d_dense_sw = nullptr;
    unsigned char *d_dense_in = nullptr, *d_dense_sw_in = nullptr;
    unsigned *d_need = nullptr;       // LCC: bit per texel that a window reads
    int *d_list = nullptr, *d_nlist = nullptr;   // LCC: those texels, listed once, and their count
    float4 *d_acache = nullptr;       // LCC 3-D weight tensors: per-texel kernel inverse and factor
    unsigned char *d_box_in = nullptr;   // box-window LCC: texel warped inside the moving image
    double *d_box_a = nullptr, *d_box_b = nullptr;   // box-window LCC: 6 planar FP64 fields each
    float *d_box_coef = nullptr;         // box-window LCC: derivative coefficient per texel
    uint32_t *d_shifts = nullptr;
    double *d_in = nullptr;          // uploaded parameters (AoS or planar) followed by weights
    unsigned *d_counters = nullptr;   // ticket counters of the fused last-block finalizations
    double *d_part = nullptr, *d_stats = nullptr, *d_deriv = nullptr, *d_rpart = nullptr, *d_out = nullptr;
    long long df_texels = 0;

    // pinned host staging
    double *h_in = nullptr, *h_out = nullptr;
    double *dh_in = nullptr, *dh_out = nullptr;   // the same staging buffers as the device addresses them
    bool weights_uploaded = false;       // h_in's weight part is on the device (skip identical weights)

    // phase-table fast path (stationary kernel, integral spacing ratio) and its tensor-core GEMMs
    TablePlan table{};
    TcPlan tc{};
    bool use_tc = true;

    // state of GpuKernelEvaluator
    double reg_rkhs = 0, reg_rd = 0, rd_scaling = 1, reg_pg = 0, pg_scaling = 1;
    unsigned long long rng_state = 0xBA5EBA11DEADBEEFULL;
    bool evaluated_once = false;
    const double *df_key = nullptr;
    RngJump jump{};
    bool use_table = true;

    // skm_metric_evaluate replays one CUDA graph (parameter upload, evaluation, result download)
    // while the metric description, the derivative request, the path and the field stay the same
    // (a few graphs, least recently used replaced: a caller may alternate derivative buffers)
    struct MetricGraph {
        cudaGraphExec_t exec = nullptr;
        skm_metric_desc desc{};
        bool deriv = false;
        int path = 0;
        const double *df = nullptr;
        const double *pdev = nullptr;  // parameter source and derivative destination the graph uses
        double *gout = nullptr;
        unsigned long long used = 0;
    };
    static constexpr int kMetricGraphs = 4;
    MetricGraph mg[kMetricGraphs];
    unsigned long long mg_clock = 0;
    void clear_metric_graphs()
    {
        for (MetricGraph &g : mg) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g = MetricGraph{};
        }
    }

    // armed by skm_evaluator_wait_drill: the next skm_get_value(_and_derivative) runs the drill
    bool drill_armed = false;

    ~skm_evaluator()
    {
        if (device >= 0) cudaSetDevice(device);
        // one device synchronisation for all buffers (no work uses them after it), then the frees
        cudaDeviceSynchronize();
        void *bufs[] = {d_fixed, d_coeffs, d_coeffs4, d_wimg, d_wten, d_wsup, d_cpd, d_df, d_samp, d_dense, d_dense_sw,
                        d_dense_in, d_need, d_list, d_nlist, d_acache, d_dense_sw_in, d_shifts, d_in, d_counters, d_part,
                        d_stats, d_deriv, d_rpart, d_out, d_box_in, d_box_a, d_box_b, d_box_coef};
        for (void *b : bufs)
            if (b) pool_release(b);
        clear_metric_graphs();
        table_tc_free(tc);
        table_free(table);
        cudaStreamSynchronize(0);
        if (h_in) cudaFreeHost(h_in);
        if (h_out) cudaFreeHost(h_out);
        if (stream) cudaStreamDestroy(stream);
    }
};

// 1 generic kernels, 2 phase table with CUDA-core GEMMs, 3 phase table with tensor-core GEMMs
static int active_path(const skm_evaluator *e)
{
    if (!(e->use_table && e->table.enabled)) return 1;
    return (e->use_tc && e->tc.enabled) ? 3 : 2;
}

// tensor-core GEMMs of the table path, when they apply and are selected
static const TcPlan *tc_of(const skm_evaluator *e)
{
    return (e->use_tc && e->tc.enabled) ? &e->tc : nullptr;
}

// the tensor-core transform's weighted control-point planes, written by every packing kernel
// whenever the plan has them (whichever path the next evaluation takes)
static RegionPlanes planes_of(const skm_evaluator *e)
{
    return e->tc.enabled ? e->tc.rp : RegionPlanes{};
}

// ------------------------------------------------------------------------------------------------
// dispatch over dimension and kernel kind
template <template <int, int> class F, typename... A>
static int dispatch(int D, int kind, A &&...a)
{
    if (D == 3) {
        if (kind == kStationary) return F<3, kStationary>::run(a...);
        if (kind == kWeightImage) return F<3, kWeightImage>::run(a...);
        return F<3, kWeightTensor>::run(a...);
    }
    if (kind == kStationary) return F<2, kStationary>::run(a...);
    if (kind == kWeightImage) return F<2, kWeightImage>::run(a...);
    return F<2, kWeightTensor>::run(a...);
}

template <int D, int KIND>
struct LaunchValue {
    static int run(skm_evaluator *e)
    {
        value_kernel<D, KIND><<<e->value_blocks, kValueThreads, 0, e->stream>>>(e->P, e->d_samp, e->d_part);
        SKM_CHECK_LAUNCH();
        return SKM_OK;
    }
};

template <int D, int KIND>
struct LaunchLccValue {
    static int run(skm_evaluator *e)
    {
        // the texels the windows read (listed once each), then the dense fields there only
        SKM_CUDA(cudaMemsetAsync(e->d_need, 0, sizeof(unsigned) * ((e->N + 31) / 32), e->stream));
        SKM_CUDA(cudaMemsetAsync(e->d_nlist, 0, sizeof(int), e->stream));
        lcc_mark_kernel<D, KIND><<<e->value_blocks, 256, 0, e->stream>>>(e->P, e->d_need, e->d_list, e->d_nlist);
        SKM_CHECK_LAUNCH();
        const int lb = grid_for(e->N);
        dense_list_kernel<D, KIND, false><<<lb, 256, 0, e->stream>>>(e->P, e->d_list, e->d_nlist, e->d_dense,
                                                                     e->d_dense_in);
        SKM_CHECK_LAUNCH();
        if (D == 3 && KIND != kStationary) {
            dense_list_kernel<D, KIND, true><<<lb, 256, 0, e->stream>>>(e->P, e->d_list, e->d_nlist, e->d_dense_sw,
                                                                        e->d_dense_sw_in, e->d_acache);
            SKM_CHECK_LAUNCH();
        }
        lcc_value_kernel<D, KIND><<<e->value_blocks, kValueThreads, 0, e->stream>>>(e->P, e->d_dense, e->d_dense_in,
                                                                                      e->d_part);
        SKM_CHECK_LAUNCH();
        return SKM_OK;
    }
};

// box-window LCC value pass: per-texel samples, window moments (x, y[, z] passes), centres (value
// partials and A, B, E), their box sums (x, y[, z]) and the texel coefficients.  Buffers alternate:
// a pass reads one of d_box_a / d_box_b and writes the other.
template <int D, int KIND>
struct LaunchBoxValue {
    static int run(skm_evaluator *e)
    {
        const long long N = e->N;
        const int nx = e->P.fixed.n[0], ny = e->P.fixed.n[1], nz = D > 2 ? e->P.fixed.n[2] : 1;
        const int lb = grid_for(N);
        cudaStream_t s = e->stream;
        double *a = e->d_box_a, *b = e->d_box_b;
        box_texel_kernel<D, KIND><<<lb, 256, 0, s>>>(e->P, e->d_samp, e->d_box_in);
        box_moments_x_kernel<<<lb, 256, 0, s>>>(e->d_fixed, e->d_samp, e->d_box_in, N, nx, a);
        box_axis_kernel<kBoxMoments><<<lb, 256, 0, s>>>(a, b, N, nx, ny);
        if (D > 2) {
            box_axis_kernel<kBoxMoments><<<lb, 256, 0, s>>>(b, a, N, (long long)nx * ny, nz);
            std::swap(a, b);
        }
        // final moments in b; the centres' A, B, E into a
        box_centers_kernel<<<e->value_blocks, kValueThreads, 0, s>>>(b, e->d_box_in, N, a, e->d_part);
        box_axis_kernel<3><<<lb, 256, 0, s>>>(a, b, N, 1, nx);
        box_axis_kernel<3><<<lb, 256, 0, s>>>(b, a, N, nx, ny);
        if (D > 2) {
            box_axis_kernel<3><<<lb, 256, 0, s>>>(a, b, N, (long long)nx * ny, nz);
            std::swap(a, b);
        }
        box_coef_kernel<<<lb, 256, 0, s>>>(a, e->d_fixed, e->d_samp, e->d_box_in, N, e->d_box_coef);
        SKM_CHECK_LAUNCH();
        return SKM_OK;
    }
};

template <int D, int KIND>
struct LaunchDeriv {
    static int run(skm_evaluator *e, DerivParams Q, bool split)
    {
        if (split)
            derivative_kernel<D, KIND, 8><<<(int)e->C, kDerivThreads, 0, e->stream>>>(e->P, Q);
        else
            derivative_kernel<D, KIND, 1><<<e->deriv_blocks, kDerivThreads, 0, e->stream>>>(e->P, Q);
        SKM_CHECK_LAUNCH();
        return SKM_OK;
    }
};

template <int D, int KIND>
struct LaunchRegValue {
    static int run(skm_evaluator *e, DerivParams Q)
    {
        regvalue_kernel<D, KIND><<<e->deriv_blocks, kDerivThreads, 0, e->stream>>>(e->P, Q);
        SKM_CHECK_LAUNCH();
        return SKM_OK;
    }
};

template <int D, int KIND>
struct LaunchDisp {
    static int run(skm_evaluator *e, double *out)
    {
        displacement_kernel<D, KIND><<<e->dense_blocks, 256, 0, e->stream>>>(e->P, out);
        SKM_CHECK_LAUNCH();
        return SKM_OK;
    }
};

// ------------------------------------------------------------------------------------------------
extern "C" const char *skm_last_error(void) { return g_last_error.c_str(); }

// lets other translation units of the library report through skm_last_error()
void skm_internal_set_error(const char *msg) { g_last_error = msg; }
extern "C" int32_t skm_abi_version(void) { return SKM_ABI_VERSION; }

extern "C" int skm_release_memory(void)
{
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SKM_OK;                               // no device: the library holds nothing
    }
    SKM_CUDA(pool_release_all());
    return SKM_OK;
}

static int validate_desc(const skm_evaluator_desc *d)
{
    if (!d) return fail(SKM_ERR_INVALID, "descriptor is NULL");
    int D = d->dimensions;
    if (D != 2 && D != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3 (got %d)", D);
    if (d->subsample < 1 || d->subsample > 100)          // metric hxx:87-89
        return fail(SKM_ERR_INVALID, "subsample must be in [1,100] (got %d)", d->subsample);
    if (d->subsample_neighborhood < 1 || d->subsample_neighborhood > 100)   // hxx:91-93
        return fail(SKM_ERR_INVALID, "subsample_neighborhood must be in [1,100] (got %d)",
                    d->subsample_neighborhood);
    if (!(d->sigma_c0 > 0.0) || !(d->sigma_c4 > 0.0))    // itkTransformAdapter.hxx:412-414
        return fail(SKM_ERR_INVALID, "kernel parameters have to be positive");
    if (!d->fixed_image || !d->moving_coefficients) return fail(SKM_ERR_INVALID, "image data is NULL");
    if (!geometry_ok(d->fixed_geometry, D) || !geometry_ok(d->moving_geometry, D) ||
        !geometry_ok(d->cp_geometry, D) || !geometry_ok(d->cpw_geometry, D))
        return fail(SKM_ERR_INVALID, "invalid geometry (size < 1 or spacing <= 0)");
    for (int k = 0; k < D; ++k) {
        if (d->moving_geometry.size[k] < 2)   // the prefilter's anti-causal start reads c[len-2]
            return fail(SKM_ERR_INVALID, "moving image must have at least 2 texels per axis");
        if (d->cpw_geometry.size[k] != d->cp_geometry.size[k])
            return fail(SKM_ERR_INVALID, "control-point weight grid must match the control-point grid");
        if (d->fixed_geometry.size[k] / d->subsample < 1)
            return fail(SKM_ERR_INVALID, "subsample larger than the fixed image");
    }
    long long C = texels(d->cp_geometry, D);
    if ((long long)d->num_parameters != C * D)
        return fail(SKM_ERR_INVALID, "num_parameters (%d) != control points (%lld) * D", d->num_parameters, C);
    if (d->use_weight_image && d->use_weight_tensor)
        return fail(SKM_ERR_INVALID, "weight image and weight tensor are exclusive");
    if (d->use_weight_image) {
        if (!d->weight_image || !geometry_ok(d->weight_image_geometry, D))
            return fail(SKM_ERR_INVALID, "weight image missing");
        long long n = texels(d->weight_image_geometry, D);
        for (long long i = 0; i < n; ++i)
            if (!(d->weight_image[i] > 1e-8))          // itkTransformAdapter.hxx:325-327
                return fail(SKM_ERR_INVALID, "weighting image has to be strictly positive everywhere");
    }
    if (d->use_weight_tensor) {
        if (!d->weight_tensor || !geometry_ok(d->weight_tensor_geometry, D))
            return fail(SKM_ERR_INVALID, "weight tensor missing");
        long long n = texels(d->weight_tensor_geometry, D);
        for (long long i = 0; i < n; ++i) {            // itkTransformAdapter.hxx:346-350
            const double *m = d->weight_tensor + i * D * D;
            double det = D == 2 ? m[0] * m[3] - m[1] * m[2]
                                : m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                                      m[2] * (m[3] * m[7] - m[4] * m[6]);
            if (!(det > 0.0)) return fail(SKM_ERR_INVALID, "weighting tensors must be positive definite");
        }
    }
    return SKM_OK;
}

extern "C" int skm_evaluator_create(const skm_evaluator_desc *d, skm_evaluator **out)
{
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int rc = validate_desc(d);
    if (rc) return rc;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SKM_ERR_CUDA, "no CUDA device available (this library has no CPU fallback)");
    }
    skm_evaluator *e = new skm_evaluator();
    int D = d->dimensions;
    e->D = D;
    if (cudaGetDevice(&e->device) != cudaSuccess) {
        delete e;
        return fail(SKM_ERR_CUDA, "cudaGetDevice failed");
    }
    rc = [&]() -> int {
        SKM_CUDA(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
        e->fixed_geo = d->fixed_geometry;
        e->cp_geo = d->cp_geometry;
        e->nparams = d->num_parameters;
        e->N = texels(d->fixed_geometry, D);
        e->C = texels(d->cp_geometry, D);
        EvalParams &P = e->P;
        P.sub = d->subsample;
        P.nbh = d->subsample_neighborhood;
        P.fixed = make_geo(d->fixed_geometry, D, 0);
        P.mov = make_geo(d->moving_geometry, D, 3);
        P.cp = make_geo(d->cp_geometry, D, 0);
        P.df = make_geo(d->fixed_geometry, D, 0);
        P.has_df = 0;
        long long ns = 1;
        for (int k = 0; k < 3; ++k) {
            P.ss[k] = k < D ? d->fixed_geometry.size[k] / d->subsample : 1;
            ns *= P.ss[k];
        }
        P.Ns = e->Ns = ns;
        P.C = e->C;
        e->value_blocks = (int)((ns + kValueThreads - 1) / kValueThreads);
        e->deriv_blocks = (int)((e->C + (kDerivThreads / 32) - 1) / (kDerivThreads / 32));
        e->dense_blocks = (int)((e->N + 255) / 256);
        e->gather_blocks = (int)((e->C + 31) / 32);

        // kernel parameters: GKernel<float> members are floats (Kernel.h:216-221)
        KernelParams &K = P.K;
        K.kind = d->use_weight_image ? kWeightImage : (d->use_weight_tensor ? kWeightTensor : kStationary);
        K.sc0 = (float)d->sigma_c0;
        K.sc4 = (float)d->sigma_c4;
        K.inv_sc0 = 1.0f / K.sc0;
        K.inv_sc4 = 1.0f / K.sc4;
        K.support_min = K.sc4 < K.sc0 ? K.sc4 : K.sc0;
        K.maxw = (float)d->maximum_weight;
        for (int i = 0; i < 9; ++i) K.maxcov[i] = (float)d->maximum_eigenvalue_covariance[i];
        K.wimg = nullptr;
        K.wten = nullptr;
        K.wsup = nullptr;
        K.sup_default = (double)K.support_min;
        K.gw = make_geo(d->weight_image_geometry, D, 0);
        K.gt = make_geo(d->weight_tensor_geometry, D, 0);

        // images: the caller's doubles (host arrays, or device memory read in place) become float
        // copies on the device, the coefficients also as rows of 4 (one aligned 16-byte load per
        // B-spline stencil row)
        long long ncoef = 1;
        for (int k = 0; k < D; ++k) ncoef *= (d->moving_geometry.size[k] + 3);
        if (ncoef >= (1LL << 31))
            return fail(SKM_ERR_UNSUPPORTED, "moving image coefficients: %lld entries, at most 2^31 - 1", ncoef);
        {
            StagedDoubles fix, coef;
            int src = fix.stage(d->fixed_image, e->N, e->stream);
            if (!src) src = coef.stage(d->moving_coefficients, ncoef, e->stream);
            if (src) return src;
            if (dalloc(&e->d_fixed, e->N) || dalloc(&e->d_coeffs, ncoef) || dalloc(&e->d_coeffs4, ncoef))
                return SKM_ERR_CUDA;
            to_float_kernel<<<grid_for(e->N), 256, 0, e->stream>>>(fix.p, e->N, e->d_fixed);
            to_float_kernel<<<grid_for(ncoef), 256, 0, e->stream>>>(coef.p, ncoef, e->d_coeffs);
            expand_rows_kernel<<<grid_for(ncoef), 256, 0, e->stream>>>(e->d_coeffs, ncoef, e->d_coeffs4);
            SKM_CHECK_LAUNCH();
            SKM_CUDA(cudaStreamSynchronize(e->stream));      // before the staging buffers go back to the pool
        }
        if (d->use_weight_image) {
            long long n = texels(d->weight_image_geometry, D);
            std::vector<float> w((size_t)n);
            for (long long i = 0; i < n; ++i) w[i] = (float)d->weight_image[i];
            if (dalloc(&e->d_wimg, n)) return SKM_ERR_CUDA;
            SKM_CUDA(cudaMemcpy(e->d_wimg, w.data(), n * sizeof(float), cudaMemcpyHostToDevice));
            K.wimg = e->d_wimg;
            std::vector<double> sup((size_t)n);
            support_table(K, D, d->weight_image, n, sup.data(), &K.sup_default);
            if (dalloc(&e->d_wsup, n)) return SKM_ERR_CUDA;
            SKM_CUDA(cudaMemcpy(e->d_wsup, sup.data(), n * sizeof(double), cudaMemcpyHostToDevice));
            K.wsup = e->d_wsup;
        }
        if (d->use_weight_tensor) {
            long long n = texels(d->weight_tensor_geometry, D) * D * D;
            std::vector<float> w((size_t)n);
            for (long long i = 0; i < n; ++i) w[i] = (float)d->weight_tensor[i];
            if (dalloc(&e->d_wten, n)) return SKM_ERR_CUDA;
            SKM_CUDA(cudaMemcpy(e->d_wten, w.data(), n * sizeof(float), cudaMemcpyHostToDevice));
            K.wten = e->d_wten;
            long long nt = texels(d->weight_tensor_geometry, D);
            std::vector<double> sup((size_t)nt);
            support_table(K, D, d->weight_tensor, nt, sup.data(), &K.sup_default);
            if (dalloc(&e->d_wsup, nt)) return SKM_ERR_CUDA;
            SKM_CUDA(cudaMemcpy(e->d_wsup, sup.data(), nt * sizeof(double), cudaMemcpyHostToDevice));
            K.wsup = e->d_wsup;
        }
        P.fixed_data = e->d_fixed;
        P.coeffs = e->d_coeffs;
        P.coeffs4 = e->d_coeffs4;

        if (dalloc(&e->d_cpd, e->C)) return SKM_ERR_CUDA;
        P.cpd = e->d_cpd;
        if (P.sub > 1) {
            if (dalloc(&e->d_shifts, e->Ns)) return SKM_ERR_CUDA;
        }
        P.shifts = e->d_shifts;
        if (dalloc(&e->d_samp, e->Ns)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_in, e->C * (D + 1))) return SKM_ERR_CUDA;
        if (dalloc(&e->d_part, (size_t)NQ * e->value_blocks)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_stats, NS)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_counters, 4)) return SKM_ERR_CUDA;
        SKM_CUDA(cudaMemset(e->d_counters, 0, 4 * sizeof(unsigned)));
        if (dalloc(&e->d_deriv, e->nparams)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_rpart, (size_t)NR * std::max<long long>(e->C, std::max(e->deriv_blocks, e->gather_blocks))))
            return SKM_ERR_CUDA;
        if (dalloc(&e->d_out, NO)) return SKM_ERR_CUDA;
        SKM_CUDA(cudaHostAlloc((void **)&e->h_in, sizeof(double) * e->C * (D + 1), cudaHostAllocMapped));
        SKM_CUDA(cudaHostAlloc((void **)&e->h_out, sizeof(double) * (e->nparams + NO), cudaHostAllocMapped));
        SKM_CUDA(cudaHostGetDevicePointer((void **)&e->dh_in, e->h_in, 0));
        SKM_CUDA(cudaHostGetDevicePointer((void **)&e->dh_out, e->h_out, 0));
        rng_jump_table(e->jump);
        int trc = table_plan(e->table, e->P, D, e->stream);
        if (trc) return fail(SKM_ERR_CUDA, "table plan failed: %s", cudaGetErrorString(cudaGetLastError()));
        if (e->table.enabled && (table_set_attributes(e->table) || table_size_grids(e->table)))
            return fail(SKM_ERR_CUDA, "table kernel attributes: %s", cudaGetErrorString(cudaGetLastError()));
        if (e->table.enabled && table_tc_plan(e->tc, e->table, e->P.cp.n, e->stream))
            return fail(SKM_ERR_CUDA, "tensor-core table plan: %s", cudaGetErrorString(cudaGetLastError()));
        if (e->table.enabled && e->tc.enabled && warp_tma_plan(e->tc.wt, e->table, e->P, e->d_coeffs, e->stream))
            return fail(SKM_ERR_CUDA, "staged warp kernel plan: %s", cudaGetErrorString(cudaGetLastError()));
        return SKM_OK;
    }();
    if (rc) {
        delete e;
        return rc;
    }
    *out = e;
    return SKM_OK;
}

extern "C" int skm_evaluator_destroy(skm_evaluator *e)
{
    delete e;
    return SKM_OK;
}

extern "C" int skm_evaluator_path(skm_evaluator *e, int32_t request, int32_t *active)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    if (request == 1) {
        e->use_table = false;
    } else if (request == 0) {
        e->use_table = true;
        e->use_tc = true;
        e->tc.fused_on = false;
    } else if (request == 2) {
        e->use_table = true;
        e->use_tc = false;
    } else if (request == 3) {
        e->use_table = true;
        e->use_tc = true;
        e->tc.fused_on = true;
    } else if (request != -1) {
        return fail(SKM_ERR_INVALID, "path request must be -1, 0, 1, 2 or 3");
    }
    if (active) *active = active_path(e);
    return SKM_OK;
}

extern "C" int skm_evaluator_describe(skm_evaluator *e, skm_evaluator_info *out)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    skm_evaluator_info r{};
    r.path = active_path(e);
    r.dimensions = e->D;
    r.fixed_texels = e->N;
    r.samples = e->Ns;
    r.control_points = e->C;
    if (e->table.enabled) {
        const TableDev &T = e->table.dev;
        r.table_phases = T.nph;
        r.table_taps = T.ntap;
        for (int d = 0; d < 3; ++d) r.table_cells_per_axis[d] = T.nq[d];
        r.table_cells = T.ncell;
        r.table_regularizer_offsets = T.nkcp;
    }
    if (e->table.enabled && e->tc.enabled) {
        const TcDev &C = e->tc.dev;
        r.tc_cells_per_tile = C.ct;
        r.tc_brick[0] = C.bx;
        r.tc_brick[1] = C.by;
        r.tc_brick[2] = C.bz;
        r.tc_transform_tiles = (int64_t)C.tiles[0] * C.tiles[1] * C.tiles[2];
        r.tc_contrib_tiles = tc_bricks(e->tc) ? (int64_t)C.nbrick[0] * C.nbrick[1] * C.nbrick[2]
                                              : (e->table.dev.ncell + C.ctc - 1) / C.ctc;
        r.tc_transform_n = 2 * C.np;
        r.tc_transform_k = C.kp;
        r.tc_contrib_n = C.npc;
        r.tc_contrib_k = C.kpc;
        r.tc_contrib_taps = C.nct;
        r.warp_staged = (e->D == 3 && e->tc.wt.enabled) ? 1 : 0;
        r.tc_region_buffers = C.nrb;
        r.tc_u_staging = C.nus;
        r.tc_record_slots = C.nrr;
        r.tc_contrib_bricks = tc_bricks(e->tc) ? 1 : 0;
    }
    *out = r;
    return SKM_OK;
}

extern "C" int skm_evaluator_wait_drill(skm_evaluator *e, int32_t armed)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    if (armed && active_path(e) != 3)
        return fail(SKM_ERR_UNSUPPORTED, "the wait drill needs the tensor-core table path (active path %d)",
                    active_path(e));
    e->drill_armed = armed != 0;
    return SKM_OK;
}

extern "C" int skm_set_regularizer_rkhs(skm_evaluator *e, double w)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    e->reg_rkhs = w;
    return SKM_OK;
}

extern "C" int skm_set_regularizer_rd(skm_evaluator *e, double w, double scaling)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    e->reg_rd = w;
    e->rd_scaling = scaling;
    return SKM_OK;
}

extern "C" int skm_set_regularizer_pg(skm_evaluator *e, double w, double scaling)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    e->reg_pg = w;
    e->pg_scaling = scaling;
    return SKM_OK;
}

// ------------------------------------------------------------------------------------------------
static int upload_field(skm_evaluator *e, const skm_field *df)
{
    const double *key = (df && df->data) ? df->data : nullptr;
    if (key == e->df_key) return SKM_OK;           // cached by host pointer (GpuEvaluator.cu:120-126)
    e->df_key = key;
    e->P.has_df = 0;
    if (!key) return SKM_OK;
    int D = e->D;
    if (!geometry_ok(df->geometry, D)) return fail(SKM_ERR_INVALID, "invalid displacement-field geometry");
    long long n = texels(df->geometry, D);
    if (n > e->df_texels) {
        e->clear_metric_graphs();                  // their kernels read the old buffer
        if (e->d_df) pool_free(e->d_df);
        e->d_df = nullptr;
        if (dalloc(&e->d_df, n)) return SKM_ERR_CUDA;
        e->df_texels = n;
    }
    if (device_memory(key)) {                      // a device field: converted in place
        field_to_float4_kernel<<<grid_for(n), 256, 0, e->stream>>>(key, n, D, e->d_df);
        SKM_CHECK_LAUNCH();
    } else {
        std::vector<float4> tmp((size_t)n);
        for (long long i = 0; i < n; ++i)
            tmp[i] = make_float4((float)key[i * D], (float)key[i * D + 1], D > 2 ? (float)key[i * D + 2] : 0.f, 0.f);
        SKM_CUDA(cudaMemcpyAsync(e->d_df, tmp.data(), n * sizeof(float4), cudaMemcpyHostToDevice, e->stream));
    }
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    e->P.df = make_geo(df->geometry, D, 0);
    e->P.dfd = e->d_df;
    e->P.has_df = 1;
    return SKM_OK;
}

// H2D of the parameters (AoS control points or planar parameters) and the weights.
static int upload_params(skm_evaluator *e, const double *cp, const double *cpw, bool planar)
{
    if (!cp || !cpw) return fail(SKM_ERR_INVALID, "control points / weights are NULL");
    const long long C = e->C, n = C * e->D;
    // (the previous call synchronised the stream, so the staging buffer is free)
    std::memcpy(e->h_in, cp, sizeof(double) * n);
    SKM_CUDA(cudaMemcpyAsync(e->d_in, e->h_in, sizeof(double) * n, cudaMemcpyHostToDevice, e->stream));
    // weights: most callers pass the same weights every time; compare with the staged copy
    if (!e->weights_uploaded || std::memcmp(e->h_in + n, cpw, sizeof(double) * C) != 0) {
        e->weights_uploaded = false;
        std::memcpy(e->h_in + n, cpw, sizeof(double) * C);
        SKM_CUDA(cudaMemcpyAsync(e->d_in + n, e->h_in + n, sizeof(double) * C, cudaMemcpyHostToDevice, e->stream));
        e->weights_uploaded = true;
    }
    int blocks = (int)((C + 255) / 256);
    if (planar)
        pack_cp_planar<<<blocks, 256, 0, e->stream>>>(e->d_in, e->d_in + n, C, e->D, e->d_cpd, planes_of(e));
    else
        pack_cp_aos<<<blocks, 256, 0, e->stream>>>(e->d_in, e->d_in + n, C, e->D, e->d_cpd, planes_of(e));
    SKM_CHECK_LAUNCH();
    return SKM_OK;
}

static int draw_shifts(skm_evaluator *e, int do_resampling)
{
    if (e->P.sub <= 1) return SKM_OK;
    if (e->evaluated_once && !do_resampling) return SKM_OK;    // GpuEvaluator.cu:107-115
    int blocks = (int)((e->Ns + 255) / 256);
    shifts_kernel<<<blocks, 256, 0, e->stream>>>(e->rng_state, e->jump, e->Ns, e->D, e->P.sub, e->d_shifts);
    SKM_CHECK_LAUNCH();
    e->rng_state = rng_advance_host(e->rng_state, (unsigned long long)e->Ns * e->D, e->jump);
    e->evaluated_once = true;
    return SKM_OK;
}

static int ensure_dense(skm_evaluator *e)
{
    if (!e->d_dense) {
        if (dalloc(&e->d_dense, e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_dense_in, e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_need, (e->N + 31) / 32)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_list, e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_nlist, 1)) return SKM_ERR_CUDA;
    }
    if (e->D == 3 && e->P.K.kind != kStationary && !e->d_dense_sw) {
        if (dalloc(&e->d_dense_sw, e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_dense_sw_in, e->N)) return SKM_ERR_CUDA;
    }
    if (e->D == 3 && e->P.K.kind == kWeightTensor && !e->d_acache)
        if (dalloc(&e->d_acache, 3 * e->N)) return SKM_ERR_CUDA;
    return SKM_OK;
}

static int check_metric_for(const skm_evaluator *e, int metric);

// box-window LCC buffers (allocated on its first use, outside any stream capture)
static int ensure_box(skm_evaluator *e)
{
    if (!e->d_box_in) {
        if (dalloc(&e->d_box_in, e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_box_a, (size_t)kBoxMoments * e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_box_b, (size_t)kBoxMoments * e->N)) return SKM_ERR_CUDA;
        if (dalloc(&e->d_box_coef, e->N)) return SKM_ERR_CUDA;
    }
    return SKM_OK;
}

struct RegWeights {
    double rkhs, rd, rd_scaling, pg, pg_scaling, l1, l21, l2;
    int with_metric, negate;
};

// The full device sequence of one evaluation (everything after the parameter upload).
// ev (optional, 6 events), for per-phase timing: after the transform (table path; the whole value
// pass on the generic path), after the warp + statistics kernel, after the statistics kernel, after
// the contrib GEMM (table path), after the derivative gather and after the result kernel.
// step (optional): the optimizer step, fused into the table gather when that kernel runs (*fused
// then says so; otherwise the caller applies the step itself)
static int run_evaluation(skm_evaluator *e, int metric, bool derivative, const RegWeights &w, const double *params,
                          cudaEvent_t *ev = nullptr, double *deriv_out = nullptr, double *res_out = nullptr,
                          const OptStep *step = nullptr, bool *fused = nullptr)
{
    if (fused) *fused = false;
    double *d_deriv = deriv_out ? deriv_out : e->d_deriv, *d_res = res_out ? res_out : e->d_out;
    int rc = SKM_OK;
    const int D = e->D, kind = e->P.K.kind;
    const bool local = metric == SKM_LCC || metric == SKM_LCC_BOX;   // generic kernels only
    if (metric == SKM_LCC) {
        if ((rc = ensure_dense(e))) return rc;
        if ((rc = dispatch<LaunchLccValue>(D, kind, e))) return rc;
    } else if (metric == SKM_LCC_BOX) {
        if ((rc = check_metric_for(e, metric))) return rc;        // every texel a sample
        if ((rc = ensure_box(e))) return rc;
        if ((rc = dispatch<LaunchBoxValue>(D, kind, e))) return rc;
    }
    const bool tab = e->use_table && e->table.enabled && !local;
    if (!local) {
        if (tab) {
            if (table_value(e->table, tc_of(e), e->P, D, metric, e->d_stats, e->d_counters, e->stream,
                            ev ? ev[0] : nullptr))
                return fail(SKM_ERR_CUDA, "table value pass: %s", cudaGetErrorString(cudaGetLastError()));
        } else if ((rc = dispatch<LaunchValue>(D, kind, e))) {
            return rc;
        }
    }
    if (ev && !tab) SKM_CUDA(cudaEventRecord(ev[0], e->stream));
    if (ev) SKM_CUDA(cudaEventRecord(ev[1], e->stream));
    if (!tab) {                                  // the table path computes the statistics in its warp kernel
        stats_kernel<<<1, 1024, 0, e->stream>>>(e->d_part, e->value_blocks, metric, e->d_stats);
        SKM_CHECK_LAUNCH();
    }
    if (ev) SKM_CUDA(cudaEventRecord(ev[2], e->stream));
    DerivParams Q{};
    Q.metric = metric;
    Q.with_metric = w.with_metric;
    Q.reg_rkhs = w.rkhs;
    Q.reg_rd = w.rd;
    Q.rd_scaling = w.rd_scaling;
    Q.reg_pg = w.pg;
    Q.pg_scaling = w.pg_scaling;
    Q.reg_l1 = w.l1;
    Q.reg_l21 = w.l21;
    Q.reg_l2 = w.l2;
    Q.negate = w.negate;
    Q.stats = e->d_stats;
    Q.params = params;
    Q.samp = e->d_samp;
    Q.dense = e->d_dense;
    Q.dense_in = e->d_dense_in;
    Q.dense_sw = e->d_dense_sw;
    Q.dense_sw_in = e->d_dense_sw_in;
    Q.acache = e->d_acache;
    Q.boxcoef = metric == SKM_LCC_BOX ? e->d_box_coef : nullptr;
    Q.deriv = d_deriv;
    Q.rpart = e->d_rpart;
    Q.out = d_res;
    Q.counter = e->d_counters + 1;
    bool any_reg = w.rkhs > 0 || w.rd > 0 || w.pg > 0 || w.with_metric;
    // few control points (coarse levels): a block per control point keeps every SM busy
    const bool split = derivative && !tab && metric != SKM_LCC && e->deriv_blocks < kSplitBelowBlocks;
    if (derivative) {
        if (tab) {
            if (step) {
                Q.step = *step;
                Q.step.on = 1;
                if (fused) *fused = true;
            }
            if (table_derivative(e->table, tc_of(e), e->P, Q, D, e->gather_blocks, e->stream, ev ? ev[3] : nullptr))
                return fail(SKM_ERR_CUDA, "table derivative: %s", cudaGetErrorString(cudaGetLastError()));
        } else {
            if (ev) SKM_CUDA(cudaEventRecord(ev[3], e->stream));
            if ((rc = dispatch<LaunchDeriv>(D, kind, e, Q, split))) return rc;
        }
    } else if (any_reg && tab) {
        // values only, through the same gather (and the same sums) as the derivative call, so
        // that GetValue and GetValueAndDerivative return identical values
        Q.values_only = 1;
        if (table_derivative_gather_only(e->table, e->P, Q, D, e->gather_blocks, e->stream))
            return fail(SKM_ERR_CUDA, "table regularizer values: %s", cudaGetErrorString(cudaGetLastError()));
    } else if (any_reg) {
        if ((rc = dispatch<LaunchRegValue>(D, kind, e, Q))) return rc;
    }
    if (ev && !derivative) SKM_CUDA(cudaEventRecord(ev[3], e->stream));
    if (ev) SKM_CUDA(cudaEventRecord(ev[4], e->stream));
    if (!((derivative || any_reg) && tab)) {    // the table gather computes the result itself
        result_kernel<<<1, 256, 0, e->stream>>>(e->d_stats, (derivative || any_reg) ? e->d_rpart : nullptr,
                                               split ? (int)e->C : e->deriv_blocks, w.rkhs, w.rd, w.pg, w.l1,
                                               w.l21, w.l2, d_res,
                                               tab ? e->table.dev.tc_err : nullptr);
        SKM_CHECK_LAUNCH();
    }
    if (ev) SKM_CUDA(cudaEventRecord(ev[5], e->stream));
    return SKM_OK;
}

// A bounded wait of a tensor-core kernel gave up: reset the sticky word and report it.
static int report_fault(skm_evaluator *e)
{
    if (e->tc.d_err) {
        cudaMemsetAsync(e->tc.d_err, 0, sizeof(unsigned), e->stream);
        cudaStreamSynchronize(e->stream);
    }
    return fail(SKM_ERR_TIMEOUT, "a tensor-core kernel gave up waiting for its MMAs; results discarded");
}

// Reads the sticky fault word (paths that do not copy the result vector back).
static int check_fault(skm_evaluator *e)
{
    if (!e->tc.d_err) return SKM_OK;
    unsigned f = 0;
    SKM_CUDA(cudaMemcpyAsync(&f, e->tc.d_err, sizeof f, cudaMemcpyDeviceToHost, e->stream));
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    return f ? report_fault(e) : SKM_OK;
}

static int fetch(skm_evaluator *e, double *derivative)
{
    SKM_CUDA(cudaMemcpyAsync(e->h_out, e->d_out, sizeof(double) * NO, cudaMemcpyDeviceToHost, e->stream));
    if (derivative)
        SKM_CUDA(cudaMemcpyAsync(e->h_out + NO, e->d_deriv, sizeof(double) * e->nparams, cudaMemcpyDeviceToHost,
                                 e->stream));
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    if (e->h_out[O_FAULT] != 0.0) return report_fault(e);
    if (derivative) std::memcpy(derivative, e->h_out + NO, sizeof(double) * e->nparams);
    return SKM_OK;
}

static int check_metric(int metric)
{
    if (metric != SKM_MSE && metric != SKM_NCC && metric != SKM_LCC && metric != SKM_LCC_BOX)
        return fail(SKM_ERR_INVALID, "unknown metric %d", metric);
    return SKM_OK;
}

// the metric against the evaluator: the box-window LCC takes every texel as a window centre
static int check_metric_for(const skm_evaluator *e, int metric)
{
    int rc = check_metric(metric);
    if (rc) return rc;
    if (metric == SKM_LCC_BOX && e->P.sub != 1)
        return fail(SKM_ERR_INVALID, "the box-window LCC needs subsample 1 (every texel a window centre)");
    return SKM_OK;
}

static int evaluate_common(skm_evaluator *e, int32_t metric, const double *cp, const double *cpw,
                           const skm_field *df, double *derivatives, int32_t do_resampling, skm_result *out)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    int rc;
    if ((rc = check_metric_for(e, metric))) return rc;
    SKM_CUDA(cudaSetDevice(e->device));
    if ((rc = upload_field(e, df))) return rc;
    if ((rc = upload_params(e, cp, cpw, false))) return rc;
    if ((rc = draw_shifts(e, do_resampling))) return rc;
    RegWeights w{};
    w.rkhs = e->reg_rkhs > 0 ? e->reg_rkhs : 0.0;
    w.rd = e->reg_rd > 0 ? e->reg_rd : 0.0;
    w.rd_scaling = e->rd_scaling;
    w.pg = e->reg_pg > 0 ? e->reg_pg : 0.0;
    w.pg_scaling = e->pg_scaling;
    const bool drill = e->drill_armed && derivatives != nullptr && active_path(e) == 3 && metric != SKM_LCC &&
                       metric != SKM_LCC_BOX;
    if (drill) {                      // one launch of the contrib kernel runs the wait drill
        e->tc.dev.drill = 1;
        e->tc.dev.wait_ns = kDrillWaitNs;
    }
    rc = run_evaluation(e, metric, derivatives != nullptr, w, nullptr);
    if (drill) {
        e->tc.dev.drill = 0;
        e->tc.dev.wait_ns = tc::kTcWaitNs;
        e->drill_armed = false;
    }
    if (rc) return rc;
    if ((rc = fetch(e, derivatives))) return rc;
    if (out) {
        out->measure = e->h_out[O_MEASURE];
        out->reg_value_rkhs = e->h_out[O_RKHS];
        out->reg_value_rd = e->h_out[O_RD];
        out->reg_value_pg = e->h_out[O_PG];
        out->num_pixels_counted = (uint32_t)e->h_out[O_COUNT];
    }
    return SKM_OK;
}

extern "C" int skm_get_value(skm_evaluator *e, int32_t metric, const double *cp, const double *cpw,
                             const skm_field *df, int32_t do_resampling, skm_result *out)
{
    return evaluate_common(e, metric, cp, cpw, df, nullptr, do_resampling, out);
}

extern "C" int skm_get_value_and_derivative(skm_evaluator *e, int32_t metric, const double *cp, const double *cpw,
                                            const skm_field *df, double *derivatives, int32_t do_resampling,
                                            skm_result *out)
{
    if (!derivatives) return fail(SKM_ERR_INVALID, "derivatives is NULL");
    return evaluate_common(e, metric, cp, cpw, df, derivatives, do_resampling, out);
}

static int validate_metric(const skm_metric_desc *m)
{
    if (!m) return fail(SKM_ERR_INVALID, "metric descriptor is NULL");
    int rc = check_metric(m->metric);
    if (rc) return rc;
    if (m->reg_l1 < 0 || m->reg_l21 < 0 || m->reg_l2 < 0 || m->reg_rkhs < 0 || m->reg_rd < 0 || m->reg_pg < 0)
        return fail(SKM_ERR_INVALID, "Regularization weights must be positive.");          // hxx:79-84
    if (!(m->reg_rd_scaling > 0) || !(m->reg_pg_scaling > 0))
        return fail(SKM_ERR_INVALID, "Robust regularization scales must be strictly positive.");   // hxx:86-88
    return SKM_OK;
}

// Device part of one metric evaluation on already-uploaded planar parameters (e->d_in); the
// derivative and the result vector go to deriv_out / res_out when given.
int skm_metric_device(skm_evaluator *e, const skm_metric_desc *m, bool derivative, double *deriv_out = nullptr,
                      double *res_out = nullptr)
{
    RegWeights w{};
    w.rkhs = m->reg_rkhs;
    w.rd = m->reg_rd;
    w.rd_scaling = m->reg_rd_scaling;
    w.pg = m->reg_pg;
    w.pg_scaling = m->reg_pg_scaling;
    w.l1 = m->reg_l1;
    w.l21 = m->reg_l21;
    w.l2 = m->reg_l2;
    w.with_metric = 1;
    w.negate = m->use_negative_gradient;
    return run_evaluation(e, m->metric, derivative, w, e->d_in, nullptr, deriv_out, res_out);
}

static bool same_metric(const skm_metric_desc &a, const skm_metric_desc &b)
{
    return a.metric == b.metric && a.reg_l1 == b.reg_l1 && a.reg_l21 == b.reg_l21 && a.reg_l2 == b.reg_l2 &&
           a.reg_rkhs == b.reg_rkhs && a.reg_rd == b.reg_rd && a.reg_rd_scaling == b.reg_rd_scaling &&
           a.reg_pg == b.reg_pg && a.reg_pg_scaling == b.reg_pg_scaling &&
           a.use_negative_gradient == b.use_negative_gradient && a.do_resampling == b.do_resampling;
}

// Enqueues (or captures) the device part of skm_metric_evaluate with no copy operations: the
// packing kernel reads the parameters from the pinned staging buffer over the bus (and keeps a
// device copy for the regularizers), and the final kernels write the derivative and the result
// vector straight into the pinned h_out.
// params_dev: the parameters as the device reads them (the pinned staging buffer, or the caller's
// own page-locked buffer); deriv_dev: where the derivative goes (staging, or the caller's buffer).
static int metric_sequence(skm_evaluator *e, const skm_metric_desc *m, bool derivative, const double *params_dev,
                           double *deriv_dev)
{
    const long long C = e->C, n = C * e->D;
    pack_cp_planar_copy<<<(int)((C + 255) / 256), 256, 0, e->stream>>>(params_dev, e->d_in + n, C, e->D, e->d_cpd,
                                                                      e->d_in, planes_of(e));
    SKM_CHECK_LAUNCH();
    return skm_metric_device(e, m, derivative, deriv_dev, e->dh_out);
}

// Device address of a page-locked host buffer the GPU can read and write directly, else nullptr.
static void *mapped_device_ptr(const void *p)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (a.type != cudaMemoryTypeHost || !a.devicePointer || (reinterpret_cast<uintptr_t>(p) & 7u)) return nullptr;
    return a.devicePointer;
}

extern "C" int skm_metric_evaluate(skm_evaluator *e, const skm_metric_desc *m, const double *parameters,
                                   const double *cpw, const skm_field *df, double *derivative,
                                   skm_metric_values *out)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    int rc;
    if ((rc = validate_metric(m))) return rc;
    if (!parameters || !cpw) return fail(SKM_ERR_INVALID, "control points / weights are NULL");
    SKM_CUDA(cudaSetDevice(e->device));
    if ((rc = upload_field(e, df))) return rc;
    const long long C = e->C, n = C * e->D;
    // page-locked caller buffers are read and written by the kernels directly; others go through the
    // pinned staging buffers (the previous call synchronised the stream, so those are free)
    const double *pdev = static_cast<const double *>(mapped_device_ptr(parameters));
    double *gdev = derivative ? static_cast<double *>(mapped_device_ptr(derivative)) : nullptr;
    if (!pdev) {
        std::memcpy(e->h_in, parameters, sizeof(double) * n);
        pdev = e->dh_in;
    }
    double *gout = gdev ? gdev : e->dh_out + NO;
    if (!e->weights_uploaded || std::memcmp(e->h_in + n, cpw, sizeof(double) * C) != 0) {
        e->weights_uploaded = false;
        std::memcpy(e->h_in + n, cpw, sizeof(double) * C);
        SKM_CUDA(cudaMemcpyAsync(e->d_in + n, e->h_in + n, sizeof(double) * C, cudaMemcpyHostToDevice, e->stream));
        e->weights_uploaded = true;
    }
    const bool deriv = derivative != nullptr;
    if (m->metric == SKM_LCC && (rc = ensure_dense(e))) return rc;   // allocates: not inside a capture
    if (m->metric == SKM_LCC_BOX && ((rc = check_metric_for(e, m->metric)) || (rc = ensure_box(e)))) return rc;
    if (e->P.sub <= 1) {
        // no sampling offsets to draw: the whole device part is one graph launch
        const int path = active_path(e);
        skm_evaluator::MetricGraph *hit = nullptr, *victim = nullptr;
        for (skm_evaluator::MetricGraph &g : e->mg) {
            if (g.exec && same_metric(g.desc, *m) && g.deriv == deriv && g.path == path && g.df == e->df_key &&
                g.pdev == pdev && g.gout == gout) {
                hit = &g;
                break;
            }
            if (!victim || (victim->exec && (!g.exec || g.used < victim->used))) victim = &g;
        }
        if (!hit) {
            if (victim->exec) cudaGraphExecDestroy(victim->exec);
            *victim = skm_evaluator::MetricGraph{};
            SKM_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
            int r = metric_sequence(e, m, deriv, pdev, gout);
            cudaGraph_t g = nullptr;
            cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
            if (r) {
                if (g) cudaGraphDestroy(g);
                return r;
            }
            if (ce != cudaSuccess) return fail(SKM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
            cudaError_t ie = cudaGraphInstantiate(&victim->exec, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) {
                victim->exec = nullptr;
                return fail(SKM_ERR_CUDA, "graph instantiation failed: %s", cudaGetErrorString(ie));
            }
            victim->desc = *m;
            victim->deriv = deriv;
            victim->path = path;
            victim->df = e->df_key;
            victim->pdev = pdev;
            victim->gout = gout;
            hit = victim;
        }
        hit->used = ++e->mg_clock;
        SKM_CUDA(cudaGraphLaunch(hit->exec, e->stream));
    } else {
        if ((rc = draw_shifts(e, m->do_resampling))) return rc;
        if ((rc = metric_sequence(e, m, deriv, pdev, gout))) return rc;
    }
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    if (e->h_out[O_FAULT] != 0.0) return report_fault(e);
    if (derivative && !gdev) std::memcpy(derivative, e->h_out + NO, sizeof(double) * e->nparams);
    if (out) {
        const double *o = e->h_out;
        out->value = o[O_VALUE];
        out->measure = o[O_MEASURE];
        out->reg_value = o[O_REG];
        out->reg_l1 = o[O_L1];
        out->reg_l21 = o[O_L21];
        out->reg_l2 = o[O_L2];
        out->reg_rkhs = o[O_RKHS];
        out->reg_rd = o[O_RD];
        out->reg_pg = o[O_PG];
        out->num_pixels_counted = (uint32_t)o[O_COUNT];
    }
    return SKM_OK;
}

extern "C" int skm_evaluate_displacement_field(skm_evaluator *e, const double *cp, const double *cpw,
                                               const skm_field *df, double *dst)
{
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    if (!dst) return fail(SKM_ERR_INVALID, "dst is NULL");
    int rc;
    SKM_CUDA(cudaSetDevice(e->device));
    if ((rc = upload_field(e, df))) return rc;
    if ((rc = upload_params(e, cp, cpw, false))) return rc;
    // a device destination is written in place, a host one through a device buffer
    const bool on_device = device_memory(dst);
    double *d_out = on_device ? dst : nullptr;
    if (!on_device && dalloc(&d_out, (size_t)e->N * e->D)) return SKM_ERR_CUDA;
    rc = dispatch<LaunchDisp>(e->D, e->P.K.kind, e, d_out);
    if (!rc) {
        cudaError_t c1 = on_device ? cudaSuccess
                                   : cudaMemcpyAsync(dst, d_out, sizeof(double) * e->N * e->D, cudaMemcpyDeviceToHost,
                                                     e->stream);
        cudaError_t c2 = cudaStreamSynchronize(e->stream);
        if (c1 != cudaSuccess || c2 != cudaSuccess)
            rc = fail(SKM_ERR_CUDA, "displacement field copy failed: %s",
                      cudaGetErrorString(c1 != cudaSuccess ? c1 : c2));
    }
    if (!on_device) pool_free(d_out);
    return rc;
}

// ------------------------------------------------------------------------------------------------
// B-spline prefilter of a device image in place (BsplineImage.h:174-195), then the mirror-padded
// coefficient volume (size + 3 per axis) into d_out
static int bspline_coefficients_device(int D, int X, int Y, int Z, double *d_img, double *d_out, cudaStream_t s)
{
    const double pole = sqrt(3.0) - 2.0;
    if (D == 3) {                                  // z, then y, then x (BsplineImage.h:182-195)
        bs_prefilter_axis<<<(int)(((long long)X * Y + 127) / 128), 128, 0, s>>>(d_img, X, Y, Z, 2, pole);
        bs_prefilter_axis<<<(int)(((long long)X * Z + 127) / 128), 128, 0, s>>>(d_img, X, Y, Z, 1, pole);
        bs_prefilter_axis<<<(int)(((long long)Y * Z + 127) / 128), 128, 0, s>>>(d_img, X, Y, Z, 0, pole);
    } else {                                       // x, then y (BsplineImage.h:174-180)
        bs_prefilter_axis<<<(Y + 127) / 128, 128, 0, s>>>(d_img, X, Y, 1, 0, pole);
        bs_prefilter_axis<<<(X + 127) / 128, 128, 0, s>>>(d_img, X, Y, 1, 1, pole);
    }
    SKM_CHECK_LAUNCH();
    const long long pn = (long long)(X + 3) * (Y + 3) * (D == 3 ? Z + 3 : 1);
    bs_mirror_pad<<<(int)((pn + 255) / 256), 256, 0, s>>>(d_img, X, Y, Z, D, d_out);
    SKM_CHECK_LAUNCH();
    return SKM_OK;
}

extern "C" int skm_bspline_coefficients(int32_t D, const int32_t *size, const double *image, double *coeffs)
{
    if (D != 2 && D != 3) return fail(SKM_ERR_INVALID, "dimensions must be 2 or 3");
    if (!size || !image || !coeffs) return fail(SKM_ERR_INVALID, "NULL argument");
    int X = size[0], Y = size[1], Z = D == 3 ? size[2] : 1;
    if (X < 2 || Y < 2 || (D == 3 && Z < 2)) return fail(SKM_ERR_INVALID, "need at least 2 texels per axis");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SKM_ERR_CUDA, "no CUDA device available (this library has no CPU fallback)");
    }
    long long n = (long long)X * Y * Z;
    long long pn = (long long)(X + 3) * (Y + 3) * (D == 3 ? Z + 3 : 1);
    double *d_img = nullptr, *d_out = nullptr;
    cudaStream_t s = nullptr;
    int rc = [&]() -> int {
        SKM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        if (dalloc(&d_img, n)) return SKM_ERR_CUDA;
        if (dalloc(&d_out, pn)) return SKM_ERR_CUDA;
        // host or device arrays on either side (the copies infer their direction)
        SKM_CUDA(cudaMemcpyAsync(d_img, image, n * sizeof(double), cudaMemcpyDefault, s));
        int rc2 = bspline_coefficients_device(D, X, Y, Z, d_img, d_out, s);
        if (rc2) return rc2;
        SKM_CUDA(cudaMemcpyAsync(coeffs, d_out, pn * sizeof(double), cudaMemcpyDefault, s));
        SKM_CUDA(cudaStreamSynchronize(s));
        return SKM_OK;
    }();
    if (d_img) pool_free(d_img);
    if (d_out) pool_free(d_out);
    if (s) cudaStreamDestroy(s);
    return rc;
}

#include "skm_optimizer.cuh"
#include "skm_driver.cuh"
#include "skm_batch.cuh"
