// skm_optimizer.cuh -- device-resident adaptive-step gradient descent (included by skm_capi.cu).
//
// Restates the optimizer the reference drives its evaluator with:
//   ITK v4 gradient-descent loop: swap(previous, gradient); metric value+derivative; step; keep best
//   AdvanceOneStep (itkStandardGradientDescentOptimizerv4.hxx:83-114)
//   EstimateLearningRate: gamma(t) = a / (A + t + 1)^alpha       (itkAdaptiveStep...hxx:86-97)
//   x = x_prev + gamma * g, orthant projection                    (itkStandard...hxx:116-157)
//   t = max(0, t + f(-<g, g_prev>)), f(x) = Fmin + (Fmax-Fmin)/(1 - (Fmax/Fmin) e^(-x/omega))  (hxx:100-128)
// `g` is the metric's (negated) derivative, so the step goes downhill.  x_prev starts as the
// zero vector: ITK's StartOptimization zero-fills the gradient buffer that the first swap turns
// into the step base (itkStandardGradientDescentOptimizerv4.hxx:71-76).  The best parameters are the
// position after the step taken from the best evaluation, as ReturnBestParametersAndValue stores them.
//
// Everything (position, gradient, previous gradient, time, best value, RNG state) lives in device
// memory; one iteration is captured once into a CUDA graph and replayed.
#pragma once

namespace {

__global__ void shifts_dev_kernel(const unsigned long long *__restrict__ state, RngJump J, long long Ns, int D,
                                  int sub, uint32_t *__restrict__ shifts)
{
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= Ns) return;
    unsigned long long s = lcg_advance(*state, (unsigned long long)t * D, J);
    uint32_t packed = 0;
    for (int d = 0; d < D; ++d) {
        unsigned out = pcg32_output(s);
        s = s * 6364136223846793005ULL + 1ULL;
        double f = (double)out / 4294967295.0;
        packed |= (uint32_t)(int)(f * (double)sub) << (8 * d);
    }
    shifts[t] = packed;
}

__global__ void rng_advance_kernel(unsigned long long *state, RngJump J, unsigned long long steps)
{
    if (threadIdx.x == 0 && blockIdx.x == 0) *state = lcg_advance(*state, steps, J);
}

// One optimizer step over all parameters; the last block (fixed-order sum of the per-block
// <g, g_prev> partials) then updates the adaptive time, the best value and the counters.  Used
// where the derivative kernel does not apply the step itself (the table gather does, see
// OptStep): a pending best position left by such a fused step is taken over first.
__global__ void __launch_bounds__(256) opt_step_kernel(const double *__restrict__ g, double *__restrict__ tmp,
                                                       double *__restrict__ base, double *__restrict__ pos,
                                                       double *__restrict__ best, double *__restrict__ scal,
                                                       const double *__restrict__ out, long long P, int orthant,
                                                       double a, double A, double alpha, double f_max, double f_min,
                                                       double omega, double *__restrict__ sp_part, unsigned *counter)
{
    __shared__ double sh[32];
    const double t = scal[T_TIME];
    const double lr = a / pow(A + t + 1.0, alpha);
    const bool improving = out[O_VALUE] < scal[T_BEST];
    const bool pending = scal[T_PENDING] != 0.0;
    double sp = 0.0;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < P; j += (long long)gridDim.x * blockDim.x) {
        const double gj = g[j];
        sp += gj * tmp[j];
        tmp[j] = gj;
        if (pending) best[j] = pos[j];
        const double b = base[j];
        double nx = b + gj * lr;
        if (orthant && nx * b < 0.0) nx = 0.0;
        pos[j] = nx;
        base[j] = nx;
        if (improving) best[j] = nx;
    }
    double v[1] = {sp};
    block_sum<1>(v, sh);
    if (threadIdx.x == 0) sp_part[blockIdx.x] = v[0];
    if (last_block_arrived(counter)) {
        double w[1];
        sum_partials<1>(sp_part, gridDim.x, w, sh);
        if (threadIdx.x == 0) {
            const double x = -w[0];
            const double f = f_min + (f_max - f_min) / (1.0 - (f_max / f_min) * exp(-x / omega));
            scal[T_TIME] = fmax(0.0, t + f);
            if (out[O_VALUE] < scal[T_BEST]) scal[T_BEST] = out[O_VALUE];
            scal[T_LR] = lr;
            scal[T_SP] = w[0];
            scal[T_VALUE] = out[O_VALUE];
            scal[T_ITER] += 1.0;
            scal[T_COUNT] = out[O_COUNT];
            scal[T_PENDING] = 0.0;
        }
    }
}

// The best parameters after a fused step from an improving evaluation: the current position.
__global__ void opt_best_pending_kernel(const double *__restrict__ scal, const double *__restrict__ pos,
                                        double *__restrict__ best, long long P)
{
    if (scal[T_PENDING] == 0.0) return;
    for (long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x; j < P; j += (long long)gridDim.x * blockDim.x)
        best[j] = pos[j];
}

}  // namespace

struct skm_optimizer {
    skm_evaluator *e = nullptr;
    skm_optimizer_desc od{};
    skm_metric_desc md{};
    long long P = 0;
    double *d_pos = nullptr, *d_base = nullptr, *d_tmp = nullptr, *d_best = nullptr, *d_cpw = nullptr;
    double *d_scal = nullptr, *d_sp = nullptr;
    unsigned long long *d_rng = nullptr;
    int step_blocks = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int iteration = 0;

    ~skm_optimizer()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        void *bufs[] = {d_pos, d_base, d_tmp, d_best, d_cpw, d_scal, d_sp, d_rng};
        for (void *b : bufs)
            if (b) pool_free(b);
    }
};

// launches of one optimizer iteration (captured into the graph).  ev (optional, 10 events):
// start, after pack, after shifts, the six events of run_evaluation, after the update -- used by
// skm_optimizer_profile.
static int optimizer_iteration(skm_optimizer *o, cudaEvent_t *ev = nullptr)
{
    skm_evaluator *e = o->e;
    const long long C = e->C;
    if (ev) SKM_CUDA(cudaEventRecord(ev[0], e->stream));
    pack_cp_planar<<<(int)((C + 255) / 256), 256, 0, e->stream>>>(o->d_pos, o->d_cpw, C, e->D, e->d_cpd,
                                                                  planes_of(e));
    SKM_CHECK_LAUNCH();
    if (ev) SKM_CUDA(cudaEventRecord(ev[1], e->stream));
    if (e->P.sub > 1 && o->md.do_resampling) {
        shifts_dev_kernel<<<(int)((e->Ns + 255) / 256), 256, 0, e->stream>>>(o->d_rng, e->jump, e->Ns, e->D, e->P.sub,
                                                                            e->d_shifts);
        SKM_CHECK_LAUNCH();
        rng_advance_kernel<<<1, 1, 0, e->stream>>>(o->d_rng, e->jump, (unsigned long long)e->Ns * e->D);
        SKM_CHECK_LAUNCH();
    }
    RegWeights w{};
    w.rkhs = o->md.reg_rkhs;
    w.rd = o->md.reg_rd;
    w.rd_scaling = o->md.reg_rd_scaling;
    w.pg = o->md.reg_pg;
    w.pg_scaling = o->md.reg_pg_scaling;
    w.l1 = o->md.reg_l1;
    w.l21 = o->md.reg_l21;
    w.l2 = o->md.reg_l2;
    w.with_metric = 1;
    w.negate = o->md.use_negative_gradient;
    if (ev) SKM_CUDA(cudaEventRecord(ev[2], e->stream));
    OptStep st{};
    st.tmp = o->d_tmp;
    st.base = o->d_base;
    st.pos = o->d_pos;
    st.best = o->d_best;
    st.scal = o->d_scal;
    st.sp_part = o->d_sp;
    st.orthant = o->od.orthant_projection;
    st.a = o->od.a;
    st.A = o->od.A;
    st.alpha = o->od.alpha;
    st.f_max = o->od.f_max;
    st.f_min = o->od.f_min;
    st.omega = o->od.omega;
    bool fused = false;
    int rc = run_evaluation(e, o->md.metric, true, w, o->d_pos, ev ? ev + 3 : nullptr, nullptr, nullptr, &st, &fused);
    if (rc) return rc;
    if (!fused) {
        opt_step_kernel<<<o->step_blocks, 256, 0, e->stream>>>(e->d_deriv, o->d_tmp, o->d_base, o->d_pos, o->d_best,
                                                              o->d_scal, e->d_out, o->P, o->od.orthant_projection,
                                                              o->od.a, o->od.A, o->od.alpha, o->od.f_max, o->od.f_min,
                                                              o->od.omega, o->d_sp, e->d_counters + 2);
        SKM_CHECK_LAUNCH();
    }
    if (ev) SKM_CUDA(cudaEventRecord(ev[9], e->stream));
    return SKM_OK;
}

extern "C" int skm_optimizer_create(skm_evaluator *e, const skm_optimizer_desc *od, const skm_metric_desc *md,
                                    const double *initial, const double *cpw, const skm_field *df,
                                    skm_optimizer **out)
{
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    *out = nullptr;
    if (!e) return fail(SKM_ERR_STATE, "evaluator is NULL");
    if (!od || !initial || !cpw) return fail(SKM_ERR_INVALID, "NULL argument");
    int rc;
    if ((rc = validate_metric(md))) return rc;
    if (od->number_of_iterations < 0) return fail(SKM_ERR_INVALID, "number_of_iterations < 0");
    if (!(od->f_min != 0.0) || !(od->omega != 0.0)) return fail(SKM_ERR_INVALID, "f_min and omega must be nonzero");
    SKM_CUDA(cudaSetDevice(e->device));
    if ((rc = upload_field(e, df))) return rc;
    // LCC's dense fields are allocated on first use: that must happen before the iteration is captured
    if (md->metric == SKM_LCC && (rc = ensure_dense(e))) return rc;
    if (md->metric == SKM_LCC_BOX && ((rc = check_metric_for(e, md->metric)) || (rc = ensure_box(e)))) return rc;
    skm_optimizer *o = new skm_optimizer();
    o->e = e;
    o->od = *od;
    o->md = *md;
    o->P = e->nparams;
    o->step_blocks = (int)std::min<long long>((o->P + 255) / 256, 1184);
    rc = [&]() -> int {
        const long long P = o->P;
        if (dalloc(&o->d_pos, P) || dalloc(&o->d_base, P) || dalloc(&o->d_tmp, P) || dalloc(&o->d_best, P) ||
            dalloc(&o->d_cpw, e->C) || dalloc(&o->d_scal, NT) ||
            dalloc(&o->d_sp, std::max<long long>(o->step_blocks, e->gather_blocks)) ||
            dalloc(&o->d_rng, 1))
            return SKM_ERR_CUDA;
        SKM_CUDA(cudaMemcpyAsync(o->d_pos, initial, sizeof(double) * P, cudaMemcpyHostToDevice, e->stream));
        SKM_CUDA(cudaMemcpyAsync(o->d_best, initial, sizeof(double) * P, cudaMemcpyHostToDevice, e->stream));
        SKM_CUDA(cudaMemsetAsync(o->d_base, 0, sizeof(double) * P, e->stream));
        SKM_CUDA(cudaMemsetAsync(o->d_tmp, 0, sizeof(double) * P, e->stream));
        SKM_CUDA(cudaMemcpyAsync(o->d_cpw, cpw, sizeof(double) * e->C, cudaMemcpyHostToDevice, e->stream));
        double scal[NT] = {0.0, 1.7976931348623157e308, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        SKM_CUDA(cudaMemcpyAsync(o->d_scal, scal, sizeof scal, cudaMemcpyHostToDevice, e->stream));
        SKM_CUDA(cudaMemcpyAsync(o->d_rng, &e->rng_state, sizeof(unsigned long long), cudaMemcpyHostToDevice,
                                 e->stream));
        SKM_CUDA(cudaStreamSynchronize(e->stream));
        // without resampling the shifts are drawn once, before the first evaluation
        if (e->P.sub > 1 && !md->do_resampling && !e->evaluated_once) {
            int r = draw_shifts(e, 1);
            if (r) return r;
        }
        // capture one iteration
        SKM_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        int r = optimizer_iteration(o);
        cudaGraph_t g = nullptr;
        cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
        if (r) {
            if (g) cudaGraphDestroy(g);
            return r;
        }
        if (ce != cudaSuccess) return fail(SKM_ERR_CUDA, "graph capture failed: %s", cudaGetErrorString(ce));
        o->graph = g;
        SKM_CUDA(cudaGraphInstantiate(&o->exec, g, 0));
        return SKM_OK;
    }();
    if (rc) {
        delete o;
        return rc;
    }
    *out = o;
    return SKM_OK;
}

extern "C" int skm_optimizer_run(skm_optimizer *o, int32_t iterations)
{
    if (!o) return fail(SKM_ERR_STATE, "optimizer is NULL");
    if (iterations < 0) return fail(SKM_ERR_INVALID, "iterations < 0");
    skm_evaluator *e = o->e;
    SKM_CUDA(cudaSetDevice(e->device));
    int n = std::min<int>(iterations, o->od.number_of_iterations - o->iteration);
    for (int i = 0; i < n; ++i) SKM_CUDA(cudaGraphLaunch(o->exec, e->stream));
    o->iteration += n;
    // keep the evaluator's generator in step with the device copy
    SKM_CUDA(cudaMemcpyAsync(&e->rng_state, o->d_rng, sizeof(unsigned long long), cudaMemcpyDeviceToHost, e->stream));
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    if (n > 0 && e->P.sub > 1) e->evaluated_once = true;
    return check_fault(e);
}

// Enqueue iterations without waiting (used for timing the device-resident loop).
extern "C" int skm_optimizer_enqueue(skm_optimizer *o, int32_t iterations, void *stream_out)
{
    if (!o) return fail(SKM_ERR_STATE, "optimizer is NULL");
    skm_evaluator *e = o->e;
    int n = std::min<int>(iterations, o->od.number_of_iterations - o->iteration);
    for (int i = 0; i < n; ++i) SKM_CUDA(cudaGraphLaunch(o->exec, e->stream));
    o->iteration += n;
    if (stream_out) *(cudaStream_t *)stream_out = e->stream;
    return SKM_OK;
}

extern "C" int skm_optimizer_get_parameters(skm_optimizer *o, int32_t best, double *params)
{
    if (!o) return fail(SKM_ERR_STATE, "optimizer is NULL");
    if (!params) return fail(SKM_ERR_INVALID, "params is NULL");
    skm_evaluator *e = o->e;
    SKM_CUDA(cudaSetDevice(e->device));
    if (best) {
        opt_best_pending_kernel<<<o->step_blocks, 256, 0, e->stream>>>(o->d_scal, o->d_pos, o->d_best, o->P);
        SKM_CHECK_LAUNCH();
    }
    SKM_CUDA(cudaMemcpyAsync(params, best ? o->d_best : o->d_pos, sizeof(double) * o->P, cudaMemcpyDeviceToHost,
                             e->stream));
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    return SKM_OK;
}

extern "C" int skm_optimizer_get_state(skm_optimizer *o, skm_optimizer_state *out)
{
    if (!o) return fail(SKM_ERR_STATE, "optimizer is NULL");
    if (!out) return fail(SKM_ERR_INVALID, "out is NULL");
    skm_evaluator *e = o->e;
    double s[NT];
    SKM_CUDA(cudaSetDevice(e->device));
    SKM_CUDA(cudaMemcpyAsync(s, o->d_scal, sizeof s, cudaMemcpyDeviceToHost, e->stream));
    SKM_CUDA(cudaStreamSynchronize(e->stream));
    int rc = check_fault(e);
    if (rc) return rc;
    out->iteration = (int32_t)s[T_ITER];
    out->current_time = s[T_TIME];
    out->learning_rate = s[T_LR];
    out->value = s[T_VALUE];
    out->best_value = s[T_BEST];
    out->scalar_product = s[T_SP];
    out->num_pixels_counted = (uint32_t)s[T_COUNT];
    return SKM_OK;
}

extern "C" int skm_optimizer_destroy(skm_optimizer *o)
{
    if (o && o->e) cudaSetDevice(o->e->device);
    delete o;
    return SKM_OK;
}

// Runs up to `iterations` iterations un-graphed with CUDA events between the phases and
// returns the mean time per phase in milliseconds: [pack, shifts, transform (generic: value pass),
// warp + statistics, statistics, contrib GEMM, derivative gather (generic: derivative pass),
// result, update].  The iterations advance the optimizer like skm_optimizer_run.
extern "C" int skm_optimizer_profile(skm_optimizer *o, int32_t iterations, double *phase_ms, int32_t nphase)
{
    if (!o) return fail(SKM_ERR_STATE, "optimizer is NULL");
    if (!phase_ms || nphase < 9) return fail(SKM_ERR_INVALID, "phase_ms needs 9 entries");
    skm_evaluator *e = o->e;
    SKM_CUDA(cudaSetDevice(e->device));
    int n = std::min<int>(iterations, o->od.number_of_iterations - o->iteration);
    cudaEvent_t ev[10];
    for (int i = 0; i < 10; ++i) SKM_CUDA(cudaEventCreate(&ev[i]));
    double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    int rc = SKM_OK;
    for (int it = 0; it < n && !rc; ++it) {
        rc = optimizer_iteration(o, ev);
        if (rc) break;
        cudaError_t ce = cudaEventSynchronize(ev[9]);
        if (ce != cudaSuccess) {
            rc = fail(SKM_ERR_CUDA, "profile: %s", cudaGetErrorString(ce));
            break;
        }
        for (int p = 0; p < 9; ++p) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[p], ev[p + 1]);
            acc[p] += ms;
        }
        o->iteration++;
    }
    for (int i = 0; i < 10; ++i) cudaEventDestroy(ev[i]);
    for (int p = 0; p < 9; ++p) phase_ms[p] = n > 0 ? acc[p] / n : 0.0;
    return rc;
}

// Number of kernel launches in one captured optimizer iteration.
extern "C" int skm_optimizer_graph_kernel_count(skm_optimizer *o, int32_t *count)
{
    if (!o || !o->graph) return fail(SKM_ERR_STATE, "optimizer has no graph");
    size_t n = 0;
    SKM_CUDA(cudaGraphGetNodes(o->graph, nullptr, &n));
    std::vector<cudaGraphNode_t> nodes(n);
    SKM_CUDA(cudaGraphGetNodes(o->graph, nodes.data(), &n));
    int k = 0;
    for (size_t i = 0; i < n; ++i) {
        cudaGraphNodeType t;
        SKM_CUDA(cudaGraphNodeGetType(nodes[i], &t));
        if (t == cudaGraphNodeTypeKernel) ++k;
    }
    *count = k;
    return SKM_OK;
}
