/*
 * skm_oracle.c -- FP64 CPU restatement of the reference SKM evaluation path.
 *
 * TEST INFRASTRUCTURE ONLY (see skm_oracle.h).  Arithmetic is double except where the
 * reference's own types make a decision in float (the kernel's float members and the weight-tensor
 * support radius); expressions are evaluated as written (C11, no contraction).  The loops follow the reference's per-thread kernels one for one, including the
 * exact index boxes (truncation toward zero, clamping) because those boxes decide
 * which control points / samples contribute.  Parallelised with OpenMP over the
 * independent outer loop; every reduction is summed per thread and then combined
 * in thread order, so results are deterministic for a fixed thread count.
 */
#include "skm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* geometry: ImageBase (include/cuda/ImageBase.h:40-100) */
typedef struct {
    int    D;
    double o[3], s[3], inv[3];
    int    n[3];
    long   st[3];
} geo_t;

static void geo_set(geo_t *g, const skm_geometry *src, int D, int pad)
{
    g->D = D;
    for (int d = 0; d < 3; ++d) {
        if (d < D) {
            g->o[d] = src->origin[d];
            g->s[d] = src->spacing[d];
            g->inv[d] = 1.0 / src->spacing[d];   /* _invScale = 1/_scale (ImageBase.h:43) */
            g->n[d] = src->size[d] + pad;
        } else {
            g->o[d] = 0.0; g->s[d] = 1.0; g->inv[d] = 1.0; g->n[d] = 1;
        }
    }
    g->st[0] = 1;
    g->st[1] = g->n[0];
    g->st[2] = (long)g->n[0] * g->n[1];
}

static inline void to_global(const geo_t *g, const double *idx, double *p)
{
    for (int d = 0; d < g->D; ++d) p[d] = g->o[d] + g->s[d] * idx[d];     /* ImageBase.h:51-54 */
}

static inline void to_local(const geo_t *g, const double *p, double *idx)
{
    for (int d = 0; d < g->D; ++d) idx[d] = g->inv[d] * (p[d] - g->o[d]); /* ImageBase.h:56-59 */
}

static inline long to_index(const geo_t *g, const int *i)
{
    long r = 0;
    for (int d = 0; d < g->D; ++d) r += g->st[d] * (long)i[d];
    return r;
}

static inline int inside_idx(const geo_t *g, const int *i)
{
    for (int d = 0; d < g->D; ++d)
        if (i[d] < 0 || i[d] >= g->n[d]) return 0;
    return 1;
}

static inline long num_texels(const geo_t *g)
{
    return (long)g->n[0] * g->n[1] * g->n[2];
}

/* ImageNearest::atGlobal (ImageNearest.h:69-84): index = int(local + 0.5), truncating. */
static inline int nearest(const geo_t *g, const double *p, long *lin)
{
    double l[3];
    int i[3] = {0, 0, 0};
    to_local(g, p, l);
    for (int d = 0; d < g->D; ++d) i[d] = (int)(l[d] + 0.5);
    if (!inside_idx(g, i)) return 0;
    *lin = to_index(g, i);
    return 1;
}

static inline int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* ------------------------------------------------------------------------- */
/* small matrices: Mat.h:228-281 */
static double det_m(const double *m, int D)
{
    if (D == 2) return m[0] * m[3] - m[2] * m[1];
    return m[0] * m[4] * m[8] + m[3] * m[7] * m[2] + m[6] * m[1] * m[5]
         - m[0] * m[7] * m[5] - m[6] * m[4] * m[2] - m[3] * m[1] * m[8];
}

static void inv_m(const double *m, int D, double *r)
{
    double dt = det_m(m, D);
    if (D == 2) {
        r[0] = m[3] / dt; r[1] = -m[1] / dt;
        r[2] = -m[2] / dt; r[3] = m[0] / dt;
        return;
    }
#define M(i, j) m[(i) * 3 + (j)]
    double a[9] = {
        M(1,1)*M(2,2) - M(1,2)*M(2,1), M(0,2)*M(2,1) - M(0,1)*M(2,2), M(0,1)*M(1,2) - M(0,2)*M(1,1),
        M(1,2)*M(2,0) - M(1,0)*M(2,2), M(0,0)*M(2,2) - M(0,2)*M(2,0), M(0,2)*M(1,0) - M(0,0)*M(1,2),
        M(1,0)*M(2,1) - M(1,1)*M(2,0), M(0,1)*M(2,0) - M(0,0)*M(2,1), M(0,0)*M(1,1) - M(0,1)*M(1,0)};
#undef M
    for (int i = 0; i < 9; ++i) r[i] = a[i] / dt;
}

/* maxEigenValue (Mat.h:259-281) with Type = float */
static float max_eig_f(const float *m, int D)
{
    if (D == 2) {
        float trace = m[0] + m[3];
        float det = m[0] * m[3] - m[2] * m[1];
        float disc = trace * trace - 4.0f * det;
        return 0.5f * (trace + sqrtf(disc > 0.0f ? disc : 0.0f));
    }
    float triSq = m[1] * m[1] + m[2] * m[2] + m[5] * m[5];
    if (triSq == 0.0f) {
        float r = m[8] > m[4] ? m[8] : m[4];
        return m[0] > r ? m[0] : r;
    }
    float q = (float)(1.0 / 3.0) * (m[0] + m[4] + m[8]);
    float pSq = 2.0f * triSq + (m[0] - q) * (m[0] - q) + (m[4] - q) * (m[4] - q) + (m[8] - q) * (m[8] - q);
    float p = sqrtf(pSq * (float)(1.0 / 6.0));
    float b0 = m[0] - q, b4 = m[4] - q, b8 = m[8] - q;
    float det = b0 * b4 * b8 + m[3] * m[7] * m[2] + m[6] * m[1] * m[5] - b0 * m[7] * m[5] - m[6] * b4 * m[2] -
                m[3] * m[1] * b8;
    float r = det * (0.5f / (p * p * p));
    if (r > 1.0f) r = 1.0f;
    if (r < -1.0f) r = -1.0f;
    float phi = (float)(1.0 / 3.0) * acosf(r);
    return q + 2.0f * p * cosf(phi);
}

/* ------------------------------------------------------------------------- */
/* kernel: GKernel (include/cuda/Kernel.h) in double */
typedef struct {
    int    D;
    double sc0, sc4;
    int    use_wi, use_wt;
    double maxw;
    double maxcov[9];
    const double *wi; geo_t gwi;
    const double *wt; geo_t gwt;
} kern_t;

/* GKernel<float> keeps sigmaC0, sigmaC4, the maximum weight and the maximum-eigenvalue
 * covariance as float members (Kernel.h:37-41, typedef at :228): the oracle rounds them the same
 * way, so that support radii (and the window and box bounds truncated from them) are the
 * reference's to the last bit.  The weight image and tensors stay double (ImageNearest<ScalarType>,
 * Kernel.h:43-44). */
static void kern_init(kern_t *K, const skm_evaluator_desc *d)
{
    K->D = d->dimensions;
    K->sc0 = (float)d->sigma_c0;
    K->sc4 = (float)d->sigma_c4;
    K->use_wi = d->use_weight_image;
    K->use_wt = d->use_weight_tensor;
    K->maxw = (float)d->maximum_weight;
    for (int i = 0; i < 9; ++i) K->maxcov[i] = (float)d->maximum_eigenvalue_covariance[i];
    K->wi = d->weight_image;
    geo_set(&K->gwi, &d->weight_image_geometry, d->dimensions, 0);
    K->wt = d->weight_tensor;
    geo_set(&K->gwt, &d->weight_tensor_geometry, d->dimensions, 0);
}

/* Wendland C4 (Kernel.h:72-77) and C0 (Kernel.h:48-53) radial profiles. */
static inline double wend_c4(double r)
{
    double f = 1.0 - r;
    if (f < 0.0) f = 0.0;
    double f2 = f * f;
    return f2 * f2 * f2 * (3.0 + 18.0 * r + 35.0 * r * r) * (560.0 / 1680.0);
}

static inline double wend_c0(double r)
{
    double f = 1.0 - r;
    if (f < 0.0) f = 0.0;
    return f * f;
}

/* p-side information of evaluate(p, q, ...): sigma/covariance at p and the support
 * radius (Kernel.h:148-171). */
typedef struct {
    double sigma;
    double cov[9];
    double support;
} pinfo_t;

static void kern_sigma_at(const kern_t *K, const double *p, double *sigma)
{
    long lin;
    *sigma = nearest(&K->gwi, p, &lin) ? K->wi[lin] : 0.0;  /* default 0 (ImageNearest.h:41-45) */
}

static void kern_cov_at(const kern_t *K, const double *p, double *cov)
{
    long lin;
    int D = K->D;
    if (nearest(&K->gwt, p, &lin)) {
        memcpy(cov, K->wt + lin * D * D, sizeof(double) * D * D);
    } else {                                           /* default identity */
        for (int i = 0; i < D * D; ++i) cov[i] = 0.0;
        for (int i = 0; i < D; ++i) cov[i * D + i] = 1.0;
    }
}

static void kern_pinfo(const kern_t *K, const double *p, pinfo_t *pi)
{
    double smin = K->sc4 < K->sc0 ? K->sc4 : K->sc0;
    if (K->use_wi) {
        kern_sigma_at(K, p, &pi->sigma);
        pi->support = smin / sqrt(2.0 / (K->maxw + pi->sigma));           /* Kernel.h:163-166 */
    } else if (K->use_wt) {
        /* Kernel.h:168-171: the float member _maximumEigenvalueCovariance plus the double tensor
         * goes through Mat<float>::operator+ (Mat.h:108), so the sum, maxEigenValue, the division
         * and the square root are float */
        float s[9];
        int D = K->D;
        kern_cov_at(K, p, pi->cov);
        for (int i = 0; i < D * D; ++i) s[i] = (float)K->maxcov[i] + (float)pi->cov[i];
        pi->support = (double)((float)smin / sqrtf(2.0f / max_eig_f(s, D)));
    } else {
        pi->support = smin;                                               /* Kernel.h:158-161 */
    }
}

static inline double dist(const double *p, const double *q, int D)
{
    double s = 0.0;
    for (int d = 0; d < D; ++d) s += (p[d] - q[d]) * (p[d] - q[d]);
    return sqrt(s);
}

/* GKernel::evaluate(p, q[, sigmaP | covP]) (Kernel.h:173-186). */
static double kern_eval(const kern_t *K, const double *p, const double *q, const pinfo_t *pi)
{
    int D = K->D;
    if (K->use_wi) {
        /* evaluateNonStationary (Kernel.h:105-117; C4/C0 :55-61,79-85) */
        double sp = pi->sigma, sq;
        kern_sigma_at(K, q, &sq);
        double F = pow(fabs(sp), 0.25) * pow(fabs(sq), 0.25) * pow(fabs((sp + sq) / 2.0), -0.5);
        double sqrtQ = sqrt(2.0 / (sp + sq)) * dist(p, q, D);
        return F * wend_c4(sqrtQ / K->sc4) * F * wend_c0(sqrtQ / K->sc0);
    }
    if (K->use_wt) {
        /* evaluateAnisotropic (Kernel.h:119-131; C4/C0 :63-70,87-94) */
        double cq[9], ms[9], mi[9], v[3], vm[3];
        kern_cov_at(K, q, cq);
        for (int i = 0; i < D * D; ++i) ms[i] = (pi->cov[i] + cq[i]) * 0.5;
        inv_m(ms, D, mi);
        for (int d = 0; d < D; ++d) v[d] = p[d] - q[d];
        for (int i = 0; i < D; ++i) {          /* Vec*Mat (Mat.h:205-215) */
            double s = 0.0;
            for (int k = 0; k < D; ++k) s += v[k] * mi[k * D + i];
            vm[i] = s;
        }
        double Q = 0.0;
        for (int d = 0; d < D; ++d) Q += vm[d] * v[d];
        double sqrtQ = sqrt(Q);
        double F = pow(det_m(pi->cov, D), 0.25) * pow(det_m(cq, D), 0.25) * pow(det_m(ms, D), -0.5);
        return F * wend_c4(sqrtQ / K->sc4) * F * wend_c0(sqrtQ / K->sc0);
    }
    double r = dist(p, q, D);                  /* evaluateStationary, C4*C0 (Kernel.h:96-103; D8) */
    return wend_c4(r / K->sc4) * wend_c0(r / K->sc0);
}

/* ------------------------------------------------------------------------- */
/* cubic B-spline image (include/cuda/BsplineImage.h) */

static double bs_initial_causal(const double *c, int len, long st, double z)
{
    double zn = z, iz = 1.0 / z;
    double z2n = pow(z, (double)(len - 1));
    double sum = c[0] + z2n * c[(len - 1) * st];
    z2n *= z2n * iz;
    for (int n = 1; n < len - 1; n++) {
        sum += (zn + z2n) * c[n * st];
        zn *= z;
        z2n *= iz;
    }
    return sum / (1.0 - zn * zn);                                     /* BsplineImage.h:42-55 */
}

static double bs_initial_anticausal(const double *c, int len, long st, double z)
{
    return (z / (z * z - 1.0)) * (z * c[(len - 2) * st] + c[(len - 1) * st]);  /* :37-40 */
}

static void bs_convert(double *c, int len, long st, double z)
{
    double lambda = 2.0 - z - 1.0 / z;                                /* :57-70 */
    for (int n = 0; n < len; n++) c[n * st] *= lambda;
    c[0] = bs_initial_causal(c, len, st, z);
    for (int n = 1; n < len; n++) c[n * st] += z * c[(n - 1) * st];
    c[(len - 1) * st] = bs_initial_anticausal(c, len, st, z);
    for (int n = len - 2; n >= 0; n--) c[n * st] = z * (c[(n + 1) * st] - c[n * st]);
}

void ora_bspline_coefficients(int D, const int32_t *size, const double *image, double *coeffs)
{
    int X = size[0], Y = size[1], Z = D == 3 ? size[2] : 1;
    long n = (long)X * Y * Z;
    double *tmp = (double *)malloc(sizeof(double) * n);
    memcpy(tmp, image, sizeof(double) * n);
    const double pole = sqrt(3.0) - 2.0;
    if (D == 3) {                                                      /* :182-195 */
        for (int y = 0; y < Y; ++y)
            for (int x = 0; x < X; x++)
                bs_convert(tmp + x + (long)y * X, Z, (long)X * Y, pole);
        for (int z = 0; z < Z; ++z)
            for (int x = 0; x < X; x++)
                bs_convert(tmp + x + (long)z * X * Y, Y, X, pole);
        for (int z = 0; z < Z; ++z)
            for (int y = 0; y < Y; ++y)
                bs_convert(tmp + (long)X * (y + (long)z * Y), X, 1, pole);
    } else {                                                           /* :174-180 */
        for (int y = 0; y < Y; y++) bs_convert(tmp + (long)y * X, X, 1, pole);
        for (int x = 0; x < X; x++) bs_convert(tmp + x, Y, X, pole);
    }
    /* mirrorCoeffBorders (:72-108): padded index x maps to W - |W - |x-1||. */
    int PX = X + 3, PY = Y + 3, PZ = D == 3 ? Z + 3 : 1;
    int W = X - 1, H = Y - 1, Dp = Z - 1;
    for (int z = 0; z < PZ; ++z)
        for (int y = 0; y < PY; ++y)
            for (int x = 0; x < PX; ++x) {
                int xi = W - abs(W - abs(x - 1));
                int yi = H - abs(H - abs(y - 1));
                int zi = D == 3 ? Dp - abs(Dp - abs(z - 1)) : 0;
                coeffs[x + (long)PX * (y + (long)z * PY)] = tmp[xi + (long)X * (yi + (long)zi * Y)];
            }
    free(tmp);
}

/* insideLocal (BsplineImage.h:285-291) on the padded geometry. */
static inline int bs_inside_local(const geo_t *gp, const double *l)
{
    for (int d = 0; d < gp->D; ++d)
        if (l[d] < -0.5 || l[d] + 3.5 >= gp->n[d]) return 0;
    return 1;
}

/* derivsLocal + reduceWithDeriv (BsplineImage.h:110-144, 247-265). */
static void bs_derivs(const double *c, const geo_t *gp, const double *l, double *val, double *grad)
{
    int D = gp->D;
    int ii[3] = {0, 0, 0};
    double W[4][3], dW[4][3];
    for (int d = 0; d < D; ++d) {
        ii[d] = (int)l[d];                        /* VecI(idx): truncation toward zero */
        double w = l[d] - ii[d];
        W[3][d] = (1.0 / 6.0) * w * w * w;
        W[0][d] = (1.0 / 6.0) + 0.5 * w * (w - 1.0) - W[3][d];
        W[2][d] = w + W[0][d] - 2.0 * W[3][d];
        W[1][d] = 1.0 - W[0][d] - W[2][d] - W[3][d];
        dW[3][d] = (3.0 / 6.0) * w * w;
        dW[0][d] = w - 0.5 - dW[3][d];
        dW[2][d] = 1.0 + dW[0][d] - 2.0 * dW[3][d];
        dW[1][d] = -dW[0][d] - dW[2][d] - dW[3][d];
    }
    if (D == 3) {
        double comb[4] = {0, 0, 0, 0};
        for (int z = 0; z < 4; ++z) {
            double wz[4] = {0, 0, 0, 0};
            for (int y = 0; y < 4; ++y) {
                double wy[4] = {0, 0, 0, 0};
                const double *row = c + (ii[0]) + (ii[1] + y) * gp->st[1] + (ii[2] + z) * gp->st[2];
                for (int x = 0; x < 4; ++x) {
                    double cv = row[x];
                    wy[0] += dW[x][0] * cv; wy[1] += W[x][0] * cv;
                    wy[2] += W[x][0] * cv;  wy[3] += W[x][0] * cv;
                }
                wz[0] += W[y][1] * wy[0]; wz[1] += dW[y][1] * wy[1];
                wz[2] += W[y][1] * wy[2]; wz[3] += W[y][1] * wy[3];
            }
            comb[0] += W[z][2] * wz[0]; comb[1] += W[z][2] * wz[1];
            comb[2] += dW[z][2] * wz[2]; comb[3] += W[z][2] * wz[3];
        }
        *val = comb[3];
        for (int d = 0; d < 3; ++d) grad[d] = comb[d] * gp->inv[d];
    } else {
        double comb[3] = {0, 0, 0};
        for (int y = 0; y < 4; ++y) {
            double wy[3] = {0, 0, 0};
            const double *row = c + ii[0] + (ii[1] + y) * gp->st[1];
            for (int x = 0; x < 4; ++x) {
                double cv = row[x];
                wy[0] += dW[x][0] * cv; wy[1] += W[x][0] * cv; wy[2] += W[x][0] * cv;
            }
            comb[0] += W[y][1] * wy[0]; comb[1] += dW[y][1] * wy[1]; comb[2] += W[y][1] * wy[2];
        }
        *val = comb[2];
        for (int d = 0; d < 2; ++d) grad[d] = comb[d] * gp->inv[d];
    }
}

void ora_bspline_sample(int D, const double *coeffs, const skm_geometry *g, int64_t n,
                        const double *pts, int32_t *inside, double *vals, double *grads)
{
    geo_t gp;
    geo_set(&gp, g, D, 3);
    for (int64_t i = 0; i < n; ++i) {
        double l[3], gr[3] = {0, 0, 0}, v = 0.0;
        to_local(&gp, pts + i * D, l);
        inside[i] = bs_inside_local(&gp, l);
        if (inside[i]) bs_derivs(coeffs, &gp, l, &v, gr);
        vals[i] = v;
        for (int d = 0; d < D; ++d) grads[i * D + d] = gr[d];
    }
}

/* ------------------------------------------------------------------------- */
/* UniformRng (include/cuda/UniformRng.h:28-55) */
uint32_t ora_pcg32_next(uint64_t *state)
{
    uint64_t old = *state;
    *state = old * 6364136223846793005ULL + (0ULL | 1ULL);   /* _sequence = 0 */
    uint32_t xorshifted = (uint32_t)(((old >> 18u) ^ old) >> 27u);
    uint32_t rot = (uint32_t)(old >> 59u);
    return (xorshifted >> rot) | (xorshifted << ((uint32_t)(-(int32_t)rot) & 31));
}

void ora_pcg32_shifts(uint64_t *state, int64_t n, int D, int sub, int32_t *shifts)
{
    /* GpuEvaluator.cu:111-112: VecI(nextV<D>() * subsample); nextF = nextI/double(UINT_MAX) */
    for (int64_t i = 0; i < n; ++i)
        for (int d = 0; d < D; ++d) {
            double f = (double)ora_pcg32_next(state) / (double)4294967295u;
            shifts[i * D + d] = (int32_t)(f * (double)sub);
        }
}

/* ------------------------------------------------------------------------- */
/* evaluator context */
struct ora_ctx {
    int D, sub, nbh, nparams;
    kern_t K;
    geo_t fixed, moving_pad, cp, cpw, ss;   /* ss: subsampled grid, geometry unused */
    const double *fixed_data, *coeffs;
    double rkhs, rd, rd_scaling, pg, pg_scaling;
    uint64_t rng;
    int evaluated_once;
    int32_t *shifts;
    long nss;
};

static int g_threads = 0;
void ora_set_num_threads(int n) { g_threads = n; }

ora_ctx *ora_create(const skm_evaluator_desc *d)
{
    ora_ctx *c = (ora_ctx *)calloc(1, sizeof(ora_ctx));
    int D = d->dimensions;
    c->D = D;
    c->sub = d->subsample;
    c->nbh = d->subsample_neighborhood;
    c->nparams = d->num_parameters;
    kern_init(&c->K, d);
    geo_set(&c->fixed, &d->fixed_geometry, D, 0);
    geo_set(&c->moving_pad, &d->moving_geometry, D, 3);
    geo_set(&c->cp, &d->cp_geometry, D, 0);
    geo_set(&c->cpw, &d->cpw_geometry, D, 0);
    c->ss = c->fixed;
    for (int k = 0; k < D; ++k) c->ss.n[k] = c->fixed.n[k] / c->sub;   /* size/subsample (cu:44) */
    c->ss.st[1] = c->ss.n[0];
    c->ss.st[2] = (long)c->ss.n[0] * c->ss.n[1];
    c->nss = num_texels(&c->ss);
    c->fixed_data = d->fixed_image;
    c->coeffs = d->moving_coefficients;
    c->rd_scaling = 1.0;
    c->pg_scaling = 1.0;
    c->rng = 0xBA5EBA11DEADBEEFULL;
    if (c->sub > 1) c->shifts = (int32_t *)calloc((size_t)c->nss * D, sizeof(int32_t));
    return c;
}

void ora_destroy(ora_ctx *c)
{
    if (!c) return;
    free(c->shifts);
    free(c);
}

void ora_set_regularizers(ora_ctx *c, double rkhs, double rd, double rd_scaling, double pg, double pg_scaling)
{
    c->rkhs = rkhs; c->rd = rd; c->rd_scaling = rd_scaling; c->pg = pg; c->pg_scaling = pg_scaling;
}

const int32_t *ora_last_shifts(const ora_ctx *c) { return c->shifts; }
int64_t ora_num_subsampled(const ora_ctx *c) { return c->nss; }

/* u(p) += sum over the cp box of w_i k(p, c_i) alpha_i (DisplacementField.cu:53-72,
 * MSE.cu:192-211).  `swap` evaluates k(c_i, p) with p-side info instead (used by the
 * 3-D LCC derivative, LCC.cu:429-442). */
static void transform_add(const ora_ctx *c, const double *p, const pinfo_t *pi,
                          const double *cp, const double *cpw, double *u, int swap)
{
    int D = c->D;
    double ip[3];
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    to_local(&c->cp, p, ip);
    for (int d = 0; d < D; ++d) {
        double sh = pi->support / c->cp.s[d];
        lo[d] = clampi((int)(ip[d] - sh + 1.0), 0, c->cp.n[d] - 1);
        hi[d] = clampi((int)(ip[d] + sh), 0, c->cp.n[d] - 1);
    }
    for (int zi = lo[2]; zi <= hi[2]; ++zi)
        for (int yi = lo[1]; yi <= hi[1]; ++yi)
            for (int xi = lo[0]; xi <= hi[0]; ++xi) {
                int ii[3] = {xi, yi, zi};
                double fi[3] = {xi, yi, zi}, q[3];
                to_global(&c->cp, fi, q);
                double k = swap ? kern_eval(&c->K, q, p, pi) : kern_eval(&c->K, p, q, pi);
                long i = to_index(&c->cp, ii);
                double wk = cpw[i] * k;
                for (int d = 0; d < D; ++d) u[d] += wk * cp[i * D + d];
            }
}

static void df_add(const ora_ctx *c, const skm_field *df, const geo_t *gdf, const double *p, double *u)
{
    long lin;
    if (df && df->data && nearest(gdf, p, &lin))
        for (int d = 0; d < c->D; ++d) u[d] += df->data[lin * c->D + d];
}

int ora_displacement_field(ora_ctx *c, const double *cp, const double *cpw, const skm_field *df, double *dst)
{
    int D = c->D;
    geo_t gdf;
    if (df && df->data) geo_set(&gdf, &df->geometry, D, 0);
    long N = num_texels(&c->fixed);
#pragma omp parallel for schedule(dynamic, 64) num_threads(g_threads > 0 ? g_threads : omp_get_max_threads())
    for (long t = 0; t < N; ++t) {
        int i[3] = {(int)(t % c->fixed.n[0]), (int)((t / c->fixed.n[0]) % c->fixed.n[1]),
                    (int)(t / ((long)c->fixed.n[0] * c->fixed.n[1]))};
        double fi[3] = {i[0], i[1], i[2]}, p[3], u[3] = {0, 0, 0};
        pinfo_t pi;
        to_global(&c->fixed, fi, p);
        df_add(c, df, &gdf, p, u);
        kern_pinfo(&c->K, p, &pi);
        transform_add(c, p, &pi, cp, cpw, u, 0);
        for (int d = 0; d < D; ++d) dst[t * D + d] = u[d];
    }
    return 0;
}

/* sample position of subsampled texel t (MSE.cu:171-174) */
static void sample_pos(const ora_ctx *c, long t, int *sp)
{
    int cell[3] = {(int)(t % c->ss.n[0]), (int)((t / c->ss.n[0]) % c->ss.n[1]),
                   (int)(t / ((long)c->ss.n[0] * c->ss.n[1]))};
    for (int d = 0; d < 3; ++d) sp[d] = cell[d];
    if (c->sub != 1)
        for (int d = 0; d < c->D; ++d) sp[d] = cell[d] * c->sub + c->shifts[t * c->D + d];
}

/* moving point of fixed-grid point p: p + DF(p) + u(p) */
static void moving_point(const ora_ctx *c, const double *cp, const double *cpw, const skm_field *df,
                         const geo_t *gdf, const double *p, double *mp, int swap)
{
    pinfo_t pi;
    for (int d = 0; d < c->D; ++d) mp[d] = p[d];
    df_add(c, df, gdf, p, mp);
    kern_pinfo(&c->K, p, &pi);
    transform_add(c, p, &pi, cp, cpw, mp, swap);
}

static double neighborhood_weight(const double *p, const double *q, float support, int D)
{
    double r = pow(dist(p, q, D) / (double)support, 10.0);   /* LCC.cu:28-35 */
    double f = 1.0 - r;
    if (f < 0.0) f = 0.0;
    return f * f;
}

typedef struct {
    double *m, *f, *grad;   /* per sample */
    int *inside;
    double *cc;
} samples_t;

/* LCC window statistics around sample point p (LCC.cu:94-191), value only. */
static double lcc_value_at(const ora_ctx *c, const double *cp, const double *cpw, const skm_field *df,
                           const geo_t *gdf, const double *p, double support)
{
    int D = c->D;
    double fi[3];
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    to_local(&c->fixed, p, fi);
    for (int d = 0; d < D; ++d) {
        double sh = support / c->fixed.s[d];
        lo[d] = clampi((int)(fi[d] - sh + 1.0), 0, c->fixed.n[d] - 1);
        hi[d] = clampi((int)(fi[d] + sh), 0, c->fixed.n[d] - 1);
    }
    double sf = 0, sm = 0, sff = 0, smm = 0, sfm = 0;
    int n = 0;
    for (int z = lo[2]; z <= hi[2]; z += c->nbh)
        for (int y = lo[1]; y <= hi[1]; y += c->nbh)
            for (int x = lo[0]; x <= hi[0]; x += c->nbh) {
                int ni[3] = {x, y, z};
                double nf[3] = {x, y, z}, q[3], mp[3], ml[3];
                pinfo_t pn;
                to_global(&c->fixed, nf, q);
                for (int d = 0; d < D; ++d) mp[d] = q[d];
                df_add(c, df, gdf, q, mp);
                kern_pinfo(&c->K, q, &pn);
                transform_add(c, q, &pn, cp, cpw, mp, 0);
                double kw = neighborhood_weight(p, q, (float)pn.support, D);
                to_local(&c->moving_pad, mp, ml);
                if (kw > 0.0 && bs_inside_local(&c->moving_pad, ml)) {
                    double mv, g[3];
                    bs_derivs(c->coeffs, &c->moving_pad, ml, &mv, g);
                    mv *= kw;
                    double fv = kw * c->fixed_data[to_index(&c->fixed, ni)];
                    sf += fv; sm += mv; sff += fv * fv; smm += mv * mv; sfm += fv * mv;
                    n++;
                }
            }
    double cc = 0.0;
    if (n > 0) {
        double msf = sf / n, msm = sm / n;
        double d1 = sff - 2.0 * msf * sf + n * msf * msf;
        double d2 = smm - 2.0 * msm * sm + n * msm * msm;
        if (d1 > 0 && d2 > 0) {
            cc = sfm - msm * sf - msf * sm + n * msf * msm;
            cc = -cc * cc / (d1 * d2);
        }
    }
    return cc;
}

static void draw_shifts(ora_ctx *c, int do_resampling)
{
    if (c->sub > 1 && (!c->evaluated_once || do_resampling)) {   /* GpuEvaluator.cu:107-115 */
        ora_pcg32_shifts(&c->rng, c->nss, c->D, c->sub, c->shifts);
        c->evaluated_once = 1;
    }
}

/* derivative box over samples for control point at fixed-local ip (MSE.cu:255-263,
 * NCC.cu:138-146 for 3-D MSE/NCC; MSE.cu:273-280 2-D, LCC.cu:236-244 otherwise). */
static void deriv_box(const ora_ctx *c, int metric, const double *ip, double support, int *lo, int *hi)
{
    int D = c->D;
    int wide = (D == 3 && metric != SKM_LCC);
    lo[2] = hi[2] = 0;
    for (int d = 0; d < D; ++d) {
        double sh = support / c->fixed.s[d];
        if (c->sub != 1) {
            double fs = (double)(float)c->sub;
            if (wide) {
                lo[d] = (int)((ip[d] - sh) / fs);
                hi[d] = (int)((ip[d] + sh) / fs + 1.0);
            } else {
                lo[d] = (int)((ip[d] - sh) / fs + 1.0);
                hi[d] = (int)((ip[d] + sh) / fs);
            }
            lo[d] = clampi(lo[d], 0, c->ss.n[d] - 1);
            hi[d] = clampi(hi[d], 0, c->ss.n[d] - 1);
        } else {
            if (wide) {
                lo[d] = (int)(ip[d] - sh);
                hi[d] = (int)(ip[d] + sh + 1.0);
            } else {
                lo[d] = (int)(ip[d] - sh + 1.0);
                hi[d] = (int)(ip[d] + sh);
            }
            lo[d] = clampi(lo[d], 0, c->fixed.n[d] - 1);
            hi[d] = clampi(hi[d], 0, c->fixed.n[d] - 1);
        }
    }
}

static void sample_point_of_cell(const ora_ctx *c, const int *cell, long idx, double *pt)
{
    double f[3] = {0, 0, 0};
    for (int d = 0; d < c->D; ++d)
        f[d] = c->sub != 1 ? (double)(cell[d] * c->sub + c->shifts[idx * c->D + d]) : (double)cell[d];
    to_global(&c->fixed, f, pt);
}

/* LCC derivative contribution of one control point (LCC.cu:206-530 / 696-962). */
static void lcc_derivative_cp(const ora_ctx *c, const double *cp, const double *cpw, const skm_field *df,
                              const geo_t *gdf, const int *j, double *der)
{
    int D = c->D;
    double jf[3] = {j[0], j[1], j[2]}, gp[3], ip[3];
    pinfo_t pj;
    to_global(&c->cp, jf, gp);
    kern_pinfo(&c->K, gp, &pj);
    to_local(&c->fixed, gp, ip);
    int lo[3], hi[3];
    deriv_box(c, SKM_LCC, ip, pj.support, lo, hi);
    for (int d = 0; d < 3; ++d) der[d] = 0.0;
    for (int zi = lo[2]; zi <= hi[2]; ++zi)
        for (int yi = lo[1]; yi <= hi[1]; ++yi)
            for (int xi = lo[0]; xi <= hi[0]; ++xi) {
                int cell[3] = {xi, yi, zi};
                long idx = c->sub != 1 ? xi + (long)c->ss.n[0] * (yi + (long)c->ss.n[1] * zi)
                                       : to_index(&c->fixed, cell);
                double pt[3], fl[3];
                pinfo_t ps;
                sample_point_of_cell(c, cell, idx, pt);
                kern_pinfo(&c->K, pt, &ps);
                to_local(&c->fixed, pt, fl);
                int flo[3] = {0, 0, 0}, fhi[3] = {0, 0, 0};
                for (int d = 0; d < D; ++d) {
                    double sh = ps.support / c->fixed.s[d];
                    flo[d] = clampi((int)(fl[d] - sh + 1.0), 0, c->fixed.n[d] - 1);
                    fhi[d] = clampi((int)(fl[d] + sh), 0, c->fixed.n[d] - 1);
                }
                double sf = 0, sm = 0, sff = 0, smm = 0, sfm = 0;
                double mkcka[3] = {0, 0, 0}, mkcmkcka[3] = {0, 0, 0}, fkcmka[3] = {0, 0, 0};
                int n = 0;
                for (int z = flo[2]; z <= fhi[2]; z += c->nbh)
                    for (int y = flo[1]; y <= fhi[1]; y += c->nbh)
                        for (int x = flo[0]; x <= fhi[0]; x += c->nbh) {
                            int ni[3] = {x, y, z};
                            double nf[3] = {x, y, z}, q[3], mp[3], ml[3];
                            pinfo_t pn;
                            to_global(&c->fixed, nf, q);
                            for (int d = 0; d < D; ++d) mp[d] = q[d];
                            df_add(c, df, gdf, q, mp);
                            kern_pinfo(&c->K, q, &pn);
                            /* 3-D evaluates k(cp_i, n) with the neighbour's sigma (LCC.cu:429-442);
                             * 2-D evaluates k(n, cp_i) (LCC.cu:876-889). */
                            transform_add(c, q, &pn, cp, cpw, mp, D == 3);
                            double kw = neighborhood_weight(pt, q, (float)pn.support, D);
                            double ka = kern_eval(&c->K, gp, q, &pn);   /* neighbour's p-side info */
                            to_local(&c->moving_pad, mp, ml);
                            if (kw > 0.0 && bs_inside_local(&c->moving_pad, ml)) {
                                double mv, g[3] = {0, 0, 0};
                                bs_derivs(c->coeffs, &c->moving_pad, ml, &mv, g);
                                mv *= kw;
                                double fv = kw * c->fixed_data[to_index(&c->fixed, ni)];
                                sf += fv; sm += mv; sff += fv * fv; smm += mv * mv; sfm += fv * mv;
                                for (int d = 0; d < D; ++d) {
                                    double gk = g[d] * kw;
                                    mkcmkcka[d] += mv * gk * ka;
                                    mkcka[d] += gk * ka;
                                    fkcmka[d] += fv * gk * ka;
                                }
                                n++;
                            }
                        }
                if (n > 0) {
                    double msf = sf / n, msm = sm / n;
                    double d1 = sff - 2.0 * msf * sf + n * msf * msf;
                    double u = d1 * (smm - 2.0 * msm * sm + n * msm * msm);
                    double v = sfm - msm * sf - msf * sm + n * msf * msm;
                    double vd[3], ud[3];
                    for (int d = 0; d < D; ++d) {
                        vd[d] = 2.0 * v * (fkcmka[d] - msf * mkcka[d]);
                        ud[d] = 2.0 * d1 * (mkcmkcka[d] - msm * mkcka[d]);
                    }
                    v = v * v;
                    if (fabs(u) > 1e-16)
                        for (int d = 0; d < D; ++d) der[d] += -(vd[d] * u - ud[d] * v) / (u * u);
                }
            }
}

/* Regularizer kernels (GpuEvaluatorRegularizers.cu): kind 0 RKHS, 1 RD, 2 PG. */
static void regularizer(const ora_ctx *c, int kind, double weight, double scale,
                        const double *cp, const double *cpw, double *deriv, double *value_out)
{
    int D = c->D;
    long C = num_texels(&c->cp);
    int nt = g_threads > 0 ? g_threads : omp_get_max_threads();
    double *partial = (double *)calloc(nt, sizeof(double));
#pragma omp parallel num_threads(nt)
    {
        int tid = omp_get_thread_num();
        double acc = 0.0;
#pragma omp for schedule(static)
        for (long t = 0; t < C; ++t) {
            int j[3] = {(int)(t % c->cp.n[0]), (int)((t / c->cp.n[0]) % c->cp.n[1]),
                        (int)(t / ((long)c->cp.n[0] * c->cp.n[1]))};
            double jf[3] = {j[0], j[1], j[2]}, gp[3];
            pinfo_t pj;
            to_global(&c->cp, jf, gp);
            long jl = to_index(&c->cp, j);
            double wj = cpw[jl];
            const double *cj = cp + jl * D;
            kern_pinfo(&c->K, gp, &pj);
            int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
            for (int d = 0; d < D; ++d) {
                double sh = pj.support / c->cp.s[d];
                lo[d] = clampi((int)(jf[d] - sh + 1.0), 0, c->cp.n[d] - 1);
                hi[d] = clampi((int)(jf[d] + sh), 0, c->cp.n[d] - 1);
            }
            double value = 0.0, der[3] = {0, 0, 0};
            for (int zi = lo[2]; zi <= hi[2]; ++zi)
                for (int yi = lo[1]; yi <= hi[1]; ++yi)
                    for (int xi = lo[0]; xi <= hi[0]; ++xi) {
                        int ii[3] = {xi, yi, zi};
                        double fi[3] = {xi, yi, zi}, q[3];
                        to_global(&c->cp, fi, q);
                        const double *ci = cp + to_index(&c->cp, ii) * D;
                        double k = kern_eval(&c->K, gp, q, &pj);
                        if (kind == 0) {                       /* Regularizers.cu:68-73 */
                            double dot = 0.0;
                            for (int d = 0; d < D; ++d) dot += k * wj * cj[d] * ci[d];
                            value += dot;
                            for (int d = 0; d < D; ++d) der[d] += 2.0 * ci[d] * k * wj;
                        } else if (kind == 1) {                /* Regularizers.cu:141-144 */
                            double l2 = 0.0;
                            for (int d = 0; d < D; ++d) l2 += (cj[d] - ci[d]) * (cj[d] - ci[d]);
                            value += l2 * k * wj;
                            for (int d = 0; d < D; ++d) der[d] += 4.0 * (cj[d] - ci[d]) * k * wj;
                        } else if (D == 3) {                   /* Regularizers.cu:218-237 */
                            double cr[3] = {ci[1] * cj[2] - ci[2] * cj[1], ci[2] * cj[0] - ci[0] * cj[2],
                                            ci[0] * cj[1] - ci[1] * cj[0]};
                            double n2 = cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2];
                            value += k * wj * scale * scale / 2.0 * log(1.0 + n2 / scale);
                            double den = 2.0 * (n2 / scale + 1.0), dev[3], dp;
                            dp = 2.0 * ci[2] * (ci[2] * cj[0] - ci[0] * cj[2]) - 2.0 * ci[1] * (ci[0] * cj[1] - ci[1] * cj[0]);
                            dev[0] = scale * dp / den;
                            dp = 2.0 * ci[0] * (ci[0] * cj[1] - ci[1] * cj[0]) - 2.0 * ci[2] * (ci[1] * cj[2] - ci[2] * cj[1]);
                            dev[1] = scale * dp / den;
                            dp = 2.0 * ci[1] * (ci[1] * cj[2] - ci[2] * cj[1]) - 2.0 * ci[0] * (ci[2] * cj[0] - ci[0] * cj[2]);
                            dev[2] = scale * dp / den;
                            for (int d = 0; d < 3; ++d) der[d] += 2.0 * k * wj * dev[d];
                        } else {                               /* Regularizers.cu:447-459 */
                            double val = ci[0] * cj[1] - ci[1] * cj[0];
                            double v2 = val * val;
                            value += k * wj * scale * scale / 2.0 * log(1.0 + v2 / scale);
                            double factor = v2 / scale + 1.0;
                            double dev0 = -scale * ci[1] * val / factor;
                            double dev1 = scale * ci[0] * val / factor;
                            der[0] += 2.0 * k * wj * dev0;
                            der[1] += 2.0 * k * wj * dev1;
                        }
                    }
            acc += value;
            if (deriv)
                for (int d = 0; d < D; ++d) deriv[jl + d * C] += der[d] * weight;
        }
        partial[tid] = acc;
    }
    double s = 0.0;
    for (int i = 0; i < nt; ++i) s += partial[i];
    free(partial);
    *value_out = s;
}

int ora_evaluate(ora_ctx *c, int metric, const double *cp, const double *cpw, const skm_field *df,
                 int do_resampling, double *derivatives, skm_result *out)
{
    int D = c->D;
    geo_t gdf;
    if (df && df->data) geo_set(&gdf, &df->geometry, D, 0);
    draw_shifts(c, do_resampling);
    long Ns = c->nss;
    long C = num_texels(&c->cp);
    double *m = (double *)calloc(Ns, sizeof(double));
    double *f = (double *)calloc(Ns, sizeof(double));
    double *cc = (double *)calloc(Ns, sizeof(double));
    double *grad = (double *)calloc(Ns * D, sizeof(double));
    int *ins = (int *)calloc(Ns, sizeof(int));
    int oob = 0;
    int nt = g_threads > 0 ? g_threads : omp_get_max_threads();

    /* value pass: one sample per subsampled texel (MSE.cu:29-95, NCC.cu:37-109, LCC.cu:38-204) */
#pragma omp parallel for schedule(dynamic, 64) num_threads(nt) reduction(| : oob)
    for (long t = 0; t < Ns; ++t) {
        int sp[3];
        sample_pos(c, t, sp);
        if (!inside_idx(&c->fixed, sp)) { oob |= 1; continue; }
        double fi[3] = {sp[0], sp[1], sp[2]}, p[3], mp[3], ml[3];
        to_global(&c->fixed, fi, p);
        moving_point(c, cp, cpw, df, &gdf, p, mp, 0);
        to_local(&c->moving_pad, mp, ml);
        if (bs_inside_local(&c->moving_pad, ml)) {
            double v, g[3] = {0, 0, 0};
            bs_derivs(c->coeffs, &c->moving_pad, ml, &v, g);
            m[t] = v;
            f[t] = c->fixed_data[to_index(&c->fixed, sp)];
            for (int d = 0; d < D; ++d) grad[t * D + d] = g[d];
            ins[t] = 1;
        }
        if (metric == SKM_LCC) {
            pinfo_t pi;
            kern_pinfo(&c->K, p, &pi);
            cc[t] = lcc_value_at(c, cp, cpw, df, &gdf, p, pi.support);
        }
    }

    /* host-side sums of the reference (GpuEvaluator.cu:460-570), per thread then combined */
    double s_d2 = 0, sf = 0, sm = 0, sff = 0, smm = 0, sfm = 0, scc = 0;
    long cnt = 0;
    for (long t = 0; t < Ns; ++t) {
        if (ins[t]) {
            double diff = m[t] - f[t];
            s_d2 += diff * diff;
            sf += f[t]; sm += m[t]; sff += f[t] * f[t]; smm += m[t] * m[t]; sfm += f[t] * m[t];
        }
        scc += cc[t];
        cnt += ins[t];
    }
    double measure = 0.0, denom = 1.0, mean_f = 0, mean_m = 0;
    if (metric == SKM_MSE) {
        measure = s_d2 / (double)cnt;
    } else if (metric == SKM_NCC) {
        sff -= sf * sf / cnt;
        smm -= sm * sm / cnt;
        sfm -= sf * sm / cnt;
        denom = -1.0 * sqrt(sff * smm);
        measure = denom != 0 ? sfm / denom : 0.0;
        mean_f = sf / cnt;
        mean_m = sm / cnt;
    } else {
        measure = scc / (double)cnt;
    }

    if (derivatives) {
        for (long i = 0; i < (long)c->nparams; ++i) derivatives[i] = 0.0;
#pragma omp parallel for schedule(dynamic, 4) num_threads(nt)
        for (long t = 0; t < C; ++t) {
            int j[3] = {(int)(t % c->cp.n[0]), (int)((t / c->cp.n[0]) % c->cp.n[1]),
                        (int)(t / ((long)c->cp.n[0] * c->cp.n[1]))};
            double der[3] = {0, 0, 0};
            long jl = to_index(&c->cp, j);
            if (metric == SKM_LCC) {
                lcc_derivative_cp(c, cp, cpw, df, &gdf, j, der);
                for (int d = 0; d < D; ++d) derivatives[jl + d * C] = der[d] / (double)cnt;
                continue;
            }
            double jf[3] = {j[0], j[1], j[2]}, gp[3], ip[3];
            pinfo_t pj;
            to_global(&c->cp, jf, gp);
            double wi = cpw[to_index(&c->cpw, j)];
            kern_pinfo(&c->K, gp, &pj);
            to_local(&c->fixed, gp, ip);
            int lo[3], hi[3];
            deriv_box(c, metric, ip, pj.support, lo, hi);
            double dF[3] = {0, 0, 0}, dM[3] = {0, 0, 0};
            for (int zi = lo[2]; zi <= hi[2]; ++zi)
                for (int yi = lo[1]; yi <= hi[1]; ++yi)
                    for (int xi = lo[0]; xi <= hi[0]; ++xi) {
                        int cell[3] = {xi, yi, zi};
                        long idx = c->sub != 1 ? xi + (long)c->ss.n[0] * (yi + (long)c->ss.n[1] * zi)
                                               : to_index(&c->fixed, cell);
                        if (!ins[idx]) continue;            /* zero gradient: no contribution */
                        double pt[3];
                        sample_point_of_cell(c, cell, idx, pt);
                        double k = kern_eval(&c->K, gp, pt, &pj);
                        for (int d = 0; d < D; ++d) {
                            double g = grad[idx * D + d];
                            if (metric == SKM_MSE) {
                                der[d] += 2.0 * (m[idx] - f[idx]) * wi * k * g;      /* MSE.cu:291 */
                            } else {
                                double diffl = wi * k * g;                           /* NCC.cu:177-179 */
                                dF[d] += f[idx] * diffl - diffl * mean_f;
                                dM[d] += m[idx] * diffl - diffl * mean_m;
                            }
                        }
                    }
            for (int d = 0; d < D; ++d) {
                double v;
                if (metric == SKM_MSE) v = der[d] / (double)cnt;                      /* cu:599-603 */
                else v = denom != 0 ? (dF[d] - (sfm / smm) * dM[d]) / denom : 0.0;     /* cu:624-633 */
                derivatives[jl + d * C] = v;
            }
        }
    }

    double vr = 0, vd = 0, vp = 0;
    if (c->rkhs > 0) regularizer(c, 0, c->rkhs, 1.0, cp, cpw, derivatives, &vr);
    if (c->rd > 0) regularizer(c, 1, c->rd, c->rd_scaling, cp, cpw, derivatives, &vd);
    if (c->pg > 0) regularizer(c, 2, c->pg, c->pg_scaling, cp, cpw, derivatives, &vp);

    out->measure = measure;
    out->reg_value_rkhs = vr;
    out->reg_value_rd = vd;
    out->reg_value_pg = vp;
    out->num_pixels_counted = (uint32_t)cnt;
    free(m); free(f); free(cc); free(grad); free(ins);
    return oob ? -1 : 0;
}

/* ------------------------------------------------------------------------- */
/* metric (itkRegularizedImageToImageMetricv4.hxx:316-573) */
int ora_metric_evaluate(ora_ctx *c, const skm_metric_desc *mt, const double *params, const double *cpw,
                        const skm_field *df, double *derivative, skm_metric_values *out)
{
    int D = c->D;
    long C = num_texels(&c->cp);
    long P = C * D;
    double *cp = (double *)malloc(sizeof(double) * P);
    for (long i = 0; i < C; ++i)
        for (int d = 0; d < D; ++d) cp[i * D + d] = params[i + d * C];   /* flat layout (Adapter.hxx:202-236) */
    /* the metric only pushes positive weights (hxx:371-380) */
    ora_set_regularizers(c, mt->reg_rkhs > 0 ? mt->reg_rkhs : 0.0, mt->reg_rd > 0 ? mt->reg_rd : 0.0,
                         mt->reg_rd_scaling, mt->reg_pg > 0 ? mt->reg_pg : 0.0, mt->reg_pg_scaling);
    skm_result r;
    double *der = derivative ? derivative : (double *)calloc(P, sizeof(double));
    int rc = ora_evaluate(c, mt->metric, cp, cpw, df, mt->do_resampling, der, &r);
    double l1 = 0, l21 = 0, l2 = 0;
    if (mt->reg_l1 > 0) {                                              /* hxx:431-467 */
        double w = mt->reg_l1;
        for (long p = 0; p < P; ++p) l1 += fabs(params[p]);
        for (long p = 0; p < P; ++p) {
            double par = params[p];
            if (fabs(par) > 0) der[p] += w * (par < 0 ? -1.0 : 1.0);
            else if (der[p] < -w) der[p] += w;
            else if (der[p] > w) der[p] -= w;
            else der[p] = 0.0;
        }
    }
    if (mt->reg_l2 > 0) {                                              /* hxx:469-489 */
        for (long i = 0; i < C; ++i) {
            double n2 = 0;
            for (int d = 0; d < D; ++d) n2 += params[i + d * C] * params[i + d * C];
            l2 += n2;
            for (int d = 0; d < D; ++d) der[i + d * C] += mt->reg_l2 * 2.0 * params[i + d * C];
        }
    }
    if (mt->reg_l21 > 0) {                                             /* hxx:491-526 */
        double w = mt->reg_l21;
        for (long i = 0; i < C; ++i) {
            double n2 = 0;
            for (int d = 0; d < D; ++d) n2 += params[i + d * C] * params[i + d * C];
            double nrm = sqrt(n2);
            l21 += nrm;
            for (int d = 0; d < D; ++d) {
                long p = i + d * C;
                if (nrm > 0) der[p] += w * params[p] / nrm;
                else if (der[p] < -w) der[p] += w;
                else if (der[p] > w) der[p] -= w;
                else der[p] = 0.0;
            }
        }
    }
    if (mt->use_negative_gradient)                                     /* hxx:528-529 */
        for (long p = 0; p < P; ++p) der[p] = -der[p];
    double reg = 0;                                                    /* hxx:531-538 */
    if (mt->reg_l1 > 0) reg += mt->reg_l1 * l1;
    if (mt->reg_l21 > 0) reg += mt->reg_l21 * l21;
    if (mt->reg_l2 > 0) reg += mt->reg_l2 * l2;
    if (mt->reg_rkhs > 0) reg += mt->reg_rkhs * r.reg_value_rkhs;
    if (mt->reg_rd > 0) reg += mt->reg_rd * r.reg_value_rd;
    if (mt->reg_pg > 0) reg += mt->reg_pg * r.reg_value_pg;
    out->measure = r.measure;
    out->reg_value = reg;
    out->value = r.measure + reg;
    out->reg_l1 = l1; out->reg_l21 = l21; out->reg_l2 = l2;
    out->reg_rkhs = r.reg_value_rkhs; out->reg_rd = r.reg_value_rd; out->reg_pg = r.reg_value_pg;
    out->num_pixels_counted = r.num_pixels_counted;
    if (!derivative) free(der);
    free(cp);
    return rc;
}

/* ------------------------------------------------------------------------- */
/* optimizer: ITK v4 gradient-descent loop + Standard/Adaptive step */
int ora_optimize(ora_ctx *c, const skm_optimizer_desc *o, const skm_metric_desc *m, const double *cpw,
                 const skm_field *df, int iterations, double *position, double *tmp_grad,
                 double *base, double *best_position, ora_opt_state *st, double *values)
{
    long P = c->nparams;
    double *g = (double *)malloc(sizeof(double) * P);
    int rc = 0;
    for (int it = 0; it < iterations && st->iteration < o->number_of_iterations; ++it) {
        skm_metric_values mv;
        /* m_Gradient <- metric derivative at the current position */
        rc |= ora_metric_evaluate(c, m, position, cpw, df, g, &mv);
        if (values) values[it] = mv.value;
        st->last_value = mv.value;
        /* EstimateLearningRate (Adaptive.hxx:86-97): gamma(t) = a/(A+t+1)^alpha */
        double lr = o->a / pow(o->A + st->current_time + 1.0, o->alpha);
        /* CalculateScalarProduct (Adaptive.hxx:100-113) */
        double sp = 0.0;
        for (long j = 0; j < P; ++j) sp += g[j] * tmp_grad[j];
        memcpy(tmp_grad, g, sizeof(double) * P);
        /* Std.hxx:132-142: x = x_prev + g*lr, orthant projection */
        for (long j = 0; j < P; ++j) {
            double nx = base[j] + g[j] * lr;
            if (o->orthant_projection && nx * base[j] < 0) nx = 0.0;
            position[j] = nx;
        }
        memcpy(base, position, sizeof(double) * P);
        /* ModifyCurrentTime (Adaptive.hxx:115-128) */
        double x = -sp;
        double fx = o->f_min + (o->f_max - o->f_min) / (1.0 - (o->f_max / o->f_min) * exp(-x / o->omega));
        st->current_time = st->current_time + fx;
        if (st->current_time < 0.0) st->current_time = 0.0;
        st->learning_rate = lr;
        st->scalar_product = sp;
        if (mv.value < st->best_value) {   /* ReturnBestParametersAndValue: position after the step */
            st->best_value = mv.value;
            if (best_position) memcpy(best_position, position, sizeof(double) * P);
        }
        st->iteration++;
    }
    free(g);
    return rc;
}

/* ------------------------------------------------------------------------- */
void ora_kernel_values(const skm_evaluator_desc *d, int64_t n, const double *p, const double *q, double *k)
{
    kern_t K;
    int D = d->dimensions;
    memset(&K, 0, sizeof K);
    kern_init(&K, d);
    for (int64_t i = 0; i < n; ++i) {
        pinfo_t pi;
        kern_pinfo(&K, p + i * D, &pi);
        k[i] = kern_eval(&K, p + i * D, q + i * D, &pi);
    }
}
