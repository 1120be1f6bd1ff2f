/*
 * skm_warmstart.h -- C-ABI of the learned warm start's tensor-core kernels.
 *
 * No counterpart in the reference (it has no learned component): a small 3-D convolutional
 * encoder-decoder predicts the coarsest scale level's kernel weights alpha from an image pair, as
 * the starting point of the plain optimizer (which stays the fallback and the judge of the final
 * metric value).  These entry points are the network's compute: BF16 implicit-GEMM 3-D
 * convolutions on the tcgen05 tensor cores with FP32 accumulation (forward, data gradient, weight
 * gradient), the weight packing they read, the loss and an Adam step.  The network itself (layers,
 * buffers, training loop) is driven from skmimageregistration_b200/warmstart.py.
 *
 * Conventions
 *  - Every pointer is DEVICE memory owned by the caller; nothing is allocated here.  Work is
 *    enqueued on `stream` (a cudaStream_t, NULL = default stream) and the call returns without
 *    waiting.
 *  - Activations are channels-last bf16: [batch][z][y][x][channels], x fastest among the voxels.
 *  - Convolutions are 3x3x3, zero padding 1, stride 1 or 2: out size = (in size - 1) / stride + 1.
 *  - Weights (FP32 master copy) are [c_out][tap][c_in] with tap = 9 kz + 3 ky + kx.
 *  - `err` is a device word that a bounded tensor-core wait sets when it gives up (the kernel then
 *    returns after freeing its tensor memory); the caller reads it after synchronising and treats a
 *    nonzero value like SKM_ERR_TIMEOUT (results of that launch are void).
 *  - Operands read with 16-byte loads (x, dy, packed weights) must be 16-byte aligned.
 *  - Return SKM_OK or an error code of include/skm_gpu.h; skm_last_error() has the message.
 */
#ifndef SKM_WARMSTART_H
#define SKM_WARMSTART_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct skm_conv3d_desc {
    int32_t batch;
    int32_t in_size[3];       /* x, y, z voxels of the input */
    int32_t in_channels;      /* <= 128 */
    int32_t out_channels;     /* <= 128 */
    int32_t stride;           /* 1 or 2 */
} skm_conv3d_desc;

/* Output size (x, y, z) of the convolution. */
int skm_conv3d_out_size(const skm_conv3d_desc *d, int32_t *out);

/* Shapes of the packed bf16 weight operands: forward [fwd_rows][fwd_ld], data gradient
 * [dgrad_rows][dgrad_ld] (rows padded to 16, leading dimensions to 64 elements). */
int skm_conv3d_weight_layout(const skm_conv3d_desc *d, int32_t *fwd_rows, int32_t *fwd_ld, int32_t *dgrad_rows,
                             int32_t *dgrad_ld);

/* FP32 master weights [c_out][27 c_in] -> the two packed bf16 operands. */
int skm_conv3d_pack_weights(const skm_conv3d_desc *d, const float *w, void *w_fwd, void *w_dgrad, void *stream);

/* y = act(conv(x, W) + bias) in bf16; y32 (may be NULL) receives the FP32 value before the ReLU.
 * relu != 0 applies max(0, .). */
int skm_conv3d_forward(const skm_conv3d_desc *d, const void *x, const void *w_fwd, const float *bias, int32_t relu,
                       void *y, float *y32, uint32_t *err, void *stream);

/* dx = conv^T(dy, W), multiplied by (mask > 0) when mask (the layer input, itself a ReLU output)
 * is not NULL; bf16, dx32 (may be NULL) the FP32 copy. */
int skm_conv3d_backward_data(const skm_conv3d_desc *d, const void *dy, const void *w_dgrad, const void *mask, void *dx,
                             float *dx32, uint32_t *err, void *stream);

/* Workspace bytes skm_conv3d_backward_weights needs for this shape. */
size_t skm_conv3d_backward_weights_workspace(const skm_conv3d_desc *d);

/* dW [c_out][27 c_in] (FP32, split-K partials summed in a fixed order) and, when db is not NULL,
 * the bias gradient db [c_out] = sum over output voxels of dy. */
int skm_conv3d_backward_weights(const skm_conv3d_desc *d, const void *x, const void *dy, float *dw, float *db,
                                void *workspace, size_t workspace_bytes, uint32_t *err, void *stream);

/* Adam (Kingma & Ba 2015) on FP32 master weights, step t >= 1 (bias-corrected moments). */
int skm_adam_step(float *w, const float *g, float *m, float *v, int64_t n, float lr, float beta1, float beta2,
                  float eps, int32_t t, void *stream);

/* loss[0] = mean (pred - target)^2 over n values (fixed-order sum); dpred (bf16) = 2 (pred - target) / n. */
int skm_mse_loss(const float *pred, const float *target, int64_t n, float *loss, void *dpred, void *stream);

/* b = bf16(a), round to nearest even. */
int skm_f32_to_bf16(const float *a, int64_t n, void *b, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* SKM_WARMSTART_H */
