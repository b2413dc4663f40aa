/*
 * picunet.h -- C-ABI of libpicunet.so, the network of the learned
 * preconditioner (a 3-level U-Net on the node grid, BF16 on the tensor cores
 * with FP32 accumulation) used inside flexible CG by pic_ife_solve.
 *
 * The reference has no learned preconditioner (its MY_PCG is Jacobi-PCG):
 * this library has no counterpart there.  Tensors are device pointers in NHWC
 * layout (pixel p = i*W + j on an H x W grid, channels fastest), filters
 * KRSC.  Every function enqueues on `stream` (a cudaStream_t, NULL = default
 * stream) and returns 0 or a negative UNET_ERR_* code.
 */
#ifndef PICUNET_H
#define PICUNET_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define UNET_OK 0
#define UNET_ERR_SHAPE (-1)
#define UNET_ERR_WORKSPACE (-2)
#define UNET_ERR_CUDA (-3)

#define UNET_FPROP_RELU 0 /* d = ReLU(conv(a = x, b = W) + bias), BF16        */
#define UNET_DGRAD 1      /* d = dx from a = dy, b = W, BF16                   */

/* 3x3 convolution ('same' padding, stride 1) of an n x h x w x c activation
 * with k filters on the tensor cores; c and k multiples of 8.  With
 * workspace == NULL, stream == NULL and ws_need != NULL the call only reports
 * the workspace bytes the convolution needs. */
int unet_conv(int32_t op, int32_t n, int32_t h, int32_t w, int32_t c, int32_t k, const void *a, const void *b,
              void *d, const void *bias, void *workspace, size_t ws_bytes, size_t *ws_need, void *stream);

/* Weight gradient of a 3x3 'same' convolution: dW[k,r,s,c] (FP32, KRSC)
 * += sum over pixels of dy[p,k] * x[p shifted by (r-1, s-1), c] (zero
 * outside the image).  dW must be zeroed by the caller before the first
 * accumulation.  Any c and k. */
int unet_wgrad(int32_t n, int32_t h, int32_t w, int32_t c, int32_t k, const void *x, const void *dy, float *dw,
               void *stream);

/* Residual scale on the device: scale[0] = s = sqrt(sum of r^2 over nodes
 * with mask > 0 / their count), scale[1] = 1/s (both 0 when r vanishes there).
 * Deterministic (fixed-order block partials).  scratch: UNET_RMS_SCRATCH
 * doubles, zero-filled before the first call and kept between calls. */
#define UNET_RMS_BLOCKS 592
#define UNET_RMS_SCRATCH (2 * UNET_RMS_BLOCKS + 1)
int unet_rms(int64_t npix, const double *r, const int32_t *mask, double *scratch, double *scale, void *stream);

/* Input features on the node grid (h x w, 8 channels, BF16):
 * [r/s, log eps_r, level set, Dirichlet mask, 0, 0, 0, 0] where r is the
 * FP64 residual on the full grid and scale = {s, 1/s} a device pointer
 * (unet_rms).  feat_static holds channels 1..3 ([h*w*3], FP32), prepared
 * once per mesh. */
int unet_features(int32_t h, int32_t w, const double *r, const double *scale, const float *feat_static,
                  void *x_out, void *stream);

/* 2x2 average pooling over the children that exist (ceil sizes), forward and
 * backward (dx written, or added to when accumulate != 0).  c multiple of 8. */
int unet_pool(int32_t n, int32_t h, int32_t w, int32_t c, const void *x, void *y, void *stream);
int unet_pool_bwd(int32_t n, int32_t h, int32_t w, int32_t c, const void *dy, void *dx, int32_t accumulate,
                  void *stream);

/* Nearest x2 upsampling of lo ((h+1)/2 x (w+1)/2 x c1) to h x w, concatenated
 * with skip (h x w x c2): y is h x w x (c1 + c2).  Backward splits dy into
 * dlo (summed over the children) and dskip (written, or added to when
 * accumulate_skip != 0).  c1, c2 multiples of 8. */
int unet_upcat(int32_t n, int32_t h, int32_t w, int32_t c1, int32_t c2, const void *lo, const void *skip,
               void *y, void *stream);
int unet_upcat_bwd(int32_t n, int32_t h, int32_t w, int32_t c1, int32_t c2, const void *dy, void *dlo,
                   void *dskip, int32_t accumulate_skip, void *stream);

/* dy *= (y > 0) in place (ReLU backward through the fused epilogue) and the
 * bias gradient db[c] += sum over pixels of dy (FP32).  c multiple of 8. */
int unet_relu_bwd(int64_t npix, int32_t c, const void *y, void *dy, float *db, void *stream);

/* 1x1 head with one output, c = 32: z[p] = sum_c w[c] y[p,c] + b (FP32 out);
 * its backward (dy BF16 = gz w; dw, db accumulated FP32); and the loss
 * sum (z - t/s)^2 and sum (t/s)^2 added to loss2[0..1], with gradient gz,
 * over nodes with mask > 0 (s = scale[0], scale[1] = 1/s from unet_rms). */
int unet_head(int64_t npix, int32_t c, const void *y, const float *w, const float *b, float *z, void *stream);
int unet_head_bwd(int64_t npix, int32_t c, const void *y, const float *w, const float *gz, void *dy, float *dw,
                  float *db, void *stream);
int unet_loss(int64_t npix, const float *z, const double *target, const double *scale, const int32_t *mask,
              float *gz, double *loss2, void *stream);

/* out = s * z on unknown nodes (mask > 0), 0 on Dirichlet nodes. */
int unet_output(int64_t npix, const float *z, const double *scale, const int32_t *mask, double *out,
                void *stream);

/* Adam on FP32 master weights (bias-corrected, step t >= 1) with a BF16 copy
 * for the tensor cores (p_bf16 may be NULL). */
int unet_adam(int64_t n, float *p, const float *g, float *m, float *v, void *p_bf16, float lr, float beta1,
              float beta2, float eps, int32_t t, void *stream);

/* Fill / convert helpers. */
int unet_fill_f32(int64_t n, float *p, float v, void *stream);
int unet_f32_to_bf16(int64_t n, const float *src, void *dst, void *stream);

#ifdef __cplusplus
}
#endif
#endif
