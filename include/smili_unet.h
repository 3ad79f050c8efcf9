/* smili_unet: BF16 kernels of the warm-start U-Net (libsmili_unet.so).
 *
 * No reference counterpart: SMILI starts every solve from a flat or Gaussian
 * prior image (smili/imaging/lbfgs.py:44-80 takes `initimage` from the
 * caller).  These kernels train and run a small U-Net that maps a dirty
 * image to a starting image for the same L-BFGS-B solve.
 *
 * All pointers are device pointers; every call is asynchronous on `stream`
 * (a cudaStream_t, NULL = the legacy default stream) and returns 0 or a
 * negative error code.  Activations are NHWC bfloat16 with a channel stride
 * `ld` (>= the channel count), so a call may read or write a channel slice
 * of a wider buffer.  Convolution weights are [Cout][3][3][Cin] bfloat16;
 * gradients and optimiser state are float32.
 */
#ifndef SMILI_UNET_H
#define SMILI_UNET_H
#ifdef __cplusplus
extern "C" {
#endif

#define SMILI_UNET_ERR_ARG (-1)
#define SMILI_UNET_ERR_CUDA (-3)

/* y (+)= act(conv3x3(x, w) + bias): pad 1, stride 1, FP32 accumulation on the
 * tensor cores.  relu != 0 applies max(0, .); accumulate != 0 adds to y.
 * When Cin and ldx are multiples of 8 and x, w are 16-byte aligned, the
 * convolution runs on the tcgen05 tensor cores (TMA-staged operands, FP32
 * accumulator in tensor memory); otherwise on mma.sync. */
int smili_unet_conv3x3(const void* x, int N, int H, int W, int Cin, int ldx, const void* w, const float* bias,
                       void* y, int ldy, int Cout, int relu, int accumulate, void* stream);

/* dw (+)= sum over pixels of dy[p][co] x[p + (ky-1, kx-1)][ci].  `partial` is
 * scratch of nsplit * Cout * 9 * Cin floats; the splits are summed in a fixed
 * order, so the result is deterministic.  When Cin, Cout, ldx and lddy are
 * multiples of 8 and x, dy are 16-byte aligned, the partials come from the
 * tcgen05 tensor cores (pixels as the K dimension, both operands TMA-staged);
 * otherwise from mma.sync. */
int smili_unet_conv3x3_wgrad(const void* x, int ldx, const void* dy, int lddy, int N, int H, int W, int Cin,
                             int Cout, float* partial, int nsplit, float* dw, int accumulate, void* stream);

/* db[c] (+)= sum over npix pixels of dy[p][c] */
int smili_unet_bias_grad(const void* dy, int ld, long long npix, int C, float* db, int accumulate, void* stream);

/* wt[ci][ky][kx][co] = w[co][2-ky][2-kx][ci]: the weights of the data-gradient
 * convolution (dx = conv3x3(dy, wt) with Cin and Cout exchanged). */
int smili_unet_flip_weights(const void* w, void* wt, int Cout, int Cin, void* stream);

/* dy[p][c] = 0 where y[p][c] <= 0 (ReLU backward on the post-activation) */
int smili_unet_relu_mask(const void* y, int ldy, void* dy, int lddy, long long npix, int C, void* stream);

/* 2x2 average pooling (H, W even) and its gradient (accumulate adds to dx) */
int smili_unet_avgpool2(const void* x, int ldx, void* y, int ldy, int N, int H, int W, int C, void* stream);
int smili_unet_avgpool2_bwd(const void* dy, int lddy, void* dx, int lddx, int N, int H, int W, int C,
                            int accumulate, void* stream);

/* nearest 2x upsampling of an H x W input and its gradient */
int smili_unet_upsample2(const void* x, int ldx, void* y, int ldy, int N, int H, int W, int C, void* stream);
int smili_unet_upsample2_bwd(const void* dy, int lddy, void* dx, int lddx, int N, int H, int W, int C,
                             int accumulate, void* stream);

/* mean squared error of n one-channel outputs against a float target:
 * loss_part[b] = block b's sum of squares (nblocks blocks); dy = 2 (y - t) / n */
int smili_unet_mse(const void* y, int ldy, const float* target, long long n, void* dy, int lddy, float* loss_part,
                   int nblocks, void* stream);

/* Adam with decoupled weight decay on float master weights w (and their
 * bfloat16 copy w16, may be NULL); step counts from 1. */
int smili_unet_adam(float* w, void* w16, const float* g, float* m, float* v, long long n, float lr, float b1,
                    float b2, float eps, float wd, int step, void* stream);

int smili_unet_f32_to_bf16(const float* x, void* y, long long n, void* stream);

/* Convolution path (forward, data gradient and weight gradient): 0 (default)
 * tcgen05 where it applies, 1 mma.sync always, 2 tcgen05 with one 128-pixel
 * tile per CTA in the forward convolution (the default gives a CTA two when
 * the image has at least 16 rows).  Process-wide; for comparisons and tests. */
int smili_unet_set_conv_path(int path);

/* Reads and clears the tcgen05 convolution's error flag (synchronous):
 * 0, or the code of a bounded wait inside the kernel that ran out (1 stage
 * release, 2 operand arrival, 3 accumulator completion, 4 outstanding copy;
 * 5-8 the same in the weight gradient), or SMILI_UNET_ERR_CUDA. */
int smili_unet_tc_status(void);

/* Why the last tcgen05 convolution call of this thread failed ("" if none). */
const char* smili_unet_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
