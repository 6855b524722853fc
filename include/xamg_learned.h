/* Kernels of the learned initial guess (libxamg_b200.so).  This part has no
 * counterpart in the reference: it is the convolutional encoder-decoder that
 * predicts x0 from the coefficient field and the right-hand side, trained and
 * evaluated on the GPU by these kernels.  The solver's own residual check
 * decides convergence, so a poor prediction costs iterations, never accuracy.
 *
 * Volumes are channels-last BF16 [nb][d][h][w][cs] (device pointers); a
 * tensor argument is a channel window (c0, c) of a buffer with cs channels
 * per voxel.  c, c0 and cs are multiples of 16.  Weights are BF16
 * [cout][27][cin] with tap t = (dz+1)*9 + (dy+1)*3 + (dx+1); biases and
 * weight gradients are FP32.  Products accumulate in FP32 on the tensor
 * cores.  Every call returns 0, 2 for invalid arguments or 3 for a CUDA
 * error; stream is a cudaStream_t (NULL = legacy default stream).
 */
#ifndef XAMG_LEARNED_H_
#define XAMG_LEARNED_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* 3x3x3 convolution with zero padding: out[v][oc0+n] = act(bias[n] + sum over
 * taps and input channels).  flags: 1 = ReLU, 2 = add to the stored output
 * (gradients that meet at a skip connection), 4 = FP32 output (out is a float
 * volume; the network's prediction).  bias may be NULL. */
int xcnn_conv3d(const void *in, int ics, int ic0, int cin, const void *w, const float *bias,
                void *out, int ocs, int oc0, int cout, int nb, int d, int h, int wd, int flags,
                void *stream);
/* Kernel choice of xcnn_conv3d (same convolution either way): 1 (default) =
 * box kernel where the volume tiles into 2 x 8 x 8 voxel boxes (each input
 * voxel staged once per 16-channel chunk), 0 = voxel-tile kernel.  Returns the
 * previous setting. */
int xcnn_set_box_conv(int on);
/* 1 = xcnn_conv3d runs on the 5th-generation tensor cores (tcgen05.mma with a
 * TMEM accumulator; the same convolution, FP32 accumulation in another order);
 * takes precedence over the box choice.  Returns the previous setting. */
int xcnn_set_tc_conv(int on);
/* 1 when a tcgen05 convolution gave up waiting on its tensor pipe (bounded
 * wait) since the last call; the flag is then cleared.  -1 on a CUDA error. */
int xcnn_tc_error(void);
/* dw[co][t][ci] += sum_p grad[p][gc0+co] * in[p + off(t)][ic0+ci]; cout is
 * 16, 32, 64 or 128. */
int xcnn_conv3d_wgrad(const void *in, int ics, int ic0, int cin, const void *grad, int gcs,
                      int gc0, int cout, float *dw, int nb, int d, int h, int wd, void *stream);
/* wt[ci][26-t][co] = w[co][t][ci]: the weights of the backward-data
 * convolution (xcnn_conv3d of the output gradient with wt). */
int xcnn_weight_flip(const void *w, void *wt, int cout, int cin, void *stream);
/* g *= (act > 0) over c channels of nvox voxels. */
int xcnn_relu_bwd(void *g, int gcs, int gc0, const void *act, int acs, int ac0, int c,
                  int64_t nvox, void *stream);
/* db[c] += sum over voxels of g[p][gc0+c] (c divides 256). */
int xcnn_bias_grad(const void *g, int gcs, int gc0, int c, int64_t nvox, float *db, void *stream);
/* 2x2x2 average pooling of the (nb, d, h, w) volume (even sides). */
int xcnn_pool2(const void *in, int ics, int ic0, void *out, int ocs, int oc0, int c, int nb, int d,
               int h, int w, void *stream);
/* Nearest upsampling to the fine volume (nb, d, h, w): mode 0 writes,
 * mode 1 adds one eighth (the backward of xcnn_pool2). */
int xcnn_up2(const void *in, int ics, int ic0, void *out, int ocs, int oc0, int c, int nb, int d,
             int h, int w, int mode, void *stream);
/* Backward of nearest upsampling: coarse gradient = sum of its 8 fine ones. */
int xcnn_up2_bwd(const void *gfine, int gcs, int gc0, void *gin, int ics, int ic0, int c, int nb,
                 int d, int h, int w, void *stream);
/* *loss += mean((pred[p][pc0] - tgt[p])^2) with pred an FP32 volume; grad
 * (BF16, may be NULL): channel 0 = 2 (pred - tgt) / nvox, channels 1..gcs-1 = 0. */
int xcnn_mse(const void *pred, int pcs, int pc0, const float *tgt, void *grad, int gcs,
             int64_t nvox, float *loss, void *stream);
/* Adam step (bias-corrected, step >= 1) on FP32 weights; wb (may be NULL)
 * receives the BF16 copy. */
int xcnn_adam(float *w, const float *g, float *m, float *v, void *wb, int64_t n, float lr, float b1,
              float b2, float eps, int step, void *stream);
/* Network input: channel 0 = a, channel 1 = b, channels 2..15 = 0 (cs 16). */
int xcnn_pack2(const float *a, const float *b, void *out, int64_t nvox, void *stream);
/* out[p] = in[p][c0] * scale[p / per], in an FP32 volume (scale may be NULL). */
int xcnn_unpack(const void *in, int cs, int c0, const float *scale, int64_t per, float *out,
                int64_t nvox, void *stream);

/* Initial guess in the solver's block-vector layout (FP64, row-major n x nv):
 * x[v*nv + s] = scale[s] * in[s*per + v][c0] for the nv samples of a batch
 * (in: FP32 volume). */
int xcnn_unpack_x0(const void *in, int cs, int c0, const float *scale, int nv, int64_t per, double *x,
                   void *stream);

#ifdef __cplusplus
}
#endif

#endif /* XAMG_LEARNED_H_ */
