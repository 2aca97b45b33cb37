/* causticws.h -- kernels of the learned warm start for the SDOT solver.
 *
 * No counterpart in the reference: its solver always starts from the
 * previous weights or zero (main.cu:193-198).  A small convolutional
 * encoder-decoder maps a target image and the site layout to initial dual
 * weights; the plain L-BFGS (cot_solve) then runs from them to the same
 * tolerance, so the network only changes where the solve starts.
 *
 * BF16 operands with FP32 accumulation.  Activations are NHWC; a 3x3
 * convolution is im2col (ws_im2col) followed by ws_gemm.  All pointers are
 * device pointers; every call is asynchronous on `stream` (a cudaStream_t,
 * NULL for the legacy default stream) and returns WS_OK or a negative code.
 * The network itself (layer list, training loop) is host code above this
 * interface (caustic_b200/warmstart.py). */
#ifndef CAUSTICWS_H
#define CAUSTICWS_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define WS_API __attribute__((visibility("default")))
#else
#define WS_API
#endif

enum { WS_OK = 0, WS_EINVAL = -1, WS_ECUDA = -2, WS_ECAPACITY = -4 };

/* GEMM layouts (row-major D[M,N] fp32 = alpha A B + beta D):
 * RC: A[M][K] K-contiguous, B stored [N][K]   -- conv forward, D = cols W^T
 * CR: A stored [K][M], B[K][N] N-contiguous  -- weight gradient, dW = dZ^T cols
 * RR: A[M][K], B[K][N] both row-major       -- input gradient, dcols = dZ W */
enum { WS_GEMM_RC = 0, WS_GEMM_CR = 1, WS_GEMM_RR = 2 };

/* Tensor-core GEMM (tcgen05, 128x128x64 tiles).  K must be a multiple of 8;
 * for CR also M and N, for RR also N (16-byte rows).  workspace: device
 * scratch of ws_gemm_workspace() bytes (may be 0). */
WS_API int ws_gemm(int layout, int M, int N, int K, const void *A, const void *B, float *D, float alpha,
                   float beta, void *workspace, size_t workspace_bytes, void *stream);
WS_API size_t ws_gemm_workspace(int layout, int M, int N, int K);

/* 3x3 / stride 1 / zero-padding 1 patches: cols[B*H*W][9*C] (bf16) from
 * in[B][H][W][C] (bf16), column = tap*C + c with tap = (dy+1)*3 + (dx+1). */
WS_API int ws_im2col(int B, int H, int W, int C, const void *in, void *cols, void *stream);
/* Adjoint of ws_im2col: dx[B][H][W][C] = sum of the patch entries that read
 * each pixel (a gather in fixed order, fp32). */
WS_API int ws_col2im(int B, int H, int W, int C, const float *dcols, float *dx, void *stream);

/* y = act(d + bias) (bf16 out; act = ReLU if relu, else identity); pre
 * (nullable) keeps d + bias in fp32.  d, pre: [M][C]. */
WS_API int ws_bias_act(long long M, int C, const float *d, const float *bias, int relu, void *y, float *pre,
                       void *stream);
/* dz = dy * act'(pre): bf16 for the GEMMs, and fp32 (dz32, nullable). */
WS_API int ws_act_back(long long n, int relu, const float *dy, const float *pre, void *dz, float *dz32,
                       void *stream);
/* db[c] = sum_m dz[m][c] (fixed order). */
WS_API int ws_colsum(long long M, int C, const float *dz, float *db, void *stream);

/* 2x2 average pooling (H, W even) and its adjoint. */
WS_API int ws_pool2(int B, int H, int W, int C, const void *in, void *out, void *stream);
WS_API int ws_pool2_back(int B, int H, int W, int C, const float *dout, float *din, void *stream);
/* Nearest 2x upsampling of in[B][H][W][C] into channels c0.. of
 * out[B][2H][2W][Ct], and its adjoint (din[B][H][W][C]). */
WS_API int ws_up2(int B, int H, int W, int C, const void *in, int Ct, int c0, void *out, void *stream);
WS_API int ws_up2_back(int B, int H, int W, int C, const float *dout, int Ct, int c0, float *din, void *stream);
/* Skip connections: out[p][c0 + c] = in[p][c] (bf16) for P pixels, and the
 * backward din[p][c] (+)= dout[p][c0 + c] (fp32; add != 0 accumulates). */
WS_API int ws_put_channels(long long P, int C, const void *in, int Ct, int c0, void *out, void *stream);
WS_API int ws_take_channels(long long P, int C, const float *dout, int Ct, int c0, int add, float *din,
                            void *stream);

/* Loss of B predictions of the weights of a gy x gx site grid (row-major)
 * against their targets, each compared after removing its mean (weights are
 * defined up to a constant).  With e = pred - target minus its mean:
 * loss_b[b] = (sum e^2 + lambda * sum of the squared differences of e between
 * grid neighbours) / (gy gx B); grad = d(sum_b loss_b) / d pred.  The
 * difference term weighs the local structure that sets the cells' masses. */
WS_API int ws_mse_centered(int B, int gy, int gx, float lambda, const float *pred, const float *target,
                           float *grad, float *loss_b, void *stream);

/* Adam step `step` (1-based) on fp32 weights w, refreshing their bf16 copy
 * w16 (nullable). */
WS_API int ws_adam(long long n, float *w, void *w16, const float *g, float *m, float *v, float lr, float b1,
                   float b2, float eps, int step, void *stream);
WS_API int ws_to_bf16(long long n, const float *x, void *y, void *stream);

/* ---- the learned warm start as one call (no counterpart in the reference:
 * its solver starts from the previous outer iteration's weights or zero,
 * main.cu:193-198) ------------------------------------------------------- */
typedef struct ws_net ws_net;

/* Load a network saved by WarmStartNet.save_bin (caustic_b200/warmstart.py)
 * onto `device`: BF16 weights and FP32 biases stay there until
 * cot_warmstart_free. */
WS_API int cot_warmstart_load(const char *path, int device, ws_net **out);
WS_API int cot_warmstart_free(ws_net *net);

/* Initial dual weights for the problem of a gx x gy jittered site lattice
 * (sites_xy[2*(a + gx*b)], caller order, inside proj_domain), target masses
 * nu[n] and density image density[ix + iy*nx] (any positive scale; nx and ny
 * whole multiples of gx and gy, gx and gy multiples of 2^(levels-1)): the
 * network's prediction with its mean removed, into w_out[n] (host memory;
 * all inputs are host arrays too).  The plain solve (cot_solve) then starts
 * from w_out; the inputs are prepared as warmstart.make_input does. */
WS_API int cot_warmstart_predict(ws_net *net, const double *sites_xy, const double *nu, int gx, int gy,
                                 const double *density, int nx, int ny, const double proj_domain[4], double *w_out,
                                 void *stream);
/* Message of the last failure of the three calls above. */
WS_API int cot_warmstart_last_error(char *buf, size_t n);

#ifdef __cplusplus
}
#endif

#endif
