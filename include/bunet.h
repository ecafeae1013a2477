/*
 * bunet.h -- C ABI of the tensor-core 3-D U-Net that supplies a learned
 * initial guess to the multigrid solve (include/bmg.h).  No counterpart in
 * the reference: Briscola's multigrid starts from the caller's x.
 *
 * All tensors are device pointers on the current device; work is queued on
 * `stream` (a cudaStream_t, NULL for the default stream) and nothing is
 * allocated.  Activations and gradients are BF16, channels-last: element
 * (i, j, k, c) of an n0 x n1 x n2 grid with C channels at
 * ((i*n1 + j)*n2 + k)*C + c (the solver's cell order, channels innermost),
 * 16-byte aligned.  Convolutions are 3x3x3, stride 1, zero padding 1, tap
 * t = (di+1)*9 + (dj+1)*3 + (dk+1); master weights are FP32 W[t][cin][cout].
 * Every function returns BUN_OK or an error code and never throws.
 */
#ifndef BUNET_H
#define BUNET_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    BUN_OK = 0,
    BUN_BAD_ARG = 3,    /* unsupported shape, channel count or alignment         */
    BUN_CUDA_ERROR = 4, /* a launch failed (see the CUDA error state)              */
};

/* Largest number of voxels (n0*n1*n2) of one convolution. */
#define BUN_MAX_VOXELS (1L << 30)

/* Tensor-core convolution, forward or data gradient:
 *   out[v][n] = epi( sum_{t,c} in[v + off(t)][c] * W[t][c][n] )
 * in: channels [0, c0) of src0 -- at half resolution (n0/2 x n1/2 x n2/2)
 *     and upsampled by nearest neighbour when up0 != 0 -- then channels
 *     [c0, c0 + c1) of src1 (the decoder's concatenation; c1 = 0: none).
 * wpack: from bun_pack_weights with the same kc and cout.
 * epi: + bias[n] (bias != NULL), max(., 0) (relu != 0), * (mask[v][n] > 0)
 *      (mask != NULL: a BF16 tensor of cout channels on the output grid).
 * kc: input channels per pipeline stage (16, 32 or 64), dividing c0 and c1.
 * Supported (kc, cout): (16: 16/32/48/64), (32: 16/32/64/96), (64: 32/64/128).
 * With kc = 16 on grids with n2 % 128 == 0 the row-marching kernel runs
 * (see bun_conv3_stage_width); the result is the same convolution.
 * err: device int set to nonzero if a CTA gave up waiting (never expected). */
int bun_conv3(int n0, int n1, int n2, const void* src0, int c0, int up0, const void* src1, int c1,
              const void* wpack, int kc, int cout, const float* bias, int relu, const void* mask, void* out,
              int* err, void* stream);

/* The stage width kc to pack weights for and pass to bun_conv3 for a
 * convolution with inputs (c0, c1), cout outputs on grids of extent n2
 * along k: 16 where the row-marching kernel applies (n2 % 128 == 0 and
 * (cin, cout) in {(16,16), (16,32), (16,48), (32,16), (32,32), (48,16)}),
 * otherwise the widest of 64/32/16 the tile kernel supports; 0: none. */
int bun_conv3_stage_width(int c0, int c1, int cout, int n2);

/* Weight gradient of a tensor-core convolution with the inputs of bun_conv3
 * and the output gradient dz (cout channels, 16/32/64):
 *   dw[t][c][n] = sum_v in[v + off(t)][c] * dz[v][n]      (FP32, overwritten)
 * split over nsplit voxel ranges; part: caller scratch of
 * bun_wgrad_part_floats(...) floats. */
size_t bun_wgrad_part_floats(int cin, int cout, int nsplit);
int bun_conv3_wgrad(int n0, int n1, int n2, const void* src0, int c0, int up0, const void* src1, int c1,
                    const void* dz, int cout, int nsplit, float* part, float* dw, int* err, void* stream);

/* BF16 weights of one convolution in the tile layout of bun_conv3:
 * transpose = 0: forward (K = cin, N = cout); transpose = 1: data gradient
 * (K = cout, N = cin, taps mirrored).  out: 27*cin*cout BF16. */
int bun_pack_weights(const float* w, int cin, int cout, int kc, int transpose, void* out, void* stream);

/* First layer, 1 -> 16 channels on the CUDA cores: out = relu(b + W * x),
 * x FP32 (one channel), w FP32 [27][16], b FP32 [16]. */
int bun_conv_in(int n0, int n1, int n2, const float* x, const float* w, const float* b, void* out, void* stream);
/* its weight gradient: dw[27*16 + 16] (weights then bias), part: nblocks*448
 * floats of scratch */
int bun_conv_in_wgrad(int n0, int n1, int n2, const float* x, const void* dz, int nblocks, float* part, float* dw,
                      void* stream);

/* Output head, 16 -> 1 channel, 1x1x1: y = b + w . d (FP32 out) */
int bun_head(long n, const void* d, const float* w, const float* b, float* y, void* stream);
/* dz = dy w (d > 0); dw[17] (weights then bias); part: nblocks*17 floats */
int bun_head_grad(long n, const void* d, const float* dy, const float* w, void* dz, int nblocks, float* part,
                  float* dw, void* stream);

/* 2x2x2 mean pooling of src (c channels, fine grid n0 x n1 x n2, even). */
int bun_pool(int n0, int n1, int n2, int c, const void* src, void* dst, void* stream);
/* Gradient of the upsampled part of a concatenated input: dz (coarse, c0
 * channels) = sum over the 8 children of dcat[..][0:c0] (fine grid, ccat
 * channels), masked by act > 0 (act: the coarse tensor that was upsampled). */
int bun_unpool_grad(int n0, int n1, int n2, int ccat, int c0, const void* dcat, const void* act, void* dz,
                    void* stream);
/* Gradient of a skip tensor src (c channels, fine grid) feeding both a
 * concatenation (channels [c0, c0+c) of dcat) and a pooling (dp: gradient of
 * the pooled tensor): dz = (src > 0) * (dcat[..][c0:c0+c] + dp(parent) / 8). */
int bun_skip_grad(int n0, int n1, int n2, int ccat, int c0, int c, const void* dcat, const void* dp,
                  const void* src, void* dz, void* stream);

/* Mean squared error: loss = mean (y - t)^2, dy = 2 (y - t) / n;
 * part: nblocks floats of scratch. */
int bun_mse(long n, const float* y, const float* t, float* dy, int nblocks, float* part, float* loss, void* stream);
/* Adam step (bias-corrected, step >= 1) on FP32 master weights. */
int bun_adam(long n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
             int step, void* stream);

/* Residual term of the training loss on a uniform n0 x n1 x n2 grid with
 * Neumann walls: r = sum over in-grid neighbours of (y_nb - y) + c f, and
 * its adjoint in y, dy += w * (the same stencil applied to g). */
int bun_laplace_residual(int n0, int n1, int n2, const float* y, const float* f, float c, float* r, void* stream);
int bun_laplace_add(int n0, int n1, int n2, const float* g, float w, float* dy, void* stream);

/* y = scale * x between the solver's FP64 fields and the network's FP32 ones */
int bun_scale_to_float(long n, const double* x, double scale, float* y, void* stream);
int bun_scale_to_double(long n, const float* x, double scale, double* y, void* stream);
/* *out = sum x^2 (FP64, fixed order); part: nblocks doubles of scratch */
int bun_sumsq(long n, const double* x, int nblocks, double* part, double* out, void* stream);
/* The network's input from a field of any size, with the scale kept on the
 * device (nothing returns to the host, so the calls can be captured into a
 * CUDA graph): *rms = sqrt(sum x^2 / n) (FP64, fixed order; part: nblocks
 * doubles of scratch) and y = sign * x / *rms (zero when *rms is zero);
 * then, for the output, x = scale * *rms * y. */
int bun_rms_normalise(long n, const float* x, float sign, int nblocks, double* part, double* rms, float* y,
                      void* stream);
int bun_rms_restore(long n, const float* y, double scale, const double* rms, float* x, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BUNET_H */
