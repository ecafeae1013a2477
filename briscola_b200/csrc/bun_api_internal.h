// bun_api_internal.h -- launchers of the U-Net's CUDA-core kernels
// (bun_elem.cu), called by the C ABI in bun_api.cu.
#pragma once

#include "bun_internal.h"

namespace bun {

cudaError_t conv_in_launch(int n0, int n1, int n2, const float* x, const float* w, const float* b, bf16* out,
                           cudaStream_t s);
cudaError_t conv_in_wgrad_launch(int n0, int n1, int n2, const float* x, const bf16* dz, float* part, int nblocks,
                                 float* dw, cudaStream_t s);
cudaError_t head_launch(long n, const bf16* d, const float* w, const float* b, float* y, cudaStream_t s);
cudaError_t head_grad_launch(long n, const bf16* d, const float* dy, const float* w, bf16* dz, float* part,
                             int nblocks, float* dw, cudaStream_t s);
cudaError_t pool_launch(int n0, int n1, int n2, int C, const bf16* src, bf16* dst, cudaStream_t s);
cudaError_t unpool_grad_launch(int n0, int n1, int n2, int ccat, int c0, const bf16* dcat, const bf16* act,
                               bf16* dz, cudaStream_t s);
cudaError_t skip_grad_launch(int n0, int n1, int n2, int ccat, int c0, int C, const bf16* dcat, const bf16* dp,
                             const bf16* src, bf16* dz, cudaStream_t s);
cudaError_t mse_launch(long n, const float* y, const float* t, float* dy, float* part, int nblocks, float* loss,
                       cudaStream_t s);
cudaError_t sum_parts_launch(const float* part, int nparts, long stride, long len, float* out, cudaStream_t s);
cudaError_t pack_launch(const float* w, int cin, int cout, int kc, int transpose, bf16* out, cudaStream_t s);
cudaError_t adam_launch(long n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2,
                        float eps, int step, cudaStream_t s);
cudaError_t to_float_launch(long n, const double* x, double scale, float* y, cudaStream_t s);
cudaError_t to_double_launch(long n, const float* x, double scale, double* y, cudaStream_t s);
cudaError_t lap_residual_launch(int n0, int n1, int n2, const float* y, const float* f, float c, float* r,
                                cudaStream_t s);
cudaError_t lap_add_launch(int n0, int n1, int n2, const float* g, float w, float* dy, cudaStream_t s);
cudaError_t sumsq_launch(long n, const double* x, double* part, int nblocks, double* out, cudaStream_t s);
cudaError_t rms_normalise_launch(long n, const float* x, float sign, double* part, int nblocks, double* rms,
                                 float* y, cudaStream_t s);
cudaError_t rms_restore_launch(long n, const float* y, double scale, const double* rms, float* x, cudaStream_t s);

}  // namespace bun
