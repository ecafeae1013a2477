// bun_internal.h -- device-side pieces of the 3-D U-Net used as a learned
// initial guess for the multigrid solve.  Kernels: bun_conv.cu (tensor-core
// convolutions), bun_elem.cu (CUDA-core kernels); C ABI: bun_api.cu.
//
// Tensors are BF16, channels-last: element (i, j, k, c) of an n0 x n1 x n2
// grid with C channels sits at ((i*n1 + j)*n2 + k)*C + c, i.e. the solver's
// k-fastest cell order with the channels innermost.  Convolutions are 3x3x3,
// stride 1, zero padding 1; tap t = (di+1)*9 + (dj+1)*3 + (dk+1).
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cstdint>

namespace bun {

using bf16 = __nv_bfloat16;

// Inputs of one convolution: channels [0, c0) from src0, [c0, c0+c1) from
// src1 (the decoder's concatenation); src0 may sit at half resolution and be
// read through a nearest-neighbour upsampling (up0 = 1).
struct ConvIn {
    const bf16* src0;
    const bf16* src1;
    int c0, c1;
    int up0;
};

// forward / data-gradient convolution on the tensor cores:
//   out[v][n] = epilogue( sum_{t, c} in[v + off(t)][c] * W[t][c][n] )
// epilogue: + bias[n] (if bias), ReLU (if relu), * (mask[v][n] > 0) (if mask)
// wpack: weights packed by the pack kernel (layout of the kernel's B tiles)
struct ConvArgs {
    int n0, n1, n2;
    ConvIn in;
    const bf16* wpack;
    const float* bias;
    const bf16* mask;
    bf16* out;
    int relu;
    int* err;
};

// weight gradient on the tensor cores, split over voxel blocks:
//   part[s][t*C + c][n] = sum over the split's voxels of in[v+off(t)][c] * dz[v][n]
struct WgradArgs {
    int n0, n1, n2;
    ConvIn in;
    const bf16* dz;
    float* part;   // [nsplit][rows_pad][cout]
    int rows;      // 27 * (c0 + c1)
    int rows_pad;  // rounded up to 128
    int nsplit;
    int* err;
};

// error code written to *err by a kernel that gave up waiting
constexpr int kErrTimeout = 1;

// launchers (bun_conv.cu); return cudaGetLastError() of the launch
cudaError_t conv_launch(const ConvArgs& a, int kc, int nout, cudaStream_t s);
cudaError_t wgrad_launch(const WgradArgs& a, int cout, cudaStream_t s);
bool conv_supported(int kc, int nout);
bool rows_supported(int cin, int nout, int n2);
cudaError_t rows_launch(const ConvArgs& a, int nout, cudaStream_t s);
bool wgrad_supported(int cout);

}  // namespace bun
