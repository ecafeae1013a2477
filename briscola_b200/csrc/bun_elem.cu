// bun_elem.cu -- the U-Net's CUDA-core kernels: the 1-channel input
// convolution and the 1x1x1 output head (too narrow for a tensor-core tile),
// pooling and its gradients, the loss, weight packing for the tensor-core
// convolutions, Adam, and the scalings between the solver's FP64 fields and
// the network's FP32 input/output.  All of them are bandwidth-trivial next
// to the 3x3x3 convolutions; reductions write one partial per block and are
// added in a fixed order.

#include "bun_api_internal.h"

namespace bun {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ void decode(long v, int n1, int n2, int& i, int& j, int& k) {
    k = (int)(v % n2);
    const long q = v / n2;
    j = (int)(q % n1);
    i = (int)(q / n1);
}

__device__ __forceinline__ float block_sum(float x, float* sh) {
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = x;
    __syncthreads();
    x = 0.f;
    if (warp == 0) {
        x = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.f;
        for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    }
    return x;
}

// a0[v][c] = relu(b[c] + sum_t w[t][c] x[v + off(t)])   (1 -> 16 channels)
// A block owns kInJ rows x kInK voxels of one plane: it stages the input
// tile with its one-voxel halo (zero outside the grid) in shared memory
// once, so each input value is read from memory about once instead of 27
// times.  A thread forms four voxels (rows tj, tj + kInJ/4, ...), reading
// each tap's weights four channels at a time, so one shared-memory load
// feeds sixteen FMAs.
constexpr int kInK = 64, kInJ = 16;  // kInK * kInJ == 4 * kBlock
__global__ void __launch_bounds__(kBlock) k_conv_in(int n0, int n1, int n2, const float* __restrict__ x,
                                                    const float* __restrict__ w, const float* __restrict__ b,
                                                    bf16* __restrict__ out) {
    __shared__ __align__(16) float sw[27 * 16 + 16];
    __shared__ float sx[3][kInJ + 2][kInK + 2];
    for (int q = threadIdx.x; q < 27 * 16; q += blockDim.x) sw[q] = w[q];
    if (threadIdx.x < 16) sw[27 * 16 + threadIdx.x] = b[threadIdx.x];
    const int k0 = blockIdx.x * kInK, j0 = blockIdx.y * kInJ, i = blockIdx.z;
    constexpr int PL = (kInJ + 2) * (kInK + 2);
    for (int q = threadIdx.x; q < 3 * PL; q += blockDim.x) {
        const int di = q / PL, r = q - di * PL, dj = r / (kInK + 2), dk = r - dj * (kInK + 2);
        const int ii = i + di - 1, jj = j0 + dj - 1, kk = k0 + dk - 1;
        const bool in = ii >= 0 && ii < n0 && jj >= 0 && jj < n1 && kk >= 0 && kk < n2;
        sx[di][dj][dk] = in ? x[((long)ii * n1 + jj) * n2 + kk] : 0.f;
    }
    __syncthreads();
    constexpr int RJ = kInJ / 4;  // rows between a thread's voxels
    const int tk = threadIdx.x % kInK, tj = threadIdx.x / kInK;
    float acc[4][16];
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[u][c] = sw[27 * 16 + c];
#pragma unroll 1
    for (int t = 0; t < 27; ++t) {
        const int di = t / 9, dj = (t / 3) % 3, dk = t % 3;
        float xv[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) xv[u] = sx[di][tj + u * RJ + dj][tk + dk];
        const float4* wt = reinterpret_cast<const float4*>(sw + t * 16);
#pragma unroll
        for (int g = 0; g < 4; ++g) {
            const float4 wv = wt[g];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                acc[u][4 * g] += wv.x * xv[u];
                acc[u][4 * g + 1] += wv.y * xv[u];
                acc[u][4 * g + 2] += wv.z * xv[u];
                acc[u][4 * g + 3] += wv.w * xv[u];
            }
        }
    }
    const int k = k0 + tk;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int j = j0 + tj + u * RJ;
        if (j >= n1 || k >= n2) continue;
        uint4 ov[2];
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(ov);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            o[q] = __floats2bfloat162_rn(fmaxf(acc[u][2 * q], 0.f), fmaxf(acc[u][2 * q + 1], 0.f));
        uint4* op = reinterpret_cast<uint4*>(out + (((long)i * n1 + j) * n2 + k) * 16);
        op[0] = ov[0];
        op[1] = ov[1];
    }
}

// partials of dW[t][c] = sum_v x[v+off(t)] dz[v][c] (t < 27) and db[c] =
// sum_v dz[v][c] (t = 27): grid (nblocks, 28), part[blk][t*16 + c]
__global__ void __launch_bounds__(kBlock) k_conv_in_wgrad(int n0, int n1, int n2, const float* __restrict__ x,
                                                          const bf16* __restrict__ dz, float* __restrict__ part) {
    __shared__ float sh[kBlock / 32];
    const int t = blockIdx.y;
    const long V = (long)n0 * n1 * n2;
    float acc[16];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc[c] = 0.f;
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
        float xv = 1.f;
        if (t < 27) {
            int i, j, k;
            decode(v, n1, n2, i, j, k);
            const int ii = i + t / 9 - 1, jj = j + (t / 3) % 3 - 1, kk = k + t % 3 - 1;
            xv = (ii < 0 || ii >= n0 || jj < 0 || jj >= n1 || kk < 0 || kk >= n2) ? 0.f
                                                                                 : x[((long)ii * n1 + jj) * n2 + kk];
        }
        const uint4* dp = reinterpret_cast<const uint4*>(dz + v * 16);
        uint4 dv[2] = {dp[0], dp[1]};
        const bf16* d = reinterpret_cast<const bf16*>(dv);
#pragma unroll
        for (int c = 0; c < 16; ++c) acc[c] += xv * __bfloat162float(d[c]);
    }
    float* dst = part + (long)blockIdx.x * (28 * 16) + t * 16;
#pragma unroll
    for (int c = 0; c < 16; ++c) {
        const float s = block_sum(acc[c], sh);
        if (threadIdx.x == 0) dst[c] = s;
    }
}

// y[v] = b + sum_c w[c] d[v][c]    (16 -> 1 channel, 1x1x1)
__global__ void __launch_bounds__(kBlock) k_head(long V, const bf16* __restrict__ d, const float* __restrict__ w,
                                                 const float* __restrict__ b, float* __restrict__ y) {
    const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    const uint4* dp = reinterpret_cast<const uint4*>(d + v * 16);
    uint4 dv[2] = {dp[0], dp[1]};
    const bf16* e = reinterpret_cast<const bf16*>(dv);
    float acc = b[0];
#pragma unroll
    for (int c = 0; c < 16; ++c) acc += w[c] * __bfloat162float(e[c]);
    y[v] = acc;
}

// dz[v][c] = dy[v] w[c] (d[v][c] > 0); partials of dW[c] = sum dy d and db
__global__ void __launch_bounds__(kBlock) k_head_grad(long V, const bf16* __restrict__ d,
                                                      const float* __restrict__ dy, const float* __restrict__ w,
                                                      bf16* __restrict__ dz, float* __restrict__ part) {
    __shared__ float sh[kBlock / 32];
    float acc[17];
#pragma unroll
    for (int c = 0; c < 17; ++c) acc[c] = 0.f;
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < V; v += (long)gridDim.x * blockDim.x) {
        const uint4* dp = reinterpret_cast<const uint4*>(d + v * 16);
        uint4 dv[2] = {dp[0], dp[1]};
        const bf16* e = reinterpret_cast<const bf16*>(dv);
        const float g = dy[v];
        uint4 ov[2];
        __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(ov);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const float a0 = __bfloat162float(e[2 * q]), a1 = __bfloat162float(e[2 * q + 1]);
            o[q] = __floats2bfloat162_rn(a0 > 0.f ? g * w[2 * q] : 0.f, a1 > 0.f ? g * w[2 * q + 1] : 0.f);
            acc[2 * q] += g * a0;
            acc[2 * q + 1] += g * a1;
        }
        acc[16] += g;
        uint4* op = reinterpret_cast<uint4*>(dz + v * 16);
        op[0] = ov[0];
        op[1] = ov[1];
    }
#pragma unroll
    for (int c = 0; c < 17; ++c) {
        const float s = block_sum(acc[c], sh);
        if (threadIdx.x == 0) part[(long)blockIdx.x * 17 + c] = s;
    }
}

// p[w][c] = mean of the 8 children of coarse voxel w (fine grid n0 x n1 x n2)
__global__ void __launch_bounds__(kBlock) k_pool(int n0, int n1, int n2, int C, const bf16* __restrict__ s,
                                                 bf16* __restrict__ p) {
    const int m0 = n0 / 2, m1 = n1 / 2, m2 = n2 / 2;
    const long total = (long)m0 * m1 * m2 * (C / 2);
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total) return;
    const int c2 = (int)(q % (C / 2));
    const long w = q / (C / 2);
    int I, J, K;
    decode(w, m1, m2, I, J, K);
    float a0 = 0.f, a1 = 0.f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const long f = ((long)(2 * I + (o >> 2)) * n1 + 2 * J + ((o >> 1) & 1)) * n2 + 2 * K + (o & 1);
        const float2 v = __bfloat1622float2(reinterpret_cast<const __nv_bfloat162*>(s + f * C)[c2]);
        a0 += v.x;
        a1 += v.y;
    }
    reinterpret_cast<__nv_bfloat162*>(p + w * C)[c2] = __floats2bfloat162_rn(0.125f * a0, 0.125f * a1);
}

// gradient of the upsampled part of a concatenated input: for coarse voxel
// w and channel c < c0, dz[w][c] = (sum over children of dcat[f][c]) *
// (act[w][c] > 0)
__global__ void __launch_bounds__(kBlock) k_unpool_grad(int n0, int n1, int n2, int ccat, int c0,
                                                        const bf16* __restrict__ dcat,
                                                        const bf16* __restrict__ act, bf16* __restrict__ dz) {
    const int m0 = n0 / 2, m1 = n1 / 2, m2 = n2 / 2;
    const long total = (long)m0 * m1 * m2 * c0;
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total) return;
    const int c = (int)(q % c0);
    const long w = q / c0;
    int I, J, K;
    decode(w, m1, m2, I, J, K);
    float a = 0.f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const long f = ((long)(2 * I + (o >> 2)) * n1 + 2 * J + ((o >> 1) & 1)) * n2 + 2 * K + (o & 1);
        a += __bfloat162float(dcat[f * ccat + c]);
    }
    dz[w * c0 + c] = __float2bfloat16_rn(__bfloat162float(act[w * c0 + c]) > 0.f ? a : 0.f);
}

// gradient of a skip tensor s (C channels, fine grid), used both by the
// decoder's concatenation (channels [c0, c0 + C) of dcat) and by the pooling
// that feeds the next encoder level (dp, coarse grid):
//   dz[v][c] = (s[v][c] > 0) * (dcat[v][c0 + c] + dp[parent(v)][c] / 8)
__global__ void __launch_bounds__(kBlock) k_skip_grad(int n0, int n1, int n2, int ccat, int c0, int C,
                                                      const bf16* __restrict__ dcat, const bf16* __restrict__ dp,
                                                      const bf16* __restrict__ s, bf16* __restrict__ dz) {
    const long total = (long)n0 * n1 * n2 * C;
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total) return;
    const int c = (int)(q % C);
    const long v = q / C;
    int i, j, k;
    decode(v, n1, n2, i, j, k);
    const long w = ((long)(i >> 1) * (n1 >> 1) + (j >> 1)) * (n2 >> 1) + (k >> 1);
    const float g = __bfloat162float(dcat[v * ccat + c0 + c]) + 0.125f * __bfloat162float(dp[w * C + c]);
    dz[v * C + c] = __float2bfloat16_rn(__bfloat162float(s[v * C + c]) > 0.f ? g : 0.f);
}

// dy = 2 (y - t) / n; partials of sum (y - t)^2
__global__ void __launch_bounds__(kBlock) k_mse(long n, const float* __restrict__ y, const float* __restrict__ t,
                                                float* __restrict__ dy, float* __restrict__ part) {
    __shared__ float sh[kBlock / 32];
    float acc = 0.f;
    const float sc = 2.f / (float)n;
    for (long v = (long)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (long)gridDim.x * blockDim.x) {
        const float e = y[v] - t[v];
        dy[v] = sc * e;
        acc += e * e;
    }
    acc = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = acc;
}

// out[q] = scale * sum_p part[p * stride + q], p in fixed order
__global__ void __launch_bounds__(kBlock) k_sum_parts(const float* __restrict__ part, int nparts, long stride,
                                                      long len, float scale, float* __restrict__ out) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= len) return;
    float a = 0.f;
    for (int p = 0; p < nparts; ++p) a += part[(long)p * stride + q];
    out[q] = scale * a;
}

// packed weights of one tensor-core convolution.  Forward (transpose = 0):
// GEMM K = cin, N = cout, element (n = co, c = ci) of block (t, g) holds
// W[t][g*kc + c][co].  Data gradient (transpose = 1): K = cout, N = cin,
// element (n = ci, c = co) of block (t, g) holds W[26 - t][ci][g*kc + c].
// Inside a block: element (n/8)*(kc*8) + (c/8)*64 + (n%8)*8 + (c%8).
__global__ void __launch_bounds__(kBlock) k_pack(const float* __restrict__ w, int cin, int cout, int kc,
                                                 int transpose, bf16* __restrict__ out) {
    const int K = transpose ? cout : cin, N = transpose ? cin : cout;
    const long total = 27L * K * N;
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= total) return;
    const long blk = q / ((long)N * kc);
    const int r = (int)(q % ((long)N * kc));
    const int ng = r / (kc * 8);
    const int r2 = r % (kc * 8);
    const int cg = r2 / 64, r3 = r2 % 64;
    const int nr = r3 / 8, cr = r3 % 8;
    const int n = ng * 8 + nr, c = cg * 8 + cr;
    const int t = (int)(blk / (K / kc)), g = (int)(blk % (K / kc));
    float val;
    if (!transpose)
        val = w[((long)t * cin + g * kc + c) * cout + n];
    else
        val = w[((long)(26 - t) * cin + n) * cout + g * kc + c];
    out[q] = __float2bfloat16_rn(val);
}

// Adam (Kingma and Ba, 2015) with bias correction, on FP32 master weights
__global__ void __launch_bounds__(kBlock) k_adam(long n, float* __restrict__ w, const float* __restrict__ g,
                                                 float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                                                 float b2, float eps, float c1, float c2) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float gq = g[q];
    const float mq = b1 * m[q] + (1.f - b1) * gq;
    const float vq = b2 * v[q] + (1.f - b2) * gq * gq;
    m[q] = mq;
    v[q] = vq;
    w[q] -= lr * (mq / c1) / (sqrtf(vq / c2) + eps);
}

__global__ void __launch_bounds__(kBlock) k_to_float(long n, const double* __restrict__ x, double scale,
                                                     float* __restrict__ y) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) y[q] = (float)(scale * x[q]);
}

__global__ void __launch_bounds__(kBlock) k_to_double(long n, const float* __restrict__ x, double scale,
                                                      double* __restrict__ y) {
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < n) y[q] = scale * (double)x[q];
}

// partials of sum x^2 (FP64)
__global__ void __launch_bounds__(kBlock) k_sumsq(long n, const double* __restrict__ x, double* __restrict__ part) {
    __shared__ double sh[kBlock / 32];
    double a = 0.0;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        a += x[q] * x[q];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < kBlock / 32; ++q) s += sh[q];
        part[blockIdx.x] = s;
    }
}

__global__ void k_sum_double(const double* __restrict__ part, int n, double* __restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int q = 0; q < n; ++q) s += part[q];
        *out = s;
    }
}

// r = sum over the (up to six) in-grid neighbours of (y_nb - y) + c * f:
// the h^2-scaled residual of the uniform-grid Neumann Laplacian for a
// network output y and the network input f (c: h^2 over the target scale)
__global__ void __launch_bounds__(kBlock) k_lap_residual(int n0, int n1, int n2, const float* __restrict__ y,
                                                         const float* __restrict__ f, float c, float* __restrict__ r) {
    const long V = (long)n0 * n1 * n2;
    const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    int i, j, k;
    decode(v, n1, n2, i, j, k);
    const float yc = y[v];
    float s = 0.f;
    if (i > 0) s += y[v - (long)n1 * n2] - yc;
    if (i < n0 - 1) s += y[v + (long)n1 * n2] - yc;
    if (j > 0) s += y[v - n2] - yc;
    if (j < n1 - 1) s += y[v + n2] - yc;
    if (k > 0) s += y[v - 1] - yc;
    if (k < n2 - 1) s += y[v + 1] - yc;
    r[v] = s + c * f[v];
}

// dy += w * (the same stencil applied to g): the adjoint of the residual's
// y-part, which is symmetric
__global__ void __launch_bounds__(kBlock) k_lap_add(int n0, int n1, int n2, const float* __restrict__ g, float w,
                                                    float* __restrict__ dy) {
    const long V = (long)n0 * n1 * n2;
    const long v = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= V) return;
    int i, j, k;
    decode(v, n1, n2, i, j, k);
    const float gc = g[v];
    float s = 0.f;
    if (i > 0) s += g[v - (long)n1 * n2] - gc;
    if (i < n0 - 1) s += g[v + (long)n1 * n2] - gc;
    if (j > 0) s += g[v - n2] - gc;
    if (j < n1 - 1) s += g[v + n2] - gc;
    if (k > 0) s += g[v - 1] - gc;
    if (k < n2 - 1) s += g[v + 1] - gc;
    dy[v] += w * s;
}

inline unsigned blocks_for(long n) { return (unsigned)((n + kBlock - 1) / kBlock); }

}  // namespace

cudaError_t conv_in_launch(int n0, int n1, int n2, const float* x, const float* w, const float* b, bf16* out,
                           cudaStream_t s) {
    const dim3 grid((unsigned)((n2 + kInK - 1) / kInK), (unsigned)((n1 + kInJ - 1) / kInJ), (unsigned)n0);
    k_conv_in<<<grid, kBlock, 0, s>>>(n0, n1, n2, x, w, b, out);
    return cudaGetLastError();
}

cudaError_t conv_in_wgrad_launch(int n0, int n1, int n2, const float* x, const bf16* dz, float* part, int nblocks,
                                 float* dw, cudaStream_t s) {
    k_conv_in_wgrad<<<dim3((unsigned)nblocks, 28), kBlock, 0, s>>>(n0, n1, n2, x, dz, part);
    k_sum_parts<<<blocks_for(28 * 16), kBlock, 0, s>>>(part, nblocks, 28 * 16, 28 * 16, 1.f, dw);
    return cudaGetLastError();
}

cudaError_t head_launch(long n, const bf16* d, const float* w, const float* b, float* y, cudaStream_t s) {
    k_head<<<blocks_for(n), kBlock, 0, s>>>(n, d, w, b, y);
    return cudaGetLastError();
}

cudaError_t head_grad_launch(long n, const bf16* d, const float* dy, const float* w, bf16* dz, float* part,
                             int nblocks, float* dw, cudaStream_t s) {
    k_head_grad<<<(unsigned)nblocks, kBlock, 0, s>>>(n, d, dy, w, dz, part);
    k_sum_parts<<<1, kBlock, 0, s>>>(part, nblocks, 17, 17, 1.f, dw);
    return cudaGetLastError();
}

cudaError_t pool_launch(int n0, int n1, int n2, int C, const bf16* src, bf16* dst, cudaStream_t s) {
    k_pool<<<blocks_for((long)(n0 / 2) * (n1 / 2) * (n2 / 2) * (C / 2)), kBlock, 0, s>>>(n0, n1, n2, C, src, dst);
    return cudaGetLastError();
}

cudaError_t unpool_grad_launch(int n0, int n1, int n2, int ccat, int c0, const bf16* dcat, const bf16* act,
                               bf16* dz, cudaStream_t s) {
    k_unpool_grad<<<blocks_for((long)(n0 / 2) * (n1 / 2) * (n2 / 2) * c0), kBlock, 0, s>>>(n0, n1, n2, ccat, c0,
                                                                                          dcat, act, dz);
    return cudaGetLastError();
}

cudaError_t skip_grad_launch(int n0, int n1, int n2, int ccat, int c0, int C, const bf16* dcat, const bf16* dp,
                             const bf16* src, bf16* dz, cudaStream_t s) {
    k_skip_grad<<<blocks_for((long)n0 * n1 * n2 * C), kBlock, 0, s>>>(n0, n1, n2, ccat, c0, C, dcat, dp, src, dz);
    return cudaGetLastError();
}

cudaError_t mse_launch(long n, const float* y, const float* t, float* dy, float* part, int nblocks, float* loss,
                       cudaStream_t s) {
    k_mse<<<(unsigned)nblocks, kBlock, 0, s>>>(n, y, t, dy, part);
    k_sum_parts<<<1, kBlock, 0, s>>>(part, nblocks, 1, 1, 1.f / (float)n, loss);
    return cudaGetLastError();
}

cudaError_t sum_parts_launch(const float* part, int nparts, long stride, long len, float* out, cudaStream_t s) {
    k_sum_parts<<<blocks_for(len), kBlock, 0, s>>>(part, nparts, stride, len, 1.f, out);
    return cudaGetLastError();
}

cudaError_t pack_launch(const float* w, int cin, int cout, int kc, int transpose, bf16* out, cudaStream_t s) {
    k_pack<<<blocks_for(27L * cin * cout), kBlock, 0, s>>>(w, cin, cout, kc, transpose, out);
    return cudaGetLastError();
}

cudaError_t adam_launch(long n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2,
                        float eps, int step, cudaStream_t s) {
    const float c1 = 1.f - powf(b1, (float)step), c2 = 1.f - powf(b2, (float)step);
    k_adam<<<blocks_for(n), kBlock, 0, s>>>(n, w, g, m, v, lr, b1, b2, eps, c1, c2);
    return cudaGetLastError();
}

cudaError_t to_float_launch(long n, const double* x, double scale, float* y, cudaStream_t s) {
    k_to_float<<<blocks_for(n), kBlock, 0, s>>>(n, x, scale, y);
    return cudaGetLastError();
}

cudaError_t to_double_launch(long n, const float* x, double scale, double* y, cudaStream_t s) {
    k_to_double<<<blocks_for(n), kBlock, 0, s>>>(n, x, scale, y);
    return cudaGetLastError();
}

cudaError_t lap_residual_launch(int n0, int n1, int n2, const float* y, const float* f, float c, float* r,
                                cudaStream_t s) {
    k_lap_residual<<<blocks_for((long)n0 * n1 * n2), kBlock, 0, s>>>(n0, n1, n2, y, f, c, r);
    return cudaGetLastError();
}

cudaError_t lap_add_launch(int n0, int n1, int n2, const float* g, float w, float* dy, cudaStream_t s) {
    k_lap_add<<<blocks_for((long)n0 * n1 * n2), kBlock, 0, s>>>(n0, n1, n2, g, w, dy);
    return cudaGetLastError();
}

// ---- RMS normalisation with the scale kept on the device ---------------------
// (for a network queued inside a captured graph: no host round trip)
__global__ void __launch_bounds__(kBlock) k_sumsq32(long n, const float* __restrict__ x, double* __restrict__ part) {
    __shared__ double sh[kBlock / 32];
    double a = 0.0;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        a += (double)x[q] * (double)x[q];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) sh[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < kBlock / 32; ++q) t += sh[q];
        part[blockIdx.x] = t;
    }
}

// *rms = sqrt(sum of the parts / n), parts added in a fixed order
__global__ void k_rms_final(const double* __restrict__ part, int nparts, long n, double* rms) {
    double a = 0.0;
    for (int q = threadIdx.x; q < nparts; q += 32) a += part[q];
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (threadIdx.x == 0) *rms = sqrt(a / (double)n);
}

// y = sign * x / rms (zero when rms is zero)
__global__ void k_div_rms(long n, const float* __restrict__ x, float sign, const double* __restrict__ rms,
                          float* __restrict__ y) {
    const double r = *rms;
    const float f = r > 0.0 ? (float)(sign / r) : 0.f;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        y[q] = f * x[q];
}

// x = y * scale * rms
__global__ void k_mul_rms(long n, const float* __restrict__ y, double scale, const double* __restrict__ rms,
                          float* __restrict__ x) {
    const float f = (float)(scale * *rms);
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        x[q] = f * y[q];
}

cudaError_t rms_normalise_launch(long n, const float* x, float sign, double* part, int nblocks, double* rms,
                                 float* y, cudaStream_t s) {
    k_sumsq32<<<(unsigned)nblocks, kBlock, 0, s>>>(n, x, part);
    k_rms_final<<<1, 32, 0, s>>>(part, nblocks, n, rms);
    k_div_rms<<<blocks_for(n), kBlock, 0, s>>>(n, x, sign, rms, y);
    return cudaGetLastError();
}

cudaError_t rms_restore_launch(long n, const float* y, double scale, const double* rms, float* x, cudaStream_t s) {
    k_mul_rms<<<blocks_for(n), kBlock, 0, s>>>(n, y, scale, rms, x);
    return cudaGetLastError();
}

cudaError_t sumsq_launch(long n, const double* x, double* part, int nblocks, double* out, cudaStream_t s) {
    k_sumsq<<<(unsigned)nblocks, kBlock, 0, s>>>(n, x, part);
    k_sum_double<<<1, 32, 0, s>>>(part, nblocks, out);
    return cudaGetLastError();
}

}  // namespace bun
