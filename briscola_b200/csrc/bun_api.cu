// bun_api.cu -- C ABI of the U-Net kernels (include/bunet.h): argument
// checks, then one launcher call each.  Nothing here allocates.

#include "../../include/bunet.h"
#include "bun_api_internal.h"

#include <cstdint>

using namespace bun;

namespace {

inline cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

inline bool aligned16(const void* p) { return p && (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

inline bool dims_ok(int n0, int n1, int n2) {
    return n0 >= 1 && n1 >= 1 && n2 >= 1 && (long)n0 * n1 * n2 <= BUN_MAX_VOXELS;
}

inline int status(cudaError_t e) { return e == cudaSuccess ? BUN_OK : BUN_CUDA_ERROR; }

// the inputs of a 3x3x3 convolution; kc = 8 accepts any channel split in
// whole 16-byte chunks (the weight-gradient kernel)
bool inputs_ok(int n0, int n1, int n2, const void* src0, int c0, int up0, const void* src1, int c1, int kc) {
    if (!dims_ok(n0, n1, n2) || c0 < kc || c0 % kc || c1 < 0 || c1 % kc || !aligned16(src0)) return false;
    if (c1 > 0 && !aligned16(src1)) return false;
    if (up0 && (n0 % 2 || n1 % 2 || n2 % 2)) return false;
    return true;
}

ConvIn make_in(const void* src0, int c0, int up0, const void* src1, int c1) {
    ConvIn in;
    in.src0 = static_cast<const bf16*>(src0);
    in.src1 = static_cast<const bf16*>(c1 > 0 ? src1 : src0);
    in.c0 = c0;
    in.c1 = c1;
    in.up0 = up0 ? 1 : 0;
    return in;
}

}  // namespace

extern "C" {

int bun_conv3(int n0, int n1, int n2, const void* src0, int c0, int up0, const void* src1, int c1,
              const void* wpack, int kc, int cout, const float* bias, int relu, const void* mask, void* out,
              int* err, void* stream) {
    if (!conv_supported(kc, cout) || !inputs_ok(n0, n1, n2, src0, c0, up0, src1, c1, kc)) return BUN_BAD_ARG;
    if (!aligned16(wpack) || !aligned16(out) || (mask && !aligned16(mask))) return BUN_BAD_ARG;
    ConvArgs a;
    a.n0 = n0;
    a.n1 = n1;
    a.n2 = n2;
    a.in = make_in(src0, c0, up0, src1, c1);
    a.wpack = static_cast<const bf16*>(wpack);
    a.bias = bias;
    a.mask = static_cast<const bf16*>(mask);
    a.out = static_cast<bf16*>(out);
    a.relu = relu ? 1 : 0;
    a.err = err;
    return status(conv_launch(a, kc, cout, S(stream)));
}

int bun_conv3_stage_width(int c0, int c1, int cout, int n2) {
    const int cin = c0 + c1;
    if (rows_supported(cin, cout, n2) && c0 % 16 == 0 && c1 % 16 == 0) return 16;
    for (int kc : {64, 32, 16})
        if (c0 % kc == 0 && c1 % kc == 0 && conv_supported(kc, cout)) return kc;
    return 0;
}

size_t bun_wgrad_part_floats(int cin, int cout, int nsplit) {
    if (cin < 8 || cout < 1 || nsplit < 1) return 0;
    const size_t rows_pad = (27 * (size_t)cin + 127) / 128 * 128;
    return (size_t)nsplit * rows_pad * (size_t)cout;
}

int bun_conv3_wgrad(int n0, int n1, int n2, const void* src0, int c0, int up0, const void* src1, int c1,
                    const void* dz, int cout, int nsplit, float* part, float* dw, int* err, void* stream) {
    if (!wgrad_supported(cout) || !inputs_ok(n0, n1, n2, src0, c0, up0, src1, c1, 8)) return BUN_BAD_ARG;
    const long V = (long)n0 * n1 * n2;
    const long nblk = (V + 127) / 128;
    if (nsplit < 1 || nsplit > nblk || nsplit > 65535 || !aligned16(dz) || !aligned16(part) || !dw)
        return BUN_BAD_ARG;
    const int cin = c0 + c1;
    WgradArgs a;
    a.n0 = n0;
    a.n1 = n1;
    a.n2 = n2;
    a.in = make_in(src0, c0, up0, src1, c1);
    a.dz = static_cast<const bf16*>(dz);
    a.part = part;
    a.rows = 27 * cin;
    a.rows_pad = (a.rows + 127) / 128 * 128;
    a.nsplit = nsplit;
    a.err = err;
    cudaError_t e = wgrad_launch(a, cout, S(stream));
    if (e != cudaSuccess) return BUN_CUDA_ERROR;
    return status(sum_parts_launch(part, nsplit, (long)a.rows_pad * cout, (long)a.rows * cout, dw, S(stream)));
}

int bun_pack_weights(const float* w, int cin, int cout, int kc, int transpose, void* out, void* stream) {
    const int K = transpose ? cout : cin, N = transpose ? cin : cout;
    if (!w || !aligned16(out) || kc < 16 || K % kc || N % 16 || N < 16) return BUN_BAD_ARG;
    return status(pack_launch(w, cin, cout, kc, transpose ? 1 : 0, static_cast<bf16*>(out), S(stream)));
}

int bun_conv_in(int n0, int n1, int n2, const float* x, const float* w, const float* b, void* out, void* stream) {
    if (!dims_ok(n0, n1, n2) || !x || !w || !b || !aligned16(out)) return BUN_BAD_ARG;
    return status(conv_in_launch(n0, n1, n2, x, w, b, static_cast<bf16*>(out), S(stream)));
}

int bun_conv_in_wgrad(int n0, int n1, int n2, const float* x, const void* dz, int nblocks, float* part, float* dw,
                      void* stream) {
    if (!dims_ok(n0, n1, n2) || !x || !aligned16(dz) || nblocks < 1 || nblocks > 65535 || !part || !dw)
        return BUN_BAD_ARG;
    return status(
        conv_in_wgrad_launch(n0, n1, n2, x, static_cast<const bf16*>(dz), part, nblocks, dw, S(stream)));
}

int bun_head(long n, const void* d, const float* w, const float* b, float* y, void* stream) {
    if (n < 1 || !aligned16(d) || !w || !b || !y) return BUN_BAD_ARG;
    return status(head_launch(n, static_cast<const bf16*>(d), w, b, y, S(stream)));
}

int bun_head_grad(long n, const void* d, const float* dy, const float* w, void* dz, int nblocks, float* part,
                  float* dw, void* stream) {
    if (n < 1 || !aligned16(d) || !dy || !w || !aligned16(dz) || nblocks < 1 || !part || !dw) return BUN_BAD_ARG;
    return status(head_grad_launch(n, static_cast<const bf16*>(d), dy, w, static_cast<bf16*>(dz), part, nblocks,
                                   dw, S(stream)));
}

int bun_pool(int n0, int n1, int n2, int c, const void* src, void* dst, void* stream) {
    if (!dims_ok(n0, n1, n2) || n0 % 2 || n1 % 2 || n2 % 2 || c < 2 || c % 2 || !src || !dst) return BUN_BAD_ARG;
    return status(pool_launch(n0, n1, n2, c, static_cast<const bf16*>(src), static_cast<bf16*>(dst), S(stream)));
}

int bun_unpool_grad(int n0, int n1, int n2, int ccat, int c0, const void* dcat, const void* act, void* dz,
                    void* stream) {
    if (!dims_ok(n0, n1, n2) || n0 % 2 || n1 % 2 || n2 % 2 || c0 < 1 || ccat < c0 || !dcat || !act || !dz)
        return BUN_BAD_ARG;
    return status(unpool_grad_launch(n0, n1, n2, ccat, c0, static_cast<const bf16*>(dcat),
                                     static_cast<const bf16*>(act), static_cast<bf16*>(dz), S(stream)));
}

int bun_skip_grad(int n0, int n1, int n2, int ccat, int c0, int c, const void* dcat, const void* dp,
                  const void* src, void* dz, void* stream) {
    if (!dims_ok(n0, n1, n2) || n0 % 2 || n1 % 2 || n2 % 2 || c < 1 || ccat < c0 + c || !dcat || !dp || !src ||
        !dz)
        return BUN_BAD_ARG;
    return status(skip_grad_launch(n0, n1, n2, ccat, c0, c, static_cast<const bf16*>(dcat),
                                   static_cast<const bf16*>(dp), static_cast<const bf16*>(src),
                                   static_cast<bf16*>(dz), S(stream)));
}

int bun_mse(long n, const float* y, const float* t, float* dy, int nblocks, float* part, float* loss, void* stream) {
    if (n < 1 || !y || !t || !dy || nblocks < 1 || !part || !loss) return BUN_BAD_ARG;
    return status(mse_launch(n, y, t, dy, part, nblocks, loss, S(stream)));
}

int bun_adam(long n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2, float eps,
             int step, void* stream) {
    if (n < 1 || !w || !g || !m || !v || step < 1) return BUN_BAD_ARG;
    return status(adam_launch(n, w, g, m, v, lr, b1, b2, eps, step, S(stream)));
}

int bun_scale_to_float(long n, const double* x, double scale, float* y, void* stream) {
    if (n < 1 || !x || !y) return BUN_BAD_ARG;
    return status(to_float_launch(n, x, scale, y, S(stream)));
}

int bun_scale_to_double(long n, const float* x, double scale, double* y, void* stream) {
    if (n < 1 || !x || !y) return BUN_BAD_ARG;
    return status(to_double_launch(n, x, scale, y, S(stream)));
}

int bun_laplace_residual(int n0, int n1, int n2, const float* y, const float* f, float c, float* r, void* stream) {
    if (!dims_ok(n0, n1, n2) || !y || !f || !r) return BUN_BAD_ARG;
    return status(lap_residual_launch(n0, n1, n2, y, f, c, r, S(stream)));
}

int bun_laplace_add(int n0, int n1, int n2, const float* g, float w, float* dy, void* stream) {
    if (!dims_ok(n0, n1, n2) || !g || !dy) return BUN_BAD_ARG;
    return status(lap_add_launch(n0, n1, n2, g, w, dy, S(stream)));
}

int bun_sumsq(long n, const double* x, int nblocks, double* part, double* out, void* stream) {
    if (n < 1 || !x || nblocks < 1 || !part || !out) return BUN_BAD_ARG;
    return status(sumsq_launch(n, x, part, nblocks, out, S(stream)));
}

int bun_rms_normalise(long n, const float* x, float sign, int nblocks, double* part, double* rms, float* y,
                      void* stream) {
    if (n < 1 || !x || nblocks < 1 || !part || !rms || !y) return BUN_BAD_ARG;
    return status(rms_normalise_launch(n, x, sign, part, nblocks, rms, y, S(stream)));
}

int bun_rms_restore(long n, const float* y, double scale, const double* rms, float* x, void* stream) {
    if (n < 1 || !y || !rms || !x) return BUN_BAD_ARG;
    return status(rms_restore_launch(n, y, scale, rms, x, S(stream)));
}

}  // extern "C"
