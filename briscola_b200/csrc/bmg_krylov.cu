// bmg_krylov.cu -- flexible conjugate gradients around the multigrid cycle:
// the FP64 outer loop of a mixed-precision solve can be Krylov-accelerated
// instead of taking one cycle per correction (no counterpart in the
// reference, whose loop is MG.C:191-242).
//
// FCG(1) (Y. Notay, "Flexible conjugate gradients", SIAM J. Sci. Comput.
// 22 (2000)), with the V-weighted inner product (u, w)_V = sum V u w, in
// which the row-scaled operator A' = A/V is self-adjoint (A is symmetric):
//   r = b - A'x,  z = cycle(r)
//   beta = -(z, V q_prev) / (p_prev, V q_prev)        (0 on the first step)
//   p = z + beta p_prev,  q = A'p = A'z + beta q_prev
//   alpha = (z, V r) / (p, V q)
//   x += alpha p,  r -= alpha q
// The truncated Gram-Schmidt form tolerates a cycle that is not exactly
// symmetric or linear (red-black smoothing, FP32 arithmetic, restriction
// and prolongation that are not transposes).  A'p is formed from A'z and
// the previous q, so p needs no ghost cells.
//
// Every kernel streams level 0 once, in FP64, with one partial sum per
// block; single-block kernels add the partials in a fixed order and derive
// the scalars on the device, so the loop runs inside the solve graph.

#include <algorithm>

#include "bmg_grid.cuh"
#include "bmg_stencil.cuh"

namespace bmg {

namespace {

__device__ __forceinline__ double cell_volume(const LevelView<double>& L, int i, int j, int k) {
    return L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
}

// r = b - A'x (FP64), written to r and to the cycle's right-hand side;
// partials: ||V r||^2 and, for mode 0, the normFactor sum (as k_residual_norm)
template <bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_residual(Bricks<double> B, Walls W, int mode, double* r_out,
                                                                 float* pre32, double* pre64, double* partials,
                                                                 long nblocks) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const int bk = brick_of(B, blockIdx.z, i);
    const LevelView<double>& L = B.v[bk];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (j < L.n1 && k < L.n2) {
        const long row = row_at(L, i, j), c = row + kpos(L, k);
        double w[6];
        const long ckm = row + kpos(L, k - 1), ckp = row + kpos(L, k + 1);
        couplings<double, VAR>(L, i, j, k, c, ckp, w);
        const double xn[6] = {L.x[c - L.si], L.x[c + L.si], L.x[c - L.sj], L.x[c + L.sj], L.x[ckm], L.x[ckp]};
        const double r = res_value(w, xn, L.x[c], L.b[c]);
        const double V = cell_volume(L, i, j, k);
        a1 = (V * r) * (V * r);
        if (mode == 0) {
            const double bb = V * L.b[c];
            const double ay =
                W.mask[bk] ? -V * *W.ybar * wall_sum(L, W, bk, i, j, k, c, ckp, false) : 0.0;
            const double t = fabs(V * r - bb + ay) + fabs(bb - ay);
            a2 = t * t;
            a3 = bb * bb;
        }
        if (mode != 2) {
            r_out[c] = r;
            if (pre32) pre32[c] = (float)r;
            if (pre64) pre64[c] = r;
        }
    }
    const long bid = block_id();
    a1 = block_sum<kReduceThreads>(a1, sh);
    if (mode == 0) {
        a2 = block_sum<kReduceThreads>(a2, sh);
        a3 = block_sum<kReduceThreads>(a3, sh);
    }
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        partials[bid] = a1;
        if (mode == 0) {
            partials[nblocks + bid] = a2;
            partials[2 * nblocks + bid] = a3;
        }
    }
}

// partials of (z, V r) and (z, V q)
template <typename T>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_dots(Bricks<double> B, const T* z, const double* r,
                                                             const double* q, double* partials, long nblocks) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a1 = 0.0, a2 = 0.0;
    if (j < L.n1 && k < L.n2) {
        const long row = row_at(L, i, j), c = row + kpos(L, k);
        const double Vz = cell_volume(L, i, j, k) * (double)z[c];
        a1 = Vz * r[c];
        a2 = Vz * q[c];
    }
    a1 = block_sum<kReduceThreads>(a1, sh);
    a2 = block_sum<kReduceThreads>(a2, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const long bid = block_id();
        partials[bid] = a1;
        partials[nblocks + bid] = a2;
    }
}

__global__ void __launch_bounds__(kFinalThreads) k_fcg_beta(const double* partials, long nblocks,
                                                            SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double a1 = sum_partials<kFinalThreads>(partials, nblocks, sh);
    const double a2 = sum_partials<kFinalThreads>(partials + nblocks, nblocks, sh);
    if (threadIdx.x == 0) {
        st->gamma = a1;
        st->beta = st->first ? 0.0 : -a2 / st->pq;
        st->first = 0;
    }
}

// p = z + beta p, q = A'z + beta q; partials of (p, V q)
template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_direction(Bricks<double> B, const T* z, double* p,
                                                                  double* q, double* partials,
                                                                  const SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a = 0.0;
    if (j < L.n1 && k < L.n2) {
        const double beta = st->beta;
        const long row = row_at(L, i, j), c = row + kpos(L, k);
        double w[6];
        const long ckm = row + kpos(L, k - 1), ckp = row + kpos(L, k + 1);
        couplings<double, VAR>(L, i, j, k, c, ckp, w);
        const double zc = (double)z[c];
        const double s = w[0] * (double)z[c - L.si] + w[1] * (double)z[c + L.si] + w[2] * (double)z[c - L.sj] +
                         w[3] * (double)z[c + L.sj] + w[4] * (double)z[ckm] + w[5] * (double)z[ckp];
        const double d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
        // on the first step p and q hold whatever the last solve left
        const double pn = beta != 0.0 ? zc + beta * p[c] : zc;
        const double qn = beta != 0.0 ? (s - d * zc) + beta * q[c] : s - d * zc;
        p[c] = pn;
        q[c] = qn;
        a = cell_volume(L, i, j, k) * pn * qn;
    }
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

__global__ void __launch_bounds__(kFinalThreads) k_fcg_alpha(const double* partials, long nblocks,
                                                             SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double a = sum_partials<kFinalThreads>(partials, nblocks, sh);
    if (threadIdx.x == 0) {
        st->pq = a;
        st->alpha = st->gamma / a;
    }
}

// x += alpha p, r -= alpha q, cycle right-hand side = r; partials ||V r||^2
__global__ void __launch_bounds__(kReduceThreads) k_fcg_update(Bricks<double> B, const double* p, double* r,
                                                               const double* q, float* pre32, double* pre64,
                                                               double* partials, const SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a = 0.0;
    if (j < L.n1 && k < L.n2) {
        const double alpha = st->alpha;
        const long row = row_at(L, i, j), c = row + kpos(L, k);
        store_x(L, c, i, j, k, L.x[c] + alpha * p[c]);
        const double rn = r[c] - alpha * q[c];
        r[c] = rn;
        if (pre32) pre32[c] = (float)rn;
        if (pre64) pre64[c] = rn;
        const double Vr = cell_volume(L, i, j, k) * rn;
        a = Vr * Vr;
    }
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

__global__ void __launch_bounds__(kFinalThreads) k_fcg_true_norm(const double* partials, long nblocks,
                                                                 SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double a = sum_partials<kFinalThreads>(partials, nblocks, sh);
    if (threadIdx.x == 0) st->l2_true = sqrt(a);
}

// ---- quad versions: a thread owns the k-quad of one row (four cells, vector
// loads) and the grid strides over the planes, so a reduction leaves few
// per-block partials for the one-block kernels to add.  Same per-cell
// arithmetic as the kernels above; used when every brick's n2 % 4 == 0.

constexpr int kQuadPlanes = 64;  // grid z: plane groups

// The logical k-quad k0 .. k0+3 at slab index p (its first cell): one
// vector in a natural row (kh = 0); in a parity-split row the even pair
// (k0, k0+2) at p and the odd pair (k0+1, k0+3) at p + kh.
template <typename T>
struct Quad4;
template <>
struct Quad4<double> {
    static __device__ __forceinline__ void ld(const double* p, int kh, double v[4]) {
        const double2 a = reinterpret_cast<const double2*>(p)[0];
        const double2 b = *reinterpret_cast<const double2*>(p + (kh ? kh : 2));
        v[0] = a.x;
        v[1] = kh ? b.x : a.y;
        v[2] = kh ? a.y : b.x;
        v[3] = b.y;
    }
    static __device__ __forceinline__ void st(double* p, int kh, const double v[4]) {
        reinterpret_cast<double2*>(p)[0] = kh ? make_double2(v[0], v[2]) : make_double2(v[0], v[1]);
        *reinterpret_cast<double2*>(p + (kh ? kh : 2)) = kh ? make_double2(v[1], v[3]) : make_double2(v[2], v[3]);
    }
};
template <>
struct Quad4<float> {
    static __device__ __forceinline__ void ld(const float* p, int kh, float v[4]) {
        if (kh) {
            const float2 a = reinterpret_cast<const float2*>(p)[0];
            const float2 b = *reinterpret_cast<const float2*>(p + kh);
            v[0] = a.x;
            v[1] = b.x;
            v[2] = a.y;
            v[3] = b.y;
        } else {
            const float4 a = *reinterpret_cast<const float4*>(p);
            v[0] = a.x;
            v[1] = a.y;
            v[2] = a.z;
            v[3] = a.w;
        }
    }
    static __device__ __forceinline__ void st(float* p, int kh, const float v[4]) {
        if (kh) {
            reinterpret_cast<float2*>(p)[0] = make_float2(v[0], v[2]);
            *reinterpret_cast<float2*>(p + kh) = make_float2(v[1], v[3]);
        } else {
            *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
        }
    }
};

// the quad grid: x over k-quads (16 per block), y over rows (16 per block),
// z over plane groups; every thread visits planes z, z + gridDim.z, ...
#define BMG_QUAD_LOOP(B, ...)                                                              \
    {                                                                                      \
        const int qx = blockIdx.x * blockDim.x + threadIdx.x;                              \
        const int j = blockIdx.y * blockDim.y + threadIdx.y;                               \
        for (int zp = blockIdx.z; zp < (B).z0[(B).nb]; zp += gridDim.z) {                  \
            int i;                                                                         \
            const LevelView<double>& L = (B).v[brick_of((B), zp, i)];                      \
            const int k0 = 4 * qx;                                                         \
            if (j < L.n1 && k0 < L.n2) {                                                   \
                const long row = row_at(L, i, j), c = row + kpos(L, k0);                   \
                const int ks = L.kh;                                                       \
                const double hij = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j];        \
                double hk[4];                                                              \
                Quad4<double>::ld(L.tab64 + L.to.h[2] + k0, 0, hk);                        \
                __VA_ARGS__                                                                \
            }                                                                              \
        }                                                                                  \
    }

// ---- two passes per flexible-CG step (the FCG(1) recurrences above with
// one reduction): pass 1 forms (z, V r), (z, V q_prev) and (z, V A'z), A'z
// by the stencil on z; k_fcg_coeffs derives beta = -(z, V q_prev) /
// (p_prev, V q_prev) and, since V A' is symmetric (so (p_prev, V A'z) =
// (z, V q_prev)),
//   (p, V q) = (z, V A'z) + 2 beta (z, V q_prev) + beta^2 (p_prev, V q_prev)
//            = (z, V A'z) + beta (z, V q_prev),
// and alpha = (z, V r) / (p, V q); pass 2 forms A'z again and updates p, q,
// x and r in one sweep, writes the cycle's right-hand side and the partials
// of ||V r||^2.  Per cell the streams are z, r, q (pass 1) and z, p, q, x,
// r in, p, q, x, r and the FP32 right-hand side out (pass 2).

// A'z of the quad at c (natural or split rows), the k couplings of the four
// cells, and their volumes: the stencil of k_fcg_direction4
#define BMG_QUAD_AZ(z, Az, zc)                                                                         \
    T zc[4], zim_[4], zip_[4], zjm_[4], zjp_[4];                                                        \
    Quad4<T>::ld(z + c, ks, zc);                                                                        \
    Quad4<T>::ld(z + c - L.si, ks, zim_);                                                               \
    Quad4<T>::ld(z + c + L.si, ks, zip_);                                                               \
    Quad4<T>::ld(z + c - L.sj, ks, zjm_);                                                               \
    Quad4<T>::ld(z + c + L.sj, ks, zjp_);                                                               \
    const long cr_ = row + kpos(L, k0 + 4);                                                             \
    const T zl_ = z[row + kpos(L, k0 - 1)], zr_ = z[cr_];                                               \
    double Az[4];                                                                                      \
    for (int e = 0; e < 4; ++e) {                                                                       \
        double w[6];                                                                                    \
        couplings<double, VAR>(L, i, j, k0 + e, c + quad_off(ks, e), e < 3 ? c + quad_off(ks, e + 1) : cr_, w); \
        const double km = e > 0 ? (double)zc[e - 1] : (double)zl_;                                      \
        const double kp = e < 3 ? (double)zc[e + 1] : (double)zr_;                                      \
        const double sv = w[0] * (double)zim_[e] + w[1] * (double)zip_[e] + w[2] * (double)zjm_[e] +     \
                          w[3] * (double)zjp_[e] + w[4] * km + w[5] * kp;                               \
        const double d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];                                       \
        Az[e] = sv - d * (double)zc[e];                                                                 \
    }

template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_dots3_4(Bricks<double> B, const T* z, const double* r,
                                                                const double* q, double* partials, long nblocks) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
    BMG_QUAD_LOOP(B, {
        BMG_QUAD_AZ(z, Az, zc)
        double rq[4], qq[4];
        Quad4<double>::ld(r + c, ks, rq);
        Quad4<double>::ld(q + c, ks, qq);
        for (int e = 0; e < 4; ++e) {
            const double Vz = (hij * hk[e]) * (double)zc[e];
            a1 += Vz * rq[e];
            a2 += Vz * qq[e];
            a3 += Vz * Az[e];
        }
    })
    a1 = block_sum<kReduceThreads>(a1, sh);
    a2 = block_sum<kReduceThreads>(a2, sh);
    a3 = block_sum<kReduceThreads>(a3, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const long bid = block_id();
        partials[bid] = a1;
        partials[nblocks + bid] = a2;
        partials[2 * nblocks + bid] = a3;
    }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_step4(Bricks<double> B, const T* z, double* p, double* q,
                                                              double* r, float* pre32, double* pre64,
                                                              double* partials, const SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    const double beta = st->beta, alpha = st->alpha;
    double a = 0.0;
    BMG_QUAD_LOOP(B, {
        BMG_QUAD_AZ(z, Az, zc)
        double pq[4], qq[4], xq[4], rq[4], rn[4];
        Quad4<double>::ld(p + c, ks, pq);
        Quad4<double>::ld(q + c, ks, qq);
        Quad4<double>::ld(L.x + c, ks, xq);
        Quad4<double>::ld(r + c, ks, rq);
        for (int e = 0; e < 4; ++e) {
            // on the first step p and q hold whatever the last solve left
            const double pn = beta != 0.0 ? (double)zc[e] + beta * pq[e] : (double)zc[e];
            const double qn = beta != 0.0 ? Az[e] + beta * qq[e] : Az[e];
            pq[e] = pn;
            qq[e] = qn;
            xq[e] = xq[e] + alpha * pn;
            rn[e] = rq[e] - alpha * qn;
            const double Vr = (hij * hk[e]) * rn[e];
            a += Vr * Vr;
        }
        Quad4<double>::st(p + c, ks, pq);
        Quad4<double>::st(q + c, ks, qq);
        Quad4<double>::st(L.x + c, ks, xq);
        if (quad_has_images(L, i, j, k0)) {
            for (int e = 0; e < 4; ++e) store_images(L, c + quad_off(ks, e), i, j, k0 + e, xq[e]);
        }
        Quad4<double>::st(r + c, ks, rn);
        if (pre32) {
            const float f[4] = {(float)rn[0], (float)rn[1], (float)rn[2], (float)rn[3]};
            Quad4<float>::st(pre32 + c, ks, f);
        }
        if (pre64) Quad4<double>::st(pre64 + c, ks, rn);
    })
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

#undef BMG_QUAD_AZ

// The two passes on a parity-split level 0 (one brick): the thread owns four
// consecutive positions of one half of a row, the cells k = 2 (m0 + e) + h of
// one parity (as k_fcg_direction_split), so z, its neighbours and the FP64
// vectors load as whole vectors.
#define BMG_SPLIT_AZ                                                                                   \
    const int h = 4 * qx >= kh ? 1 : 0;                                                                 \
    const int m0 = 4 * qx - h * kh;                                                                     \
    const long row = row_at(L, i, j), c = row + 4 * qx;                                                 \
    const long co = row + (1 - h) * kh + m0; /* the other half, same slots */                          \
    const long ce = h == 0 ? (m0 > 0 ? co - 1 : row - 1) : (m0 + 4 < kh ? co + 4 : row + 2 * kh);       \
    T zc[4], zo[4], zim[4], zip[4], zjm[4], zjp[4];                                                     \
    Quad4<T>::ld(z + c, 0, zc);                                                                         \
    Quad4<T>::ld(z + co, 0, zo);                                                                        \
    Quad4<T>::ld(z + c - L.si, 0, zim);                                                                 \
    Quad4<T>::ld(z + c + L.si, 0, zip);                                                                 \
    Quad4<T>::ld(z + c - L.sj, 0, zjm);                                                                 \
    Quad4<T>::ld(z + c + L.sj, 0, zjp);                                                                 \
    const T ze = z[ce];                                                                                 \
    const double wil = L.tab64[L.to.wl[0] + i], wih = L.tab64[L.to.wh[0] + i];                          \
    const double hij = L.tab64[L.to.h[0] + i] * hj;                                                     \
    double wkl[4], wkh[4], hk[4];                                                                      \
    Quad4<double>::ld(L.tab64 + L.to.kwl + 4 * qx, 0, wkl);                                            \
    Quad4<double>::ld(L.tab64 + L.to.kwh + 4 * qx, 0, wkh);                                            \
    Quad4<double>::ld(L.tab64 + L.to.ksz + 4 * qx, 0, hk);                                             \
    double l0[4], l0p[4], l1[4], l1p[4], l2[4], l2o[4], l2e = 1.0;                                      \
    if (VAR) {                                                                                          \
        Quad4<double>::ld(L.lam0 + c, 0, l0);                                                           \
        Quad4<double>::ld(L.lam0 + c + L.si, 0, l0p);                                                   \
        Quad4<double>::ld(L.lam1 + c, 0, l1);                                                           \
        Quad4<double>::ld(L.lam1 + c + L.sj, 0, l1p);                                                   \
        Quad4<double>::ld(L.lam2 + c, 0, l2);                                                           \
        Quad4<double>::ld(L.lam2 + co, 0, l2o);                                                         \
        l2e = L.lam2[ce];                                                                               \
    }                                                                                                   \
    double Az[4];                                                                                      \
    for (int e = 0; e < 4; ++e) {                                                                       \
        double w[6] = {wil, wih, wjl, wjh, wkl[e], wkh[e]};                                             \
        if (VAR) {                                                                                      \
            w[0] *= l0[e];                                                                              \
            w[1] *= l0p[e];                                                                             \
            w[2] *= l1[e];                                                                              \
            w[3] *= l1p[e];                                                                             \
            w[4] *= l2[e];                                                                              \
            w[5] *= h == 0 ? l2o[e] : (e < 3 ? l2o[e + 1] : l2e);                                       \
        }                                                                                               \
        const double km = h == 0 ? (double)(e == 0 ? ze : zo[e - 1]) : (double)zo[e];                   \
        const double kp = h == 0 ? (double)zo[e] : (double)(e == 3 ? ze : zo[e + 1]);                   \
        const double sv = w[0] * (double)zim[e] + w[1] * (double)zip[e] + w[2] * (double)zjm[e] +        \
                          w[3] * (double)zjp[e] + w[4] * km + w[5] * kp;                                \
        const double d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];                                       \
        Az[e] = sv - d * (double)zc[e];                                                                 \
    }

#define BMG_SPLIT_LOOP(...)                                                                            \
    {                                                                                                   \
        const LevelView<double>& L = B.v[0];                                                            \
        const int qx = blockIdx.x * blockDim.x + threadIdx.x;                                           \
        const int j = blockIdx.y * blockDim.y + threadIdx.y;                                            \
        const int kh = L.kh;                                                                            \
        if (j < L.n1 && 4 * qx < L.n2) {                                                                \
            const double wjl = L.tab64[L.to.wl[1] + j], wjh = L.tab64[L.to.wh[1] + j];                  \
            const double hj = L.tab64[L.to.h[1] + j];                                                   \
            for (int i = blockIdx.z; i < L.n0; i += gridDim.z) {                                        \
                BMG_SPLIT_AZ                                                                            \
                __VA_ARGS__                                                                             \
            }                                                                                           \
        }                                                                                               \
    }

template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads, VAR ? 2 : 3) k_fcg_dots3_split(Bricks<double> B, const T* z,
                                                                                  const double* r, const double* q,
                                                                                  double* partials, long nblocks) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
    BMG_SPLIT_LOOP({
        double rq[4], qq[4];
        Quad4<double>::ld(r + c, 0, rq);
        Quad4<double>::ld(q + c, 0, qq);
        for (int e = 0; e < 4; ++e) {
            const double Vz = (hij * hk[e]) * (double)zc[e];
            a1 += Vz * rq[e];
            a2 += Vz * qq[e];
            a3 += Vz * Az[e];
        }
    })
    a1 = block_sum<kReduceThreads>(a1, sh);
    a2 = block_sum<kReduceThreads>(a2, sh);
    a3 = block_sum<kReduceThreads>(a3, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const long bid = block_id();
        partials[bid] = a1;
        partials[nblocks + bid] = a2;
        partials[2 * nblocks + bid] = a3;
    }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads, VAR ? 2 : 3) k_fcg_step_split(Bricks<double> B, const T* z,
                                                                                 double* p, double* q, double* r,
                                                                                 float* pre32, double* pre64,
                                                                                 double* partials,
                                                                                 const SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    const double beta = st->beta, alpha = st->alpha;
    double a = 0.0;
    BMG_SPLIT_LOOP({
        double pq[4], qq[4], xq[4], rq[4], rn[4];
        Quad4<double>::ld(p + c, 0, pq);
        Quad4<double>::ld(q + c, 0, qq);
        Quad4<double>::ld(L.x + c, 0, xq);
        Quad4<double>::ld(r + c, 0, rq);
        for (int e = 0; e < 4; ++e) {
            const double pn = beta != 0.0 ? (double)zc[e] + beta * pq[e] : (double)zc[e];
            const double qn = beta != 0.0 ? Az[e] + beta * qq[e] : Az[e];
            pq[e] = pn;
            qq[e] = qn;
            xq[e] = xq[e] + alpha * pn;
            rn[e] = rq[e] - alpha * qn;
            const double Vr = (hij * hk[e]) * rn[e];
            a += Vr * Vr;
        }
        Quad4<double>::st(p + c, 0, pq);
        Quad4<double>::st(q + c, 0, qq);
        Quad4<double>::st(L.x + c, 0, xq);
        if ((L.per0 && (i == 0 || i == L.n0 - 1)) || (L.per1 && (j == 0 || j == L.n1 - 1)) ||
            (L.per2 && ((h == 0 && m0 == 0) || (h == 1 && m0 + 4 == kh)))) {
            for (int e = 0; e < 4; ++e) store_images(L, c + e, i, j, 2 * (m0 + e) + h, xq[e]);
        }
        Quad4<double>::st(r + c, 0, rn);
        if (pre32) {
            const float f[4] = {(float)rn[0], (float)rn[1], (float)rn[2], (float)rn[3]};
            Quad4<float>::st(pre32 + c, 0, f);
        }
        if (pre64) Quad4<double>::st(pre64 + c, 0, rn);
    })
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

#undef BMG_SPLIT_LOOP
#undef BMG_SPLIT_AZ

// The level-0 FP64 residual of k_residual_norm / k_fcg_residual on a
// parity-split level (one brick): the thread owns four consecutive positions
// of one half of a row, the cells k = 2 (m0 + e) + h of one parity (as
// k_fcg_step_split), so x, its neighbours and b load as whole vectors.  Per
// cell r = res_value(...), the arithmetic of the natural-order kernels; the
// partials: ||V r||^2 and, for mode 0, the normFactor sums; r, pre32 and
// pre64 written where given.
template <bool VAR>
__global__ void __launch_bounds__(kReduceThreads, 2) k_residual_split(Bricks<double> B, Walls W, int mode,
                                                                                 double* r_out, float* pre32,
                                                                                 double* pre64, double* partials,
                                                                                 long nblocks) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
    const LevelView<double>& L = B.v[0];
    const int qx = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int kh = L.kh;
    if (j < L.n1 && 4 * qx < L.n2) {
        const double wjl = L.tab64[L.to.wl[1] + j], wjh = L.tab64[L.to.wh[1] + j];
        const double hj = L.tab64[L.to.h[1] + j];
        const int h = 4 * qx >= kh ? 1 : 0;
        const int m0 = 4 * qx - h * kh;
        double wkl[4], wkh[4], hk[4];
        Quad4<double>::ld(L.tab64 + L.to.kwl + 4 * qx, 0, wkl);
        Quad4<double>::ld(L.tab64 + L.to.kwh + 4 * qx, 0, wkh);
        Quad4<double>::ld(L.tab64 + L.to.ksz + 4 * qx, 0, hk);
        for (int i = blockIdx.z; i < L.n0; i += gridDim.z) {
            const long row = row_at(L, i, j), c = row + 4 * qx;
            const long co = row + (1 - h) * kh + m0;  // the other half, same slots
            const long ce = h == 0 ? (m0 > 0 ? co - 1 : row - 1) : (m0 + 4 < kh ? co + 4 : row + 2 * kh);
            double xc[4], xo[4], xim[4], xip[4], xjm[4], xjp[4], bq[4];
            Quad4<double>::ld(L.x + c, 0, xc);
            Quad4<double>::ld(L.x + co, 0, xo);
            Quad4<double>::ld(L.x + c - L.si, 0, xim);
            Quad4<double>::ld(L.x + c + L.si, 0, xip);
            Quad4<double>::ld(L.x + c - L.sj, 0, xjm);
            Quad4<double>::ld(L.x + c + L.sj, 0, xjp);
            Quad4<double>::ld(L.b + c, 0, bq);
            const double xe = L.x[ce];
            const double wil = L.tab64[L.to.wl[0] + i], wih = L.tab64[L.to.wh[0] + i];
            const double hij = L.tab64[L.to.h[0] + i] * hj;
            double l0[4], l0p[4], l1[4], l1p[4], l2[4], l2o[4], l2e = 1.0;
            if (VAR) {
                Quad4<double>::ld(L.lam0 + c, 0, l0);
                Quad4<double>::ld(L.lam0 + c + L.si, 0, l0p);
                Quad4<double>::ld(L.lam1 + c, 0, l1);
                Quad4<double>::ld(L.lam1 + c + L.sj, 0, l1p);
                Quad4<double>::ld(L.lam2 + c, 0, l2);
                Quad4<double>::ld(L.lam2 + co, 0, l2o);  // lower faces of the other half's slots
                l2e = L.lam2[ce];
            }
            double rq[4];
#pragma unroll
            for (int e = 0; e < 4; ++e) {
                double w[6] = {wil, wih, wjl, wjh, wkl[e], wkh[e]};
                if (VAR) {
                    w[0] *= l0[e];
                    w[1] *= l0p[e];
                    w[2] *= l1[e];
                    w[3] *= l1p[e];
                    w[4] *= l2[e];
                    w[5] *= h == 0 ? l2o[e] : (e < 3 ? l2o[e + 1] : l2e);
                }
                const double km = h == 0 ? (e == 0 ? xe : xo[e - 1]) : xo[e];
                const double kp = h == 0 ? xo[e] : (e == 3 ? xe : xo[e + 1]);
                const double xn[6] = {xim[e], xip[e], xjm[e], xjp[e], km, kp};
                const double r = res_value(w, xn, xc[e], bq[e]);
                rq[e] = r;
                const double V = hij * hk[e];
                const double rr = V * r;
                a1 += rr * rr;
                if (mode == 0) {
                    const double bb = V * bq[e];
                    double ay = 0.0;
                    if (W.mask[0]) {  // A*mean(x): nonzero only in the rows of Dirichlet faces
                        const int k = 2 * (m0 + e) + h;
                        ay = -V * *W.ybar * wall_sum(L, W, 0, i, j, k, c + e, row + kpos(L, k + 1), false);
                    }
                    const double t = fabs(rr - bb + ay) + fabs(bb - ay);
                    a2 += t * t;
                    a3 += bb * bb;
                }
            }
            if (r_out) Quad4<double>::st(r_out + c, 0, rq);
            if (pre64) Quad4<double>::st(pre64 + c, 0, rq);
            if (pre32) {
                const float f[4] = {(float)rq[0], (float)rq[1], (float)rq[2], (float)rq[3]};
                Quad4<float>::st(pre32 + c, 0, f);
            }
        }
    }
    const long bid = block_id();
    a1 = block_sum<kReduceThreads>(a1, sh);
    if (mode == 0) {
        a2 = block_sum<kReduceThreads>(a2, sh);
        a3 = block_sum<kReduceThreads>(a3, sh);
    }
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        partials[bid] = a1;
        if (mode == 0) {
            partials[nblocks + bid] = a2;
            partials[2 * nblocks + bid] = a3;
        }
    }
}

// beta, (p, V q) and alpha from the one reduction of pass 1
__global__ void __launch_bounds__(kFinalThreads) k_fcg_coeffs(const double* partials, long nblocks, SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double zr = sum_partials<kFinalThreads>(partials, nblocks, sh);
    const double zq = sum_partials<kFinalThreads>(partials + nblocks, nblocks, sh);
    const double zaz = sum_partials<kFinalThreads>(partials + 2 * nblocks, nblocks, sh);
    if (threadIdx.x == 0) {
        const double beta = st->first ? 0.0 : -zq / st->pq;
        const double pq = st->first ? zaz : zaz + beta * zq;
        st->gamma = zr;
        st->beta = beta;
        st->pq = pq;
        st->alpha = zr / pq;
        st->first = 0;
    }
}

#undef BMG_QUAD_LOOP

bool fcg_quads(const Bricks<double>& B) {
    for (int b = 0; b < B.nb; ++b)
        if (B.v[b].n2 % 4) return false;
    return true;
}

dim3 quad_grid(const Bricks<double>& B) {
    return dim3((unsigned)((B.max2 / 4 + 15) / 16), (unsigned)((B.max1 + 15) / 16),
                (unsigned)std::min(B.z0[B.nb], kQuadPlanes));
}

}  // namespace

long fcg_partials(const Bricks<double>& B) {
    if (!fcg_quads(B)) return reduce_blocks(B);
    const dim3 g = quad_grid(B);
    return (long)g.x * g.y * g.z;
}

template <bool VAR>
long launch_residual_split(const Bricks<double>& B, const Walls& W, int mode, double* r, float* pre32,
                           double* pre64, double* partials, cudaStream_t s) {
    const long nb = fcg_partials(B);
    launch_k(k_residual_split<VAR>, quad_grid(B), dim3(16, 16, 1), 0, s, B, W, mode, r, pre32, pre64, partials, nb);
    return nb;
}

template <bool VAR>
long launch_fcg_residual(const Bricks<double>& B, const Walls& W, int mode, double* r, float* pre32, double* pre64,
                         double* partials, cudaStream_t s) {
    if (B.v[0].kh) return launch_residual_split<VAR>(B, W, mode, r, pre32, pre64, partials, s);
    const dim3 blk = block_for(B.max2);
    launch_k(k_fcg_residual<VAR>, grid_for(B, B.max2, blk), blk, 0, s, B, W, mode, r, pre32, pre64, partials,
                                                                   reduce_blocks(B));
    return reduce_blocks(B);
}

template <typename T, bool VAR>
void launch_fcg_step(const Bricks<double>& B, const T* z, double* p, double* q, double* r, float* pre32,
                     double* pre64, double* partials, SolveState* st, cudaStream_t s) {
    const long nb = fcg_partials(B);
    if (fcg_quads(B)) {
        // two passes and one reduction (k_fcg_coeffs)
        const dim3 g = quad_grid(B), blk(16, 16, 1);
        if (B.v[0].kh)
            launch_k(k_fcg_dots3_split<T, VAR>, g, blk, 0, s, B, z, r, q, partials, nb);
        else
            launch_k(k_fcg_dots3_4<T, VAR>, g, blk, 0, s, B, z, r, q, partials, nb);
        launch_k(k_fcg_coeffs, 1, kFinalThreads, 0, s, partials, nb, st);
        if (B.v[0].kh)
            launch_k(k_fcg_step_split<T, VAR>, g, blk, 0, s, B, z, p, q, r, pre32, pre64, partials, st);
        else
            launch_k(k_fcg_step4<T, VAR>, g, blk, 0, s, B, z, p, q, r, pre32, pre64, partials, st);
        return;
    }
    // rows of n2 % 4 != 0: one cell per thread, three passes
    const dim3 blk = block_for(B.max2);
    const dim3 g = grid_for(B, B.max2, blk);
    launch_k(k_fcg_dots<T>, g, blk, 0, s, B, z, r, q, partials, nb);
    launch_k(k_fcg_beta, 1, kFinalThreads, 0, s, partials, nb, st);
    launch_k(k_fcg_direction<T, VAR>, g, blk, 0, s, B, z, p, q, partials, st);
    launch_k(k_fcg_alpha, 1, kFinalThreads, 0, s, partials, nb, st);
    launch_k(k_fcg_update, g, blk, 0, s, B, p, r, q, pre32, pre64, partials, st);
}

int fcg_step_launches(const Bricks<double>& B) { return fcg_quads(B) ? 3 : 5; }

void launch_fcg_true_norm(const double* partials, long n, SolveState* st, cudaStream_t s) {
    launch_k(k_fcg_true_norm, 1, kFinalThreads, 0, s, partials, n, st);
}

template long launch_fcg_residual<false>(const Bricks<double>&, const Walls&, int, double*, float*, double*,
                                         double*, cudaStream_t);
template long launch_fcg_residual<true>(const Bricks<double>&, const Walls&, int, double*, float*, double*,
                                        double*, cudaStream_t);
template long launch_residual_split<false>(const Bricks<double>&, const Walls&, int, double*, float*, double*,
                                           double*, cudaStream_t);
template long launch_residual_split<true>(const Bricks<double>&, const Walls&, int, double*, float*, double*,
                                          double*, cudaStream_t);
#define BMG_INST(T, V)                                                                                         \
    template void launch_fcg_step<T, V>(const Bricks<double>&, const T*, double*, double*, double*, float*, \
                                        double*, double*, SolveState*, cudaStream_t);
BMG_INST(float, false)
BMG_INST(float, true)
BMG_INST(double, false)
BMG_INST(double, true)
#undef BMG_INST

}  // namespace bmg
