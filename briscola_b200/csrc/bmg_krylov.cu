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

// The next cycle's first colour pass for cell (i,j,k) of right-hand side f
// (FirstPass): gs_value with zero neighbours on the cells of fp.colour, the
// arithmetic of the colour-pass kernels on x = 0, and 0 elsewhere.
__device__ __forceinline__ float first_pass_value(const LevelView<double>& L, const FirstPass& fp, int i, int j,
                                                  int k, float f) {
    if (((i + j + k + L.cpar) & 1) != fp.colour) return 0.f;
    const float w[6] = {ldg(fp.tab + L.to.wl[0] + i), ldg(fp.tab + L.to.wh[0] + i), ldg(fp.tab + L.to.wl[1] + j),
                        ldg(fp.tab + L.to.wh[1] + j), ldg(fp.tab + L.to.wl[2] + k), ldg(fp.tab + L.to.wh[2] + k)};
    const float zero[6] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
    return gs_value(w, zero, f);
}

// r = b - A'x (FP64), written to r and to the cycle's right-hand side;
// partials: ||V r||^2 and, for mode 0, the normFactor sum (as k_residual_norm)
template <bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_residual(Bricks<double> B, Walls W, int mode, double* r_out,
                                                                 float* pre32, double* pre64, double* partials,
                                                                 long nblocks, FirstPass fp) {
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const int bk = brick_of(B, blockIdx.z, i);
    const LevelView<double>& L = B.v[bk];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a1 = 0.0, a2 = 0.0, a3 = 0.0;
    if (j < L.n1 && k < L.n2) {
        const long row = row_at(L, i, j), c = row + kpos(L, k);
        double w[6], s, d;
        const long ckm = row + kpos(L, k - 1), ckp = row + kpos(L, k + 1);
        couplings<double, VAR>(L, i, j, k, c, ckp, w);
        stencil(L.x, c, ckm, ckp, L.si, L.sj, w, s, d);
        const double r = L.b[c] + d * L.x[c] - s;
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
            if (fp.z) {
                const float z = first_pass_value(L, fp, i, j, k, (float)r);
                fp.z[c] = z;
                store_images_to(L, fp.z, c, i, j, k, z);
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

// partials of (z, V r) and (z, V q)
template <typename T>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_dots(Bricks<double> B, const T* z, const double* r,
                                                             const double* q, double* partials, long nblocks) {
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

template <typename T>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_dots4(Bricks<double> B, const T* z, const double* r,
                                                              const double* q, double* partials, long nblocks) {
    __shared__ double sh[kReduceThreads / 32];
    double a1 = 0.0, a2 = 0.0;
    BMG_QUAD_LOOP(B, {
        T zq[4];
        double rq[4], qq[4];
        Quad4<T>::ld(z + c, ks, zq);
        Quad4<double>::ld(r + c, ks, rq);
        Quad4<double>::ld(q + c, ks, qq);
        for (int e = 0; e < 4; ++e) {
            const double Vz = (hij * hk[e]) * (double)zq[e];
            a1 += Vz * rq[e];
            a2 += Vz * qq[e];
        }
    })
    a1 = block_sum<kReduceThreads>(a1, sh);
    a2 = block_sum<kReduceThreads>(a2, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const long bid = block_id();
        partials[bid] = a1;
        partials[nblocks + bid] = a2;
    }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_fcg_direction4(Bricks<double> B, const T* z, double* p,
                                                                   double* q, double* partials,
                                                                   const SolveState* st) {
    __shared__ double sh[kReduceThreads / 32];
    const double beta = st->beta;
    double a = 0.0;
    BMG_QUAD_LOOP(B, {
        T zc[4], zim[4], zip[4], zjm[4], zjp[4];
        Quad4<T>::ld(z + c, ks, zc);
        Quad4<T>::ld(z + c - L.si, ks, zim);
        Quad4<T>::ld(z + c + L.si, ks, zip);
        Quad4<T>::ld(z + c - L.sj, ks, zjm);
        Quad4<T>::ld(z + c + L.sj, ks, zjp);
        const long cr = row + kpos(L, k0 + 4);
        const T zl = z[row + kpos(L, k0 - 1)], zr = z[cr];
        double pq[4], qq[4], pn[4], qn[4];
        Quad4<double>::ld(p + c, ks, pq);
        Quad4<double>::ld(q + c, ks, qq);
        for (int e = 0; e < 4; ++e) {
            double w[6];
            couplings<double, VAR>(L, i, j, k0 + e, c + quad_off(ks, e), e < 3 ? c + quad_off(ks, e + 1) : cr, w);
            const double km = e > 0 ? (double)zc[e - 1] : (double)zl;
            const double kp = e < 3 ? (double)zc[e + 1] : (double)zr;
            const double zz = (double)zc[e];
            const double sv = w[0] * (double)zim[e] + w[1] * (double)zip[e] + w[2] * (double)zjm[e] +
                              w[3] * (double)zjp[e] + w[4] * km + w[5] * kp;
            const double d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
            // on the first step p and q hold whatever the last solve left
            pn[e] = beta != 0.0 ? zz + beta * pq[e] : zz;
            qn[e] = beta != 0.0 ? (sv - d * zz) + beta * qq[e] : sv - d * zz;
            a += (hij * hk[e]) * pn[e] * qn[e];
        }
        Quad4<double>::st(p + c, ks, pn);
        Quad4<double>::st(q + c, ks, qn);
    })
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

// The same direction step on a parity-split level 0 (one brick): the
// thread owns four consecutive positions of one half of a row, the cells
// k = 2 (m0 + e) + h of one parity, so z, its neighbours and p and q load as
// whole vectors; the k neighbours are the other half's same slots and one
// beyond them (as in k_colour_split).  Per cell the arithmetic is
// k_fcg_direction4's; the partial sums group the cells differently.
template <typename T, bool VAR>
__global__ void __launch_bounds__(kReduceThreads, VAR ? 2 : 3) k_fcg_direction_split(Bricks<double> B, const T* z, double* p,
                                                                        double* q, double* partials,
                                                                        const SolveState* st) {
    __shared__ double sh[kReduceThreads / 32];
    const double beta = st->beta;
    double a = 0.0;
    const LevelView<double>& L = B.v[0];
    const int qx = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int kh = L.kh;
    if (j < L.n1 && 4 * qx < L.n2) {
        const int h = 4 * qx >= kh ? 1 : 0;
        const int m0 = 4 * qx - h * kh;
        const double wjl = L.tab64[L.to.wl[1] + j], wjh = L.tab64[L.to.wh[1] + j];
        const double hj = L.tab64[L.to.h[1] + j];
        for (int i = blockIdx.z; i < L.n0; i += gridDim.z) {
            const long row = row_at(L, i, j), c = row + 4 * qx;
            const long co = row + (1 - h) * kh + m0;  // the other half, same slots
            const long ce = h == 0 ? (m0 > 0 ? co - 1 : row - 1) : (m0 + 4 < kh ? co + 4 : row + 2 * kh);
            T zc[4], zo[4], zim[4], zip[4], zjm[4], zjp[4];
            Quad4<T>::ld(z + c, 0, zc);
            Quad4<T>::ld(z + co, 0, zo);
            Quad4<T>::ld(z + c - L.si, 0, zim);
            Quad4<T>::ld(z + c + L.si, 0, zip);
            Quad4<T>::ld(z + c - L.sj, 0, zjm);
            Quad4<T>::ld(z + c + L.sj, 0, zjp);
            const T ze = z[ce];
            double pq[4], qq[4], pn[4], qn[4];
            Quad4<double>::ld(p + c, 0, pq);
            Quad4<double>::ld(q + c, 0, qq);
            const double wil = L.tab64[L.to.wl[0] + i], wih = L.tab64[L.to.wh[0] + i];
            const double hij = L.tab64[L.to.h[0] + i] * hj;
            // k couplings and cell sizes of the four cells, from the tables
            // kept in the rows' storage order (contiguous)
            double wkl[4], wkh[4], hk[4];
            Quad4<double>::ld(L.tab64 + L.to.kwl + 4 * qx, 0, wkl);
            Quad4<double>::ld(L.tab64 + L.to.kwh + 4 * qx, 0, wkh);
            Quad4<double>::ld(L.tab64 + L.to.ksz + 4 * qx, 0, hk);
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
            for (int e = 0; e < 4; ++e) {
                // the couplings of couplings(): l, r, b, t, a, f
                double w[6] = {wil, wih, wjl, wjh, wkl[e], wkh[e]};
                if (VAR) {
                    w[0] *= l0[e];
                    w[1] *= l0p[e];
                    w[2] *= l1[e];
                    w[3] *= l1p[e];
                    w[4] *= l2[e];
                    w[5] *= h == 0 ? l2o[e] : (e < 3 ? l2o[e + 1] : l2e);
                }
                const double km = h == 0 ? (double)(e == 0 ? ze : zo[e - 1]) : (double)zo[e];
                const double kp = h == 0 ? (double)zo[e] : (double)(e == 3 ? ze : zo[e + 1]);
                const double zz = (double)zc[e];
                const double sv = w[0] * (double)zim[e] + w[1] * (double)zip[e] + w[2] * (double)zjm[e] +
                                  w[3] * (double)zjp[e] + w[4] * km + w[5] * kp;
                const double d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
                pn[e] = beta != 0.0 ? zz + beta * pq[e] : zz;
                qn[e] = beta != 0.0 ? (sv - d * zz) + beta * qq[e] : sv - d * zz;
                a += (hij * hk[e]) * pn[e] * qn[e];
            }
            Quad4<double>::st(p + c, 0, pn);
            Quad4<double>::st(q + c, 0, qn);
        }
    }
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

__global__ void __launch_bounds__(kReduceThreads) k_fcg_update4(Bricks<double> B, const double* p, double* r,
                                                                const double* q, float* pre32, double* pre64,
                                                                double* partials, const SolveState* st,
                                                                FirstPass fp) {
    __shared__ double sh[kReduceThreads / 32];
    const double alpha = st->alpha;
    double a = 0.0;
    BMG_QUAD_LOOP(B, {
        double xq[4], pq[4], rq[4], qq[4], rn[4];
        Quad4<double>::ld(L.x + c, ks, xq);
        Quad4<double>::ld(p + c, ks, pq);
        Quad4<double>::ld(r + c, ks, rq);
        Quad4<double>::ld(q + c, ks, qq);
        for (int e = 0; e < 4; ++e) {
            xq[e] = xq[e] + alpha * pq[e];
            rn[e] = rq[e] - alpha * qq[e];
            const double Vr = (hij * hk[e]) * rn[e];
            a += Vr * Vr;
        }
        Quad4<double>::st(L.x + c, ks, xq);
        if (quad_has_images(L, i, j, k0)) {
            for (int e = 0; e < 4; ++e) store_images(L, c + quad_off(ks, e), i, j, k0 + e, xq[e]);
        }
        Quad4<double>::st(r + c, ks, rn);
        if (pre32) {
            const float f[4] = {(float)rn[0], (float)rn[1], (float)rn[2], (float)rn[3]};
            Quad4<float>::st(pre32 + c, ks, f);
            if (fp.z) {
                float zq[4];
                for (int e = 0; e < 4; ++e) zq[e] = first_pass_value(L, fp, i, j, k0 + e, f[e]);
                Quad4<float>::st(fp.z + c, ks, zq);
                if (quad_has_images(L, i, j, k0)) {
                    for (int e = 0; e < 4; ++e) store_images_to(L, fp.z, c + quad_off(ks, e), i, j, k0 + e, zq[e]);
                }
            }
        }
        if (pre64) Quad4<double>::st(pre64 + c, ks, rn);
    })
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
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
void launch_fcg_residual(const Bricks<double>& B, const Walls& W, int mode, double* r, float* pre32, double* pre64,
                         double* partials, FirstPass fp, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    k_fcg_residual<VAR><<<grid_for(B, B.max2, blk), blk, 0, s>>>(B, W, mode, r, pre32, pre64, partials,
                                                                   reduce_blocks(B), fp);
}

template <typename T>
void launch_fcg_beta(const Bricks<double>& B, const T* z, const double* r, const double* q, double* partials,
                     SolveState* st, cudaStream_t s) {
    const long nb = fcg_partials(B);
    if (fcg_quads(B)) {
        k_fcg_dots4<T><<<quad_grid(B), dim3(16, 16, 1), 0, s>>>(B, z, r, q, partials, nb);
    } else {
        const dim3 blk = block_for(B.max2);
        k_fcg_dots<T><<<grid_for(B, B.max2, blk), blk, 0, s>>>(B, z, r, q, partials, nb);
    }
    k_fcg_beta<<<1, kFinalThreads, 0, s>>>(partials, nb, st);
}

template <typename T, bool VAR>
void launch_fcg_direction(const Bricks<double>& B, const T* z, double* p, double* q, double* partials,
                          SolveState* st, cudaStream_t s) {
    if (B.v[0].kh) {
        k_fcg_direction_split<T, VAR><<<quad_grid(B), dim3(16, 16, 1), 0, s>>>(B, z, p, q, partials, st);
    } else if (fcg_quads(B)) {
        k_fcg_direction4<T, VAR><<<quad_grid(B), dim3(16, 16, 1), 0, s>>>(B, z, p, q, partials, st);
    } else {
        const dim3 blk = block_for(B.max2);
        k_fcg_direction<T, VAR><<<grid_for(B, B.max2, blk), blk, 0, s>>>(B, z, p, q, partials, st);
    }
    k_fcg_alpha<<<1, kFinalThreads, 0, s>>>(partials, fcg_partials(B), st);
}

void launch_fcg_update(const Bricks<double>& B, const double* p, double* r, const double* q, float* pre32,
                       double* pre64, double* partials, const SolveState* st, FirstPass fp, cudaStream_t s) {
    if (fcg_quads(B)) {
        k_fcg_update4<<<quad_grid(B), dim3(16, 16, 1), 0, s>>>(B, p, r, q, pre32, pre64, partials, st, fp);
        return;
    }
    const dim3 blk = block_for(B.max2);
    k_fcg_update<<<grid_for(B, B.max2, blk), blk, 0, s>>>(B, p, r, q, pre32, pre64, partials, st);
}

void launch_fcg_true_norm(const Bricks<double>& B, const double* partials, SolveState* st, cudaStream_t s) {
    k_fcg_true_norm<<<1, kFinalThreads, 0, s>>>(partials, reduce_blocks(B), st);
}

template void launch_fcg_residual<false>(const Bricks<double>&, const Walls&, int, double*, float*, double*, double*,
                                         FirstPass, cudaStream_t);
template void launch_fcg_residual<true>(const Bricks<double>&, const Walls&, int, double*, float*, double*, double*,
                                        FirstPass, cudaStream_t);
template void launch_fcg_beta<float>(const Bricks<double>&, const float*, const double*, const double*, double*,
                                     SolveState*, cudaStream_t);
template void launch_fcg_beta<double>(const Bricks<double>&, const double*, const double*, const double*,
                                      double*, SolveState*, cudaStream_t);
template void launch_fcg_direction<float, false>(const Bricks<double>&, const float*, double*, double*, double*,
                                                 SolveState*, cudaStream_t);
template void launch_fcg_direction<float, true>(const Bricks<double>&, const float*, double*, double*, double*,
                                                SolveState*, cudaStream_t);
template void launch_fcg_direction<double, false>(const Bricks<double>&, const double*, double*, double*,
                                                  double*, SolveState*, cudaStream_t);
template void launch_fcg_direction<double, true>(const Bricks<double>&, const double*, double*, double*,
                                                 double*, SolveState*, cudaStream_t);

}  // namespace bmg
