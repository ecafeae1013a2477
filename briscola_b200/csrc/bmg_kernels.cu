// bmg_kernels.cu -- sm_100a kernels of the multigrid V-cycle.
//
// Every kernel here is HBM- (fine levels) or L2-bound (levels up to 128^3
// fit the 126 MB L2): no tensor cores, coalesced k-fastest access, FP64 or
// FP32 arithmetic chosen by the template parameter.  Layout and coefficient
// conventions are described in bmg_internal.h.  Each per-cell kernel runs
// over all bricks of a level in one launch: the grid's z index walks the
// planes of brick 0, then brick 1, and so on.

#include <algorithm>
#include <cmath>

#include "bmg_grid.cuh"
#include "bmg_stencil.cuh"

namespace bmg {

namespace {

template <typename T>
struct Pair;
template <>
struct Pair<float> {
    using type = float2;
};
template <>
struct Pair<double> {
    using type = double2;
};

// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel: one colour pass (one pass of rbgsSmoother.C:65-183
// over the whole level).  Colour 0 = (i+j+k+cpar) even, cpar the parity of
// the brick origin, so colours agree across brick contacts.  The thread owns
// the k-pair (2p, 2p+1) and updates its member of the requested colour.
// Neighbour rows and planes are read as whole pairs (8/16-byte loads), so a
// warp's loads fill every L1 wavefront; the k neighbour outside the pair is
// one scalar load.
// ---------------------------------------------------------------------------
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_colour_pass(Bricks<T> B, int colour) {
    grid_dep_sync();
    using V2 = typename Pair<T>::type;
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = 2 * p;
    if (j >= L.n1 || k0 >= L.n2) return;
    const int e = ((i + j + k0 + L.cpar) & 1) == colour ? 0 : 1;
    const int k = k0 + e;
    if (k >= L.n2) return;
    const long r = L.base + (long)i * L.si + (long)j * L.sj;
    const T* x = L.x;
    const long c0 = r + k0;
    const V2 xm = *reinterpret_cast<const V2*>(x + c0 - L.si);
    const V2 xp = *reinterpret_cast<const V2*>(x + c0 + L.si);
    const V2 ym = *reinterpret_cast<const V2*>(x + c0 - L.sj);
    const V2 yp = *reinterpret_cast<const V2*>(x + c0 + L.sj);
    const V2 own = *reinterpret_cast<const V2*>(x + c0);
    const long c = r + k;
    if (L.pin && (i | j | k) == 0) return;  // the pinned cell stays zero
    T w[6];
    couplings<T, VAR>(L, i, j, k, c, c + 1, w);  // natural rows only (n2 % 4 != 0)
    const T xn[6] = {e ? xm.y : xm.x, e ? xp.y : xp.x, e ? ym.y : ym.x, e ? yp.y : yp.x,
                     e ? own.x : x[c0 - 1], e ? x[c0 + 2] : own.y};
    store_x(L, c, i, j, k, gs_value(w, xn, L.b[c]));
}

// Four consecutive values of a row (16-byte aligned for FP32, two 16-byte
// halves for FP64).
template <typename T>
struct Row4;
template <>
struct Row4<float> {
    static __device__ __forceinline__ void ld(const float* p, float v[4]) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
    static __device__ __forceinline__ void ldg4(const float* p, float v[4]) {
        const float4 a = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
    static __device__ __forceinline__ void st(float* p, const float v[4]) {
        *reinterpret_cast<float4*>(p) = make_float4(v[0], v[1], v[2], v[3]);
    }
    // two consecutive values from an 8-byte aligned address
    static __device__ __forceinline__ void ld2(const float* p, float& a, float& b) {
        const float2 v = *reinterpret_cast<const float2*>(p);
        a = v.x;
        b = v.y;
    }
};
template <>
struct Row4<double> {
    static __device__ __forceinline__ void ld(const double* p, double v[4]) {
        const double2 a = reinterpret_cast<const double2*>(p)[0], b = reinterpret_cast<const double2*>(p)[1];
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
    static __device__ __forceinline__ void ldg4(const double* p, double v[4]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
    static __device__ __forceinline__ void st(double* p, const double v[4]) {
        reinterpret_cast<double2*>(p)[0] = make_double2(v[0], v[1]);
        reinterpret_cast<double2*>(p)[1] = make_double2(v[2], v[3]);
    }
    // two consecutive values from a 16-byte aligned address
    static __device__ __forceinline__ void ld2(const double* p, double& a, double& b) {
        const double2 v = *reinterpret_cast<const double2*>(p);
        a = v.x;
        b = v.y;
    }
};

// The logical k-quad k0 .. k0+3 (k0 % 4 == 0) of a row, at slab index c
// = the quad's first cell: one vector in a natural row (kh = 0); in a
// parity-split row the even pair (k0, k0+2) at c and the odd pair
// (k0+1, k0+3) at c + kh.
template <typename T>
__device__ __forceinline__ void ldq(const T* p, int kh, T v[4]) {
    if (kh) {
        Row4<T>::ld2(p, v[0], v[2]);
        Row4<T>::ld2(p + kh, v[1], v[3]);
    } else {
        Row4<T>::ld(p, v);
    }
}
template <typename T>
__device__ __forceinline__ void ldgq(const T* p, int kh, T v[4]) {
    if (kh) {
        v[0] = ldg(p);
        v[2] = ldg(p + 1);
        v[1] = ldg(p + kh);
        v[3] = ldg(p + kh + 1);
    } else {
        Row4<T>::ldg4(p, v);
    }
}
template <typename T>
__device__ __forceinline__ void stq(T* p, int kh, const T v[4]);
template <>
__device__ __forceinline__ void stq<float>(float* p, int kh, const float v[4]) {
    if (kh) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[2]);
        *reinterpret_cast<float2*>(p + kh) = make_float2(v[1], v[3]);
    } else {
        Row4<float>::st(p, v);
    }
}
template <>
__device__ __forceinline__ void stq<double>(double* p, int kh, const double v[4]) {
    if (kh) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[2]);
        *reinterpret_cast<double2*>(p + kh) = make_double2(v[1], v[3]);
    } else {
        Row4<double>::st(p, v);
    }
}

// ---------------------------------------------------------------------------
// Red-black colour pass, four cells per thread: the thread owns the k-quad
// (4p .. 4p+3) of one row and updates the two cells of the requested colour.
// The rows j-1, j, j+1, the i neighbours, b and the k couplings are read as
// whole vectors, and the quad is written back as one vector (the other
// colour's values are unchanged during the pass, so writing them back is
// safe; a quad is never a ghost).  colour_quad_item is shared with the
// single-CTA coarse cycle (k_tail_cycle).  The arithmetic is gs_value's, so results are
// bit-identical to k_colour_pass and the fused smoother.  Needs every
// brick's n2 % 4 == 0 and natural rows (parity-split levels take
// k_colour_split).
// ---------------------------------------------------------------------------
template <typename T, bool VAR>
__device__ __forceinline__ void colour_quad_item(const LevelView<T>& L, int i, int j, int p, int colour) {
    const int k0 = 4 * p;
    const int c = cell32(L, i, j, k0), si = (int)L.si, sj = (int)L.sj;
    const T* x = L.x;
    // rows j-1, j, j+1 of this plane (j+1 may be the ghost row)
    T ym[4], own[4], yp[4], xm[4], xp[4], bb[4], wkl[4], wkh[4];
    Row4<T>::ld(x + c - sj, ym);
    Row4<T>::ld(x + c, own);
    Row4<T>::ld(x + c + sj, yp);
    Row4<T>::ld(x + c - si, xm);
    Row4<T>::ld(x + c + si, xp);
    Row4<T>::ld(L.b + c, bb);
    Row4<T>::ldg4(L.tab + L.to.wl[2] + k0, wkl);
    Row4<T>::ldg4(L.tab + L.to.wh[2] + k0, wkh);
    const T wil = ldg(L.tab + L.to.wl[0] + i), wih = ldg(L.tab + L.to.wh[0] + i);
    const T left = x[c - 1], right = x[c + 4];
    const T wjl = ldg(L.tab + L.to.wl[1] + j), wjh = ldg(L.tab + L.to.wh[1] + j);
    // the two cells of the colour: (0, 2) or (1, 3); every array index
    // below is a compile-time constant picked by a select
    const bool odd = ((colour ^ (i + j + k0 + L.cpar)) & 1) != 0;
#define BMG_SEL(a, e) (odd ? a[(e) + 1] : a[e])
    T w0[6] = {wil, wih, wjl, wjh, BMG_SEL(wkl, 0), BMG_SEL(wkh, 0)};
    T w2[6] = {wil, wih, wjl, wjh, BMG_SEL(wkl, 2), BMG_SEL(wkh, 2)};
    if (VAR) {
        T l0[4], l0p[4], l1[4], l1p[4], l2[4];
        Row4<T>::ldg4(L.lam0 + c, l0);
        Row4<T>::ldg4(L.lam0 + c + si, l0p);
        Row4<T>::ldg4(L.lam1 + c, l1);
        Row4<T>::ldg4(L.lam1 + c + sj, l1p);
        Row4<T>::ldg4(L.lam2 + c, l2);
        const T l2r = ldg(L.lam2 + c + 4);
        w0[0] *= BMG_SEL(l0, 0);
        w0[1] *= BMG_SEL(l0p, 0);
        w0[2] *= BMG_SEL(l1, 0);
        w0[3] *= BMG_SEL(l1p, 0);
        w0[4] *= BMG_SEL(l2, 0);
        w0[5] *= BMG_SEL(l2, 1);
        w2[0] *= BMG_SEL(l0, 2);
        w2[1] *= BMG_SEL(l0p, 2);
        w2[2] *= BMG_SEL(l1, 2);
        w2[3] *= BMG_SEL(l1p, 2);
        w2[4] *= BMG_SEL(l2, 2);
        w2[5] *= odd ? l2r : l2[3];
    }
    const T xn0[6] = {BMG_SEL(xm, 0), BMG_SEL(xp, 0), BMG_SEL(ym, 0), BMG_SEL(yp, 0), odd ? own[0] : left,
                      odd ? own[2] : own[1]};
    const T xn2[6] = {BMG_SEL(xm, 2), BMG_SEL(xp, 2), BMG_SEL(ym, 2), BMG_SEL(yp, 2), odd ? own[2] : own[1],
                      odd ? right : own[3]};
    // the pinned cell (0,0,0), when this pass updates it, stays zero
    const T v0 = (L.pin && (i | j | k0) == 0 && !odd) ? own[0] : gs_value(w0, xn0, BMG_SEL(bb, 0));
    const T v2 = gs_value(w2, xn2, BMG_SEL(bb, 2));
#undef BMG_SEL
    const T out[4] = {odd ? own[0] : v0, odd ? v0 : own[1], odd ? own[2] : v2, odd ? v2 : own[3]};
    Row4<T>::st(L.x + c, out);
    // periodic images of the two updated cells
    if (quad_has_images(L, i, j, k0)) {
        const int q0 = odd ? 1 : 0;
        store_images(L, c + q0, i, j, k0 + q0, v0);
        store_images(L, c + q0 + 2, i, j, k0 + q0 + 2, v2);
    }
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_colour_quad(Bricks<T> B, int colour) {
    grid_dep_sync();
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || 4 * p >= L.n2) return;
    colour_quad_item<T, VAR>(L, i, j, p, colour);
}

// ---------------------------------------------------------------------------
// Red-black colour pass on a parity-split level (bmg_internal.h): the
// thread owns one 16-byte vector of the pass's colour, NC = 16 / sizeof(T)
// consecutive slots (4 FP32 or 2 FP64 cells) of its row's half of that
// colour, so a warp's loads and stores are whole contiguous runs.  Every
// value it reads is one the update needs: the other colour's same slots of
// its own row and one k neighbour beyond them, the same slots of the four
// neighbouring rows, b of its own cells, and the k couplings from tables
// kept in the same order.  Per cell the arithmetic is gs_value's with
// colour_quad_item's couplings and neighbour order, so the pass is
// bit-identical to the natural-order kernels.  The FP32 constant-coefficient
// instance is held to 48 registers (five blocks per SM): latency-bound,
// it runs 16 % faster with the extra warps.
// ---------------------------------------------------------------------------
template <typename T>
struct Vec16;
template <>
struct Vec16<float> {
    static constexpr int N = 4;
    static __device__ __forceinline__ void ld(const float* p, float v[4]) { Row4<float>::ld(p, v); }
    static __device__ __forceinline__ void ldg(const float* p, float v[4]) { Row4<float>::ldg4(p, v); }
    static __device__ __forceinline__ void st(float* p, const float v[4]) { Row4<float>::st(p, v); }
};
template <>
struct Vec16<double> {
    static constexpr int N = 2;
    static __device__ __forceinline__ void ld(const double* p, double v[2]) { Row4<double>::ld2(p, v[0], v[1]); }
    static __device__ __forceinline__ void ldg(const double* p, double v[2]) {
        const double2 a = __ldg(reinterpret_cast<const double2*>(p));
        v[0] = a.x;
        v[1] = a.y;
    }
    static __device__ __forceinline__ void st(double* p, const double v[2]) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    }
};

// ZERO: the first pass of a cycle that starts from x = 0 -- no x is read
// (every neighbour is zero), and the thread also writes zero to the other
// half's same slots, so the pass leaves the whole level written (the
// arithmetic of a pass over a zeroed x).
template <typename T, bool VAR, bool ZERO>
__global__ void __launch_bounds__(256, sizeof(T) == 4 && !VAR ? 5 : 1) k_colour_split(LevelView<T> L, int colour) {
    grid_dep_sync();
    constexpr int NC = Vec16<T>::N;  // cells per thread
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    const int kh = L.kh;
    if (j >= L.n1 || t * NC >= kh) return;
    const int m0 = t * NC;  // first slot of the thread in its half row
    // h = 0: the even k of this row have the pass's colour (k = 2m + h)
    const int h = (colour ^ (i + j + L.cpar)) & 1;
    const int si = (int)L.si, sj = (int)L.sj;
    const int row = (int)L.base + i * si + j * sj;
    const int own = row + h * kh + m0;
    const int oth = row + (1 - h) * kh + m0;
    // the k neighbour beyond the slots: below the first cell (h = 0; the
    // previous slot of the odd half, or the ghost k = -1) or above the last
    // one (h = 1; the next slot of the even half, or the ghost k = n2)
    const int ext = h == 0 ? (m0 > 0 ? oth - 1 : row - 1) : (m0 + NC < kh ? oth + NC : row + 2 * kh);
    // every load is issued before any is used, so one memory latency covers them
    T xo[NC], xm[NC], xp[NC], ym[NC], yp[NC], bb[NC], wkl[NC], wkh[NC];
    T e = T(0);
    if constexpr (ZERO) {
#pragma unroll
        for (int m = 0; m < NC; ++m) xo[m] = xm[m] = xp[m] = ym[m] = yp[m] = T(0);
    } else {
        Vec16<T>::ld(L.x + oth, xo);
        Vec16<T>::ld(L.x + own - si, xm);
        Vec16<T>::ld(L.x + own + si, xp);
        Vec16<T>::ld(L.x + own - sj, ym);
        Vec16<T>::ld(L.x + own + sj, yp);
        e = L.x[ext];
    }
    Vec16<T>::ld(L.b + own, bb);
    Vec16<T>::ldg(L.tab + L.to.kwl + (own - row), wkl);
    Vec16<T>::ldg(L.tab + L.to.kwh + (own - row), wkh);
    const T wil = ldg(L.tab + L.to.wl[0] + i), wih = ldg(L.tab + L.to.wh[0] + i);
    const T wjl = ldg(L.tab + L.to.wl[1] + j), wjh = ldg(L.tab + L.to.wh[1] + j);
    T l0[NC], l0p[NC], l1[NC], l1p[NC], l2[NC], l2u[NC], l2e = T(1);
    if (VAR) {
        Vec16<T>::ldg(L.lam0 + own, l0);
        Vec16<T>::ldg(L.lam0 + own + si, l0p);
        Vec16<T>::ldg(L.lam1 + own, l1);
        Vec16<T>::ldg(L.lam1 + own + sj, l1p);
        Vec16<T>::ldg(L.lam2 + own, l2);
        Vec16<T>::ldg(L.lam2 + oth, l2u);  // lower faces of the other colour's slots
        // the upper k face of the last cell (h = 1) is the lower face of the
        // next even slot, or the face at k = n2 (both at ext)
        l2e = ldg(L.lam2 + ext);
    }
    T v[NC];
#pragma unroll
    for (int m = 0; m < NC; ++m) {
        // k neighbours: h = 0 reads (e, xo[0]), (xo[0], xo[1]), ...;
        // h = 1 reads (xo[0], xo[1]), ..., (xo[NC-1], e)
        const T klo = h == 0 ? (m == 0 ? e : xo[m - 1]) : xo[m];
        const T khi = h == 0 ? xo[m] : (m == NC - 1 ? e : xo[m + 1]);
        T w[6] = {wil, wih, wjl, wjh, wkl[m], wkh[m]};
        if (VAR) {
            w[0] *= l0[m];
            w[1] *= l0p[m];
            w[2] *= l1[m];
            w[3] *= l1p[m];
            w[4] *= l2[m];
            w[5] *= h == 0 ? l2u[m] : (m == NC - 1 ? l2e : l2u[m + 1]);
        }
        const T xn[6] = {xm[m], xp[m], ym[m], yp[m], klo, khi};
        v[m] = gs_value(w, xn, bb[m]);
    }
    // the pinned cell (0,0,0), when this pass updates it, keeps its value
    if (L.pin && (i | j | h | m0) == 0) v[0] = ZERO ? T(0) : L.x[own];
    Vec16<T>::st(L.x + own, v);
    const bool edge_ij = (L.per0 && (i == 0 || i == L.n0 - 1)) || (L.per1 && (j == 0 || j == L.n1 - 1));
    if (edge_ij || (L.per2 && (((h | m0) == 0) || (h == 1 && m0 + NC == kh)))) {
#pragma unroll
        for (int m = 0; m < NC; ++m) store_images(L, own + m, i, j, 2 * (m0 + m) + h, v[m]);
    }
    if constexpr (ZERO) {
        T zero[NC];
#pragma unroll
        for (int m = 0; m < NC; ++m) zero[m] = T(0);
        Vec16<T>::st(L.x + oth, zero);
        const int ho = 1 - h;
        if (edge_ij || (L.per2 && (((ho | m0) == 0) || (ho == 1 && m0 + NC == kh)))) {
#pragma unroll
            for (int m = 0; m < NC; ++m) store_images(L, oth + m, i, j, 2 * (m0 + m) + ho, T(0));
        }
    }
}

// Damped Jacobi (omega = 0.8, jacSmoother.C:15) into a temporary, then copy.
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_jacobi(Bricks<T> B, T* tmp) {
    grid_dep_sync();
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    T w[6], s, d;
    const long ckm = row + kpos(L, k - 1), ckp = row + kpos(L, k + 1);
    couplings<T, VAR>(L, i, j, k, c, ckp, w);
    stencil(L.x, c, ckm, ckp, L.si, L.sj, w, s, d);
    const T omega = T(0.8);
    tmp[c] = (L.pin && (i | j | k) == 0) ? T(0) : (T(1) - omega) * L.x[c] + omega * (s - L.b[c]) / d;
}

template <typename T>
__global__ void __launch_bounds__(256) k_copy_interior(Bricks<T> B, const T* src) {
    grid_dep_sync();
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    store_x(L, c, i, j, k, src[c]);
}

// ---------------------------------------------------------------------------
// Fused residual + restriction: coarse b' = sum over the (up to 8) children
// of (V_child / V_coarse) * (b' - A' x)_child.  On a rectilinear brick this
// equals the reference's scaled linear restriction V_c * sum w_q r_q / V_q
// (linearRestrictionScheme.C:118-159): the trilinear weight of each child
// along an axis is its share of the coarse cell length along that axis.
// ---------------------------------------------------------------------------
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_residual_restrict(Bricks<T> FB, Bricks<T> CB, TransferSet ts) {
    grid_dep_sync();
    int I;
    const int b = brick_of(CB, blockIdx.z, I);
    const LevelView<T>& C = CB.v[b];
    const LevelView<T>& F = FB.v[b];
    const TransferTabs& t = ts.t[b];
    const int K = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    if (J >= C.n1 || K >= C.n2) return;
    const T* ratio;
    if constexpr (sizeof(T) == 8)
        ratio = reinterpret_cast<const T*>(t.ratio64);
    else
        ratio = reinterpret_cast<const T*>(t.ratio32);
    T acc = T(0);
    for (int a = 0; a < t.R0; ++a) {
        const int i = I * t.R0 + a;
        const T ra = ldg(ratio + i);
        for (int bb = 0; bb < t.R1; ++bb) {
            const int j = J * t.R1 + bb;
            const T rab = ra * ldg(ratio + F.n0 + j);
            for (int e = 0; e < t.R2; ++e) {
                const int k = K * t.R2 + e;
                const long row = row_at(F, i, j), c = row + kpos(F, k);
                const long ckm = row + kpos(F, k - 1), ckp = row + kpos(F, k + 1);
                T w[6], s, d;
                couplings<T, VAR>(F, i, j, k, c, ckp, w);
                stencil(F.x, c, ckm, ckp, F.si, F.sj, w, s, d);
                const T r = F.b[c] + d * F.x[c] - s;
                acc += rab * ldg(ratio + F.n0 + F.n1 + k) * r;
            }
        }
    }
    C.b[row_at(C, I, J) + kpos(C, K)] = acc;
}

// ---------------------------------------------------------------------------
// Fused prolongation + correction: x_f += trilinear interpolation of the
// coarse correction (linearProlongationScheme.C:12-147).  Per fine index the
// host tables give the two coarse indices (own parent and the neighbour on
// the fine cell's side) and the neighbour's weight.  On a single brick the
// neighbour index is wrapped on periodic axes and the weight is zero at
// walls (the reference's zero-gradient ghost gives the same value); between
// bricks the neighbour is the coarse ghost cell, refreshed before the call.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_prolong_correct(Bricks<T> FB, Bricks<T> CB, TransferSet ts) {
    grid_dep_sync();
    int i;
    const int b = brick_of(FB, blockIdx.z, i);
    const LevelView<T>& F = FB.v[b];
    const LevelView<T>& C = CB.v[b];
    const TransferTabs& t = ts.t[b];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= F.n1 || k >= F.n2) return;
    const int* pidx = t.pidx;
    const T* pw;
    if constexpr (sizeof(T) == 8)
        pw = reinterpret_cast<const T*>(t.pw64);
    else
        pw = reinterpret_cast<const T*>(t.pw32);
    const int I0 = ldg(pidx + 2 * i), I1 = ldg(pidx + 2 * i + 1);
    const int J0 = ldg(pidx + 2 * F.n0 + 2 * j), J1 = ldg(pidx + 2 * F.n0 + 2 * j + 1);
    const int K0 = ldg(pidx + 2 * (F.n0 + F.n1) + 2 * k);
    const int K1 = ldg(pidx + 2 * (F.n0 + F.n1) + 2 * k + 1);
    const T wi = ldg(pw + i), wj = ldg(pw + F.n0 + j), wk = ldg(pw + F.n0 + F.n1 + k);
    const T* X = C.x;
    const long r00 = C.base + (long)I0 * C.si + (long)J0 * C.sj;
    const long r01 = C.base + (long)I0 * C.si + (long)J1 * C.sj;
    const long r10 = C.base + (long)I1 * C.si + (long)J0 * C.sj;
    const long r11 = C.base + (long)I1 * C.si + (long)J1 * C.sj;
    const T uk = T(1) - wk, uj = T(1) - wj, ui = T(1) - wi;
    const int P0 = kpos(C, K0), P1 = kpos(C, K1);
    const T v00 = uk * X[r00 + P0] + wk * X[r00 + P1];
    const T v01 = uk * X[r01 + P0] + wk * X[r01 + P1];
    const T v10 = uk * X[r10 + P0] + wk * X[r10 + P1];
    const T v11 = uk * X[r11 + P0] + wk * X[r11 + P1];
    const T v = ui * (uj * v00 + wj * v01) + wi * (uj * v10 + wj * v11);
    const long c = row_at(F, i, j) + kpos(F, k);
    store_x(F, c, i, j, k, F.x[c] + v);
}

// ---------------------------------------------------------------------------
// The same two transfers for factor-2 coarsening along every axis with
// n2 % 4 == 0 (fine) -- the shape of every level the solver builds from
// even brick extents: a thread owns four fine cells along k.  Prolongation:
// the coarse i/j indices and weights are set up once for the four cells and
// the fine quad is read and written as one vector.  Restriction: the thread
// owns the two coarse cells over those four fine cells and evaluates the
// residual of each of its four fine rows from whole-vector loads.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void prolong_quad_item(const LevelView<T>& F, const LevelView<T>& C,
                                                  const TransferTabs& t, int i, int j, int p) {
    const int k0 = 4 * p;
    const int* pidx = t.pidx;
    const T* pw;
    if constexpr (sizeof(T) == 8)
        pw = reinterpret_cast<const T*>(t.pw64);
    else
        pw = reinterpret_cast<const T*>(t.pw32);
    const int I0 = ldg(pidx + 2 * i), I1 = ldg(pidx + 2 * i + 1);
    const int J0 = ldg(pidx + 2 * F.n0 + 2 * j), J1 = ldg(pidx + 2 * F.n0 + 2 * j + 1);
    const T wi = ldg(pw + i), wj = ldg(pw + F.n0 + j);
    const T ui = T(1) - wi, uj = T(1) - wj;
    const T* X = C.x;
    const int r00 = cell32(C, I0, J0, 0), r01 = cell32(C, I0, J1, 0);
    const int r10 = cell32(C, I1, J0, 0), r11 = cell32(C, I1, J1, 0);
    const int c0 = cell32(F, i, j, k0);
    T xf[4];
    ldq(F.x + c0, F.kh, xf);
    const int* pk = pidx + 2 * (F.n0 + F.n1);
    const T* wk = pw + F.n0 + F.n1;
    // Fine cells k0 .. k0+3 (k0 = 4p) have parents 2p, 2p, 2p+1, 2p+1 and
    // second coarse cells Ka, 2p+1, 2p, Kd: four coarse values per row,
    // the middle pair (2p, 2p+1) one aligned vector (interior k starts at an
    // offset of 4 in every row, so 2p sits at an even offset).
    const int Ka = kpos(C, ldg(pk + 2 * k0 + 1)), Kb = ldg(pk + 2 * k0), Kd = kpos(C, ldg(pk + 2 * (k0 + 3) + 1));
    const int Pb = kpos(C, Kb), Pc = kpos(C, Kb + 1);
    T w[4], u[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        w[q] = ldg(wk + k0 + q);
        u[q] = T(1) - w[q];
    }
    const int rows[4] = {r00, r01, r10, r11};
    T v[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        T xb, xc;
        if (C.kh) {
            xb = X[rows[r] + Pb];
            xc = X[rows[r] + Pc];
        } else {
            Row4<T>::ld2(X + rows[r] + Kb, xb, xc);
        }
        const T xa = X[rows[r] + Ka], xd = X[rows[r] + Kd];
        v[r][0] = u[0] * xb + w[0] * xa;
        v[r][1] = u[1] * xb + w[1] * xc;
        v[r][2] = u[2] * xc + w[2] * xb;
        v[r][3] = u[3] * xc + w[3] * xd;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        xf[q] += ui * (uj * v[0][q] + wj * v[1][q]) + wi * (uj * v[2][q] + wj * v[3][q]);
    stq(F.x + c0, F.kh, xf);
    if (quad_has_images(F, i, j, k0)) {
#pragma unroll
        for (int q = 0; q < 4; ++q) store_images(F, c0 + quad_off(F.kh, q), i, j, k0 + q, xf[q]);
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong_quad(Bricks<T> FB, Bricks<T> CB, TransferSet ts) {
    grid_dep_sync();
    int i;
    const int b = brick_of(FB, blockIdx.z, i);
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= FB.v[b].n1 || 4 * p >= FB.v[b].n2) return;
    prolong_quad_item<T>(FB.v[b], CB.v[b], ts.t[b], i, j, p);
}

template <typename T, bool VAR>
__device__ __forceinline__ void restrict_quad_item(const LevelView<T>& F, const LevelView<T>& C,
                                                   const TransferTabs& t, int I, int J, int P) {
    const int K0 = 2 * P;  // the thread's coarse k-pair
    const T* ratio;
    if constexpr (sizeof(T) == 8)
        ratio = reinterpret_cast<const T*>(t.ratio64);
    else
        ratio = reinterpret_cast<const T*>(t.ratio32);
    const int k0 = 2 * K0;
    T rk[4], wkl[4], wkh[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) rk[q] = ldg(ratio + F.n0 + F.n1 + k0 + q);
    Row4<T>::ldg4(F.tab + F.to.wl[2] + k0, wkl);
    Row4<T>::ldg4(F.tab + F.to.wh[2] + k0, wkh);
    T acc0 = T(0), acc1 = T(0);
#pragma unroll
    for (int a = 0; a < 2; ++a) {
        const int i = 2 * I + a;
        const T ra = ldg(ratio + i);
        const T wil = ldg(F.tab + F.to.wl[0] + i), wih = ldg(F.tab + F.to.wh[0] + i);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int j = 2 * J + e;
            const T rab = ra * ldg(ratio + F.n0 + j);
            const T wjl = ldg(F.tab + F.to.wl[1] + j), wjh = ldg(F.tab + F.to.wh[1] + j);
            const int row = (int)row_at(F, i, j), si = (int)F.si, sj = (int)F.sj;
            const int c = row + kpos(F, k0), kh = F.kh;
            T own[4], xm[4], xp[4], ym[4], yp[4], bb[4];
            ldq(F.x + c, kh, own);
            ldq(F.x + c - si, kh, xm);
            ldq(F.x + c + si, kh, xp);
            ldq(F.x + c - sj, kh, ym);
            ldq(F.x + c + sj, kh, yp);
            ldq(F.b + c, kh, bb);
            const int cl = row + kpos(F, k0 - 1), cr = row + kpos(F, k0 + 4);
            const T left = F.x[cl], right = F.x[cr];
            T l0[4], l0p[4], l1[4], l1p[4], l2[4], l2r = T(1);
            if (VAR) {
                ldgq(F.lam0 + c, kh, l0);
                ldgq(F.lam0 + c + si, kh, l0p);
                ldgq(F.lam1 + c, kh, l1);
                ldgq(F.lam1 + c + sj, kh, l1p);
                ldgq(F.lam2 + c, kh, l2);
                l2r = ldg(F.lam2 + cr);
            }
            T r[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                T w[6] = {wil, wih, wjl, wjh, wkl[q], wkh[q]};
                if (VAR) {
                    w[0] *= l0[q];
                    w[1] *= l0p[q];
                    w[2] *= l1[q];
                    w[3] *= l1p[q];
                    w[4] *= l2[q];
                    w[5] *= q < 3 ? l2[q + 1] : l2r;
                }
                const T km = q > 0 ? own[q - 1] : left, kp = q < 3 ? own[q + 1] : right;
                const T sv = w[0] * xm[q] + w[1] * xp[q] + w[2] * ym[q] + w[3] * yp[q] + w[4] * km + w[5] * kp;
                const T d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
                r[q] = bb[q] + d * own[q] - sv;
            }
            acc0 += rab * (rk[0] * r[0] + rk[1] * r[1]);
            acc1 += rab * (rk[2] * r[2] + rk[3] * r[3]);
        }
    }
    C.b[cell32(C, I, J, K0)] = acc0;
    C.b[cell32(C, I, J, K0 + 1)] = acc1;
}

template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_restrict_quad(Bricks<T> FB, Bricks<T> CB, TransferSet ts) {
    grid_dep_sync();
    int I;
    const int b = brick_of(CB, blockIdx.z, I);
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    if (J >= CB.v[b].n1 || 2 * P >= CB.v[b].n2) return;
    restrict_quad_item<T, VAR>(FB.v[b], CB.v[b], ts.t[b], I, J, P);
}

// ---------------------------------------------------------------------------
// The same two transfers for a parity-split fine level (single brick,
// factor 2 along every axis): a thread owns the fine slots 4P .. 4P+3 of
// both halves of a row -- the eight consecutive cells k = 8P .. 8P+7, four
// even and four odd -- so every fine array moves as whole vectors.  The
// restriction writes the coarse cells K = 4P .. 4P+3 (the parents of
// those eight), the prolongation reads them and their two outer
// neighbours.  Per cell the arithmetic and its order are those of
// restrict_quad_item and prolong_quad_item, so the results are
// bit-identical.
// ---------------------------------------------------------------------------
template <typename T, bool VAR>
__global__ void __launch_bounds__(256, sizeof(T) == 4 && !VAR ? 3 : 2) k_restrict_split(Bricks<T> FB, Bricks<T> CB,
                                                                                   TransferSet ts) {
    grid_dep_sync();
    const LevelView<T>& F = FB.v[0];
    const LevelView<T>& C = CB.v[0];
    const TransferTabs& t = ts.t[0];
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    const int I = blockIdx.z;
    const int kh = F.kh;
    if (J >= C.n1 || 4 * P >= kh) return;
    const T* ratio;
    if constexpr (sizeof(T) == 8)
        ratio = reinterpret_cast<const T*>(t.ratio64);
    else
        ratio = reinterpret_cast<const T*>(t.ratio32);
    const int m0 = 4 * P;
    // k couplings and k shares of the even (k = 2(m0+m)) and odd cells: the
    // eight consecutive k = 8P .. 8P+7 of the natural tables, as vectors
    T wke[4], whe[4], wko[4], who[4], rke[4], rko[4];
    {
        T a[8], b[8], r[8];
        Row4<T>::ldg4(F.tab + F.to.wl[2] + 2 * m0, a);
        Row4<T>::ldg4(F.tab + F.to.wl[2] + 2 * m0 + 4, a + 4);
        Row4<T>::ldg4(F.tab + F.to.wh[2] + 2 * m0, b);
        Row4<T>::ldg4(F.tab + F.to.wh[2] + 2 * m0 + 4, b + 4);
        const T* rp = ratio + F.n0 + F.n1 + 2 * m0;
        if (((F.n0 + F.n1) & 3) == 0) {  // 16-byte aligned: two vectors
            Row4<T>::ldg4(rp, r);
            Row4<T>::ldg4(rp + 4, r + 4);
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) r[q] = ldg(rp + q);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            wke[m] = a[2 * m];
            wko[m] = a[2 * m + 1];
            whe[m] = b[2 * m];
            who[m] = b[2 * m + 1];
            rke[m] = r[2 * m];
            rko[m] = r[2 * m + 1];
        }
    }
    T acc[4] = {T(0), T(0), T(0), T(0)};
    // FP64 and variable-coefficient rows hold twice the registers: one fine
    // plane at a time there
#pragma unroll(sizeof(T) == 4 && !VAR ? 2 : 1)
    for (int a = 0; a < 2; ++a) {
        const int i = 2 * I + a;
        const T ra = ldg(ratio + i);
        const T wil = ldg(F.tab + F.to.wl[0] + i), wih = ldg(F.tab + F.to.wh[0] + i);
#pragma unroll
        for (int e = 0; e < 2; ++e) {
            const int j = 2 * J + e;
            const T rab = ra * ldg(ratio + F.n0 + j);
            const T wjl = ldg(F.tab + F.to.wl[1] + j), wjh = ldg(F.tab + F.to.wh[1] + j);
            const int si = (int)F.si, sj = (int)F.sj;
            const int row = (int)row_at(F, i, j);
            const int ce = row + m0, co = row + kh + m0;           // even and odd slots
            const int clo = m0 > 0 ? co - 1 : row - 1;            // k = 8P - 1
            const int chi = m0 + 4 < kh ? ce + 4 : row + 2 * kh;  // k = 8P + 8
            T xe[4], xo[4], me[4], mo[4], pe[4], po[4], ne[4], no[4], qe[4], qo[4], be[4], bo[4];
            Row4<T>::ld(F.x + ce, xe);
            Row4<T>::ld(F.x + co, xo);
            Row4<T>::ld(F.x + ce - si, me);
            Row4<T>::ld(F.x + co - si, mo);
            Row4<T>::ld(F.x + ce + si, pe);
            Row4<T>::ld(F.x + co + si, po);
            Row4<T>::ld(F.x + ce - sj, ne);
            Row4<T>::ld(F.x + co - sj, no);
            Row4<T>::ld(F.x + ce + sj, qe);
            Row4<T>::ld(F.x + co + sj, qo);
            Row4<T>::ld(F.b + ce, be);
            Row4<T>::ld(F.b + co, bo);
            const T left = F.x[clo], right = F.x[chi];
            T l0e[4], l0o[4], l0pe[4], l0po[4], l1e[4], l1o[4], l1pe[4], l1po[4], l2e[4], l2o[4], l2r = T(1);
            if (VAR) {
                Row4<T>::ldg4(F.lam0 + ce, l0e);
                Row4<T>::ldg4(F.lam0 + co, l0o);
                Row4<T>::ldg4(F.lam0 + ce + si, l0pe);
                Row4<T>::ldg4(F.lam0 + co + si, l0po);
                Row4<T>::ldg4(F.lam1 + ce, l1e);
                Row4<T>::ldg4(F.lam1 + co, l1o);
                Row4<T>::ldg4(F.lam1 + ce + sj, l1pe);
                Row4<T>::ldg4(F.lam1 + co + sj, l1po);
                Row4<T>::ldg4(F.lam2 + ce, l2e);
                Row4<T>::ldg4(F.lam2 + co, l2o);
                l2r = ldg(F.lam2 + chi);
            }
#pragma unroll
            for (int m = 0; m < 4; ++m) {
                // the even cell k = 2(m0+m) and the odd cell k + 1, in that order
                T r2[2];
#pragma unroll
                for (int sd = 0; sd < 2; ++sd) {
                    T w[6] = {wil, wih, wjl, wjh, sd ? wko[m] : wke[m], sd ? who[m] : whe[m]};
                    if (VAR) {
                        w[0] *= sd ? l0o[m] : l0e[m];
                        w[1] *= sd ? l0po[m] : l0pe[m];
                        w[2] *= sd ? l1o[m] : l1e[m];
                        w[3] *= sd ? l1po[m] : l1pe[m];
                        w[4] *= sd ? l2o[m] : l2e[m];
                        // upper k face: the lower face of the next cell
                        w[5] *= sd ? (m < 3 ? l2e[m + 1] : l2r) : l2o[m];
                    }
                    const T own = sd ? xo[m] : xe[m];
                    const T km = sd ? xe[m] : (m > 0 ? xo[m - 1] : left);
                    const T kp = sd ? (m < 3 ? xe[m + 1] : right) : xo[m];
                    const T xmv = sd ? mo[m] : me[m], xpv = sd ? po[m] : pe[m];
                    const T ymv = sd ? no[m] : ne[m], ypv = sd ? qo[m] : qe[m];
                    const T sv = w[0] * xmv + w[1] * xpv + w[2] * ymv + w[3] * ypv + w[4] * km + w[5] * kp;
                    const T d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
                    r2[sd] = (sd ? bo[m] : be[m]) + d * own - sv;
                }
                acc[m] += rab * (rke[m] * r2[0] + rko[m] * r2[1]);
            }
        }
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) C.b[cell32(C, I, J, m0 + m)] = acc[m];
}

template <typename T>
__global__ void __launch_bounds__(256) k_prolong_split(Bricks<T> FB, Bricks<T> CB, TransferSet ts) {
    grid_dep_sync();
    const LevelView<T>& F = FB.v[0];
    const LevelView<T>& C = CB.v[0];
    const TransferTabs& t = ts.t[0];
    const int P = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    const int kh = F.kh;
    if (j >= F.n1 || 4 * P >= kh) return;
    const int m0 = 4 * P;
    const int* pidx = t.pidx;
    const T* pw;
    if constexpr (sizeof(T) == 8)
        pw = reinterpret_cast<const T*>(t.pw64);
    else
        pw = reinterpret_cast<const T*>(t.pw32);
    const int I0 = ldg(pidx + 2 * i), I1 = ldg(pidx + 2 * i + 1);
    const int J0 = ldg(pidx + 2 * F.n0 + 2 * j), J1 = ldg(pidx + 2 * F.n0 + 2 * j + 1);
    const T wi = ldg(pw + i), wj = ldg(pw + F.n0 + j);
    const T ui = T(1) - wi, uj = T(1) - wj;
    const int* pk = pidx + 2 * (F.n0 + F.n1);
    const T* wk = pw + F.n0 + F.n1;
    // parents of the eight cells: K = m0 .. m0+3; second coarse cells: K - 1
    // for the even cells and K + 1 for the odd ones, the outer two from the
    // tables (they may be a wrapped, a ghost or the parent's own index)
    const int Klo = kpos(C, ldg(pk + 2 * (2 * m0) + 1));
    const int Khi = kpos(C, ldg(pk + 2 * (2 * m0 + 7) + 1));
    T we[4], ue[4], wo[4], uo[4];
    {
        T a[8];  // the weights of k = 8P .. 8P+7 (natural order, contiguous)
        if (((F.n0 + F.n1) & 3) == 0) {  // 16-byte aligned: two vectors
            Row4<T>::ldg4(wk + 2 * m0, a);
            Row4<T>::ldg4(wk + 2 * m0 + 4, a + 4);
        } else {
#pragma unroll
            for (int q = 0; q < 8; ++q) a[q] = ldg(wk + 2 * m0 + q);
        }
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            we[m] = a[2 * m];
            wo[m] = a[2 * m + 1];
            ue[m] = T(1) - we[m];
            uo[m] = T(1) - wo[m];
        }
    }
    const int rows[4] = {cell32(C, I0, J0, 0), cell32(C, I0, J1, 0), cell32(C, I1, J0, 0), cell32(C, I1, J1, 0)};
    T ve[4][4], vo[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const T* X = C.x + rows[r];
        T xc[4];  // the parents K = m0 .. m0+3
        if (C.kh) {
            Row4<T>::ld2(X + m0 / 2, xc[0], xc[2]);
            Row4<T>::ld2(X + C.kh + m0 / 2, xc[1], xc[3]);
        } else {
            Row4<T>::ld(X + m0, xc);
        }
        const T xlo = X[Klo], xhi = X[Khi];
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            ve[r][m] = ue[m] * xc[m] + we[m] * (m > 0 ? xc[m - 1] : xlo);
            vo[r][m] = uo[m] * xc[m] + wo[m] * (m < 3 ? xc[m + 1] : xhi);
        }
    }
    const int row = (int)row_at(F, i, j);
    const int ce = row + m0, co = row + kh + m0;
    T xe[4], xo[4];
    Row4<T>::ld(F.x + ce, xe);
    Row4<T>::ld(F.x + co, xo);
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        xe[m] += ui * (uj * ve[0][m] + wj * ve[1][m]) + wi * (uj * ve[2][m] + wj * ve[3][m]);
        xo[m] += ui * (uj * vo[0][m] + wj * vo[1][m]) + wi * (uj * vo[2][m] + wj * vo[3][m]);
    }
    Row4<T>::st(F.x + ce, xe);
    Row4<T>::st(F.x + co, xo);
    if ((F.per0 && (i == 0 || i == F.n0 - 1)) || (F.per1 && (j == 0 || j == F.n1 - 1)) ||
        (F.per2 && (m0 == 0 || m0 + 4 == kh))) {
#pragma unroll
        for (int m = 0; m < 4; ++m) {
            store_images(F, ce + m, i, j, 2 * (m0 + m), xe[m]);
            store_images(F, co + m, i, j, 2 * (m0 + m) + 1, xo[m]);
        }
    }
}

// ---------------------------------------------------------------------------
// Coarse direct solve: x = inverse(A'_pinned) b' with b'(0) = 0 (MG.C:37-40,
// solver.C:201-231, APLU.C:91-128); a singular system's inverse comes with
// its first column zeroed, which is that b'(0) = 0.  One CTA; the inverse is
// factored once per matrix on the host in FP64.  cidx gives the slab index of every
// unknown (bricks one after another, k fastest).
// ---------------------------------------------------------------------------
// rows r0, r0 + rstep, ... of x = A^-1 b, one warp per row (the CTA's
// warps take consecutive rows); sb: n doubles of shared memory.  A row's
// sum is formed the same way whichever CTA forms it.
template <typename T>
__device__ __forceinline__ void coarse_solve_block(const Bricks<T>& CB, const double* __restrict__ ainv,
                                                   const int* __restrict__ cidx, int n, double* sb, int r0 = 0,
                                                   int rstep = 0) {
    const T* bsrc = CB.v[0].b;
    for (int q = threadIdx.x; q < n; q += blockDim.x) sb[q] = (double)bsrc[cidx[q]];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    if (rstep == 0) rstep = nw;
    for (int r = r0 + warp; r < n; r += rstep) {
        double s = 0.0;
        for (int l = lane; l < n; l += 32) s += ainv[(long)r * n + l] * sb[l];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            if (CB.nb == 1) {
                // single brick: also refresh the periodic ghost images
                const LevelView<T>& C = CB.v[0];
                const int nn = C.n1 * C.n2;
                const int i = r / nn, j = (r / C.n2) % C.n1, k = r % C.n2;
                store_x(C, row_at(C, i, j) + kpos(C, k), i, j, k, (T)s);
            } else {
                CB.v[0].x[cidx[r]] = (T)s;
            }
        }
    }
}

// the dense coarse solve over many CTAs: CTA c takes rows 8c .. 8c + 7,
// then 8 (c + gridDim.x) .., so the inverse streams through all SMs
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_solve(Bricks<T> CB, const double* __restrict__ ainv,
                                                      const int* __restrict__ cidx, int n) {
    grid_dep_sync();
    extern __shared__ double sb[];
    const int nw = blockDim.x >> 5;
    coarse_solve_block<T>(CB, ainv, cidx, n, sb, blockIdx.x * nw, gridDim.x * nw);
}

// ---------------------------------------------------------------------------
// The coarse end of a V-cycle in one CTA: on the small levels every pass is
// a few thousand cells, so a launch per pass costs more than the pass.  The
// levels from P.first down to the coarse solve level run here with a barrier
// between passes: pre-smoothing colour passes, restriction (and the zeroed
// coarse x), the dense coarse solve, then prolongation and post-smoothing on
// the way up -- the same per-item functions as the per-pass kernels, so the
// result is bit-identical to the per-pass path (MG.C:19-130, V cycle).
// ---------------------------------------------------------------------------
template <typename T, bool VAR>
__global__ void __launch_bounds__(kTailThreads) k_tail_cycle(TailPlan<T> P) {
    grid_dep_sync();
    extern __shared__ double sb[];
    const int nt = blockDim.x;
    const int nl = P.nlev;
    auto smooth = [&](int q, const int* seq, int nseq) {
        const LevelView<T>& L = P.v[q];
        const int nq = L.n2 / 4;
        const int items = L.n0 * L.n1 * nq;
        for (int s = 0; s < nseq; ++s) {
            for (int it = threadIdx.x; it < items; it += nt) {
                const int p = it % nq, ij = it / nq;
                colour_quad_item<T, VAR>(L, ij / L.n1, ij % L.n1, p, seq[s]);
            }
            __syncthreads();
        }
    };
    for (int q = 0; q < nl - 1; ++q) {
        smooth(q, P.pre[q], P.npre[q]);
        const LevelView<T>& F = P.v[q];
        const LevelView<T>& C = P.v[q + 1];
        const int np = C.n2 / 2;
        const int items = C.n0 * C.n1 * np;
        for (int it = threadIdx.x; it < items; it += nt) {
            const int pp = it % np, IJ = it / np;
            restrict_quad_item<T, VAR>(F, C, P.t[q], IJ / C.n1, IJ % C.n1, pp);
        }
        // x(q+1) = 0 over the whole slab (the per-pass path's memset)
        for (long c = threadIdx.x; c < C.cells; c += nt) C.x[c] = T(0);
        __syncthreads();
    }
    Bricks<T> CB{};
    CB.v[0] = P.v[nl - 1];
    CB.nb = 1;
    coarse_solve_block<T>(CB, P.ainv, P.cidx, P.ncoarse, sb);
    __syncthreads();
    for (int q = nl - 2; q >= 0; --q) {
        const LevelView<T>& F = P.v[q];
        const int nq = F.n2 / 4;
        const int items = F.n0 * F.n1 * nq;
        for (int it = threadIdx.x; it < items; it += nt) {
            const int p = it % nq, ij = it / nq;
            prolong_quad_item<T>(F, P.v[q + 1], P.t[q], ij / F.n1, ij % F.n1, p);
        }
        __syncthreads();
        smooth(q, P.post[q], P.npost[q]);
    }
}

template <typename T>
__global__ void k_fill_ghosts(T* x, const int* __restrict__ dst, const int* __restrict__ src, long n) {
    grid_dep_sync();
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        x[dst[q]] = x[src[q]];
}

// residual r = b - A x of any level, unscaled, into a compact array
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_residual_out(Bricks<T> B, double* out) {
    grid_dep_sync();
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    T w[6], s, d;
    const long ckm = row + kpos(L, k - 1), ckp = row + kpos(L, k + 1);
    couplings<T, VAR>(L, i, j, k, c, ckp, w);
    stencil(L.x, c, ckm, ckp, L.si, L.sj, w, s, d);
    const double r = (double)(L.b[c] + d * L.x[c] - s);
    const double V = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
    out[compact_index(L, i, j, k)] = r * V;
}

// ---------------------------------------------------------------------------
// Level-0 residual norms in FP64 (MG.C:163-174,223-230; solver.C:13-61).
// One cell per thread over the same grid as the other cell kernels, one
// partial sum per block; the finalize kernel adds the partials in a fixed
// order, so sums are reproducible.  mode 0 also accumulates the normFactor
// sum (|r - b + A ybar| + |b - A ybar|)^2, ybar = mean(x): the row sums of
// the level-0 operator vanish (every coupling is paired with the centre)
// except in the rows of Dirichlet faces.
// ---------------------------------------------------------------------------
template <bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_residual_norm(Bricks<double> B, Walls W, int mode,
                                                                  double* partials, long nblocks, float* b32) {
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
        const double V = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
        const double rr = V * r;
        a1 = rr * rr;
        if (mode == 0) {
            const double bb = V * L.b[c];
            // A*mean(x): nonzero only in the rows of Dirichlet faces
            const double ay =
                W.mask[bk] ? -V * *W.ybar * wall_sum(L, W, bk, i, j, k, c, ckp, false) : 0.0;
            const double t = fabs(rr - bb + ay) + fabs(bb - ay);
            a2 = t * t;
            a3 = bb * bb;
        }
        if (b32) b32[c] = (float)r;
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

// solver.C:13-95 on the reduced sums; also decides whether the loop goes on
// (MG.C:191-195) and, inside the solve graph, hands that decision to the
// WHILE node (bounded by maxIter, so the device loop always ends).
__global__ void __launch_bounds__(kFinalThreads) k_finalize(const double* partials, long nblocks,
                                                             SolveState* st, int mode,
                                                             cudaGraphConditionalHandle cond,
                                                             int setCondition) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double a1 = sum_partials<kFinalThreads>(partials, nblocks, sh);
    double a2 = 0.0, a3 = 0.0;
    if (mode == 0) {
        a2 = sum_partials<kFinalThreads>(partials + nblocks, nblocks, sh);
        a3 = sum_partials<kFinalThreads>(partials + 2 * nblocks, nblocks, sh);
    }
    if (threadIdx.x == 0) {
        const double l2 = sqrt(a1);
        if (mode == 0) {
            // normFactor floor: 1e-12 per cell (solver.C:53-58)
            st->nf = fmax(sqrt(a2), st->ncells * 1e-12);
            st->init = l2 / st->nf;
            st->cur = st->init;
            st->l2_0 = l2;
            st->bnorm = sqrt(a3);
            st->iter = 0;
        } else {
            st->cur = l2 / st->nf;
            st->iter += 1;
        }
        st->l2 = l2;
        st->nan = !isfinite(st->cur);
        // solver.C:64-95; criterion 1 measures the residual against ||b||
        // instead of the initial residual
        if (st->criterion == 1)
            st->converged = !((st->bnorm > 0.0) && (st->cur > st->abs_tol) && (l2 > st->rel_tol * st->bnorm));
        else
            st->converged = !((st->init > 0.0) && (st->cur > st->abs_tol) &&
                              (st->cur / (st->init + 1e-20) > st->rel_tol));
        st->keep_going = !st->nan && ((st->iter < st->max_iter && !st->converged) ||
                                      st->iter < st->min_iter);
        if (setCondition) cudaGraphSetConditional(cond, st->keep_going ? 1u : 0u);
    }
}

__global__ void __launch_bounds__(kReduceThreads) k_mean_partials(Bricks<double> B, double* partials) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a = 0.0;
    if (j < L.n1 && k < L.n2) {
        const long row = row_at(L, i, j), c = row + kpos(L, k);
        a = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k] * L.x[c];
    }
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

__global__ void __launch_bounds__(kFinalThreads) k_mean_finalize(const double* partials, long nblocks,
                                                                 SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double a = sum_partials<kFinalThreads>(partials, nblocks, sh);
    if (threadIdx.x == 0) st->mean = a / st->vol_total;
}

// plain (unweighted) sum of the interior x per block, then the mean
__global__ void __launch_bounds__(kReduceThreads) k_plain_partials(Bricks<double> B, double* partials) {
    grid_dep_sync();
    __shared__ double sh[kReduceThreads / 32];
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    double a = 0.0;
    if (j < L.n1 && k < L.n2) a = L.x[row_at(L, i, j) + kpos(L, k)];
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0 && threadIdx.y == 0) partials[block_id()] = a;
}

__global__ void __launch_bounds__(kFinalThreads) k_plain_finalize(const double* partials, long nblocks,
                                                                  SolveState* st) {
    grid_dep_sync();
    __shared__ double sh[kFinalThreads / 32];
    const double a = sum_partials<kFinalThreads>(partials, nblocks, sh);
    if (threadIdx.x == 0) st->ybar = a / st->ncells;
}

// subtract the mean everywhere, ghosts included (a constant shift keeps the
// periodic images consistent)
__global__ void k_sub_mean(double* x, long n, const SolveState* st) {
    grid_dep_sync();
    const double m = st->mean;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        x[q] -= m;
}

__global__ void __launch_bounds__(256) k_load_b(Bricks<double> B, Walls W, const double* compact) {
    grid_dep_sync();
    int i;
    const int bk = brick_of(B, blockIdx.z, i);
    const LevelView<double>& L = B.v[bk];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    const double V = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
    double v = compact[compact_index(L, i, j, k)] / V;
    // face values: Dirichlet b -= 2 A_f g, Neumann b -= A_f g / delta
    if (W.mask[bk] | W.nmask[bk]) v -= wall_sum(L, W, bk, i, j, k, c, row + kpos(L, k + 1), true);
    L.b[c] = v;
}

__global__ void __launch_bounds__(256) k_load_x(Bricks<double> B, const double* compact) {
    grid_dep_sync();
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    store_x(L, c, i, j, k, compact[compact_index(L, i, j, k)]);
}

__global__ void __launch_bounds__(256) k_store_x(Bricks<double> B, double* compact) {
    grid_dep_sync();
    int i;
    const LevelView<double>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    compact[compact_index(L, i, j, k)] = L.x[c];
}

template <typename T>
__global__ void __launch_bounds__(256) k_load_field(Bricks<T> B, int field, const double* compact, int unscale) {
    grid_dep_sync();
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    double v = compact[compact_index(L, i, j, k)];
    if (field == 0) {
        store_x(L, c, i, j, k, (T)v);
    } else {
        if (unscale) v /= L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
        L.b[c] = (T)v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_store_field(Bricks<T> B, int field, double* compact, int unscale) {
    grid_dep_sync();
    int i;
    const LevelView<T>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    double v = field == 0 ? (double)L.x[c] : (double)L.b[c];
    if (field == 1 && unscale)
        v *= L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
    compact[compact_index(L, i, j, k)] = v;
}

// A single-brick FP32 level and a plain interior array (index (i n1 + j) n2
// + k, the level's own frame): b to the array, the array to x (with its
// periodic images) -- the two ends of a level solver (bmg_set_level_solver).
__global__ void __launch_bounds__(256) k_b_to_plain32(Bricks<float> B, float* out) {
    grid_dep_sync();
    int i;
    const LevelView<float>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    out[((long)i * L.n1 + j) * L.n2 + k] = L.b[row_at(L, i, j) + kpos(L, k)];
}

__global__ void __launch_bounds__(256) k_plain32_to_x(Bricks<float> B, const float* in) {
    grid_dep_sync();
    int i;
    const LevelView<float>& L = B.v[brick_of(B, blockIdx.z, i)];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    store_x(L, row_at(L, i, j) + kpos(L, k), i, j, k, in[((long)i * L.n1 + j) * L.n2 + k]);
}

__global__ void __launch_bounds__(256) k_add_correction(Bricks<double> B, Bricks<float> E) {
    grid_dep_sync();
    int i;
    const int b = brick_of(B, blockIdx.z, i);
    const LevelView<double>& L = B.v[b];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (j >= L.n1 || k >= L.n2) return;
    const long row = row_at(L, i, j), c = row + kpos(L, k);
    store_x(L, c, i, j, k, L.x[c] + (double)E.v[b].x[c]);
}

}  // namespace

// ---- launchers --------------------------------------------------------------

long reduce_blocks(const Bricks<double>& B) {
    const dim3 blk = block_for(B.max2);
    const dim3 g = grid_for(B, B.max2, blk);
    return (long)g.x * g.y * g.z;
}

template <typename T, bool VAR>
void launch_colour_pass(const Bricks<T>& B, int colour, cudaStream_t s, bool zero) {
    if (B.v[0].kh) {  // parity-split rows (single brick, n2 % 16 == 0)
        const LevelView<T>& L = B.v[0];
        const int tr = L.kh / (16 / (int)sizeof(T));  // threads per half row
        int bx = 1;
        while (bx < tr && bx < 32) bx *= 2;
        const dim3 blk(bx, 256 / bx, 1);
        const dim3 grid((tr + bx - 1) / bx, (L.n1 + blk.y - 1) / blk.y, L.n0);
        if (zero)
            launch_k(k_colour_split<T, VAR, true>, grid, blk, 0, s, L, colour);
        else
            launch_k(k_colour_split<T, VAR, false>, grid, blk, 0, s, L, colour);
        return;
    }
    bool quads = true;
    for (int b = 0; b < B.nb; ++b) quads = quads && B.v[b].n2 % 4 == 0;
    if (quads) {
        // one row per thread: two rows per thread (R = 2) measured no faster
        // on the 256^3 level and costs registers in FP64
        const int nq = B.max2 / 4;
        const dim3 blk = nq >= 32 ? dim3(32, 8, 1) : nq >= 8 ? dim3(8, 32, 1) : dim3(2, 128, 1);
        launch_k(k_colour_quad<T, VAR>, grid_for(B, nq, blk), blk, 0, s, B, colour);
        return;
    }
    const int pairs = (B.max2 + 1) / 2;
    const dim3 blk = pairs >= 32 ? dim3(32, 8, 1) : pairs >= 8 ? dim3(8, 32, 1) : dim3(2, 128, 1);
    launch_k(k_colour_pass<T, VAR>, grid_for(B, pairs, blk), blk, 0, s, B, colour);
}

template <typename T, bool VAR>
void launch_jacobi(const Bricks<T>& B, T* tmp, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_jacobi<T, VAR>, grid_for(B, B.max2, blk), blk, 0, s, B, tmp);
    launch_k(k_copy_interior<T>, grid_for(B, B.max2, blk), blk, 0, s, B, tmp);
}

// factor-2 coarsening along every axis and n2 % 4 == 0 on the fine level
template <typename T>
bool quad_transfers(const Bricks<T>& F, const TransferSet& t) {
    for (int b = 0; b < F.nb; ++b)
        if (t.t[b].R0 != 2 || t.t[b].R1 != 2 || t.t[b].R2 != 2 || F.v[b].n2 % 4) return false;
    return true;
}

// the split-level transfers: blocks of 256 threads over (slot groups, rows), one plane per grid z
inline dim3 split_block(int groups) {
    int bx = 1;
    while (bx < groups && bx < 32) bx *= 2;
    return dim3(bx, 256 / bx, 1);
}

template <typename T, bool VAR>
void launch_residual_restrict(const Bricks<T>& F, const Bricks<T>& C, const TransferSet& t, cudaStream_t s) {
    if (F.v[0].kh && quad_transfers(F, t)) {
        const int groups = F.v[0].kh / 4;
        const dim3 blk = split_block(groups);
        const dim3 grid((groups + blk.x - 1) / blk.x, (C.v[0].n1 + blk.y - 1) / blk.y, C.v[0].n0);
        launch_k(k_restrict_split<T, VAR>, grid, blk, 0, s, F, C, t);
        return;
    }
    if (quad_transfers(F, t)) {
        const int np = C.max2 / 2;
        const dim3 blk = np >= 32 ? dim3(32, 8, 1) : np >= 8 ? dim3(8, 32, 1) : dim3(2, 128, 1);
        launch_k(k_restrict_quad<T, VAR>, grid_for(C, np, blk), blk, 0, s, F, C, t);
        return;
    }
    const dim3 blk = block_for(C.max2);
    launch_k(k_residual_restrict<T, VAR>, grid_for(C, C.max2, blk), blk, 0, s, F, C, t);
}

template <typename T>
void launch_prolong_correct(const Bricks<T>& F, const Bricks<T>& C, const TransferSet& t, cudaStream_t s) {
    if (F.v[0].kh && quad_transfers(F, t)) {
        const int groups = F.v[0].kh / 4;
        const dim3 blk = split_block(groups);
        const dim3 grid((groups + blk.x - 1) / blk.x, (F.v[0].n1 + blk.y - 1) / blk.y, F.v[0].n0);
        launch_k(k_prolong_split<T>, grid, blk, 0, s, F, C, t);
        return;
    }
    if (quad_transfers(F, t)) {
        const int nq = F.max2 / 4;
        const dim3 blk = nq >= 32 ? dim3(32, 8, 1) : nq >= 8 ? dim3(8, 32, 1) : dim3(2, 128, 1);
        launch_k(k_prolong_quad<T>, grid_for(F, nq, blk), blk, 0, s, F, C, t);
        return;
    }
    const dim3 blk = block_for(F.max2);
    launch_k(k_prolong_correct<T>, grid_for(F, F.max2, blk), blk, 0, s, F, C, t);
}

template <typename T>
void launch_coarse_solve(const Bricks<T>& C, const double* ainv, const int* cidx, int n, cudaStream_t s) {
    const int grid = std::min((n + 7) / 8, 1184);  // 8 rows (warps) per CTA
    launch_k(k_coarse_solve<T>, grid, 256, n * sizeof(double), s, C, ainv, cidx, n);
}

template <typename T, bool VAR>
void launch_tail_cycle(const TailPlan<T>& P, cudaStream_t s) {
    launch_k(k_tail_cycle<T, VAR>, 1, kTailThreads, P.ncoarse * sizeof(double), s, P);
}

template <typename T>
void launch_fill_ghosts(T* x, const int* dst, const int* src, long n, cudaStream_t s) {
    const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 8);
    launch_k(k_fill_ghosts<T>, blocks, 256, 0, s, x, dst, src, n);
}

template <typename T, bool VAR>
void launch_residual_out(const Bricks<T>& B, double* out, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_residual_out<T, VAR>, grid_for(B, B.max2, blk), blk, 0, s, B, out);
}

template <bool VAR>
long launch_residual_norm(const Bricks<double>& B, const Walls& W, int mode, double* partials, float* b32,
                          cudaStream_t s) {
    if (B.v[0].kh) return launch_residual_split<VAR>(B, W, mode, nullptr, b32, nullptr, partials, s);
    const dim3 blk = block_for(B.max2);
    launch_k(k_residual_norm<VAR>, grid_for(B, B.max2, blk), blk, 0, s, B, W, mode, partials, reduce_blocks(B), b32);
    return reduce_blocks(B);
}

void launch_finalize(const Bricks<double>& B, const double* partials, SolveState* st, int mode,
                     cudaGraphConditionalHandle cond, int setCondition, cudaStream_t s) {
    launch_k(k_finalize, 1, kFinalThreads, 0, s, partials, reduce_blocks(B), st, mode, cond, setCondition);
}

void launch_finalize_n(const double* partials, long n, SolveState* st, int mode, cudaGraphConditionalHandle cond,
                       int setCondition, cudaStream_t s) {
    launch_k(k_finalize, 1, kFinalThreads, 0, s, partials, n, st, mode, cond, setCondition);
}

void launch_mean(const Bricks<double>& B, double* partials, SolveState* st, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_mean_partials, grid_for(B, B.max2, blk), blk, 0, s, B, partials);
    launch_k(k_mean_finalize, 1, kFinalThreads, 0, s, partials, reduce_blocks(B), st);
    const long n = B.v[0].cells;
    const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 16);
    launch_k(k_sub_mean, blocks, 256, 0, s, B.v[0].x, n, st);
}

void launch_plain_mean(const Bricks<double>& B, double* partials, SolveState* st, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_plain_partials, grid_for(B, B.max2, blk), blk, 0, s, B, partials);
    launch_k(k_plain_finalize, 1, kFinalThreads, 0, s, partials, reduce_blocks(B), st);
}

void launch_load_b(const Bricks<double>& B, const Walls& W, const double* compact, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_load_b, grid_for(B, B.max2, blk), blk, 0, s, B, W, compact);
}

void launch_load_x(const Bricks<double>& B, const double* compact, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_load_x, grid_for(B, B.max2, blk), blk, 0, s, B, compact);
}

void launch_store_x(const Bricks<double>& B, double* compact, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_store_x, grid_for(B, B.max2, blk), blk, 0, s, B, compact);
}

template <typename T>
void launch_load_field(const Bricks<T>& B, int field, const double* compact, int unscale, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_load_field<T>, grid_for(B, B.max2, blk), blk, 0, s, B, field, compact, unscale);
}

template <typename T>
void launch_store_field(const Bricks<T>& B, int field, double* compact, int unscale, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_store_field<T>, grid_for(B, B.max2, blk), blk, 0, s, B, field, compact, unscale);
}

void launch_b_to_plain32(const Bricks<float>& B, float* out, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_b_to_plain32, grid_for(B, B.max2, blk), blk, 0, s, B, out);
}

void launch_plain32_to_x(const Bricks<float>& B, const float* in, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_plain32_to_x, grid_for(B, B.max2, blk), blk, 0, s, B, in);
}

void launch_add_correction(const Bricks<double>& B, const Bricks<float>& E, cudaStream_t s) {
    const dim3 blk = block_for(B.max2);
    launch_k(k_add_correction, grid_for(B, B.max2, blk), blk, 0, s, B, E);
}

// explicit instantiations
#define BMG_INST(T, V)                                                                                   \
    template void launch_colour_pass<T, V>(const Bricks<T>&, int, cudaStream_t, bool);                   \
    template void launch_jacobi<T, V>(const Bricks<T>&, T*, cudaStream_t);                               \
    template void launch_residual_restrict<T, V>(const Bricks<T>&, const Bricks<T>&, const TransferSet&, \
                                                 cudaStream_t);                                          \
    template void launch_residual_out<T, V>(const Bricks<T>&, double*, cudaStream_t);
BMG_INST(double, false)
BMG_INST(double, true)
BMG_INST(float, false)
BMG_INST(float, true)
#undef BMG_INST
template void launch_prolong_correct<double>(const Bricks<double>&, const Bricks<double>&, const TransferSet&,
                                             cudaStream_t);
template void launch_prolong_correct<float>(const Bricks<float>&, const Bricks<float>&, const TransferSet&,
                                            cudaStream_t);
template void launch_coarse_solve<double>(const Bricks<double>&, const double*, const int*, int, cudaStream_t);
template void launch_coarse_solve<float>(const Bricks<float>&, const double*, const int*, int, cudaStream_t);
template void launch_tail_cycle<double, false>(const TailPlan<double>&, cudaStream_t);
template void launch_tail_cycle<double, true>(const TailPlan<double>&, cudaStream_t);
template void launch_tail_cycle<float, false>(const TailPlan<float>&, cudaStream_t);
template void launch_tail_cycle<float, true>(const TailPlan<float>&, cudaStream_t);
template void launch_fill_ghosts<double>(double*, const int*, const int*, long, cudaStream_t);
template void launch_fill_ghosts<float>(float*, const int*, const int*, long, cudaStream_t);
template long launch_residual_norm<false>(const Bricks<double>&, const Walls&, int, double*, float*, cudaStream_t);
template long launch_residual_norm<true>(const Bricks<double>&, const Walls&, int, double*, float*, cudaStream_t);
template void launch_load_field<double>(const Bricks<double>&, int, const double*, int, cudaStream_t);
template void launch_load_field<float>(const Bricks<float>&, int, const double*, int, cudaStream_t);
template void launch_store_field<double>(const Bricks<double>&, int, double*, int, cudaStream_t);
template void launch_store_field<float>(const Bricks<float>&, int, double*, int, cudaStream_t);

}  // namespace bmg
