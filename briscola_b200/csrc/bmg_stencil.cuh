// bmg_stencil.cuh -- the 7-point stencil arithmetic shared by every kernel
// that updates or evaluates a cell, so that the per-colour and the fused
// smoothers produce bit-identical values.
#pragma once

#include "bmg_internal.h"

namespace bmg {

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
    return __ldg(p);
}

// Storage position of logical k (-1 .. n2) in a row: k itself in natural
// rows (kh = 0); in a parity-split row (kh = n2/2) the even k first, then
// the odd k, with the ghosts k = -1 and k = n2 at their natural places.
__device__ __forceinline__ int kpos_split(int k, int kh) {
    return (k >= 0 && k < 2 * kh) ? (k & 1) * kh + (k >> 1) : k;
}

template <typename T>
__device__ __forceinline__ int kpos(const LevelView<T>& L, int k) {
    return L.kh ? kpos_split(k, L.kh) : k;
}

// Row-scaled couplings of cell (i,j,k) to its six neighbours in the order
// of the reference's row product: l, r, b, t, a, f (linearSystemFunctions.H
// :96-102), i.e. axis 0 lower/upper, axis 1 lower/upper, axis 2 lower/upper.
// c is the cell's slab index, ckp the slab index of cell (i,j,k+1), whose
// lower face is the cell's upper k face.
template <typename T, bool VAR>
__device__ __forceinline__ void couplings(const LevelView<T>& L, int i, int j, int k, long c, long ckp,
                                          T w[6]) {
    w[0] = ldg(L.tab + L.to.wl[0] + i);
    w[1] = ldg(L.tab + L.to.wh[0] + i);
    w[2] = ldg(L.tab + L.to.wl[1] + j);
    w[3] = ldg(L.tab + L.to.wh[1] + j);
    w[4] = ldg(L.tab + L.to.wl[2] + k);
    w[5] = ldg(L.tab + L.to.wh[2] + k);
    if (VAR) {
        w[0] *= ldg(L.lam0 + c);
        w[1] *= ldg(L.lam0 + c + L.si);
        w[2] *= ldg(L.lam1 + c);
        w[3] *= ldg(L.lam1 + c + L.sj);
        w[4] *= ldg(L.lam2 + c);
        w[5] *= ldg(L.lam2 + ckp);
    }
}

// Gauss-Seidel value of a cell from its couplings w, neighbour values xn
// (same order) and right-hand side b: (sum w*xn - b) / sum w, which is
// (b - offdiag row product) / centre of rbgsSmoother.C:76-81 for the
// row-scaled operator.
// The FP32 smoother divides with the hardware reciprocal (about 2 ulp, two
// instructions); the FP64 path keeps IEEE division.  Both smoother kernels
// call this one function, so they stay bit-identical to each other.
// The sums are written with explicit round-to-nearest intrinsics, so the
// compiler cannot contract them into fused multiply-adds differently in
// different kernels: every smoother evaluates the same sequence of roundings.
__device__ __forceinline__ float gs_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double gs_div(double a, double b) { return a / b; }
__device__ __forceinline__ float rn_mul(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double rn_mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float rn_fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double rn_fma(double a, double b, double c) { return __fma_rn(a, b, c); }
__device__ __forceinline__ float rn_add(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double rn_add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float rn_sub(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double rn_sub(double a, double b) { return __dsub_rn(a, b); }

template <typename T>
__device__ __forceinline__ T gs_value(const T w[6], const T xn[6], T b) {
    T s = rn_mul(w[0], xn[0]);
    s = rn_fma(w[1], xn[1], s);
    s = rn_fma(w[2], xn[2], s);
    s = rn_fma(w[3], xn[3], s);
    s = rn_fma(w[4], xn[4], s);
    s = rn_fma(w[5], xn[5], s);
    const T d = rn_add(rn_add(rn_add(rn_add(rn_add(w[0], w[1]), w[2]), w[3]), w[4]), w[5]);
    return gs_div(rn_sub(s, b), d);
}

// the residual b + d x - s of one cell (s = sum of couplings times
// neighbour values, d = sum of couplings), rounded step by step in a fixed
// order, so the level-0 residual kernels give the same bits on natural and
// parity-split rows
__device__ __forceinline__ double res_value(const double w[6], const double xn[6], double xc, double b) {
    double s = rn_mul(w[0], xn[0]);
    s = rn_fma(w[1], xn[1], s);
    s = rn_fma(w[2], xn[2], s);
    s = rn_fma(w[3], xn[3], s);
    s = rn_fma(w[4], xn[4], s);
    s = rn_fma(w[5], xn[5], s);
    const double d = rn_add(rn_add(rn_add(rn_add(rn_add(w[0], w[1]), w[2]), w[3]), w[4]), w[5]);
    return rn_sub(rn_fma(d, xc, b), s);
}

// sum of couplings times neighbour values, and the sum of couplings; ckm
// and ckp are the slab indices of the k neighbours
template <typename T>
__device__ __forceinline__ void stencil(const T* x, long c, long ckm, long ckp, long si, long sj, const T w[6],
                                        T& s, T& d) {
    s = w[0] * x[c - si] + w[1] * x[c + si] + w[2] * x[c - sj] + w[3] * x[c + sj] +
        w[4] * x[ckm] + w[5] * x[ckp];
    d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
}

// Wall faces of cell (i,j,k) on level 0 (FP64).  values == false: the sum
// over its Dirichlet faces of the face coupling (the eliminated 2 A_f / V,
// times the face lambda), the cell's row sum up to sign.  values == true:
// the right-hand-side term of the face values, sum over Dirichlet faces of
// 2 A_f g / V (DirichletBoundaryCondition.C:47-48) plus, over Neumann faces
// with a gradient g, A_f g / (delta V) = lambda g / h
// (NeumannBoundaryCondition.C:44-50).
__device__ __forceinline__ double wall_sum(const LevelView<double>& L, const Walls& W, int b, int i, int j, int k,
                                           long c, long ckp, bool values) {
    double s = 0.0;
    const int at[6] = {i == 0, i == L.n0 - 1, j == 0, j == L.n1 - 1, k == 0, k == L.n2 - 1};
    const int q[3] = {i, j, k};
    const long st[3] = {L.si, L.sj, 1};
    const int faces = values ? (W.mask[b] | W.nmask[b]) : W.mask[b];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
        if (!((faces >> f) & 1) || !at[f]) continue;
        const int d = f >> 1, up = f & 1;
        const bool dir = (W.mask[b] >> f) & 1;
        double w = dir ? L.tab64[(up ? L.to.wh[d] : L.to.wl[d]) + q[d]] : 1.0 / L.tab64[L.to.h[d] + q[d]];
        const double* lam = d == 0 ? L.lam0 : d == 1 ? L.lam1 : L.lam2;
        if (lam) w *= lam[!up ? c : d == 2 ? ckp : c + st[d]];
        s += values ? w * W.g[b][f] : w;
    }
    return s;
}

// whether any cell of the k-quad (i, j, k0 .. k0+3) has a periodic ghost
// image (k0 % 4 == 0, n2 % 4 == 0): a cheap test that spares the other
// quads store_images' per-cell offset arithmetic
template <typename T>
__device__ __forceinline__ bool quad_has_images(const LevelView<T>& L, int i, int j, int k0) {
    return (L.per0 && (i == 0 || i == L.n0 - 1)) || (L.per1 && (j == 0 || j == L.n1 - 1)) ||
           (L.per2 && (k0 == 0 || k0 + 4 >= L.n2));
}

// slab index of cell (i,j,k) in 32-bit arithmetic (the host rejects levels
// of 2^31 cells or more); k is logical, its storage position comes from kpos
template <typename T>
__device__ __forceinline__ int cell32(const LevelView<T>& L, int i, int j, int k) {
    return (int)L.base + i * (int)L.si + j * (int)L.sj + kpos(L, k);
}

// slab index of the first (logical k = 0) position of row (i, j)
template <typename T>
__device__ __forceinline__ long row_at(const LevelView<T>& L, int i, int j) {
    return L.base + (long)i * L.si + (long)j * L.sj;
}

// Position, relative to the quad's first cell, of cell e (0..3) of the
// logical k-quad k0 .. k0+3 (k0 % 4 == 0): consecutive in natural rows
// (kh = 0); in a parity-split row the even pair sits at kpos(k0),
// kpos(k0)+1 and the odd pair kh further on.
__device__ __forceinline__ int quad_off(int kh, int e) { return kh ? (e & 1) * kh + (e >> 1) : e; }

// index of cell (i,j,k) in the caller's (compact, brick-frame) arrays
template <typename T>
__device__ __forceinline__ long compact_index(const LevelView<T>& L, int i, int j, int k) {
    return L.cbase + (long)i * L.cs[0] + (long)j * L.cs[1] + (long)k * L.cs[2];
}

// Store an interior value and its periodic ghost images (faces, edges and
// corners), replacing the reference's per-sweep periodic ghost copy
// (periodicBoundaryCondition.C:53-92).  Per axis a cell has up to two
// images: in the upper ghost layer (cell 0) and in the lower one (cell
// n-1); both when n == 1.  All combinations are unrolled into predicated
// stores, so nothing lives in local memory.
template <typename T>
__device__ __forceinline__ void store_images(const LevelView<T>& L, long c, int i, int j, int k, T v);
template <typename T, typename U>
__device__ __forceinline__ void store_images_to(const LevelView<T>& L, U* x, long c, int i, int j, int k, U v);

template <typename T>
__device__ __forceinline__ void store_x(const LevelView<T>& L, long c, int i, int j, int k, T v) {
    L.x[c] = v;
    store_images(L, c, i, j, k, v);
}

// the periodic ghost images alone, for kernels that store the interior
// value themselves (as part of a vector store)
template <typename T>
__device__ __forceinline__ void store_images(const LevelView<T>& L, long c, int i, int j, int k, T v) {
    store_images_to(L, L.x, c, i, j, k, v);
}

// the same images of a value of another array with L's geometry
template <typename T, typename U>
__device__ __forceinline__ void store_images_to(const LevelView<T>& L, U* x, long c, int i, int j, int k, U v) {
    const long up0 = (L.per0 && i == 0) ? (long)L.n0 * L.si : 0;
    const long dn0 = (L.per0 && i == L.n0 - 1) ? -(long)L.n0 * L.si : 0;
    const long up1 = (L.per1 && j == 0) ? (long)L.n1 * L.sj : 0;
    const long dn1 = (L.per1 && j == L.n1 - 1) ? -(long)L.n1 * L.sj : 0;
    const long up2 = (L.per2 && k == 0) ? (long)L.n2 : 0;
    const long dn2 = (L.per2 && k == L.n2 - 1) ? -(long)L.n2 : 0;
    if (!(up0 | dn0 | up1 | dn1 | up2 | dn2)) return;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const long o0 = a == 0 ? 0 : a == 1 ? up0 : dn0;
        if (a && !o0) continue;
#pragma unroll
        for (int e = 0; e < 3; ++e) {
            const long o1 = e == 0 ? 0 : e == 1 ? up1 : dn1;
            if (e && !o1) continue;
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                const long o2 = f == 0 ? 0 : f == 1 ? up2 : dn2;
                if (f && !o2) continue;
                if (a | e | f) x[c + o0 + o1 + o2] = v;
            }
        }
    }
}

}  // namespace bmg
