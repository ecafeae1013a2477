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

// Row-scaled couplings of cell (i,j,k) to its six neighbours in the order
// of the reference's row product: l, r, b, t, a, f (linearSystemFunctions.H
// :96-102), i.e. axis 0 lower/upper, axis 1 lower/upper, axis 2 lower/upper.
template <typename T, bool VAR>
__device__ __forceinline__ void couplings(const LevelView<T>& L, int i, int j, int k, long c,
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
        w[5] *= ldg(L.lam2 + c + 1);
    }
}

// Gauss-Seidel value of a cell from its couplings w, neighbour values xn
// (same order) and right-hand side b: (sum w*xn - b) / sum w, which is
// (b - offdiag row product) / centre of rbgsSmoother.C:76-81 for the
// row-scaled operator.
// The FP32 smoother divides with the hardware reciprocal (about 2 ulp, two
// instructions); the FP64 path keeps IEEE division.  Both smoother kernels
// call this one function, so they stay bit-identical to each other.
__device__ __forceinline__ float gs_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double gs_div(double a, double b) { return a / b; }

template <typename T>
__device__ __forceinline__ T gs_value(const T w[6], const T xn[6], T b) {
    const T s = w[0] * xn[0] + w[1] * xn[1] + w[2] * xn[2] + w[3] * xn[3] + w[4] * xn[4] + w[5] * xn[5];
    const T d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
    return gs_div(s - b, d);
}

// sum of couplings times neighbour values, and the sum of couplings
template <typename T>
__device__ __forceinline__ void stencil(const T* x, long c, long si, long sj, const T w[6], T& s,
                                        T& d) {
    s = w[0] * x[c - si] + w[1] * x[c + si] + w[2] * x[c - sj] + w[3] * x[c + sj] +
        w[4] * x[c - 1] + w[5] * x[c + 1];
    d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
}

// Store an interior value and its periodic ghost images (faces, edges and
// corners), replacing the reference's per-sweep periodic ghost copy
// (periodicBoundaryCondition.C:53-92).  Per axis a cell has up to two
// images: in the upper ghost layer (cell 0) and in the lower one (cell
// n-1); both when n == 1.  All combinations are unrolled into predicated
// stores, so nothing lives in local memory.
template <typename T>
__device__ __forceinline__ void store_x(const LevelView<T>& L, long c, int i, int j, int k, T v) {
    L.x[c] = v;
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
                if (a | e | f) L.x[c + o0 + o1 + o2] = v;
            }
        }
    }
}

}  // namespace bmg
