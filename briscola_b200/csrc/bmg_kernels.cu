// bmg_kernels.cu -- sm_100a kernels of the multigrid V-cycle.
//
// Every kernel here is HBM- (fine levels) or L2-bound (levels up to 128^3
// fit the 126 MB L2): no tensor cores, coalesced k-fastest access, FP64 or
// FP32 arithmetic chosen by the template parameter.  Layout and coefficient
// conventions are described in bmg_internal.h.

#include "bmg_internal.h"

#include <cmath>

namespace bmg {

namespace {

template <typename T>
__device__ __forceinline__ T ldg(const T* p) {
    return __ldg(p);
}

// Row-scaled couplings of cell (i,j,k) to its six neighbours, in the order
// of the reference's row product: l, r, b, t, a, f (linearSystemFunctions.H
// :96-102).
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

// sum of couplings times neighbour values, and the sum of couplings
// (= minus the centre coefficient)
template <typename T>
__device__ __forceinline__ void stencil(const T* x, long c, long si, long sj, const T w[6], T& s,
                                        T& d) {
    s = w[0] * x[c - si] + w[1] * x[c + si] + w[2] * x[c - sj] + w[3] * x[c + sj] +
        w[4] * x[c - 1] + w[5] * x[c + 1];
    d = w[0] + w[1] + w[2] + w[3] + w[4] + w[5];
}

// Store an interior value and its periodic ghost images (faces, edges and
// corners), replacing the reference's per-sweep periodic ghost copy
// (periodicBoundaryCondition.C:53-92).
// Per axis a cell has up to two images: in the upper ghost layer (cell 0)
// and in the lower one (cell n-1); both when n == 1.  All 26 combinations
// are unrolled into predicated stores, so nothing lives in local memory.
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

// ---------------------------------------------------------------------------
// Red-black Gauss-Seidel: one colour pass.  Thread per (i, j, k-pair); the
// pair member of the requested colour is updated.  Colour 0 = (i+j+k) even.
// Equivalent to one pass of rbgsSmoother.C:65-183 over the whole level.
// ---------------------------------------------------------------------------
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_colour_pass(LevelView<T> L, int colour) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1) return;
    const int k = 2 * m + ((colour + i + j) & 1);
    if (k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    T w[6], s, d;
    couplings<T, VAR>(L, i, j, k, c, w);
    stencil(L.x, c, L.si, L.sj, w, s, d);
    const T v = (s - L.b[c]) / d;
    store_x(L, c, i, j, k, v);
}

// Damped Jacobi (omega = 0.8, jacSmoother.C:15) into a temporary, then copy.
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_jacobi(LevelView<T> L, T* tmp) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    T w[6], s, d;
    couplings<T, VAR>(L, i, j, k, c, w);
    stencil(L.x, c, L.si, L.sj, w, s, d);
    const T omega = T(0.8);
    tmp[c] = (T(1) - omega) * L.x[c] + omega * (s - L.b[c]) / d;
}

template <typename T>
__global__ void __launch_bounds__(256) k_copy_interior(LevelView<T> L, const T* src) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
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
__global__ void __launch_bounds__(256) k_residual_restrict(LevelView<T> F, LevelView<T> C,
                                                           const T* ratio, int R0, int R1,
                                                           int R2) {
    const int K = blockIdx.x * blockDim.x + threadIdx.x;
    const int J = blockIdx.y * blockDim.y + threadIdx.y;
    const int I = blockIdx.z;
    if (J >= C.n1 || K >= C.n2) return;
    T acc = T(0);
    for (int a = 0; a < R0; ++a) {
        const int i = I * R0 + a;
        const T ra = ldg(ratio + i);
        for (int bb = 0; bb < R1; ++bb) {
            const int j = J * R1 + bb;
            const T rab = ra * ldg(ratio + F.n0 + j);
            for (int e = 0; e < R2; ++e) {
                const int k = K * R2 + e;
                const long c = F.base + (long)i * F.si + (long)j * F.sj + k;
                T w[6], s, d;
                couplings<T, VAR>(F, i, j, k, c, w);
                stencil(F.x, c, F.si, F.sj, w, s, d);
                const T r = F.b[c] + d * F.x[c] - s;
                acc += rab * ldg(ratio + F.n0 + F.n1 + k) * r;
            }
        }
    }
    const long cc = C.base + (long)I * C.si + (long)J * C.sj + K;
    C.b[cc] = acc;
}

// ---------------------------------------------------------------------------
// Fused prolongation + correction: x_f += trilinear interpolation of the
// coarse correction (linearProlongationScheme.C:12-147).  Per fine index the
// host tables give the two coarse indices (own parent and the neighbour on
// the fine cell's side, wrapped on periodic axes) and the neighbour's weight;
// at walls the weight is zero, which equals the reference's use of a
// zero-gradient ghost there.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_prolong_correct(LevelView<T> F, LevelView<T> C,
                                                         const int* pidx, const T* pw) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= F.n1 || k >= F.n2) return;
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
    const T v00 = uk * X[r00 + K0] + wk * X[r00 + K1];
    const T v01 = uk * X[r01 + K0] + wk * X[r01 + K1];
    const T v10 = uk * X[r10 + K0] + wk * X[r10 + K1];
    const T v11 = uk * X[r11 + K0] + wk * X[r11 + K1];
    const T v = ui * (uj * v00 + wj * v01) + wi * (uj * v10 + wj * v11);
    const long c = F.base + (long)i * F.si + (long)j * F.sj + k;
    store_x(F, c, i, j, k, F.x[c] + v);
}

// ---------------------------------------------------------------------------
// Coarse direct solve: x = inverse(A'_pinned) b' with b'(0) = 0 (MG.C:37-40,
// solver.C:201-231, APLU.C:91-128).  One CTA; the inverse is factored once
// per matrix on the host in FP64.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_coarse_solve(LevelView<T> C, const double* __restrict__ ainv,
                                                      int n) {
    extern __shared__ double sb[];
    const int nn = C.n1 * C.n2;
    for (int q = threadIdx.x; q < n; q += blockDim.x) {
        const int i = q / nn, j = (q / C.n2) % C.n1, k = q % C.n2;
        sb[q] = q == 0 ? 0.0 : (double)C.b[C.base + (long)i * C.si + (long)j * C.sj + k];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int r = warp; r < n; r += nw) {
        double s = 0.0;
        for (int l = lane; l < n; l += 32) s += ainv[(long)r * n + l] * sb[l];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const int i = r / nn, j = (r / C.n2) % C.n1, k = r % C.n2;
            store_x(C, C.base + (long)i * C.si + (long)j * C.sj + k, i, j, k, (T)s);
        }
    }
}

// residual r = b - A x of any level, unscaled, into a compact array
template <typename T, bool VAR>
__global__ void __launch_bounds__(256) k_residual_out(LevelView<T> L, double* out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    T w[6], s, d;
    couplings<T, VAR>(L, i, j, k, c, w);
    stencil(L.x, c, L.si, L.sj, w, s, d);
    const double r = (double)(L.b[c] + d * L.x[c] - s);
    const double V = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
    out[((long)i * L.n1 + j) * L.n2 + k] = r * V;
}

template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) sh[warp] = v;
    __syncthreads();
    v = 0.0;
    if (warp == 0) {
        v = lane < NT / 32 ? sh[lane] : 0.0;
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    }
    return v;
}

// ---------------------------------------------------------------------------
// Level-0 residual norms in FP64 (MG.C:163-174,223-230; solver.C:13-61).
// Fixed grid and fixed reduction tree: the result does not depend on timing.
// mode 0 also accumulates the normFactor sum (|r - b| + |b|)^2, where the
// row sums of the level-0 operator vanish (all couplings are paired with the
// centre), so A*mean(x) drops out of the reference's expression.
// ---------------------------------------------------------------------------
template <bool VAR>
__global__ void __launch_bounds__(kReduceThreads) k_residual_norm(LevelView<double> L, int mode,
                                                                  double* partials, float* b32) {
    __shared__ double sh[kReduceThreads / 32];
    double a1 = 0.0, a2 = 0.0;
    const int rows = L.n0 * L.n1;
    for (int q = blockIdx.x; q < rows; q += gridDim.x) {
        const int i = q / L.n1, j = q % L.n1;
        const double hij = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j];
        for (int k = threadIdx.x; k < L.n2; k += blockDim.x) {
            const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
            double w[6], s, d;
            couplings<double, VAR>(L, i, j, k, c, w);
            stencil(L.x, c, L.si, L.sj, w, s, d);
            const double r = L.b[c] + d * L.x[c] - s;
            const double V = hij * L.tab64[L.to.h[2] + k];
            const double rr = V * r;
            a1 += rr * rr;
            if (mode == 0) {
                const double bb = V * L.b[c];
                const double t = fabs(rr - bb) + fabs(bb);
                a2 += t * t;
            }
            if (b32) b32[c] = (float)r;
        }
    }
    a1 = block_sum<kReduceThreads>(a1, sh);
    if (mode == 0) a2 = block_sum<kReduceThreads>(a2, sh);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = a1;
        if (mode == 0) partials[kReduceBlocks + blockIdx.x] = a2;
    }
}

// solver.C:13-95 on the reduced sums; also decides whether the loop goes on
// (MG.C:191-195).
__global__ void __launch_bounds__(kReduceThreads) k_finalize(const double* partials, SolveState* st,
                                                              int mode) {
    __shared__ double sh[kReduceThreads / 32];
    double a1 = 0.0, a2 = 0.0;
    for (int q = threadIdx.x; q < kReduceBlocks; q += blockDim.x) {
        a1 += partials[q];
        if (mode == 0) a2 += partials[kReduceBlocks + q];
    }
    a1 = block_sum<kReduceThreads>(a1, sh);
    if (mode == 0) a2 = block_sum<kReduceThreads>(a2, sh);
    if (threadIdx.x == 0) {
        const double l2 = sqrt(a1);
        if (mode == 0) {
            // normFactor floor: 1e-12 per cell (solver.C:53-58)
            st->nf = fmax(sqrt(a2), st->ncells * 1e-12);
            st->init = l2 / st->nf;
            st->cur = st->init;
            st->l2_0 = l2;
            st->iter = 0;
        } else {
            st->cur = l2 / st->nf;
            st->iter += 1;
        }
        st->l2 = l2;
        st->nan = !isfinite(st->cur);
        // solver.C:64-95
        st->converged = !((st->init > 0.0) && (st->cur > st->abs_tol) &&
                          (st->cur / (st->init + 1e-20) > st->rel_tol));
        st->keep_going = !st->nan && ((st->iter < st->max_iter && !st->converged) ||
                                      st->iter < st->min_iter);
    }
}

__global__ void __launch_bounds__(kReduceThreads) k_mean_partials(LevelView<double> L, double* partials) {
    __shared__ double sh[kReduceThreads / 32];
    double a = 0.0;
    const int rows = L.n0 * L.n1;
    for (int q = blockIdx.x; q < rows; q += gridDim.x) {
        const int i = q / L.n1, j = q % L.n1;
        const double hij = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j];
        for (int k = threadIdx.x; k < L.n2; k += blockDim.x) {
            const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
            a += hij * L.tab64[L.to.h[2] + k] * L.x[c];
        }
    }
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0) partials[blockIdx.x] = a;
}

__global__ void __launch_bounds__(kReduceThreads) k_mean_finalize(const double* partials, SolveState* st) {
    __shared__ double sh[kReduceThreads / 32];
    double a = 0.0;
    for (int q = threadIdx.x; q < kReduceBlocks; q += blockDim.x) a += partials[q];
    a = block_sum<kReduceThreads>(a, sh);
    if (threadIdx.x == 0) st->mean = a / st->vol_total;
}

// subtract the mean everywhere, ghosts included (a constant shift keeps the
// periodic images consistent)
__global__ void k_sub_mean(double* x, long n, const SolveState* st) {
    const double m = st->mean;
    for (long q = blockIdx.x * (long)blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        x[q] -= m;
}

__global__ void __launch_bounds__(256) k_load_b(LevelView<double> L, const double* compact) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    const double V = L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
    L.b[c] = compact[((long)i * L.n1 + j) * L.n2 + k] / V;
}

__global__ void __launch_bounds__(256) k_load_x(LevelView<double> L, const double* compact) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    store_x(L, c, i, j, k, compact[((long)i * L.n1 + j) * L.n2 + k]);
}

__global__ void __launch_bounds__(256) k_store_x(LevelView<double> L, double* compact) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    compact[((long)i * L.n1 + j) * L.n2 + k] = L.x[c];
}

template <typename T>
__global__ void __launch_bounds__(256) k_load_field(LevelView<T> L, int field, const double* compact,
                                                    int unscale) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    double v = compact[((long)i * L.n1 + j) * L.n2 + k];
    if (field == 0) {
        store_x(L, c, i, j, k, (T)v);
    } else {
        if (unscale) v /= L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
        L.b[c] = (T)v;
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_store_field(LevelView<T> L, int field, double* compact,
                                                     int unscale) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    double v = field == 0 ? (double)L.x[c] : (double)L.b[c];
    if (field == 1 && unscale)
        v *= L.tab64[L.to.h[0] + i] * L.tab64[L.to.h[1] + j] * L.tab64[L.to.h[2] + k];
    compact[((long)i * L.n1 + j) * L.n2 + k] = v;
}

__global__ void __launch_bounds__(256) k_add_correction(LevelView<double> L, const float* e) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (j >= L.n1 || k >= L.n2) return;
    const long c = L.base + (long)i * L.si + (long)j * L.sj + k;
    store_x(L, c, i, j, k, L.x[c] + (double)e[c]);
}

inline dim3 grid_cells(int n0, int n1, int n2, dim3 blk) {
    return dim3((n2 + blk.x - 1) / blk.x, (n1 + blk.y - 1) / blk.y, n0);
}

inline dim3 block_for(int n2) {
    // k extent on lanes; small rows give the spare lanes to j
    if (n2 >= 64) return dim3(64, 4, 1);
    if (n2 >= 32) return dim3(32, 8, 1);
    if (n2 >= 16) return dim3(16, 16, 1);
    return dim3(8, 32, 1);
}

}  // namespace

// ---- launchers --------------------------------------------------------------

template <typename T, bool VAR>
void launch_colour_pass(const LevelView<T>& L, int colour, cudaStream_t s) {
    const int pairs = (L.n2 + 1) / 2;
    const dim3 blk = pairs >= 32 ? dim3(32, 8, 1) : pairs >= 8 ? dim3(8, 32, 1) : dim3(2, 128, 1);
    k_colour_pass<T, VAR><<<grid_cells(L.n0, L.n1, pairs, blk), blk, 0, s>>>(L, colour);
}

template <typename T, bool VAR>
void launch_jacobi(const LevelView<T>& L, T* tmp, cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_jacobi<T, VAR><<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, tmp);
    k_copy_interior<T><<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, tmp);
}

template <typename T, bool VAR>
void launch_residual_restrict(const LevelView<T>& F, const LevelView<T>& C, const TransferTabs& t,
                              cudaStream_t s) {
    const dim3 blk = block_for(C.n2);
    const T* ratio;
    if constexpr (sizeof(T) == 8)
        ratio = reinterpret_cast<const T*>(t.ratio64);
    else
        ratio = reinterpret_cast<const T*>(t.ratio32);
    k_residual_restrict<T, VAR>
        <<<grid_cells(C.n0, C.n1, C.n2, blk), blk, 0, s>>>(F, C, ratio, t.R0, t.R1, t.R2);
}

template <typename T>
void launch_prolong_correct(const LevelView<T>& F, const LevelView<T>& C, const TransferTabs& t,
                            cudaStream_t s) {
    const dim3 blk = block_for(F.n2);
    const T* pw;
    if constexpr (sizeof(T) == 8)
        pw = reinterpret_cast<const T*>(t.pw64);
    else
        pw = reinterpret_cast<const T*>(t.pw32);
    k_prolong_correct<T><<<grid_cells(F.n0, F.n1, F.n2, blk), blk, 0, s>>>(F, C, t.pidx, pw);
}

template <typename T>
void launch_coarse_solve(const LevelView<T>& C, const double* ainv, int n, cudaStream_t s) {
    k_coarse_solve<T><<<1, 256, n * sizeof(double), s>>>(C, ainv, n);
}

template <typename T, bool VAR>
void launch_residual_out(const LevelView<T>& L, double* out, cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_residual_out<T, VAR><<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, out);
}

template <bool VAR>
void launch_residual_norm(const LevelView<double>& L, int mode, double* partials, float* b32,
                          const LevelView<float>*, cudaStream_t s) {
    k_residual_norm<VAR><<<kReduceBlocks, kReduceThreads, 0, s>>>(L, mode, partials, b32);
}

void launch_finalize(const double* partials, SolveState* st, int mode, cudaStream_t s) {
    k_finalize<<<1, kReduceThreads, 0, s>>>(partials, st, mode);
}

void launch_mean(const LevelView<double>& L, double* partials, SolveState* st, cudaStream_t s) {
    k_mean_partials<<<kReduceBlocks, kReduceThreads, 0, s>>>(L, partials);
    k_mean_finalize<<<1, kReduceThreads, 0, s>>>(partials, st);
    const long n = L.cells;
    const int blocks = (int)std::min<long>((n + 255) / 256, 148L * 16);
    k_sub_mean<<<blocks, 256, 0, s>>>(L.x, n, st);
}

void launch_load_b(const LevelView<double>& L, const double* compact, cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_load_b<<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, compact);
}

void launch_load_x(const LevelView<double>& L, const double* compact, cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_load_x<<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, compact);
}

void launch_store_x(const LevelView<double>& L, double* compact, cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_store_x<<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, compact);
}

template <typename T>
void launch_load_field(const LevelView<T>& L, int field, const double* compact, int unscale,
                       cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_load_field<T><<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, field, compact, unscale);
}

template <typename T>
void launch_store_field(const LevelView<T>& L, int field, double* compact, int unscale,
                        cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_store_field<T><<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, field, compact, unscale);
}

void launch_add_correction(const LevelView<double>& L, const LevelView<float>& E, cudaStream_t s) {
    const dim3 blk = block_for(L.n2);
    k_add_correction<<<grid_cells(L.n0, L.n1, L.n2, blk), blk, 0, s>>>(L, E.x);
}

// explicit instantiations
#define BMG_INST(T, V)                                                                          \
    template void launch_colour_pass<T, V>(const LevelView<T>&, int, cudaStream_t);             \
    template void launch_jacobi<T, V>(const LevelView<T>&, T*, cudaStream_t);                   \
    template void launch_residual_restrict<T, V>(const LevelView<T>&, const LevelView<T>&,      \
                                                 const TransferTabs&, cudaStream_t);            \
    template void launch_residual_out<T, V>(const LevelView<T>&, double*, cudaStream_t);
BMG_INST(double, false)
BMG_INST(double, true)
BMG_INST(float, false)
BMG_INST(float, true)
#undef BMG_INST
template void launch_prolong_correct<double>(const LevelView<double>&, const LevelView<double>&,
                                             const TransferTabs&, cudaStream_t);
template void launch_prolong_correct<float>(const LevelView<float>&, const LevelView<float>&,
                                            const TransferTabs&, cudaStream_t);
template void launch_coarse_solve<double>(const LevelView<double>&, const double*, int, cudaStream_t);
template void launch_coarse_solve<float>(const LevelView<float>&, const double*, int, cudaStream_t);
template void launch_residual_norm<false>(const LevelView<double>&, int, double*, float*,
                                          const LevelView<float>*, cudaStream_t);
template void launch_residual_norm<true>(const LevelView<double>&, int, double*, float*,
                                         const LevelView<float>*, cudaStream_t);
template void launch_load_field<double>(const LevelView<double>&, int, const double*, int, cudaStream_t);
template void launch_load_field<float>(const LevelView<float>&, int, const double*, int, cudaStream_t);
template void launch_store_field<double>(const LevelView<double>&, int, double*, int, cudaStream_t);
template void launch_store_field<float>(const LevelView<float>&, int, double*, int, cudaStream_t);

}  // namespace bmg
