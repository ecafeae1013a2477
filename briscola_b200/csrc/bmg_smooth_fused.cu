// bmg_smooth_fused.cu -- several red-black colour passes in one pass over
// memory (temporal blocking of red-black Gauss-Seidel), software-pipelined.
//
// A smoothing step of the reference is a sequence of red-black colour
// passes (rbgsSmoother.C:65-183; after dropping back-to-back repeats the
// colours alternate, e.g. 0,1,0,1,0 for two sweeps on an even brick).  Done
// pass by pass, every pass streams x and b through HBM.  Here one CTA owns
// a tile of KR x 4*kQ cells across (j, k) and a chunk of planes along i,
// and runs S consecutive passes as a wavefront: at each plane step one new
// plane enters and stage s updates the plane s steps behind it.  Per cell x
// and b are read once and x written once for all S passes.
//
// Each thread owns the k-quad of one row (four cells) through every plane
// and keeps it in registers split by colour: two cells of colour 0 and two
// of colour 1, with the i neighbours (planes entering .. S+1 behind) in a
// register window.  A colour-c cell's six neighbours all have colour 1-c,
// and its i and j neighbours sit at the same k, so in colour-split form
// they are the same element of the neighbouring quad: no per-cell parity
// selects.  Only the in-plane neighbours that other threads own go through
// shared memory, and a stage only reads the colour the previous stage
// wrote, so each buffer holds half a plane: the colour-(1-c1) half of the
// entering plane, and the output half of stages 1..S-1, each double-
// buffered by step parity, so one barrier per step both publishes the
// previous step's halves and retires the ones this step overwrites.
//
// Correctness of the wavefront: stage s at plane p needs plane p+1 at stage
// s-1 (computed earlier in the same step, same thread), plane p at stage s-1
// (previous step) and plane p-1 at stage s-1; plane p-1 is already at stage
// s, but a stage only changes cells of its own colour and the (p-1)
// neighbour of a colour-c cell has the other colour, so the value read is
// its stage s-1 value.  Periodic extents are even (the host checks), so a
// wrapped neighbour has the other colour too and raw indices give the
// colour parity.
//
// Tiles recompute a halo of S rows in j, one quad in k and S planes at chunk
// ends, valid one cell less per stage; only the tile proper is written,
// into a second buffer (ping-pong), so neighbouring CTAs always read the
// input.  Planes arrive by cp.async KP steps ahead into shared-memory
// landing slots; when a plane enters, its b quad is split by colour into a
// colour-major ring that its S stages read.  The step loop is
// unrolled by U (even), so register-window slots, ring slots and buffer
// parities are compile-time.  The
// arithmetic is gs_value() of bmg_stencil.cuh with the same coupling and
// neighbour order as the colour-pass kernels: results are bit-identical to
// S separate colour passes.

#include <algorithm>

#include "bmg_stencil.cuh"

namespace bmg {

namespace {

constexpr int kQ = 16;  // quads per tile row (64 cells)

template <typename T, int S, int KR>
struct SweepShape {
    static constexpr int EQ = kQ + 2;         // quads incl. one halo quad each side
    static constexpr int EA = KR + 2 * S;     // rows incl. S halo rows each side
    static constexpr int NT = EA * EQ;        // threads, one quad each
    static constexpr int RH = 2 * EQ;         // half row: 2 cells per quad
    static constexpr int PH = (EA + 2) * RH;  // half plane: a guard row each side
    static constexpr int QP = NT * 4;         // natural quads of one plane
    static constexpr int U = 8;               // step unroll
    static constexpr int KP = 3;              // planes loaded ahead (cp.async groups in flight)
    static constexpr int NX = KP + 1;         // landing slots of x and b
    static constexpr int NB = 4;              // colour-split b slots
    static_assert(U % NX == 0 && U % NB == 0 && S + 1 <= NB && S + 2 <= U, "ring sizes");
    static constexpr int WMAX = 128 + 2 * S;  // planes of a chunk (at most 128) with halos
    static constexpr size_t elems = (size_t)(2 * S) * PH + (size_t)(2 * NX + NB) * QP + 2 * WMAX;
    static constexpr size_t smem = sizeof(T) * elems;
    static constexpr int threads = NT;
    static constexpr int min_ctas = sizeof(T) == 8 ? 1 : KR > 8 ? 2 : 3;
};

template <typename T>
struct Vec;
template <>
struct Vec<float> {
    static __device__ __forceinline__ void ld4s(const float* p, float v[4]) {
        const float4 a = *reinterpret_cast<const float4*>(p);
        v[0] = a.x;
        v[1] = a.y;
        v[2] = a.z;
        v[3] = a.w;
    }
    static __device__ __forceinline__ void st4(float* p, float a, float b, float c, float d) {
        *reinterpret_cast<float4*>(p) = make_float4(a, b, c, d);
    }
    static __device__ __forceinline__ void ld2(const float* p, float v[2]) {
        const float2 a = *reinterpret_cast<const float2*>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
    static __device__ __forceinline__ void st2(float* p, const float v[2]) {
        *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    }
};
template <>
struct Vec<double> {
    static __device__ __forceinline__ void ld4s(const double* p, double v[4]) {
        const double2 a = reinterpret_cast<const double2*>(p)[0];
        const double2 b = reinterpret_cast<const double2*>(p)[1];
        v[0] = a.x;
        v[1] = a.y;
        v[2] = b.x;
        v[3] = b.y;
    }
    static __device__ __forceinline__ void st4(double* p, double a, double b, double c, double d) {
        reinterpret_cast<double2*>(p)[0] = make_double2(a, b);
        reinterpret_cast<double2*>(p)[1] = make_double2(c, d);
    }
    static __device__ __forceinline__ void ld2(const double* p, double v[2]) {
        const double2 a = *reinterpret_cast<const double2*>(p);
        v[0] = a.x;
        v[1] = a.y;
    }
    static __device__ __forceinline__ void st2(double* p, const double v[2]) {
        *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
    }
};

__device__ __forceinline__ int wrapa(int r, int n, int periodic, bool& valid) {
    valid = (r >= 0 && r < n) || periodic != 0;
    return ((r % n) + n) % n;
}

// plane index along i -> (index, valid) with one periodic wrap at most
__device__ __forceinline__ int wrapm(int r, int n, int periodic, bool& valid) {
    valid = (r >= 0 && r < n);
    if (!valid && periodic) {
        valid = true;
        return r < 0 ? r + n : r - n;
    }
    return valid ? r : 0;
}

// 16-byte cp.async, zero-filled (and nothing read) when !valid
__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// a quad of T values: 16 bytes (FP32) or 2 x 16 bytes (FP64)
template <typename T>
__device__ __forceinline__ void cp_quad(T* smem, const T* gmem, bool valid) {
    cp16(smem, gmem, valid);
    if constexpr (sizeof(T) == 8) cp16(smem + 2, gmem + 2, valid);
}

template <typename T, bool VAR, int S, int KR, int C1>
__global__ void __launch_bounds__(SweepShape<T, S, KR>::threads, SweepShape<T, S, KR>::min_ctas)
    k_sweep(LevelView<T> L, T* __restrict__ xout, FusedGeom g) {
    grid_dep_sync();
    using F = SweepShape<T, S, KR>;
    constexpr int EQ = F::EQ, NT = F::NT, RH = F::RH, PH = F::PH, QP = F::QP, U = F::U, KP = F::KP,
                  NX = F::NX, NB = F::NB;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // half planes: buffer (stage s in 0..S-1, parity p) at (2s + p) * PH;
    // stage 0 is the entering plane's colour-(1-C1) half.  A half row is
    // the threads' pairs back to back, so a warp's pairs are contiguous.
    T* const sh = reinterpret_cast<T*>(smem_raw);
    T* const rx = sh + 2 * S * PH;  // [NX][QP] landing natural quads of x, plane t in slot t % NX
    T* const rb = rx + NX * QP;     // [NX][QP] landing natural quads of b
    T* const cb = rb + NX * QP;     // [NB][2 colours][NT][2] colour-split b, plane t in slot t % NB
    T* const wm = cb + NB * QP;     // [2][WMAX] couplings of the chunk's planes along i

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int a_raw = blockIdx.y * KR - S + ty;
    const int q_raw = blockIdx.x * kQ - 1 + tx;
    const int k0_raw = 4 * q_raw;
    const int m0 = blockIdx.z * g.ti;
    const int mcount = min(g.ti, g.nm - m0);
    const int steps = mcount + 2 * S;

    bool va, vk;
    const int a = wrapa(a_raw, g.na, g.pera, va);
    const int k0 = 4 * wrapa(q_raw, g.nk / 4, g.perk, vk);
    const bool vq = va && vk;

    const T* tab = L.tab;
    const T wal = va ? ldg(tab + g.wl_a + a) : T(0), wah = va ? ldg(tab + g.wh_a + a) : T(0);
    // cell indices of a level fit 32 bits (the host only fuses such levels)
    const int rowa = (int)(L.base + (long)a * g.sa);
    const int sm = (int)g.sm;

    // Colour of (P, a, k) is (P + a + k + cpar) & 1 and k0 is even, so the
    // colour-0 cells of the quad at plane P sit at q = lo, lo + 2 with
    // lo = (P + a + cpar) & 1.  At unrolled step u (chunks start at even
    // steps) the entering plane Lp has lo = lpar ^ (u & 1), and every stage
    // of the step updates the cells at q = o, o + 2 with o = opar ^ (u & 1):
    // stage s works on plane Lp - s in colour C1 ^ ((s-1) & 1), and the two
    // parities cancel.
    const int rowpar = (a_raw + L.cpar) & 1;
    const int lpar = (m0 - S + rowpar) & 1;
    const int opar = (m0 - S + rowpar + C1 + 1) & 1;
    T wkL[2][2], wkH[2][2];  // by step parity: k couplings of the two updated cells
    int ext[2];              // by step parity: offset of the neighbour another thread owns
    bool oo[2], lo[2], so[2];
#pragma unroll
    for (int p = 0; p < 2; ++p) {
        oo[p] = (opar ^ p) != 0;
        lo[p] = (lpar ^ p) != 0;
        so[p] = (lpar ^ p ^ (S & 1)) != 0;  // plane Lp - S (the one written)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const int q = 2 * i + (oo[p] ? 1 : 0);
            wkL[p][i] = vk ? ldg(tab + L.to.wl[2] + k0 + q) : T(0);
            wkH[p][i] = vk ? ldg(tab + L.to.wh[2] + k0 + q) : T(0);
        }
        ext[p] = oo[p] ? 2 : -1;
    }

    const int tid = ty * EQ + tx;
    // own pair in a half plane; the pairs either side of the tile row are
    // the neighbouring rows' (or a guard row's) and only reach halo cells
    const int me = RH + 2 * tid;
    const int mq = tid * 4;  // own quad in a landing slot

    // guard rows stay zero for good; the couplings of the chunk's planes
    for (int q = tid; q < 2 * S * PH; q += F::threads) sh[q] = T(0);
    for (int q = tid; q < steps; q += F::threads) {
        bool vm;
        const int mp = wrapm(m0 - S + q, g.nm, g.perm, vm);
        wm[q] = vm ? ldg(tab + g.wl_m + mp) : T(0);
        wm[F::WMAX + q] = vm ? ldg(tab + g.wh_m + mp) : T(0);
    }

    // queue plane tt (one cp.async group per step, empty past the end, so
    // that group counting stays uniform)
    auto issue = [&](int tt, int xslot) {
        if (tt < steps) {
            bool vm;
            const int mp = wrapm(m0 - S + tt, g.nm, g.perm, vm);
            const bool v = vm && vq;
            const int r = rowa + mp * sm + k0;
            cp_quad<T>(rx + xslot * QP + mq, v ? L.x + r : L.x, v);
            cp_quad<T>(rb + xslot * QP + mq, v ? L.b + r : L.b, v);
        }
        cp_commit();
    };
#pragma unroll
    for (int tt = 0; tt < KP; ++tt) issue(tt, tt % NX);

    // register window by plane slot (t % U): [colour][cell] of x
    T X[U][2][2];
#pragma unroll
    for (int p = 0; p < U; ++p)
#pragma unroll
        for (int c = 0; c < 2; ++c) X[p][c][0] = X[p][c][1] = T(0);

    const bool outRow = ty >= S && ty < S + KR && a_raw < g.na;
    const bool outCol = tx >= 1 && tx < 1 + kQ && k0_raw < g.nk;
    LevelView<T> O = L;
    O.x = xout;
    const bool images = L.per0 | L.per1 | L.per2;

    for (int t0 = 0; t0 < steps; t0 += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int t = t0 + u;
            if (t >= steps) break;  // uniform across the CTA
            const int Lp = m0 - S + t;
            cp_wait<KP - 1>();  // this thread's copies of plane t have landed
            // Publishes the halves written in step t-1 (and, at t = 0, the
            // couplings and zeroed guards) and orders every read of the
            // halves and ring slots this step overwrites (all made in step
            // t-1 or earlier).
            __syncthreads();
            issue(t + KP, (u + KP) % NX);

            // the entering plane: split its quads by colour
            {
                T q[4], r[4];
                Vec<T>::ld4s(rx + (u % NX) * QP + mq, q);
                Vec<T>::ld4s(rb + (u % NX) * QP + mq, r);
                const bool l = lo[u & 1];
                T(&x)[2][2] = X[u];
                x[0][0] = l ? q[1] : q[0];
                x[0][1] = l ? q[3] : q[2];
                x[1][0] = l ? q[0] : q[1];
                x[1][1] = l ? q[2] : q[3];
                Vec<T>::st2(sh + (u & 1) * PH + me, x[1 - C1]);
                const T b0[2] = {l ? r[1] : r[0], l ? r[3] : r[2]};
                const T b1[2] = {l ? r[0] : r[1], l ? r[2] : r[3]};
                T* const c = cb + (u % NB) * QP + 2 * tid;
                Vec<T>::st2(c, b0);
                Vec<T>::st2(c + 2 * NT, b1);
            }

#pragma unroll
            for (int s = 1; s <= S; ++s) {
                const int C = C1 ^ ((s - 1) & 1);  // colour of this stage
                const int P = Lp - s;
                const int sp = (u - s + 2 * U) % U;      // plane P
                const int sM = (u - s - 1 + 2 * U) % U;  // plane P - 1
                const int sP = (u - s + 1 + 2 * U) % U;  // plane P + 1
                const bool inP = (P >= 0 && P < g.nm) || g.perm;
                // t < s: plane P lies below the loaded planes (nothing to do)
                if (t >= s && inP && vq) {
                    // plane P after stage s-1, written in step t-1
                    const T* Bs = sh + (2 * (s - 1) + ((u + 1) & 1)) * PH;
                    T ym[2], yp[2];
                    Vec<T>::ld2(Bs + me - RH, ym);
                    Vec<T>::ld2(Bs + me + RH, yp);
                    const T e = Bs[me + ext[u & 1]];
                    const bool o = oo[u & 1];
                    T bb[2];
                    Vec<T>::ld2(cb + ((u - s + 2 * NB) % NB) * QP + C * 2 * NT + 2 * tid, bb);
                    const T* Y = X[sp][1 - C];  // own row, other colour
                    const T l0 = o ? Y[0] : e;
                    const T r0 = o ? Y[1] : Y[0];
                    const T r1 = o ? e : Y[1];
                    const T wml = wm[t - s], wmh = wm[F::WMAX + t - s];
                    T w0[6] = {wml, wmh, wal, wah, wkL[u & 1][0], wkH[u & 1][0]};
                    T w1[6] = {wml, wmh, wal, wah, wkL[u & 1][1], wkH[u & 1][1]};
                    if (VAR) {
                        bool vP;
                        const int mP = wrapm(P, g.nm, g.perm, vP);
                        // the updated cells are k0 + o and k0 + o + 2
                        const long c = (long)rowa + (long)mP * sm + k0 + (o ? 1 : 0);
                        w0[0] *= ldg(L.lam0 + c);
                        w0[1] *= ldg(L.lam0 + c + L.si);
                        w0[2] *= ldg(L.lam1 + c);
                        w0[3] *= ldg(L.lam1 + c + L.sj);
                        w0[4] *= ldg(L.lam2 + c);
                        w0[5] *= ldg(L.lam2 + c + 1);
                        w1[0] *= ldg(L.lam0 + c + 2);
                        w1[1] *= ldg(L.lam0 + c + 2 + L.si);
                        w1[2] *= ldg(L.lam1 + c + 2);
                        w1[3] *= ldg(L.lam1 + c + 2 + L.sj);
                        w1[4] *= ldg(L.lam2 + c + 2);
                        w1[5] *= ldg(L.lam2 + c + 3);
                    }
                    const T xn0[6] = {X[sM][1 - C][0], X[sP][1 - C][0], ym[0], yp[0], l0, r0};
                    const T xn1[6] = {X[sM][1 - C][1], X[sP][1 - C][1], ym[1], yp[1], r0, r1};
                    X[sp][C][0] = gs_value(w0, xn0, bb[0]);
                    X[sp][C][1] = gs_value(w1, xn1, bb[1]);
                }
                if (s < S) {
                    Vec<T>::st2(sh + (2 * s + (u & 1)) * PH + me, X[sp][C]);
                } else if (outRow && outCol && P >= m0 && P < m0 + mcount) {
                    const bool l = so[u & 1];
                    const T q0 = l ? X[sp][1][0] : X[sp][0][0];
                    const T q1 = l ? X[sp][0][0] : X[sp][1][0];
                    const T q2 = l ? X[sp][1][1] : X[sp][0][1];
                    const T q3 = l ? X[sp][0][1] : X[sp][1][1];
                    const long c = (long)rowa + (long)P * sm + k0_raw;
                    Vec<T>::st4(xout + c, q0, q1, q2, q3);
                    if (images && quad_has_images(O, P, a, k0_raw)) {
                        store_images(O, c, P, a, k0_raw, q0);
                        store_images(O, c + 1, P, a, k0_raw + 1, q1);
                        store_images(O, c + 2, P, a, k0_raw + 2, q2);
                        store_images(O, c + 3, P, a, k0_raw + 3, q3);
                    }
                }
            }
        }
    }
    cp_wait<0>();  // no copy outlives the CTA
}

// rows per tile: FP32 tiles of 12 (three stages) or 16 rows (two), two
// CTAs per SM, cut the j-halo overhead of 8-row tiles; FP64 keeps 8 rows
// (registers)
template <typename T, int S>
constexpr int tile_rows() {
    return sizeof(T) == 8 || S == 1 ? 8 : S == 3 ? 12 : 16;
}

template <typename T, bool VAR, int S, int C1>
void configure_one() {
    constexpr int KR = tile_rows<T, S>();
    cudaFuncSetAttribute(k_sweep<T, VAR, S, KR, C1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)SweepShape<T, S, KR>::smem);
}

template <typename T, bool VAR, int S>
void launch_one(const LevelView<T>& L, T* xout, const FusedGeom& g, int c1, cudaStream_t s) {
    constexpr int KR = tile_rows<T, S>();
    using F = SweepShape<T, S, KR>;
    // the couplings of a chunk's planes are staged for at most 128 planes
    FusedGeom gg = g;
    gg.ti = std::min(g.ti, 128);
    const dim3 grid((g.nk + 4 * kQ - 1) / (4 * kQ), (g.na + KR - 1) / KR, (gg.nm + gg.ti - 1) / gg.ti);
    const dim3 blk(F::EQ, F::EA, 1);
    if (c1)
        launch_k(k_sweep<T, VAR, S, KR, 1>, grid, blk, F::smem, s, L, xout, gg);
    else
        launch_k(k_sweep<T, VAR, S, KR, 0>, grid, blk, F::smem, s, L, xout, gg);
}

template <typename T, bool VAR>
void configure_type() {
    configure_one<T, VAR, 1, 0>();
    configure_one<T, VAR, 1, 1>();
    configure_one<T, VAR, 2, 0>();
    configure_one<T, VAR, 2, 1>();
    configure_one<T, VAR, 3, 0>();
    configure_one<T, VAR, 3, 1>();
}

}  // namespace

void configure_fused_kernels() {
    configure_type<float, false>();
    configure_type<float, true>();
    configure_type<double, false>();
    configure_type<double, true>();
}

template <typename T, bool VAR>
void launch_smooth_fused(const LevelView<T>& L, T* xout, const FusedGeom& g, int c1, int stages,
                         cudaStream_t s) {
    switch (stages) {
        case 1: launch_one<T, VAR, 1>(L, xout, g, c1, s); break;
        case 2: launch_one<T, VAR, 2>(L, xout, g, c1, s); break;
        default: launch_one<T, VAR, 3>(L, xout, g, c1, s); break;
    }
}

template void launch_smooth_fused<float, false>(const LevelView<float>&, float*, const FusedGeom&, int, int,
                                                cudaStream_t);
template void launch_smooth_fused<float, true>(const LevelView<float>&, float*, const FusedGeom&, int, int,
                                               cudaStream_t);
template void launch_smooth_fused<double, false>(const LevelView<double>&, double*, const FusedGeom&, int, int,
                                                 cudaStream_t);
template void launch_smooth_fused<double, true>(const LevelView<double>&, double*, const FusedGeom&, int, int,
                                                cudaStream_t);

}  // namespace bmg
