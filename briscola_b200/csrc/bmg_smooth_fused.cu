// bmg_smooth_fused.cu -- several red-black colour passes in one pass over
// memory (temporal blocking of red-black Gauss-Seidel), software-pipelined.
//
// A smoothing step of the reference is a sequence of red-black colour
// passes (rbgsSmoother.C:65-183; after dropping back-to-back repeats the
// colours alternate, e.g. 0,1,0,1,0 for two sweeps on an even brick).  Done
// pass by pass, every pass streams x and b through HBM.  Here one CTA owns
// a tile of TA x 2*TKP cells across (j, k) and a chunk of planes along i,
// and runs S consecutive passes as a wavefront: at each plane step one new
// plane enters and stage s updates the plane s steps behind it.  Per cell x
// and b are read once and x written once for all S passes.
//
// Correctness of the wavefront: stage s at plane p needs plane p+1 at stage
// s-1 (computed earlier in the same step), plane p at stage s-1 (previous
// step) and plane p-1 at stage s-1; plane p-1 is already at stage s, but a
// stage only changes cells of its own colour and the (p-1) neighbour of a
// colour-c cell has the other colour, so the value read is its stage s-1
// value.  In-plane neighbours come from per-stage shared-memory planes,
// double-buffered by step parity.
//
// Pipelining: planes of x and b (and the i-direction couplings) stream into
// a ring of R = S + D + 1 shared-memory slots with cp.async, D steps ahead
// of use, so a step never waits on its own global loads; the one barrier per
// step both publishes the landed plane and retires the slots and stage
// buffers the step overwrites.
//
// Tiles recompute a halo of S cells (S planes at chunk ends), valid one
// cell less per stage; only the tile proper is written, into a second
// buffer (ping-pong), so neighbouring CTAs always read the input.
//
// Arithmetic is gs_value() of bmg_stencil.cuh, shared with k_colour_pass:
// results are bit-identical to S separate colour passes.

#include "bmg_stencil.cuh"

namespace bmg {

namespace {

constexpr int kPrefetch = 3;  // planes in flight ahead of the one being consumed

template <typename T>
struct Vec2;
template <>
struct Vec2<float> {
    using type = float2;
};
template <>
struct Vec2<double> {
    using type = double2;
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

// cp.async of N bytes; bytes past src_bytes are zero-filled (src_bytes = 0
// writes zeros and reads nothing)
template <int N>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int src_bytes) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(s), "l"(gmem), "n"(N), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <typename T, int S, int TA, int TKP>
struct FusedShape {
    static constexpr int HKP = (S + 1) / 2;    // k halo in pairs
    static constexpr int EKP = TKP + 2 * HKP;  // expanded tile width in pairs
    static constexpr int EK = 2 * EKP;         // ... in cells
    static constexpr int EA = TA + 2 * S;      // expanded tile height
    static constexpr int RK = EK + 4;          // padded row: 2 guard cells each side
    static constexpr int PL = (EA + 2) * RK;   // padded plane: 1 guard row each side
    static constexpr int BP = EA * EK;         // b plane (no guards)
    static constexpr int R = S + kPrefetch + 1;
    static constexpr int WM = (2 * R + 3) / 4 * 4;  // coupling slots, keeps 32-byte alignment
    static constexpr int NB = S > 1 ? S - 1 : 1;   // stage-output planes per parity
    static constexpr size_t smem = sizeof(T) * ((size_t)R * PL + (size_t)R * BP + WM + 2 * (size_t)NB * PL);
    static constexpr int threads = EKP * EA;
};

// Threads: (EKP pairs along k) x (EA rows along j).  Each thread owns the
// cell pair (k0, k0+1) of one row; in every stage exactly one of the two has
// the stage's colour, and which one depends only on the plane step.
template <typename T, bool VAR, int S, int TA, int TKP>
__global__ void __launch_bounds__(FusedShape<T, S, TA, TKP>::threads, 1)
    k_smooth_fused(LevelView<T> L, T* __restrict__ xout, FusedGeom g, int c1) {
    using F = FusedShape<T, S, TA, TKP>;
    constexpr int EKP = F::EKP, EK = F::EK, EA = F::EA, RK = F::RK, PL = F::PL, BP = F::BP, R = F::R;
    constexpr int HKP = F::HKP, D = kPrefetch;
    using V2 = typename Vec2<T>::type;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    T* xr = reinterpret_cast<T*>(smem_raw);  // [R][PL] planes of x (stage 0)
    T* br = xr + R * PL;                     // [R][BP] planes of b
    T* wr = br + R * BP;                     // [R][2] couplings along i
    T* B = wr + F::WM;                       // [2 parities][NB][PL] stage outputs

    const int tx = threadIdx.x, ty = threadIdx.y;
    const int a_raw = blockIdx.y * TA - S + ty;
    const int k0_raw = blockIdx.x * (2 * TKP) - 2 * HKP + 2 * tx;
    const int m0 = blockIdx.z * g.ti;
    const int mcount = min(g.ti, g.nm - m0);
    const int steps = mcount + 2 * S;

    bool va, vk0, vk1;
    const int a = wrapa(a_raw, g.na, g.pera, va);
    const int k0 = wrapa(k0_raw, g.nk, g.perk, vk0);
    const int k1 = wrapa(k0_raw + 1, g.nk, g.perk, vk1);
    const bool pairOK = va && vk0 && vk1 && k1 == k0 + 1;

    const T* tab = L.tab;
    const T wa_lo = va ? ldg(tab + g.wl_a + a) : T(0), wa_hi = va ? ldg(tab + g.wh_a + a) : T(0);
    const T wk_lo0 = vk0 ? ldg(tab + L.to.wl[2] + k0) : T(0), wk_hi0 = vk0 ? ldg(tab + L.to.wh[2] + k0) : T(0);
    const T wk_lo1 = vk1 ? ldg(tab + L.to.wl[2] + k1) : T(0), wk_hi1 = vk1 ? ldg(tab + L.to.wh[2] + k1) : T(0);
    // cell indices of a level fit 32 bits (the host only fuses such levels)
    const int rowa = (int)(L.base + (long)a * g.sa);
    const int sm = (int)g.sm;

    const int me = (ty + 1) * RK + 2 + 2 * tx;  // own pair in a padded plane
    const int mb = ty * EK + 2 * tx;            // own pair in a b plane

    // zero everything once: guard cells stay zero for good
    for (int q = ty * EKP + tx; q < (int)(F::smem / sizeof(T)); q += EKP * EA) xr[q] = T(0);
    __syncthreads();

    // queue the planes of step tt into ring slot tt % R (one cp.async group
    // per step, empty past the end so group counting stays uniform)
    auto issue = [&](int tt) {
        if (tt < steps) {
            bool vm;
            const int mp = wrapm(m0 - S + tt, g.nm, g.perm, vm);
            const int slot = tt % R;
            T* xd = xr + slot * PL + me;
            T* bd = br + slot * BP + mb;
            const int r = rowa + mp * sm;
            if (vm && pairOK) {
                cp_async<2 * sizeof(T)>(xd, L.x + r + k0, 2 * sizeof(T));
                cp_async<2 * sizeof(T)>(bd, L.b + r + k0, 2 * sizeof(T));
            } else {
                const bool v0 = vm && va && vk0, v1 = vm && va && vk1;
                cp_async<sizeof(T)>(xd, v0 ? L.x + r + k0 : L.x, v0 ? sizeof(T) : 0);
                cp_async<sizeof(T)>(xd + 1, v1 ? L.x + r + k1 : L.x, v1 ? sizeof(T) : 0);
                cp_async<sizeof(T)>(bd, v0 ? L.b + r + k0 : L.b, v0 ? sizeof(T) : 0);
                cp_async<sizeof(T)>(bd + 1, v1 ? L.b + r + k1 : L.b, v1 ? sizeof(T) : 0);
            }
            if (tx == 0 && ty == 0) {
                cp_async<sizeof(T)>(wr + 2 * slot, tab + g.wl_m + mp, vm ? sizeof(T) : 0);
                cp_async<sizeof(T)>(wr + 2 * slot + 1, tab + g.wh_m + mp, vm ? sizeof(T) : 0);
            }
        }
        cp_commit();
    };
#pragma unroll
    for (int tt = 0; tt < D; ++tt) issue(tt);

    // x of planes Lp .. Lp-S-1 for the own pair
    T xw[S + 2][2];
#pragma unroll
    for (int q = 0; q < S + 2; ++q) xw[q][0] = xw[q][1] = T(0);

    const bool outRow = ty >= S && ty < S + TA && a_raw < g.na;
    const bool outCol = tx >= HKP && tx < HKP + TKP;
    LevelView<T> O = L;
    O.x = xout;

    for (int t = 0; t < steps; ++t) {
        const int Lp = m0 - S + t;  // plane entering the window (raw index)
        cp_wait<D - 1>();           // this thread's copies of step t have landed
        // Publishes step t's plane and orders every read of the slots and
        // stage buffers rewritten below (all last read in step t-1 or earlier).
        __syncthreads();
        issue(t + D);

#pragma unroll
        for (int q = S + 1; q > 0; --q) {
            xw[q][0] = xw[q - 1][0];
            xw[q][1] = xw[q - 1][1];
        }
        {
            const V2 v = *reinterpret_cast<const V2*>(xr + (t % R) * PL + me);
            xw[0][0] = v.x;
            xw[0][1] = v.y;
        }
        // the pair member of the stage's colour is the same in every stage of
        // this step (plane and colour both flip from stage to stage)
        const int e = ((Lp - 1 + a_raw + k0_raw) & 1) == c1 ? 0 : 1;
        const bool ve = e ? vk1 : vk0;
        const int ce = me + e;
        T* const Bw = B + ((t + 1) & 1) * F::NB * PL;
        const T* const Bp = B + (t & 1) * F::NB * PL;

#pragma unroll
        for (int s = 1; s <= S; ++s) {
            const int P = Lp - s;
            bool vP;
            const int mP = wrapm(P, g.nm, g.perm, vP);
            const int slot = (t - s + R) % R;  // ring slot of plane P
            if (vP && va && ve) {
                // plane P after stage s-1: the loaded plane for s = 1
                const T* Bs = s == 1 ? xr + ((t - 1 + R) % R) * PL : Bp + (s - 2) * PL;
                T w[6], xn[6];
                w[0] = wr[2 * slot];
                w[1] = wr[2 * slot + 1];
                w[2] = wa_lo;
                w[3] = wa_hi;
                w[4] = e ? wk_lo1 : wk_lo0;
                w[5] = e ? wk_hi1 : wk_hi0;
                xn[0] = e ? xw[s + 1][1] : xw[s + 1][0];
                xn[1] = e ? xw[s - 1][1] : xw[s - 1][0];
                xn[2] = Bs[ce - RK];
                xn[3] = Bs[ce + RK];
                xn[4] = e ? xw[s][0] : Bs[ce - 1];
                xn[5] = e ? Bs[ce + 1] : xw[s][1];
                if (VAR) {
                    const long c = (long)rowa + (long)mP * sm + (e ? k1 : k0);
                    w[0] *= ldg(L.lam0 + c);
                    w[1] *= ldg(L.lam0 + c + L.si);
                    w[2] *= ldg(L.lam1 + c);
                    w[3] *= ldg(L.lam1 + c + L.sj);
                    w[4] *= ldg(L.lam2 + c);
                    w[5] *= ldg(L.lam2 + c + 1);
                }
                const T v = gs_value(w, xn, br[slot * BP + mb + e]);
                if (e)
                    xw[s][1] = v;
                else
                    xw[s][0] = v;
            }
            if (s < S) {
                V2 st;
                st.x = xw[s][0];
                st.y = xw[s][1];
                *reinterpret_cast<V2*>(Bw + (s - 1) * PL + me) = st;
            } else if (outRow && outCol && P >= m0 && P < m0 + mcount) {
                const long r = (long)rowa + (long)P * sm;
                if (k0_raw < g.nk) store_x(O, r + k0_raw, P, a, k0_raw, xw[S][0]);
                if (k0_raw + 1 < g.nk) store_x(O, r + k0_raw + 1, P, a, k0_raw + 1, xw[S][1]);
            }
        }
    }
    cp_wait<0>();  // no copy outlives the CTA
}

template <typename T, bool VAR, int S, int TA, int TKP>
void configure_one() {
    cudaFuncSetAttribute(k_smooth_fused<T, VAR, S, TA, TKP>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)FusedShape<T, S, TA, TKP>::smem);
}

template <typename T, bool VAR, int S, int TA, int TKP>
void launch_one(const LevelView<T>& L, T* xout, const FusedGeom& g, int c1, cudaStream_t s) {
    using F = FusedShape<T, S, TA, TKP>;
    const dim3 grid((g.nk + 2 * TKP - 1) / (2 * TKP), (g.na + TA - 1) / TA, (g.nm + g.ti - 1) / g.ti);
    const dim3 blk(F::EKP, F::EA, 1);
    k_smooth_fused<T, VAR, S, TA, TKP><<<grid, blk, F::smem, s>>>(L, xout, g, c1);
}

constexpr int kTA = 16, kTKP = 32;  // 16 x 64 cells per tile
// FP64 with three stages: 12 rows, so the register window and the ring fit
template <typename T>
constexpr int kTA3 = sizeof(T) == 8 ? 12 : 16;

template <typename T, bool VAR>
void configure_type() {
    configure_one<T, VAR, 1, kTA, kTKP>();
    configure_one<T, VAR, 2, kTA, kTKP>();
    configure_one<T, VAR, 3, kTA3<T>, kTKP>();
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
        case 1: launch_one<T, VAR, 1, kTA, kTKP>(L, xout, g, c1, s); break;
        case 2: launch_one<T, VAR, 2, kTA, kTKP>(L, xout, g, c1, s); break;
        default: launch_one<T, VAR, 3, kTA3<T>, kTKP>(L, xout, g, c1, s); break;
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
