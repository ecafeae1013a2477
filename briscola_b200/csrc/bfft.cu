// bfft.cu -- the FFT Poisson solver on B200 (C ABI: include/bfft.h).
//
// The reference solves a constant-coefficient Poisson (or Helmholtz, with
// ddt) problem on a rectilinear brick with two uniform directions by fast
// transforms in those two directions and a tridiagonal solve per mode in the
// third (FFTPoissonSolver.C:88-446).  Here the field stays in one k-fastest
// FP64 array in HBM and every step is a pass over it:
//   prep        -b - shift x_old - face terms, times 1/normalisation
//               (FFTPoissonSolver.C:116-183; the reference divides at the
//               end, FourierTransforms.C:414-420 -- the steps are linear)
//   transforms  k_transform along each transform axis: a CTA loads a tile
//               of lines into shared memory, runs one radix-2 complex FFT of
//               length M per line and writes the line back.  Every FFTW r2r
//               kind the reference uses is one zero-padded FFT with a
//               pre-twiddle of the input and a post-twiddle of the output:
//               REDFT10/01/11 and RODFT10/01/11 with M = 2N, R2HC/HC2R with
//               M = N (FourierTransforms.C:228-242).
//   tridiagonal k_tridiag: one thread per mode marches along the solve
//               axis (Thomas, or the cyclic two-system form for a periodic
//               solve axis, tridiagonalSolver.C:330-450); lines of
//               consecutive k are consecutive threads, so every step is a
//               coalesced load or store.
// Along the strided axes a transform tile is a run of consecutive k, so its
// loads and stores are runs of contiguous doubles too.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/bfft.h"

struct bfft_ctx;

namespace bfft {

// boundary pair of an axis (FourierTransforms.C:130-226)
enum Pair { P_EMPTY = 0, P_DD = 1, P_NN = 2, P_DN = 3, P_ND = 4, P_CC = 5 };
// output of a transform: halfcomplex of Z, Re(Z), Re(post Z), -Im(post Z)
enum Mode { M_R2HC = 0, M_HC2R = 1, M_RE = 2, M_NEG_IM = 3 };

constexpr int kThreads = 256;
constexpr int kMaxN = 512;

// lines along one axis: line l starts at (l / inner) * outer + (l % inner) * inner_stride
struct Lines {
    int n;             // cells along the axis
    long stride;       // element stride along the axis
    long inner;        // lines per outer index
    long inner_stride;
    long outer_stride;
    long count;
    int line_fast;     // consecutive lines are adjacent in memory (strided axes)
};

struct Transform {
    int M, logM, mode;
    int kind;             // Kind
    int odd;              // K_DCT2 / K_DCT3: the sine kinds RODFT10 / RODFT01
    int logN;             // log2 of the line length (transformed extents are powers of two)
    int logLB;            // log2 of the lines per CTA
    const double2* pre;   // n entries, nullptr: 1
    const double2* post;  // n entries, nullptr: 1
    const double2* tw;    // M entries: exp(-2 pi i q / M)
};

struct Tri {
    int ns, cyclic;
    double shift;
    double s0;            // first diagonal entry of a pinned (singular) mode
    int pin;              // the solve direction is N-N or periodic: the mode whose two
                          // eigenvalues are zero is singular and pinned (tridiagonalSolver.C)
    const double* A;      // D_k = ((e - A_k) - B_k)
    const double* B;
    const double* DU;
    const double* DL;
    const double* ev1;    // eigenvalue / h^2 of the first transform direction
    const double* ev2;
    int dir1_inner;       // the first transform direction is the inner line coordinate
    // modes with equal eigenvalues share one factorisation: class of each
    // inner / outer line coordinate, a representative coordinate per class
    const int* clsI;
    const int* clsO;
    const int* repI;
    const int* repO;
    int nci, nco;
    double* mfac;         // [ns][modes]: DL_k / Dh_{k-1}
    double* rfac;         // [ns][modes]: 1 / Dh_k
};

constexpr int kTriAhead = 8;  // rows a tridiagonal sweep loads ahead
constexpr int kSplitBlocks = 592;  // partial maxima of the face coefficients

struct Prep {
    int n0, n1, n2;
    double shift, scale;
    double corr[6];       // face terms subtracted on the boundary cells of each face
};

__device__ __forceinline__ long line_base(const Lines& L, long l) {
    // along axes 0 and 2 the outer stride is inner * inner_stride: no division
    if (L.outer_stride == L.inner * L.inner_stride) return l * L.inner_stride;
    const unsigned lu = (unsigned)l, in = (unsigned)L.inner;  // line counts fit 32 bits
    const unsigned o = lu / in;
    return (long)o * L.outer_stride + (long)(lu - o * in) * L.inner_stride;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// cos and sin of a pi / 8, a = 0..7: the twiddles of the register DFTs (R <= 16)
__host__ __device__ constexpr double cos8(int a) {
    return a == 0   ? 1.0
           : a == 1 ? 0.92387953251128675613
           : a == 2 ? 0.70710678118654752440
           : a == 3 ? 0.38268343236508977173
           : a == 4 ? 0.0
           : a == 5 ? -0.38268343236508977173
           : a == 6 ? -0.70710678118654752440
                    : -0.92387953251128675613;
}
__host__ __device__ constexpr double sin8(int a) { return a <= 4 ? cos8(4 - a) : cos8(a - 4); }

__host__ __device__ constexpr int brev_c(int i, int logR) {
    int r = 0;
    for (int b = 0; b < logR; ++b) r |= ((i >> b) & 1) << (logR - 1 - b);
    return r;
}

// x * exp(-i pi p / h) for compile-time p < h <= 8
template <int P, int H>
__device__ __forceinline__ double2 rot(double2 x) {
    constexpr int a = P * (8 / H);
    if constexpr (a == 0) {
        return x;
    } else if constexpr (a == 4) {
        return make_double2(x.y, -x.x);
    } else {
        constexpr double c = cos8(a), sn = sin8(a);
        return make_double2(x.x * c + x.y * sn, x.y * c - x.x * sn);
    }
}

template <int H, int I, int P, int R>
__device__ __forceinline__ void bfly(double2 (&v)[R]) {
    const double2 u = v[I + P];
    const double2 t = rot<P, H>(v[I + P + H]);
    v[I + P] = make_double2(u.x + t.x, u.y + t.y);
    v[I + P + H] = make_double2(u.x - t.x, u.y - t.y);
}

template <int H, int I, int P, int R>
__device__ __forceinline__ void bfly_group(double2 (&v)[R]) {
    if constexpr (P < H) {
        bfly<H, I, P, R>(v);
        bfly_group<H, I, P + 1, R>(v);
    }
}

template <int H, int I, int R>
__device__ __forceinline__ void bfly_stage(double2 (&v)[R]) {
    if constexpr (I < R) {
        bfly_group<H, I, 0, R>(v);
        bfly_stage<H, I + 2 * H, R>(v);
    }
}

template <int H, int R>
__device__ __forceinline__ void bfly_stages(double2 (&v)[R]) {
    if constexpr (H < R) {
        bfly_stage<H, 0, R>(v);
        bfly_stages<2 * H, R>(v);
    }
}

// in-register DFT of R points (natural order in and out): bit reversal,
// then radix-2 stages with the exact twiddles of kCos8 / kSin8
template <int R, int LOGR>
__device__ __forceinline__ void dft_regs(double2 (&v)[R]) {
    double2 t[R];
#pragma unroll
    for (int i = 0; i < R; ++i) t[i] = v[brev_c(i, LOGR)];
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = t[i];
    bfly_stages<1, R>(v);
}

constexpr int kTransformThreads = 128;
constexpr int kTileComplex = 2048;                              // complex values of a tile (LB lines of M)
constexpr int kPerThread = kTileComplex / kTransformThreads;    // 16 values per thread and pass
constexpr int kMaxLines = 256;  // lines of a tile (short lines fill less than the tile)

// tile index -> shared-memory slot: one pad slot after every 16, so the
// first Stockham pass's writes (stride R) do not pile onto one bank group,
// and for lines of 16 points or more one more after every line, so that
// the same point of consecutive lines (the strided axes' staging and
// output, thread by thread) falls in consecutive 16-byte bank groups
// instead of one (a line of M points and its pads is 17 M / 16 slots, a
// multiple of the eight groups)
template <int LOGM>
__device__ __forceinline__ int pad(int i) {
    return i + (i >> 4) + (LOGM >= 4 ? (i >> LOGM) : 0);
}

// pad(base + r 2^S) for r = 0..R-1 as pad(base) + r * stride (all inside
// one line): exact when S >= 4, or when base is a multiple of 16 and
// R 2^S <= 16
template <int S>
__device__ __forceinline__ constexpr int padded_step() {
    return S >= 4 ? 17 << (S - 4) : 1 << S;
}
constexpr int kTileSlots = kTileComplex + kTileComplex / 16 + kTileComplex / 16;
constexpr int kStage = 2 * kTileComplex;  // real values of a staged tile (two real lines per complex one)
constexpr int kTransformSmem = kTileSlots * 16 + kStage * 8;  // tile and staging buffer

// One Stockham radix-R pass (Govindaraju et al., SC 2008) in place over the
// tile: group j of a line reads points j + r M/R, twiddles them by
// exp(-2 pi i r (j mod Ns) / (Ns R)), takes their R-point DFT and writes
// them to (j / Ns) Ns R + (j mod Ns) + r Ns; natural order after the last
// pass.  Every thread holds its 16 / R groups in registers across the
// barrier between the reads and the writes.
template <int R, int LOGR, int LOGM, int LOGNS, int LB>
__device__ __forceinline__ void stockham_pass(double2* __restrict__ buf, const double2* __restrict__ tw) {
    constexpr int G = kPerThread / R;
    constexpr int LOGG = LOGM - LOGR;
    constexpr int groups = (1 << LOGG) * LB;
    constexpr int nsMask = (1 << LOGNS) - 1;
    double2 v[G][R];
    // a tile of short lines has fewer groups than threads x G: the extra
    // groups read group 0 and write nothing (predicated, so v stays in
    // registers)
    // reads: stride 2^LOGG, affine after padding when LOGG >= 4
    constexpr bool affineRead = LOGG >= 4;
    // writes: stride 2^LOGNS from idxD; idxD is a multiple of R when Ns = 1
    constexpr bool affineWrite = LOGNS >= 4 || (LOGNS == 0 && R <= 16);
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        const int g0 = threadIdx.x + gi * kTransformThreads;
        const int g = (groups >= kTileComplex / R || g0 < groups) ? g0 : 0;
        const int t = g >> LOGG, j = g & ((1 << LOGG) - 1);
        const int row = (t << LOGM) + j;
        if constexpr (affineRead) {
            const double2* src = buf + pad<LOGM>(row);
#pragma unroll
            for (int r = 0; r < R; ++r) v[gi][r] = src[r * padded_step<LOGG>()];
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r) v[gi][r] = buf[pad<LOGM>(row + (r << LOGG))];
        }
    }
    __syncthreads();
#pragma unroll
    for (int gi = 0; gi < G; ++gi) {
        const int g0 = threadIdx.x + gi * kTransformThreads;
        const bool ok = groups >= kTileComplex / R || g0 < groups;
        const int g = ok ? g0 : 0;
        const int t = g >> LOGG, j = g & ((1 << LOGG) - 1);
        const int jm = j & nsMask;
        if constexpr (LOGNS > 0) {
            const int step = jm << (LOGM - LOGNS - LOGR);
#pragma unroll
            for (int r = 1; r < R; ++r) v[gi][r] = cmul(v[gi][r], __ldg(tw + r * step));
        }
        dft_regs<R, LOGR>(v[gi]);
        const int idxD = (t << LOGM) + ((j >> LOGNS) << (LOGNS + LOGR)) + jm;
        if constexpr (affineWrite) {
            double2* dst = buf + pad<LOGM>(idxD);
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (ok) dst[r * padded_step<LOGNS>()] = v[gi][r];
        } else {
#pragma unroll
            for (int r = 0; r < R; ++r)
                if (ok) buf[pad<LOGM>(idxD + (r << LOGNS))] = v[gi][r];
        }
    }
    __syncthreads();
}

// all passes of an M = 2^LOGM point FFT: radix 16 while 16 points or more
// remain, then one radix 8, 4 or 2 pass
template <int LOGM, int LOGNS, int LB>
__device__ __forceinline__ void stockham_all(double2* __restrict__ buf, const double2* __restrict__ tw) {
    constexpr int rem = LOGM - LOGNS;
    if constexpr (rem >= 4) {
        stockham_pass<16, 4, LOGM, LOGNS, LB>(buf, tw);
        stockham_all<LOGM, LOGNS + 4, LB>(buf, tw);
    } else if constexpr (rem == 3) {
        stockham_pass<8, 3, LOGM, LOGNS, LB>(buf, tw);
    } else if constexpr (rem == 2) {
        stockham_pass<4, 2, LOGM, LOGNS, LB>(buf, tw);
    } else if constexpr (rem == 1) {
        stockham_pass<2, 1, LOGM, LOGNS, LB>(buf, tw);
    }
}

// the prep of the first transform's input: -b - shift x_old - face terms,
// times 1/normalisation (FFTPoissonSolver.C:116-183)
struct LoadPrep {
    int on;
    int axis;             // the transform axis
    int n1, n2;
    const double* xo;     // nullptr: no ddt term
    Prep P;
};

__device__ __forceinline__ void cp8(void* smem, const void* gmem, bool valid) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(valid ? 8 : 0)
                 : "memory");
}
// 16 bytes, of which `bytes` (0, 8 or 16) are read and the rest zero-filled
__device__ __forceinline__ void cp16(void* smem, const void* gmem, int bytes) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa), "l"(gmem), "r"(bytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Transform kinds.  K_TRIG: one zero-padded M = 2N point complex FFT per
// line with a pre-twiddle of the input and a post-twiddle of the output
// (the quarter-wave kinds REDFT11 / RODFT11).  The others put two real lines
// into one N-point complex FFT (line 2u as the real part, line 2u + 1 as the
// imaginary part) and separate the two spectra afterwards from
// Z(k) and conj Z(N - k):
//   K_R2HC  forward real FFT, halfcomplex output
//   K_HC2R  inverse real FFT of halfcomplex input (unnormalised)
//   K_DCT2  REDFT10 by Makhoul's reordering (J. Makhoul, "A fast cosine
//           transform in one and two dimensions", IEEE TASSP 28 (1980)):
//           v = (x0, x2, x4, ..., x5, x3, x1), X_k = 2 Re(e^{-i pi k/2N} V_k);
//           with `odd`, RODFT10 as REDFT10 of (-1)^n x_n, read backwards
//   K_DCT3  REDFT01, the inverse of that reordering: V_k = e^{i pi k/2N}
//           (X_k - i X_{N-k}) (X_N = 0), v = IDFT(V), x_2n = v_n,
//           x_2n+1 = v_{N-1-n}; with `odd`, RODFT01 as (-1)^n REDFT01 of
//           the reversed input
// so every kind the solver meets on a periodic, Dirichlet-Dirichlet or
// Neumann-Neumann axis costs half an N-point complex FFT per line.
enum Kind { K_R2HC = 0, K_HC2R = 1, K_TRIG = 2, K_DCT2 = 3, K_DCT3 = 4 };

// the slot of point p in Makhoul's reordering (even points first, then the
// odd ones backwards)
template <int N>
__device__ __forceinline__ int makhoul(int p) {
    return (p & 1) ? N - 1 - (p >> 1) : p >> 1;
}

// out(line) = transform of in(line), tile by tile, persistent: while a
// tile's FFT runs, the next tile's lines are already on their way into a
// staging buffer by cp.async, so the loads of HBM overlap the arithmetic.
// in == out is allowed: every element belongs to one tile, which the same
// CTA loads before it writes.  A tile holds LB lines of N points:
// LB = min(4096 / N, 256) for the paired kinds (LB / 2 complex lines of M =
// N points), min(2048 / M, 256) for K_TRIG.
//
// Element q of a tile is point p of tile line t, with t fastest along the
// strided axes (LF: a run of lines is a run of consecutive k) and p fastest
// along k (a tile is then one contiguous block).  Each thread handles the
// elements q = 2 (tid + u NT) and q + 1: with LF that is one pair of lines
// for the whole tile, so its addresses are affine in u.  With `pair` the two
// elements are adjacent in memory and move as one 16-byte copy.
template <int LOGM, int KIND, bool LF>
__global__ void __launch_bounds__(kTransformThreads, 3) k_transform(const double* in, double* out, Lines L,
                                                                    Transform T, LoadPrep LP, long tiles, int pair) {
    extern __shared__ double2 dsm[];
    double2* buf = dsm;                                          // [kTileSlots]
    double* stage = reinterpret_cast<double*>(dsm + kTileSlots);  // [kStage]
    constexpr int NT = kTransformThreads;
    constexpr bool PK = KIND != K_TRIG;  // two real lines per complex FFT
    constexpr int M = 1 << LOGM;
    constexpr int LOGN = PK ? LOGM : LOGM - 1;
    constexpr int N = 1 << LOGN;
    constexpr int LOGLB0 = PK ? 12 - LOGM : 11 - LOGM;
    constexpr int LOGLB = LOGLB0 < 8 ? LOGLB0 : 8;
    constexpr int LB = 1 << LOGLB;
    constexpr int LBC = PK ? LB / 2 : LB;            // complex lines of a tile
    constexpr int TOTAL = LB << LOGN;             // elements of a tile
    constexpr int PAIRS = (TOTAL / 2 + NT - 1) / NT;  // element pairs per thread
    static_assert(LB >= 2 && TOTAL >= 2 && TOTAL <= kStage, "tiles hold pairs");
    const int tid = threadIdx.x;
    double* bufd = reinterpret_cast<double*>(buf);

    // element q -> (line t, point p)
    auto tp = [&](int q, int& t, int& p) {
        if constexpr (LF) {
            t = q & (LB - 1);
            p = q >> LOGLB;
        } else {
            t = q >> LOGN;
            p = q & (N - 1);
        }
    };
    // global index of element q of the tile (lb: base of the thread's line
    // pair along LF axes)
    auto gidx = [&](long tile, long lb, int q) -> long {
        if constexpr (LF) {
            return lb + (long)(q >> LOGLB) * L.stride;
        } else {
            return tile * TOTAL + q;  // axis-2 lines are consecutive rows of n points
        }
    };
    // the lines of the thread's element pairs: fixed along LF axes
    auto pair_line = [&](long tile) { return tile * LB + ((2 * tid) & (LB - 1)); };
    // the first transform forms the right-hand side as it loads b: the face
    // terms of line l's two fixed coordinates...
    auto fixed_terms = [&](long l) {
        if (l >= L.count) return 0.0;
        const unsigned in = (unsigned)L.inner;
        const long co = (unsigned)l / in, ci = (unsigned)l - (unsigned)co * in;
        const int a0 = LP.axis == 0 ? 1 : 0, a1 = LP.axis == 2 ? 1 : 2;
        const int e0 = a0 == 0 ? LP.P.n0 : LP.P.n1, e1 = a1 == 1 ? LP.P.n1 : LP.P.n2;
        double f = 0.0;
        if (co == 0) f += LP.P.corr[2 * a0];
        if (co == e0 - 1) f += LP.P.corr[2 * a0 + 1];
        if (ci == 0) f += LP.P.corr[2 * a1];
        if (ci == e1 - 1) f += LP.P.corr[2 * a1 + 1];
        return f;
    };
    // ... and then those of its varying one (fixed: the line's fixed terms)
    auto prep = [&](double x, long tile, int t, int p, double fixed) {
        const long l = tile * LB + t;
        if (l >= L.count) return 0.0;
        double v = -x;
        if (LP.xo) v -= LP.P.shift * LP.xo[line_base(L, l) + (long)p * L.stride];
        double f = fixed;
        if (p == 0) f += LP.P.corr[2 * LP.axis];
        if (p == N - 1) f += LP.P.corr[2 * LP.axis + 1];
        return (v - f) * LP.P.scale;
    };
    auto issue = [&](long tile) {
        const long l = pair_line(tile);
        const long lb = LF ? line_base(L, l < L.count ? l : 0) : 0;
        // elements of the pair that exist: both, the first only (odd line
        // count), or none
        const long lines_left = L.count - tile * LB;
#pragma unroll
        for (int u = 0; u < PAIRS; ++u) {
            const int q = 2 * (tid + u * NT);
            if (q >= TOTAL) break;
            int t, p;
            tp(q, t, p);
            int nvalid;
            if constexpr (LF || N == 1) {
                nvalid = (int)min(max(lines_left - t, 0L), 2L);
            } else {
                nvalid = t < lines_left ? 2 : 0;
            }
            const long g = gidx(tile, lb, q);
            if (pair) {
                cp16(stage + q, nvalid ? in + g : in, 8 * nvalid);
            } else {
                // the pair's second element is the next line (LF) or point
                const long g1 = LF ? (nvalid > 1 ? line_base(L, l + 1) + (long)p * L.stride : 0) : g + 1;
                cp8(stage + q, nvalid > 0 ? in + g : in, nvalid > 0);
                cp8(stage + q + 1, nvalid > 1 ? in + g1 : in, nvalid > 1);
            }
        }
        cp_commit();
    };

    long tile = blockIdx.x;
    if (tile < tiles) issue(tile);
    for (; tile < tiles; tile += gridDim.x) {
        const long lines_left = L.count - tile * LB;
        cp_wait_all();
        // the staged tile is complete, and the previous tile's output phase
        // has finished reading buf
        __syncthreads();
        if constexpr (KIND == K_HC2R || KIND == K_DCT3) {
            // spectral input: point p of staged line t (the first
            // transform's prep applied)
            auto h = [&](int t, int p) {
                const int q = LF ? (p << LOGLB) + t : (t << LOGN) + p;
                const double x = stage[q];
                return LP.on ? prep(x, tile, t, p, fixed_terms(tile * LB + t)) : x;
            };
            // slot (u, k) of the complex tile from lines 2u and 2u + 1:
            // conj of the combined spectrum, so the forward FFT below gives
            // the conjugate of the inverse transform
            constexpr int SLOTS = TOTAL / 2;
#pragma unroll 4
            for (int s = tid; s < SLOTS; s += NT) {
                // consecutive threads take consecutive points along k, or
                // along the strided axes consecutive lines (adjacent in the
                // staged tile there)
                const int u = LF ? s & (LBC - 1) : s >> LOGN;
                const int k = LF ? s >> (LOGLB - 1) : s & (N - 1);
                const int ta = 2 * u, tb = 2 * u + 1;
                double ar, ai, br, bi;
                if constexpr (KIND == K_HC2R) {
                    // A_k of a halfcomplex line: (r_k, i_k), i_k stored at N - k
                    auto hc = [&](int t, double& re, double& im) {
                        if (k == 0) {
                            re = h(t, 0);
                            im = 0.0;
                        } else if (2 * k < N) {
                            re = h(t, k);
                            im = h(t, N - k);
                        } else if (2 * k == N) {
                            re = h(t, k);
                            im = 0.0;
                        } else {
                            re = h(t, N - k);
                            im = -h(t, k);
                        }
                    };
                    hc(ta, ar, ai);
                    hc(tb, br, bi);
                } else {
                    // V_k = c_k (X_k - i X_{N-k}), c_k = e^{i pi k / 2N}
                    const double2 c = __ldg(T.pre + k);
                    auto v = [&](int t, double& re, double& im) {
                        double xk, xn;
                        if (T.odd) {  // the reversed line
                            xk = h(t, N - 1 - k);
                            xn = k ? h(t, k - 1) : 0.0;
                        } else {
                            xk = h(t, k);
                            xn = k ? h(t, N - k) : 0.0;
                        }
                        re = c.x * xk + c.y * xn;
                        im = c.y * xk - c.x * xn;
                    };
                    v(ta, ar, ai);
                    v(tb, br, bi);
                }
                // conj(A + i B)
                buf[pad<LOGM>((u << LOGM) + k)] = make_double2(ar - bi, -(ai + br));
            }
        } else {
            // along LF axes the thread's line pair is fixed for the tile
            double fx[2] = {0.0, 0.0};
            if (LF && LP.on) {
                fx[0] = fixed_terms(pair_line(tile));
                fx[1] = fixed_terms(pair_line(tile) + 1);
            }
#pragma unroll
            for (int u = 0; u < PAIRS; ++u) {
                const int q = 2 * (tid + u * NT);
                if (q >= TOTAL) break;
                const double2 x2 = *reinterpret_cast<const double2*>(stage + q);
                double xs[2] = {x2.x, x2.y};
                int tq[2], pq[2];
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    tp(q + e, tq[e], pq[e]);
                    double x = xs[e];
                    if (LP.on) x = prep(x, tile, tq[e], pq[e], LF ? fx[e] : fixed_terms(tile * LB + tq[e]));
                    if constexpr (KIND == K_DCT2) {
                        if (T.odd && (pq[e] & 1)) x = -x;
                    }
                    xs[e] = x;
                }
                if constexpr (KIND == K_TRIG) {
#pragma unroll
                    for (int e = 0; e < 2; ++e) {
                        double2 c = make_double2(xs[e], 0.0);
                        if (T.pre) {
                            const double2 w = __ldg(T.pre + pq[e]);
                            c = make_double2(w.x * xs[e], w.y * xs[e]);
                        }
                        buf[pad<LOGM>((tq[e] << LOGM) + pq[e])] = c;
                    }
                } else {
                    // real part from the even line of a pair, imaginary part
                    // from the odd one; DCT2 reorders the points
                    const int p0 = KIND == K_DCT2 ? makhoul<N>(pq[0]) : pq[0];
                    if constexpr (LF) {  // the two elements are lines t, t + 1 at one point
                        buf[pad<LOGM>(((tq[0] >> 1) << LOGM) + p0)] = make_double2(xs[0], xs[1]);
                    } else {  // points p, p + 1 of one line
                        const int p1 = KIND == K_DCT2 ? makhoul<N>(pq[1]) : pq[1];
                        const int base = (tq[0] >> 1) << LOGM, part = tq[0] & 1;
                        bufd[2 * pad<LOGM>(base + p0) + part] = xs[0];
                        bufd[2 * pad<LOGM>(base + p1) + part] = xs[1];
                    }
                }
            }
            if constexpr (KIND == K_TRIG) {  // zero padding: points N..2N-1 of every line
#pragma unroll
                for (int u = 0; u < 2 * PAIRS; ++u) {
                    const int q = tid + u * NT;
                    if (q < TOTAL) buf[pad<LOGM>(((q >> LOGN) << LOGM) + N + (q & (N - 1)))] = make_double2(0.0, 0.0);
                }
            }
        }
        __syncthreads();
        // stage is free: the next tile's loads run under this tile's FFT
        if (tile + gridDim.x < tiles) issue(tile + gridDim.x);

        stockham_all<LOGM, 0, LBC>(buf, T.tw);

        // output: element q of the tile from spectrum entry (t, k)
        const long l = pair_line(tile);
        const long lb = LF ? line_base(L, l < L.count ? l : 0) : 0;
#pragma unroll
        for (int u = 0; u < PAIRS; ++u) {
            const int q = 2 * (tid + u * NT);
            if (q >= TOTAL) break;
            double y[2];
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                int t, k;
                tp(q + e, t, k);
                if constexpr (KIND == K_TRIG) {
                    const double2 z = buf[pad<LOGM>((t << LOGM) + k)];
                    const double2 c = T.post ? cmul(__ldg(T.post + k), z) : z;
                    y[e] = T.mode == M_RE ? c.x : -c.y;
                } else {
                    const int row = (t >> 1) << LOGM, part = t & 1;
                    if constexpr (KIND == K_R2HC) {
                        // A = (Z_k + conj Z_{N-k}) / 2, B = (Z_k - conj Z_{N-k}) / 2i;
                        // halfcomplex: Re at k <= N/2, Im of N - k above
                        const int kk = 2 * k <= N ? k : N - k;
                        const double2 zk = buf[pad<LOGM>(row + kk)], zn = buf[pad<LOGM>(row + ((N - kk) & (N - 1)))];
                        if (2 * k <= N)
                            y[e] = part == 0 ? 0.5 * (zk.x + zn.x) : 0.5 * (zk.y + zn.y);
                        else
                            y[e] = part == 0 ? 0.5 * (zk.y - zn.y) : -0.5 * (zk.x - zn.x);
                    } else if constexpr (KIND == K_DCT2) {
                        // 2 Re(w_k A_k) or 2 Re(w_k B_k), w_k = e^{-i pi k / 2N}
                        const int kk = T.odd ? N - 1 - k : k;
                        const double2 zk = buf[pad<LOGM>(row + kk)], zn = buf[pad<LOGM>(row + ((N - kk) & (N - 1)))];
                        const double2 w = __ldg(T.post + kk);
                        y[e] = part == 0 ? w.x * (zk.x + zn.x) - w.y * (zk.y - zn.y)
                                         : w.x * (zk.y + zn.y) + w.y * (zk.x - zn.x);
                    } else {
                        // the forward FFT of conj(A + i B) is conj(a + i b)
                        const int slot = KIND == K_DCT3 ? makhoul<N>(k) : k;
                        const double2 z = buf[pad<LOGM>(row + slot)];
                        double v = part == 0 ? z.x : -z.y;
                        if (KIND == K_DCT3 && T.odd && (k & 1)) v = -v;
                        y[e] = v;
                    }
                }
            }
            int t, p;
            tp(q, t, p);
            int nvalid;
            if constexpr (LF || N == 1) {
                nvalid = (int)min(max(lines_left - t, 0L), 2L);
            } else {
                nvalid = t < lines_left ? 2 : 0;
            }
            const long g = gidx(tile, lb, q);
            if (pair && nvalid == 2) {
                *reinterpret_cast<double2*>(out + g) = make_double2(y[0], y[1]);
            } else {
                if (nvalid > 0) out[g] = y[0];
                if (nvalid > 1) out[LF ? line_base(L, l + 1) + (long)p * L.stride : g + 1] = y[1];
            }
        }
    }
    cp_wait_all();  // no copy outlives the CTA
}

// Thomas per mode (tridiagonalSolver.C:330-374), or the cyclic form with
// two auxiliary systems (:376-450); dh and vv are scratch of the field's size
__global__ void __launch_bounds__(kThreads) k_tridiag(double* __restrict__ w, double* __restrict__ dh,
                                                      double* __restrict__ vv, Lines L, Tri T) {
    const long l = (long)blockIdx.x * kThreads + threadIdx.x;
    if (l >= L.count) return;
    const long base = line_base(L, l);
    const long st = L.stride;
    const int ns = T.ns;
    const unsigned inner = (unsigned)L.inner;
    const long co = (unsigned)l / inner, ci = (unsigned)l - (unsigned)co * inner;
    const long c1 = T.dir1_inner ? ci : co, c2 = T.dir1_inner ? co : ci;
    const double e1 = T.ev1[c1], e2 = T.ev2[c2];
    const double e = e1 + e2;
    const bool singular = T.pin && e1 == 0.0 && e2 == 0.0;
    auto diag = [&](int k) {
        const double d = (k == 0 && singular) ? T.s0 : (e - T.A[k]) - T.B[k];
        return d - T.shift;
    };
    if (!T.cyclic) {
        double Dp = diag(0);
        double fp = w[base];
        dh[base] = Dp;
        // loads run kTriAhead rows ahead of the elimination
        double fa[kTriAhead];
#pragma unroll
        for (int u = 0; u < kTriAhead; ++u) fa[u] = 1 + u < ns ? w[base + (1 + u) * st] : 0.0;
        for (int k0 = 1; k0 < ns; k0 += kTriAhead) {
#pragma unroll
            for (int u = 0; u < kTriAhead; ++u) {
                const int k = k0 + u;
                if (k < ns) {
                    const long c = base + k * st;
                    const double fk = fa[u];
                    const int kn = k + kTriAhead;
                    fa[u] = kn < ns ? w[base + kn * st] : 0.0;
                    const double m = T.DL[k] / Dp;
                    const double D = diag(k) - m * T.DU[k - 1];
                    const double f = fk - m * fp;
                    w[c] = f;
                    dh[c] = D;
                    Dp = D;
                    fp = f;
                }
            }
        }
        double p = fp / Dp;
        w[base + (ns - 1) * st] = p;
        double wa[kTriAhead], da[kTriAhead];
#pragma unroll
        for (int u = 0; u < kTriAhead; ++u) {
            const int k = ns - 2 - u;
            wa[u] = k >= 0 ? w[base + k * st] : 0.0;
            da[u] = k >= 0 ? dh[base + k * st] : 1.0;
        }
        for (int k0 = ns - 2; k0 >= 0; k0 -= kTriAhead) {
#pragma unroll
            for (int u = 0; u < kTriAhead; ++u) {
                const int k = k0 - u;
                if (k >= 0) {
                    const double wk = wa[u], dk = da[u];
                    const int kn = k - kTriAhead;
                    wa[u] = kn >= 0 ? w[base + kn * st] : 0.0;
                    da[u] = kn >= 0 ? dh[base + kn * st] : 1.0;
                    p = (wk - T.DU[k] * p) / dk;
                    w[base + k * st] = p;
                }
            }
        }
        return;
    }
    // cyclic: u solves the system without row 0 for f, v for the couplings
    // of row 0 (both from row 1, start = 1)
    const double f0 = w[base];
    double Dp = diag(1);
    double up = w[base + st];
    double vp = ns - 1 == 1 ? -T.DU[ns - 1] : -T.DL[1];
    dh[base + st] = Dp;
    vv[base + st] = vp;
    for (int k = 2; k < ns; ++k) {
        const long c = base + k * st;
        const double m = T.DL[k] / Dp;
        const double D = diag(k) - m * T.DU[k - 1];
        const double fu = w[c] - m * up;
        const double fv = (k == ns - 1 ? -T.DU[ns - 1] : 0.0) - m * vp;
        w[c] = fu;
        vv[c] = fv;
        dh[c] = D;
        Dp = D;
        up = fu;
        vp = fv;
    }
    double u = up / Dp, v = vp / Dp;
    const double uN = u, vN = v;
    w[base + (ns - 1) * st] = u;
    vv[base + (ns - 1) * st] = v;
    for (int k = ns - 2; k >= 1; --k) {
        const long c = base + k * st;
        u = (w[c] - T.DU[k] * u) / dh[c];
        v = (vv[c] - T.DU[k] * v) / dh[c];
        w[c] = u;
        vv[c] = v;
    }
    // u, v now hold row 1
    const double p0 = (f0 - T.DL[0] * uN - T.DU[0] * u) / (diag(0) + T.DL[0] * vN + T.DU[0] * v);
    w[base] = p0;
    for (int k = 1; k < ns; ++k) {
        const long c = base + k * st;
        w[c] = w[c] + p0 * vv[c];
    }
}

// Thomas elimination factors of each class of modes (the forward sweep of
// tridiagonalSolver.C:343-353 without the right-hand side): m_k and 1/Dh_k
__global__ void k_tri_factor(Tri T) {
    const int mode = blockIdx.x * blockDim.x + threadIdx.x;
    const int modes = T.nci * T.nco;
    if (mode >= modes) return;
    const int ci = T.repI[mode % T.nci], co = T.repO[mode / T.nci];
    const int c1 = T.dir1_inner ? ci : co, c2 = T.dir1_inner ? co : ci;
    const double e1 = T.ev1[c1], e2 = T.ev2[c2];
    const double e = e1 + e2;
    const bool singular = T.pin && e1 == 0.0 && e2 == 0.0;
    auto diag = [&](int k) {
        const double d = (k == 0 && singular) ? T.s0 : (e - T.A[k]) - T.B[k];
        return d - T.shift;
    };
    double Dp = diag(0);
    T.mfac[mode] = 0.0;
    T.rfac[mode] = 1.0 / Dp;
    for (int k = 1; k < T.ns; ++k) {
        const double m = T.DL[k] / Dp;
        const double D = diag(k) - m * T.DU[k - 1];
        T.mfac[(long)k * modes + mode] = m;
        T.rfac[(long)k * modes + mode] = 1.0 / D;
        Dp = D;
    }
}

// the Thomas sweeps with the factors of the line's mode class: one FMA chain
// forward, one backward, the field read and written once each way
__global__ void __launch_bounds__(kThreads) k_tri_apply(double* __restrict__ w, Lines L, Tri T) {
    const long l = (long)blockIdx.x * kThreads + threadIdx.x;
    if (l >= L.count) return;
    const long base = line_base(L, l);
    const long st = L.stride;
    const int ns = T.ns;
    const unsigned inner = (unsigned)L.inner;
    const int co = (int)((unsigned)l / inner), ci = (int)((unsigned)l - (unsigned)co * inner);
    const int modes = T.nci * T.nco;
    const int mode = T.clsO[co] * T.nci + T.clsI[ci];
    const double* mf = T.mfac + mode;
    const double* rf = T.rfac + mode;
    // field values and factors run kTriAhead rows ahead of the FMA chains
    double fp = w[base];
    double fa[kTriAhead], ma[kTriAhead];
#pragma unroll
    for (int u = 0; u < kTriAhead; ++u) {
        const int k = 1 + u;
        fa[u] = k < ns ? w[base + k * st] : 0.0;
        ma[u] = k < ns ? __ldg(mf + (long)k * modes) : 0.0;
    }
    for (int k0 = 1; k0 < ns; k0 += kTriAhead) {
#pragma unroll
        for (int u = 0; u < kTriAhead; ++u) {
            const int k = k0 + u;
            if (k < ns) {
                const double fk = fa[u], mk = ma[u];
                const int kn = k + kTriAhead;
                fa[u] = kn < ns ? w[base + kn * st] : 0.0;
                ma[u] = kn < ns ? __ldg(mf + (long)kn * modes) : 0.0;
                fp = fk - mk * fp;
                w[base + k * st] = fp;
            }
        }
    }
    double p = fp * __ldg(rf + (long)(ns - 1) * modes);
    w[base + (ns - 1) * st] = p;
    double ra[kTriAhead], ua[kTriAhead];
#pragma unroll
    for (int u = 0; u < kTriAhead; ++u) {
        const int k = ns - 2 - u;
        fa[u] = k >= 0 ? w[base + k * st] : 0.0;
        ra[u] = k >= 0 ? __ldg(rf + (long)k * modes) : 0.0;
        ua[u] = k >= 0 ? T.DU[k] : 0.0;
    }
    for (int k0 = ns - 2; k0 >= 0; k0 -= kTriAhead) {
#pragma unroll
        for (int u = 0; u < kTriAhead; ++u) {
            const int k = k0 - u;
            if (k >= 0) {
                const double wk = fa[u], rk = ra[u], duk = ua[u];
                const int kn = k - kTriAhead;
                fa[u] = kn >= 0 ? w[base + kn * st] : 0.0;
                ra[u] = kn >= 0 ? __ldg(rf + (long)kn * modes) : 0.0;
                ua[u] = kn >= 0 ? T.DU[kn] : 0.0;
                p = (wk - duk * p) * rk;
                w[base + k * st] = p;
            }
        }
    }
}

// ---- split Poisson solver -------------------------------------------------

struct SplitGeom {
    int n[3];
    const double* h[3];   // cell sizes per axis
    int bc[6];            // BFFT_BC_* per face
    double value[6];      // Dirichlet value or Neumann gradient
};

// largest of the three face arrays: per-block maxima, then one block
__global__ void k_max3(const double* __restrict__ a, long na, const double* __restrict__ b, long nb,
                       const double* __restrict__ c, long nc, double* __restrict__ part) {
    double m = -1e308;
    const long stride = (long)gridDim.x * blockDim.x;
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < na + nb + nc; q += stride) {
        const double v = q < na ? a[q] : q < na + nb ? b[q - na] : c[q - na - nb];
        m = fmax(m, v);
    }
    __shared__ double sm[kThreads];
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sm[0];
}

__global__ void k_max_final(double* __restrict__ part, int n) {
    __shared__ double sm[kThreads];
    double m = -1e308;
    for (int q = threadIdx.x; q < n; q += kThreads) m = fmax(m, part[q]);
    sm[threadIdx.x] = m;
    __syncthreads();
    for (int w = kThreads / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) sm[threadIdx.x] = fmax(sm[threadIdx.x], sm[threadIdx.x + w]);
        __syncthreads();
    }
    if (threadIdx.x == 0) part[0] = sm[0];
}

// one face's flux term lambda' (x_nb - x_c) delta, with the neighbour or the
// ghost the face condition sets (DirichletBoundaryCondition.C:51-71,
// NeumannBoundaryCondition.C:59-85; mirrored ghost cells: delta = 1/h)
__device__ __forceinline__ double face_term(const SplitGeom& G, int axis, int side, int idx, double lamp, double xc,
                                            double xnb, bool boundary, double delta) {
    if (!boundary) return lamp * (xnb - xc) * delta;
    const int f = 2 * axis + side;
    const int bc = G.bc[f];
    if (bc == BFFT_BC_NEUMANN) return lamp * G.value[f];  // (x_g - x_c) delta = g
    if (bc == BFFT_BC_DIRICHLET) return lamp * (2.0 * G.value[f] - 2.0 * xc) * delta;
    return 0.0;  // empty
}

// bhat = b / lambda0 + div((lambda / lambda0 - 1) faceGrad(x) faceArea)
__global__ void k_split_source(const double* __restrict__ x, const double* __restrict__ b,
                               const double* __restrict__ lam0, const double* __restrict__ lam1,
                               const double* __restrict__ lam2, double lambda0, double* __restrict__ bhat,
                               SplitGeom G) {
    const int n1 = G.n[1], n2 = G.n[2];
    // one CTA row of k per (i, j): grid (k chunks, n1, n0)
    const int i = blockIdx.z, j = blockIdx.y;
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n2; k += gridDim.x * blockDim.x) {
        const long c = ((long)i * n1 + j) * n2 + k;
        const int ijk[3] = {i, j, k};
        const long sx[3] = {(long)n1 * n2, n2, 1};
        const double xc = x[c];
        double div = 0.0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const int q = ijk[a], n = G.n[a];
            const double* h = G.h[a];
            const bool per = G.bc[2 * a] == BFFT_BC_PERIODIC;
            const double hc = h[q];
            // lower and upper faces of the cell along axis a
            const double hlo = q > 0 ? h[q - 1] : (per ? h[n - 1] : hc);
            const double hhi = q < n - 1 ? h[q + 1] : (per ? h[0] : hc);
            const double dw = 0.5 * (hc + hlo), de = 0.5 * (hc + hhi);
            long flo, fhi;  // face indices in the face array of axis a
            if (a == 0) {
                flo = ((long)i * n1 + j) * n2 + k;
                fhi = ((long)(i + 1) * n1 + j) * n2 + k;
            } else if (a == 1) {
                flo = ((long)i * (n1 + 1) + j) * n2 + k;
                fhi = ((long)i * (n1 + 1) + j + 1) * n2 + k;
            } else {
                flo = ((long)i * n1 + j) * (n2 + 1) + k;
                fhi = flo + 1;
            }
            const double* lam = a == 0 ? lam0 : a == 1 ? lam1 : lam2;
            const double llo = lam[flo] / lambda0 - 1.0, lhi = lam[fhi] / lambda0 - 1.0;
            const bool blo = q == 0 && !per, bhi = q == n - 1 && !per;
            double xlo = 0.0, xhi = 0.0;
            if (!blo) xlo = x[q > 0 ? c - sx[a] : c + (long)(n - 1) * sx[a]];
            if (!bhi) xhi = x[q < n - 1 ? c + sx[a] : c - (long)(n - 1) * sx[a]];
            // lower face: outward gradient (x_lo - x_c) delta; upper face enters with a minus sign
            // of its own outward gradient, i.e. (x_hi - x_c) delta
            const double tlo = face_term(G, a, 0, q, llo, xc, xlo, blo, 1.0 / dw);
            const double thi = face_term(G, a, 1, q, lhi, xc, xhi, bhi, 1.0 / de);
            div += (tlo + thi) / hc;
        }
        bhat[c] = b[c] / lambda0 + div;
    }
}

__global__ void k_axpby(double a, const double* x, double c, const double* y, double* out, long n) {
    for (long q = (long)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (long)gridDim.x * blockDim.x)
        out[q] = a * x[q] + c * y[q];
}

// w = (-b - shift x_old - face terms) * scale
__global__ void k_prep(double* __restrict__ w, const double* __restrict__ b, const double* __restrict__ xo, Prep P) {
    const long total = (long)P.n0 * P.n1 * P.n2;
    for (long c = (long)blockIdx.x * blockDim.x + threadIdx.x; c < total; c += (long)gridDim.x * blockDim.x) {
        const int k = (int)(c % P.n2);
        const long ij = c / P.n2;
        const int j = (int)(ij % P.n1), i = (int)(ij / P.n1);
        double v = -b[c];
        if (xo) v -= P.shift * xo[c];
        if (i == 0) v -= P.corr[0];
        if (i == P.n0 - 1) v -= P.corr[1];
        if (j == 0) v -= P.corr[2];
        if (j == P.n1 - 1) v -= P.corr[3];
        if (k == 0) v -= P.corr[4];
        if (k == P.n2 - 1) v -= P.corr[5];
        w[c] = v * P.scale;
    }
}

// the line lengths of a kind: M = N = 1 .. kMaxN for the paired kinds,
// M = 2N = 2 .. 2 kMaxN for K_TRIG
constexpr int kMinLogM(int kind) { return kind == K_TRIG ? 1 : 0; }

template <int KIND, bool LF, int LOGM = kMinLogM(KIND)>
void launch_kind(int logM, unsigned grid, cudaStream_t st, const double* in, double* out, const Lines& L,
                 const Transform& T, const LoadPrep& lp, long tiles, int pair) {
    if constexpr (LOGM <= kMinLogM(KIND) + 9) {
        if (logM == LOGM)
            k_transform<LOGM, KIND, LF><<<grid, kTransformThreads, kTransformSmem, st>>>(in, out, L, T, lp, tiles, pair);
        else
            launch_kind<KIND, LF, LOGM + 1>(logM, grid, st, in, out, L, T, lp, tiles, pair);
    }
}

template <bool LF>
void launch_lf(int kind, int logM, unsigned grid, cudaStream_t st, const double* in, double* out, const Lines& L,
               const Transform& T, const LoadPrep& lp, long tiles, int pair) {
    switch (kind) {
        case K_R2HC: launch_kind<K_R2HC, LF>(logM, grid, st, in, out, L, T, lp, tiles, pair); break;
        case K_HC2R: launch_kind<K_HC2R, LF>(logM, grid, st, in, out, L, T, lp, tiles, pair); break;
        case K_DCT2: launch_kind<K_DCT2, LF>(logM, grid, st, in, out, L, T, lp, tiles, pair); break;
        case K_DCT3: launch_kind<K_DCT3, LF>(logM, grid, st, in, out, L, T, lp, tiles, pair); break;
        default: launch_kind<K_TRIG, LF>(logM, grid, st, in, out, L, T, lp, tiles, pair); break;
    }
}

void launch_transform(int kind, int logM, unsigned grid, cudaStream_t st, const double* in, double* out,
                      const Lines& L, const Transform& T, const LoadPrep& lp, long tiles, int pair) {
    if (L.line_fast)
        launch_lf<true>(kind, logM, grid, st, in, out, L, T, lp, tiles, pair);
    else
        launch_lf<false>(kind, logM, grid, st, in, out, L, T, lp, tiles, pair);
}

template <int KIND, bool LF, int LOGM = kMinLogM(KIND)>
void allow_kind() {
    if constexpr (LOGM <= kMinLogM(KIND) + 9) {
        cudaFuncSetAttribute(k_transform<LOGM, KIND, LF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             kTransformSmem);
        allow_kind<KIND, LF, LOGM + 1>();
    }
}

void allow_smem_all() {
    allow_kind<K_R2HC, true>();
    allow_kind<K_R2HC, false>();
    allow_kind<K_HC2R, true>();
    allow_kind<K_HC2R, false>();
    allow_kind<K_DCT2, true>();
    allow_kind<K_DCT2, false>();
    allow_kind<K_DCT3, true>();
    allow_kind<K_DCT3, false>();
    allow_kind<K_TRIG, true>();
    allow_kind<K_TRIG, false>();
}

struct BadArg {
    int code;
    std::string msg;
};

template <typename T>
T* dalloc(size_t n) {
    void* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) throw BadArg{BMG_CUDA_ERROR, std::string("cudaMalloc: ") + cudaGetErrorString(e)};
    return static_cast<T*>(p);
}

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw BadArg{BMG_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e)};
}

struct AxisPlan {
    int pair = P_EMPTY;
    Lines lines{};
    Transform fwd{}, bwd{};
    int LB = 1;
    int adjacent = 0;   // the two elements of a thread's pair are adjacent in memory
    bool identity = false;  // a periodic axis of one cell: nothing to transform
};

}  // namespace bfft

using namespace bfft;

struct bfft_ctx {
    int dev = 0;
    int sms = 148;
    int n[3] = {0, 0, 0};
    int s = 0, dir1 = 0, dir2 = 0;
    AxisPlan ax[3];
    Lines solveLines{};
    Tri tri{};
    Prep prep{};
    double* w = nullptr;
    double* dh = nullptr;
    double* vv = nullptr;
    std::vector<void*> owned;
    cudaStream_t stream = nullptr;
    bool ownStream = false;
    SplitGeom split{};
    double* part = nullptr;     // reduction partials (split solver)
    bool factored = false;      // the Thomas factors hold for factorShift
    double factorShift = 0.0;
    std::string err;
};

namespace {

bool power_of_two(int n) { return n > 0 && (n & (n - 1)) == 0; }

int log2i(int n) {
    int l = 0;
    while ((1 << l) < n) ++l;
    return l;
}

template <typename T>
T* upload(bfft_ctx* c, const std::vector<T>& v) {
    T* p = dalloc<T>(v.size());
    c->owned.push_back(p);
    check(cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice), "cudaMemcpy");
    return p;
}

double2 expi(long double angle, long double scale = 1.0L) {
    return make_double2((double)(scale * cosl(angle)), (double)(scale * sinl(angle)));
}

// transform tables of one axis (the kinds of FourierTransforms.C:228-242)
void planTransforms(bfft_ctx* c, int d) {
    AxisPlan& A = c->ax[d];
    const int N = c->n[d];
    if (A.pair == P_EMPTY) return;
    const long double pi = 3.141592653589793238462643383279502884L;
    // periodic, D-D and N-N axes: two real lines per N-point complex FFT;
    // the quarter-wave kinds (D-N, N-D): a zero-padded 2N-point FFT per line
    const bool paired = A.pair == P_CC || A.pair == P_NN || A.pair == P_DD;
    const int M = paired ? N : 2 * N;
    std::vector<double2> tw(M);
    for (int j = 0; j < M; ++j) tw[j] = expi(-2.0L * pi * j / M);
    const double2* twd = upload(c, tw);
    auto table = [&](auto f) {
        std::vector<double2> t(N);
        for (int q = 0; q < N; ++q) t[q] = f(q);
        return upload(c, t);
    };
    const int LB = paired ? std::min(kStage / N, kMaxLines) : std::min(kTileComplex / M, kMaxLines);
    Transform f{M, log2i(M), M_RE, K_TRIG, 0, log2i(N), log2i(LB), nullptr, nullptr, twd};
    Transform b = f;
    switch (A.pair) {
        case P_CC:
            f.mode = M_R2HC;
            b.mode = M_HC2R;
            f.kind = K_R2HC;
            b.kind = K_HC2R;
            break;
        case P_NN:  // REDFT10 / REDFT01
        case P_DD:  // RODFT10 / RODFT01
            f.kind = K_DCT2;
            b.kind = K_DCT3;
            f.odd = b.odd = A.pair == P_DD;
            f.post = table([&](int k) { return expi(-pi * k / (2.0L * N)); });
            b.pre = table([&](int k) { return expi(pi * k / (2.0L * N)); });
            break;
        case P_DN:  // RODFT11 both ways
        case P_ND:  // REDFT11 both ways
            f.mode = b.mode = A.pair == P_DN ? M_NEG_IM : M_RE;
            f.pre = b.pre = table([&](int q) { return expi(-pi * q / (2.0L * N)); });
            f.post = b.post = table([&](int k) { return expi(-pi * (2 * k + 1) / (4.0L * N), 2.0L); });
            break;
    }
    A.fwd = f;
    A.bwd = b;
    A.LB = LB;
    A.identity = A.pair == P_CC && N == 1;
    // pairs: consecutive lines along the strided axes (adjacent when the k
    // rows hold an even number of cells), consecutive points along k
    const long n1 = c->n[1], n2 = c->n[2];
    A.adjacent = d == 2 ? 1 : d == 1 ? (n2 % 2 == 0) : ((n1 * n2) % 2 == 0);
}

Lines linesAlong(const int n[3], int d) {
    const long n0 = n[0], n1 = n[1], n2 = n[2];
    Lines L{};
    L.n = n[d];
    if (d == 2) {
        L.stride = 1;
        L.inner = n1;
        L.inner_stride = n2;
        L.outer_stride = n1 * n2;
        L.count = n0 * n1;
        L.line_fast = 0;
    } else if (d == 1) {
        L.stride = n2;
        L.inner = n2;
        L.inner_stride = 1;
        L.outer_stride = n1 * n2;
        L.count = n0 * n2;
        L.line_fast = 1;
    } else {
        L.stride = n1 * n2;
        L.inner = n2;
        L.inner_stride = 1;
        L.outer_stride = n2;
        L.count = n1 * n2;
        L.line_fast = 1;
    }
    return L;
}

int pairOf(int lo, int hi) {
    if (lo == BFFT_BC_EMPTY || hi == BFFT_BC_EMPTY) return lo == hi ? P_EMPTY : -1;
    if (lo == BFFT_BC_PERIODIC || hi == BFFT_BC_PERIODIC) return lo == hi ? P_CC : -1;
    if (lo == BFFT_BC_DIRICHLET) return hi == BFFT_BC_DIRICHLET ? P_DD : P_DN;
    return hi == BFFT_BC_DIRICHLET ? P_ND : P_NN;
}

// eigenvalues of tridiagonalSolver.C:20-115
std::vector<double> eigen(int N, int pair) {
    std::vector<double> l(N, 0.0);
    const double pi = 3.14159265358979323846;
    for (int i = 0; i < N; ++i) {
        double s = 0.0;
        switch (pair) {
            case P_DD: s = std::sin((i + 1) * pi / (2.0 * N)); break;
            case P_NN: s = std::sin(i * pi / (2.0 * N)); break;
            case P_DN:
            case P_ND: s = std::sin((2.0 * (i + 1) - 1.0) * pi / (4.0 * N)); break;
            case P_CC: s = std::sin(i * pi / N); break;
            default: s = 0.0;
        }
        l[i] = -4.0 * s * s;
    }
    return l;
}

void build(bfft_ctx* c, const bfft_desc* d) {
    for (int a = 0; a < 3; ++a) {
        if (d->n[a] < 1) throw BadArg{BMG_BAD_ARG, "extents must be positive"};
        if (!d->points[a]) throw BadArg{BMG_BAD_ARG, "missing vertex coordinates"};
        c->n[a] = d->n[a];
        const int p = pairOf(d->bc[2 * a], d->bc[2 * a + 1]);
        if (p < 0) throw BadArg{BMG_BAD_ARG, "incorrect boundary condition pair"};
        if (p == P_EMPTY && d->n[a] != 1) throw BadArg{BMG_BAD_ARG, "an empty axis has one cell"};
        c->ax[a].pair = p;
        for (int q = 0; q < d->n[a]; ++q)
            if (!(d->points[a][q + 1] > d->points[a][q])) throw BadArg{BMG_BAD_ARG, "vertex coordinates must increase"};
    }
    // planner.C:60-99 on one process: the first non-uniform axis solves
    std::vector<double> h[3];
    bool uniform[3];
    for (int a = 0; a < 3; ++a) {
        h[a].resize(c->n[a]);
        double lo = 1e300, hi = -1e300;
        for (int q = 0; q < c->n[a]; ++q) {
            h[a][q] = d->points[a][q + 1] - d->points[a][q];
            lo = std::min(lo, h[a][q]);
            hi = std::max(hi, h[a][q]);
        }
        uniform[a] = hi - lo <= 1e-12 * hi;
    }
    c->s = -1;
    for (int a = 0; a < 3 && c->s < 0; ++a)
        if (!uniform[a]) c->s = a;
    if (c->s < 0) c->s = c->n[0] > 1 ? 0 : 2;
    for (int a = 0; a < 3; ++a)
        if (a != c->s && !uniform[a])
            throw BadArg{BMG_BAD_ARG, "at least two mesh directions must be uniform for the FFT solver"};
    // tridiagonalSolver.C:300-325
    c->dir1 = c->s == 0 ? 2 : 0;
    c->dir2 = c->s == 1 ? 2 : 1;
    const int s = c->s;
    if (c->ax[s].pair == P_EMPTY || c->n[s] < 2) throw BadArg{BMG_UNSUPPORTED, "the solve direction needs two cells or more"};
    for (int a : {c->dir1, c->dir2}) {
        if (c->ax[a].pair == P_EMPTY) continue;
        if (!power_of_two(c->n[a]) || c->n[a] > kMaxN)
            throw BadArg{BMG_UNSUPPORTED, "transformed extents must be powers of two up to 512"};
    }

    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= c->dev || c->dev < 0)
        throw BadArg{BMG_NO_DEVICE, "no usable CUDA device"};
    check(cudaSetDevice(c->dev), "cudaSetDevice");
    check(cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->dev), "cudaDeviceGetAttribute");
    allow_smem_all();
    for (int a : {c->dir1, c->dir2}) {
        c->ax[a].lines = linesAlong(c->n, a);
        planTransforms(c, a);
    }

    // tridiagonal coefficients (tridiagonalSolver.C:117-280), ghost cell
    // sizes from levelPoints.C:198-236 / 326-400
    const int ns = c->n[s];
    const int ps = c->ax[s].pair;
    std::vector<double> hg(ns + 2);
    for (int q = 0; q < ns; ++q) hg[q + 1] = h[s][q];
    hg[0] = ps == P_CC ? h[s][ns - 1] : h[s][0];
    hg[ns + 1] = ps == P_CC ? h[s][0] : h[s][ns - 1];
    std::vector<double> A(ns), B(ns), DU(ns), DL(ns);
    for (int k = 0; k < ns; ++k) {
        const double d3 = hg[k + 1], d3e = (hg[k + 1] + hg[k + 2]) / 2.0, d3w = (hg[k + 1] + hg[k]) / 2.0;
        A[k] = 1.0 / (d3e * d3);
        B[k] = 1.0 / (d3 * d3w);
        DU[k] = 1.0 / (d3 * d3e);
        DL[k] = 1.0 / (d3 * d3w);
    }
    const double d30 = hg[1], d3e0 = (hg[1] + hg[2]) / 2.0, d3w0 = (hg[1] + hg[0]) / 2.0;
    const double d3L = hg[ns], d3eL = (hg[ns] + hg[ns + 1]) / 2.0, d3wL = (hg[ns] + hg[ns - 1]) / 2.0;
    double s0 = 0.0;
    switch (ps) {
        case P_DD:
            B[0] = 2.0 / (d30 * d3w0);
            A[ns - 1] = 2.0 / (d3eL * d3L);
            break;
        case P_NN:
            B[0] = 0.0;
            A[ns - 1] = 0.0;
            s0 = -1.0 / (d3e0 * d30) - 2.0 / (d30 * d3w0);
            break;
        case P_DN:
            B[0] = 2.0 / (d30 * d3w0);
            A[ns - 1] = 0.0;
            break;
        case P_ND:
            B[0] = 0.0;
            A[ns - 1] = 2.0 / (d3eL * d3L);
            break;
        case P_CC:
            s0 = -1.0 / (d3e0 * d30) - 2.0 / (d30 * d3w0);
            break;
    }
    // a pinned mode exists only where the solve direction has no Dirichlet
    // face (N-N or periodic) and both transform directions have a zero
    // eigenvalue; with a Dirichlet face in the solve direction the mode of
    // zero eigenvalues is an ordinary one
    auto ev = [&](int a) {
        std::vector<double> l = eigen(c->n[a], c->ax[a].pair);
        const double hh = h[a][0] * h[a][0];
        for (double& x : l) x /= hh;
        return l;
    };
    Tri& T = c->tri;
    T.ns = ns;
    T.cyclic = ps == P_CC;
    T.s0 = s0;
    T.pin = ps == P_NN || ps == P_CC;
    T.A = upload(c, A);
    T.B = upload(c, B);
    T.DU = upload(c, DU);
    T.DL = upload(c, DL);
    T.ev1 = upload(c, ev(c->dir1));
    T.ev2 = upload(c, ev(c->dir2));
    c->solveLines = linesAlong(c->n, s);
    // the lines' inner coordinate: k for s = 0 and 1, j for s = 2
    const int innerAxis = s == 2 ? 1 : 2;
    const int outerAxis = s == 0 ? 1 : 0;
    T.dir1_inner = c->dir1 == innerAxis;
    // classes of equal eigenvalues: frequencies p and N - p of a real
    // Fourier axis (halfcomplex positions), every position otherwise
    auto classes = [&](int a, std::vector<int>& cls, std::vector<int>& rep) {
        const int N = c->n[a];
        cls.assign(N, 0);
        rep.clear();
        if (c->ax[a].pair == P_CC) {
            for (int q = 0; q < N; ++q) cls[q] = q <= N / 2 ? q : N - q;
            for (int q = 0; q <= N / 2; ++q) rep.push_back(q);
        } else {
            for (int q = 0; q < N; ++q) {
                cls[q] = q;
                rep.push_back(q);
            }
        }
    };
    std::vector<int> cI, rI, cO, rO;
    classes(innerAxis, cI, rI);
    classes(outerAxis, cO, rO);
    T.clsI = upload(c, cI);
    T.repI = upload(c, rI);
    T.clsO = upload(c, cO);
    T.repO = upload(c, rO);
    T.nci = (int)rI.size();
    T.nco = (int)rO.size();
    if (!T.cyclic) {
        const size_t f = (size_t)T.nci * T.nco * ns;
        T.mfac = dalloc<double>(f);
        T.rfac = dalloc<double>(f);
        c->owned.push_back(T.mfac);
        c->owned.push_back(T.rfac);
    }

    // right-hand side terms of the faces (FFTPoissonSolver.C:140-183)
    Prep& P = c->prep;
    P.n0 = c->n[0];
    P.n1 = c->n[1];
    P.n2 = c->n[2];
    double norm = 1.0;
    for (int a : {c->dir1, c->dir2}) {
        const int p = c->ax[a].pair;
        if (p != P_EMPTY) norm *= p == P_CC ? c->n[a] : 2.0 * c->n[a];
    }
    P.scale = 1.0 / norm;
    for (int f = 0; f < 6; ++f) {
        const int a = f / 2, side = f % 2;
        P.corr[f] = 0.0;
        const int p = c->ax[a].pair;
        if (p == P_EMPTY || p == P_CC || d->value[f] == 0.0) continue;
        const double hb = side == 0 ? h[a][0] : h[a][c->n[a] - 1];
        if (d->bc[f] == BFFT_BC_DIRICHLET)
            P.corr[f] = 2.0 * d->value[f] / (hb * hb);
        else  // ghost centre one mirrored cell away
            P.corr[f] = d->value[f] * hb / (hb * hb);
    }

    // geometry of the split solver's source kernel
    for (int a = 0; a < 3; ++a) {
        c->split.n[a] = c->n[a];
        c->split.h[a] = upload(c, h[a]);
    }
    for (int f = 0; f < 6; ++f) {
        c->split.bc[f] = d->bc[f];
        c->split.value[f] = d->value[f];
    }
    c->part = dalloc<double>(kSplitBlocks);
    c->owned.push_back(c->part);

    const size_t cells = (size_t)c->n[0] * c->n[1] * c->n[2];
    c->w = dalloc<double>(cells);
    c->dh = dalloc<double>(cells);
    if (T.cyclic) c->vv = dalloc<double>(cells);
    check(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    c->ownStream = true;
}

void freeAll(bfft_ctx* c) {
    for (void* p : c->owned) cudaFree(p);
    c->owned.clear();
    cudaFree(c->w);
    cudaFree(c->dh);
    cudaFree(c->vv);
    c->w = c->dh = c->vv = nullptr;
    if (c->ownStream && c->stream) cudaStreamDestroy(c->stream);
    c->stream = nullptr;
}

template <typename F>
int guarded(bfft_ctx* c, F&& f) {
    try {
        return f();
    } catch (const BadArg& e) {
        if (c) c->err = e.msg;
        return e.code;
    } catch (const std::exception& e) {
        if (c) c->err = e.what();
        return BMG_CUDA_ERROR;
    }
}

void transform(bfft_ctx* c, int a, bool forward, const double* in, double* out, const LoadPrep& lp) {
    const AxisPlan& A = c->ax[a];
    const Transform& T = forward ? A.fwd : A.bwd;
    const long tiles = (A.lines.count + A.LB - 1) / A.LB;
    // persistent: as many CTAs as fit at once (three per SM)
    const long grid = std::min<long>(tiles, 3L * c->sms);
    launch_transform(T.kind, T.logM, (unsigned)grid, c->stream, in, out, A.lines, T, lp, tiles, A.adjacent);
    check(cudaGetLastError(), "k_transform");
}

}  // namespace

extern "C" {

int bfft_create(bfft_ctx** out, const bfft_desc* desc) {
    if (!out || !desc) return BMG_BAD_ARG;
    *out = nullptr;
    bfft_ctx* c = new bfft_ctx;
    c->dev = desc->device;
    const int rc = guarded(c, [&] {
        build(c, desc);
        return (int)BMG_OK;
    });
    if (rc != BMG_OK) {
        fprintf(stderr, "bfft_create: %s\n", c->err.c_str());
        freeAll(c);
        delete c;
        return rc;
    }
    *out = c;
    return BMG_OK;
}

void bfft_destroy(bfft_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->dev);
    if (c->stream) cudaStreamSynchronize(c->stream);
    freeAll(c);
    delete c;
}

int bfft_set_stream(bfft_ctx* c, void* stream) {
    if (!c) return BMG_BAD_ARG;
    return guarded(c, [&] {
        check(cudaSetDevice(c->dev), "cudaSetDevice");
        check(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        if (c->ownStream) cudaStreamDestroy(c->stream);
        c->ownStream = false;
        c->stream = static_cast<cudaStream_t>(stream);
        return (int)BMG_OK;
    });
}

int bfft_solve(bfft_ctx* c, const double* b, double* x, const double* x_old, double shift, int flags) {
    if (!c || !b || !x) return BMG_BAD_ARG;
    return guarded(c, [&] {
        check(cudaSetDevice(c->dev), "cudaSetDevice");
        const bool dev = flags & BMG_DEVICE_PTRS;
        const size_t cells = (size_t)c->n[0] * c->n[1] * c->n[2];
        const double* bd = b;
        const double* xo = x_old;
        if (!dev) {
            check(cudaMemcpyAsync(c->w, b, cells * sizeof(double), cudaMemcpyHostToDevice, c->stream), "copy b");
            bd = c->w;
            if (x_old) {
                // the Thomas scratch is free until the tridiagonal step
                check(cudaMemcpyAsync(c->dh, x_old, cells * sizeof(double), cudaMemcpyHostToDevice, c->stream),
                      "copy x_old");
                xo = c->dh;
            }
        }
        Prep P = c->prep;
        P.shift = shift;
        std::vector<int> fwd;
        for (int a : {c->dir1, c->dir2})
            if (c->ax[a].pair != P_EMPTY && !c->ax[a].identity) fwd.push_back(a);
        const LoadPrep none{};
        if (fwd.empty()) {
            const int blocks = (int)std::min<size_t>((cells + kThreads - 1) / kThreads, 148 * 16);
            k_prep<<<blocks, kThreads, 0, c->stream>>>(c->w, bd, shift != 0.0 ? xo : nullptr, P);
            check(cudaGetLastError(), "k_prep");
        }
        for (size_t q = 0; q < fwd.size(); ++q) {
            // the first transform forms the right-hand side as it loads b
            LoadPrep lp{};
            if (q == 0) {
                lp.on = 1;
                lp.axis = fwd[0];
                lp.n1 = c->n[1];
                lp.n2 = c->n[2];
                lp.xo = shift != 0.0 ? xo : nullptr;
                lp.P = P;
            }
            transform(c, fwd[q], true, q == 0 ? bd : c->w, c->w, q == 0 ? lp : none);
        }
        Tri T = c->tri;
        T.shift = shift;
        if (!T.cyclic && (!c->factored || c->factorShift != shift)) {
            const int modes = T.nci * T.nco;
            k_tri_factor<<<(modes + 127) / 128, 128, 0, c->stream>>>(T);
            check(cudaGetLastError(), "k_tri_factor");
            c->factored = true;
            c->factorShift = shift;
        }
        const long lines = c->solveLines.count;
        if (T.cyclic)
            k_tridiag<<<(unsigned)((lines + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(c->w, c->dh, c->vv,
                                                                                              c->solveLines, T);
        else
            k_tri_apply<<<(unsigned)((lines + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(c->w, c->solveLines,
                                                                                                T);
        check(cudaGetLastError(), "k_tridiag");
        // backward in reverse order; the last one writes the device x
        std::vector<int> back;
        for (int a : {c->dir2, c->dir1})
            if (c->ax[a].pair != P_EMPTY && !c->ax[a].identity) back.push_back(a);
        for (size_t q = 0; q < back.size(); ++q) {
            const bool last = q + 1 == back.size();
            transform(c, back[q], false, c->w, last && dev ? x : c->w, none);
        }
        if (dev && back.empty())
            check(cudaMemcpyAsync(x, c->w, cells * sizeof(double), cudaMemcpyDeviceToDevice, c->stream), "copy x");
        if (!dev) {
            check(cudaMemcpyAsync(x, c->w, cells * sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy x");
            check(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        }
        return (int)BMG_OK;
    });
}

int bfft_split_lambda0(bfft_ctx* c, const double* lam0, const double* lam1, const double* lam2, double* lambda0) {
    if (!c || !lam0 || !lam1 || !lam2 || !lambda0) return BMG_BAD_ARG;
    return guarded(c, [&] {
        check(cudaSetDevice(c->dev), "cudaSetDevice");
        const long n0 = c->n[0], n1 = c->n[1], n2 = c->n[2];
        k_max3<<<kSplitBlocks, kThreads, 0, c->stream>>>(lam0, (n0 + 1) * n1 * n2, lam1, n0 * (n1 + 1) * n2, lam2,
                                                        n0 * n1 * (n2 + 1), c->part);
        k_max_final<<<1, kThreads, 0, c->stream>>>(c->part, kSplitBlocks);
        check(cudaGetLastError(), "k_max3");
        check(cudaMemcpyAsync(lambda0, c->part, sizeof(double), cudaMemcpyDeviceToHost, c->stream), "copy lambda0");
        check(cudaStreamSynchronize(c->stream), "cudaStreamSynchronize");
        if (!(*lambda0 > 0.0)) throw BadArg{BMG_BAD_ARG, "face coefficients must be positive"};
        return (int)BMG_OK;
    });
}

int bfft_split_source(bfft_ctx* c, const double* x, const double* b, const double* lam0, const double* lam1,
                      const double* lam2, double lambda0, double* bhat) {
    if (!c || !x || !b || !lam0 || !lam1 || !lam2 || !bhat || !(lambda0 > 0.0)) return BMG_BAD_ARG;
    return guarded(c, [&] {
        check(cudaSetDevice(c->dev), "cudaSetDevice");
        const dim3 grid((unsigned)std::min((c->n[2] + 127) / 128, 8), (unsigned)c->n[1], (unsigned)c->n[0]);
        k_split_source<<<grid, 128, 0, c->stream>>>(x, b, lam0, lam1, lam2, lambda0, bhat, c->split);
        check(cudaGetLastError(), "k_split_source");
        return (int)BMG_OK;
    });
}

int bfft_axpby(bfft_ctx* c, double a, const double* x, double cc, const double* y, double* out) {
    if (!c || !x || !y || !out) return BMG_BAD_ARG;
    return guarded(c, [&] {
        check(cudaSetDevice(c->dev), "cudaSetDevice");
        const long n = (long)c->n[0] * c->n[1] * c->n[2];
        k_axpby<<<4 * c->sms, kThreads, 0, c->stream>>>(a, x, cc, y, out, n);
        check(cudaGetLastError(), "k_axpby");
        return (int)BMG_OK;
    });
}

int bfft_solve_direction(const bfft_ctx* c) { return c ? c->s : -1; }

const char* bfft_last_error(const bfft_ctx* c) { return c ? c->err.c_str() : ""; }

}  // extern "C"
