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
constexpr int kTileComplex = 2048;  // complex values of a transform tile (32 KB)
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
    const double2* pre;   // n entries, nullptr: 1
    const double2* post;  // n entries, nullptr: 1
    const double2* tw;    // M/2 entries: exp(-2 pi i j / M)
};

struct Tri {
    int ns, cyclic;
    double shift;
    double s0;            // first diagonal entry of a pinned (singular) mode
    const double* A;      // D_k = ((e - A_k) - B_k)
    const double* B;
    const double* DU;
    const double* DL;
    const double* ev1;    // eigenvalue / h^2 of the first transform direction
    const double* ev2;
    int dir1_inner;       // the first transform direction is the inner line coordinate
};

struct Prep {
    int n0, n1, n2;
    double shift, scale;
    double corr[6];       // face terms subtracted on the boundary cells of each face
};

__device__ __forceinline__ long line_base(const Lines& L, long l) {
    return (l / L.inner) * L.outer_stride + (l % L.inner) * L.inner_stride;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// w_out(line) = transform of w_in(line) for LB lines per CTA (in place allowed:
// a CTA reads all its lines before it writes)
__global__ void __launch_bounds__(kThreads) k_transform(const double* __restrict__ in, double* __restrict__ out,
                                                        Lines L, Transform T, int LB) {
    extern __shared__ double2 sm[];
    const int M = T.M, n = L.n;
    double2* a = sm;                        // [LB][M]
    double2* tw = a + (long)LB * M;         // [M/2]
    long* base = reinterpret_cast<long*>(tw + M / 2);  // [LB]
    double* raw = reinterpret_cast<double*>(base + LB); // [LB][n] (HC2R input)
    const int tid = threadIdx.x;
    const long l0 = (long)blockIdx.x * LB;
    const int lines = (int)min((long)LB, L.count - l0);

    for (int q = tid; q < M / 2; q += kThreads) tw[q] = T.tw[q];
    for (int t = tid; t < LB; t += kThreads) base[t] = t < lines ? line_base(L, l0 + t) : 0;
    __syncthreads();

    const int shift = 32 - T.logM;
    auto brev = [&](int p) { return T.logM ? (int)(__brev((unsigned)p) >> shift) : 0; };
    // element q of the tile: line-fast order along strided axes
    auto split = [&](int q, int& t, int& p) {
        if (L.line_fast) {
            t = q % LB;
            p = q / LB;
        } else {
            t = q / n;
            p = q % n;
        }
    };

    if (T.mode == M_HC2R) {
        for (int q = tid; q < LB * n; q += kThreads) {
            int t, p;
            split(q, t, p);
            raw[t * n + p] = t < lines ? in[base[t] + p * L.stride] : 0.0;
        }
        __syncthreads();
        // conj(Y_k) of the halfcomplex spectrum, bit-reversed
        for (int q = tid; q < LB * M; q += kThreads) {
            const int t = q / M, k = q % M;
            const double* h = raw + t * n;
            double re, im;
            if (k == 0) {
                re = h[0];
                im = 0.0;
            } else if (2 * k < n) {
                re = h[k];
                im = -h[n - k];
            } else if (2 * k == n) {
                re = h[k];
                im = 0.0;
            } else {
                re = h[n - k];
                im = h[k];
            }
            a[t * M + brev(k)] = make_double2(re, im);
        }
    } else {
        for (int q = tid; q < LB * n; q += kThreads) {
            int t, p;
            split(q, t, p);
            const double x = t < lines ? in[base[t] + p * L.stride] : 0.0;
            const double2 c = T.pre ? T.pre[p] : make_double2(1.0, 0.0);
            a[t * M + brev(p)] = make_double2(c.x * x, c.y * x);
        }
        if (M > n)  // zero padding
            for (int q = tid; q < LB * (M - n); q += kThreads) {
                const int t = q / (M - n), p = n + q % (M - n);
                a[t * M + brev(p)] = make_double2(0.0, 0.0);
            }
    }
    __syncthreads();

    // radix-2 decimation in time, natural-order output
    for (int h = 1, ts = M / 2; h < M; h <<= 1, ts >>= 1) {
        for (int q = tid; q < LB * (M / 2); q += kThreads) {
            const int t = q / (M / 2), b = q % (M / 2);
            const int pos = b & (h - 1);
            const int i0 = t * M + ((b - pos) << 1) + pos, i1 = i0 + h;
            const double2 u = a[i0];
            const double2 v = cmul(a[i1], tw[pos * ts]);
            a[i0] = make_double2(u.x + v.x, u.y + v.y);
            a[i1] = make_double2(u.x - v.x, u.y - v.y);
        }
        __syncthreads();
    }

    for (int q = tid; q < LB * n; q += kThreads) {
        int t, k;
        split(q, t, k);
        if (t >= lines) continue;
        const double2* z = a + t * M;
        double y;
        if (T.mode == M_R2HC) {
            y = 2 * k <= n ? z[k].x : z[n - k].y;
        } else if (T.mode == M_HC2R) {
            y = z[k].x;
        } else {
            const double2 c = T.post ? cmul(T.post[k], z[k]) : z[k];
            y = T.mode == M_RE ? c.x : -c.y;
        }
        out[base[t] + k * L.stride] = y;
    }
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
    const long ci = l % L.inner, co = l / L.inner;
    const long c1 = T.dir1_inner ? ci : co, c2 = T.dir1_inner ? co : ci;
    const double e1 = T.ev1[c1], e2 = T.ev2[c2];
    const double e = e1 + e2;
    const bool singular = e1 == 0.0 && e2 == 0.0;
    auto diag = [&](int k) {
        const double d = (k == 0 && singular) ? T.s0 : (e - T.A[k]) - T.B[k];
        return d - T.shift;
    };
    if (!T.cyclic) {
        double Dp = diag(0);
        double fp = w[base];
        dh[base] = Dp;
#pragma unroll 4
        for (int k = 1; k < ns; ++k) {
            const long c = base + k * st;
            const double m = T.DL[k] / Dp;
            const double D = diag(k) - m * T.DU[k - 1];
            const double f = w[c] - m * fp;
            w[c] = f;
            dh[c] = D;
            Dp = D;
            fp = f;
        }
        double p = fp / Dp;
        w[base + (ns - 1) * st] = p;
#pragma unroll 4
        for (int k = ns - 2; k >= 0; --k) {
            const long c = base + k * st;
            p = (w[c] - T.DU[k] * p) / dh[c];
            w[c] = p;
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
    size_t smem = 0;
};

}  // namespace bfft

using namespace bfft;

struct bfft_ctx {
    int dev = 0;
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
    const bool cc = A.pair == P_CC;
    const int M = cc ? N : 2 * N;
    std::vector<double2> tw(std::max(M / 2, 1));
    for (int j = 0; j < M / 2; ++j) tw[j] = expi(-2.0L * pi * j / M);
    const double2* twd = upload(c, tw);
    auto table = [&](auto f) {
        std::vector<double2> t(N);
        for (int q = 0; q < N; ++q) t[q] = f(q);
        return upload(c, t);
    };
    Transform f{M, log2i(M), M_RE, nullptr, nullptr, twd};
    Transform b = f;
    switch (A.pair) {
        case P_CC:
            f.mode = M_R2HC;
            b.mode = M_HC2R;
            break;
        case P_NN:  // REDFT10 / REDFT01
            f.post = table([&](int k) { return expi(-pi * k / (2.0L * N), 2.0L); });
            b.pre = table([&](int q) { return expi(-pi * q / (2.0L * N), q == 0 ? 1.0L : 2.0L); });
            break;
        case P_DD:  // RODFT10 / RODFT01
            f.mode = b.mode = M_NEG_IM;
            f.pre = table([&](int q) { return expi(-pi * q / N); });
            f.post = table([&](int k) { return expi(-pi * (k + 1) / (2.0L * N), 2.0L); });
            b.pre = table([&](int q) { return expi(-pi * q / (2.0L * N), q == N - 1 ? 1.0L : 2.0L); });
            b.post = table([&](int k) { return expi(-pi * (2 * k + 1) / (2.0L * N)); });
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
    A.LB = std::max(1, std::min(32, kTileComplex / M));
    A.smem = sizeof(double2) * ((size_t)A.LB * M + std::max(M / 2, 1)) + sizeof(long) * A.LB +
             (cc ? sizeof(double) * (size_t)A.LB * N : 0);
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
    size_t smem = 0;
    for (int a : {c->dir1, c->dir2}) {
        c->ax[a].lines = linesAlong(c->n, a);
        planTransforms(c, a);
        smem = std::max(smem, c->ax[a].smem);
    }
    check(cudaFuncSetAttribute(k_transform, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
          "cudaFuncSetAttribute");

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
    // a pinned mode exists only where both transform directions can have a
    // zero eigenvalue; elsewhere s0 is never used
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
    T.A = upload(c, A);
    T.B = upload(c, B);
    T.DU = upload(c, DU);
    T.DL = upload(c, DL);
    T.ev1 = upload(c, ev(c->dir1));
    T.ev2 = upload(c, ev(c->dir2));
    c->solveLines = linesAlong(c->n, s);
    // the lines' inner coordinate: k for s = 0 and 1, j for s = 2
    const int innerAxis = s == 2 ? 1 : 2;
    T.dir1_inner = c->dir1 == innerAxis;

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

void transform(bfft_ctx* c, int a, bool forward, const double* in, double* out) {
    const AxisPlan& A = c->ax[a];
    const Transform& T = forward ? A.fwd : A.bwd;
    const long grid = (A.lines.count + A.LB - 1) / A.LB;
    k_transform<<<(unsigned)grid, kThreads, A.smem, c->stream>>>(in, out, A.lines, T, A.LB);
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
        const int blocks = (int)std::min<size_t>((cells + kThreads - 1) / kThreads, 148 * 16);
        k_prep<<<blocks, kThreads, 0, c->stream>>>(c->w, bd, shift != 0.0 ? xo : nullptr, P);
        check(cudaGetLastError(), "k_prep");
        for (int a : {c->dir1, c->dir2})
            if (c->ax[a].pair != P_EMPTY) transform(c, a, true, c->w, c->w);
        Tri T = c->tri;
        T.shift = shift;
        const long lines = c->solveLines.count;
        k_tridiag<<<(unsigned)((lines + kThreads - 1) / kThreads), kThreads, 0, c->stream>>>(c->w, c->dh, c->vv,
                                                                                          c->solveLines, T);
        check(cudaGetLastError(), "k_tridiag");
        // backward in reverse order; the last one writes the device x
        std::vector<int> back;
        for (int a : {c->dir2, c->dir1})
            if (c->ax[a].pair != P_EMPTY) back.push_back(a);
        for (size_t q = 0; q < back.size(); ++q) {
            const bool last = q + 1 == back.size();
            transform(c, back[q], false, c->w, last && dev ? x : c->w);
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

int bfft_solve_direction(const bfft_ctx* c) { return c ? c->s : -1; }

const char* bfft_last_error(const bfft_ctx* c) { return c ? c->err.c_str() : ""; }

}  // extern "C"
