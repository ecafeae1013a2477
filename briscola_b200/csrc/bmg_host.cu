// bmg_host.cu -- host side of the B200 multigrid solver: level hierarchy of
// one or more bricks, geometry tables, inter-brick ghost lists, the V/W/F
// cycle driver, mixed-precision refinement, the whole-solve CUDA graph, the
// launch-shape autotuner and the C ABI declared in include/bmg.h.
//
// Reference behaviour followed (paths relative to the Briscola tree, with
// FV = src/briscolaFiniteVolume):
//   level sizes          src/briscolaCore/include/utils.H:1152-1170, src/briscolaMesh/mesh/mesh.C:19-53
//   coarse points/ghosts src/briscolaMesh/level/levelPoints.C:151-155,198-236,326-400
//   operator             FV/schemes/laplacianSchemes/linearGaussLaplacianScheme/linearGaussLaplacianScheme.C:59-94
//                        FV/fvMeshMetrics.C:848-893, NeumannBoundaryCondition.C:19-56
//   cycle                FV/solvers/MG/MG.C:19-130, MG.H:106-124
//   loop / convergence   FV/solvers/MG/MG.C:132-254, FV/solvers/solver/solver.C:13-95
//   pin + coarse solve   FV/solvers/solver/solver.C:201-231, FV/solvers/externalSolvers/APLU/APLU.C:26-128
//   transfers            linearRestrictionScheme.C:15-187, linearProlongationScheme.C:12-147,
//                        areaWeightedFaceRestrictionScheme.C:19-57
//   brick contacts       FV/boundaryConditions/parallelBoundaryCondition/parallelBoundaryCondition.C:84-174

#include "../../include/bmg.h"
#include "bmg_internal.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

using namespace bmg;

namespace {

struct Axis {
    std::vector<double> pts;  // n+3 entries, entry q+1 = point q (q = -1..n+1)
    std::vector<double> cc;   // n+2 entries, entry i+1 = centre of cell i (i = -1..n)
    std::vector<double> h;    // n+2 entries, same indexing
};

// one brick on one level
struct HostBrick {
    int n[3] = {0, 0, 0};
    int R[3] = {1, 1, 1};     // ratio to the parent level
    int origin[3] = {0, 0, 0};  // cell offset in the level's global lattice
    Axis ax[3];
    bool open[6] = {false, false, false, false, false, false};  // periodic or touching another brick
    // Dirichlet wall faces, and the Dirichlet value or Neumann gradient of
    // each wall face (level 0; coarse levels keep the Dirichlet flags)
    int dirichlet[6] = {0, 0, 0, 0, 0, 0};
    double dval[6] = {0, 0, 0, 0, 0, 0};
    int nbr[6] = {-1, -1, -1, -1, -1, -1};  // a brick touching the face (its ghost points come from it)
    // orientation of the caller's arrays: local axis d runs along axis
    // tax[d] of this (global) frame, reversed when tfl[d]
    int tax[3] = {0, 1, 2};
    int tfl[3] = {0, 0, 0};
    long si = 0, sj = 0;      // strides
    long off = 0;             // slab offset of the brick's block
    long base = 0;            // slab index of interior cell (0,0,0)
    long cells = 0;           // size of the brick's block
    long cbase = 0;           // offset in compact arrays
    TabOff to{};              // offsets into the level's table
    int cpar = 0;
    std::vector<double> lam_user[3];  // restricted user lambda, block-local indexing
    long ncell() const { return (long)n[0] * n[1] * n[2]; }
    long at(int i, int j, int k) const { return base + (long)i * si + (long)j * sj + k; }
    long loc(int i, int j, int k) const { return at(i, j, k) - off; }
};

struct HostLevel {
    std::vector<HostBrick> br;
    // multi-brick lattice box: lowest cell lo, extent ext; axes with wrap
    // set are periodic (a brick face on the box boundary meets the bricks
    // on the opposite boundary), period = their length in coordinates
    int lo[3] = {0, 0, 0};
    int ext[3] = {0, 0, 0};
    int wrap[3] = {0, 0, 0};
    double period[3] = {0.0, 0.0, 0.0};
    long cells = 0;   // slab size
    long ncell = 0;   // interior cells of all bricks
    int planes = 0;   // sum of n0
    std::vector<double> tab;  // 1-D tables of all bricks
    std::vector<double> lam_host[3];  // face lambda of the slab (variable coefficient)
    double* x64 = nullptr;
    double* b64 = nullptr;
    float* x32 = nullptr;
    float* b32 = nullptr;
    double* tab64 = nullptr;
    float* tab32 = nullptr;
    double* lam64[3] = {nullptr, nullptr, nullptr};
    float* lam32[3] = {nullptr, nullptr, nullptr};
    double* jtmp64 = nullptr;
    float* jtmp32 = nullptr;
    double* x64b = nullptr;  // second x buffers: fused smoothing writes here, then swaps
    float* x32b = nullptr;
    bool fusedOK = false;    // single brick large enough for the fused smoother
    bool ks = false;         // parity-split rows (bmg_internal.h)
    // per precision (0: FP64, 1: FP32), picked by autotune():
    int fusedS[2] = {kFusedMaxStages, kFusedMaxStages};  // colour stages per fused launch
    int fusedTi[2] = {64, 64};                             // planes per CTA chunk
    // ghost refresh between bricks: slab[gdst[q]] = slab[gsrc[q]]
    int* gdst = nullptr;
    int* gsrc = nullptr;
    long nghost = 0;
};

struct BrickTransfer {
    double* ratio64 = nullptr;
    float* ratio32 = nullptr;
    int* pidx = nullptr;
    double* pw64 = nullptr;
    float* pw32 = nullptr;
    int R[3] = {1, 1, 1};
};

struct CudaError {
    std::string msg;
};

#define BMG_CUDA(call)                                                                     \
    do {                                                                                   \
        cudaError_t e__ = (call);                                                          \
        if (e__ != cudaSuccess)                                                            \
            throw CudaError{std::string(#call) + ": " + cudaGetErrorString(e__)};          \
    } while (0)

struct BadArg {
    int code;
    std::string msg;
};

}  // namespace

struct bmg_ctx {
    bmg_options opt{};
    int periodic[3] = {0, 0, 0};  // single brick only
    bool singular = true;         // no Dirichlet face (linearSystem.H:227-230)
    bool multi = false;           // more than one brick
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<HostLevel> lv;
    std::vector<std::vector<BrickTransfer>> tr;  // [level][brick]
    int lc = 0;  // coarse solve level
    int tail = -1;  // first level of the single-CTA coarse cycle, -1: none
    double* ainv = nullptr;
    int* cidx = nullptr;
    int ncoarse = 0;
    bool userLambda = false;  // a variable coefficient was given
    bool variable = false;    // kernels read face lambdas (user lambda or brick contacts)
    bool conforming = true;   // every brick face in contact is wholly in contact (no contact mask)
    double* partials = nullptr;
    SolveState* st = nullptr;
    SolveState* st_host = nullptr;
    double* stage_b = nullptr;
    double* stage_x = nullptr;
    // flexible CG outer loop (level-0 slabs): solution, scaled right-hand
    // side, residual, direction p and q = A'p
    double* fx = nullptr;
    double* fb = nullptr;
    double* fr = nullptr;
    double* fp = nullptr;
    double* fq = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    long launches = 0;  // kernels launched by the current solve
    std::vector<int> visits;
    // whole-solve CUDA graph (captured on the first solve, reused)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    cudaStream_t capStream = nullptr;  // private stream used only for capture
    // a level solver in place of the FP32 cycle's recursion below hookLevel
    // (bmg_set_level_solver), with its right-hand side and result arrays
    // the next FP32 cycle starts from z = 0 on a parity-split level 0: its
    // first colour pass writes the whole level (no memset before it)
    bool zeroFirst0 = false;
    int hookLevel = -1;
    int hookMode = BMG_LEVEL_REPLACE;
    bmg_level_solver hook = nullptr;
    void* hookUser = nullptr;
    float* hookRhs = nullptr;
    float* hookX = nullptr;
    bool graphZero = false;
    long launchesInitPost = 0, launchesBody = 0;
};

namespace {

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
// levelPoints.C:198-236 (walls: project by one spacing) and :326-400
// (periodic: the opposite side's spacing).  A face touching another brick
// takes the neighbour's point (glo / ghi, NaN where there is none), as the
// reference's processor-boundary ghost points do.
void finishAxis(Axis& a, int n, bool periodic, double glo, double ghi) {
    std::vector<double>& p = a.pts;
    if (periodic) {
        p[0] = p[1] - (p[n + 1] - p[n]);
        p[n + 2] = p[n + 1] + (p[2] - p[1]);
    } else {
        p[0] = std::isnan(glo) ? p[1] + (p[1] - p[2]) : glo;
        p[n + 2] = std::isnan(ghi) ? p[n + 1] + (p[n + 1] - p[n]) : ghi;
    }
    a.cc.assign(n + 2, 0.0);
    a.h.assign(n + 2, 0.0);
    for (int i = -1; i <= n; ++i) {
        a.cc[i + 1] = 0.5 * (p[i + 1] + p[i + 2]);
        a.h[i + 1] = p[i + 2] - p[i + 1];
    }
}

// storage position of interior k in a parity-split row of n2 cells
// (kpos_split of bmg_stencil.cuh): the even k first, then the odd k
inline int kposSplit(int k, int n2) { return (k & 1) * (n2 / 2) + (k >> 1); }

// a slab field in natural row order -> parity-split order (interior k of
// every row of the brick, ghost rows included; the k ghosts stay)
void splitRows(const HostBrick& B, std::vector<double>& f) {
    std::vector<double> tmp(B.n[2]);
    for (int i = -1; i <= B.n[0]; ++i)
        for (int j = -1; j <= B.n[1]; ++j) {
            const long r = B.base + (long)i * B.si + (long)j * B.sj;
            for (int k = 0; k < B.n[2]; ++k) tmp[kposSplit(k, B.n[2])] = f[r + k];
            for (int k = 0; k < B.n[2]; ++k) f[r + k] = tmp[k];
        }
}

// Rows of pitch p2 = round_up(n2 + 5, 4) with interior k = 0 at offset 4:
// rows and interiors start on 16-byte (FP32) / 32-byte (FP64) boundaries so
// pairs of k-neighbours load as one vector; the k ghosts sit at offsets 3
// and n2 + 4.  Bricks follow one another in the slab.
void layout(HostLevel& L) {
    long off = 0, coff = 0;
    int planes = 0;
    for (auto& B : L.br) {
        const long p2 = ((B.n[2] + 5) + 3) / 4 * 4, p1 = B.n[1] + 2, p0 = B.n[0] + 2;
        B.sj = p2;
        B.si = p1 * p2;
        B.off = off;
        B.base = off + B.si + B.sj + 4;
        B.cells = p0 * p1 * p2;
        B.cbase = coff;
        B.cpar = (B.origin[0] + B.origin[1] + B.origin[2]) & 1;
        off += B.cells;
        coff += B.ncell();
        planes += B.n[0];
    }
    L.cells = off;
    L.ncell = coff;
    L.planes = planes;
}

// row-scaled couplings (A'/V): lower neighbour delta(i)/h(i), upper
// delta(i+1)/h(i); zero across a Neumann wall face (NeumannBoundaryCondition
// .C:19-56), twice the ghost coupling across a Dirichlet one, whose ghost
// cells stay zero: A_c -= A_f after A_c = -(sum of all faces)
// (DirichletBoundaryCondition.C:19-51).  Faces touching another brick keep
// their coupling and get their wall parts zeroed through the face lambdas.
void buildTables(HostLevel& L) {
    int off = 0;
    L.tab.clear();
    // every sub-table starts on a multiple of 4 entries, so the colour pass
    // can read 4 consecutive k couplings as one vector
    auto next = [](int o, int n) { return (o + n + 3) / 4 * 4; };
    for (auto& B : L.br) {
        TabOff& to = B.to;
        for (int d = 0; d < 3; ++d) {
            to.wl[d] = off;
            off = next(off, B.n[d]);
            to.wh[d] = off;
            off = next(off, B.n[d]);
            to.h[d] = off;
            off = next(off, B.n[d]);
        }
        to.kwl = to.kwh = to.ksz = -1;
        if (L.ks) {
            to.kwl = off;
            off = next(off, B.n[2]);
            to.kwh = off;
            off = next(off, B.n[2]);
            to.ksz = off;
            off = next(off, B.n[2]);
        }
        to.total = off;
        L.tab.resize(off, 0.0);
        for (int d = 0; d < 3; ++d) {
            const Axis& a = B.ax[d];
            const int n = B.n[d];
            for (int i = 0; i < n; ++i) {
                const double hi = a.h[i + 1];
                const double dlo = 1.0 / std::fabs(a.cc[i + 1] - a.cc[i]);
                const double dhi = 1.0 / std::fabs(a.cc[i + 2] - a.cc[i + 1]);
                double wl = dlo / hi, wh = dhi / hi;
                if (!B.open[2 * d] && i == 0) wl = B.dirichlet[2 * d] ? 2.0 * wl : 0.0;
                if (!B.open[2 * d + 1] && i == n - 1) wh = B.dirichlet[2 * d + 1] ? 2.0 * wh : 0.0;
                L.tab[to.wl[d] + i] = wl;
                L.tab[to.wh[d] + i] = wh;
                L.tab[to.h[d] + i] = hi;
            }
        }
        if (L.ks)  // the k couplings once more, in the rows' storage order
            for (int k = 0; k < B.n[2]; ++k) {
                L.tab[to.kwl + kposSplit(k, B.n[2])] = L.tab[to.wl[2] + k];
                L.tab[to.kwh + kposSplit(k, B.n[2])] = L.tab[to.wh[2] + k];
                L.tab[to.ksz + kposSplit(k, B.n[2])] = L.tab[to.h[2] + k];
            }
    }
}

template <typename T>
Bricks<T> bricks(const bmg_ctx* c, int l) {
    const HostLevel& H = c->lv[l];
    Bricks<T> B{};
    B.nb = (int)H.br.size();
    int z = 0;
    for (int b = 0; b < B.nb; ++b) {
        const HostBrick& K = H.br[b];
        LevelView<T>& v = B.v[b];
        v.n0 = K.n[0];
        v.n1 = K.n[1];
        v.n2 = K.n[2];
        v.si = K.si;
        v.sj = K.sj;
        v.base = K.base;
        v.cells = H.cells;
        // compact (caller) index of cell (i,j,k) of this frame: the brick's
        // own k-fastest order, cbase + i*cs[0] + j*cs[1] + k*cs[2]
        {
            long ls[3];
            ls[2] = 1;
            ls[1] = K.n[K.tax[2]];
            ls[0] = ls[1] * K.n[K.tax[1]];
            long off = 0;
            for (int d = 0; d < 3; ++d) {
                v.cs[K.tax[d]] = (int)(K.tfl[d] ? -ls[d] : ls[d]);
                if (K.tfl[d]) off += (long)(K.n[K.tax[d]] - 1) * ls[d];
            }
            v.cbase = K.cbase + off;
        }
        v.to = K.to;
        v.tab64 = H.tab64;
        if constexpr (sizeof(T) == 8) {
            v.x = reinterpret_cast<T*>(H.x64);
            v.b = reinterpret_cast<T*>(H.b64);
            v.tab = reinterpret_cast<const T*>(H.tab64);
            for (int d = 0; d < 3; ++d) (&v.lam0)[d] = reinterpret_cast<const T*>(H.lam64[d]);
        } else {
            v.x = reinterpret_cast<T*>(H.x32);
            v.b = reinterpret_cast<T*>(H.b32);
            v.tab = reinterpret_cast<const T*>(H.tab32);
            for (int d = 0; d < 3; ++d) (&v.lam0)[d] = reinterpret_cast<const T*>(H.lam32[d]);
        }
        v.per0 = c->periodic[0];
        v.per1 = c->periodic[1];
        v.per2 = c->periodic[2];
        v.cpar = K.cpar;
        v.kh = H.ks ? K.n[2] / 2 : 0;
        // a smoothed coarse level of a singular system keeps global cell 0
        // (brick 0's first cell) at zero
        v.pin = l == c->lc && b == 0 && c->singular && c->opt.coarse_mode == BMG_COARSE_SMOOTH;
        B.z0[b] = z;
        z += K.n[0];
        B.max1 = std::max(B.max1, K.n[1]);
        B.max2 = std::max(B.max2, K.n[2]);
    }
    B.z0[B.nb] = z;
    return B;
}

// the face values of the level-0 bricks (Dirichlet values, Neumann gradients)
Walls walls(const bmg_ctx* c) {
    Walls W{};
    const HostLevel& L0 = c->lv[0];
    for (size_t b = 0; b < L0.br.size(); ++b) {
        const HostBrick& K = L0.br[b];
        for (int f = 0; f < 6; ++f) {
            W.mask[b] |= K.dirichlet[f] << f;
            W.nmask[b] |= (!K.dirichlet[f] && K.dval[f] != 0.0) << f;
            W.g[b][f] = K.dval[f];
        }
    }
    W.ybar = c->st ? &c->st->ybar : nullptr;
    return W;
}

TransferSet ttabs(const bmg_ctx* c, int l) {
    TransferSet s{};
    for (size_t b = 0; b < c->tr[l].size(); ++b) {
        const BrickTransfer& t = c->tr[l][b];
        TransferTabs& u = s.t[b];
        u.ratio64 = t.ratio64;
        u.ratio32 = t.ratio32;
        u.pidx = t.pidx;
        u.pw64 = t.pw64;
        u.pw32 = t.pw32;
        u.R0 = t.R[0];
        u.R1 = t.R[1];
        u.R2 = t.R[2];
    }
    return s;
}

template <typename T>
T* dalloc(size_t n) {
    void* p = nullptr;
    BMG_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    BMG_CUDA(cudaMemset(p, 0, std::max<size_t>(n, 1) * sizeof(T)));
    return static_cast<T*>(p);
}

template <typename T>
void upload(T* d, const std::vector<T>& h) {
    BMG_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice));
}

std::vector<float> to_f32(const std::vector<double>& v) {
    std::vector<float> f(v.size());
    for (size_t i = 0; i < v.size(); ++i) f[i] = (float)v[i];
    return f;
}

// Gauss-Jordan inverse with partial pivoting, FP64
bool invert(std::vector<double>& M, int n, std::vector<double>& inv) {
    inv.assign((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i) inv[(size_t)i * n + i] = 1.0;
    for (int k = 0; k < n; ++k) {
        int p = k;
        double best = std::fabs(M[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i)
            if (std::fabs(M[(size_t)i * n + k]) > best) {
                best = std::fabs(M[(size_t)i * n + k]);
                p = i;
            }
        if (best == 0.0) return false;
        if (p != k)
            for (int j = 0; j < n; ++j) {
                std::swap(M[(size_t)k * n + j], M[(size_t)p * n + j]);
                std::swap(inv[(size_t)k * n + j], inv[(size_t)p * n + j]);
            }
        const double d = M[(size_t)k * n + k];
        for (int j = 0; j < n; ++j) {
            M[(size_t)k * n + j] /= d;
            inv[(size_t)k * n + j] /= d;
        }
        for (int i = 0; i < n; ++i) {
            if (i == k) continue;
            const double f = M[(size_t)i * n + k];
            if (f == 0.0) continue;
            for (int j = 0; j < n; ++j) {
                M[(size_t)i * n + j] -= f * M[(size_t)k * n + j];
                inv[(size_t)i * n + j] -= f * inv[(size_t)k * n + j];
            }
        }
    }
    return true;
}

// brick of a level containing global lattice cell g (wrapped around the
// box on periodic axes), with the local cell
int findBrick(const HostLevel& L, const int g0[3], int loc[3]) {
    int g[3];
    for (int d = 0; d < 3; ++d)
        g[d] = L.wrap[d] ? L.lo[d] + (((g0[d] - L.lo[d]) % L.ext[d]) + L.ext[d]) % L.ext[d] : g0[d];
    for (size_t b = 0; b < L.br.size(); ++b) {
        const HostBrick& B = L.br[b];
        bool in = true;
        for (int d = 0; d < 3; ++d) {
            loc[d] = g[d] - B.origin[d];
            in = in && loc[d] >= 0 && loc[d] < B.n[d];
        }
        if (in) return (int)b;
    }
    return -1;
}

// coupling of interior cell (b; i,j,k) through stencil slot s (0..5: axis 0
// lower/upper, axis 1, axis 2), as the kernels form it
double couplingOf(const bmg_ctx* c, const HostLevel& L, int b, int i, int j, int k, int s) {
    const HostBrick& B = L.br[b];
    const int d = s / 2;
    const bool up = s % 2;
    const int ijk[3] = {i, j, k};
    double w = L.tab[(up ? B.to.wh[d] : B.to.wl[d]) + ijk[d]];
    if (c->variable) {
        long fc = B.at(i, j, k);
        if (up) fc += d == 0 ? B.si : d == 1 ? B.sj : 1;
        w *= L.lam_host[d][fc];
    }
    return w;
}

// Dense row-scaled operator of the coarse solve level with, for a singular
// system, the pin of solver.C:201-231 (row of the first cell = identity,
// every coupling to it removed, periodic images included), inverted once
// per matrix.
// Unknowns: bricks one after another, k fastest.
void buildCoarseInverse(bmg_ctx* c) {
    const HostLevel& L = c->lv[c->lc];
    const int n = (int)L.ncell;
    std::vector<double> M((size_t)n * n, 0.0);
    std::vector<int> cidx(n);
    for (int b = 0; b < (int)L.br.size(); ++b) {
        const HostBrick& B = L.br[b];
        for (int i = 0; i < B.n[0]; ++i)
            for (int j = 0; j < B.n[1]; ++j)
                for (int k = 0; k < B.n[2]; ++k) {
                    const long row = B.cbase + ((long)i * B.n[1] + j) * B.n[2] + k;
                    cidx[row] = (int)B.at(i, j, k);
                    double diag = 0.0;
                    for (int s = 0; s < 6; ++s) {
                        const double w = couplingOf(c, L, b, i, j, k, s);
                        if (w == 0.0) continue;
                        const int d = s / 2;
                        int nbl[3] = {i, j, k};
                        nbl[d] += (s % 2) ? 1 : -1;
                        long col;
                        if (nbl[d] >= 0 && nbl[d] < B.n[d]) {
                            col = B.cbase + ((long)nbl[0] * B.n[1] + nbl[1]) * B.n[2] + nbl[2];
                        } else if (c->periodic[d]) {
                            nbl[d] = (nbl[d] + B.n[d]) % B.n[d];
                            col = B.cbase + ((long)nbl[0] * B.n[1] + nbl[1]) * B.n[2] + nbl[2];
                        } else {
                            const int g[3] = {B.origin[0] + nbl[0], B.origin[1] + nbl[1], B.origin[2] + nbl[2]};
                            int loc[3];
                            const int nb = findBrick(L, g, loc);
                            if (nb < 0) {
                                // a Dirichlet wall: eliminated coupling, zero ghost
                                diag -= w;
                                continue;
                            }
                            const HostBrick& N = L.br[nb];
                            col = N.cbase + ((long)loc[0] * N.n[1] + loc[1]) * N.n[2] + loc[2];
                        }
                        diag -= w;
                        M[(size_t)row * n + col] += w;
                    }
                    M[(size_t)row * n + row] += diag;
                }
    }
    if (c->singular) {
        for (int j = 0; j < n; ++j) M[j] = j == 0 ? 1.0 : 0.0;
        for (int r = 1; r < n; ++r) M[(size_t)r * n] = 0.0;
    }
    std::vector<double> inv;
    if (!invert(M, n, inv)) throw BadArg{BMG_BAD_ARG, "coarse level matrix is singular"};
    // MG.C:37-40: the pinned cell's right-hand side is zero
    if (c->singular)
        for (int r = 0; r < n; ++r) inv[(size_t)r * n] = 0.0;
    if (!c->ainv || c->ncoarse != n) {
        if (c->ainv) cudaFree(c->ainv);
        if (c->cidx) cudaFree(c->cidx);
        c->ainv = dalloc<double>((size_t)n * n);
        c->cidx = dalloc<int>(n);
    }
    c->ncoarse = n;
    upload(c->ainv, inv);
    upload(c->cidx, cidx);
}

// the dense inverse exists for coarse levels of at most 4096 cells (the
// direct coarse solve, and the building block of either coarse mode)
void refreshCoarseInverse(bmg_ctx* c) {
    if (c->lv[c->lc].ncell <= 4096)
        buildCoarseInverse(c);
    else
        c->ncoarse = 0;
}

void destroyGraph(bmg_ctx* c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->gexec = nullptr;
    c->graph = nullptr;
}

void freeTransfers(bmg_ctx* c);

void freeAll(bmg_ctx* c) {
    for (auto& L : c->lv) {
        for (void* p : {(void*)L.x64, (void*)L.b64, (void*)L.x32, (void*)L.b32, (void*)L.tab64, (void*)L.tab32,
                        (void*)L.jtmp64, (void*)L.jtmp32, (void*)L.x64b, (void*)L.x32b, (void*)L.gdst,
                        (void*)L.gsrc})
            if (p) cudaFree(p);
        for (int d = 0; d < 3; ++d) {
            if (L.lam64[d]) cudaFree(L.lam64[d]);
            if (L.lam32[d]) cudaFree(L.lam32[d]);
        }
    }
    freeTransfers(c);
    for (void* p : {(void*)c->ainv, (void*)c->cidx, (void*)c->partials, (void*)c->st, (void*)c->stage_b,
                    (void*)c->stage_x, (void*)c->fx, (void*)c->fb, (void*)c->fr, (void*)c->fp, (void*)c->fq})
        if (p) cudaFree(p);
    if (c->st_host) cudaFreeHost(c->st_host);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    destroyGraph(c);
    if (c->capStream) cudaStreamDestroy(c->capStream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    if (c->hookRhs) cudaFree(c->hookRhs);
    if (c->hookX) cudaFree(c->hookX);
}

void validateOptions(const bmg_options* o) {
    if (!(o->rel_tol >= 0.0) || !(o->abs_tol >= 0.0)) throw BadArg{BMG_BAD_ARG, "negative tolerance"};
    if (o->max_iter < 0 || o->min_iter < 0) throw BadArg{BMG_BAD_ARG, "negative iteration bound"};
    if (o->n_pre < 0 || o->n_post < 0) throw BadArg{BMG_BAD_ARG, "negative sweep count"};
    if (o->cycle_type < 0 || o->cycle_type > 2) throw BadArg{BMG_BAD_ARG, "unknown cycleType"};
    if (o->smoother < 0 || o->smoother > 1) throw BadArg{BMG_BAD_ARG, "unsupported smoother type"};
    if (o->precision < 0 || o->precision > 1) throw BadArg{BMG_BAD_ARG, "unknown precision"};
    if (o->coarse_level < 0) throw BadArg{BMG_BAD_ARG, "negative coarseLevel"};
    if (o->fused < 0) throw BadArg{BMG_BAD_ARG, "negative fused stage count"};
    if (o->fused_chunk < 1 || o->fused_chunk > 128) throw BadArg{BMG_BAD_ARG, "fusedChunk outside 1..128"};
    if (o->krylov < 0 || o->krylov > 1) throw BadArg{BMG_BAD_ARG, "unknown krylov"};
    if (o->criterion < 0 || o->criterion > 1) throw BadArg{BMG_BAD_ARG, "unknown criterion"};
    if (o->coarse_mode < 0 || o->coarse_mode > 1) throw BadArg{BMG_BAD_ARG, "unknown coarseMode"};
    if (o->restrict_scheme < 0 || o->restrict_scheme > 1) throw BadArg{BMG_BAD_ARG, "unknown restriction scheme"};
    if (o->prolong_scheme < 0 || o->prolong_scheme > 1) throw BadArg{BMG_BAD_ARG, "unknown prolongation scheme"};
    if (o->row_layout < 0 || o->row_layout > 1) throw BadArg{BMG_BAD_ARG, "unknown rowLayout"};
}

// Level-0 bricks from the mesh description; contacts between bricks.
void readBricks(bmg_ctx* c, const bmg_mesh_desc* mesh, HostLevel& L0) {
    if (!mesh || mesh->n_bricks < 1 || !mesh->bricks) throw BadArg{BMG_BAD_ARG, "empty mesh"};
    const int nb = mesh->n_bricks;
    if (nb > kMaxBricks) throw BadArg{BMG_UNSUPPORTED, "more bricks than this build handles (8)"};
    c->multi = nb > 1;
    for (int b = 0; b < nb; ++b) {
        const bmg_brick& B = mesh->bricks[b];
        HostBrick K;
        // Orientation (the transform T of parallelBoundaryCondition.C:148-163
        // between a brick's frame and its neighbours'): the brick is kept in
        // the mesh's frame on the device, and only the caller's arrays are
        // read and written in the brick's own frame.
        const bool ident = B.transform[0] == 0 && B.transform[1] == 0 && B.transform[2] == 0;
        int seen = 0;
        for (int d = 0; d < 3 && !ident; ++d) {
            const int t = B.transform[d], a = std::abs(t) - 1;
            if (a < 0 || a > 2 || ((seen >> a) & 1))
                throw BadArg{BMG_BAD_ARG, "brick transform is not a signed permutation of the axes"};
            seen |= 1 << a;
            K.tax[d] = a;
            K.tfl[d] = t < 0;
        }
        // the brick in the mesh's frame: extents, vertex coordinates (given
        // in local order along each local axis), face conditions and values
        int gn[3] = {0, 0, 0}, gbc[6];
        double gval[6];
        std::vector<double> gp[3];
        for (int d = 0; d < 3; ++d) {
            if (B.n[d] < 1) throw BadArg{BMG_BAD_ARG, "brick with fewer than one cell along an axis"};
            if (!B.points[d]) throw BadArg{BMG_BAD_ARG, "missing vertex coordinates"};
            const int a = K.tax[d], n = B.n[d];
            gn[a] = n;
            gp[a].resize(n + 1);
            for (int q = 0; q <= n; ++q) gp[a][q] = K.tfl[d] ? B.points[d][n - q] : B.points[d][q];
            for (int side = 0; side < 2; ++side) {
                const int gs = K.tfl[d] ? 1 - side : side;
                gbc[2 * a + gs] = B.bc[2 * d + side];
                gval[2 * a + gs] = B.value[2 * d + side];
            }
        }
        for (int d = 0; d < 3; ++d) {
            for (int q = 0; q < gn[d]; ++q)
                if (!(gp[d][q + 1] > gp[d][q]))
                    throw BadArg{BMG_BAD_ARG, "vertex coordinates must be strictly monotone (increasing along an "
                                              "axis, decreasing along a reversed one)"};
            const int lo = gbc[2 * d], hi = gbc[2 * d + 1];
            if ((lo == BMG_BC_PERIODIC) != (hi == BMG_BC_PERIODIC))
                throw BadArg{BMG_BAD_ARG, "periodic faces must come in opposite pairs"};
            for (int side = 0; side < 2; ++side) {
                const int t = gbc[2 * d + side];
                const double v = gval[2 * d + side];
                if (t != BMG_BC_PERIODIC && t != BMG_BC_NEUMANN && t != BMG_BC_DIRICHLET)
                    throw BadArg{BMG_BAD_ARG, "unknown boundary condition type"};
                if (t == BMG_BC_PERIODIC) continue;
                if (!std::isfinite(v)) throw BadArg{BMG_BAD_ARG, "a face value is not finite"};
                K.dval[2 * d + side] = v;
                K.dirichlet[2 * d + side] = t == BMG_BC_DIRICHLET;
            }
            if (lo == BMG_BC_PERIODIC && c->multi) L0.wrap[d] |= 1 << b;  // resolved below
            if (!c->multi) c->periodic[d] = lo == BMG_BC_PERIODIC;
            K.n[d] = gn[d];
            K.origin[d] = c->multi ? B.origin[d] : 0;
            K.ax[d].pts.assign(gn[d] + 3, 0.0);
            for (int q = 0; q <= gn[d]; ++q) K.ax[d].pts[q + 1] = gp[d][q];
            K.open[2 * d] = K.open[2 * d + 1] = c->periodic[d];
        }
        L0.br.push_back(std::move(K));
    }
    if (!c->multi) return;
    // the lattice box; an axis is periodic for every brick or for none
    for (int d = 0; d < 3; ++d) {
        int lo = L0.br[0].origin[d], hi = lo + L0.br[0].n[d];
        for (const auto& K : L0.br) {
            lo = std::min(lo, K.origin[d]);
            hi = std::max(hi, K.origin[d] + K.n[d]);
        }
        L0.lo[d] = lo;
        L0.ext[d] = hi - lo;
        const int all = (1 << nb) - 1;
        if (L0.wrap[d] != 0 && L0.wrap[d] != all)
            throw BadArg{BMG_BAD_ARG, "on a multi-brick mesh an axis is periodic for every brick or for none"};
        L0.wrap[d] = L0.wrap[d] != 0;
    }
    // bricks must not overlap; faces in the same plane with overlapping
    // extents are contacts, which need matching vertex coordinates (on a
    // periodic axis the box's two ends meet, one period apart)
    for (int a = 0; a < nb; ++a)
        for (int b = a + 1; b < nb; ++b) {
            const HostBrick& A = L0.br[a];
            const HostBrick& B = L0.br[b];
            long overlap = 1;
            for (int d = 0; d < 3; ++d)
                overlap *= std::max(0, std::min(A.origin[d] + A.n[d], B.origin[d] + B.n[d]) -
                                           std::max(A.origin[d], B.origin[d]));
            if (overlap > 0) throw BadArg{BMG_BAD_ARG, "bricks overlap"};
        }
    for (int a = 0; a < nb; ++a)
        for (int b = 0; b < nb; ++b) {
            HostBrick& A = L0.br[a];
            const HostBrick& B = L0.br[b];
            for (int d = 0; d < 3; ++d) {
                // A's upper face meets B's lower face, directly or across
                // the periodic ends of the box (a brick may meet itself)
                const bool across = L0.wrap[d] && A.origin[d] + A.n[d] == L0.lo[d] + L0.ext[d] &&
                                    B.origin[d] == L0.lo[d];
                if (!across && (a == b || A.origin[d] + A.n[d] != B.origin[d])) continue;
                const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
                const int lo1 = std::max(A.origin[t1], B.origin[t1]);
                const int hi1 = std::min(A.origin[t1] + A.n[t1], B.origin[t1] + B.n[t1]);
                const int lo2 = std::max(A.origin[t2], B.origin[t2]);
                const int hi2 = std::min(A.origin[t2] + A.n[t2], B.origin[t2] + B.n[t2]);
                if (hi1 <= lo1 || hi2 <= lo2) continue;
                const double scale = std::fabs(A.ax[d].pts[A.n[d] + 1] - A.ax[d].pts[1]) + 1.0;
                const double tol = 1e-12 * scale;
                if (across) {
                    const double P = A.ax[d].pts[A.n[d] + 1] - B.ax[d].pts[1];
                    if (L0.period[d] == 0.0) L0.period[d] = P;
                    if (!(P > 0.0) || std::fabs(P - L0.period[d]) > tol)
                        throw BadArg{BMG_BAD_ARG, "the periodic ends of the bricks are not one period apart"};
                } else if (std::fabs(A.ax[d].pts[A.n[d] + 1] - B.ax[d].pts[1]) > tol) {
                    throw BadArg{BMG_BAD_ARG, "bricks meet on a lattice face but their coordinates differ"};
                }
                for (int t : {t1, t2}) {
                    const int lo = t == t1 ? lo1 : lo2, hi = t == t1 ? hi1 : hi2;
                    for (int g = lo; g <= hi; ++g)
                        if (std::fabs(A.ax[t].pts[g - A.origin[t] + 1] - B.ax[t].pts[g - B.origin[t] + 1]) > tol)
                            throw BadArg{BMG_BAD_ARG, "brick contact is not cell-conforming"};
                }
                A.open[2 * d + 1] = true;
                L0.br[b].open[2 * d] = true;
                if (A.nbr[2 * d + 1] < 0) A.nbr[2 * d + 1] = b;
                if (L0.br[b].nbr[2 * d] < 0) L0.br[b].nbr[2 * d] = a;
            }
        }
    // A face wholly in contact with other bricks is an interface and carries
    // no boundary condition (the reference links whole faces of bricks,
    // brickFaceLink.C); a face partly in contact keeps zero-gradient walls on
    // the rest, which cannot take a Dirichlet value or a gradient.
    for (auto& B : L0.br)
        for (int d = 0; d < 3; ++d)
            for (int side = 0; side < 2; ++side) {
                const int f = 2 * d + side;
                if (!B.open[f]) continue;
                const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
                long touching = 0;
                for (int u = 0; u < B.n[t1]; ++u)
                    for (int v = 0; v < B.n[t2]; ++v) {
                        int g[3], loc[3];
                        g[d] = side ? B.origin[d] + B.n[d] : B.origin[d] - 1;
                        g[t1] = B.origin[t1] + u;
                        g[t2] = B.origin[t2] + v;
                        touching += findBrick(L0, g, loc) >= 0;
                    }
                if (touching == (long)B.n[t1] * B.n[t2]) {
                    B.dirichlet[f] = 0;
                    B.dval[f] = 0.0;
                    continue;
                }
                c->conforming = false;  // walls beside a contact: the contact mask
                if (B.dirichlet[f] || B.dval[f] != 0.0) {
                    throw BadArg{BMG_UNSUPPORTED,
                                 "a Dirichlet value or a Neumann gradient on a brick face partly in contact with "
                                 "another brick"};
                }
            }
}

// a system with no Dirichlet face anywhere is singular (linearSystem.H:227-230)
bool singularSystem(const HostLevel& L0) {
    for (const auto& B : L0.br)
        for (int f = 0; f < 6; ++f)
            if (B.dirichlet[f]) return false;
    return true;
}

// Coarse level: halve every extent (single brick: the reference's rule,
// dimensions of 3 or fewer cells stay; several bricks: all bricks halve in
// every direction together, so contacts stay cell-conforming).
bool coarsenLevel(const bmg_ctx* c, const HostLevel& F, HostLevel& C) {
    bool anyChange = false;
    if (!c->multi) {
        const HostBrick& B = F.br[0];
        HostBrick K;
        for (int d = 0; d < 3; ++d) {
            const int nc = B.n[d] <= 3 ? B.n[d] : B.n[d] / 2;
            if (B.n[d] > 3 && B.n[d] % 2)
                throw BadArg{BMG_BAD_ARG, "non-coarsenable brick size (an extent above 3 is odd on some level)"};
            anyChange = anyChange || nc != B.n[d];
            K.n[d] = nc;
            K.R[d] = B.n[d] / nc;
        }
        if (!anyChange) return false;
        for (int d = 0; d < 3; ++d) {
            K.tax[d] = B.tax[d];
            K.tfl[d] = B.tfl[d];
            K.ax[d].pts.assign(K.n[d] + 3, 0.0);
            for (int q = 0; q <= K.n[d]; ++q) K.ax[d].pts[q + 1] = B.ax[d].pts[q * K.R[d] + 1];
            K.open[2 * d] = K.open[2 * d + 1] = c->periodic[d];
            K.dirichlet[2 * d] = B.dirichlet[2 * d];
            K.dirichlet[2 * d + 1] = B.dirichlet[2 * d + 1];
        }
        C.br.push_back(std::move(K));
        return true;
    }
    for (const auto& B : F.br)
        for (int d = 0; d < 3; ++d)
            if (B.n[d] < 4 || B.n[d] % 2 || B.origin[d] % 2) return false;
    for (int d = 0; d < 3; ++d) {
        C.lo[d] = F.lo[d] / 2;
        C.ext[d] = F.ext[d] / 2;
        C.wrap[d] = F.wrap[d];
        C.period[d] = F.period[d];
    }
    for (const auto& B : F.br) {
        HostBrick K;
        for (int d = 0; d < 3; ++d) {
            K.n[d] = B.n[d] / 2;
            K.R[d] = 2;
            K.origin[d] = B.origin[d] / 2;
            K.ax[d].pts.assign(K.n[d] + 3, 0.0);
            for (int q = 0; q <= K.n[d]; ++q) K.ax[d].pts[q + 1] = B.ax[d].pts[2 * q + 1];
        }
        for (int f = 0; f < 6; ++f) {
            K.open[f] = B.open[f];
            K.nbr[f] = B.nbr[f];
            K.dirichlet[f] = B.dirichlet[f];
        }
        for (int d = 0; d < 3; ++d) {
            K.tax[d] = B.tax[d];
            K.tfl[d] = B.tfl[d];
        }
        C.br.push_back(std::move(K));
    }
    return true;
}

// ghost points and cell tables of every brick of a level; every brick
// touching a face must agree on the ghost point it gives
void finishLevel(const bmg_ctx* c, HostLevel& L) {
    // lattice planes a and b coincide, directly or as the two ends of a
    // periodic axis
    auto samePlane = [&](int d, int a, int b) {
        return a == b || (L.wrap[d] && ((a == L.lo[d] && b == L.lo[d] + L.ext[d]) ||
                                        (b == L.lo[d] && a == L.lo[d] + L.ext[d])));
    };
    for (auto& B : L.br)
        for (int d = 0; d < 3; ++d) {
            double g[2] = {NAN, NAN};
            for (int side = 0; side < 2; ++side) {
                if (B.nbr[2 * d + side] < 0) continue;
                const HostBrick& N = L.br[B.nbr[2 * d + side]];
                // across the periodic ends the neighbour's coordinates are
                // one period away
                const bool across = L.wrap[d] && (side ? B.origin[d] + B.n[d] == L.lo[d] + L.ext[d]
                                                       : B.origin[d] == L.lo[d]);
                const double shift = across ? (side ? L.period[d] : -L.period[d]) : 0.0;
                g[side] = (side ? N.ax[d].pts[2] : N.ax[d].pts[N.n[d]]) + shift;
                for (const auto& M : L.br) {
                    if (&M == &B || &M == &N) continue;
                    // another brick across the same face plane, overlapping it
                    const int plane = side ? B.origin[d] + B.n[d] : B.origin[d];
                    if (!samePlane(d, side ? M.origin[d] : M.origin[d] + M.n[d], plane)) continue;
                    bool touch = true;
                    for (int t : {(d + 1) % 3, (d + 2) % 3})
                        touch = touch && std::min(B.origin[t] + B.n[t], M.origin[t] + M.n[t]) >
                                             std::max(B.origin[t], M.origin[t]);
                    if (!touch) continue;
                    const double gm = (side ? M.ax[d].pts[2] : M.ax[d].pts[M.n[d]]) + shift;
                    const double h = std::fabs(B.ax[d].pts[side ? B.n[d] + 1 : 1] - g[side]);
                    if (std::fabs(gm - g[side]) > 1e-9 * h)
                        throw BadArg{BMG_UNSUPPORTED,
                                     "bricks touching one face have different cell sizes normal to it"};
                }
            }
            finishAxis(B.ax[d], B.n[d], c->periodic[d], g[0], g[1]);
        }
}

// face lambdas of a multi-brick level: 1 inside bricks and where a face
// touches another brick, 0 on the wall parts of open faces
void contactMask(const HostLevel& L, std::vector<double> mask[3]) {
    for (int d = 0; d < 3; ++d) mask[d].assign(L.cells, 1.0);
    for (const auto& B : L.br)
        for (int d = 0; d < 3; ++d)
            for (int side = 0; side < 2; ++side) {
                if (!B.open[2 * d + side]) continue;
                const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
                for (int u = 0; u < B.n[t1]; ++u)
                    for (int v = 0; v < B.n[t2]; ++v) {
                        int cell[3];
                        cell[d] = side ? B.n[d] - 1 : 0;
                        cell[t1] = u;
                        cell[t2] = v;
                        int g[3] = {B.origin[0] + cell[0], B.origin[1] + cell[1], B.origin[2] + cell[2]};
                        g[d] += side ? 1 : -1;
                        int loc[3];
                        const bool touch = findBrick(L, g, loc) >= 0;
                        int face[3] = {cell[0], cell[1], cell[2]};
                        if (side) face[d] += 1;  // upper face = lower face of the next cell
                        mask[d][B.at(face[0], face[1], face[2])] = touch ? 1.0 : 0.0;
                    }
            }
}

// Ghost frame of every brick: from the brick that owns the position, else a
// zero-gradient copy of the brick's own nearest cell (what the reference's
// unset-boundary copies give at walls, meshLevel.C:301-328), except beyond a
// Dirichlet face, where the ghost is left at zero as on a single brick.
void ghostList(const HostLevel& L, std::vector<int>& dst, std::vector<int>& src) {
    dst.clear();
    src.clear();
    for (const auto& B : L.br)
        for (int i = -1; i <= B.n[0]; ++i)
            for (int j = -1; j <= B.n[1]; ++j)
                for (int k = -1; k <= B.n[2]; ++k) {
                    const int l3[3] = {i, j, k};
                    bool ghost = false;
                    for (int d = 0; d < 3; ++d) ghost = ghost || l3[d] < 0 || l3[d] >= B.n[d];
                    if (!ghost) continue;
                    const int g[3] = {B.origin[0] + i, B.origin[1] + j, B.origin[2] + k};
                    int loc[3];
                    const int nb = findBrick(L, g, loc);
                    long s;
                    if (nb >= 0) {
                        s = L.br[nb].at(loc[0], loc[1], loc[2]);
                    } else {
                        // beyond a Dirichlet wall the ghost stays zero: the
                        // eliminated coupling (twice the face's) reads it
                        bool dir = false;
                        for (int d = 0; d < 3; ++d)
                            dir = dir || (l3[d] < 0 && B.dirichlet[2 * d]) || (l3[d] >= B.n[d] && B.dirichlet[2 * d + 1]);
                        if (dir) continue;
                        // elsewhere a zero-gradient copy of the nearest cell
                        const int ci = std::min(std::max(i, 0), B.n[0] - 1);
                        const int cj = std::min(std::max(j, 0), B.n[1] - 1);
                        const int ck = std::min(std::max(k, 0), B.n[2] - 1);
                        s = B.at(ci, cj, ck);
                    }
                    dst.push_back((int)B.at(i, j, k));
                    src.push_back((int)s);
                }
}

// face lambdas on the device: restricted user lambda (if any) times the
// contact mask (multi-brick), per level
void uploadLambda(bmg_ctx* c) {
    for (auto& L : c->lv) {
        std::vector<double> mask[3];
        if (c->multi) contactMask(L, mask);
        for (int d = 0; d < 3; ++d) {
            L.lam_host[d].assign(L.cells, c->multi ? 0.0 : 1.0);
            for (const auto& B : L.br)
                for (long q = 0; q < B.cells; ++q) {
                    double v = c->userLambda ? B.lam_user[d][q] : 1.0;
                    if (c->multi) v *= mask[d][B.off + q];
                    L.lam_host[d][B.off + q] = v;
                }
            if (!L.lam64[d]) L.lam64[d] = dalloc<double>(L.cells);
            if (!L.lam32[d]) L.lam32[d] = dalloc<float>(L.cells);
            // lam_host keeps the natural order (the coarse matrix reads it)
            std::vector<double> dev = L.lam_host[d];
            if (L.ks) splitRows(L.br[0], dev);
            upload(L.lam64[d], dev);
            upload(L.lam32[d], to_f32(dev));
        }
    }
}

// transfer tables per brick between levels l and l+1: restriction shares
// and prolongation indices/weights, for the configured schemes
void freeTransfers(bmg_ctx* c) {
    for (auto& lt : c->tr)
        for (auto& t : lt)
            for (void* p : {(void*)t.ratio64, (void*)t.ratio32, (void*)t.pidx, (void*)t.pw64, (void*)t.pw32})
                if (p) cudaFree(p);
    c->tr.clear();
}

void buildTransfers(bmg_ctx* c) {
    freeTransfers(c);
    const int nl = (int)c->lv.size();
    c->tr.assign(nl > 1 ? nl - 1 : 0, {});
    for (int l = 0; l + 1 < nl; ++l) {
        for (size_t b = 0; b < c->lv[l].br.size(); ++b) {
            const HostBrick& F = c->lv[l].br[b];
            const HostBrick& C = c->lv[l + 1].br[b];
            BrickTransfer t;
            std::vector<double> ratio, pw;
            std::vector<int> pidx;
            for (int d = 0; d < 3; ++d) {
                const int R = C.R[d];
                t.R[d] = R;
                const Axis& fa = F.ax[d];
                const Axis& ca = C.ax[d];
                for (int i = 0; i < F.n[d]; ++i) {
                    const int I0 = i / R;
                    // linear: the trilinear weight of the coarse centre between
                    // the two fine centres, h_f / H_c per axis
                    // (linearRestrictionScheme.C:15-80); average: 1/R per axis
                    // (averageRestrictionScheme.C:35-77)
                    ratio.push_back(R == 1 ? 1.0
                                    : c->opt.restrict_scheme == BMG_RESTRICT_AVERAGE ? 0.5
                                                                                     : fa.h[i + 1] / ca.h[I0 + 1]);
                    int I1 = I0;
                    double w = 0.0;
                    // injection (injectionProlongationScheme.C:14-33): the
                    // parent's value, weight 0 on every second coarse cell
                    if (R > 1 && c->opt.prolong_scheme == BMG_PROLONG_LINEAR) {
                        const int off = (i % 2) ? 1 : -1;
                        const int In = I0 + off;
                        // linearProlongationScheme.C:49-104: weight of the coarse
                        // neighbour on the fine cell's side, ghost centres included
                        w = (fa.cc[i + 1] - ca.cc[I0 + 1]) / (ca.cc[In + 1] - ca.cc[I0 + 1]);
                        if (In < 0 || In >= C.n[d]) {
                            if (c->periodic[d]) {
                                I1 = (In + C.n[d]) % C.n[d];
                            } else if (C.open[2 * d + (In >= C.n[d])]) {
                                I1 = In;  // ghost cell, refreshed from the neighbouring brick
                            } else if (C.dirichlet[2 * d + (In >= C.n[d])]) {
                                // the coarse ghost is -x (DirichletBoundaryCondition.C
                                // :59-80 above level 0): (1 - w) x + w (-x) = (1 - 2w) x,
                                // read as weight 2w on the ghost cell, which holds zero
                                I1 = In;
                                w = 2.0 * w;
                            } else {
                                I1 = I0;  // zero-gradient ghost: the value equals the parent's
                                w = 0.0;
                            }
                        } else {
                            I1 = In;
                        }
                    }
                    pidx.push_back(I0);
                    pidx.push_back(I1);
                    pw.push_back(w);
                }
            }
            t.ratio64 = dalloc<double>(ratio.size());
            t.ratio32 = dalloc<float>(ratio.size());
            t.pidx = dalloc<int>(pidx.size());
            t.pw64 = dalloc<double>(pw.size());
            t.pw32 = dalloc<float>(pw.size());
            upload(t.ratio64, ratio);
            upload(t.ratio32, to_f32(ratio));
            upload(t.pidx, pidx);
            upload(t.pw64, pw);
            upload(t.pw32, to_f32(pw));
            c->tr[l].push_back(t);
        }
    }
}

void build(bmg_ctx* c, HostLevel&& L0) {
    finishLevel(c, L0);
    c->lv.push_back(std::move(L0));
    // mesh.C:19-53: levels while coarsen(N) != N
    for (;;) {
        HostLevel C;
        if (!coarsenLevel(c, c->lv.back(), C)) break;
        finishLevel(c, C);
        c->lv.push_back(std::move(C));
    }
    const int nl = (int)c->lv.size();
    for (auto& L : c->lv) {
        for (auto& B : L.br)
            for (int d = 0; d < 3; ++d)
                if (c->periodic[d] && B.n[d] > 1 && B.n[d] % 2)
                    throw BadArg{BMG_UNSUPPORTED, "odd cell count along a periodic axis on some level"};
        // red-black colours alternate across the periodic ends of the box
        for (int d = 0; d < 3; ++d)
            if (L.wrap[d] && L.ext[d] > 1 && L.ext[d] % 2)
                throw BadArg{BMG_UNSUPPORTED, "odd cell count along a periodic axis on some level"};
    }
    for (auto& L : c->lv) {
        layout(L);
        if (L.cells >= (1L << 31)) throw BadArg{BMG_UNSUPPORTED, "a level above 2^31 cells"};
        // parity-split rows on the single-brick levels the per-pass kernels
        // run (above the single-CTA coarse end's size) whose rows are whole
        // 16-cell blocks
        L.ks = c->opt.row_layout == BMG_ROWS_SPLIT && !c->multi && L.br[0].n[2] % 16 == 0 &&
               L.ncell > kSplitMinCells;
        buildTables(L);
        L.x64 = dalloc<double>(L.cells);
        L.b64 = dalloc<double>(L.cells);
        L.x32 = dalloc<float>(L.cells);
        L.b32 = dalloc<float>(L.cells);
        L.tab64 = dalloc<double>(L.tab.size());
        L.tab32 = dalloc<float>(L.tab.size());
        upload(L.tab64, L.tab);
        upload(L.tab32, to_f32(L.tab));
        // the fused smoother handles one brick and marches along axis 0 in
        // chunks, wrapping at most one period there; its threads own k-quads,
        // and it relies on periodic extents being even (a wrapped neighbour
        // then has the other colour, as an interior one does)
        const HostBrick& B = L.br[0];
        L.fusedOK = !c->multi && !L.ks && B.n[0] >= 16 && B.n[1] >= 16 && B.n[2] >= 16 && B.n[2] % 4 == 0;
        for (int d = 0; d < 3; ++d)
            if (c->periodic[d] && B.n[d] % 2) L.fusedOK = false;
        if (L.fusedOK) {
            L.x64b = dalloc<double>(L.cells);
            L.x32b = dalloc<float>(L.cells);
        }
        if (c->multi) {
            std::vector<int> dst, src;
            ghostList(L, dst, src);
            L.nghost = (long)dst.size();
            L.gdst = dalloc<int>(dst.size());
            L.gsrc = dalloc<int>(src.size());
            upload(L.gdst, dst);
            upload(L.gsrc, src);
        }
    }
    // multi-brick meshes whose faces are partly in contact carry face
    // lambdas (the contact mask); where every contact covers whole faces
    // the tables alone describe the operator
    c->variable = c->multi && !c->conforming;
    if (c->multi) uploadLambda(c);
    buildTransfers(c);
    c->partials = dalloc<double>(3 * reduce_blocks(bricks<double>(c, 0)));
    c->st = dalloc<SolveState>(1);
    BMG_CUDA(cudaMallocHost(&c->st_host, sizeof(SolveState)));
    c->stage_b = dalloc<double>(c->lv[0].ncell);
    c->stage_x = dalloc<double>(c->lv[0].ncell);
    BMG_CUDA(cudaEventCreate(&c->ev0));
    BMG_CUDA(cudaEventCreate(&c->ev1));
    c->visits.assign(nl, 0);
}

// the coarse solve level the options ask for, checked against the hierarchy
int coarseLevelFor(const bmg_ctx* c, const bmg_options& o) {
    const int nl = (int)c->lv.size();
    if (nl < 2 || o.coarse_level > nl - 2)
        throw BadArg{BMG_BAD_ARG, "coarseLevel too high: at most (number of levels - 2)"};
    const int lc = nl - 1 - o.coarse_level;
    if (c->lv[lc].ncell > 4096 && o.coarse_mode == BMG_COARSE_DIRECT)
        throw BadArg{BMG_UNSUPPORTED, "coarse solve level above 4096 cells; raise coarseLevel"};
    return lc;
}

void configureCoarse(bmg_ctx* c) {
    c->lc = coarseLevelFor(c, c->opt);
    refreshCoarseInverse(c);
}

void ensureKrylovBuffers(bmg_ctx* c) {
    const long n = c->lv[0].cells;
    for (double** p : {&c->fx, &c->fb, &c->fr, &c->fp, &c->fq})
        if (!*p) *p = dalloc<double>(n);
}

void ensureJacobiBuffers(bmg_ctx* c) {
    for (auto& L : c->lv) {
        if (!L.jtmp64) L.jtmp64 = dalloc<double>(L.cells);
        if (!L.jtmp32) L.jtmp32 = dalloc<float>(L.cells);
    }
}

// ---------------------------------------------------------------------------
// cycle driver
// ---------------------------------------------------------------------------
// Colour order of one reference RBGS sweep over a whole level: forward even,
// forward odd, then the backward passes whose loop-counter parity maps to
// colour q = (n0+n1+n2+1) % 2 first (rbgsSmoother.C:125-183, utils.H:736-745).
// A colour repeated back to back recomputes the same values and is dropped.
// Several bricks follow the first brick's order.
std::vector<int> colourSequence(const HostLevel& L, int sweeps) {
    const HostBrick& B = L.br[0];
    const int q = (B.n[0] + B.n[1] + B.n[2] + 1) % 2;
    std::vector<int> seq;
    for (int s = 0; s < sweeps; ++s)
        for (int col : {0, 1, q, 1 - q})
            if (seq.empty() || seq.back() != col) seq.push_back(col);
    return seq;
}

FusedGeom fusedGeom(const bmg_ctx* c, const HostLevel& L, int prec) {
    const HostBrick& B = L.br[0];
    FusedGeom g{};
    g.m_axis = 0;
    g.nm = B.n[0];
    g.na = B.n[1];
    g.nk = B.n[2];
    g.sm = B.si;
    g.sa = B.sj;
    g.perm = c->periodic[0];
    g.pera = c->periodic[1];
    g.perk = c->periodic[2];
    g.ti = std::min(L.fusedTi[prec], B.n[0]);
    g.wl_m = B.to.wl[0];
    g.wh_m = B.to.wh[0];
    g.wl_a = B.to.wl[1];
    g.wh_a = B.to.wh[1];
    return g;
}

template <typename T>
void swapX(HostLevel& L) {
    if constexpr (sizeof(T) == 8)
        std::swap(L.x64, L.x64b);
    else
        std::swap(L.x32, L.x32b);
}

// refresh the ghost frames of a multi-brick level (device-side exchange)
template <typename T>
void exchangeField(bmg_ctx* c, int l, T* x) {
    HostLevel& L = c->lv[l];
    if (!L.nghost) return;
    c->launches += 1;
    launch_fill_ghosts<T>(x, L.gdst, L.gsrc, L.nghost, c->stream);
}

template <typename T>
void exchange(bmg_ctx* c, int l) {
    HostLevel& L = c->lv[l];
    if constexpr (sizeof(T) == 8)
        exchangeField<T>(c, l, reinterpret_cast<T*>(L.x64));
    else
        exchangeField<T>(c, l, reinterpret_cast<T*>(L.x32));
}

template <typename T>
void smooth(bmg_ctx* c, int l, int sweeps) {
    cudaStream_t s = c->stream;
    HostLevel& H = c->lv[l];
    const int prec = sizeof(T) == 8 ? 0 : 1;
    const std::vector<int> seq = colourSequence(H, sweeps);
    bool zeroFirst = false;  // the first pass starts from x = 0 (zeroFirst0)
    if (sizeof(T) == 4 && l == 0 && c->zeroFirst0) {
        zeroFirst = true;
        c->zeroFirst0 = false;
    }
    // (the fused smoother does not keep a pinned cell: a pinned level runs
    // pass by pass)
    const bool pinned = l == c->lc && c->singular && c->opt.coarse_mode == BMG_COARSE_SMOOTH;
    if (c->opt.smoother == BMG_SMOOTHER_RBGS && c->opt.fused > 0 && H.fusedOK && H.fusedS[prec] > 0 && !pinned) {
        // the colour sequence alternates; run it in launches of up to
        // maxS stages, each writing the other x buffer
        const FusedGeom g = fusedGeom(c, H, prec);
        const size_t maxS = (size_t)std::min({c->opt.fused, H.fusedS[prec], kFusedMaxStages});
        for (size_t p = 0; p < seq.size(); p += maxS) {
            const int stages = (int)std::min<size_t>(maxS, seq.size() - p);
            const LevelView<T> in = bricks<T>(c, l).v[0];
            T* out;
            if constexpr (sizeof(T) == 8)
                out = reinterpret_cast<T*>(H.x64b);
            else
                out = reinterpret_cast<T*>(H.x32b);
            c->launches += 1;
            if (c->variable)
                launch_smooth_fused<T, true>(in, out, g, seq[p], stages, s);
            else
                launch_smooth_fused<T, false>(in, out, g, seq[p], stages, s);
            swapX<T>(H);
        }
        return;
    }
    const Bricks<T> B = bricks<T>(c, l);
    if (c->opt.smoother == BMG_SMOOTHER_JACOBI) {
        T* tmp;
        if constexpr (sizeof(T) == 8)
            tmp = reinterpret_cast<T*>(H.jtmp64);
        else
            tmp = reinterpret_cast<T*>(H.jtmp32);
        for (int k = 0; k < sweeps; ++k) {
            exchange<T>(c, l);
            c->launches += 2;
            if (c->variable)
                launch_jacobi<T, true>(B, tmp, s);
            else
                launch_jacobi<T, false>(B, tmp, s);
        }
        return;
    }
    for (int col : seq) {
        exchange<T>(c, l);
        c->launches += 1;
        if (c->variable)
            launch_colour_pass<T, true>(B, col, s, zeroFirst);
        else
            launch_colour_pass<T, false>(B, col, s, zeroFirst);
        zeroFirst = false;
    }
}

template <typename T>
void residualRestrict(bmg_ctx* c, int l) {
    exchange<T>(c, l);
    const Bricks<T> F = bricks<T>(c, l);
    const Bricks<T> C = bricks<T>(c, l + 1);
    c->launches += 1;
    if (c->variable)
        launch_residual_restrict<T, true>(F, C, ttabs(c, l), c->stream);
    else
        launch_residual_restrict<T, false>(F, C, ttabs(c, l), c->stream);
    BMG_CUDA(cudaMemsetAsync(C.v[0].x, 0, C.v[0].cells * sizeof(T), c->stream));
}

template <typename T>
void prolongCorrect(bmg_ctx* c, int l) {
    exchange<T>(c, l + 1);
    c->launches += 1;
    launch_prolong_correct<T>(bricks<T>(c, l), bricks<T>(c, l + 1), ttabs(c, l), c->stream);
}

template <typename T>
void coarseSolve(bmg_ctx* c) {
    c->launches += 1;
    launch_coarse_solve<T>(bricks<T>(c, c->lc), c->ainv, c->cidx, c->ncoarse, c->stream);
}

// Launch-shape autotuner: for every level the fused smoother can handle,
// time one smoothing step (the configured sweep count) with one launch per
// colour pass and with the fused smoother at each number of colour stages
// per launch and plane-chunk length, and keep the fastest.  The tile (8 x
// 64 cells) is fixed by the fused kernel's thread block; stages and chunk
// length trade halo recomputation against memory passes and CTA count.
// Each candidate is timed as a captured graph of kTuneReps smoothing steps,
// the way the solve graph launches it (stream launches would charge the
// per-colour passes launch costs the solve does not pay).
constexpr int kTuneReps = 4;

template <typename T>
float timeSmoothGraph(bmg_ctx* c, int l, int sweeps, cudaEvent_t e0, cudaEvent_t e1) {
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    {
        // capture on the private stream; an exception ends the capture and
        // gives the context its stream back
        struct Capture {
            bmg_ctx* c;
            cudaStream_t user;
            ~Capture() {
                cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
                if (cudaStreamIsCapturing(c->capStream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                    cudaGraph_t dropped = nullptr;
                    cudaStreamEndCapture(c->capStream, &dropped);
                    if (dropped) cudaGraphDestroy(dropped);
                }
                c->stream = user;
            }
        } guard{c, c->stream};
        c->stream = c->capStream;
        BMG_CUDA(cudaStreamBeginCapture(c->capStream, cudaStreamCaptureModeThreadLocal));
        for (int r = 0; r < kTuneReps; ++r) smooth<T>(c, l, sweeps);
        BMG_CUDA(cudaStreamEndCapture(c->capStream, &g));
    }
    cudaError_t err = cudaSuccess;
    float ms = 0.f;
    err = cudaGraphInstantiate(&ge, g, 0);
    if (err == cudaSuccess) err = cudaGraphLaunch(ge, c->stream);  // warm-up
    if (err == cudaSuccess) err = cudaEventRecord(e0, c->stream);
    if (err == cudaSuccess) err = cudaGraphLaunch(ge, c->stream);
    if (err == cudaSuccess) err = cudaEventRecord(e1, c->stream);
    if (err == cudaSuccess) err = cudaEventSynchronize(e1);
    if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    BMG_CUDA(err);
    return ms;
}

template <typename T>
void autotuneLevel(bmg_ctx* c, int l, int sweeps, cudaEvent_t e0, cudaEvent_t e1) {
    HostLevel& H = c->lv[l];
    const int prec = sizeof(T) == 8 ? 0 : 1;
    float best = 1e30f;
    int bestS = H.fusedS[prec], bestTi = H.fusedTi[prec];
    const int n0 = H.br[0].n[0];
    for (int S = 0; S <= kFusedMaxStages; ++S) {
        bool whole = false;  // chunks at least as long as the level are all one launch shape
        for (int ti : {16, 24, 32, 48, 64, 128}) {
            if (S == 0 && ti != 16) continue;
            if (ti >= n0) {
                if (whole) continue;
                whole = true;
            }
            H.fusedS[prec] = S;
            H.fusedTi[prec] = ti;
            const float ms = timeSmoothGraph<T>(c, l, sweeps, e0, e1);
            if (ms < best) {
                best = ms;
                bestS = S;
                bestTi = ti;
            }
        }
    }
    H.fusedS[prec] = bestS;
    H.fusedTi[prec] = bestTi;
}

// planes per chunk of the fused smoother from the options (autotune off)
void applyChunk(bmg_ctx* c) {
    for (auto& L : c->lv) L.fusedTi[0] = L.fusedTi[1] = c->opt.fused_chunk;
}

void autotune(bmg_ctx* c) {
    if (c->opt.smoother != BMG_SMOOTHER_RBGS || c->opt.fused <= 0) return;
    const int sweeps = std::max({c->opt.n_pre, c->opt.n_post, 1});
    cudaEvent_t e0, e1;
    BMG_CUDA(cudaEventCreate(&e0));
    BMG_CUDA(cudaEventCreate(&e1));
    for (int l = 0; l < (int)c->lv.size(); ++l) {
        if (!c->lv[l].fusedOK) continue;
        autotuneLevel<double>(c, l, sweeps, e0, e1);
        autotuneLevel<float>(c, l, sweeps, e0, e1);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    // the timing runs smoothed whatever the buffers held: start clean
    for (auto& L : c->lv) {
        BMG_CUDA(cudaMemsetAsync(L.x64, 0, L.cells * sizeof(double), c->stream));
        BMG_CUDA(cudaMemsetAsync(L.x32, 0, L.cells * sizeof(float), c->stream));
        if (L.x64b) BMG_CUDA(cudaMemsetAsync(L.x64b, 0, L.cells * sizeof(double), c->stream));
        if (L.x32b) BMG_CUDA(cudaMemsetAsync(L.x32b, 0, L.cells * sizeof(float), c->stream));
    }
    BMG_CUDA(cudaStreamSynchronize(c->stream));
}

int levelReps(const bmg_ctx* c, int l) {  // MG.H:106-124
    if (c->opt.cycle_type == BMG_CYCLE_V) return 1;
    if (c->opt.cycle_type == BMG_CYCLE_W) return 1 + (l > 0);
    return 1 + (l > 0 && c->visits[l] == 0);
}

// MG.C:19-130.  x(l) = 0 for l > 0 is done by the restriction step that
// produces b(l).  The finest-level residual is always recomputed after
// pre-smoothing (the reference skips it on the first repetition, MG.C:72).
// The levels from tailFirst(c) to the coarse solve level run in one CTA
// (k_tail_cycle) when the cycle is a single-brick V cycle with red-black
// smoothing and factor-2 quad transfers on every one of them; -1 otherwise.
int tailFirst(const bmg_ctx* c) {
    if (!c->opt.fuse_coarse || c->multi || c->opt.cycle_type != BMG_CYCLE_V ||
        c->opt.smoother != BMG_SMOOTHER_RBGS || c->opt.coarse_mode != BMG_COARSE_DIRECT)
        return -1;
    const int lc = c->lc;
    int first = lc;
    while (first > 0 && c->lv[first - 1].ncell <= kTailCells) --first;
    if (first == lc || lc - first + 1 > kMaxTail) return -1;
    // a level solver inside the tail's levels would be skipped by it
    if (c->hook && c->hookLevel >= first) return -1;
    for (int q = first; q < lc; ++q) {
        const HostBrick& F = c->lv[q].br[0];
        const HostBrick& C = c->lv[q + 1].br[0];
        if (F.n[2] % 4 || C.R[0] != 2 || C.R[1] != 2 || C.R[2] != 2) return -1;
        const int lens[2] = {(int)colourSequence(c->lv[q], c->opt.n_pre).size(),
                             (int)colourSequence(c->lv[q], c->opt.n_post).size()};
        if (lens[0] > kMaxSeq || lens[1] > kMaxSeq) return -1;
    }
    return first;
}

template <typename T>
void tailCycle(bmg_ctx* c, int first) {
    TailPlan<T> P{};
    P.nlev = c->lc - first + 1;
    for (int q = 0; q < P.nlev; ++q) {
        const int l = first + q;
        P.v[q] = bricks<T>(c, l).v[0];
        if (l < c->lc) {
            P.t[q] = ttabs(c, l).t[0];
            const std::vector<int> pre = c->opt.n_pre > 0 ? colourSequence(c->lv[l], c->opt.n_pre) : std::vector<int>();
            const std::vector<int> post =
                c->opt.n_post > 0 ? colourSequence(c->lv[l], c->opt.n_post) : std::vector<int>();
            P.npre[q] = (int)pre.size();
            P.npost[q] = (int)post.size();
            for (size_t e = 0; e < pre.size(); ++e) P.pre[q][e] = pre[e];
            for (size_t e = 0; e < post.size(); ++e) P.post[q][e] = post[e];
        }
        c->visits[l]++;
    }
    P.ainv = c->ainv;
    P.cidx = c->cidx;
    P.ncoarse = c->ncoarse;
    c->launches += 1;
    if (c->variable)
        launch_tail_cycle<T, true>(P, c->stream);
    else
        launch_tail_cycle<T, false>(P, c->stream);
}

// The level solver's turn (bmg_set_level_solver): the level's right-hand
// side out to the solver, its result back as the level's x.
void hookSolve(bmg_ctx* c, int l) {
    const Bricks<float> B = bricks<float>(c, l);
    const HostBrick& K = c->lv[l].br[0];
    c->launches += 2;
    launch_b_to_plain32(B, c->hookRhs, c->stream);
    const int n[3] = {K.n[0], K.n[1], K.n[2]};
    if (c->hook(c->hookUser, c->stream, c->hookRhs, c->hookX, n) != 0)
        throw CudaError{"the level solver returned an error"};
    launch_plain32_to_x(B, c->hookX, c->stream);
}

template <typename T>
void cycle(bmg_ctx* c, int l) {
    if constexpr (sizeof(T) == 4) {
        if (c->hook && l == c->hookLevel) {
            hookSolve(c, l);
            if (c->hookMode == BMG_LEVEL_REPLACE) {
                // the solver's result is the level's correction: post-smooth
                // it; nothing below the level runs
                if (c->opt.n_post > 0) smooth<float>(c, l, c->opt.n_post);
                c->visits[l]++;
                return;
            }
            // BMG_LEVEL_GUESS: the usual cycle below, from the solver's x
        }
    }
    if (l == c->tail) return tailCycle<T>(c, l);
    if (c->opt.n_pre > 0) smooth<T>(c, l, c->opt.n_pre);
    if (l < c->lc) {
        const int reps = levelReps(c, l);
        for (int rep = 0; rep < reps; ++rep) {
            residualRestrict<T>(c, l);
            cycle<T>(c, l + 1);
            prolongCorrect<T>(c, l);
            if (c->opt.n_post > 0) smooth<T>(c, l, c->opt.n_post);
        }
    } else if (c->opt.coarse_mode == BMG_COARSE_SMOOTH) {
        smooth<T>(c, l, std::max(c->opt.n_post, 2));  // MG.C:116-125
    } else {
        coarseSolve<T>(c);
    }
    c->visits[l]++;
}

void checkLaunch() {
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw CudaError{std::string("kernel launch: ") + cudaGetErrorString(e)};
}

// level-0 FP64 residual norm and the convergence decision; inside a graph
// the decision also sets the WHILE node's condition
void residualNorm(bmg_ctx* c, int mode, bool setCondition) {
    exchange<double>(c, 0);
    const Bricks<double> L = bricks<double>(c, 0);
    float* b32 = c->opt.precision == BMG_PRECISION_MIXED ? c->lv[0].b32 : nullptr;
    c->launches += 2;
    const long n = c->variable ? launch_residual_norm<true>(L, walls(c), mode, c->partials, b32, c->stream)
                               : launch_residual_norm<false>(L, walls(c), mode, c->partials, b32, c->stream);
    launch_finalize_n(c->partials, n, c->st, mode, c->cond, setCondition ? 1 : 0, c->stream);
}

SolveState initialState(const bmg_ctx* c) {
    SolveState init{};
    init.rel_tol = c->opt.rel_tol;
    init.abs_tol = c->opt.abs_tol;
    init.min_iter = c->opt.min_iter;
    init.max_iter = c->opt.max_iter;
    init.ncells = (double)c->lv[0].ncell;
    double vol = 0.0;
    for (const auto& B : c->lv[0].br) {
        double v[3] = {0.0, 0.0, 0.0};
        for (int d = 0; d < 3; ++d)
            for (int i = 0; i < B.n[d]; ++i) v[d] += B.ax[d].h[i + 1];
        vol += v[0] * v[1] * v[2];
    }
    init.vol_total = vol;
    init.first = 1;
    init.criterion = c->opt.criterion;
    return init;
}

// MG.C:144-190: load b (scaled) and x, initial residual, normFactor and the
// first convergence test.  The state is copied from the pinned host copy,
// which the caller fills before every solve (also when replayed as a graph).
void segInitFcg(bmg_ctx* c, const double* bsrc, const double* xsrc, bool zero, bool setCondition);
bool zeroFirst(const bmg_ctx* c);
void segBodyFcg(bmg_ctx* c, bool setCondition);
void segPostFcg(bmg_ctx* c, double* xdst);

void segInit(bmg_ctx* c, const double* bsrc, const double* xsrc, bool zero, bool setCondition) {
    if (c->opt.krylov == BMG_KRYLOV_FCG) return segInitFcg(c, bsrc, xsrc, zero, setCondition);
    cudaStream_t s = c->stream;
    HostLevel& L0 = c->lv[0];
    const Bricks<double> V0 = bricks<double>(c, 0);
    launch_load_b(V0, walls(c), bsrc, s);
    BMG_CUDA(cudaMemsetAsync(L0.x64, 0, L0.cells * sizeof(double), s));
    c->launches += 1;
    if (!zero) {
        launch_load_x(V0, xsrc, s);
        c->launches += 1;
    }
    BMG_CUDA(cudaMemcpyAsync(c->st, c->st_host, sizeof(SolveState), cudaMemcpyHostToDevice, s));
    if (!zero && !c->singular) {
        launch_plain_mean(V0, c->partials, c->st, s);
        c->launches += 2;
    }
    residualNorm(c, 0, setCondition);
}

// MG.C:191-242: one cycle and the new residual.  Mixed precision: the FP32
// cycle solves for the correction of the FP64 residual (written in FP32 by
// the residual kernel), which is then added in FP64.
void segBody(bmg_ctx* c, bool setCondition) {
    if (c->opt.krylov == BMG_KRYLOV_FCG) return segBodyFcg(c, setCondition);
    cudaStream_t s = c->stream;
    HostLevel& L0 = c->lv[0];
    std::fill(c->visits.begin(), c->visits.end(), 0);
    if (c->opt.precision == BMG_PRECISION_MIXED) {
        BMG_CUDA(cudaMemsetAsync(L0.x32, 0, L0.cells * sizeof(float), s));
        cycle<float>(c, 0);
        launch_add_correction(bricks<double>(c, 0), bricks<float>(c, 0), s);
        c->launches += 1;
    } else {
        cycle<double>(c, 0);
    }
    residualNorm(c, 1, setCondition);
}

void segPost(bmg_ctx* c, double* xdst) {
    if (c->opt.krylov == BMG_KRYLOV_FCG) return segPostFcg(c, xdst);
    const Bricks<double> V0 = bricks<double>(c, 0);
    if (c->opt.remove_mean && c->singular) {
        launch_mean(V0, c->partials, c->st, c->stream);
        c->launches += 3;
    }
    launch_store_x(V0, xdst, c->stream);
    c->launches += 1;
}

// ---- flexible CG outer loop (bmg_krylov.cu) ----------------------------------
// level-0 FP64 view whose x and b are the outer loop's solution and RHS
Bricks<double> fcgView(const bmg_ctx* c) {
    Bricks<double> V = bricks<double>(c, 0);
    for (int b = 0; b < V.nb; ++b) {
        V.v[b].x = c->fx;
        V.v[b].b = c->fb;
    }
    return V;
}

// Whether each FP32 cycle of a mixed flexible-CG solve starts with a
// zero-start first colour pass on level 0 (fuseFirstPass) instead of a
// memset and a pass: a parity-split level 0 smoothed by red-black passes
// before anything else reads its x.
bool zeroFirst(const bmg_ctx* c) {
    return c->opt.fuse_first && c->opt.precision == BMG_PRECISION_MIXED && c->opt.krylov == BMG_KRYLOV_FCG &&
           c->lv[0].ks && c->opt.smoother == BMG_SMOOTHER_RBGS && c->opt.n_pre >= 1 && c->tail != 0 &&
           c->hookLevel != 0;
}

void segInitFcg(bmg_ctx* c, const double* bsrc, const double* xsrc, bool zero, bool setCondition) {
    cudaStream_t s = c->stream;
    const Bricks<double> V = fcgView(c);
    const bool mixed = c->opt.precision == BMG_PRECISION_MIXED;
    launch_load_b(V, walls(c), bsrc, s);
    BMG_CUDA(cudaMemsetAsync(c->fx, 0, c->lv[0].cells * sizeof(double), s));
    c->launches += 1;
    if (!zero) {
        launch_load_x(V, xsrc, s);
        c->launches += 1;
    }
    BMG_CUDA(cudaMemcpyAsync(c->st, c->st_host, sizeof(SolveState), cudaMemcpyHostToDevice, s));
    exchangeField<double>(c, 0, c->fx);
    if (!zero && !c->singular) {
        launch_plain_mean(V, c->partials, c->st, s);
        c->launches += 2;
    }
    float* pre32 = mixed ? c->lv[0].b32 : nullptr;
    double* pre64 = mixed ? nullptr : c->lv[0].b64;
    long n;
    if (c->variable)
        n = launch_fcg_residual<true>(V, walls(c), 0, c->fr, pre32, pre64, c->partials, s);
    else
        n = launch_fcg_residual<false>(V, walls(c), 0, c->fr, pre32, pre64, c->partials, s);
    launch_finalize_n(c->partials, n, c->st, 0, c->cond, setCondition ? 1 : 0, s);
    c->launches += 2;
}

template <typename T>
void fcgStep(bmg_ctx* c, const T* z, float* pre32, double* pre64, bool setCondition) {
    cudaStream_t s = c->stream;
    const Bricks<double> V = fcgView(c);
    if (c->variable)
        launch_fcg_step<T, true>(V, z, c->fp, c->fq, c->fr, pre32, pre64, c->partials, c->st, s);
    else
        launch_fcg_step<T, false>(V, z, c->fp, c->fq, c->fr, pre32, pre64, c->partials, c->st, s);
    launch_finalize_n(c->partials, fcg_partials(V), c->st, 1, c->cond, setCondition ? 1 : 0, s);
    c->launches += fcg_step_launches(V) + 1;
}

// one preconditioning cycle z = cycle(r) from a zero guess, then one FCG step
void segBodyFcg(bmg_ctx* c, bool setCondition) {
    cudaStream_t s = c->stream;
    HostLevel& L0 = c->lv[0];
    std::fill(c->visits.begin(), c->visits.end(), 0);
    if (c->opt.precision == BMG_PRECISION_MIXED) {
        // z starts from zero: the cycle's first level-0 pass writes all of
        // it (zeroFirst), or a memset does
        if (zeroFirst(c))
            c->zeroFirst0 = true;
        else
            BMG_CUDA(cudaMemsetAsync(L0.x32, 0, L0.cells * sizeof(float), s));
        cycle<float>(c, 0);
        c->zeroFirst0 = false;
        exchange<float>(c, 0);
        fcgStep<float>(c, L0.x32, L0.b32, nullptr, setCondition);
    } else {
        BMG_CUDA(cudaMemsetAsync(L0.x64, 0, L0.cells * sizeof(double), s));
        cycle<double>(c, 0);
        exchange<double>(c, 0);
        fcgStep<double>(c, L0.x64, nullptr, L0.b64, setCondition);
    }
}

// the true residual of the final x, mean removal and store
void segPostFcg(bmg_ctx* c, double* xdst) {
    cudaStream_t s = c->stream;
    const Bricks<double> V = fcgView(c);
    exchangeField<double>(c, 0, c->fx);
    long n;
    if (c->variable)
        n = launch_fcg_residual<true>(V, walls(c), 2, nullptr, nullptr, nullptr, c->partials, s);
    else
        n = launch_fcg_residual<false>(V, walls(c), 2, nullptr, nullptr, nullptr, c->partials, s);
    launch_fcg_true_norm(c->partials, n, c->st, s);
    c->launches += 2;
    if (c->opt.remove_mean && c->singular) {
        launch_mean(V, c->partials, c->st, s);
        c->launches += 3;
    }
    launch_store_x(V, xdst, s);
    c->launches += 1;
}

// Whole solve as one graph: init -> WHILE(keep_going){ cycle, residual,
// decision } -> mean removal and store.  Reads b from stage_b (and x from
// stage_x), writes x to stage_x.
void captureGraph(bmg_ctx* c, bool zero) {
    destroyGraph(c);
    // capture on the context's private stream (capturing the legacy default
    // stream is not allowed); the instantiated graph runs on any stream
    const cudaStream_t user = c->stream;
    c->stream = c->capStream;
    struct Restore {
        bmg_ctx* c;
        cudaStream_t s;
        ~Restore() {
            // a capture left open by an error is ended and dropped
            cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
            if (cudaStreamIsCapturing(c->capStream, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(c->capStream, &g);
                if (g && g != c->graph) cudaGraphDestroy(g);
            }
            c->stream = s;
        }
    } restore{c, user};
    cudaStream_t s = c->stream;
    BMG_CUDA(cudaGraphCreate(&c->graph, 0));
    BMG_CUDA(cudaGraphConditionalHandleCreate(&c->cond, c->graph, 0, 0));
    const long l0 = c->launches;
    BMG_CUDA(cudaStreamBeginCaptureToGraph(s, c->graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    segInit(c, c->stage_b, c->stage_x, zero, true);
    cudaStreamCaptureStatus cs;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    cudaGraph_t capg = nullptr;
    BMG_CUDA(cudaStreamGetCaptureInfo(s, &cs, nullptr, &capg, &deps, &ndeps));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = c->cond;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t loop;
    BMG_CUDA(cudaGraphAddNode(&loop, c->graph, deps, ndeps, &p));
    cudaGraph_t body = p.conditional.phGraph_out[0];
    BMG_CUDA(cudaStreamUpdateCaptureDependencies(s, &loop, 1, cudaStreamSetCaptureDependencies));
    segPost(c, c->stage_x);
    BMG_CUDA(cudaStreamEndCapture(s, &capg));
    const long l1 = c->launches;

    double* x0 = c->lv[0].x64;
    BMG_CUDA(cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    segBody(c, true);
    // the fused smoother swaps x buffers; level-0 x must come back to the
    // buffer the next iteration (and the post segment) reads (the flexible
    // CG loop keeps its solution elsewhere)
    if (c->lv[0].x64 != x0 && c->opt.krylov != BMG_KRYLOV_FCG) {
        BMG_CUDA(cudaMemcpyAsync(x0, c->lv[0].x64, c->lv[0].cells * sizeof(double), cudaMemcpyDeviceToDevice, s));
        std::swap(c->lv[0].x64, c->lv[0].x64b);
    }
    BMG_CUDA(cudaStreamEndCapture(s, &body));
    c->launchesInitPost = l1 - l0;
    c->launchesBody = c->launches - l1;
    BMG_CUDA(cudaGraphInstantiate(&c->gexec, c->graph, 0));
    c->graphZero = zero;
}

int solveImpl(bmg_ctx* c, const double* b, double* x, int flags, bmg_report* rep) {
    BMG_CUDA(cudaSetDevice(c->opt.device));
    cudaStream_t s = c->stream;
    const long n = c->lv[0].ncell;
    const bool dev = flags & BMG_DEVICE_PTRS;
    const bool zero = flags & BMG_ZERO_GUESS;
    if (c->opt.smoother == BMG_SMOOTHER_JACOBI) ensureJacobiBuffers(c);
    if (c->opt.krylov == BMG_KRYLOV_FCG) ensureKrylovBuffers(c);
    const auto t0 = std::chrono::steady_clock::now();
    *c->st_host = initialState(c);
    int status = BMG_OK;
    // the graph runs the loop on the device; a wall-clock budget needs the
    // host between cycles
    const bool useGraph = c->opt.use_graph && !(c->opt.timeout_ms > 0);

    if (useGraph) {
        if (!c->gexec || c->graphZero != zero) captureGraph(c, zero);
        const cudaMemcpyKind kin = dev ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        BMG_CUDA(cudaEventRecord(c->ev0, s));
        BMG_CUDA(cudaMemcpyAsync(c->stage_b, b, n * sizeof(double), kin, s));
        if (!zero) BMG_CUDA(cudaMemcpyAsync(c->stage_x, x, n * sizeof(double), kin, s));
        BMG_CUDA(cudaGraphLaunch(c->gexec, s));
        BMG_CUDA(cudaMemcpyAsync(x, c->stage_x, n * sizeof(double),
                                 dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, s));
    } else {
        c->launches = 0;
        BMG_CUDA(cudaEventRecord(c->ev0, s));
        const double* bsrc = b;
        const double* xsrc = x;
        if (!dev) {
            BMG_CUDA(cudaMemcpyAsync(c->stage_b, b, n * sizeof(double), cudaMemcpyHostToDevice, s));
            bsrc = c->stage_b;
            if (!zero) {
                BMG_CUDA(cudaMemcpyAsync(c->stage_x, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
                xsrc = c->stage_x;
            }
        }
        segInit(c, bsrc, xsrc, zero, false);
        checkLaunch();
        for (;;) {
            BMG_CUDA(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
            BMG_CUDA(cudaStreamSynchronize(s));
            if (!c->st_host->keep_going) break;
            if (c->opt.timeout_ms > 0) {
                const double ms =
                    std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
                if (ms > c->opt.timeout_ms) {
                    status = BMG_TIMEOUT;
                    break;
                }
            }
            segBody(c, false);
            checkLaunch();
        }
        double* xdst = dev ? x : c->stage_x;
        segPost(c, xdst);
        if (!dev) BMG_CUDA(cudaMemcpyAsync(x, c->stage_x, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    BMG_CUDA(cudaEventRecord(c->ev1, s));
    BMG_CUDA(cudaMemcpyAsync(c->st_host, c->st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
    BMG_CUDA(cudaStreamSynchronize(s));
    checkLaunch();
    const SolveState& st = *c->st_host;
    if (status == BMG_OK) {
        if (st.nan)
            status = BMG_NAN_DETECTED;
        else if (!st.converged)
            status = BMG_NOT_CONVERGED;
    }
    if (rep) {
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        rep->status = status;
        rep->cycles = st.iter;
        rep->outer_iterations = st.iter;
        rep->initial_residual = st.init;
        rep->final_residual = st.cur;
        // the flexible CG loop updates r recursively; report the residual of x
        const double l2 = c->opt.krylov == BMG_KRYLOV_FCG ? st.l2_true : st.l2;
        rep->rel_residual = st.l2_0 > 0 ? l2 / st.l2_0 : 0.0;
        rep->final_l2 = l2;
        rep->rhs_rel_residual = st.bnorm > 0 ? l2 / st.bnorm : 0.0;
        rep->norm_factor = st.nf;
        rep->ms = ms;
        rep->kernel_launches = useGraph ? c->launchesInitPost + c->launchesBody * st.iter : c->launches;
    }
    return status;
}

// restrict the level-0 face lambda to every level, area-weighted
// (areaWeightedFaceRestrictionScheme.C:19-57), per brick
void restrictLambda(bmg_ctx* c, const double* src[3]) {
    HostLevel& L0 = c->lv[0];
    long q[3] = {0, 0, 0};
    for (auto& B : L0.br) {
        for (int fd = 0; fd < 3; ++fd) B.lam_user[fd].assign(B.cells, 1.0);
        // the caller's arrays are in the brick's own frame: local face
        // direction ld, local face/cell indices l[] in local order
        for (int ld = 0; ld < 3; ++ld) {
            int ln[3];
            for (int d = 0; d < 3; ++d) ln[d] = B.n[B.tax[d]] + (d == ld);
            int l[3];
            for (l[0] = 0; l[0] < ln[0]; ++l[0])
                for (l[1] = 0; l[1] < ln[1]; ++l[1])
                    for (l[2] = 0; l[2] < ln[2]; ++l[2]) {
                        int g[3];
                        for (int d = 0; d < 3; ++d) g[B.tax[d]] = B.tfl[d] ? ln[d] - 1 - l[d] : l[d];
                        B.lam_user[B.tax[ld]][B.loc(g[0], g[1], g[2])] = src[ld][q[ld]++];
                    }
        }
    }
    for (size_t l = 0; l + 1 < c->lv.size(); ++l)
        for (size_t b = 0; b < c->lv[l].br.size(); ++b) {
            const HostBrick& F = c->lv[l].br[b];
            HostBrick& C = c->lv[l + 1].br[b];
            for (int fd = 0; fd < 3; ++fd) {
                C.lam_user[fd].assign(C.cells, 1.0);
                const int e0 = fd == 0, e1 = fd == 1, e2 = fd == 2;
                for (int I = 0; I < C.n[0] + e0; ++I)
                    for (int J = 0; J < C.n[1] + e1; ++J)
                        for (int K = 0; K < C.n[2] + e2; ++K) {
                            double area = 0.0, value = 0.0;
                            for (int ox = 0; ox < (fd == 0 ? 1 : C.R[0]); ++ox)
                                for (int oy = 0; oy < (fd == 1 ? 1 : C.R[1]); ++oy)
                                    for (int oz = 0; oz < (fd == 2 ? 1 : C.R[2]); ++oz) {
                                        const int fi = I * C.R[0] + ox, fj = J * C.R[1] + oy,
                                                  fk = K * C.R[2] + oz;
                                        const double a = fd == 0   ? F.ax[1].h[fj + 1] * F.ax[2].h[fk + 1]
                                                         : fd == 1 ? F.ax[0].h[fi + 1] * F.ax[2].h[fk + 1]
                                                                   : F.ax[0].h[fi + 1] * F.ax[1].h[fj + 1];
                                        area += a;
                                        value += a * F.lam_user[fd][F.loc(fi, fj, fk)];
                                    }
                            C.lam_user[fd][C.loc(I, J, K)] = value / area;
                        }
            }
        }
}

template <class F>
int guarded(bmg_ctx* c, F&& f) {
    try {
        return f();
    } catch (const BadArg& e) {
        if (c) c->err = e.msg;
        return e.code;
    } catch (const CudaError& e) {
        if (c) c->err = e.msg;
        return BMG_CUDA_ERROR;
    } catch (const std::exception& e) {
        if (c) c->err = e.what();
        return BMG_CUDA_ERROR;
    }
}

bool validLevel(const bmg_ctx* c, int l) { return c && l >= 0 && l < (int)c->lv.size(); }

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int bmg_default_options(bmg_options* o) {
    if (!o) return BMG_BAD_ARG;
    o->rel_tol = 1e-8;
    o->abs_tol = 0.0;
    o->min_iter = 0;
    o->max_iter = 999;
    o->n_pre = 0;
    o->n_post = 2;
    o->cycle_type = BMG_CYCLE_F;
    o->coarse_level = 0;
    o->smoother = BMG_SMOOTHER_RBGS;
    o->precision = BMG_PRECISION_FP64;
    o->use_graph = 1;
    o->remove_mean = 1;
    o->fused = kFusedMaxStages;
    o->autotune = 1;
    o->device = 0;
    o->timeout_ms = 0.0;
    o->krylov = BMG_KRYLOV_NONE;
    o->criterion = BMG_CRITERION_INITIAL;
    o->fused_chunk = 64;
    o->fuse_coarse = 1;
    o->coarse_mode = BMG_COARSE_DIRECT;
    o->restrict_scheme = BMG_RESTRICT_LINEAR;
    o->prolong_scheme = BMG_PROLONG_LINEAR;
    o->row_layout = BMG_ROWS_SPLIT;
    o->fuse_first = 1;
    return BMG_OK;
}

int bmg_create(bmg_ctx** out, const bmg_mesh_desc* mesh, const bmg_options* opts) {
    if (!out) return BMG_BAD_ARG;
    *out = nullptr;
    bmg_ctx* c = new bmg_ctx();
    if (opts)
        c->opt = *opts;
    else
        bmg_default_options(&c->opt);
    const int rc = guarded(c, [&] {
        validateOptions(&c->opt);
        // the mesh is checked on the host before any device work
        HostLevel L0;
        readBricks(c, mesh, L0);
        c->singular = singularSystem(L0);
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= c->opt.device || c->opt.device < 0)
            throw BadArg{BMG_NO_DEVICE, "no CUDA device with the requested ordinal"};
        cudaDeviceProp prop;
        BMG_CUDA(cudaGetDeviceProperties(&prop, c->opt.device));
        if (prop.major < 10) throw BadArg{BMG_NO_DEVICE, "device is not sm_100 class"};
        BMG_CUDA(cudaSetDevice(c->opt.device));
        BMG_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
        BMG_CUDA(cudaStreamCreateWithFlags(&c->capStream, cudaStreamNonBlocking));
        configure_fused_kernels();
        build(c, std::move(L0));
        configureCoarse(c);
        c->tail = tailFirst(c);
        applyChunk(c);
        if (c->opt.autotune) autotune(c);
        return BMG_OK;
    });
    if (rc != BMG_OK) {
        fprintf(stderr, "bmg_create: %s\n", c->err.c_str());
        freeAll(c);
        delete c;
        return rc;
    }
    *out = c;
    return BMG_OK;
}

void bmg_destroy(bmg_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->opt.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    freeAll(c);
    delete c;
}

int bmg_set_options(bmg_ctx* c, const bmg_options* o) {
    if (!c || !o) return BMG_BAD_ARG;
    return guarded(c, [&] {
        validateOptions(o);
        if (o->device != c->opt.device) throw BadArg{BMG_BAD_ARG, "the device of a context is fixed"};
        if (o->row_layout != c->opt.row_layout)
            throw BadArg{BMG_BAD_ARG, "the row layout of a context is fixed at creation"};
        const bool coarseChanged = o->coarse_level != c->opt.coarse_level || o->coarse_mode != c->opt.coarse_mode;
        const bool transfersChanged =
            o->restrict_scheme != c->opt.restrict_scheme || o->prolong_scheme != c->opt.prolong_scheme;
        const bool retune = o->autotune && (!c->opt.autotune || o->fused != c->opt.fused ||
                                            o->n_pre != c->opt.n_pre || o->n_post != c->opt.n_post);
        // options the hierarchy cannot take are refused before anything changes
        if (coarseChanged && c->hook && c->hookLevel > coarseLevelFor(c, *o))
            throw BadArg{BMG_BAD_ARG, "the level solver's level would lie below the coarse solve level"};
        if (coarseChanged) coarseLevelFor(c, *o);
        c->opt = *o;
        destroyGraph(c);
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (coarseChanged) configureCoarse(c);
        if (transfersChanged) buildTransfers(c);
        c->tail = tailFirst(c);
        if (!o->autotune) applyChunk(c);
        if (retune) autotune(c);
        return BMG_OK;
    });
}

int bmg_set_level_solver(bmg_ctx* c, int level, bmg_level_solver fn, void* user, int mode) {
    if (!c) return BMG_BAD_ARG;
    return guarded(c, [&] {
        if (mode != BMG_LEVEL_REPLACE && mode != BMG_LEVEL_GUESS)
            throw BadArg{BMG_BAD_ARG, "level solver: unknown mode"};
        if (fn && (level < 1 || level > c->lc))
            throw BadArg{BMG_BAD_ARG, "level solver: level outside 1 .. the coarse solve level"};
        if (fn && c->multi) throw BadArg{BMG_UNSUPPORTED, "level solver on a multi-brick mesh"};
        BMG_CUDA(cudaSetDevice(c->opt.device));
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        destroyGraph(c);
        if (c->hookRhs) cudaFree(c->hookRhs);
        if (c->hookX) cudaFree(c->hookX);
        c->hookRhs = c->hookX = nullptr;
        c->hook = fn;
        c->hookUser = fn ? user : nullptr;
        c->hookLevel = fn ? level : -1;
        c->hookMode = mode;
        if (fn) {
            c->hookRhs = dalloc<float>(c->lv[level].ncell);
            c->hookX = dalloc<float>(c->lv[level].ncell);
        }
        c->tail = tailFirst(c);
        return BMG_OK;
    });
}

int bmg_set_coefficients(bmg_ctx* c, const double* lx, const double* ly, const double* lz) {
    if (!c) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        if (!lx || !ly || !lz) {
            if (lx || ly || lz) throw BadArg{BMG_BAD_ARG, "give all three face coefficient arrays or none"};
            c->userLambda = false;
        } else {
            const double* src[3] = {lx, ly, lz};
            long nf[3] = {0, 0, 0};
            for (const auto& B : c->lv[0].br)
                for (int fd = 0; fd < 3; ++fd) {  // local face direction, local extents
                    long m = 1;
                    for (int d = 0; d < 3; ++d) m *= B.n[B.tax[d]] + (d == fd);
                    nf[fd] += m;
                }
            for (int fd = 0; fd < 3; ++fd)
                for (long q = 0; q < nf[fd]; ++q)
                    if (!(src[fd][q] > 0.0) || !std::isfinite(src[fd][q]))
                        throw BadArg{BMG_BAD_ARG, "face coefficients must be positive and finite"};
            restrictLambda(c, src);
            c->userLambda = true;
        }
        c->variable = c->userLambda || (c->multi && !c->conforming);
        if (c->variable) uploadLambda(c);
        refreshCoarseInverse(c);
        destroyGraph(c);  // kernels differ between constant and variable coefficients
        return BMG_OK;
    });
}

int bmg_set_stream(bmg_ctx* c, void* stream) {
    if (!c) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        if (c->own_stream) BMG_CUDA(cudaStreamDestroy(c->stream));
        c->own_stream = false;
        c->stream = static_cast<cudaStream_t>(stream);
        return BMG_OK;
    });
}

int bmg_solve(bmg_ctx* c, const double* b, double* x, int flags, bmg_report* rep) {
    if (!c || !b || !x) return BMG_BAD_ARG;
    const int rc = guarded(c, [&] { return solveImpl(c, b, x, flags, rep); });
    if (rep && (rc == BMG_BAD_ARG || rc == BMG_CUDA_ERROR || rc == BMG_UNSUPPORTED)) rep->status = rc;
    return rc;
}

long bmg_num_cells(const bmg_ctx* c) { return c ? c->lv[0].ncell : 0; }
int bmg_num_levels(const bmg_ctx* c) { return c ? (int)c->lv.size() : 0; }
int bmg_coarse_level_index(const bmg_ctx* c) { return c ? c->lc : -1; }

int bmg_level_tuning(const bmg_ctx* c, int l, int prec, int* stages, int* chunk) {
    if (!validLevel(c, l) || prec < 0 || prec > 1 || !stages || !chunk) return BMG_BAD_ARG;
    const HostLevel& L = c->lv[l];
    const bool fused = c->opt.smoother == BMG_SMOOTHER_RBGS && c->opt.fused > 0 && L.fusedOK && L.fusedS[prec] > 0;
    *stages = fused ? std::min({c->opt.fused, L.fusedS[prec], kFusedMaxStages}) : 0;
    *chunk = fused ? std::min(L.fusedTi[prec], L.br[0].n[0]) : 0;
    return BMG_OK;
}

int bmg_set_level_tuning(bmg_ctx* c, int l, int prec, int stages, int chunk) {
    if (!validLevel(c, l) || prec < 0 || prec > 1 || stages < 0 || stages > kFusedMaxStages || chunk < 1 ||
        chunk > 128)
        return BMG_BAD_ARG;
    HostLevel& L = c->lv[l];
    if (stages > 0 && !L.fusedOK) return BMG_UNSUPPORTED;
    return guarded(c, [&] {
        destroyGraph(c);
        L.fusedS[prec] = stages;
        L.fusedTi[prec] = chunk;
        return BMG_OK;
    });
}

namespace {

ProjGeom projGeom(const bmg_ctx* c) {
    if (c->multi) throw BadArg{BMG_UNSUPPORTED, "projection steps take a single-brick mesh"};
    const HostLevel& L = c->lv[0];
    const HostBrick& B = L.br[0];
    for (int d = 0; d < 3; ++d)
        if (B.tax[d] != d || B.tfl[d])
            throw BadArg{BMG_UNSUPPORTED, "projection steps take a brick in the mesh's own orientation"};
    ProjGeom G{};
    for (int d = 0; d < 3; ++d) {
        G.n[d] = B.n[d];
        G.per[d] = c->periodic[d];
        G.h[d] = L.tab64 + B.to.h[d];
    }
    return G;
}

}  // namespace

int bmg_project_rhs(bmg_ctx* c, const double* u0, const double* u1, const double* u2, double c_dt, double* out,
                    int flags) {
    if (!c || !u0 || !u1 || !u2 || !out || c_dt == 0.0) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        ProjGeom G = projGeom(c);
        G.cdt = c_dt;
        G.perVolume = (flags & BMG_PER_VOLUME) ? 1 : 0;
        launch_project_rhs(u0, u1, u2, out, G, c->stream);
        BMG_CUDA(cudaGetLastError());
        return BMG_OK;
    });
}

int bmg_project_correct(bmg_ctx* c, double* u0, double* u1, double* u2, const double* p, const double* lam0,
                        const double* lam1, const double* lam2, double c_dt) {
    if (!c || !u0 || !u1 || !u2 || !p) return BMG_BAD_ARG;
    if ((lam0 || lam1 || lam2) && !(lam0 && lam1 && lam2)) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        ProjGeom G = projGeom(c);
        G.cdt = c_dt;
        launch_project_correct(u0, u1, u2, p, lam0, lam1, lam2, G, c->stream);
        BMG_CUDA(cudaGetLastError());
        return BMG_OK;
    });
}

int bmg_level_shape(const bmg_ctx* c, int l, int brick, int n[3]) {
    if (!validLevel(c, l) || !n || brick < 0 || brick >= (int)c->lv[l].br.size()) return BMG_BAD_ARG;
    const auto& K = c->lv[l].br[brick];
    for (int d = 0; d < 3; ++d) n[d] = K.n[K.tax[d]];  // in the brick's own frame
    return BMG_OK;
}

const char* bmg_status_string(int s) {
    switch (s) {
        case BMG_OK: return "ok";
        case BMG_NOT_CONVERGED: return "not converged within maxIter";
        case BMG_NAN_DETECTED: return "residual became NaN or Inf";
        case BMG_BAD_ARG: return "invalid argument";
        case BMG_CUDA_ERROR: return "CUDA error";
        case BMG_TIMEOUT: return "solve exceeded its time budget";
        case BMG_NO_DEVICE: return "no usable sm_100 device";
        case BMG_UNSUPPORTED: return "unsupported configuration";
        default: return "unknown status";
    }
}

const char* bmg_last_error(const bmg_ctx* c) { return c ? c->err.c_str() : "no context"; }

// ---- building blocks --------------------------------------------------------

int bmg_level_upload(bmg_ctx* c, int l, int field, int prec, const double* host) {
    if (!validLevel(c, l) || !host || field < 0 || field > 1) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        HostLevel& L = c->lv[l];
        BMG_CUDA(cudaMemcpyAsync(c->stage_b, host, L.ncell * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (prec == 0) {
            if (field == 0) BMG_CUDA(cudaMemsetAsync(L.x64, 0, L.cells * sizeof(double), c->stream));
            launch_load_field<double>(bricks<double>(c, l), field, c->stage_b, 1, c->stream);
        } else {
            if (field == 0) BMG_CUDA(cudaMemsetAsync(L.x32, 0, L.cells * sizeof(float), c->stream));
            launch_load_field<float>(bricks<float>(c, l), field, c->stage_b, 1, c->stream);
        }
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_level_download(bmg_ctx* c, int l, int field, int prec, double* host) {
    if (!validLevel(c, l) || !host || field < 0 || field > 1) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (prec == 0)
            launch_store_field<double>(bricks<double>(c, l), field, c->stage_x, 1, c->stream);
        else
            launch_store_field<float>(bricks<float>(c, l), field, c->stage_x, 1, c->stream);
        checkLaunch();
        BMG_CUDA(cudaMemcpyAsync(host, c->stage_x, c->lv[l].ncell * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_colour_pass(bmg_ctx* c, int l, int colour, int prec) {
    if (!validLevel(c, l) || colour < 0 || colour > 1) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (prec == 0) {
            exchange<double>(c, l);
            if (c->variable) launch_colour_pass<double, true>(bricks<double>(c, l), colour, c->stream);
            else launch_colour_pass<double, false>(bricks<double>(c, l), colour, c->stream);
        } else {
            exchange<float>(c, l);
            if (c->variable) launch_colour_pass<float, true>(bricks<float>(c, l), colour, c->stream);
            else launch_colour_pass<float, false>(bricks<float>(c, l), colour, c->stream);
        }
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_smooth(bmg_ctx* c, int l, int sweeps, int prec) {
    if (!validLevel(c, l) || sweeps < 0) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (c->opt.smoother == BMG_SMOOTHER_JACOBI) ensureJacobiBuffers(c);
        if (prec == 0) smooth<double>(c, l, sweeps);
        else smooth<float>(c, l, sweeps);
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_residual(bmg_ctx* c, int l, int prec, double* host_r) {
    if (!validLevel(c, l) || !host_r) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (prec == 0) {
            exchange<double>(c, l);
            if (c->variable) launch_residual_out<double, true>(bricks<double>(c, l), c->stage_x, c->stream);
            else launch_residual_out<double, false>(bricks<double>(c, l), c->stage_x, c->stream);
        } else {
            exchange<float>(c, l);
            if (c->variable) launch_residual_out<float, true>(bricks<float>(c, l), c->stage_x, c->stream);
            else launch_residual_out<float, false>(bricks<float>(c, l), c->stage_x, c->stream);
        }
        checkLaunch();
        BMG_CUDA(cudaMemcpyAsync(host_r, c->stage_x, c->lv[l].ncell * sizeof(double), cudaMemcpyDeviceToHost,
                                 c->stream));
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_residual_restrict(bmg_ctx* c, int l, int prec) {
    if (!validLevel(c, l) || l + 1 >= (int)c->lv.size()) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (prec == 0) residualRestrict<double>(c, l);
        else residualRestrict<float>(c, l);
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_prolong_correct(bmg_ctx* c, int l, int prec) {
    if (!validLevel(c, l) || l + 1 >= (int)c->lv.size()) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (prec == 0) prolongCorrect<double>(c, l);
        else prolongCorrect<float>(c, l);
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_coarse_solve(bmg_ctx* c, int prec) {
    if (!c) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (c->ncoarse == 0) throw BadArg{BMG_UNSUPPORTED, "no dense coarse solve on a level above 4096 cells"};
        if (prec == 0) coarseSolve<double>(c);
        else coarseSolve<float>(c);
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

}  // extern "C"
