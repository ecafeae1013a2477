// bmg_host.cu -- host side of the B200 multigrid solver: level hierarchy,
// geometry tables, the V/W/F cycle driver, mixed-precision refinement and
// the C ABI declared in include/bmg.h.
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

struct HostLevel {
    int n[3] = {0, 0, 0};
    int R[3] = {1, 1, 1};  // ratio to the parent level
    Axis ax[3];
    long si = 0, sj = 0, base = 0, cells = 0;
    TabOff to{};
    std::vector<double> tab;  // host copy of the 1-D tables
    double* x64 = nullptr;
    double* b64 = nullptr;
    float* x32 = nullptr;
    float* b32 = nullptr;
    double* tab64 = nullptr;
    float* tab32 = nullptr;
    double* lam64[3] = {nullptr, nullptr, nullptr};
    float* lam32[3] = {nullptr, nullptr, nullptr};
    std::vector<double> lam_host[3];  // ghost-framed face lambda (variable coefficient)
    double* jtmp64 = nullptr;
    float* jtmp32 = nullptr;
    double* x64b = nullptr;  // second x buffers: fused smoothing writes here, then swaps
    float* x32b = nullptr;
    bool fusedOK = false;    // level large enough for the fused smoother
    // per precision (0: FP64, 1: FP32), picked by autotune():
    int fusedS[2] = {kFusedMaxStages, kFusedMaxStages};  // colour stages per fused launch
    int fusedTi[2] = {64, 64};                             // planes per CTA chunk
    long ncell() const { return (long)n[0] * n[1] * n[2]; }
    long at(int i, int j, int k) const { return base + (long)i * si + (long)j * sj + k; }
};

struct HostTransfer {
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
    int periodic[3] = {0, 0, 0};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    std::vector<HostLevel> lv;
    std::vector<HostTransfer> tr;
    int lc = 0;  // coarse solve level
    double* ainv = nullptr;
    int ncoarse = 0;
    bool variable = false;
    double* partials = nullptr;
    SolveState* st = nullptr;
    SolveState* st_host = nullptr;
    double* stage_b = nullptr;
    double* stage_x = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::string err;
    long launches = 0;  // kernels launched by the current solve
    std::vector<int> visits;
    // whole-solve CUDA graph (captured on the first solve, reused)
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    cudaGraphConditionalHandle cond = 0;
    cudaStream_t capStream = nullptr;  // private stream used only for capture
    bool graphZero = false;
    long launchesInitPost = 0, launchesBody = 0;
};

namespace {

// ---------------------------------------------------------------------------
// geometry
// ---------------------------------------------------------------------------
void finishAxis(Axis& a, int n, bool periodic) {
    std::vector<double>& p = a.pts;
    // levelPoints.C:198-236 (walls: project by one spacing) and :326-400
    // (periodic: the opposite side's spacing)
    if (periodic) {
        p[0] = p[1] - (p[n + 1] - p[n]);
        p[n + 2] = p[n + 1] + (p[2] - p[1]);
    } else {
        p[0] = p[1] + (p[1] - p[2]);
        p[n + 2] = p[n + 1] + (p[n + 1] - p[n]);
    }
    a.cc.assign(n + 2, 0.0);
    a.h.assign(n + 2, 0.0);
    for (int i = -1; i <= n; ++i) {
        a.cc[i + 1] = 0.5 * (p[i + 1] + p[i + 2]);
        a.h[i + 1] = p[i + 2] - p[i + 1];
    }
}

// Rows of pitch p2 = round_up(n2 + 5, 4) with interior k = 0 at offset 4:
// rows and interiors start on 16-byte (FP32) / 32-byte (FP64) boundaries so
// pairs and quads of k-neighbours load as one vector; the k ghosts sit at
// offsets 3 and n2 + 4.
void layout(HostLevel& L) {
    const long p2 = ((L.n[2] + 5) + 3) / 4 * 4, p1 = L.n[1] + 2, p0 = L.n[0] + 2;
    L.sj = p2;
    L.si = p1 * p2;
    L.base = L.si + L.sj + 4;
    L.cells = p0 * p1 * p2;
}

// row-scaled couplings (A'/V): lower neighbour delta(i)/h(i), upper
// delta(i+1)/h(i); zero across a wall, i.e. after the Neumann elimination
void buildTables(HostLevel& L, const int periodic[3]) {
    TabOff& to = L.to;
    int off = 0;
    for (int d = 0; d < 3; ++d) {
        to.wl[d] = off;
        off += L.n[d];
        to.wh[d] = off;
        off += L.n[d];
        to.h[d] = off;
        off += L.n[d];
    }
    to.total = off;
    L.tab.assign(off, 0.0);
    for (int d = 0; d < 3; ++d) {
        const Axis& a = L.ax[d];
        const int n = L.n[d];
        for (int i = 0; i < n; ++i) {
            const double hi = a.h[i + 1];
            const double dlo = 1.0 / std::fabs(a.cc[i + 1] - a.cc[i]);
            const double dhi = 1.0 / std::fabs(a.cc[i + 2] - a.cc[i + 1]);
            double wl = dlo / hi, wh = dhi / hi;
            if (!periodic[d] && i == 0) wl = 0.0;
            if (!periodic[d] && i == n - 1) wh = 0.0;
            L.tab[to.wl[d] + i] = wl;
            L.tab[to.wh[d] + i] = wh;
            L.tab[to.h[d] + i] = hi;
        }
    }
}

template <typename T>
LevelView<T> view(const bmg_ctx* c, int l) {
    const HostLevel& L = c->lv[l];
    LevelView<T> v{};
    v.n0 = L.n[0];
    v.n1 = L.n[1];
    v.n2 = L.n[2];
    v.si = L.si;
    v.sj = L.sj;
    v.base = L.base;
    v.cells = L.cells;
    v.to = L.to;
    v.tab64 = L.tab64;
    if constexpr (sizeof(T) == 8) {
        v.x = reinterpret_cast<T*>(L.x64);
        v.b = reinterpret_cast<T*>(L.b64);
        v.tab = reinterpret_cast<const T*>(L.tab64);
        for (int d = 0; d < 3; ++d) (&v.lam0)[d] = reinterpret_cast<const T*>(L.lam64[d]);
    } else {
        v.x = reinterpret_cast<T*>(L.x32);
        v.b = reinterpret_cast<T*>(L.b32);
        v.tab = reinterpret_cast<const T*>(L.tab32);
        for (int d = 0; d < 3; ++d) (&v.lam0)[d] = reinterpret_cast<const T*>(L.lam32[d]);
    }
    v.per0 = c->periodic[0];
    v.per1 = c->periodic[1];
    v.per2 = c->periodic[2];
    return v;
}

TransferTabs ttabs(const bmg_ctx* c, int l) {
    const HostTransfer& t = c->tr[l];
    TransferTabs s{};
    s.ratio64 = t.ratio64;
    s.ratio32 = t.ratio32;
    s.pidx = t.pidx;
    s.pw64 = t.pw64;
    s.pw32 = t.pw32;
    s.R0 = t.R[0];
    s.R1 = t.R[1];
    s.R2 = t.R[2];
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

// Dense row-scaled operator of the coarse solve level with the singularity
// pin of solver.C:201-231 (row of cell 0 = identity, every coupling to cell
// 0 removed, periodic images included), inverted once per matrix.
void buildCoarseInverse(bmg_ctx* c) {
    const HostLevel& L = c->lv[c->lc];
    const int n = (int)L.ncell();
    std::vector<double> M((size_t)n * n, 0.0);
    auto num = [&](int i, int j, int k) { return ((long)i * L.n[1] + j) * L.n[2] + k; };
    for (int i = 0; i < L.n[0]; ++i)
        for (int j = 0; j < L.n[1]; ++j)
            for (int k = 0; k < L.n[2]; ++k) {
                const long row = num(i, j, k);
                const int ijk[3] = {i, j, k};
                double diag = 0.0;
                for (int s = 0; s < 6; ++s) {
                    const int d = s / 2;
                    const bool up = s % 2;
                    double w = L.tab[(up ? L.to.wh[d] : L.to.wl[d]) + ijk[d]];
                    if (c->variable) {
                        long fc = L.at(i, j, k);
                        if (up) fc += d == 0 ? L.si : d == 1 ? L.sj : 1;
                        w *= L.lam_host[d][fc];
                    }
                    if (w == 0.0) continue;
                    diag -= w;
                    int nb[3] = {i, j, k};
                    nb[d] += up ? 1 : -1;
                    nb[d] = (nb[d] + L.n[d]) % L.n[d];
                    M[(size_t)row * n + num(nb[0], nb[1], nb[2])] += w;
                }
                M[(size_t)row * n + row] += diag;
            }
    for (int j = 0; j < n; ++j) M[j] = j == 0 ? 1.0 : 0.0;
    for (int r = 1; r < n; ++r) M[(size_t)r * n] = 0.0;
    std::vector<double> inv;
    if (!invert(M, n, inv)) throw BadArg{BMG_BAD_ARG, "coarse level matrix is singular"};
    if (!c->ainv || c->ncoarse != n) {
        if (c->ainv) cudaFree(c->ainv);
        c->ainv = dalloc<double>((size_t)n * n);
    }
    c->ncoarse = n;
    upload(c->ainv, inv);
}

void freeAll(bmg_ctx* c) {
    for (auto& L : c->lv) {
        for (void* p : {(void*)L.x64, (void*)L.b64, (void*)L.x32, (void*)L.b32, (void*)L.tab64,
                        (void*)L.tab32, (void*)L.jtmp64, (void*)L.jtmp32, (void*)L.x64b, (void*)L.x32b})
            if (p) cudaFree(p);
        for (int d = 0; d < 3; ++d) {
            if (L.lam64[d]) cudaFree(L.lam64[d]);
            if (L.lam32[d]) cudaFree(L.lam32[d]);
        }
    }
    for (auto& t : c->tr)
        for (void* p : {(void*)t.ratio64, (void*)t.ratio32, (void*)t.pidx, (void*)t.pw64, (void*)t.pw32})
            if (p) cudaFree(p);
    for (void* p : {(void*)c->ainv, (void*)c->partials, (void*)c->st, (void*)c->stage_b, (void*)c->stage_x})
        if (p) cudaFree(p);
    if (c->st_host) cudaFreeHost(c->st_host);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    if (c->capStream) cudaStreamDestroy(c->capStream);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
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
}

void build(bmg_ctx* c, const bmg_mesh_desc* mesh) {
    if (!mesh || mesh->n_bricks < 1 || !mesh->bricks) throw BadArg{BMG_BAD_ARG, "empty mesh"};
    if (mesh->n_bricks != 1)
        throw BadArg{BMG_UNSUPPORTED, "this build solves single-brick meshes"};
    const bmg_brick& B = mesh->bricks[0];
    for (int d = 0; d < 3; ++d) {
        if (B.n[d] < 1) throw BadArg{BMG_BAD_ARG, "brick with fewer than one cell along an axis"};
        if (!B.points[d]) throw BadArg{BMG_BAD_ARG, "missing vertex coordinates"};
        for (int q = 0; q < B.n[d]; ++q)
            if (!(B.points[d][q + 1] > B.points[d][q]))
                throw BadArg{BMG_BAD_ARG, "vertex coordinates must increase strictly"};
        const int lo = B.bc[2 * d], hi = B.bc[2 * d + 1];
        if ((lo == BMG_BC_PERIODIC) != (hi == BMG_BC_PERIODIC))
            throw BadArg{BMG_BAD_ARG, "periodic faces must come in opposite pairs"};
        if ((lo != BMG_BC_PERIODIC && lo != BMG_BC_NEUMANN) || (hi != BMG_BC_PERIODIC && hi != BMG_BC_NEUMANN))
            throw BadArg{BMG_UNSUPPORTED, "boundary condition type not supported"};
        c->periodic[d] = lo == BMG_BC_PERIODIC;
    }
    // mesh.C:19-53: levels while coarsen(N) != N
    HostLevel L0;
    for (int d = 0; d < 3; ++d) {
        L0.n[d] = B.n[d];
        L0.ax[d].pts.assign(B.n[d] + 3, 0.0);
        for (int q = 0; q <= B.n[d]; ++q) L0.ax[d].pts[q + 1] = B.points[d][q];
        finishAxis(L0.ax[d], B.n[d], c->periodic[d]);
    }
    c->lv.push_back(std::move(L0));
    for (;;) {
        const HostLevel& F = c->lv.back();
        int nc[3];
        bool same = true;
        for (int d = 0; d < 3; ++d) {
            nc[d] = F.n[d] <= 3 ? F.n[d] : F.n[d] / 2;
            if (F.n[d] > 3 && F.n[d] % 2)
                throw BadArg{BMG_BAD_ARG, "non-coarsenable brick size (an extent above 3 is odd on some level)"};
            same = same && nc[d] == F.n[d];
        }
        if (same) break;
        HostLevel C;
        for (int d = 0; d < 3; ++d) {
            C.n[d] = nc[d];
            C.R[d] = F.n[d] / nc[d];
            C.ax[d].pts.assign(nc[d] + 3, 0.0);
            for (int q = 0; q <= nc[d]; ++q) C.ax[d].pts[q + 1] = F.ax[d].pts[q * C.R[d] + 1];
            finishAxis(C.ax[d], nc[d], c->periodic[d]);
        }
        c->lv.push_back(std::move(C));
    }
    const int nl = (int)c->lv.size();
    for (auto& L : c->lv)
        for (int d = 0; d < 3; ++d)
            if (c->periodic[d] && L.n[d] > 1 && L.n[d] % 2)
                throw BadArg{BMG_UNSUPPORTED, "odd cell count along a periodic axis on some level"};
    for (auto& L : c->lv) {
        layout(L);
        buildTables(L, c->periodic);
        L.x64 = dalloc<double>(L.cells);
        L.b64 = dalloc<double>(L.cells);
        L.x32 = dalloc<float>(L.cells);
        L.b32 = dalloc<float>(L.cells);
        L.tab64 = dalloc<double>(L.tab.size());
        L.tab32 = dalloc<float>(L.tab.size());
        // the fused smoother marches along axis 0 in chunks and wraps at most
        // one period there (extent >= 2 * stages)
        L.fusedOK = L.n[0] >= 16 && L.n[1] >= 16 && L.n[2] >= 16;
        if (L.fusedOK) {
            L.x64b = dalloc<double>(L.cells);
            L.x32b = dalloc<float>(L.cells);
        }
        upload(L.tab64, L.tab);
        upload(L.tab32, to_f32(L.tab));
    }
    // transfer tables: restriction shares and prolongation indices/weights
    c->tr.resize(nl > 1 ? nl - 1 : 0);
    for (int l = 0; l + 1 < nl; ++l) {
        const HostLevel& F = c->lv[l];
        const HostLevel& C = c->lv[l + 1];
        HostTransfer& t = c->tr[l];
        std::vector<double> ratio, pw;
        std::vector<int> pidx;
        for (int d = 0; d < 3; ++d) {
            const int R = C.R[d];
            t.R[d] = R;
            const Axis& fa = F.ax[d];
            const Axis& ca = C.ax[d];
            for (int i = 0; i < F.n[d]; ++i) {
                const int I0 = i / R;
                ratio.push_back(R == 1 ? 1.0 : fa.h[i + 1] / ca.h[I0 + 1]);
                int I1 = I0;
                double w = 0.0;
                if (R > 1) {
                    const int off = (i % 2) ? 1 : -1;
                    const int In = I0 + off;
                    // linearProlongationScheme.C:49-104: weight of the coarse
                    // neighbour on the fine cell's side, ghost centres included
                    w = (fa.cc[i + 1] - ca.cc[I0 + 1]) / (ca.cc[In + 1] - ca.cc[I0 + 1]);
                    if (In < 0 || In >= C.n[d]) {
                        if (c->periodic[d]) {
                            I1 = (In + C.n[d]) % C.n[d];
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
    }
    c->partials = dalloc<double>(2 * reduce_blocks(view<double>(c, 0)));
    c->st = dalloc<SolveState>(1);
    BMG_CUDA(cudaMallocHost(&c->st_host, sizeof(SolveState)));
    c->stage_b = dalloc<double>(c->lv[0].ncell());
    c->stage_x = dalloc<double>(c->lv[0].ncell());
    BMG_CUDA(cudaEventCreate(&c->ev0));
    BMG_CUDA(cudaEventCreate(&c->ev1));
    c->visits.assign(nl, 0);
}

void configureCoarse(bmg_ctx* c) {
    const int nl = (int)c->lv.size();
    if (nl < 2 || c->opt.coarse_level > nl - 2)
        throw BadArg{BMG_BAD_ARG, "coarseLevel too high: at most (number of levels - 2)"};
    const int lc = nl - 1 - c->opt.coarse_level;
    if (c->lv[lc].ncell() > 4096)
        throw BadArg{BMG_UNSUPPORTED, "coarse solve level above 4096 cells; raise coarseLevel"};
    c->lc = lc;
    buildCoarseInverse(c);
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
std::vector<int> colourSequence(const HostLevel& L, int sweeps) {
    const int q = (L.n[0] + L.n[1] + L.n[2] + 1) % 2;
    std::vector<int> seq;
    for (int s = 0; s < sweeps; ++s)
        for (int col : {0, 1, q, 1 - q})
            if (seq.empty() || seq.back() != col) seq.push_back(col);
    return seq;
}

FusedGeom fusedGeom(const bmg_ctx* c, const HostLevel& L, int prec) {
    FusedGeom g{};
    g.m_axis = 0;
    g.nm = L.n[0];
    g.na = L.n[1];
    g.nk = L.n[2];
    g.sm = L.si;
    g.sa = L.sj;
    g.perm = c->periodic[0];
    g.pera = c->periodic[1];
    g.perk = c->periodic[2];
    g.ti = std::min(L.fusedTi[prec], L.n[0]);
    g.wl_m = L.to.wl[0];
    g.wh_m = L.to.wh[0];
    g.wl_a = L.to.wl[1];
    g.wh_a = L.to.wh[1];
    return g;
}

template <typename T>
void swapX(HostLevel& L) {
    if constexpr (sizeof(T) == 8)
        std::swap(L.x64, L.x64b);
    else
        std::swap(L.x32, L.x32b);
}

template <typename T>
void smooth(bmg_ctx* c, int l, int sweeps) {
    const LevelView<T> L = view<T>(c, l);
    cudaStream_t s = c->stream;
    HostLevel& H = c->lv[l];
    const int precIdx = sizeof(T) == 8 ? 0 : 1;
    if (c->opt.smoother == BMG_SMOOTHER_RBGS && c->opt.fused > 0 && H.fusedOK && H.fusedS[precIdx] > 0) {
        // the colour sequence alternates; run it in launches of up to
        // maxS stages, each writing the other x buffer
        const std::vector<int> seq = colourSequence(H, sweeps);
        const int prec = sizeof(T) == 8 ? 0 : 1;
        const FusedGeom g = fusedGeom(c, H, prec);
        const size_t maxS = (size_t)std::min({c->opt.fused, H.fusedS[prec], kFusedMaxStages});
        for (size_t p = 0; p < seq.size(); p += maxS) {
            const int stages = (int)std::min<size_t>(maxS, seq.size() - p);
            const LevelView<T> in = view<T>(c, l);
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
    if (c->opt.smoother == BMG_SMOOTHER_JACOBI) {
        T* tmp;
        if constexpr (sizeof(T) == 8)
            tmp = reinterpret_cast<T*>(c->lv[l].jtmp64);
        else
            tmp = reinterpret_cast<T*>(c->lv[l].jtmp32);
        for (int k = 0; k < sweeps; ++k) {
            c->launches += 2;
            if (c->variable)
                launch_jacobi<T, true>(L, tmp, s);
            else
                launch_jacobi<T, false>(L, tmp, s);
        }
        return;
    }
    for (int col : colourSequence(c->lv[l], sweeps)) {
        c->launches += 1;
        if (c->variable)
            launch_colour_pass<T, true>(L, col, s);
        else
            launch_colour_pass<T, false>(L, col, s);
    }
}

template <typename T>
void residualRestrict(bmg_ctx* c, int l) {
    const LevelView<T> F = view<T>(c, l);
    const LevelView<T> C = view<T>(c, l + 1);
    c->launches += 1;
    if (c->variable)
        launch_residual_restrict<T, true>(F, C, ttabs(c, l), c->stream);
    else
        launch_residual_restrict<T, false>(F, C, ttabs(c, l), c->stream);
    BMG_CUDA(cudaMemsetAsync(C.x, 0, C.cells * sizeof(T), c->stream));
}

template <typename T>
void prolongCorrect(bmg_ctx* c, int l) {
    c->launches += 1;
    launch_prolong_correct<T>(view<T>(c, l), view<T>(c, l + 1), ttabs(c, l), c->stream);
}

template <typename T>
void coarseSolve(bmg_ctx* c) {
    c->launches += 1;
    launch_coarse_solve<T>(view<T>(c, c->lc), c->ainv, c->ncoarse, c->stream);
}

// Launch-shape autotuner: for every level the fused smoother handles, time
// one smoothing step (the configured sweep count) for each number of colour
// stages per launch and each plane-chunk length, and keep the fastest.  The
// tile (16 x 64 cells) is fixed by the kernel's register window; stages and
// chunk length trade halo recomputation against memory passes and CTA count.
template <typename T>
void autotuneLevel(bmg_ctx* c, int l, int sweeps, cudaEvent_t e0, cudaEvent_t e1) {
    HostLevel& H = c->lv[l];
    const int prec = sizeof(T) == 8 ? 0 : 1;
    float best = 1e30f;
    int bestS = H.fusedS[prec], bestTi = H.fusedTi[prec];
    // S = 0: one launch per colour pass (no temporal blocking)
    for (int S = 0; S <= kFusedMaxStages; ++S)
        for (int ti : {32, 64, 128}) {
            if (ti > 2 * H.n[0] && ti != 32) continue;
            if (S == 0 && ti != 32) continue;
            H.fusedS[prec] = S;
            H.fusedTi[prec] = ti;
            smooth<T>(c, l, sweeps);  // warm-up
            BMG_CUDA(cudaEventRecord(e0, c->stream));
            for (int r = 0; r < 3; ++r) smooth<T>(c, l, sweeps);
            BMG_CUDA(cudaEventRecord(e1, c->stream));
            BMG_CUDA(cudaEventSynchronize(e1));
            float ms = 0.f;
            BMG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) {
                best = ms;
                bestS = S;
                bestTi = ti;
            }
        }
    H.fusedS[prec] = bestS;
    H.fusedTi[prec] = bestTi;
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
template <typename T>
void cycle(bmg_ctx* c, int l) {
    if (c->opt.n_pre > 0) smooth<T>(c, l, c->opt.n_pre);
    if (l < c->lc) {
        const int reps = levelReps(c, l);
        for (int rep = 0; rep < reps; ++rep) {
            residualRestrict<T>(c, l);
            cycle<T>(c, l + 1);
            prolongCorrect<T>(c, l);
            if (c->opt.n_post > 0) smooth<T>(c, l, c->opt.n_post);
        }
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
    const LevelView<double> L = view<double>(c, 0);
    float* b32 = c->opt.precision == BMG_PRECISION_MIXED ? c->lv[0].b32 : nullptr;
    c->launches += 2;
    if (c->variable)
        launch_residual_norm<true>(L, mode, c->partials, b32, nullptr, c->stream);
    else
        launch_residual_norm<false>(L, mode, c->partials, b32, nullptr, c->stream);
    launch_finalize(L, c->partials, c->st, mode, c->cond, setCondition ? 1 : 0, c->stream);
}

SolveState initialState(const bmg_ctx* c) {
    const HostLevel& L0 = c->lv[0];
    SolveState init{};
    init.rel_tol = c->opt.rel_tol;
    init.abs_tol = c->opt.abs_tol;
    init.min_iter = c->opt.min_iter;
    init.max_iter = c->opt.max_iter;
    init.ncells = (double)L0.ncell();
    double v[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < 3; ++d)
        for (int i = 0; i < L0.n[d]; ++i) v[d] += L0.ax[d].h[i + 1];
    init.vol_total = v[0] * v[1] * v[2];
    return init;
}

// MG.C:144-190: load b (scaled) and x, initial residual, normFactor and the
// first convergence test.  The state is copied from the pinned host copy,
// which the caller fills before every solve (also when replayed as a graph).
void segInit(bmg_ctx* c, const double* bsrc, const double* xsrc, bool zero, bool setCondition) {
    cudaStream_t s = c->stream;
    HostLevel& L0 = c->lv[0];
    const LevelView<double> V0 = view<double>(c, 0);
    launch_load_b(V0, bsrc, s);
    BMG_CUDA(cudaMemsetAsync(L0.x64, 0, L0.cells * sizeof(double), s));
    c->launches += 1;
    if (!zero) {
        launch_load_x(V0, xsrc, s);
        c->launches += 1;
    }
    BMG_CUDA(cudaMemcpyAsync(c->st, c->st_host, sizeof(SolveState), cudaMemcpyHostToDevice, s));
    residualNorm(c, 0, setCondition);
}

// MG.C:191-242: one cycle and the new residual.  Mixed precision: the FP32
// cycle solves for the correction of the FP64 residual (written in FP32 by
// the residual kernel), which is then added in FP64.
void segBody(bmg_ctx* c, bool setCondition) {
    cudaStream_t s = c->stream;
    HostLevel& L0 = c->lv[0];
    std::fill(c->visits.begin(), c->visits.end(), 0);
    if (c->opt.precision == BMG_PRECISION_MIXED) {
        BMG_CUDA(cudaMemsetAsync(L0.x32, 0, L0.cells * sizeof(float), s));
        cycle<float>(c, 0);
        launch_add_correction(view<double>(c, 0), view<float>(c, 0), s);
        c->launches += 1;
    } else {
        cycle<double>(c, 0);
    }
    residualNorm(c, 1, setCondition);
}

void segPost(bmg_ctx* c, double* xdst) {
    const LevelView<double> V0 = view<double>(c, 0);
    if (c->opt.remove_mean) {
        launch_mean(V0, c->partials, c->st, c->stream);
        c->launches += 3;
    }
    launch_store_x(V0, xdst, c->stream);
    c->launches += 1;
}

void destroyGraph(bmg_ctx* c) {
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->gexec = nullptr;
    c->graph = nullptr;
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
    // buffer the next iteration (and the post segment) reads
    if (c->lv[0].x64 != x0) {
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
    const long n = c->lv[0].ncell();
    const bool dev = flags & BMG_DEVICE_PTRS;
    const bool zero = flags & BMG_ZERO_GUESS;
    if (c->opt.smoother == BMG_SMOOTHER_JACOBI) ensureJacobiBuffers(c);
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
        rep->rel_residual = st.l2_0 > 0 ? st.l2 / st.l2_0 : 0.0;
        rep->final_l2 = st.l2;
        rep->norm_factor = st.nf;
        rep->ms = ms;
        rep->kernel_launches = useGraph ? c->launchesInitPost + c->launchesBody * st.iter : c->launches;
    }
    return status;
}

// restrict the level-0 face lambda to every level, area-weighted
// (areaWeightedFaceRestrictionScheme.C:19-57), into ghost-framed face arrays
void restrictLambda(bmg_ctx* c, const double* src[3]) {
    HostLevel& L0 = c->lv[0];
    for (int fd = 0; fd < 3; ++fd) {
        L0.lam_host[fd].assign(L0.cells, 0.0);
        const int e0 = fd == 0, e1 = fd == 1, e2 = fd == 2;
        long q = 0;
        for (int i = 0; i < L0.n[0] + e0; ++i)
            for (int j = 0; j < L0.n[1] + e1; ++j)
                for (int k = 0; k < L0.n[2] + e2; ++k) L0.lam_host[fd][L0.at(i, j, k)] = src[fd][q++];
    }
    for (size_t l = 0; l + 1 < c->lv.size(); ++l) {
        const HostLevel& F = c->lv[l];
        HostLevel& C = c->lv[l + 1];
        for (int fd = 0; fd < 3; ++fd) {
            C.lam_host[fd].assign(C.cells, 0.0);
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
                                    value += a * F.lam_host[fd][F.at(fi, fj, fk)];
                                }
                        C.lam_host[fd][C.at(I, J, K)] = value / area;
                    }
        }
    }
    for (auto& L : c->lv)
        for (int fd = 0; fd < 3; ++fd) {
            if (!L.lam64[fd]) L.lam64[fd] = dalloc<double>(L.cells);
            if (!L.lam32[fd]) L.lam32[fd] = dalloc<float>(L.cells);
            upload(L.lam64[fd], L.lam_host[fd]);
            upload(L.lam32[fd], to_f32(L.lam_host[fd]));
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
        build(c, mesh);
        configureCoarse(c);
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
        const bool coarseChanged = o->coarse_level != c->opt.coarse_level;
        const bool retune = o->autotune && (!c->opt.autotune || o->fused != c->opt.fused ||
                                            o->n_pre != c->opt.n_pre || o->n_post != c->opt.n_post);
        c->opt = *o;
        destroyGraph(c);
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (coarseChanged) configureCoarse(c);
        if (retune) autotune(c);
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
            c->variable = false;
        } else {
            const double* src[3] = {lx, ly, lz};
            for (int fd = 0; fd < 3; ++fd) {
                const HostLevel& L0 = c->lv[0];
                long nf = (long)(L0.n[0] + (fd == 0)) * (L0.n[1] + (fd == 1)) * (L0.n[2] + (fd == 2));
                for (long q = 0; q < nf; ++q)
                    if (!(src[fd][q] > 0.0) || !std::isfinite(src[fd][q]))
                        throw BadArg{BMG_BAD_ARG, "face coefficients must be positive and finite"};
            }
            restrictLambda(c, src);
            c->variable = true;
        }
        buildCoarseInverse(c);
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

long bmg_num_cells(const bmg_ctx* c) { return c ? c->lv[0].ncell() : 0; }
int bmg_num_levels(const bmg_ctx* c) { return c ? (int)c->lv.size() : 0; }
int bmg_coarse_level_index(const bmg_ctx* c) { return c ? c->lc : -1; }

int bmg_level_tuning(const bmg_ctx* c, int l, int prec, int* stages, int* chunk) {
    if (!validLevel(c, l) || prec < 0 || prec > 1 || !stages || !chunk) return BMG_BAD_ARG;
    const HostLevel& L = c->lv[l];
    const bool fused = c->opt.smoother == BMG_SMOOTHER_RBGS && c->opt.fused > 0 && L.fusedOK && L.fusedS[prec] > 0;
    *stages = fused ? std::min({c->opt.fused, L.fusedS[prec], kFusedMaxStages}) : 0;
    *chunk = fused ? std::min(L.fusedTi[prec], L.n[0]) : 0;
    return BMG_OK;
}

int bmg_level_shape(const bmg_ctx* c, int l, int brick, int n[3]) {
    if (!validLevel(c, l) || brick != 0 || !n) return BMG_BAD_ARG;
    for (int d = 0; d < 3; ++d) n[d] = c->lv[l].n[d];
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
        const long n = c->lv[l].ncell();
        BMG_CUDA(cudaMemcpyAsync(c->stage_b, host, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
        if (prec == 0) {
            if (field == 0) BMG_CUDA(cudaMemsetAsync(c->lv[l].x64, 0, c->lv[l].cells * sizeof(double), c->stream));
            launch_load_field<double>(view<double>(c, l), field, c->stage_b, 1, c->stream);
        } else {
            if (field == 0) BMG_CUDA(cudaMemsetAsync(c->lv[l].x32, 0, c->lv[l].cells * sizeof(float), c->stream));
            launch_load_field<float>(view<float>(c, l), field, c->stage_b, 1, c->stream);
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
        const long n = c->lv[l].ncell();
        if (prec == 0)
            launch_store_field<double>(view<double>(c, l), field, c->stage_x, 1, c->stream);
        else
            launch_store_field<float>(view<float>(c, l), field, c->stage_x, 1, c->stream);
        checkLaunch();
        BMG_CUDA(cudaMemcpyAsync(host, c->stage_x, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

int bmg_op_colour_pass(bmg_ctx* c, int l, int colour, int prec) {
    if (!validLevel(c, l) || colour < 0 || colour > 1) return BMG_BAD_ARG;
    return guarded(c, [&] {
        BMG_CUDA(cudaSetDevice(c->opt.device));
        if (prec == 0) {
            if (c->variable) launch_colour_pass<double, true>(view<double>(c, l), colour, c->stream);
            else launch_colour_pass<double, false>(view<double>(c, l), colour, c->stream);
        } else {
            if (c->variable) launch_colour_pass<float, true>(view<float>(c, l), colour, c->stream);
            else launch_colour_pass<float, false>(view<float>(c, l), colour, c->stream);
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
            if (c->variable) launch_residual_out<double, true>(view<double>(c, l), c->stage_x, c->stream);
            else launch_residual_out<double, false>(view<double>(c, l), c->stage_x, c->stream);
        } else {
            if (c->variable) launch_residual_out<float, true>(view<float>(c, l), c->stage_x, c->stream);
            else launch_residual_out<float, false>(view<float>(c, l), c->stage_x, c->stream);
        }
        checkLaunch();
        BMG_CUDA(cudaMemcpyAsync(host_r, c->stage_x, c->lv[l].ncell() * sizeof(double),
                                 cudaMemcpyDeviceToHost, c->stream));
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
        if (prec == 0) coarseSolve<double>(c);
        else coarseSolve<float>(c);
        checkLaunch();
        BMG_CUDA(cudaStreamSynchronize(c->stream));
        return BMG_OK;
    });
}

}  // extern "C"
