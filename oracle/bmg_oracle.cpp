// bmg_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU restatement of the
// reference multigrid solve that the CUDA solver is checked against.  The
// file list it follows is in bmg_oracle.h.  Paths below are relative to the
// Briscola source tree; "FV/" abbreviates src/briscolaFiniteVolume/.

#include "bmg_oracle.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <thread>
#include <vector>

namespace {

// ---------------------------------------------------------------------------
// A small persistent thread pool.  The reference runs one rank per brick
// part; here threads split loops over i-planes inside one pass, which for
// single-colour passes, residuals and transfers leaves every value exactly
// as the sequential loop computes it.
// ---------------------------------------------------------------------------
class Pool {
public:
    explicit Pool(int n) : n_(std::max(1, n)) {
        for (int t = 1; t < n_; ++t)
            workers_.emplace_back([this, t] { loop(t); });
    }
    ~Pool() {
        {
            std::lock_guard<std::mutex> g(m_);
            stop_ = true;
            ++gen_;
        }
        cv_.notify_all();
        for (auto& w : workers_) w.join();
    }
    int size() const { return n_; }

    // f(begin, end) over [0, n) split into size() contiguous chunks
    void run(int n, const std::function<void(int, int)>& f) {
        if (n_ == 1 || n < 2 * n_ || n < 16) {
            f(0, n);
            return;
        }
        {
            std::lock_guard<std::mutex> g(m_);
            job_ = &f;
            jobN_ = n;
            pending_ = n_ - 1;
            ++gen_;
        }
        cv_.notify_all();
        chunk(0, n, f);
        std::unique_lock<std::mutex> lk(m_);
        done_.wait(lk, [this] { return pending_ == 0; });
        job_ = nullptr;
    }

private:
    void chunk(int t, int n, const std::function<void(int, int)>& f) {
        const int b = (int)((long)n * t / n_);
        const int e = (int)((long)n * (t + 1) / n_);
        if (b < e) f(b, e);
    }
    void loop(int t) {
        long seen = 0;
        for (;;) {
            const std::function<void(int, int)>* job;
            int n;
            {
                std::unique_lock<std::mutex> lk(m_);
                cv_.wait(lk, [&] { return gen_ != seen; });
                seen = gen_;
                if (stop_) return;
                job = job_;
                n = jobN_;
            }
            chunk(t, n, *job);
            {
                std::lock_guard<std::mutex> g(m_);
                if (--pending_ == 0) done_.notify_one();
            }
        }
    }

    int n_;
    std::vector<std::thread> workers_;
    std::mutex m_;
    std::condition_variable cv_, done_;
    const std::function<void(int, int)>* job_ = nullptr;
    int jobN_ = 0;
    int pending_ = 0;
    long gen_ = 0;
    bool stop_ = false;
};

// utils.H:1152-1170: halve every dimension larger than 3
inline void coarsen(const int N[3], int Nc[3]) {
    for (int d = 0; d < 3; ++d) Nc[d] = N[d] <= 3 ? N[d] : N[d] / 2;
}

struct Level {
    int N[3];
    int R[3];            // ratio parent/this level (1 or 2); 1 on level 0
    int S[3];            // shape including the ghost frame
    long Si, Sj;         // strides of i and j (k is contiguous)
    std::vector<double> pts[3];  // N+3 points, entry p+1 holds point p (p = -1..N+1)
    std::vector<double> cc[3];   // N+2 centres, entry i+1 holds cell i (i = -1..N)
    std::vector<double> h[3];    // N+2 cell sizes, same indexing
    std::vector<double> A;       // 7 coefficients per (ghost-framed) cell
    std::vector<double> x, b, r;
    std::vector<double> lam[3];  // face lambda on lower faces, ghost-framed indexing

    long cells() const { return (long)S[0] * S[1] * S[2]; }
    long n_interior() const { return (long)N[0] * N[1] * N[2]; }
    // index from ghost-inclusive coordinates (0..N+1)
    long gidx(int i, int j, int k) const { return ((long)i * S[1] + j) * S[2] + k; }
    // index from interior coordinates (-1..N)
    long at(int i, int j, int k) const { return gidx(i + 1, j + 1, k + 1); }
    double ccen(int d, int i) const { return cc[d][i + 1]; }
    double hsz(int d, int i) const { return h[d][i + 1]; }
};

}  // namespace

struct bmgo_problem {
    std::vector<Level> lv;
    int periodic[3];
    int dirichlet[6] = {0, 0, 0, 0, 0, 0};  // walls with a Dirichlet condition
    double dval[6] = {0, 0, 0, 0, 0, 0};    // their (uniform) boundary values
    std::vector<double> bdir;               // level-0 right-hand-side term of the Dirichlet values
    int restrictAverage = 0;                // restriction / prolongation schemes
    int prolongInjection = 0;
    bool variable = false;
    Pool pool;
    int coarseLevelIdx = -1;  // level index that carries the pin
    explicit bmgo_problem(int nt) : pool(nt) {}
    // linearSystem.H:227-230, meshLevel.C:555-583: singular unless a wall
    // carries a Dirichlet condition
    bool singular() const {
        for (int f = 0; f < 6; ++f)
            if (dirichlet[f]) return false;
        return true;
    }
};

namespace {

using P = bmgo_problem;

// levelPoints.C:198-236 (face ghost points projected by one spacing) and
// levelPoints.C:326-400 (periodic ghost points from the opposite spacing)
void setGhostPoints(Level& L, const int periodic[3]) {
    for (int d = 0; d < 3; ++d) {
        std::vector<double>& p = L.pts[d];
        const int N = L.N[d];
        // p[q+1] = point q
        if (periodic[d]) {
            p[0] = p[1] - (p[N + 1] - p[N]);
            p[N + 2] = p[N + 1] + (p[2] - p[1]);
        } else {
            p[0] = p[1] + (p[1] - p[2]);
            p[N + 2] = p[N + 1] + (p[N + 1] - p[N]);
        }
        L.cc[d].assign(N + 2, 0.0);
        L.h[d].assign(N + 2, 0.0);
        for (int i = -1; i <= N; ++i) {
            L.cc[d][i + 1] = 0.5 * (p[i + 1] + p[i + 2]);
            L.h[d][i + 1] = p[i + 2] - p[i + 1];
        }
    }
}

void allocLevel(Level& L) {
    for (int d = 0; d < 3; ++d) L.S[d] = L.N[d] + 2;
    L.Sj = L.S[2];
    L.Si = (long)L.S[1] * L.S[2];
    const long n = L.cells();
    L.A.assign(7 * n, 0.0);
    L.x.assign(n, 0.0);
    L.b.assign(n, 0.0);
    L.r.assign(n, 0.0);
}

// mesh.C:19-53 with level.H:144-147: add levels while coarsen(N) != N;
// coarse points are every R-th parent point (levelPoints.C:151-155).
void buildLevels(P& p, const int N[3], const double* pts[3]) {
    Level L0;
    for (int d = 0; d < 3; ++d) {
        L0.N[d] = N[d];
        L0.R[d] = 1;
        L0.pts[d].assign(N[d] + 3, 0.0);
        for (int q = 0; q <= N[d]; ++q) L0.pts[d][q + 1] = pts[d][q];
    }
    setGhostPoints(L0, p.periodic);
    allocLevel(L0);
    p.lv.push_back(std::move(L0));
    for (;;) {
        const Level& F = p.lv.back();
        int Nc[3];
        coarsen(F.N, Nc);
        if (Nc[0] == F.N[0] && Nc[1] == F.N[1] && Nc[2] == F.N[2]) break;
        Level C;
        for (int d = 0; d < 3; ++d) {
            C.N[d] = Nc[d];
            C.R[d] = F.N[d] / Nc[d];
            C.pts[d].assign(Nc[d] + 3, 0.0);
            for (int q = 0; q <= Nc[d]; ++q)
                C.pts[d][q + 1] = F.pts[d][q * C.R[d] + 1];
        }
        setGhostPoints(C, p.periodic);
        allocLevel(C);
        p.lv.push_back(std::move(C));
    }
}

// Ghost fill of a level field (meshLevel.C:231-253), axis by axis over
// growing extents: periodic images, zero-gradient copies at Neumann walls
// (NeumannBoundaryCondition.C evaluate with zero gradient) and the mirror
// H 2 g - x at Dirichlet walls (DirichletBoundaryCondition.C:59-80, H = 1 on
// level 0 only).  Edge and corner ghosts then hold the composition of the
// per-axis rules, which is what the reference's periodic edge boundaries
// give.  Where only walls meet (no periodic axis among them), the
// reference's unset-boundary copy of the diagonal interior cell
// (meshLevel.C:301-328) applies instead; it differs from the composition
// only where a Dirichlet wall takes part, so it is written over the
// composition there.
void fillGhostsAll(const P& p, const Level& L, std::vector<double>& f, int level) {
    const double H = level == 0 ? 1.0 : 0.0;
    int n[3] = {L.N[0], L.N[1], L.N[2]};
    int lo[3] = {0, 0, 0}, hi[3] = {n[0], n[1], n[2]};
    for (int d = 0; d < 3; ++d) {
        const int t1 = (d + 1) % 3, t2 = (d + 2) % 3;
        for (int u = lo[t1]; u < hi[t1]; ++u)
            for (int v = lo[t2]; v < hi[t2]; ++v)
                for (int side = 0; side < 2; ++side) {
                    int g[3], in[3];
                    g[t1] = in[t1] = u;
                    g[t2] = in[t2] = v;
                    g[d] = side ? n[d] : -1;
                    if (p.periodic[d])
                        in[d] = side ? 0 : n[d] - 1;
                    else
                        in[d] = side ? n[d] - 1 : 0;
                    const double val = f[L.at(in[0], in[1], in[2])];
                    if (!p.periodic[d] && p.dirichlet[2 * d + side])
                        f[L.at(g[0], g[1], g[2])] = H * 2.0 * p.dval[2 * d + side] - val;
                    else
                        f[L.at(g[0], g[1], g[2])] = val;
                }
        lo[d] = -1;
        hi[d] = n[d] + 1;
    }
    if (p.singular()) return;
    // wall-only edges and corners: copy of the diagonal interior cell
    for (int i = -1; i <= n[0]; ++i)
        for (int j = -1; j <= n[1]; ++j)
            for (int k = -1; k <= n[2]; ++k) {
                const int q[3] = {i, j, k};
                int out = 0;
                bool wallOnly = true;
                int in[3];
                for (int d = 0; d < 3; ++d) {
                    const bool o = q[d] < 0 || q[d] >= n[d];
                    out += o;
                    if (o && p.periodic[d]) wallOnly = false;
                    in[d] = std::min(std::max(q[d], 0), n[d] - 1);
                }
                if (out < 2 || !wallOnly) continue;
                f[L.at(i, j, k)] = f[L.at(in[0], in[1], in[2])];
            }
}

// periodicBoundaryCondition.C:53-92: same-rank periodic faces copy the
// boundary layer into the opposite ghost layer (face ghosts only, degree 1).
void evaluatePeriodicFaces(const P& p, const Level& L, std::vector<double>& f) {
    const int N0 = L.N[0], N1 = L.N[1], N2 = L.N[2];
    if (p.periodic[0])
        for (int j = 0; j < N1; ++j)
            for (int k = 0; k < N2; ++k) {
                f[L.at(N0, j, k)] = f[L.at(0, j, k)];
                f[L.at(-1, j, k)] = f[L.at(N0 - 1, j, k)];
            }
    if (p.periodic[1])
        for (int i = 0; i < N0; ++i)
            for (int k = 0; k < N2; ++k) {
                f[L.at(i, N1, k)] = f[L.at(i, 0, k)];
                f[L.at(i, -1, k)] = f[L.at(i, N1 - 1, k)];
            }
    if (p.periodic[2])
        for (int i = 0; i < N0; ++i)
            for (int j = 0; j < N1; ++j) {
                f[L.at(i, j, N2)] = f[L.at(i, j, 0)];
                f[L.at(i, j, -1)] = f[L.at(i, j, N2 - 1)];
            }
}

// areaWeightedFaceRestrictionScheme.C:19-57
void restrictLambda(P& p) {
    for (size_t l = 0; l + 1 < p.lv.size(); ++l) {
        const Level& F = p.lv[l];
        Level& C = p.lv[l + 1];
        for (int fd = 0; fd < 3; ++fd) {
            C.lam[fd].assign(C.cells(), 0.0);
            const int e0 = fd == 0, e1 = fd == 1, e2 = fd == 2;
            for (int I = 0; I < C.N[0] + e0; ++I)
                for (int J = 0; J < C.N[1] + e1; ++J)
                    for (int K = 0; K < C.N[2] + e2; ++K) {
                        double area = 0.0, value = 0.0;
                        for (int ox = 0; ox < (fd == 0 ? 1 : C.R[0]); ++ox)
                            for (int oy = 0; oy < (fd == 1 ? 1 : C.R[1]); ++oy)
                                for (int oz = 0; oz < (fd == 2 ? 1 : C.R[2]); ++oz) {
                                    const int fi = I * C.R[0] + ox;
                                    const int fj = J * C.R[1] + oy;
                                    const int fk = K * C.R[2] + oz;
                                    double a;
                                    if (fd == 0)
                                        a = F.hsz(1, fj) * F.hsz(2, fk);
                                    else if (fd == 1)
                                        a = F.hsz(0, fi) * F.hsz(2, fk);
                                    else
                                        a = F.hsz(0, fi) * F.hsz(1, fj);
                                    area += a;
                                    value += a * F.lam[fd][F.at(fi, fj, fk)];
                                }
                        C.lam[fd][C.at(I, J, K)] = value / area;
                    }
        }
    }
}

// linearGaussLaplacianScheme.C:59-94 with the face metrics of
// fvMeshMetrics.C:848-893 (delta = 1/|cc_P - cc_N|) on a rectilinear brick
// (face area = product of the two transverse cell sizes).
void assembleLevel(const P& p, Level& L) {
    std::fill(L.A.begin(), L.A.end(), 0.0);
    const long off[3] = {L.Si, L.Sj, 1};
    for (int fd = 0; fd < 3; ++fd) {
        const int e0 = fd == 0, e1 = fd == 1, e2 = fd == 2;
        for (int i = 0; i < L.N[0] + e0; ++i)
            for (int j = 0; j < L.N[1] + e1; ++j)
                for (int k = 0; k < L.N[2] + e2; ++k) {
                    const int ijk[3] = {i, j, k};
                    const double fa = fd == 0   ? L.hsz(1, j) * L.hsz(2, k)
                                      : fd == 1 ? L.hsz(0, i) * L.hsz(2, k)
                                                : L.hsz(0, i) * L.hsz(1, j);
                    const double dc = L.ccen(fd, ijk[fd]) - L.ccen(fd, ijk[fd] - 1);
                    const double delta = 1.0 / std::fabs(dc);
                    double value = fa * delta;
                    if (p.variable) value = fa * delta * L.lam[fd][L.at(i, j, k)];
                    const long c = L.at(i, j, k);
                    const long n = c - off[fd];
                    L.A[7 * c + 2 * fd + 1] = value;
                    L.A[7 * n + 2 * fd + 2] = value;
                    L.A[7 * c] -= value;
                    L.A[7 * n] -= value;
                }
    }
}

// Wall elimination (linearSystem.C:326-341): NeumannBoundaryCondition.C:19-56
// folds the ghost coefficient into the centre, DirichletBoundaryCondition.C
// :19-51 subtracts it; both drop it.  On level 0 the face values enter the
// right-hand side, -2 A_f g (Dirichlet value g) or -A_f g / delta (Neumann
// gradient g), kept in bdir and added to b at every solve.
void eliminateWalls(P& p, Level& L, int level) {
    if (level == 0) p.bdir.assign(L.cells(), 0.0);
    for (int f = 0; f < 6; ++f) {
        const int fd = f / 2;
        if (p.periodic[fd]) continue;
        const bool dir = p.dirichlet[f] != 0;
        const int lo[3] = {0, 0, 0};
        int S[3] = {lo[0], lo[1], lo[2]};
        int E[3] = {L.N[0], L.N[1], L.N[2]};
        if (f % 2 == 0)
            E[fd] = 1;
        else
            S[fd] = L.N[fd] - 1;
        for (int i = S[0]; i < E[0]; ++i)
            for (int j = S[1]; j < E[1]; ++j)
                for (int k = S[2]; k < E[2]; ++k) {
                    const long c = L.at(i, j, k);
                    const double g = L.A[7 * c + f + 1];
                    if (dir) {
                        L.A[7 * c] -= g;
                        if (level == 0) p.bdir[c] -= g * 2.0 * p.dval[f];
                    } else {
                        L.A[7 * c] += g;
                        // NeumannBoundaryCondition.C:44-50: b -= A_f grad / delta,
                        // delta of the wall face = 1 / (centre - ghost centre)
                        if (level == 0 && p.dval[f] != 0.0) {
                            const int ijk[3] = {i, j, k};
                            const int gq = ijk[fd] + (f % 2 ? 1 : -1);
                            const double dist = std::fabs(L.ccen(fd, ijk[fd]) - L.ccen(fd, gq));
                            p.bdir[c] -= g * p.dval[f] * dist;
                        }
                    }
                    L.A[7 * c + f + 1] = 0.0;
                }
    }
}

// neighbour (interior or ghost) of interior cell (i,j,k) through stencil
// slot s mapped to its interior cell number, or -1 across a wall
long neighbourNumber(const P& p, const Level& L, int i, int j, int k, int s) {
    int c[3] = {i, j, k};
    const int fd = (s - 1) / 2;
    c[fd] += (s % 2 == 1) ? -1 : 1;
    if (c[fd] < 0 || c[fd] >= L.N[fd]) {
        if (!p.periodic[fd]) return -1;
        c[fd] = (c[fd] + L.N[fd]) % L.N[fd];
    }
    return ((long)c[0] * L.N[1] + c[1]) * L.N[2] + c[2];
}

// solver.C:201-231: pin global cell 0 on the coarse solve level
void setSingularityConstraint(const P& p, Level& L) {
    const long c0 = L.at(0, 0, 0);
    for (int s = 0; s < 7; ++s) L.A[7 * c0 + s] = s == 0 ? 1.0 : 0.0;
    for (int i = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) {
                const long c = L.at(i, j, k);
                for (int s = 1; s < 7; ++s)
                    if (L.A[7 * c + s] != 0.0 && neighbourNumber(p, L, i, j, k, s) == 0)
                        L.A[7 * c + s] = 0.0;
            }
}

// linearSystemFunctions.H:82-104
inline double offDiag(const double* A, const double* x, long c, long Si, long Sj) {
    return A[c * 7 + 1] * x[c - Si] + A[c * 7 + 2] * x[c + Si] + A[c * 7 + 3] * x[c - Sj] +
           A[c * 7 + 4] * x[c + Sj] + A[c * 7 + 5] * x[c - 1] + A[c * 7 + 6] * x[c + 1];
}
// linearSystemFunctions.H:28-51
inline double rowProd(const double* A, const double* x, long c, long Si, long Sj) {
    return A[c * 7] * x[c] + A[c * 7 + 1] * x[c - Si] + A[c * 7 + 2] * x[c + Si] +
           A[c * 7 + 3] * x[c - Sj] + A[c * 7 + 4] * x[c + Sj] + A[c * 7 + 5] * x[c - 1] +
           A[c * 7 + 6] * x[c + 1];
}

// One of the four passes of rbgsSmoother.C:65-183 over the ghost-inclusive
// region [S,E): loop-counter parity `want` (0 even, 1 odd); forward counters
// start at S, backward counters at E-1.  Cells of one parity do not couple,
// so splitting the i loop over threads keeps every value.
void rbgsPass(P& p, Level& L, const int S[3], const int E[3], int want, bool backward) {
    double* x = L.x.data();
    const double* b = L.b.data();
    const double* A = L.A.data();
    const long Si = L.Si, Sj = L.Sj;
    p.pool.run(E[0] - S[0], [&](int ib, int ie) {
        for (int ci = S[0] + ib; ci < S[0] + ie; ++ci)
            for (int cj = S[1]; cj < E[1]; ++cj)
                for (int ck = S[2]; ck < E[2]; ++ck) {
                    const int par = backward ? ((E[0] - 1 - ci) + (E[1] - 1 - cj) + (E[2] - 1 - ck)) & 1
                                             : ((ci - S[0]) + (cj - S[1]) + (ck - S[2])) & 1;
                    if (par != want) continue;
                    const long c = L.gidx(ci, cj, ck);
                    x[c] = (b[c] - offDiag(A, x, c, Si, Sj)) / A[c * 7];
                }
    });
}

void rbgsRegion(P& p, Level& L, const int S[3], const int E[3]) {
    if (S[0] >= E[0] || S[1] >= E[1] || S[2] >= E[2]) return;
    rbgsPass(p, L, S, E, 0, false);
    rbgsPass(p, L, S, E, 1, false);
    rbgsPass(p, L, S, E, 0, true);
    rbgsPass(p, L, S, E, 1, true);
}

// jacSmoother.C:18-127 on one ghost-inclusive region
void jacRegion(P& p, Level& L, const int S[3], const int E[3]) {
    if (S[0] >= E[0] || S[1] >= E[1] || S[2] >= E[2]) return;
    const double omega = 0.8;
    const int M[3] = {E[0] - S[0], E[1] - S[1], E[2] - S[2]};
    std::vector<double> y((size_t)M[0] * M[1] * M[2]);
    double* x = L.x.data();
    const double* b = L.b.data();
    const double* A = L.A.data();
    const long Si = L.Si, Sj = L.Sj;
    p.pool.run(M[0], [&](int ib, int ie) {
        for (int i = ib; i < ie; ++i)
            for (int j = 0; j < M[1]; ++j)
                for (int k = 0; k < M[2]; ++k) {
                    const long c = L.gidx(S[0] + i, S[1] + j, S[2] + k);
                    y[((size_t)i * M[1] + j) * M[2] + k] =
                        (1.0 - omega) * x[c] + omega * (b[c] - offDiag(A, x, c, Si, Sj)) / A[c * 7];
                }
    });
    p.pool.run(M[0], [&](int ib, int ie) {
        for (int i = ib; i < ie; ++i)
            for (int j = 0; j < M[1]; ++j)
                for (int k = 0; k < M[2]; ++k)
                    x[L.gidx(S[0] + i, S[1] + j, S[2] + k)] = y[((size_t)i * M[1] + j) * M[2] + k];
    });
}

// rbgsSmoother.C:377-437 / jacSmoother.C:285-321: interior sweep padded by
// one layer at non-eliminated (periodic) faces, periodic ghost evaluation,
// then one sweep per padded boundary layer (SweepBoundary).
void smoothLevel(P& p, int l, int smoother, int sweeps) {
    Level& L = p.lv[l];
    int pad[6];
    for (int f = 0; f < 6; ++f) pad[f] = p.periodic[f / 2] ? 1 : 0;
    for (int s = 0; s < sweeps; ++s) {
        int S[3], E[3];
        for (int d = 0; d < 3; ++d) {
            S[d] = 1 + pad[2 * d];
            E[d] = 1 + L.N[d] - pad[2 * d + 1];
        }
        if (smoother == 0)
            rbgsRegion(p, L, S, E);
        else
            jacRegion(p, L, S, E);
        evaluatePeriodicFaces(p, L, L.x);
        for (int f = 0; f < 6; ++f) {
            if (!pad[f]) continue;
            const int fd = f / 2;
            int Sb[3], Eb[3];
            for (int d = 0; d < 3; ++d) {
                Sb[d] = 1;
                Eb[d] = 1 + L.N[d];
            }
            if (f % 2 == 0)
                Eb[fd] = Sb[fd] + 1;
            else
                Sb[fd] = Eb[fd] - 1;
            if (smoother == 0)
                rbgsRegion(p, L, Sb, Eb);
            else
                jacRegion(p, L, Sb, Eb);
        }
    }
}

// linearSystemResidual.C:13-130 + :280-332 with boundary correction; the
// interior/boundary split leaves values unchanged because x is read only.
void residualLevel(P& p, Level& L, bool corrBcs) {
    if (corrBcs) evaluatePeriodicFaces(p, L, L.x);
    double* r = L.r.data();
    const double* x = L.x.data();
    const double* b = L.b.data();
    const double* A = L.A.data();
    const long Si = L.Si, Sj = L.Sj;
    p.pool.run(L.N[0], [&](int ib, int ie) {
        for (int i = ib; i < ie; ++i)
            for (int j = 0; j < L.N[1]; ++j)
                for (int k = 0; k < L.N[2]; ++k) {
                    const long c = L.at(i, j, k);
                    r[c] = b[c] - rowProd(A, x, c, Si, Sj);
                }
    });
}

// per-axis trilinear weight: local coordinate of point q between centres
// a (weight 1-w) and b (weight w); interpolationWeights() on an axis-aligned
// hexahedron reduces to this on every axis.
inline double axisWeight(double q, double a, double b) { return (q - a) / (b - a); }

// linearRestrictionScheme.C:15-80 (weights) and :103-187 (restrict)
void restrictLevel(P& p, int lf, const std::vector<double>& fine, std::vector<double>& coarse,
                   bool scale) {
    const Level& F = p.lv[lf];
    const Level& C = p.lv[lf + 1];
    const int R0 = C.R[0], R1 = C.R[1], R2 = C.R[2];
    const int ox = R0 > 1, oy = R1 > 1, oz = R2 > 1;
    p.pool.run(C.N[0], [&](int Ib, int Ie) {
        for (int I = Ib; I < Ie; ++I)
            for (int J = 0; J < C.N[1]; ++J)
                for (int K = 0; K < C.N[2]; ++K) {
                    // averageRestrictionScheme.C:35-77: the children's mean
                    // (weight 1/2 per coarsened axis)
                    const bool avg = p.restrictAverage != 0;
                    const double wx = avg ? 0.5 : axisWeight(C.ccen(0, I), F.ccen(0, I * R0), F.ccen(0, I * R0 + 1));
                    const double wy = avg ? 0.5 : axisWeight(C.ccen(1, J), F.ccen(1, J * R1), F.ccen(1, J * R1 + 1));
                    const double wz = avg ? 0.5 : axisWeight(C.ccen(2, K), F.ccen(2, K * R2), F.ccen(2, K * R2 + 1));
                    double w[8] = {(1.0 - wx) * (1.0 - wy) * (1.0 - wz), (wx) * (1.0 - wy) * (1.0 - wz),
                                   (1.0 - wx) * (wy) * (1.0 - wz),       (wx) * (wy) * (1.0 - wz),
                                   (1.0 - wx) * (1.0 - wy) * (wz),       (wx) * (1.0 - wy) * (wz),
                                   (1.0 - wx) * (wy) * (wz),             (wx) * (wy) * (wz)};
                    for (int q = 0; q < 8; ++q)
                        if (w[q] <= 1e-12) w[q] = 0.0;
                    double v = 0.0;
                    int q = 0;
                    for (int c = 0; c < 2; ++c)
                        for (int bb = 0; bb < 2; ++bb)
                            for (int a = 0; a < 2; ++a) {
                                const double wq = w[q++];
                                if (wq == 0.0) continue;
                                const int fi = I * R0 + a * ox, fj = J * R1 + bb * oy, fk = K * R2 + c * oz;
                                if (scale) {
                                    const double icv =
                                        1.0 / (F.hsz(0, fi) * F.hsz(1, fj) * F.hsz(2, fk));
                                    v += wq * fine[F.at(fi, fj, fk)] * icv;
                                } else {
                                    v += wq * fine[F.at(fi, fj, fk)];
                                }
                            }
                    if (scale) v *= C.hsz(0, I) * C.hsz(1, J) * C.hsz(2, K);
                    coarse[C.at(I, J, K)] = v;
                }
    });
}

// linearProlongationScheme.C:12-110 (weights and indices) and :112-147
void prolongLevel(P& p, int lf, std::vector<double>& coarse, std::vector<double>& fine, int op,
                  bool fillGhosts = true) {
    const Level& F = p.lv[lf];
    const Level& C = p.lv[lf + 1];
    if (fillGhosts) fillGhostsAll(p, C, coarse, lf + 1);
    const int R0 = C.R[0], R1 = C.R[1], R2 = C.R[2];
    p.pool.run(F.N[0], [&](int ib, int ie) {
        for (int i = ib; i < ie; ++i)
            for (int j = 0; j < F.N[1]; ++j)
                for (int k = 0; k < F.N[2]; ++k) {
                    const int o0 = i % 2 ? 1 : -1, o1 = j % 2 ? 1 : -1, o2 = k % 2 ? 1 : -1;
                    const int I = i / R0, J = j / R1, K = k / R2;
                    // injectionProlongationScheme.C:14-33: the parent's value
                    const bool inj = p.prolongInjection != 0;
                    const double wx = inj ? 0.0 : axisWeight(F.ccen(0, i), C.ccen(0, I), C.ccen(0, I + o0));
                    const double wy = inj ? 0.0 : axisWeight(F.ccen(1, j), C.ccen(1, J), C.ccen(1, J + o1));
                    const double wz = inj ? 0.0 : axisWeight(F.ccen(2, k), C.ccen(2, K), C.ccen(2, K + o2));
                    double v = 0.0;
                    for (int c = 0; c < 2; ++c)
                        for (int bb = 0; bb < 2; ++bb)
                            for (int a = 0; a < 2; ++a) {
                                const double w = (1.0 - a + wx * (2 * a - 1)) * (1.0 - bb + wy * (2 * bb - 1)) *
                                                 (1.0 - c + wz * (2 * c - 1));
                                if (w != 0.0) v += w * coarse[C.at(I + a * o0, J + bb * o1, K + c * o2)];
                            }
                    double& t = fine[F.at(i, j, k)];
                    if (op == 0)
                        t = v;
                    else
                        t += v;
                }
    });
}

// APLU.C:26-128: the coarse level gathered into a dense matrix, factored
// with partial pivoting and back-substituted.
struct DenseLU {
    int n = 0;
    std::vector<double> M;
    std::vector<int> piv;
    void factor() {
        piv.resize(n);
        for (int k = 0; k < n; ++k) {
            int pr = k;
            double best = std::fabs(M[(size_t)k * n + k]);
            for (int i = k + 1; i < n; ++i)
                if (std::fabs(M[(size_t)i * n + k]) > best) {
                    best = std::fabs(M[(size_t)i * n + k]);
                    pr = i;
                }
            piv[k] = pr;
            if (pr != k)
                for (int j = 0; j < n; ++j) std::swap(M[(size_t)k * n + j], M[(size_t)pr * n + j]);
            const double d = M[(size_t)k * n + k];
            for (int i = k + 1; i < n; ++i) {
                const double f = M[(size_t)i * n + k] / d;
                M[(size_t)i * n + k] = f;
                if (f != 0.0)
                    for (int j = k + 1; j < n; ++j) M[(size_t)i * n + j] -= f * M[(size_t)k * n + j];
            }
        }
    }
    void solve(std::vector<double>& v) const {
        for (int k = 0; k < n; ++k) {
            std::swap(v[k], v[piv[k]]);
            for (int i = k + 1; i < n; ++i) v[i] -= M[(size_t)i * n + k] * v[k];
        }
        for (int i = n - 1; i >= 0; --i) {
            double s = v[i];
            for (int j = i + 1; j < n; ++j) s -= M[(size_t)i * n + j] * v[j];
            v[i] = s / M[(size_t)i * n + i];
        }
    }
};

DenseLU buildCoarseLU(const P& p, const Level& L) {
    DenseLU lu;
    lu.n = (int)L.n_interior();
    lu.M.assign((size_t)lu.n * lu.n, 0.0);
    for (int i = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) {
                const long row = ((long)i * L.N[1] + j) * L.N[2] + k;
                const long c = L.at(i, j, k);
                lu.M[(size_t)row * lu.n + row] += L.A[7 * c];
                for (int s = 1; s < 7; ++s) {
                    const double a = L.A[7 * c + s];
                    if (a == 0.0) continue;
                    const long col = neighbourNumber(p, L, i, j, k, s);
                    if (col >= 0) lu.M[(size_t)row * lu.n + col] += a;
                }
            }
    lu.factor();
    return lu;
}

void coarseSolve(Level& L, const DenseLU& lu) {
    std::vector<double> v(lu.n);
    for (int i = 0, q = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) v[q++] = L.b[L.at(i, j, k)];
    lu.solve(v);
    for (int i = 0, q = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) L.x[L.at(i, j, k)] = v[q++];
}

// plane-ordered sums: deterministic for any thread count
template <class F>
double planeSum(P& p, const Level& L, F f) {
    std::vector<double> part(L.N[0], 0.0);
    p.pool.run(L.N[0], [&](int ib, int ie) {
        for (int i = ib; i < ie; ++i) {
            double s = 0.0;
            for (int j = 0; j < L.N[1]; ++j)
                for (int k = 0; k < L.N[2]; ++k) s += f(L.at(i, j, k));
            part[i] = s;
        }
    });
    double s = 0.0;
    for (double v : part) s += v;
    return s;
}

struct Solver {
    P& p;
    bmgo_options o;
    int coarseLevel;  // absolute level index of the coarse solve
    DenseLU lu;
    std::vector<int> visits;

    int levelReps(int l) const {  // MG.H:106-124
        if (o.cycle_type == 0) return 1;
        if (o.cycle_type == 1) return 1 + (l > 0);
        return 1 + (l > 0 && visits[l] == 0);
    }

    // MG.C:19-130
    void cycle(int l) {
        Level& L = p.lv[l];
        if (l == coarseLevel && p.singular()) L.b[L.at(0, 0, 0)] = 0.0;
        if (l > 0) std::fill(L.x.begin(), L.x.end(), 0.0);
        if (o.n_pre > 0) smoothLevel(p, l, o.smoother, o.n_pre);
        if (l < coarseLevel) {
            Level& C = p.lv[l + 1];
            const int reps = levelReps(l);
            for (int rep = 0; rep < reps; ++rep) {
                if (rep > 0 || l > 0 || !o.stale_residual) residualLevel(p, L, true);
                restrictLevel(p, l, L.r, C.b, true);
                cycle(l + 1);
                prolongLevel(p, l, C.x, L.x, 1);
                if (o.n_post > 0) smoothLevel(p, l, o.smoother, o.n_post);
            }
        } else {
            if (o.coarse_direct)
                coarseSolve(L, lu);
            else
                smoothLevel(p, l, o.smoother, std::max(o.n_post, 2));
        }
        visits[l]++;
    }
};

int absCoarseLevel(const P& p, const bmgo_options& o) {
    return (int)p.lv.size() - o.coarse_level - 1;
}

void assembleAll(P& p, const bmgo_options& o) {
    p.restrictAverage = o.restrict_average;
    p.prolongInjection = o.prolong_injection;
    const int lc = absCoarseLevel(p, o);
    for (size_t l = 0; l < p.lv.size(); ++l) assembleLevel(p, p.lv[l]);
    // MG.C:431-445: pin first (solver.C:201-231), then eliminate ghosts
    if (lc >= 0 && lc < (int)p.lv.size() && p.singular()) setSingularityConstraint(p, p.lv[lc]);
    for (size_t l = 0; l < p.lv.size(); ++l) eliminateWalls(p, p.lv[l], (int)l);
    p.coarseLevelIdx = lc;
}

void copyIn(const Level& L, const double* src, std::vector<double>& dst) {
    for (int i = 0, q = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) dst[L.at(i, j, k)] = src[q++];
}
void copyOut(const Level& L, const std::vector<double>& src, double* dst) {
    for (int i = 0, q = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) dst[q++] = src[L.at(i, j, k)];
}

}  // namespace

extern "C" {

void bmgo_default_options(bmgo_options* o) {
    o->rel_tol = 1e-10;
    o->abs_tol = 0.0;
    o->min_iter = 0;
    o->max_iter = 999;
    o->n_pre = 0;
    o->n_post = 2;
    o->cycle_type = 2;
    o->coarse_level = 0;
    o->coarse_direct = 1;
    o->smoother = 0;
    o->stale_residual = 1;
    o->restrict_average = 0;
    o->prolong_injection = 0;
}

bmgo_problem* bmgo_create(const int N[3], const double* px, const double* py, const double* pz,
                          const int periodic[3], int nthreads) {
    if (nthreads <= 0) nthreads = (int)std::max(1u, std::thread::hardware_concurrency());
    bmgo_problem* p = new bmgo_problem(nthreads);
    for (int d = 0; d < 3; ++d) p->periodic[d] = periodic[d] != 0;
    const double* pts[3] = {px, py, pz};
    buildLevels(*p, N, pts);
    return p;
}

int bmgo_set_faces(bmgo_problem* p, const int dirichlet[6], const double value[6]) {
    for (int f = 0; f < 6; ++f)
        if ((dirichlet[f] || (value && value[f] != 0.0)) && p->periodic[f / 2]) return -1;
    for (int f = 0; f < 6; ++f) {
        p->dirichlet[f] = dirichlet[f] != 0;
        p->dval[f] = value ? value[f] : 0.0;
    }
    return 0;
}

void bmgo_destroy(bmgo_problem* p) { delete p; }

int bmgo_num_levels(const bmgo_problem* p) { return (int)p->lv.size(); }

void bmgo_level_shape(const bmgo_problem* p, int l, int N[3]) {
    for (int d = 0; d < 3; ++d) N[d] = p->lv[l].N[d];
}

void bmgo_level_ratio(const bmgo_problem* p, int l, int R[3]) {
    for (int d = 0; d < 3; ++d) R[d] = p->lv[l + 1].R[d];
}

void bmgo_cell_centres(const bmgo_problem* p, int l, int axis, double* out) {
    const Level& L = p->lv[l];
    for (int i = 0; i < L.N[axis] + 2; ++i) out[i] = L.cc[axis][i];
}

void bmgo_cell_volumes(const bmgo_problem* p, int l, double* out) {
    const Level& L = p->lv[l];
    long q = 0;
    for (int i = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) out[q++] = L.hsz(0, i) * L.hsz(1, j) * L.hsz(2, k);
}

void bmgo_set_lambda(bmgo_problem* p, const double* lx, const double* ly, const double* lz) {
    if (!lx || !ly || !lz) {
        p->variable = false;
        for (auto& L : p->lv)
            for (int d = 0; d < 3; ++d) L.lam[d].clear();
        return;
    }
    p->variable = true;
    Level& L = p->lv[0];
    const double* src[3] = {lx, ly, lz};
    for (int fd = 0; fd < 3; ++fd) {
        L.lam[fd].assign(L.cells(), 0.0);
        const int e0 = fd == 0, e1 = fd == 1, e2 = fd == 2;
        long q = 0;
        for (int i = 0; i < L.N[0] + e0; ++i)
            for (int j = 0; j < L.N[1] + e1; ++j)
                for (int k = 0; k < L.N[2] + e2; ++k) L.lam[fd][L.at(i, j, k)] = src[fd][q++];
    }
    restrictLambda(*p);
}

void bmgo_get_lambda(const bmgo_problem* p, int l, int fd, double* out) {
    const Level& L = p->lv[l];
    const int e0 = fd == 0, e1 = fd == 1, e2 = fd == 2;
    long q = 0;
    for (int i = 0; i < L.N[0] + e0; ++i)
        for (int j = 0; j < L.N[1] + e1; ++j)
            for (int k = 0; k < L.N[2] + e2; ++k) out[q++] = L.lam[fd][L.at(i, j, k)];
}

void bmgo_assemble(bmgo_problem* p, const bmgo_options* o) { assembleAll(*p, *o); }

void bmgo_get_matrix(const bmgo_problem* p, int l, double* out7) {
    const Level& L = p->lv[l];
    long q = 0;
    for (int i = 0; i < L.N[0]; ++i)
        for (int j = 0; j < L.N[1]; ++j)
            for (int k = 0; k < L.N[2]; ++k) {
                const long c = L.at(i, j, k);
                for (int s = 0; s < 7; ++s) out7[q++] = L.A[7 * c + s];
            }
}

// MG.C:402-483 (solve) and MG.C:132-254 (Solve)
int bmgo_solve(bmgo_problem* pp, const bmgo_options* o, const double* b, double* x, bmgo_report* rep,
               double* history, int max_hist) {
    P& p = *pp;
    Solver s{p, *o, absCoarseLevel(p, *o), {}, {}};
    if (s.coarseLevel < 0 || s.coarseLevel > (int)p.lv.size() - 1) return -1;
    assembleAll(p, *o);
    if (o->coarse_direct) s.lu = buildCoarseLU(p, p.lv[s.coarseLevel]);
    Level& L0 = p.lv[0];
    for (auto& L : p.lv) {
        std::fill(L.x.begin(), L.x.end(), 0.0);
        std::fill(L.b.begin(), L.b.end(), 0.0);
        std::fill(L.r.begin(), L.r.end(), 0.0);
    }
    copyIn(L0, b, L0.b);
    for (long c = 0; c < L0.cells(); ++c) L0.b[c] += p.bdir[c];
    copyIn(L0, x, L0.x);
    fillGhostsAll(p, L0, L0.x, 0);

    residualLevel(p, L0, false);  // initial residual without boundary correction

    // solver.C:13-61
    const double nCells = (double)L0.n_interior();
    const double ybar = planeSum(p, L0, [&](long c) { return L0.x[c]; }) / nCells;
    double nf = std::sqrt(planeSum(p, L0, [&](long c) {
        double rs = 0.0;
        for (int q = 0; q < 7; ++q) rs += L0.A[7 * c + q];
        const double Ay = rs * ybar;
        const double t = std::fabs(L0.r[c] - L0.b[c] + Ay) + std::fabs(L0.b[c] - Ay);
        return t * t;
    }));
    nf = std::max(nf, nCells * 1e-12);
    const double bl2 = std::sqrt(planeSum(p, L0, [&](long c) { return L0.b[c] * L0.b[c]; }));

    auto l2r = [&]() { return std::sqrt(planeSum(p, L0, [&](long c) { return L0.r[c] * L0.r[c]; })); };
    double rl2 = l2r();
    const double init = rl2 / nf;
    double cur = init;
    // solver.C:64-95
    auto conv = [&](double c) {
        return !((init > 0.0) && (c > o->abs_tol) && (c / (init + 1e-20) > o->rel_tol));
    };
    bool converged = conv(cur);
    int iter = 0;
    s.visits.assign(p.lv.size(), 0);
    while ((iter < o->max_iter && !converged) || iter < o->min_iter) {
        std::fill(s.visits.begin(), s.visits.end(), 0);
        s.cycle(0);
        residualLevel(p, L0, true);
        rl2 = l2r();
        cur = rl2 / nf;
        converged = conv(cur);
        if (history && iter < max_hist) history[iter] = cur;
        ++iter;
    }
    copyOut(L0, L0.x, x);
    if (rep) {
        rep->iterations = iter;
        rep->initial_residual = init;
        rep->final_residual = cur;
        rep->norm_factor = nf;
        rep->final_l2 = rl2;
        rep->b_l2 = bl2;
    }
    return converged ? 0 : 1;
}

void bmgo_residual(bmgo_problem* p, int l, const double* x, const double* b, double* r) {
    Level& L = p->lv[l];
    std::fill(L.x.begin(), L.x.end(), 0.0);
    copyIn(L, x, L.x);
    copyIn(L, b, L.b);
    fillGhostsAll(*p, L, L.x, l);
    residualLevel(*p, L, true);
    copyOut(L, L.r, r);
}

void bmgo_smooth(bmgo_problem* p, int l, int smoother, int sweeps, double* x, const double* b) {
    Level& L = p->lv[l];
    std::fill(L.x.begin(), L.x.end(), 0.0);
    copyIn(L, x, L.x);
    copyIn(L, b, L.b);
    fillGhostsAll(*p, L, L.x, l);
    smoothLevel(*p, l, smoother, sweeps);
    copyOut(L, L.x, x);
}

void bmgo_colour_pass(bmgo_problem* p, int l, int colour, double* x, const double* b) {
    Level& L = p->lv[l];
    std::fill(L.x.begin(), L.x.end(), 0.0);
    copyIn(L, x, L.x);
    copyIn(L, b, L.b);
    fillGhostsAll(*p, L, L.x, l);
    const int S[3] = {1, 1, 1};
    const int E[3] = {1 + L.N[0], 1 + L.N[1], 1 + L.N[2]};
    rbgsPass(*p, L, S, E, colour, false);
    copyOut(L, L.x, x);
}

void bmgo_restrict(bmgo_problem* p, int lf, const double* fine, double* coarse, int scale) {
    Level& F = p->lv[lf];
    Level& C = p->lv[lf + 1];
    copyIn(F, fine, F.r);
    restrictLevel(*p, lf, F.r, C.b, scale != 0);
    copyOut(C, C.b, coarse);
}

void bmgo_prolong(bmgo_problem* p, int lf, const double* coarse, double* fine, int op) {
    Level& F = p->lv[lf];
    Level& C = p->lv[lf + 1];
    std::fill(C.x.begin(), C.x.end(), 0.0);
    copyIn(C, coarse, C.x);
    copyIn(F, fine, F.x);
    prolongLevel(*p, lf, C.x, F.x, op);
    copyOut(F, F.x, fine);
}

void bmgo_prolong_ghosted(bmgo_problem* p, int lf, const double* coarse_g, double* fine, int op) {
    Level& F = p->lv[lf];
    Level& C = p->lv[lf + 1];
    std::copy(coarse_g, coarse_g + C.cells(), C.x.begin());
    copyIn(F, fine, F.x);
    prolongLevel(*p, lf, C.x, F.x, op, false);
    copyOut(F, F.x, fine);
}

void bmgo_coarse_solve(bmgo_problem* p, int l, const double* b, double* x) {
    Level& L = p->lv[l];
    DenseLU lu = buildCoarseLU(*p, L);
    copyIn(L, b, L.b);
    coarseSolve(L, lu);
    copyOut(L, L.x, x);
}

}  // extern "C"
