// bmg_internal.h -- device-side views and kernel launchers of the B200
// multigrid solver.  Host driver: bmg_host.cu.  Kernels: bmg_kernels.cu,
// bmg_smooth_fused.cu.
//
// Data layout in HBM (per level):
//   all bricks of a level live in one slab per field.  Each brick is a
//   ghost-framed block of (n0+2) x (n1+2) x p2 values, k fastest (the
//   reference's lin(), utils.H:569, with its one-cell ghost frame,
//   meshDirection.H:35); rows are padded to p2 = round_up(n2 + 5, 4) so that
//   interior rows start on 16-byte (FP32) / 32-byte (FP64) boundaries.
//   Interior cell (i,j,k) of a brick sits at base + i*si + j*sj + k.
//   Compact (interior-only) arrays list the bricks one after another, each
//   k fastest, as the C ABI does.
//
// Parity-split rows (LevelView::kh > 0, single-brick levels above
// kTailCells cells with n2 % 16 == 0): the interior of every row is stored
// as its n2/2 even-k cells followed by its n2/2 odd-k cells, so cell
// (i,j,k) sits at base + i*si + j*sj + kpos(k), kpos(k) = (k & 1) * kh +
// (k >> 1) with kh = n2/2.  In a row the even k have one red-black colour
// and the odd k the other, and the same-k cells of the neighbouring rows
// have the other colour of the same k parity: a colour pass reads and
// writes contiguous half-rows of one colour only (whole sectors, coalesced
// warp loads), where the natural order reads every sector of x and b to
// update half of them.  The k ghosts keep their natural places (k = -1 and
// k = n2), and so do the periodic images (a cell and its k image are n2
// apart in both orders).
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

namespace bmg {

constexpr int kMaxBricks = 8;

// ---- programmatic dependent launch (sm_90 and later) -------------------------
// The solve's kernels follow one another on one stream, each reading what the
// previous one wrote.  They are launched with programmatic stream
// serialization, and every one of them begins with grid_dep_sync(): it waits
// until the preceding grid has completed and its writes are visible
// (griddepcontrol.wait), then lets the next grid be scheduled
// (griddepcontrol.launch_dependents).  The next kernel's launch then
// overlaps this one's execution instead of following its completion; its
// CTAs take only the slots this grid leaves free and wait at their own
// grid_dep_sync.  After a kernel launched without the attribute, or after a
// memset or a copy, the wait returns at once.
__device__ __forceinline__ void grid_dep_sync() {
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
}

constexpr bool kProgrammaticLaunch = true;

template <typename... KArgs, typename... Args>
inline void launch_k(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                     Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = kProgrammaticLaunch ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kernel, static_cast<Args&&>(args)...);
}

// 1-D table offsets inside one level's coefficient table
struct TabOff {
    int wl[3];   // coupling to the lower neighbour, per cell along the axis
    int wh[3];   // coupling to the upper neighbour
    int h[3];    // cell sizes (volume factors)
    int kwl, kwh;  // parity-split levels: the k couplings in the row's storage
                   // order (entry kpos(k) holds wl[2] / wh[2] of k); -1 otherwise
    int ksz;       // ... and the cell sizes along k (h[2]) in the same order
    int total;
};

// One brick on one level.
template <typename T>
struct LevelView {
    int n0, n1, n2;
    long si, sj;       // strides of i and j (k contiguous)
    long base;         // slab index of interior cell (0,0,0)
    long cells;        // size of the whole slab (all bricks)
    long cbase;        // compact index of cell (0,0,0): with cs[], the caller's
    int cs[3];         // array index cbase + i*cs[0] + j*cs[1] + k*cs[2]
                       // (the brick's own frame, k fastest there)
    T* x;              // slab pointers
    T* b;
    const T* tab;      // 1-D tables (TabOff layout) in precision T
    const double* tab64;  // the same tables in FP64 (norms, volumes)
    TabOff to;
    const T* lam0;     // face lambda (lower face of the cell, ghost-framed
    const T* lam1;     // indexing), nullptr for a constant coefficient
    const T* lam2;
    int per0, per1, per2;  // periodic write-through (single brick only)
    int cpar;          // parity of the brick origin: colour = (i+j+k+cpar) & 1
    int pin;           // smoothers keep cell (0,0,0) at zero: the singularity pin
                       // of an iteratively smoothed coarse level (solver.C:201-231)
    int kh;            // parity-split rows: offset n2/2 of the odd-k half (see
                       // above); 0: natural k order
};

// Wall faces of a single-brick level 0: bit f of mask for a Dirichlet face
// f (x-lo, x-hi, y-lo, y-hi, z-lo, z-hi; DirichletBoundaryCondition.C:19-80),
// of nmask for a Neumann face with a nonzero gradient
// (NeumannBoundaryCondition.C:19-56), g the face values.  On every level the
// 1-D tables hold the eliminated coupling 2 A_f / V at Dirichlet faces and
// the ghost cells stay zero, so each stencil kernel applies the eliminated
// operator as it is; only the right-hand side (b -= 2 A_f g, or A_f g /
// delta) and the normFactor's A*mean(x) term (solver.C:28-45) need the faces
// themselves.  ybar: the plain mean of the initial x (SolveState::ybar).
// Both masks are 0 on coarse levels.
// Face values of the level-0 bricks: per brick, bit f of mask marks a
// Dirichlet face, bit f of nmask a Neumann face with a nonzero gradient,
// g[b][f] the value or gradient
struct Walls {
    int mask[kMaxBricks];
    int nmask[kMaxBricks];
    double g[kMaxBricks][6];
    const double* ybar;
};

// All bricks of a level, for one launch across bricks: the grid's z index
// runs over the planes of brick 0, then brick 1, ...
template <typename T>
struct Bricks {
    LevelView<T> v[kMaxBricks];
    int z0[kMaxBricks + 1];  // first plane of each brick; z0[nb] = total planes
    int nb;
    int max1, max2;          // largest n1 and n2 (grid extents)
};

// Transfer tables between level l (fine) and l+1 (coarse), fine-indexed.
struct TransferTabs {
    // restriction: coarse b' = sum over children of ratio_x*ratio_y*ratio_z * r'
    const double* ratio64;  // [n0f | n1f | n2f]
    const float* ratio32;
    // prolongation per axis: coarse indices i0, i1 and the weight of i1
    const int* pidx;        // [2*n0f | 2*n1f | 2*n2f]
    const double* pw64;     // [n0f | n1f | n2f]
    const float* pw32;
    int R0, R1, R2;
};

struct TransferSet {
    TransferTabs t[kMaxBricks];
};

// Device-resident solve state: one cache line read back (or tested by the
// graph's loop condition) per cycle.
struct SolveState {
    double nf;         // normalisation factor (solver.C:13-61)
    double init;       // initial normalised residual
    double cur;        // current normalised residual
    double l2;         // current ||b - A x||_2 (unscaled)
    double l2_0;       // initial ||b - A x0||_2
    double rel_tol, abs_tol;
    double mean;       // volume-weighted mean of x (mean removal)
    double ybar;       // plain mean of the initial x (normFactor with Dirichlet faces)
    double vol_total;
    double ncells;
    int iter;
    int min_iter, max_iter;
    int converged;
    int nan;
    int keep_going;
    int first;         // flexible CG: no previous direction yet
    int criterion;     // 0: relative to the initial residual, 1: relative to ||b||
    // flexible CG scalars
    double alpha;      // step length of the last update
    double gamma;      // (z, V r) of the current direction
    double beta;
    double pq;         // (p, V q) of the current direction
    double l2_true;    // ||b - A x||_2 recomputed from x after the loop
    double bnorm;      // ||b||_2 (unscaled)
};

// Geometry of a fused smoothing launch (single brick): march axis m (0),
// the other non-contiguous axis a (1), and k (axis 2); see
// bmg_smooth_fused.cu.
struct FusedGeom {
    int m_axis;
    int nm, na, nk;
    long sm, sa;        // strides of m and a (k contiguous)
    int perm, pera, perk;
    int ti;             // planes per CTA chunk along m
    int wl_m, wh_m;     // coupling-table offsets of the m axis
    int wl_a, wh_a;     // ... of the a axis
};

// all `stages` colour passes (colours c1, 1-c1, c1, ...) of one smoothing
// step in one launch, reading L.x and writing xout
template <typename T, bool VAR>
void launch_smooth_fused(const LevelView<T>& L, T* xout, const FusedGeom& g, int c1, int stages,
                         cudaStream_t s);
constexpr int kFusedMaxStages = 3;

constexpr int kReduceThreads = 256;

// The coarse end of a V-cycle in one CTA (k_tail_cycle): levels v[0] (the
// first fused level) .. v[nlev-1] (the coarse solve level) of one brick,
// the transfers between them, and each level's colour sequences.
constexpr int kMaxTail = 6;
constexpr int kMaxSeq = 16;
constexpr int kTailThreads = 512;
constexpr long kTailCells = 4096;  // levels this small run in the fused tail
constexpr long kSplitMinCells = kTailCells;  // parity-split rows on single-brick levels above this

template <typename T>
struct TailPlan {
    LevelView<T> v[kMaxTail];
    TransferTabs t[kMaxTail];
    int pre[kMaxTail][kMaxSeq];
    int post[kMaxTail][kMaxSeq];
    int npre[kMaxTail];
    int npost[kMaxTail];
    int nlev;
    const double* ainv;
    const int* cidx;
    int ncoarse;
};

// ---- launchers (bmg_kernels.cu) -------------------------------------------
// zero (parity-split levels only): the pass starts from x = 0 -- x is not
// read, and the whole level (both colours, periodic images) is written
template <typename T, bool VAR>
void launch_colour_pass(const Bricks<T>& B, int colour, cudaStream_t s, bool zero = false);
template <typename T, bool VAR>
void launch_jacobi(const Bricks<T>& B, T* tmp, cudaStream_t s);
template <typename T, bool VAR>
void launch_residual_restrict(const Bricks<T>& F, const Bricks<T>& C, const TransferSet& t, cudaStream_t s);
template <typename T>
void launch_prolong_correct(const Bricks<T>& F, const Bricks<T>& C, const TransferSet& t, cudaStream_t s);
// dense solve on the coarse level; cidx lists the slab index of each unknown
template <typename T>
void launch_coarse_solve(const Bricks<T>& C, const double* ainv, const int* cidx, int n, cudaStream_t s);
template <typename T, bool VAR>
void launch_tail_cycle(const TailPlan<T>& P, cudaStream_t s);
template <typename T, bool VAR>
void launch_residual_out(const Bricks<T>& B, double* r_unscaled_compact, cudaStream_t s);
// x[dst[q]] = x[src[q]]: ghost refresh between bricks
template <typename T>
void launch_fill_ghosts(T* x, const int* dst, const int* src, long n, cudaStream_t s);

// residual norms of level 0 in FP64.  mode 0: initial (also the norm-factor
// sum and ||b||^2: three partial arrays), 1: current.  When b32 is given the scaled residual is also written
// there in FP32 (the right-hand side of the next mixed-precision cycle).
// Returns the number of per-block partials written (for launch_finalize_n).
template <bool VAR>
long launch_residual_norm(const Bricks<double>& B, const Walls& W, int mode, double* partials, float* b32,
                          cudaStream_t s);
void launch_finalize(const Bricks<double>& B, const double* partials, SolveState* st, int mode,
                     cudaGraphConditionalHandle cond, int setCondition, cudaStream_t s);
void launch_mean(const Bricks<double>& B, double* partials, SolveState* st, cudaStream_t s);
// st->ybar = plain mean of the interior x (gAverage, solver.C:24)
void launch_plain_mean(const Bricks<double>& B, double* partials, SolveState* st, cudaStream_t s);
// number of per-block partial sums the level-0 reductions write
long reduce_blocks(const Bricks<double>& B);
// sets the dynamic shared memory limits of the fused smoother instances
void configure_fused_kernels();

// ---- flexible CG outer loop (bmg_krylov.cu), level 0, FP64 ------------------
// r = b - A'x into r (and the cycle's right-hand side pre32 or pre64);
// partials as launch_residual_norm.  mode 2: only ||V r||^2, nothing written.
template <bool VAR>
long launch_fcg_residual(const Bricks<double>& B, const Walls& W, int mode, double* r, float* pre32, double* pre64,
                         double* partials, cudaStream_t s);
// the same residual on a parity-split level 0 (four same-parity cells per
// thread); returns the number of partials
template <bool VAR>
long launch_residual_split(const Bricks<double>& B, const Walls& W, int mode, double* r, float* pre32,
                           double* pre64, double* partials, cudaStream_t s);
// one FCG(1) step after the cycle z = M(r): beta, p = z + beta p,
// q = A'z + beta q, alpha, x += alpha p (B.x, periodic write-through),
// r -= alpha q, pre = r, and the partials of ||V r||^2 -- two passes and
// one reduction on rows of whole quads, three passes otherwise
template <typename T, bool VAR>
void launch_fcg_step(const Bricks<double>& B, const T* z, double* p, double* q, double* r, float* pre32,
                     double* pre64, double* partials, SolveState* st, cudaStream_t s);
// kernels launch_fcg_step launches
int fcg_step_launches(const Bricks<double>& B);
// number of per-block partials the FCG step kernels write
long fcg_partials(const Bricks<double>& B);
// the convergence decision from n partials (as launch_finalize)
void launch_finalize_n(const double* partials, long n, SolveState* st, int mode, cudaGraphConditionalHandle cond,
                       int setCondition, cudaStream_t s);
// st->l2_true from the partials of a mode-2 residual
void launch_fcg_true_norm(const double* partials, long n, SolveState* st, cudaStream_t s);

// ---- projection steps either side of the pressure solve (bmg_project.cu) ----
struct ProjGeom {
    int n[3];
    int per[3];
    const double* h[3];  // cell sizes per axis (device)
    double cdt;          // C dt of the staggered solver's stage
    int perVolume;       // 1: the Poisson source coloDiv(U) / (-C dt); 0: the system form -V times it
};
void launch_project_rhs(const double* u0, const double* u1, const double* u2, double* out, const ProjGeom& G,
                        cudaStream_t s);
void launch_project_correct(double* u0, double* u1, double* u2, const double* p, const double* lam0,
                            const double* lam1, const double* lam2, const ProjGeom& G, cudaStream_t s);

// compact interior <-> ghost-framed conversions
void launch_load_b(const Bricks<double>& B, const Walls& W, const double* compact, cudaStream_t s);
void launch_load_x(const Bricks<double>& B, const double* compact, cudaStream_t s);
void launch_store_x(const Bricks<double>& B, double* compact, cudaStream_t s);
template <typename T>
void launch_load_field(const Bricks<T>& B, int field, const double* compact, int unscale, cudaStream_t s);
template <typename T>
void launch_store_field(const Bricks<T>& B, int field, double* compact, int unscale, cudaStream_t s);
// x64 += x32 on the interior (write-through)
void launch_add_correction(const Bricks<double>& B, const Bricks<float>& E, cudaStream_t s);
// single-brick FP32 level b -> plain interior array, and plain array -> x
void launch_b_to_plain32(const Bricks<float>& B, float* out, cudaStream_t s);
void launch_plain32_to_x(const Bricks<float>& B, const float* in, cudaStream_t s);

}  // namespace bmg
