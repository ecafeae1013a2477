// bmg_internal.h -- device-side views and kernel launchers of the B200
// multigrid solver.  Host driver: bmg_host.cu.  Kernels: bmg_kernels.cu.
//
// Data layout in HBM (per level, per brick):
//   every cell field is a ghost-framed block of (n0+2) x (n1+2) x (n2+2)
//   values, k fastest (the reference's lin(), utils.H:569, with its one-cell
//   ghost frame, meshDirection.H:35).  Interior cell (i,j,k) sits at
//   base + i*si + j*sj + k with base = si + sj + 1.
//   Periodic axes keep their ghost layers (faces, edges, corners) current by
//   write-through: every kernel that stores an interior value also stores it
//   into the ghost images of that cell, so stencils read ghosts without
//   a separate exchange step (the reference exchanges them per sweep,
//   rbgsSmoother.C:405-428).  Wall (Neumann) ghosts are never read: their
//   couplings are zero after elimination (NeumannBoundaryCondition.C:19-56).
//
// The operator is stored row-scaled by the inverse cell volume (A' = A/V,
// b' = b/V), which leaves every Gauss-Seidel, Jacobi and coarse-solve
// update unchanged and makes the constant-coefficient couplings pure 1-D
// tables: coupling to the lower x neighbour = delta_x(i)/h_x(i) (times the
// face lambda for a variable coefficient).  No 7-coefficient array exists
// on the device.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace bmg {

// 1-D table offsets inside one level's coefficient table
struct TabOff {
    int wl[3];   // coupling to the lower neighbour, per cell along the axis
    int wh[3];   // coupling to the upper neighbour
    int h[3];    // cell sizes (volume factors)
    int total;
};

template <typename T>
struct LevelView {
    int n0, n1, n2;
    long si, sj;       // strides of i and j (k contiguous)
    long base;         // index of interior cell (0,0,0)
    long cells;        // size of the ghost-framed block
    T* x;
    T* b;
    const T* tab;      // 1-D tables (TabOff layout) in precision T
    const double* tab64;  // the same tables in FP64 (norms, volumes)
    TabOff to;
    const T* lam0;     // face lambda (lower face of the cell, ghost-framed
    const T* lam1;     // indexing), nullptr for a constant coefficient
    const T* lam2;
    int per0, per1, per2;
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
    double vol_total;
    double ncells;
    int iter;
    int min_iter, max_iter;
    int converged;
    int nan;
    int keep_going;
    int pad[2];
};

// Geometry of a fused smoothing launch: march axis m (0 or 1), the other
// non-contiguous axis a, and k (axis 2); see bmg_smooth_fused.cu.
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

// ---- launchers (bmg_kernels.cu) -------------------------------------------
template <typename T, bool VAR>
void launch_colour_pass(const LevelView<T>& L, int colour, cudaStream_t s);
template <typename T, bool VAR>
void launch_jacobi(const LevelView<T>& L, T* tmp, cudaStream_t s);
template <typename T, bool VAR>
void launch_residual_restrict(const LevelView<T>& F, const LevelView<T>& C, const TransferTabs& t,
                              cudaStream_t s);
template <typename T>
void launch_prolong_correct(const LevelView<T>& F, const LevelView<T>& C, const TransferTabs& t,
                            cudaStream_t s);
template <typename T>
void launch_coarse_solve(const LevelView<T>& C, const double* ainv, int n, cudaStream_t s);
template <typename T, bool VAR>
void launch_residual_out(const LevelView<T>& L, double* r_unscaled_compact, cudaStream_t s);

// residual norms of level 0 in FP64.  mode 0: initial (also the norm-factor
// sum), 1: current.  When b32 is given the scaled residual is also written
// there in FP32 (the right-hand side of the next mixed-precision cycle).
template <bool VAR>
void launch_residual_norm(const LevelView<double>& L, int mode, double* partials, float* b32,
                          const LevelView<float>* L32, cudaStream_t s);
void launch_finalize(const LevelView<double>& L, const double* partials, SolveState* st, int mode,
                     cudaGraphConditionalHandle cond, int setCondition, cudaStream_t s);
// number of per-block partial sums the level-0 reductions write
long reduce_blocks(const LevelView<double>& L);
// sets the dynamic shared memory limits of the fused smoother instances
void configure_fused_kernels();
void launch_mean(const LevelView<double>& L, double* partials, SolveState* st, cudaStream_t s);

// compact interior <-> ghost-framed conversions (level 0, FP64)
void launch_load_b(const LevelView<double>& L, const double* compact, cudaStream_t s);
void launch_load_x(const LevelView<double>& L, const double* compact, cudaStream_t s);
void launch_store_x(const LevelView<double>& L, double* compact, cudaStream_t s);
template <typename T>
void launch_load_field(const LevelView<T>& L, int field, const double* compact, int unscale,
                       cudaStream_t s);
template <typename T>
void launch_store_field(const LevelView<T>& L, int field, double* compact, int unscale,
                        cudaStream_t s);
// x64 += x32 on the interior (write-through)
void launch_add_correction(const LevelView<double>& L, const LevelView<float>& E, cudaStream_t s);

}  // namespace bmg
