/*
 * bmg.h -- C ABI of the B200 geometric-multigrid Poisson solver.
 *
 * This is the boundary a Briscola linear-solver plugin (type "GPUMG") binds.
 * It replaces the reference's multigrid solve behind
 *   solver<SType,Type,MeshType>::solve(linearSystem&, bool constMatrix)
 *       src/briscolaFiniteVolume/solvers/solver/solver.H:280-284
 * selected by name through the runtime table
 *   src/briscolaFiniteVolume/solvers/solver/solver.H:240-251,
 *   src/briscolaFiniteVolume/solvers/solver/solver.C:130-157,
 *   registered as in src/briscolaFiniteVolume/solvers/MG/MGSolvers.C:13-21.
 *
 * Plain pointers and sizes only.  Every function returns a bmg_status code
 * and never throws.  One context owns its device memory and serves one
 * stream; a context is not thread-safe, distinct contexts are independent.
 *
 * Arrays: per brick, interior cells only, k fastest:
 *   lin(i,j,k) = (i*Ny + j)*Nz + k     (src/briscolaCore/include/utils.H:569)
 * and bricks concatenated in brick order.  The system follows the
 * reference's sign convention: A is negative semi-definite (off-diagonal
 * +area*delta*lambda, centre minus their sum; linearGaussLaplacianScheme.C
 * :59-94), and b is the system right-hand side (b_sys = -V f for the
 * Poisson source f, linearSystem.C:547-556).
 */
#ifndef BMG_H
#define BMG_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bmg_status {
    BMG_OK = 0,
    BMG_NOT_CONVERGED = 1, /* maxIter reached (the reference prints stats and returns, MG.C:246-253) */
    BMG_NAN_DETECTED = 2,  /* a residual norm became NaN or Inf                                     */
    BMG_BAD_ARG = 3,       /* invalid argument (the reference aborts with FatalError)                */
    BMG_CUDA_ERROR = 4,    /* a CUDA runtime call failed; see bmg_last_error()                       */
    BMG_TIMEOUT = 5,       /* the solve exceeded its wall-clock budget (bmg_options.timeout_ms)      */
    BMG_NO_DEVICE = 6,     /* no usable sm_100 device                                                */
    BMG_UNSUPPORTED = 7    /* a valid option this build does not implement                           */
} bmg_status;

/* Boundary condition of one outer brick face.  Dirichlet faces follow
 * DirichletBoundaryCondition.C:19-80: the ghost coefficient is eliminated
 * into the centre (A_c -= A_f), the face value g enters the right-hand side
 * as b -= 2 A_f g at every solve, and the system is not singular (no pin, no
 * mean removal; linearSystem.H:227-230).  A Neumann face's value is its
 * gradient g: b -= A_f g / delta (NeumannBoundaryCondition.C:19-56).  On a
 * multi-brick mesh a face wholly in contact with other bricks is an
 * interface and its condition is ignored; a face partly in contact keeps
 * zero-gradient walls on the rest and takes neither a Dirichlet condition
 * nor a gradient there (BMG_UNSUPPORTED). */
enum { BMG_BC_NEUMANN = 0, BMG_BC_PERIODIC = 1, BMG_BC_DIRICHLET = 2 };

/* Cycle types (MG.H:106-124) and smoothers (MG.C:313-373). */
enum { BMG_CYCLE_V = 0, BMG_CYCLE_W = 1, BMG_CYCLE_F = 2 };
enum { BMG_SMOOTHER_RBGS = 0, BMG_SMOOTHER_JACOBI = 1 };
/* Arithmetic of the cycles: plain FP64, or FP32 cycles inside FP64
 * iterative refinement (FP64 residual, update, coarse solve, mean). */
enum { BMG_PRECISION_FP64 = 0, BMG_PRECISION_MIXED = 1 };
/* Outer loop: the reference's one cycle per iteration (MG.C:191-242), or
 * flexible conjugate gradients (Notay's FCG(1)) on the FP64 residual with
 * one cycle as the preconditioner.  No counterpart in the reference. */
enum { BMG_KRYLOV_NONE = 0, BMG_KRYLOV_FCG = 1 };
/* Coarsest level of a cycle (coarseMode, MG.C:110-126): the direct solve
 * (APLU), or max(nSweepsPost, 2) sweeps of the smoother, with the
 * singularity pin (solver.C:201-231) kept by the smoothers on that level. */
enum { BMG_COARSE_DIRECT = 0, BMG_COARSE_SMOOTH = 1 };
/* Grid transfers of the cycle (MG.C:289-305): the residual restriction
 * linear (linearRestrictionScheme.C:15-187) or average
 * (averageRestrictionScheme.C:17-77), the correction's prolongation linear
 * (linearProlongationScheme.C:12-147) or injection
 * (injectionProlongationScheme.C:14-33). */
enum { BMG_RESTRICT_LINEAR = 0, BMG_RESTRICT_AVERAGE = 1 };
enum { BMG_PROLONG_LINEAR = 0, BMG_PROLONG_INJECTION = 1 };
/* Convergence test: relTol relative to the initial residual (solver.C:64-95,
 * the reference's), or relative to ||b||_2, i.e. ||b - A x||_2 <= relTol
 * ||b||_2 whatever the initial guess (used to compare solves that start from
 * different guesses).  The absolute tolerance applies in both. */
enum { BMG_CRITERION_INITIAL = 0, BMG_CRITERION_RHS = 1 };
/* Storage order of the rows of the device levels (rowLayout; no counterpart
 * in the reference, whose arrays are k fastest, utils.H:569).  Split: on
 * single-brick levels above 4096 cells with n2 % 16 == 0, each row's cells
 * are kept in blocks of 16, the 8 even k before the 8 odd k, so a red-black
 * colour pass reads and writes only sectors of the colours it needs; the
 * caller's arrays keep the reference's order.  Natural: k fastest on every
 * level.  Both give bit-identical results.  Fixed when the context is
 * created. */
enum { BMG_ROWS_SPLIT = 0, BMG_ROWS_NATURAL = 1 };

/* bmg_solve flags */
enum {
    BMG_DEVICE_PTRS = 1, /* b and x are device pointers on the context's device */
    BMG_ZERO_GUESS = 2,  /* ignore the incoming x and start from zero           */
    BMG_PER_VOLUME = 4   /* bmg_project_rhs: the Poisson source, not the system form */
};

typedef struct bmg_brick {
    int n[3];                 /* cells along x, y, z                                   */
    const double* points[3];  /* n[d]+1 vertex coordinates along axis d (host memory)  */
    int bc[6];                /* x-lo, x-hi, y-lo, y-hi, z-lo, z-hi: BMG_BC_*          */
    int origin[3];            /* cell offset in the global lattice (multi-brick)       */
    double value[6];          /* Dirichlet value or Neumann gradient of each face
                                 (uniform; ignored on periodic faces)             */
    int transform[3];         /* orientation of the brick's own frame: local axis d
                                 runs along mesh axis |transform[d]|-1, reversed
                                 when negative (parallelBoundaryCondition.C:148-163's
                                 T); {0,0,0} = identity.  n, points, bc, value and
                                 the brick's parts of b, x and lambda are in the
                                 brick's frame (points in local order, decreasing
                                 along a reversed axis); origin is in the mesh's. */
} bmg_brick;

typedef struct bmg_mesh_desc {
    int n_bricks;
    const bmg_brick* bricks;
} bmg_mesh_desc;

/* Dictionary keys of the reference MG (MG.C:257-305, solver.C:115-123) plus
 * the B200-specific ones. */
typedef struct bmg_options {
    double rel_tol;     /* relTol                                              */
    double abs_tol;     /* tolerance                                           */
    int min_iter;       /* minIter      (0)                                    */
    int max_iter;       /* maxIter      (999)                                  */
    int n_pre;          /* nSweepsPre   (0)                                    */
    int n_post;         /* nSweepsPost  (2)                                    */
    int cycle_type;     /* cycleType    (F)                                    */
    int coarse_level;   /* coarseLevel  (0), counted from the coarsest level   */
    int smoother;       /* smoother     (rbgs)                                 */
    int precision;      /* precision    (fp64)                                 */
    int use_graph;      /* graph        (1): whole solve as one CUDA graph     */
    int remove_mean;    /* subtract the volume-weighted mean of x; singular
                           systems only (no Dirichlet face)                    */
    int fused;          /* fused (3): up to this many colour passes of a
                           smoothing step per pass over memory (1..3); 0: one
                           launch per colour pass                              */
    int autotune;       /* autotune (1): time the fused smoother's launch
                           shapes per level at creation and keep the fastest   */
    int device;         /* CUDA device ordinal                                 */
    double timeout_ms;  /* wall-clock budget per solve, <= 0: none             */
    int krylov;         /* krylov (none): outer loop, BMG_KRYLOV_*             */
    int criterion;      /* criterion (initial): BMG_CRITERION_*                */
    int fused_chunk;    /* fusedChunk (64): planes along i per CTA of the
                           fused smoother when autotune is off (1..128)        */
    int fuse_coarse;    /* fuseCoarse (1): run the levels of at most 4096
                           cells and the coarse solve of a single-brick V
                           cycle in one kernel                                 */
    int coarse_mode;    /* coarseMode (direct): BMG_COARSE_* (MG.C:110-126)     */
    int restrict_scheme;/* restrict (linear): BMG_RESTRICT_*                   */
    int prolong_scheme; /* prolong (linear): BMG_PROLONG_*                     */
    int row_layout;     /* rowLayout (split): BMG_ROWS_*, fixed at creation    */
    int fuse_first;     /* fuseFirstPass (1): a mixed flexible-CG solve starts
                           each FP32 cycle with a zero-start colour pass on
                           a parity-split level 0 (no memset of z, no read
                           of z); results bit-identical                      */
} bmg_options;

typedef struct bmg_report {
    int status;
    int cycles;               /* V/W/F cycles performed (inner cycles when mixed) */
    int outer_iterations;     /* FP64 refinement steps (mixed), else = cycles     */
    double initial_residual;  /* Briscola-normalised (solver.C:13-61)             */
    double final_residual;    /* Briscola-normalised                              */
    double rel_residual;      /* ||b - A x||_2 / ||b - A x0||_2 (recomputed from x
                                 at the end of an FCG solve)                      */
    double final_l2;          /* ||b - A x||_2                                    */
    double norm_factor;       /* normFactor of solver.C:13-61                     */
    float ms;                 /* device time of the solve (CUDA events)           */
    long kernel_launches;     /* kernels this solve launched (graph nodes count)  */
    double rhs_rel_residual;  /* ||b - A x||_2 / ||b||_2                            */
} bmg_report;

int bmg_default_options(bmg_options* opts);

/* Build the level hierarchy and device buffers for a mesh.  Replaces the MG
 * constructor (MG.C:257-399) and the per-solve setup of MG.C:431-459. */
int bmg_create(struct bmg_ctx** ctx, const bmg_mesh_desc* mesh, const bmg_options* opts);
void bmg_destroy(struct bmg_ctx* ctx);

/* Variable coefficient lambda on the level-0 faces (host arrays), one per
 * face direction with shapes (Nx+1,Ny,Nz), (Nx,Ny+1,Nz), (Nx,Ny,Nz+1) per
 * brick, concatenated.  Restricted to coarse levels area-weighted
 * (areaWeightedFaceRestrictionScheme.C:19-57).  NULLs: constant coefficient. */
int bmg_set_coefficients(struct bmg_ctx* ctx, const double* lambda_x, const double* lambda_y,
                         const double* lambda_z);

int bmg_set_stream(struct bmg_ctx* ctx, void* cuda_stream);
int bmg_set_options(struct bmg_ctx* ctx, const bmg_options* opts);

/* Solve A x = b.  Replaces MG::solve (MG.C:402-483).  x holds the initial
 * guess on entry unless BMG_ZERO_GUESS, and the solution on return. */
int bmg_solve(struct bmg_ctx* ctx, const double* b, double* x, int flags, bmg_report* report);

/* Number of cells of all bricks on level 0 (length of b and x). */
long bmg_num_cells(const struct bmg_ctx* ctx);
int bmg_num_levels(const struct bmg_ctx* ctx);
int bmg_level_shape(const struct bmg_ctx* ctx, int level, int brick, int n[3]);

const char* bmg_status_string(int status);
const char* bmg_last_error(const struct bmg_ctx* ctx);

/* ---- Building blocks, for per-kernel parity tests --------------------------
 * They act on the context's level buffers.  Fields: 0 = x, 1 = b (both as
 * the reference's unscaled values), interior cells of every brick in brick
 * order.  The precision argument selects the FP64 (0) or FP32 (1) buffers. */
int bmg_level_upload(struct bmg_ctx* ctx, int level, int field, int precision, const double* host);
int bmg_level_download(struct bmg_ctx* ctx, int level, int field, int precision, double* host);
/* one red-black colour pass (colour 0: (i+j+k) even) on level l:
 * replaces one pass of rbgsSmoother.C:65-183 */
int bmg_op_colour_pass(struct bmg_ctx* ctx, int level, int colour, int precision);
/* n_sweeps sweeps of the configured smoother on level l */
int bmg_op_smooth(struct bmg_ctx* ctx, int level, int n_sweeps, int precision);
/* r = b - A x on level l, written into host r (unscaled); replaces
 * linearSystemResidual.C:280-332 */
int bmg_op_residual(struct bmg_ctx* ctx, int level, int precision, double* host_r);
/* b(l+1) = restriction of b(l) - A x(l) (fused residual + restriction,
 * linearRestrictionScheme.C:103-159 with scale); x(l+1) = 0 */
int bmg_op_residual_restrict(struct bmg_ctx* ctx, int level, int precision);
/* x(l) += prolongation of x(l+1) (linearProlongationScheme.C:112-147) */
int bmg_op_prolong_correct(struct bmg_ctx* ctx, int level, int precision);
/* direct solve on the coarse solve level (APLU.C:91-128) */
int bmg_op_coarse_solve(struct bmg_ctx* ctx, int precision);
/* the configured coarse solve level index */
int bmg_coarse_level_index(const struct bmg_ctx* ctx);
/* launch shape of the fused smoother on a level (precision 0: FP64, 1:
 * FP32): colour stages per launch (0 when the level is smoothed pass by
 * pass) and planes per CTA chunk, as chosen by the autotuner */
int bmg_level_tuning(const struct bmg_ctx* ctx, int level, int precision, int* stages, int* chunk);
/* pins that launch shape (stages 0: pass by pass; 1..3 needs a level the
 * fused smoother handles; chunk 1..128), e.g. to replay a tuning measured
 * in another process; the solve graph is rebuilt at the next solve */
int bmg_set_level_tuning(struct bmg_ctx* ctx, int level, int precision, int stages, int chunk);

/* ---- Either side of the solve in a projection step --------------------------
 * Single-brick contexts, device arrays on the context's stream.  Staggered
 * face arrays of axis d hold n[d]+1 faces along d (the face below cell q,
 * then the top face), k fastest: u0 (n0+1) x n1 x n2, u1 n0 x (n1+1) x n2,
 * u2 n0 x n1 x (n2+1); on a periodic axis the last face repeats the first.
 *
 * out (interior cells, k fastest) = the right-hand side of the pressure solve
 * of a staggered projection, coloDiv(U) / (-c_dt) (briscolaStaggered.C:92,
 * divergenceScheme.C:116-150), in the system form -V times it that
 * bmg_solve takes (linearSystem.C:547-556), or as that Poisson source itself
 * with BMG_PER_VOLUME (for the FFT solver, bfft.h). */
int bmg_project_rhs(struct bmg_ctx* ctx, const double* u0, const double* u1, const double* u2, double c_dt,
                    double* out, int flags);
/* U -= c_dt * stagReconstruct(lambda faceGrad(p) A) = c_dt lambda (p_c - p_below) delta
 * on every face (briscolaStaggered.C:96, defaultPoissonSolver.C:110-123,
 * exSchemesReconstruction.H:187-206); lambda arrays as the face arrays of U,
 * NULL for 1; wall faces (zero gradient) are left unchanged. */
int bmg_project_correct(struct bmg_ctx* ctx, double* u0, double* u1, double* u2, const double* p,
                        const double* lam0, const double* lam1, const double* lam2, double c_dt);

/* ---- A level solver in place of the cycle's coarse recursion ---------------
 * No counterpart in the reference: the learned coarse-level correction.  In
 * the cycle MG.C:19-130 a level l > 0 receives the restricted residual as
 * its right-hand side and returns the correction its sub-cycle computes
 * (MG.C:77-99).  With a level solver set at level l, the FP32 cycles of a
 * mixed-precision solve (precision mixed) instead hand that level's
 * right-hand side to fn and take fn's result as the level's correction,
 * then post-smooth it (nSweepsPost sweeps); the levels below l are not
 * visited.  FP64 cycles keep the multigrid recursion.
 *
 * With mode BMG_LEVEL_GUESS the solver's result instead starts the level's
 * usual cycle (pre-smoothing, the recursion below, post-smoothing) in place
 * of zero: the levels below keep their work, and the network only has to
 * improve the level's starting point.
 *
 * fn(user, stream, rhs, x, n) is called on the host while the cycle is
 * being launched: rhs and x are device arrays of the level's interior
 * cells (n[0]*n[1]*n[2] floats, k fastest), rhs the row-scaled right-hand
 * side b/V of the level (equal to -f for a Poisson source f), x to be
 * filled with the correction.  fn must queue all its work on `stream` (a
 * cudaStream_t) and neither synchronise nor allocate: inside a graphed
 * solve it runs while the solve graph is being captured, and its kernels
 * become part of the graph.  A nonzero return aborts the solve with
 * BMG_CUDA_ERROR.  Single-brick meshes, 1 <= level <= the coarse solve
 * level; fn NULL removes the solver.  The context keeps two level-sized
 * FP32 arrays for rhs and x. */
typedef int (*bmg_level_solver)(void* user, void* stream, const float* rhs, float* x, const int n[3]);
enum { BMG_LEVEL_REPLACE = 0, BMG_LEVEL_GUESS = 1 };
int bmg_set_level_solver(struct bmg_ctx* ctx, int level, bmg_level_solver fn, void* user, int mode);

/* ---- Residual norm without any device allocation ---------------------------
 * No counterpart in the reference: an addition for callers that must not
 * call cudaMalloc when they want a residual -- an application whose device
 * memory belongs to its own pool, a loop that cannot take the device-wide
 * synchronisation an allocation may bring, or a failure path running after
 * device memory ran out.
 *
 * *norm_out = ||b - A x||_2 for one brick with the solver's level-0 operator
 * (constant coefficient).  x, b: device arrays of interior cells, k fastest;
 * points_*: device arrays of n[d]+1 vertex coordinates; bc: host array of
 * BMG_BC_* per face (Dirichlet faces homogeneous: the eliminated operator,
 * with any face values already in b); norm_out: one device double.  Work is queued on
 * `stream` (a cudaStream_t, NULL for the default stream); the result is
 * ready once the stream has reached that point.
 *
 * Scratch: a file-scope static device array of BMG_NOALLOC_MAX_ROWS doubles
 * (512 KB on every GPU that loads the library, until exit), one partial sum
 * per (i, j) row: n[0]*n[1] above the limit is rejected with BMG_BAD_ARG and
 * a message on stderr.  Every call overwrites the partials it reads, so no
 * state carries over, but all calls on a device share the array: calls that
 * overlap on the GPU (different streams, or threads without ordering) race.
 * Every call looks up the array's device address (cudaGetSymbolAddress)
 * with the current device; the first call on a device also loads the
 * library's device code there, so make that first call before any stream
 * capture.  An error that earlier work left pending (cudaPeekAtLastError)
 * is returned as BMG_CUDA_ERROR before anything is launched, and left
 * pending for its owner. */
#define BMG_NOALLOC_MAX_ROWS 65536
int bmg_residual_norm_noalloc(const double* x, const double* b, const int n[3],
                              const double* points_x, const double* points_y,
                              const double* points_z, const int bc[6], double* norm_out,
                              void* stream);

#ifdef __cplusplus
}
#endif

#endif /* BMG_H */
