/*
 * bmg_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement of the reference (Briscola) geometric-multigrid solve for
 * one rectilinear, cell-centred brick on one rank.  It is the parity checker
 * for the CUDA solver in briscola_b200/csrc: only tests, the smoke check and
 * the CPU-baseline leg of the benchmark may load it.  Nothing in the product
 * path links or calls it.
 *
 * What it follows (paths relative to the Briscola source tree):
 *   cycle / loop / convergence  src/briscolaFiniteVolume/solvers/MG/MG.C:19-254,402-483
 *                               src/briscolaFiniteVolume/solvers/MG/MG.H:106-124
 *   norms, convergence, pin     src/briscolaFiniteVolume/solvers/solver/solver.C:13-95,201-231
 *   RBGS smoother               src/briscolaFiniteVolume/solvers/smoothers/rbgsSmoother/rbgsSmoother.C:15-437
 *   Jacobi smoother (w = 0.8)   src/briscolaFiniteVolume/solvers/smoothers/jacSmoother/jacSmoother.C:15-321
 *   residual                    src/briscolaFiniteVolume/linearSystems/linearSystem/linearSystemResidual.C:13-332
 *   row products                src/briscolaFiniteVolume/linearSystems/linearSystem/linearSystemFunctions.H:28-104
 *   linear restriction          src/briscolaFiniteVolume/schemes/restrictionSchemes/linearRestrictionScheme/linearRestrictionScheme.C:15-187
 *   linear prolongation         src/briscolaFiniteVolume/schemes/prolongationSchemes/linearProlongationScheme/linearProlongationScheme.C:12-147
 *   average restriction         src/briscolaFiniteVolume/schemes/restrictionSchemes/averageRestrictionScheme/averageRestrictionScheme.C:17-77
 *   injection prolongation      src/briscolaFiniteVolume/schemes/prolongationSchemes/injectionProlongationScheme/injectionProlongationScheme.C:14-33
 *   area-weighted lambda        src/briscolaFiniteVolume/schemes/restrictionSchemes/areaWeightedFaceRestrictionScheme/areaWeightedFaceRestrictionScheme.C:19-57
 *   Laplacian assembly          src/briscolaFiniteVolume/schemes/laplacianSchemes/linearGaussLaplacianScheme/linearGaussLaplacianScheme.C:22-102
 *   face deltas                 src/briscolaFiniteVolume/fvMeshMetrics.C:848-893
 *   Neumann elimination         src/briscolaFiniteVolume/boundaryConditions/NeumannBoundaryCondition/NeumannBoundaryCondition.C:19-85
 *   Dirichlet elimination/ghost src/briscolaFiniteVolume/boundaryConditions/DirichletBoundaryCondition/DirichletBoundaryCondition.C:19-80
 *   Neumann gradient values     NeumannBoundaryCondition.C:44-50 (b -= A_f g / delta on level 0)
 *   singularity test            src/briscolaFiniteVolume/linearSystems/linearSystem/linearSystem.H:227-230,
 *                               src/briscolaFiniteVolume/fields/meshLevels/meshLevel/meshLevel.C:555-583
 *   ghost fill order            src/briscolaFiniteVolume/fields/meshLevels/meshLevel/meshLevel.C:231-253,301-328
 *   periodic ghost copy         src/briscolaFiniteVolume/boundaryConditions/periodicBoundaryCondition/periodicBoundaryCondition.C:47-92
 *   level sizes                 src/briscolaCore/include/utils.H:1152-1170, src/briscolaMesh/mesh/mesh.C:19-53,
 *                               src/briscolaMesh/level/level.H:144-147
 *   coarse points / ghosts      src/briscolaMesh/level/levelPoints.C:151-155,198-236,326-400
 *   coarse direct solve (APLU)  src/briscolaFiniteVolume/solvers/externalSolvers/APLU/APLU.C:26-128
 *                               (OpenFOAM's LUDecompose is not in the tree; a partial-pivot LU of our own)
 *
 * Restatement choices (each documented where it is made in the source):
 *   - rectilinear geometry only: the trilinear interpolation weights of the
 *     transfer operators factor into per-axis weights, which are computed
 *     on the fly instead of being cached per cell;
 *   - edge and corner ghosts of a level are filled axis by axis (periodic
 *     image, zero-gradient copy or Dirichlet mirror), which is what the
 *     reference's periodic edge boundaries give; where only walls meet, the
 *     reference's unset-boundary copy of the diagonal interior cell;
 *   - sums that the reference performs with gSum are done per i-plane and
 *     combined in plane order, so results are independent of the thread count.
 */
#ifndef BMG_ORACLE_H
#define BMG_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct bmgo_problem bmgo_problem;

typedef struct bmgo_options {
    double rel_tol;        /* relTol                                  */
    double abs_tol;        /* tolerance                               */
    int    min_iter;       /* minIter (default 0)                     */
    int    max_iter;       /* maxIter (default 999)                   */
    int    n_pre;          /* nSweepsPre                              */
    int    n_post;         /* nSweepsPost                             */
    int    cycle_type;     /* 0 = V, 1 = W, 2 = F                     */
    int    coarse_level;   /* coarseLevel, counted from the coarsest  */
    int    coarse_direct;  /* 1 = direct (APLU), 0 = smoothing        */
    int    smoother;       /* 0 = rbgs, 1 = jacobi                    */
    int    stale_residual; /* 1 = keep MG.C:72 (skip fine residual on rep 0) */
    int    restrict_average;  /* restrict average (averageRestrictionScheme.C) instead of linear */
    int    prolong_injection; /* prolong injection (injectionProlongationScheme.C) instead of linear */
} bmgo_options;

typedef struct bmgo_report {
    int    iterations;
    double initial_residual;   /* Briscola-normalised (solver.C:13-61) */
    double final_residual;     /* Briscola-normalised                   */
    double norm_factor;
    double final_l2;           /* ||b - A x||_2                          */
    double b_l2;               /* ||b||_2                                */
} bmgo_report;

void bmgo_default_options(bmgo_options* o);

/* One brick with N[d] cells; pts_d holds N[d]+1 vertex coordinates along
 * axis d.  periodic[d] != 0 makes both faces of axis d periodic, otherwise
 * both are homogeneous Neumann walls (bmgo_set_faces makes walls Dirichlet).
 * nthreads <= 0 uses all cores. */
bmgo_problem* bmgo_create(const int N[3], const double* pts_x,
                          const double* pts_y, const double* pts_z,
                          const int periodic[3], int nthreads);
void bmgo_destroy(bmgo_problem* p);
/* Wall conditions: dirichlet[f] != 0 turns wall face f (x-lo, x-hi, y-lo,
 * y-hi, z-lo, z-hi) into a Dirichlet face with the uniform value value[f];
 * on the other walls value[f] is the Neumann gradient (NULL: homogeneous
 * everywhere).  A Dirichlet face makes the system non-singular: no pin, no
 * forced coarse cell (linearSystem.H:227-230).  Returns -1 (and changes
 * nothing) for a Dirichlet face or a nonzero value on a periodic axis.
 * Takes effect at the next assembly. */
int  bmgo_set_faces(bmgo_problem* p, const int dirichlet[6], const double* value);

int  bmgo_num_levels(const bmgo_problem* p);
void bmgo_level_shape(const bmgo_problem* p, int l, int N[3]);
/* coarse level l+1 relative factor R (1 or 2 per axis) */
void bmgo_level_ratio(const bmgo_problem* p, int l, int R[3]);
/* cell centres along one axis, N[axis]+2 values including both ghosts */
void bmgo_cell_centres(const bmgo_problem* p, int l, int axis, double* out);
/* cell volumes, interior, k fastest */
void bmgo_cell_volumes(const bmgo_problem* p, int l, double* out);

/* Variable coefficient: level-0 face values of lambda for the x, y, z faces,
 * shapes (Nx+1,Ny,Nz), (Nx,Ny+1,Nz), (Nx,Ny,Nz+1), k fastest.  Restricted to
 * every level with the area-weighted face restriction.  Pass NULLs to return
 * to the constant-coefficient operator. */
void bmgo_set_lambda(bmgo_problem* p, const double* lx, const double* ly,
                     const double* lz);
/* lambda of one level, face direction fd, shape as above for that level */
void bmgo_get_lambda(const bmgo_problem* p, int l, int fd, double* out);

/* Build A on every level (Laplacian + wall elimination + singular pin on
 * the coarsest solve level given by opts->coarse_level, when singular);
 * also selects the transfer schemes of opts for the building blocks. */
void bmgo_assemble(bmgo_problem* p, const bmgo_options* o);
/* 7 coefficients per interior cell {c,l,r,b,t,a,f}, k fastest */
void bmgo_get_matrix(const bmgo_problem* p, int l, double* out7);

/* Full solve of A x = b on level 0.  b and x are interior arrays (k fastest);
 * x is the initial guess on entry.  history (may be NULL) receives up to
 * max_hist normalised residuals, one per cycle. */
int  bmgo_solve(bmgo_problem* p, const bmgo_options* o, const double* b,
                double* x, bmgo_report* rep, double* history, int max_hist);

/* Building blocks on interior arrays of level l, for per-kernel parity. */
void bmgo_residual(bmgo_problem* p, int l, const double* x, const double* b,
                   double* r);
void bmgo_smooth(bmgo_problem* p, int l, int smoother, int sweeps, double* x,
                 const double* b);
/* one clean colour pass over the whole level (parity of the interior
 * index i+j+k), ghosts refreshed before the pass */
void bmgo_colour_pass(bmgo_problem* p, int l, int colour, double* x,
                      const double* b);
/* coarse = restriction of fine (level lf -> lf+1), scale as MG uses it */
void bmgo_restrict(bmgo_problem* p, int lf, const double* fine, double* coarse,
                   int scale);
/* fine (level lf) op= prolongation of coarse (level lf+1); op 0: =, 1: += */
void bmgo_prolong(bmgo_problem* p, int lf, const double* coarse, double* fine,
                  int op);
/* as bmgo_prolong, but the coarse array carries its ghost frame
 * ((Nx+2)(Ny+2)(Nz+2), k fastest) and is used as given: the known-answer
 * test of the reference sets ghosts to the exact field */
void bmgo_prolong_ghosted(bmgo_problem* p, int lf, const double* coarse_g,
                          double* fine, int op);
/* direct solve on level l (matrix as assembled, including the pin) */
void bmgo_coarse_solve(bmgo_problem* p, int l, const double* b, double* x);

#ifdef __cplusplus
}
#endif

#endif
