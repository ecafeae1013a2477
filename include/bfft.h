/*
 * bfft.h -- C ABI of the B200 FFT Poisson solver.
 *
 * Replaces the reference's constant-coefficient direct solver
 *   FFTPoissonSolver<SType>::solve(x, bPtr, lambdaPtr, ddt, dtFrac)
 *       src/briscolaFiniteVolume/solvers/PoissonSolvers/FFTPoissonSolver/FFTPoissonSolver.H:98-106,
 *       FFTPoissonSolver.C:88-446
 * selected as PoissonSolver type "FFT" (FFTPoissonSolver.C:14-21).  The
 * method is the reference's: fast trigonometric / real Fourier transforms
 * along the two uniform directions (FFTW r2r kinds chosen per boundary pair,
 * FourierTransforms.C:130-282), a tridiagonal (Thomas, or cyclic) solve per
 * mode along the third direction (tridiagonalSolver.C:117-450), inverse
 * transforms and normalisation.
 *
 * Plain pointers and sizes only; every function returns a bmg_status code
 * (bmg.h) and never throws.  One brick, interior cells only, k fastest:
 * lin(i,j,k) = (i*Ny + j)*Nz + k.  Every extent that is transformed must be
 * a power of two up to 512 (BMG_UNSUPPORTED otherwise); the solve direction
 * may have any extent >= 2.
 */
#ifndef BFFT_H
#define BFFT_H

#include "bmg.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Face conditions (FourierTransforms.C:96-101): an "empty" axis has one cell
 * and carries no transform. */
enum { BFFT_BC_DIRICHLET = 0, BFFT_BC_NEUMANN = 1, BFFT_BC_PERIODIC = 2, BFFT_BC_EMPTY = 3 };

typedef struct bfft_desc {
    int n[3];                /* cells along x, y, z                                      */
    const double* points[3]; /* n[d]+1 vertex coordinates along axis d (host memory)     */
    int bc[6];               /* x-lo, x-hi, y-lo, y-hi, z-lo, z-hi: BFFT_BC_*            */
    double value[6];         /* Dirichlet value or Neumann gradient of each face (uniform)*/
    int device;              /* CUDA device ordinal                                      */
} bfft_desc;

typedef struct bfft_ctx bfft_ctx;

/* Plans the solve (solve direction as planner.C:60-99, transform tables,
 * tridiagonal coefficients) and allocates the device work arrays. */
int bfft_create(bfft_ctx** ctx, const bfft_desc* desc);
void bfft_destroy(bfft_ctx* ctx);
/* Work is queued on this stream (a cudaStream_t); the default is a stream
 * the context owns.  Host-pointer solves synchronise it before returning. */
int bfft_set_stream(bfft_ctx* ctx, void* stream);

/* x solves  Laplacian(x) - shift x = -b - shift x_old  with the face values
 * of the descriptor (the reference's solve with ddt: shift = 1/(dt dtFrac),
 * FFTPoissonSolver.C:117-131, tridiagonalSolver.C:347-350; shift 0 and
 * x_old NULL without ddt).  b, x, x_old: n[0]*n[1]*n[2] doubles, host
 * arrays, or device arrays with BMG_DEVICE_PTRS.  The Laplacian is the
 * reference's cell-centred one (face distances from cell centres, ghost
 * cells mirrored at walls); a mode whose two transform eigenvalues are zero
 * (all-Neumann or periodic transform directions) is fixed by the
 * reference's pin of its first diagonal entry (tridiagonalSolver.C:180-186,
 * 225-231). */
int bfft_solve(bfft_ctx* ctx, const double* b, double* x, const double* x_old, double shift, int flags);

/* ---- split Poisson solver (splitPoissonSolver.C:53-155) -------------------
 * Device arrays only.  Face coefficients: lam0 (n0+1) x n1 x n2 (the face
 * below cell i along x, then the top face), lam1 n0 x (n1+1) x n2, lam2
 * n0 x n1 x (n2+1), k fastest.
 *
 * *lambda0 = the largest face coefficient (splitPoissonSolver.C:97-104). */
int bfft_split_lambda0(bfft_ctx* ctx, const double* lam0, const double* lam1, const double* lam2, double* lambda0);
/* bhat = b / lambda0 + div((lambda / lambda0 - 1) faceGrad(x) faceArea), the
 * modified source of splitPoissonSolver.C:118-138 with the reference's
 * outward face gradient and flux divergence (linearFaceGradientScheme.C,
 * divergenceScheme.C:68-96); boundary faces see the ghost values of the
 * descriptor's face conditions. */
int bfft_split_source(bfft_ctx* ctx, const double* x, const double* b, const double* lam0, const double* lam1,
                      const double* lam2, double lambda0, double* bhat);
/* out = a x + c y (the split solver's prediction from two old levels,
 * splitPoissonSolver.C:75-84); out may alias x or y. */
int bfft_axpby(bfft_ctx* ctx, double a, const double* x, double c, const double* y, double* out);

/* the planned solve direction (0, 1, 2) */
int bfft_solve_direction(const bfft_ctx* ctx);
/* last error message of the context ("" if none) */
const char* bfft_last_error(const bfft_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif
