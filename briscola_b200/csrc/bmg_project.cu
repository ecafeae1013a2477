// bmg_project.cu -- the steps either side of the pressure solve of a
// projection method, on the device, so that a time step keeps the velocity
// and the pressure in HBM (C ABI: bmg_project_rhs / bmg_project_correct in
// include/bmg.h).
//
// Right-hand side: the colocated divergence of the staggered velocity,
//   coloDiv(U)_c = sum over the cell's faces of U_f A_f (outward) / V_c
//   (divergenceScheme.C:116-150), divided by -C dt as the staggered solver
//   passes it (briscolaStaggered.C:92), or multiplied into the system form
//   b_sys = -V b of the linear solve (linearSystem.C:547-556).
// Correction: U_f -= C dt * stagReconstruct(flux)_f with the Poisson flux
//   lambda faceGrad(p) A (defaultPoissonSolver.C:110-123) and
//   stagReconstruct = -flux / A (exSchemesReconstruction.H:187-206): with the
//   outward face gradient (p_lo - p_c) delta, the face velocity loses
//   C dt lambda (p_c - p_lo) delta.  Zero-gradient walls leave their faces
//   unchanged; periodic faces wrap.
//
// Face arrays of axis d hold n_d + 1 faces along d (the face below cell q,
// then the top face), k fastest; on a periodic axis the last face is the
// first again and both are written.

#include "bmg_internal.h"

namespace bmg {

namespace {

__global__ void k_project_rhs(const double* __restrict__ u0, const double* __restrict__ u1,
                              const double* __restrict__ u2, double* __restrict__ out, ProjGeom G) {
    const int n1 = G.n[1], n2 = G.n[2];
    const int i = blockIdx.z, j = blockIdx.y;
    const double h0 = G.h[0][i], h1 = G.h[1][j];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n2; k += gridDim.x * blockDim.x) {
        const long f0 = ((long)i * n1 + j) * n2 + k;
        const long f1 = ((long)i * (n1 + 1) + j) * n2 + k;
        const long f2 = ((long)i * n1 + j) * (n2 + 1) + k;
        const double h2 = G.h[2][k];
        // sum of U A over the faces, then divided by V (A / V = 1 / h along each axis)
        const double div = (u0[f0 + (long)n1 * n2] - u0[f0]) / h0 + (u1[f1 + n2] - u1[f1]) / h1 +
                           (u2[f2 + 1] - u2[f2]) / h2;
        const double b = div / (-G.cdt);
        out[((long)i * n1 + j) * n2 + k] = G.perVolume ? b : -(h0 * h1 * h2) * b;
    }
}

// faces of axis A: grid over (faces along k for A == 2 / cells along k, rows)
template <int A>
__global__ void k_project_correct(double* __restrict__ u, const double* __restrict__ p,
                                  const double* __restrict__ lam, ProjGeom G) {
    const int n0 = G.n[0], n1 = G.n[1], n2 = G.n[2];
    const int i = blockIdx.z, j = blockIdx.y;  // face coordinates (the face index along A is i, j or k)
    const int e0 = A == 0 ? n0 + 1 : n0, e1 = A == 1 ? n1 + 1 : n1, e2 = A == 2 ? n2 + 1 : n2;
    if (i >= e0 || j >= e1) return;
    const int nA = G.n[A];
    const double* h = G.h[A];
    for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < e2; k += gridDim.x * blockDim.x) {
        const int q = A == 0 ? i : A == 1 ? j : k;  // face index along A
        const long f = ((long)i * e1 + j) * e2 + k;
        int qc = q, ql = q - 1;  // cells above and below the face
        if (q == 0 || q == nA) {
            if (!G.per[A]) continue;  // a wall: zero gradient
            qc = 0;  // across the periodic seam: the first and the last cell
            ql = nA - 1;
        }
        const double delta = 1.0 / (0.5 * (h[qc] + h[ql]));
        auto cell = [&](int qq) {
            const int ci = A == 0 ? qq : i, cj = A == 1 ? qq : j, ck = A == 2 ? qq : k;
            return ((long)ci * n1 + cj) * n2 + ck;
        };
        const double g = (p[cell(qc)] - p[cell(ql)]) * delta;
        const double l = lam ? lam[f] : 1.0;
        u[f] -= G.cdt * (l * g);
    }
}

}  // namespace

void launch_project_rhs(const double* u0, const double* u1, const double* u2, double* out, const ProjGeom& G,
                        cudaStream_t s) {
    const dim3 grid((unsigned)std::min((G.n[2] + 127) / 128, 8), (unsigned)G.n[1], (unsigned)G.n[0]);
    k_project_rhs<<<grid, 128, 0, s>>>(u0, u1, u2, out, G);
}

void launch_project_correct(double* u0, double* u1, double* u2, const double* p, const double* lam0,
                            const double* lam1, const double* lam2, const ProjGeom& G, cudaStream_t s) {
    const int n0 = G.n[0], n1 = G.n[1], n2 = G.n[2];
    k_project_correct<0><<<dim3((unsigned)std::min((n2 + 127) / 128, 8), n1, n0 + 1), 128, 0, s>>>(u0, p, lam0, G);
    k_project_correct<1><<<dim3((unsigned)std::min((n2 + 127) / 128, 8), n1 + 1, n0), 128, 0, s>>>(u1, p, lam1, G);
    k_project_correct<2><<<dim3((unsigned)std::min((n2 + 128) / 128, 8), n1, n0), 128, 0, s>>>(u2, p, lam2, G);
}

}  // namespace bmg
