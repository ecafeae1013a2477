// bmg_noalloc.cu -- residual norm ||b - A x||_2 of one brick that allocates
// no device memory.
//
// Who needs it: callers that may not call cudaMalloc at the moment they want
// a residual -- an application that hands all device memory to its own pool
// and forbids stray allocations, a time-step loop that cannot afford the
// device-wide synchronisation an allocation may cause, or a failure path that
// runs after device memory is exhausted and still has to report how far a
// solve got.  They pass their own device arrays; the per-row partial sums go
// to a fixed static device array instead of a temporary buffer.
//
// The arithmetic is the level-0 residual of the solver (the same operator as
// k_residual_norm in bmg_kernels.cu): row-scaled couplings delta/h per axis,
// periodic neighbours wrapped, Neumann wall couplings zero, Dirichlet wall
// couplings doubled against a zero ghost (homogeneous: face values belong
// in b).

#include "../../include/bmg.h"

#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>

namespace {

constexpr int kThreads = 256;

// Scratch shared by every call on a device: one partial sum per (i, j) row.
// 512 KB, held by every GPU that loads the library until the process exits.
static __device__ __align__(256) double g_row_partials[BMG_NOALLOC_MAX_ROWS];

// row-scaled coupling between cell i and its lower (up = 0) or upper (up = 1)
// neighbour along an axis with vertices p[0..n]: 1 / (centre distance * h_i).
// At a wall the neighbour is a ghost: a Neumann wall drops the coupling, a
// (homogeneous) Dirichlet wall doubles it, with the ghost one spacing h_i
// away and read as zero (DirichletBoundaryCondition.C:19-51).  *inner: the
// neighbour is a cell of the brick (or its periodic image).
__device__ __forceinline__ double coupling(const double* p, int n, int i, int up, int periodic, int dirichlet,
                                           bool* inner) {
    const double h = p[i + 1] - p[i];
    double dist;
    *inner = true;
    if (!up) {
        if (i > 0)
            dist = 0.5 * (p[i + 1] - p[i - 1]);
        else if (periodic)
            dist = 0.5 * (h + (p[n] - p[n - 1]));
        else {
            *inner = false;
            return dirichlet ? 2.0 / h / h : 0.0;
        }
    } else {
        if (i < n - 1)
            dist = 0.5 * (p[i + 2] - p[i]);
        else if (periodic)
            dist = 0.5 * (h + (p[1] - p[0]));
        else {
            *inner = false;
            return dirichlet ? 2.0 / h / h : 0.0;
        }
    }
    return 1.0 / dist / h;
}

__device__ __forceinline__ int wrap(int i, int n) { return i < 0 ? i + n : (i >= n ? i - n : i); }

__global__ void __launch_bounds__(kThreads) k_rows(const double* __restrict__ x, const double* __restrict__ b,
                                                   int n0, int n1, int n2, const double* __restrict__ p0,
                                                   const double* __restrict__ p1, const double* __restrict__ p2,
                                                   int per0, int per1, int per2, int dir, double* rows) {
    __shared__ double sh[kThreads / 32];
    const int nrows = n0 * n1;
    for (int q = blockIdx.x; q < nrows; q += gridDim.x) {
        const int i = q / n1, j = q % n1;
        bool in0, in1, in2, in3, in4, in5;
        const double w0 = coupling(p0, n0, i, 0, per0, dir & 1, &in0);
        const double w1 = coupling(p0, n0, i, 1, per0, dir & 2, &in1);
        const double w2 = coupling(p1, n1, j, 0, per1, dir & 4, &in2);
        const double w3 = coupling(p1, n1, j, 1, per1, dir & 8, &in3);
        const double hij = (p0[i + 1] - p0[i]) * (p1[j + 1] - p1[j]);
        const long rim = (long)wrap(i - 1, n0) * n1 + j, rip = (long)wrap(i + 1, n0) * n1 + j;
        const long rjm = (long)i * n1 + wrap(j - 1, n1), rjp = (long)i * n1 + wrap(j + 1, n1);
        double acc = 0.0;
        for (int k = threadIdx.x; k < n2; k += blockDim.x) {
            const double w4 = coupling(p2, n2, k, 0, per2, dir & 16, &in4);
            const double w5 = coupling(p2, n2, k, 1, per2, dir & 32, &in5);
            const int km = wrap(k - 1, n2), kp = wrap(k + 1, n2);
            const long c = (long)q * n2 + k;
            // ghost neighbours (walls) are never read: zero-gradient walls
            // have no coupling, Dirichlet ghosts are zero
            const double s = (in0 ? w0 * x[rim * n2 + k] : 0.0) + (in1 ? w1 * x[rip * n2 + k] : 0.0) +
                             (in2 ? w2 * x[rjm * n2 + k] : 0.0) + (in3 ? w3 * x[rjp * n2 + k] : 0.0) +
                             (in4 ? w4 * x[(long)q * n2 + km] : 0.0) + (in5 ? w5 * x[(long)q * n2 + kp] : 0.0);
            const double d = w0 + w1 + w2 + w3 + w4 + w5;
            const double V = hij * (p2[k + 1] - p2[k]);
            const double r = b[c] + V * (d * x[c] - s);
            acc += r * r;
        }
        for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) t += sh[w];
            rows[q] = t;
        }
        __syncthreads();
    }
}

// fixed-order sum of the row partials: the result does not depend on timing
__global__ void __launch_bounds__(kThreads) k_sum_rows(const double* rows, int nrows, double* out) {
    __shared__ double sh[kThreads];
    double a = 0.0;
    for (int q = threadIdx.x; q < nrows; q += blockDim.x) a += rows[q];
    sh[threadIdx.x] = a;
    __syncthreads();
    for (int s = kThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sqrt(sh[0]);
}

// Device address of the static scratch on the current device.  Host code
// must not pass the symbol itself to a kernel (in host code it names a
// host-side stand-in).  The address is looked up on every call rather than
// cached: a cached address would go stale if the application reset the
// device or recreated its primary context between calls.
int scratchForCurrentDevice(double** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return BMG_NO_DEVICE;
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_row_partials);
    if (e != cudaSuccess) {
        fprintf(stderr, "bmg_residual_norm_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                cudaGetErrorString(e));
        return BMG_CUDA_ERROR;
    }
    *out = static_cast<double*>(p);
    return BMG_OK;
}

}  // namespace

extern "C" int bmg_residual_norm_noalloc(const double* x, const double* b, const int n[3],
                                         const double* points_x, const double* points_y,
                                         const double* points_z, const int bc[6], double* norm_out,
                                         void* stream) {
    if (!x || !b || !n || !points_x || !points_y || !points_z || !bc || !norm_out) return BMG_BAD_ARG;
    int dir = 0;
    for (int d = 0; d < 3; ++d) {
        if (n[d] < 1) return BMG_BAD_ARG;
        if ((bc[2 * d] == BMG_BC_PERIODIC) != (bc[2 * d + 1] == BMG_BC_PERIODIC)) return BMG_BAD_ARG;
        for (int side = 0; side < 2; ++side) {
            const int t = bc[2 * d + side];
            if (t != BMG_BC_NEUMANN && t != BMG_BC_PERIODIC && t != BMG_BC_DIRICHLET) return BMG_BAD_ARG;
            if (t == BMG_BC_DIRICHLET) dir |= 1 << (2 * d + side);
        }
    }
    const long nrows = (long)n[0] * n[1];
    if (nrows > BMG_NOALLOC_MAX_ROWS) {
        fprintf(stderr,
                "bmg_residual_norm_noalloc: n[0]*n[1] = %ld rows exceeds the static scratch of %d rows\n",
                nrows, BMG_NOALLOC_MAX_ROWS);
        return BMG_BAD_ARG;
    }
    // an error left pending by the caller's earlier work is reported, not
    // cleared, and nothing is launched: this call must not swallow it
    if (cudaPeekAtLastError() != cudaSuccess) return BMG_CUDA_ERROR;
    double* rows = nullptr;
    const int rc = scratchForCurrentDevice(&rows);
    if (rc != BMG_OK) return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1)
        return BMG_CUDA_ERROR;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const long grid = 8L * sms;  // eight resident blocks of 256 threads per SM
    const int blocks = (int)(nrows < grid ? nrows : grid);
    k_rows<<<blocks, kThreads, 0, s>>>(x, b, n[0], n[1], n[2], points_x, points_y, points_z,
                                       bc[0] == BMG_BC_PERIODIC, bc[2] == BMG_BC_PERIODIC,
                                       bc[4] == BMG_BC_PERIODIC, dir, rows);
    k_sum_rows<<<1, kThreads, 0, s>>>(rows, (int)nrows, norm_out);
    return cudaGetLastError() == cudaSuccess ? BMG_OK : BMG_CUDA_ERROR;
}
