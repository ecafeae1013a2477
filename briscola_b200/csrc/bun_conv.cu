// bun_conv.cu -- 3x3x3 convolutions of the U-Net as implicit GEMMs on the
// sm_100a tensor cores (tcgen05.mma kind::f16, BF16 operands, FP32
// accumulators in tensor memory).
//
// Forward and data-gradient kernel (k_conv): one CTA computes a tile of 128
// consecutive voxels x all output channels.  GEMM view: M = voxels, N =
// output channels, K = 27 taps x input channels, walked in stages of one tap
// and KC channels.  Warps 0-3 load the stages with cp.async (the A tile is
// the tile's voxels shifted by the tap, zero-filled outside the grid; the B
// tile is a contiguous block of the packed weights) and signal a full
// barrier per stage; one thread of warp 4 issues KC/16 MMAs per stage and
// releases the stage through tcgen05.commit; after the last stage warps 0-3
// read the accumulator rows from tensor memory (thread = voxel = TMEM lane)
// and apply bias, ReLU or a ReLU mask before storing BF16.
//
// Weight-gradient kernel (k_wgrad): GEMM view M = (tap, input channel) rows
// in tiles of 128, N = output channels, K = voxels; both operands are read
// MN-major (channels contiguous), which is the channels-last layout of the
// activations, so the A tile is 16 row groups of 8 channels x 128 voxels of
// the tap-shifted input and the B tile the matching 128 voxels of the output
// gradient.  K is split over grid.y; each split writes FP32 partial sums
// that a CUDA-core kernel adds in a fixed order.
//
// Shared-memory operand layouts are the canonical no-swizzle (interleaved)
// ones of the tcgen05 matrix descriptors: a core matrix is 8 rows of 16
// bytes (128 contiguous bytes).  K-major tiles: a row is one M/N index with
// 8 consecutive K elements; core matrices 128 bytes apart along K (leading
// byte offset) and one row group apart along M/N (stride byte offset).
// MN-major tiles: a row is one K index with 8 consecutive M/N elements; core
// matrices 128 bytes apart along K (leading) and 2 KB apart along M/N
// (stride).
//
// Every wait on a barrier is bounded (about two seconds of SM clock); a
// thread that gives up records kErrTimeout, stops issuing work, and the CTA
// still waits for its issued MMAs before freeing tensor memory.

#include "bun_internal.h"

namespace bun {

namespace {

constexpr int kTile = 128;       // voxels per conv tile / per wgrad K block
constexpr int kProducers = 128;  // warps 0-3: loads, then the epilogue
constexpr int kThreads = 160;    // + warp 4: TMEM allocation and MMA issue
constexpr long long kWaitCycles = 4000000000LL;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// wait until the phase with this parity has completed; false on timeout
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const long long t0 = clock64();
    while (!mbar_test(bar, parity))
        if (clock64() - t0 > kWaitCycles) return false;
    return true;
}

// 16-byte global -> shared copy; zero-filled when !valid (src is not read)
__device__ __forceinline__ void cp16(uint32_t dst, const void* src, bool valid) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(valid ? 16 : 0)
                 : "memory");
}

// arrive on the barrier once this thread's cp.async copies have landed
__device__ __forceinline__ void cp_arrive(uint64_t* bar) {
    asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// whole warp
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_free(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// no-swizzle shared-memory matrix descriptor (version 1)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// instruction descriptor: BF16 x BF16 -> FP32, M x N, operand majorness
__host__ __device__ constexpr uint32_t idesc_bf16(int m, int n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((a_mn ? 1u : 0u) << 15) | ((b_mn ? 1u : 0u) << 16) |
           ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void umma(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// arrive on the barrier when every MMA issued so far has completed
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int q = 0; q < 16; ++q) v[q] = __uint_as_float(r[q]);
}

// the 8-channel chunk starting at channel ch of full-resolution voxel
// (i, j, k) of the (possibly concatenated, possibly upsampled) input
__device__ __forceinline__ const bf16* in_ptr(const ConvIn& in, int n1, int n2, int i, int j, int k, int ch) {
    if (ch < in.c0) {
        if (in.up0) {
            i >>= 1;
            j >>= 1;
            k >>= 1;
            n1 >>= 1;
            n2 >>= 1;
        }
        return in.src0 + (((long)i * n1 + j) * n2 + k) * in.c0 + ch;
    }
    return in.src1 + (((long)i * n1 + j) * n2 + k) * in.c1 + (ch - in.c0);
}

template <int NOUT>
__host__ __device__ constexpr int tmem_cols() {
    return NOUT <= 32 ? 32 : NOUT <= 64 ? 64 : NOUT <= 128 ? 128 : 256;
}

// ---------------------------------------------------------------------------
// forward / data-gradient convolution
// ---------------------------------------------------------------------------
template <int KC, int NOUT, int S>
__global__ void __launch_bounds__(kThreads) k_conv(ConvArgs a) {
    constexpr int A_BYTES = kTile * KC * 2;
    constexpr int B_BYTES = NOUT * KC * 2;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t NCOLS = tmem_cols<NOUT>();
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
    uint64_t* empty = full + S;
    uint64_t* accb = empty + S;
    uint32_t* slot = reinterpret_cast<uint32_t*>(accb + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
    const int nq = (a.in.c0 + a.in.c1) / KC;
    const int iters = 27 * nq;
    const long V = (long)n0 * n1 * n2;
    const long v = (long)blockIdx.x * kTile + (tid & (kTile - 1));

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], kProducers);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accb, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 4) tmem_alloc(slot, NCOLS);
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = *slot;
    bool ok = true;

    if (warp < 4) {
        // ---- producers: one voxel row of every A tile, a share of the B tile
        const bool row = v < V;
        int i = 0, j = 0, k = 0;
        if (row) {
            k = (int)(v % n2);
            const long q = v / n2;
            j = (int)(q % n1);
            i = (int)(q / n1);
        }
        const uint32_t a_off = (uint32_t)(tid >> 3) * (KC * 16) + (uint32_t)(tid & 7) * 16;
        const uint32_t base = smem_u32(smem);
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            const uint32_t use = (uint32_t)(it / S);
            if (!mbar_wait(&empty[s], (use & 1) ^ 1)) {
                ok = false;
                break;
            }
            const int t = it / nq, qq = it - t * nq;
            const int ii = i + t / 9 - 1, jj = j + (t / 3) % 3 - 1, kk = k + t % 3 - 1;
            const bool valid = row && ii >= 0 && ii < n0 && jj >= 0 && jj < n1 && kk >= 0 && kk < n2;
            const bf16* src = valid ? in_ptr(a.in, n1, n2, ii, jj, kk, qq * KC) : a.wpack;
            const uint32_t As = base + s * STAGE;
#pragma unroll
            for (int h = 0; h < KC / 8; ++h) cp16(As + a_off + h * 128, src + (valid ? h * 8 : 0), valid);
            const bf16* w = a.wpack + (long)it * (NOUT * KC);
            const uint32_t Bs = As + A_BYTES;
            for (int c = tid; c < NOUT * KC / 8; c += kProducers) cp16(Bs + c * 16, w + c * 8, true);
            cp_arrive(&full[s]);
        }
    } else if (tid == kProducers) {
        // ---- MMA issue: KC/16 MMAs of 128 x NOUT x 16 per stage
        constexpr uint32_t idesc = idesc_bf16(kTile, NOUT, false, false);
        const uint32_t base = smem_u32(smem);
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            const uint32_t use = (uint32_t)(it / S);
            if (!mbar_wait(&full[s], use & 1)) {
                ok = false;
                break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_after();
            const uint32_t As = base + s * STAGE, Bs = As + A_BYTES;
#pragma unroll
            for (int q = 0; q < KC / 16; ++q)
                umma(tmem, sdesc(As + q * 256, 128, KC * 16), sdesc(Bs + q * 256, 128, KC * 16), idesc,
                     (it | q) != 0);
            umma_commit(&empty[s]);
        }
        umma_commit(accb);
    }

    if (warp < 4) {
        // ---- epilogue: thread = voxel = TMEM lane
        bool done = mbar_wait(accb, 0);
        done = __all_sync(0xffffffffu, done);
        tc_after();
        if (!done) ok = false;
        if (done) {
            const bool row = v < V;
#pragma unroll 1
            for (int c0 = 0; c0 < NOUT; c0 += 16) {
                float acc[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
                if (!row) continue;
                if (a.bias) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) acc[q] += a.bias[c0 + q];
                }
                if (a.relu) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) acc[q] = fmaxf(acc[q], 0.f);
                }
                if (a.mask) {
                    const uint4* mp = reinterpret_cast<const uint4*>(a.mask + v * NOUT + c0);
                    uint4 mv[2] = {mp[0], mp[1]};
                    const bf16* m = reinterpret_cast<const bf16*>(mv);
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (!(__bfloat162float(m[q]) > 0.f)) acc[q] = 0.f;
                }
                uint4 ov[2];
                __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(ov);
#pragma unroll
                for (int q = 0; q < 8; ++q) o[q] = __floats2bfloat162_rn(acc[2 * q], acc[2 * q + 1]);
                uint4* op = reinterpret_cast<uint4*>(a.out + v * NOUT + c0);
                op[0] = ov[0];
                op[1] = ov[1];
            }
        }
    }

    if (!ok && a.err) atomicExch(a.err, kErrTimeout);
    tc_before();
    __syncthreads();
    if (warp == 4) {
        tc_after();
        mbar_wait(accb, 0);  // no MMA may still write the accumulator
        tmem_free(tmem, NCOLS);
    }
}

// ---------------------------------------------------------------------------
// weight gradient
// ---------------------------------------------------------------------------
template <int NOUT, int S>
__global__ void __launch_bounds__(kThreads) k_wgrad(WgradArgs a) {
    constexpr int A_BYTES = 128 * kTile * 2;  // 16 row groups x 16 voxel groups x 128 B
    constexpr int B_BYTES = NOUT * kTile * 2;
    constexpr int STAGE = A_BYTES + B_BYTES;
    constexpr uint32_t NCOLS = tmem_cols<NOUT>();
    extern __shared__ __align__(1024) uint8_t smem[];
    uint64_t* full = reinterpret_cast<uint64_t*>(smem + S * STAGE);
    uint64_t* empty = full + S;
    uint64_t* accb = empty + S;
    uint32_t* slot = reinterpret_cast<uint32_t*>(accb + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
    const int cin = a.in.c0 + a.in.c1;
    const long V = (long)n0 * n1 * n2;
    const long nblk = (V + kTile - 1) / kTile;
    const int split = blockIdx.y;
    const int iters = split < nblk ? (int)((nblk - 1 - split) / a.nsplit + 1) : 0;
    const int mt = blockIdx.x;

    if (tid == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], kProducers);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accb, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 4) tmem_alloc(slot, NCOLS);
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = *slot;
    bool ok = true;

    if (warp < 4) {
        // the 16 row groups of this M tile: tap offset and first channel
        int gdi[16], gdj[16], gdk[16], gch[16];
        bool gon[16];
#pragma unroll
        for (int g = 0; g < 16; ++g) {
            const int r0 = mt * 128 + g * 8;
            const int t = r0 / cin;
            gon[g] = r0 < a.rows;
            gch[g] = r0 - t * cin;
            gdi[g] = t / 9 - 1;
            gdj[g] = (t / 3) % 3 - 1;
            gdk[g] = t % 3 - 1;
        }
        const uint32_t off = (uint32_t)(tid >> 3) * 128 + (uint32_t)(tid & 7) * 16;
        const uint32_t base = smem_u32(smem);
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            const uint32_t use = (uint32_t)(it / S);
            if (!mbar_wait(&empty[s], (use & 1) ^ 1)) {
                ok = false;
                break;
            }
            const long v = ((long)split + (long)it * a.nsplit) * kTile + tid;
            const bool row = v < V;
            int i = 0, j = 0, k = 0;
            if (row) {
                k = (int)(v % n2);
                const long q = v / n2;
                j = (int)(q % n1);
                i = (int)(q / n1);
            }
            const uint32_t As = base + s * STAGE, Bs = As + A_BYTES;
#pragma unroll
            for (int g = 0; g < 16; ++g) {
                const int ii = i + gdi[g], jj = j + gdj[g], kk = k + gdk[g];
                const bool valid = row && gon[g] && ii >= 0 && ii < n0 && jj >= 0 && jj < n1 && kk >= 0 && kk < n2;
                const bf16* src = valid ? in_ptr(a.in, n1, n2, ii, jj, kk, gch[g]) : a.dz;
                cp16(As + g * 2048 + off, src, valid);
            }
#pragma unroll
            for (int g = 0; g < NOUT / 8; ++g) cp16(Bs + g * 2048 + off, row ? a.dz + v * NOUT + g * 8 : a.dz, row);
            cp_arrive(&full[s]);
        }
    } else if (tid == kProducers) {
        constexpr uint32_t idesc = idesc_bf16(128, NOUT, true, true);
        const uint32_t base = smem_u32(smem);
        for (int it = 0; it < iters; ++it) {
            const int s = it % S;
            const uint32_t use = (uint32_t)(it / S);
            if (!mbar_wait(&full[s], use & 1)) {
                ok = false;
                break;
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_after();
            const uint32_t As = base + s * STAGE, Bs = As + A_BYTES;
#pragma unroll
            for (int q = 0; q < kTile / 16; ++q)
                umma(tmem, sdesc(As + q * 256, 128, 2048), sdesc(Bs + q * 256, 128, 2048), idesc, (it | q) != 0);
            umma_commit(&empty[s]);
        }
        umma_commit(accb);
    }

    if (warp < 4) {
        bool done = mbar_wait(accb, 0);
        done = __all_sync(0xffffffffu, done);
        tc_after();
        if (!done) ok = false;
        if (done) {
            float* dst = a.part + ((long)split * a.rows_pad + (long)mt * 128 + tid) * NOUT;
#pragma unroll 1
            for (int c0 = 0; c0 < NOUT; c0 += 16) {
                float acc[16];
                tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, acc);
                if (iters == 0) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) acc[q] = 0.f;  // nothing was accumulated
                }
#pragma unroll
                for (int q = 0; q < 16; q += 4)
                    *reinterpret_cast<float4*>(dst + c0 + q) = make_float4(acc[q], acc[q + 1], acc[q + 2], acc[q + 3]);
            }
        }
    }

    if (!ok && a.err) atomicExch(a.err, kErrTimeout);
    tc_before();
    __syncthreads();
    if (warp == 4) {
        tc_after();
        mbar_wait(accb, 0);
        tmem_free(tmem, NCOLS);
    }
}

// ---------------------------------------------------------------------------
// forward / data-gradient convolution marching along j (n2 % 128 == 0)
// ---------------------------------------------------------------------------
// A CTA owns plane i and the 128-voxel k-segment k0 .. k0+127 and walks the
// rows j of a segment of kJSeg rows.  For output row j it needs the input
// rows (i+di, j+dj), di, dj in {-1, 0, 1}, over k0-1 .. k0+128; they live in
// a ring of NR row-sets (a row-set = the three rows di = -1, 0, 1 of one j')
// filled once per j' by cp.async, laid out per row as [8-channel chunk h]
// [voxel 0 .. 129] x 16 bytes.  The operand of tap (di, dj, dk) and channels
// 16u .. 16u+15 is then a K-major no-swizzle matrix starting at
//   row(j+dj, di) + 2u * 2080 + (dk + 1) * 16
// with 2080 bytes between channel chunks (leading byte offset) and 128 bytes
// between groups of 8 voxels (stride byte offset): shifting along k is a
// change of start address, so every input row is loaded once, not 27 times.
// All weights stay in shared memory; the TMEM accumulator is double-
// buffered so the epilogue of row j overlaps the MMAs of row j+1.
// Warps 0-3: epilogue (thread = voxel = TMEM lane); warps 4-7: row loader;
// warp 8: TMEM allocation, one thread issues the MMAs.
constexpr int kRowVox = 130;                 // k0-1 .. k0+128
constexpr int kRowChunk = kRowVox * 16;      // bytes of one 8-channel chunk of a row
constexpr int kJSeg = 32;                    // rows per CTA
constexpr int kRowThreads = 288;

template <int CIN, int NOUT, int NR>
struct RowShape {
    static constexpr int ROW = (CIN / 8) * kRowChunk;  // one input row
    static constexpr int SET = 3 * ROW;                // rows di = -1, 0, 1
    static constexpr int WBYTES = 27 * CIN * NOUT * 2;
    static constexpr int NCOLS = NOUT <= 32 ? 32 : NOUT <= 64 ? 64 : 128;
    static constexpr int smem = NR * SET + WBYTES + (2 * NR + 6) * 8 + 16;
};

template <int CIN, int NOUT, int NR>
__global__ void __launch_bounds__(kRowThreads, 1) k_conv_rows(ConvArgs a) {
    using F = RowShape<CIN, NOUT, NR>;
    constexpr int NQ = CIN / 16;
    extern __shared__ __align__(1024) uint8_t smem[];
    // the NR row slots start at smem (addressed through `base` below)
    uint8_t* wts = smem + NR * F::SET;
    uint64_t* full = reinterpret_cast<uint64_t*>(wts + F::WBYTES);
    uint64_t* empty = full + NR;
    uint64_t* wbar = empty + NR;
    uint64_t* tfull = wbar + 1;   // [2]
    uint64_t* tempty = tfull + 2; // [2]
    uint64_t* fin = tempty + 2;   // every MMA of the CTA has completed
    uint32_t* slot = reinterpret_cast<uint32_t*>(fin + 1);

    const int tid = threadIdx.x, warp = tid >> 5;
    const int n0 = a.n0, n1 = a.n1, n2 = a.n2;
    const int k0 = blockIdx.x * kTile;
    const int i = blockIdx.y;
    const int js = blockIdx.z * kJSeg;
    const int je = min(js + kJSeg, n1);
    const int nsteps = je - js;

    if (tid == 0) {
        for (int r = 0; r < NR; ++r) {
            mbar_init(&full[r], kProducers);
            mbar_init(&empty[r], 1);
        }
        mbar_init(wbar, kProducers);
        for (int q = 0; q < 2; ++q) {
            mbar_init(&tfull[q], 1);
            mbar_init(&tempty[q], kProducers);
        }
        mbar_init(fin, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 8) tmem_alloc(slot, 2 * F::NCOLS);
    tc_before();
    __syncthreads();
    tc_after();
    const uint32_t tmem = *slot;
    bool ok = true;
    const uint32_t base = smem_u32(smem);

    if (warp >= 4 && warp < 8) {
        // ---- loader: weights once, then the row-sets js-1 .. je
        const int lt = tid - 128;
        const uint32_t wb = base + NR * F::SET;
        for (int c = lt; c < F::WBYTES / 16; c += kProducers) cp16(wb + c * 16, a.wpack + c * 8, true);
        cp_arrive(wbar);
        for (int jj = js - 1; jj <= je; ++jj) {
            const int q = jj - (js - 1);
            const int r = q % NR;
            const uint32_t use = (uint32_t)(q / NR);
            if (!mbar_wait(&empty[r], (use & 1) ^ 1)) {
                ok = false;
                break;
            }
            const uint32_t sb = base + r * F::SET;
            const bool jok = jj >= 0 && jj < n1;
            // 3 rows x 130 voxels x CIN/8 chunks
            for (int e = lt; e < 3 * kRowVox * (CIN / 8); e += kProducers) {
                const int di = e / (kRowVox * (CIN / 8));
                const int rem = e - di * (kRowVox * (CIN / 8));
                const int h = rem / kRowVox, kk = rem - h * kRowVox;
                const int ii = i + di - 1, k = k0 - 1 + kk;
                const bool valid = jok && ii >= 0 && ii < n0 && k >= 0 && k < n2;
                const bf16* src = valid ? in_ptr(a.in, n1, n2, ii, jj, k, h * 8) : a.wpack;
                cp16(sb + di * F::ROW + h * kRowChunk + kk * 16, src, valid);
            }
            cp_arrive(&full[r]);
        }
    } else if (tid == 256) {
        // ---- MMA issue
        constexpr uint32_t idesc = idesc_bf16(kTile, NOUT, false, false);
        const uint32_t wb = base + NR * F::SET;
        if (!mbar_wait(wbar, 0)) ok = false;
        for (int st = 0; ok && st < nsteps; ++st) {
            const int acc = st & 1;
            const uint32_t ause = (uint32_t)(st >> 1);
            if (!mbar_wait(&tempty[acc], (ause & 1) ^ 1)) {
                ok = false;
                break;
            }
            // row-sets st-1+1 .. st+1+1 in ring order (q = jj - (js-1))
            for (int q = (st == 0 ? 0 : st + 2); q <= st + 2; ++q) {
                if (!mbar_wait(&full[q % NR], (uint32_t)(q / NR) & 1)) ok = false;
            }
            if (!ok) break;
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            tc_after();
            const uint32_t d = tmem + (uint32_t)(acc * F::NCOLS);
            bool first = true;
#pragma unroll 1
            for (int dj = 0; dj < 3; ++dj) {
                const uint32_t set = base + ((st + dj) % NR) * F::SET;
#pragma unroll 1
                for (int di = 0; di < 3; ++di) {
#pragma unroll
                    for (int dk = 0; dk < 3; ++dk) {
                        const int t = di * 9 + dj * 3 + dk;
#pragma unroll
                        for (int u = 0; u < NQ; ++u) {
                            const uint32_t as = set + di * F::ROW + 2 * u * kRowChunk + dk * 16;
                            const uint32_t bs = wb + (uint32_t)((t * NQ + u) * NOUT * 32);
                            umma(d, sdesc(as, kRowChunk, 128), sdesc(bs, 128, 256), idesc, first ? 0u : 1u);
                            first = false;
                        }
                    }
                }
            }
            umma_commit(&tfull[acc]);
            umma_commit(&empty[st % NR]);  // row-set js-1+st is not needed again
        }
        umma_commit(fin);  // one phase, after every MMA issued above
    }

    if (warp < 4) {
        // ---- epilogue
        for (int st = 0; st < nsteps; ++st) {
            const int acc = st & 1;
            bool done = mbar_wait(&tfull[acc], (uint32_t)(st >> 1) & 1);
            done = __all_sync(0xffffffffu, done);
            if (!done) {
                ok = false;
                break;
            }
            tc_after();
            const int j = js + st;
            const long v = ((long)i * n1 + j) * n2 + k0 + tid;
#pragma unroll 1
            for (int c0 = 0; c0 < NOUT; c0 += 16) {
                float accv[16];
                tmem_ld16(tmem + (uint32_t)(acc * F::NCOLS) + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, accv);
                if (a.bias) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) accv[q] += a.bias[c0 + q];
                }
                if (a.relu) {
#pragma unroll
                    for (int q = 0; q < 16; ++q) accv[q] = fmaxf(accv[q], 0.f);
                }
                if (a.mask) {
                    const uint4* mp = reinterpret_cast<const uint4*>(a.mask + v * NOUT + c0);
                    uint4 mv[2] = {mp[0], mp[1]};
                    const bf16* m = reinterpret_cast<const bf16*>(mv);
#pragma unroll
                    for (int q = 0; q < 16; ++q)
                        if (!(__bfloat162float(m[q]) > 0.f)) accv[q] = 0.f;
                }
                uint4 ov[2];
                __nv_bfloat162* o = reinterpret_cast<__nv_bfloat162*>(ov);
#pragma unroll
                for (int q = 0; q < 8; ++q) o[q] = __floats2bfloat162_rn(accv[2 * q], accv[2 * q + 1]);
                uint4* op = reinterpret_cast<uint4*>(a.out + v * NOUT + c0);
                op[0] = ov[0];
                op[1] = ov[1];
            }
            tc_before();
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(&tempty[acc])) : "memory");
        }
    }

    if (!ok && a.err) atomicExch(a.err, kErrTimeout);
    tc_before();
    __syncthreads();
    if (warp == 8) {
        tc_after();
        mbar_wait(fin, 0);  // no MMA may still write the accumulators
        tmem_free(tmem, 2 * F::NCOLS);
    }
}

constexpr int conv_stages(int kc, int nout) {
    return (96 * 1024) / (kc * 2 * (kTile + nout)) > 6   ? 6
           : (96 * 1024) / (kc * 2 * (kTile + nout)) < 2 ? 2
                                                          : (96 * 1024) / (kc * 2 * (kTile + nout));
}

template <int KC, int NOUT>
cudaError_t conv_inst(const ConvArgs& a, cudaStream_t s) {
    constexpr int S = conv_stages(KC, NOUT);
    constexpr int smem = S * (KC * 2 * (kTile + NOUT)) + (2 * S + 1) * 8 + 16;
    cudaError_t e = cudaFuncSetAttribute(k_conv<KC, NOUT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long V = (long)a.n0 * a.n1 * a.n2;
    k_conv<KC, NOUT, S><<<(unsigned)((V + kTile - 1) / kTile), kThreads, smem, s>>>(a);
    return cudaGetLastError();
}

template <int NOUT>
cudaError_t wgrad_inst(const WgradArgs& a, cudaStream_t s) {
    constexpr int S = 3;
    constexpr int smem = S * (128 * kTile * 2 + NOUT * kTile * 2) + (2 * S + 1) * 8 + 16;
    cudaError_t e = cudaFuncSetAttribute(k_wgrad<NOUT, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    k_wgrad<NOUT, S><<<dim3((unsigned)(a.rows_pad / 128), (unsigned)a.nsplit), kThreads, smem, s>>>(a);
    return cudaGetLastError();
}

template <int CIN, int NOUT>
cudaError_t rows_inst(const ConvArgs& a, cudaStream_t s) {
    constexpr int NR = RowShape<CIN, NOUT, 4>::smem <= 200 * 1024 ? 4 : 3;
    constexpr int smem = RowShape<CIN, NOUT, NR>::smem;
    static_assert(smem <= 227 * 1024, "row kernel does not fit shared memory");
    cudaError_t e = cudaFuncSetAttribute(k_conv_rows<CIN, NOUT, NR>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         smem);
    if (e != cudaSuccess) return e;
    const dim3 grid((unsigned)(a.n2 / kTile), (unsigned)a.n0, (unsigned)((a.n1 + kJSeg - 1) / kJSeg));
    k_conv_rows<CIN, NOUT, NR><<<grid, kRowThreads, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace

// the row-marching kernel covers these (input channels, output channels)
// on grids with n2 % 128 == 0; other shapes use k_conv
bool rows_supported(int cin, int nout, int n2) {
    if (n2 % 128) return false;
    return (cin == 16 && (nout == 16 || nout == 32 || nout == 48)) || (cin == 32 && (nout == 16 || nout == 32)) ||
           (cin == 48 && nout == 16);
}

cudaError_t rows_launch(const ConvArgs& a, int nout, cudaStream_t s) {
    const int cin = a.in.c0 + a.in.c1;
    if (cin == 16 && nout == 16) return rows_inst<16, 16>(a, s);
    if (cin == 16 && nout == 32) return rows_inst<16, 32>(a, s);
    if (cin == 16 && nout == 48) return rows_inst<16, 48>(a, s);
    if (cin == 32 && nout == 16) return rows_inst<32, 16>(a, s);
    if (cin == 32 && nout == 32) return rows_inst<32, 32>(a, s);
    if (cin == 48 && nout == 16) return rows_inst<48, 16>(a, s);
    return cudaErrorInvalidValue;
}

bool conv_supported(int kc, int nout) {
    switch (kc) {
        case 16: return nout == 16 || nout == 32 || nout == 48 || nout == 64;
        case 32: return nout == 16 || nout == 32 || nout == 64 || nout == 96;
        case 64: return nout == 32 || nout == 64 || nout == 128;
        default: return false;
    }
}

bool wgrad_supported(int cout) { return cout == 16 || cout == 32 || cout == 64; }

#define BUN_CONV_CASE(KC, N) \
    if (kc == KC && nout == N) return conv_inst<KC, N>(a, s);

cudaError_t conv_launch(const ConvArgs& a, int kc, int nout, cudaStream_t s) {
    // rows of 128 voxels with 16-channel weight blocks: the row-marching kernel
    if (kc == 16 && rows_supported(a.in.c0 + a.in.c1, nout, a.n2)) return rows_launch(a, nout, s);
    BUN_CONV_CASE(16, 16)
    BUN_CONV_CASE(16, 32)
    BUN_CONV_CASE(16, 48)
    BUN_CONV_CASE(16, 64)
    BUN_CONV_CASE(32, 16)
    BUN_CONV_CASE(32, 32)
    BUN_CONV_CASE(32, 64)
    BUN_CONV_CASE(32, 96)
    BUN_CONV_CASE(64, 32)
    BUN_CONV_CASE(64, 64)
    BUN_CONV_CASE(64, 128)
    return cudaErrorInvalidValue;
}
#undef BUN_CONV_CASE

cudaError_t wgrad_launch(const WgradArgs& a, int cout, cudaStream_t s) {
    if (cout == 16) return wgrad_inst<16>(a, s);
    if (cout == 32) return wgrad_inst<32>(a, s);
    if (cout == 64) return wgrad_inst<64>(a, s);
    return cudaErrorInvalidValue;
}

}  // namespace bun
