"""CPU emulation of the tensor-core convolutions' shared-memory tiles.

The loaders of bun_conv.cu write each pipeline stage byte by byte into the
canonical no-swizzle layouts; the MMAs read them back through matrix
descriptors (start address, leading byte offset along K, stride byte offset
along M/N).  Emulating both sides with the same index arithmetic as the
kernels -- and the weight packing of bun_elem.cu -- must reproduce the
convolution, its data gradient and its weight gradient exactly (up to
summation order)."""
import numpy as np
import pytest

from tests import unet_ref as R

TILE = 128


def kmajor(start, lbo, sbo, mn, k):
    """byte address of element (mn, k) of a K-major no-swizzle operand"""
    return start + (mn // 8) * sbo + (k // 8) * lbo + (mn % 8) * 16 + (k % 8) * 2


def mnmajor(start, lbo, sbo, mn, k):
    """byte address of element (mn, k) of an MN-major no-swizzle operand"""
    return start + (mn // 8) * sbo + (k // 8) * lbo + (k % 8) * 16 + (mn % 8) * 2


def pack(W, kc, transpose):
    """bun_elem.cu k_pack: element index -> value, as a flat array"""
    cin, cout = W.shape[1], W.shape[2]
    K, N = (cout, cin) if transpose else (cin, cout)
    out = np.zeros(27 * K * N)
    q = np.arange(out.size)
    blk = q // (N * kc)
    r = q % (N * kc)
    ng, r2 = r // (kc * 8), r % (kc * 8)
    cg, r3 = r2 // 64, r2 % 64
    n, c = ng * 8 + r3 // 8, cg * 8 + r3 % 8
    t, g = blk // (K // kc), blk % (K // kc)
    if not transpose:
        out[:] = W[t, g * kc + c, n]
    else:
        out[:] = W[26 - t, n, g * kc + c]
    return out


def in_value(src0, c0, up0, src1, i, j, k, ch):
    """channel ch of full-resolution voxel (i, j, k) of the kernel's input"""
    if ch < c0:
        if up0:
            return src0[i // 2, j // 2, k // 2, ch]
        return src0[i, j, k, ch]
    return src1[i, j, k, ch - c0]


def emulate_conv(dims, src0, c0, up0, src1, c1, W, kc, transpose=False):
    n0, n1, n2 = dims
    cout = W.shape[1] if transpose else W.shape[2]
    wp = pack(W, kc, transpose)
    V = n0 * n1 * n2
    cin = c0 + c1
    nq = cin // kc
    out = np.zeros((V, cout))
    a_bytes = TILE * kc * 2
    for tile in range(-(-V // TILE)):
        acc = np.zeros((TILE, cout))
        for it in range(27 * nq):
            t, qq = divmod(it, nq)
            di, dj, dk = R.TAPS[t]
            smem = np.zeros((a_bytes + cout * kc * 2) // 2)  # one value per BF16 slot
            # A: producer thread m writes its row
            for m in range(TILE):
                v = tile * TILE + m
                if v >= V:
                    continue
                i, r = divmod(v, n1 * n2)
                j, k = divmod(r, n2)
                ii, jj, kk = i + di, j + dj, k + dk
                if not (0 <= ii < n0 and 0 <= jj < n1 and 0 <= kk < n2):
                    continue
                a_off = (m >> 3) * (kc * 16) + (m & 7) * 16
                for h in range(kc // 8):
                    for e in range(8):
                        smem[(a_off + h * 128) // 2 + e] = in_value(src0, c0, up0, src1, ii, jj, kk,
                                                                     qq * kc + h * 8 + e)
            # B: contiguous block of the packed weights
            smem[a_bytes // 2:] = wp[it * cout * kc:(it + 1) * cout * kc]
            # MMAs: kc/16 of 128 x cout x 16
            mm, kk_ = np.meshgrid(np.arange(TILE), np.arange(16), indexing="ij")
            nn, kb = np.meshgrid(np.arange(cout), np.arange(16), indexing="ij")
            for q in range(kc // 16):
                A = smem[kmajor(q * 256, 128, kc * 16, mm, kk_) // 2]
                B = smem[kmajor(a_bytes + q * 256, 128, kc * 16, nn, kb) // 2]
                acc += A @ B.T
        hi = min(V, (tile + 1) * TILE)
        out[tile * TILE:hi] = acc[:hi - tile * TILE]
    return out.reshape(n0, n1, n2, cout)


def emulate_wgrad(dims, src0, c0, up0, src1, c1, dz, nsplit):
    n0, n1, n2 = dims
    cin = c0 + c1
    cout = dz.shape[3]
    rows = 27 * cin
    rows_pad = -(-rows // 128) * 128
    V = n0 * n1 * n2
    nblk = -(-V // TILE)
    dzf = dz.reshape(V, cout)
    part = np.zeros((nsplit, rows_pad, cout))
    a_bytes = 128 * TILE * 2
    for mt in range(rows_pad // 128):
        for split in range(nsplit):
            acc = np.zeros((128, cout))
            for blk in range(split, nblk, nsplit):
                smem = np.zeros((a_bytes + cout * TILE * 2) // 2)
                for tid in range(TILE):
                    v = blk * TILE + tid
                    if v >= V:
                        continue
                    i, r = divmod(v, n1 * n2)
                    j, k = divmod(r, n2)
                    off = (tid >> 3) * 128 + (tid & 7) * 16
                    for g in range(16):
                        r0 = mt * 128 + g * 8
                        if r0 >= rows:
                            continue
                        t, ch = divmod(r0, cin)
                        di, dj, dk = R.TAPS[t]
                        ii, jj, kk = i + di, j + dj, k + dk
                        if 0 <= ii < n0 and 0 <= jj < n1 and 0 <= kk < n2:
                            for e in range(8):
                                smem[(g * 2048 + off) // 2 + e] = in_value(src0, c0, up0, src1, ii, jj, kk, ch + e)
                    for g in range(cout // 8):
                        smem[(a_bytes + g * 2048 + off) // 2:(a_bytes + g * 2048 + off) // 2 + 8] = \
                            dzf[v, g * 8:g * 8 + 8]
                mm, kk_ = np.meshgrid(np.arange(128), np.arange(16), indexing="ij")
                nn, kb = np.meshgrid(np.arange(cout), np.arange(16), indexing="ij")
                for q in range(TILE // 16):
                    A = smem[mnmajor(q * 256, 128, 2048, mm, kk_) // 2]
                    B = smem[mnmajor(a_bytes + q * 256, 128, 2048, nn, kb) // 2]
                    acc += A @ B.T
            part[split, mt * 128:(mt + 1) * 128] = acc
    return part.sum(axis=0)[:rows].reshape(27, cin, cout)


def _case(rng, dims, c0, up0, c1):
    half = tuple(d // 2 for d in dims) if up0 else dims
    src0 = rng.standard_normal(half + (c0,))
    src1 = rng.standard_normal(dims + (c1,)) if c1 else None
    x = np.concatenate([R.up(src0) if up0 else src0, src1], axis=3) if c1 else (R.up(src0) if up0 else src0)
    return src0, src1, x


@pytest.mark.parametrize("dims,c0,up0,c1,cout,kc", [
    ((2, 4, 20), 16, 0, 0, 16, 16),    # 160 voxels: a partial second tile
    ((4, 4, 8), 32, 1, 16, 32, 16),    # upsampled source + skip
    ((2, 2, 32), 64, 0, 0, 32, 64),
])
def test_conv_tiles_reproduce_convolution(dims, c0, up0, c1, cout, kc):
    rng = np.random.default_rng(7)
    src0, src1, x = _case(rng, dims, c0, up0, c1)
    W = rng.standard_normal((27, c0 + c1, cout))
    got = emulate_conv(dims, src0, c0, up0, src1, c1, W, kc)
    assert np.allclose(got, R.conv3(x, W), rtol=1e-12, atol=1e-10)


def test_dgrad_tiles_reproduce_adjoint():
    rng = np.random.default_rng(8)
    dims, cin, cout = (2, 4, 16), 48, 16
    W = rng.standard_normal((27, cin, cout))
    dz = rng.standard_normal(dims + (cout,))
    got = emulate_conv(dims, dz, cout, 0, None, 0, W, 16, transpose=True)
    assert np.allclose(got, R.conv3_dgrad(dz, W), rtol=1e-12, atol=1e-10)


@pytest.mark.parametrize("dims,c0,up0,c1,cout,nsplit", [
    ((2, 4, 20), 16, 0, 0, 16, 1),
    ((4, 4, 8), 32, 1, 16, 32, 2),
])
def test_wgrad_tiles_reproduce_weight_gradient(dims, c0, up0, c1, cout, nsplit):
    rng = np.random.default_rng(9)
    src0, src1, x = _case(rng, dims, c0, up0, c1)
    dz = rng.standard_normal(dims + (cout,))
    got = emulate_wgrad(dims, src0, c0, up0, src1, c1, dz, nsplit)
    assert np.allclose(got, R.conv3_wgrad(x, dz), rtol=1e-12, atol=1e-10)


def test_descriptor_reads_stay_inside_the_stage():
    """every address an MMA reads lies inside its stage buffer"""
    for kc in (16, 32, 64):
        for cout in (16, 32, 48, 64, 96, 128):
            a_bytes = TILE * kc * 2
            stage = a_bytes + cout * kc * 2
            mm, kk = np.meshgrid(np.arange(128), np.arange(16), indexing="ij")
            nn, kb = np.meshgrid(np.arange(cout), np.arange(16), indexing="ij")
            for q in range(kc // 16):
                assert kmajor(q * 256, 128, kc * 16, mm, kk).max() + 2 <= a_bytes
                assert kmajor(a_bytes + q * 256, 128, kc * 16, nn, kb).max() + 2 <= stage
    for cout in (16, 32, 64):
        a_bytes = 128 * TILE * 2
        stage = a_bytes + cout * TILE * 2
        mm, kk = np.meshgrid(np.arange(128), np.arange(16), indexing="ij")
        nn, kb = np.meshgrid(np.arange(cout), np.arange(16), indexing="ij")
        for q in range(TILE // 16):
            assert mnmajor(q * 256, 128, 2048, mm, kk).max() + 2 <= a_bytes
            assert mnmajor(a_bytes + q * 256, 128, 2048, nn, kb).max() + 2 <= stage


ROW_VOX, ROW_CHUNK = 130, 130 * 16


def emulate_rows(dims, src0, c0, up0, src1, c1, W):
    """bun_conv.cu k_conv_rows: row-sets of 3 rows x 130 voxels laid out
    [chunk][voxel] x 16 B, tap operands by start-address shifts"""
    n0, n1, n2 = dims
    cin, cout = c0 + c1, W.shape[2]
    nq = cin // 16
    wp = pack(W, 16, False)
    row_b = (cin // 8) * ROW_CHUNK
    set_b = 3 * row_b
    out = np.zeros((n0, n1, n2, cout))
    mm, kk_ = np.meshgrid(np.arange(TILE), np.arange(16), indexing="ij")
    nn, kb = np.meshgrid(np.arange(cout), np.arange(16), indexing="ij")
    for k0 in range(0, n2, TILE):
        for i in range(n0):
            for j in range(n1):
                # the three row-sets j-1, j, j+1 (one value per BF16 slot)
                smem = np.zeros(3 * set_b // 2)
                wbase = 3 * set_b
                for dj in range(3):
                    jj = j + dj - 1
                    for di in range(3):
                        ii = i + di - 1
                        for kk in range(ROW_VOX):
                            k = k0 - 1 + kk
                            if not (0 <= jj < n1 and 0 <= ii < n0 and 0 <= k < n2):
                                continue
                            for h in range(cin // 8):
                                a = (dj * set_b + di * row_b + h * ROW_CHUNK + kk * 16) // 2
                                for e in range(8):
                                    smem[a + e] = in_value(src0, c0, up0, src1, ii, jj, k, h * 8 + e)
                wsm = wp  # weights follow the ring in shared memory
                acc = np.zeros((TILE, cout))
                for dj in range(3):
                    for di in range(3):
                        for dk in range(3):
                            t = di * 9 + dj * 3 + dk
                            for u in range(nq):
                                st = dj * set_b + di * row_b + 2 * u * ROW_CHUNK + dk * 16
                                A = smem[kmajor(st, ROW_CHUNK, 128, mm, kk_) // 2]
                                bs = (t * nq + u) * cout * 32
                                B = wsm[kmajor(bs, 128, 256, nn, kb) // 2]
                                acc += A @ B.T
                out[i, j, k0:k0 + TILE] = acc
    return out


@pytest.mark.parametrize("dims,c0,up0,c1,cout", [((2, 3, 128), 16, 0, 0, 16), ((2, 2, 128), 32, 1, 16, 16),
                                                  ((2, 2, 128), 16, 0, 0, 48)])
def test_row_kernel_tiles_reproduce_convolution(dims, c0, up0, c1, cout):
    rng = np.random.default_rng(10)
    src0, src1, x = _case(rng, dims, c0, up0, c1)
    W = rng.standard_normal((27, c0 + c1, cout))
    got = emulate_rows(dims, src0, c0, up0, src1, c1, W)
    assert np.allclose(got, R.conv3(x, W), rtol=1e-12, atol=1e-10)


def test_row_kernel_reads_stay_inside_the_ring():
    """the farthest operand element of the last row-set slot (row di = +1,
    last channel pair, tap dk = +1) lies inside the ring, and an operand
    never reads past voxel 129 of its row"""
    mm, kk = np.meshgrid(np.arange(128), np.arange(16), indexing="ij")
    for cin in (16, 32, 48):
        row_b = (cin // 8) * ROW_CHUNK
        for nr in (3, 4):
            start = (nr - 1) * 3 * row_b + 2 * row_b + 2 * (cin // 16 - 1) * ROW_CHUNK + 2 * 16
            assert kmajor(start, ROW_CHUNK, 128, mm, kk).max() + 2 <= nr * 3 * row_b
    # within one channel chunk (k < 8): voxel 2 + 127 = 129 at most
    m8, k8 = np.meshgrid(np.arange(128), np.arange(8), indexing="ij")
    assert (kmajor(2 * 16, ROW_CHUNK, 128, m8, k8) // 16).max() == 129
