"""The U-Net kernels of libbunet.so on the GPU against the FP64 reference
(tests/unet_ref.py).  Inputs are rounded to BF16 first, so a kernel's only
errors are its FP32 accumulation and the BF16 rounding of its output:
  * tensor-core convolution (forward, data gradient): relative L2 error
    <= 4e-3 (BF16 output rounding is 2^-9 relative);
  * weight gradient (FP32 output): <= 1e-4;
  * the whole network, 18 layers of BF16 activations: output <= 3e-2,
    parameter gradients <= 1e-1 (relative L2 per layer)."""
import ctypes

import numpy as np
import pytest

from tests import unet_ref as R

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def L():
    from briscola_b200 import unet
    from briscola_b200.build import build_unet

    build_unet()
    return unet.load()


def dev(a, dtype):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to("cuda").to(dtype)


def host(t):
    return t.float().cpu().numpy().astype(np.float64)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def S():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


CONV_CASES = [
    # dims, c0, up0, c1, cout, kc
    ((8, 8, 8), 16, 0, 0, 16, 16),
    ((6, 10, 12), 16, 0, 0, 32, 16),   # 720 voxels: a partial last tile
    ((8, 8, 16), 32, 0, 0, 64, 32),
    ((8, 8, 8), 64, 0, 0, 64, 64),
    ((8, 8, 8), 64, 1, 64, 64, 64),    # decoder: upsampled + skip
    ((8, 16, 8), 64, 1, 32, 32, 32),
    ((16, 8, 8), 32, 1, 16, 16, 16),
    # rows of 128 voxels with kc = 16: the row-marching kernel
    ((2, 3, 128), 16, 0, 0, 16, 16),
    ((4, 4, 128), 16, 0, 0, 32, 16),
    ((2, 4, 128), 32, 1, 16, 16, 16),   # upsampled + skip, 48 channels
    ((2, 2, 128), 32, 0, 0, 32, 16),
    ((2, 2, 256), 32, 0, 0, 16, 16),    # two k-segments
    ((1, 40, 128), 16, 0, 0, 16, 16),   # two j-segments (32 + 8 rows)
]


def _inputs(rng, dims, c0, up0, c1):
    half = tuple(d // 2 for d in dims) if up0 else dims
    s0 = R.bf16(rng.standard_normal(half + (c0,)))
    s1 = R.bf16(rng.standard_normal(dims + (c1,))) if c1 else None
    u = R.up(s0) if up0 else s0
    x = np.concatenate([u, s1], axis=3) if c1 else u
    return s0, s1, x


@pytest.mark.parametrize("dims,c0,up0,c1,cout,kc", CONV_CASES)
@pytest.mark.parametrize("relu", [0, 1])
def test_conv_forward(L, dims, c0, up0, c1, cout, kc, relu):
    rng = np.random.default_rng(hash((dims, c0, c1, cout)) % 2**32)
    s0, s1, x = _inputs(rng, dims, c0, up0, c1)
    W = rng.standard_normal((27, c0 + c1, cout)) / np.sqrt(27 * (c0 + c1))
    Wd = dev(W, torch.float32)
    wp = torch.zeros(W.size, dtype=torch.bfloat16, device="cuda")
    assert L.bun_pack_weights(Wd.data_ptr(), c0 + c1, cout, kc, 0, wp.data_ptr(), S()) == 0
    out = torch.zeros(int(np.prod(dims)) * cout, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0, t1 = dev(s0, torch.bfloat16), (dev(s1, torch.bfloat16) if c1 else None)
    rc = L.bun_conv3(*dims, t0.data_ptr(), c0, up0, t1.data_ptr() if c1 else None, c1, wp.data_ptr(), kc, cout,
                     None, relu, None, out.data_ptr(), err.data_ptr(), S())
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = R.conv3(x, R.bf16(W))
    if relu:
        ref = np.maximum(ref, 0)
    got = host(out).reshape(dims + (cout,))
    assert rel(got, ref) <= 4e-3


@pytest.mark.parametrize("dims,cin,cout,kc", [((8, 8, 8), 48, 16, 16), ((8, 8, 8), 128, 64, 64),
                                               ((8, 8, 8), 96, 32, 32), ((8, 8, 8), 16, 32, 32),
                                               ((8, 8, 8), 32, 64, 64),
                                               ((2, 3, 128), 48, 16, 16), ((2, 3, 128), 16, 32, 16),
                                               ((2, 3, 128), 32, 32, 16)])
def test_conv_data_gradient_with_mask(L, dims, cin, cout, kc):
    rng = np.random.default_rng(cin * 7 + cout)
    W = rng.standard_normal((27, cin, cout)) / np.sqrt(27 * cout)
    dz = R.bf16(rng.standard_normal(dims + (cout,)))
    act = R.bf16(np.maximum(rng.standard_normal(dims + (cin,)), 0))
    wp = torch.zeros(W.size, dtype=torch.bfloat16, device="cuda")
    Wd = dev(W, torch.float32)
    assert L.bun_pack_weights(Wd.data_ptr(), cin, cout, kc, 1, wp.data_ptr(), S()) == 0
    out = torch.zeros(int(np.prod(dims)) * cin, dtype=torch.bfloat16, device="cuda")
    dzd, actd = dev(dz, torch.bfloat16), dev(act, torch.bfloat16)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = L.bun_conv3(*dims, dzd.data_ptr(), cout, 0, None, 0, wp.data_ptr(), kc, cin, None, 0, actd.data_ptr(),
                     out.data_ptr(), err.data_ptr(), S())
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = R.conv3_dgrad(dz, R.bf16(W)) * (act > 0)
    assert rel(host(out).reshape(dims + (cin,)), ref) <= 4e-3


@pytest.mark.parametrize("dims,c0,up0,c1,cout,nsplit", [
    ((8, 8, 8), 16, 0, 0, 16, 1),
    ((8, 8, 8), 16, 0, 0, 16, 3),
    ((6, 10, 12), 32, 0, 0, 32, 2),   # partial voxel block
    ((8, 8, 8), 64, 1, 64, 64, 4),
    ((8, 8, 16), 64, 1, 32, 32, 5),
    ((16, 8, 8), 32, 1, 16, 16, 2),
])
def test_conv_weight_gradient(L, dims, c0, up0, c1, cout, nsplit):
    rng = np.random.default_rng(c0 * 3 + c1 + cout + nsplit)
    s0, s1, x = _inputs(rng, dims, c0, up0, c1)
    dz = R.bf16(rng.standard_normal(dims + (cout,)))
    t0, t1 = dev(s0, torch.bfloat16), (dev(s1, torch.bfloat16) if c1 else None)
    dzd = dev(dz, torch.bfloat16)
    part = torch.zeros(L.bun_wgrad_part_floats(c0 + c1, cout, nsplit), dtype=torch.float32, device="cuda")
    dw = torch.zeros(27 * (c0 + c1) * cout, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):  # a second call overwrites, not accumulates
        rc = L.bun_conv3_wgrad(*dims, t0.data_ptr(), c0, up0, t1.data_ptr() if c1 else None, c1, dzd.data_ptr(),
                               cout, nsplit, part.data_ptr(), dw.data_ptr(), err.data_ptr(), S())
        assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = R.conv3_wgrad(x, dz)
    assert rel(host(dw).reshape(27, c0 + c1, cout), ref) <= 1e-4


def test_small_kernels(L):
    rng = np.random.default_rng(3)
    dims = (8, 8, 16)
    V = int(np.prod(dims))
    half = (4, 4, 8)
    # pooling
    s = R.bf16(rng.standard_normal(dims + (32,)))
    sd = dev(s, torch.bfloat16)
    p = torch.zeros(V // 8 * 32, dtype=torch.bfloat16, device="cuda")
    assert L.bun_pool(*dims, 32, sd.data_ptr(), p.data_ptr(), S()) == 0
    assert rel(host(p).reshape(half + (32,)), R.pool(s)) <= 4e-3
    # gradient of the upsampled part of a concatenation
    dcat = R.bf16(rng.standard_normal(dims + (96,)))
    act = R.bf16(np.maximum(rng.standard_normal(half + (64,)), 0))
    dz = torch.zeros(V // 8 * 64, dtype=torch.bfloat16, device="cuda")
    dcd, acd = dev(dcat, torch.bfloat16), dev(act, torch.bfloat16)
    assert L.bun_unpool_grad(*dims, 96, 64, dcd.data_ptr(), acd.data_ptr(), dz.data_ptr(), S()) == 0
    assert rel(host(dz).reshape(half + (64,)), R.sumpool(dcat[..., :64]) * (act > 0)) <= 4e-3
    # skip gradient
    dp = R.bf16(rng.standard_normal(half + (32,)))
    src = R.bf16(np.maximum(rng.standard_normal(dims + (32,)), 0))
    dpd, srd = dev(dp, torch.bfloat16), dev(src, torch.bfloat16)
    dzs = torch.zeros(V * 32, dtype=torch.bfloat16, device="cuda")
    assert L.bun_skip_grad(*dims, 96, 64, 32, dcd.data_ptr(), dpd.data_ptr(), srd.data_ptr(), dzs.data_ptr(),
                           S()) == 0
    ref = (dcat[..., 64:] + R.up(dp) / 8) * (src > 0)
    assert rel(host(dzs).reshape(dims + (32,)), ref) <= 4e-3
    # input convolution and its weight gradient
    x = rng.standard_normal(dims)
    w = rng.standard_normal((27, 16)) * 0.2
    b = rng.standard_normal(16) * 0.1
    xd, wd, bd = dev(x, torch.float32), dev(w, torch.float32), dev(b, torch.float32)
    a0 = torch.zeros(V * 16, dtype=torch.bfloat16, device="cuda")
    assert L.bun_conv_in(*dims, xd.data_ptr(), wd.data_ptr(), bd.data_ptr(), a0.data_ptr(), S()) == 0
    x32 = x.astype(np.float32).astype(np.float64)
    ref = np.maximum(R.conv3(x32[..., None], w.astype(np.float32)[:, None, :]) + b.astype(np.float32), 0)
    assert rel(host(a0).reshape(dims + (16,)), ref) <= 4e-3
    g = R.bf16(rng.standard_normal(dims + (16,)))
    gd = dev(g, torch.bfloat16)
    part = torch.zeros(64 * 28 * 16, dtype=torch.float32, device="cuda")
    dw = torch.zeros(28 * 16, dtype=torch.float32, device="cuda")
    assert L.bun_conv_in_wgrad(*dims, xd.data_ptr(), gd.data_ptr(), 64, part.data_ptr(), dw.data_ptr(), S()) == 0
    dwr = np.concatenate([R.conv3_wgrad(x32[..., None], g)[:, 0, :].ravel(), g.sum(axis=(0, 1, 2))])
    assert rel(host(dw), dwr) <= 1e-4
    # head
    d0 = R.bf16(np.maximum(rng.standard_normal(dims + (16,)), 0))
    hw = rng.standard_normal(16)
    hb = np.array([0.3])
    d0d, hwd, hbd = dev(d0, torch.bfloat16), dev(hw, torch.float32), dev(hb, torch.float32)
    y = torch.zeros(V, dtype=torch.float32, device="cuda")
    assert L.bun_head(V, d0d.data_ptr(), hwd.data_ptr(), hbd.data_ptr(), y.data_ptr(), S()) == 0
    assert rel(host(y).reshape(dims), d0 @ hw.astype(np.float32) + 0.3) <= 1e-5
    dy = rng.standard_normal(dims)
    dyd = dev(dy, torch.float32)
    dzh = torch.zeros(V * 16, dtype=torch.bfloat16, device="cuda")
    dwh = torch.zeros(17, dtype=torch.float32, device="cuda")
    assert L.bun_head_grad(V, d0d.data_ptr(), dyd.data_ptr(), hwd.data_ptr(), dzh.data_ptr(), 16, part.data_ptr(),
                           dwh.data_ptr(), S()) == 0
    dy32 = dy.astype(np.float32).astype(np.float64)
    assert rel(host(dwh), np.concatenate([np.einsum("ijkc,ijk->c", d0, dy32), [dy32.sum()]])) <= 1e-4
    assert rel(host(dzh).reshape(dims + (16,)), dy32[..., None] * hw.astype(np.float32) * (d0 > 0)) <= 4e-3


def _lap(y):
    """sum over in-grid neighbours of (y_nb - y)"""
    out = np.zeros_like(y)
    for ax in range(3):
        d = np.diff(y, axis=ax)
        lo = [slice(None)] * 3
        hi = [slice(None)] * 3
        lo[ax] = slice(0, -1)
        hi[ax] = slice(1, None)
        out[tuple(lo)] += d
        out[tuple(hi)] -= d
    return out


def test_laplace_residual_kernels(L):
    rng = np.random.default_rng(4)
    dims = (8, 12, 16)
    y, f, g, dy = (rng.standard_normal(dims) for _ in range(4))
    yd, fd, gd, dyd = (dev(a, torch.float32) for a in (y, f, g, dy))
    r = torch.zeros(int(np.prod(dims)), dtype=torch.float32, device="cuda")
    assert L.bun_laplace_residual(*dims, yd.data_ptr(), fd.data_ptr(), 0.25, r.data_ptr(), S()) == 0
    assert L.bun_laplace_add(*dims, gd.data_ptr(), 0.5, dyd.data_ptr(), S()) == 0
    assert rel(host(r).reshape(dims), _lap(y) + 0.25 * f) <= 1e-6
    assert rel(host(dyd).reshape(dims), dy + 0.5 * _lap(g)) <= 1e-6


def test_argument_checks(L):
    t = torch.zeros(4096, dtype=torch.bfloat16, device="cuda")
    # unsupported (kc, cout), misaligned pointer, channel count not a multiple of kc
    assert L.bun_conv3(8, 8, 8, t.data_ptr(), 16, 0, None, 0, t.data_ptr(), 16, 128, None, 0, None,
                       t.data_ptr(), None, S()) == 3
    assert L.bun_conv3(8, 8, 8, t.data_ptr() + 2, 16, 0, None, 0, t.data_ptr(), 16, 16, None, 0, None,
                       t.data_ptr(), None, S()) == 3
    assert L.bun_conv3(8, 8, 8, t.data_ptr(), 24, 0, None, 0, t.data_ptr(), 16, 16, None, 0, None,
                       t.data_ptr(), None, S()) == 3
    # upsampled source needs even extents
    assert L.bun_conv3(7, 8, 8, t.data_ptr(), 16, 1, t.data_ptr(), 16, t.data_ptr(), 16, 16, None, 0, None,
                       t.data_ptr(), None, S()) == 3
    assert L.bun_conv3_wgrad(8, 8, 8, t.data_ptr(), 16, 0, None, 0, t.data_ptr(), 48, 1, None, None, None,
                             S()) == 3


def test_network_matches_reference(L):
    from briscola_b200 import unet

    rng = np.random.default_rng(5)
    dims = (16, 16, 16)
    p = unet.init_params(11)
    layout, n = unet.param_layout()
    for name, shape, off in layout:
        if name.endswith(".b"):
            p[off:off + int(np.prod(shape))] = 0.05 * rng.standard_normal(int(np.prod(shape)))
    net = unet.UNet(dims, params=p)
    x = rng.standard_normal(dims)
    target = rng.standard_normal(dims)
    xd = dev(x, torch.float32).reshape(-1)
    td = dev(target, torch.float32).reshape(-1)
    y = net.forward(xd)
    net.mse(td)
    net.backward()
    torch.cuda.synchronize()
    net.check_errors()
    P = R.unpack(p.astype(np.float64))
    x32 = x.astype(np.float32).astype(np.float64)
    yr, act = R.forward(P, x32)
    assert rel(host(y).reshape(dims), yr) <= 3e-2
    # gradient of the loss computed from the GPU's own output
    dy = 2.0 * (host(y).reshape(dims) - target.astype(np.float32)) / x.size
    G = R.flat(R.backward(P, x32, act, dy))
    g = host(net.g)
    for name, shape, off in layout:
        size = int(np.prod(shape))
        e = rel(g[off:off + size], G[off:off + size])
        assert e <= 1e-1, (name, e)
    loss = float(net.loss.item())
    assert abs(loss - np.mean((host(y).reshape(dims) - target.astype(np.float32)) ** 2)) <= 1e-4 * loss


def test_network_row_kernels_match_reference(L):
    """level 0 on 128-voxel rows runs the row-marching kernel"""
    from briscola_b200 import unet

    rng = np.random.default_rng(6)
    dims = (8, 8, 128)
    p = unet.init_params(12)
    net = unet.UNet(dims, params=p)
    assert net.kcf["e0b"] == 16 and net.kcf["d0a"] == 16 and net.kcd["d0a"] == 16
    x = rng.standard_normal(dims)
    target = rng.standard_normal(dims)
    y = net.forward(dev(x, torch.float32).reshape(-1))
    net.mse(dev(target, torch.float32).reshape(-1))
    net.backward()
    torch.cuda.synchronize()
    net.check_errors()
    P = R.unpack(p.astype(np.float64))
    x32 = x.astype(np.float32).astype(np.float64)
    yr, act = R.forward(P, x32)
    assert rel(host(y).reshape(dims), yr) <= 3e-2
    dy = 2.0 * (host(y).reshape(dims) - target.astype(np.float32)) / x.size
    G = R.flat(R.backward(P, x32, act, dy))
    g = host(net.g)
    layout, n = unet.param_layout()
    for name, shape, off in layout:
        size = int(np.prod(shape))
        assert rel(g[off:off + size], G[off:off + size]) <= 1e-1, name


def test_training_reduces_loss(L):
    """Fit the network to a fixed smooth target: the loss must fall."""
    from briscola_b200 import unet

    dims = (16, 16, 16)
    rng = np.random.default_rng(2)
    net = unet.UNet(dims, seed=4)
    x = rng.standard_normal(dims)
    ii, jj, kk = np.meshgrid(*[np.arange(16)] * 3, indexing="ij")
    target = np.sin(np.pi * (ii + 0.5) / 16) * np.cos(np.pi * (jj + 0.5) / 16) * 0.5
    xd = dev(x, torch.float32).reshape(-1)
    td = dev(target, torch.float32).reshape(-1)
    losses = []
    for _ in range(60):
        losses.append(float(net.train_step(xd, td, lr=2e-3).item()))
    net.check_errors()
    assert np.isfinite(losses).all()
    assert losses[-1] < 0.2 * losses[0], losses[::10]
