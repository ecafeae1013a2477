"""The FP64 reference of the U-Net (tests/unet_ref.py) on the CPU: its
hand-written backward pass agrees with finite differences, its operators
with their definitions, and the parameter layout matches the network."""
import numpy as np
import pytest

from briscola_b200 import unet
from tests import unet_ref as R


def test_param_layout_is_contiguous():
    layout, n = unet.param_layout()
    off = 0
    for name, shape, o in layout:
        assert o == off
        off += int(np.prod(shape))
    assert off == n
    names = [x[0] for x in layout]
    # the kernels write weights then bias in one block
    assert names.index("in.b") == names.index("in.w") + 1
    assert names.index("head.b") == names.index("head.w") + 1


def test_conv_adjoints():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((4, 6, 8, 3))
    W = rng.standard_normal((27, 3, 5))
    dz = rng.standard_normal((4, 6, 8, 5))
    # <conv(x, W), dz> = <x, dgrad(dz, W)> = <W, wgrad(x, dz)>
    lhs = (R.conv3(x, W) * dz).sum()
    assert np.isclose(lhs, (x * R.conv3_dgrad(dz, W)).sum())
    assert np.isclose(lhs, (W * R.conv3_wgrad(x, dz)).sum())
    # pool / up / sumpool adjoints
    u = rng.standard_normal((4, 6, 8, 2))
    v = rng.standard_normal((2, 3, 4, 2))
    assert np.isclose((R.up(v) * u).sum(), (v * R.sumpool(u)).sum())
    assert np.isclose((R.pool(u) * v).sum(), (u * R.up(v) / 8).sum())


def test_backward_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = unet.init_params(3).astype(np.float64)
    # small nonzero biases so that the bias paths are exercised
    layout, n = unet.param_layout()
    for name, shape, off in layout:
        if name.endswith(".b"):
            p[off:off + int(np.prod(shape))] = 0.1 * rng.standard_normal(int(np.prod(shape)))
    x = rng.standard_normal((8, 8, 8))
    dy = rng.standard_normal((8, 8, 8))
    P = R.unpack(p)
    y, a = R.forward(P, x)
    g = R.flat(R.backward(P, x, a, dy))
    eps = 1e-6
    for name, shape, off in layout:
        size = int(np.prod(shape))
        for q in rng.choice(size, size=min(3, size), replace=False):
            pp, pm = p.copy(), p.copy()
            pp[off + q] += eps
            pm[off + q] -= eps
            fd = ((R.forward(R.unpack(pp), x)[0] - R.forward(R.unpack(pm), x)[0]) * dy).sum() / (2 * eps)
            assert abs(fd - g[off + q]) <= 1e-5 * (1 + abs(fd)), (name, q, fd, g[off + q])


def test_bf16_rounding():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3])
    r = R.bf16(a)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7
    assert r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8


def test_checkpoint_roundtrip_and_checks(tmp_path):
    layout, n = unet.param_layout()
    rng = np.random.default_rng(2)
    p = rng.standard_normal(n).astype(np.float32)
    m = rng.standard_normal(n).astype(np.float32)
    v = rng.random(n).astype(np.float32)
    f = tmp_path / "w.bunet"
    unet.save_state(str(f), p, m, v, step=17, meta={"target_scale": 0.5, "training_grid": 64})
    p2, m2, v2, step, meta = unet.load_state(str(f))
    assert np.array_equal(p, p2) and np.array_equal(m, m2) and np.array_equal(v, v2)
    assert step == 17 and meta == {"target_scale": 0.5, "training_grid": 64}
    # parameters only
    unet.save_state(str(f), p)
    p3, m3, v3, _, _ = unet.load_state(str(f))
    assert np.array_equal(p, p3) and m3 is None and v3 is None
    # wrong magic, truncated file, wrong length
    bad = tmp_path / "bad"
    bad.write_bytes(b"NOTACKPT" + bytes(16))
    with pytest.raises(unet.UNetError):
        unet.load_state(str(bad))
    raw = f.read_bytes()
    (tmp_path / "cut").write_bytes(raw[:-8])
    with pytest.raises(unet.UNetError):
        unet.load_state(str(tmp_path / "cut"))
    with pytest.raises(unet.UNetError):
        unet.save_state(str(f), p[:-1])
