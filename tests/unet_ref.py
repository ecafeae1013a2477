"""FP64 numpy restatement of the U-Net in briscola_b200/unet.py, with a
hand-written backward pass: the reference the GPU kernels are checked
against (test infrastructure only)."""
from __future__ import annotations

import numpy as np

from briscola_b200.unet import CONVS, param_layout

TAPS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]


def shift(x, d):
    """y[v] = x[v + d] with zeros outside; x: (n0, n1, n2, C)"""
    n0, n1, n2 = x.shape[:3]
    xp = np.pad(x, ((1, 1), (1, 1), (1, 1), (0, 0)))
    return xp[1 + d[0]:1 + d[0] + n0, 1 + d[1]:1 + d[1] + n1, 1 + d[2]:1 + d[2] + n2]


def conv3(x, W):
    """out[v][n] = sum_t sum_c x[v + off(t)][c] W[t][c][n]"""
    out = np.zeros(x.shape[:3] + (W.shape[2],))
    for t, d in enumerate(TAPS):
        out += shift(x, d) @ W[t]
    return out


def conv3_wgrad(x, dz):
    return np.stack([np.einsum("ijkc,ijkn->cn", shift(x, d), dz) for d in TAPS])


def conv3_dgrad(dz, W):
    out = np.zeros(dz.shape[:3] + (W.shape[1],))
    for t, d in enumerate(TAPS):
        out += shift(dz, (-d[0], -d[1], -d[2])) @ W[t].T
    return out


def pool(x):
    n0, n1, n2, c = x.shape
    return x.reshape(n0 // 2, 2, n1 // 2, 2, n2 // 2, 2, c).mean(axis=(1, 3, 5))


def up(x):
    return x.repeat(2, 0).repeat(2, 1).repeat(2, 2)


def sumpool(x):
    n0, n1, n2, c = x.shape
    return x.reshape(n0 // 2, 2, n1 // 2, 2, n2 // 2, 2, c).sum(axis=(1, 3, 5))


relu = lambda z: np.maximum(z, 0.0)  # noqa: E731


def unpack(p):
    layout, _ = param_layout()
    return {name: np.asarray(p[off:off + int(np.prod(shape))], dtype=np.float64).reshape(shape)
            for name, shape, off in layout}


def forward(P, x):
    """x: (n0, n1, n2) -> (y, activations)"""
    a = {}
    a["a0"] = relu(conv3(x[..., None], P["in.w"][:, None, :]) + P["in.b"])
    W = {c[0]: P[c[0] + ".w"] for c in CONVS}
    a["s0"] = relu(conv3(a["a0"], W["e0b"]))
    a["p0"] = pool(a["s0"])
    a["a1"] = relu(conv3(a["p0"], W["e1a"]))
    a["s1"] = relu(conv3(a["a1"], W["e1b"]))
    a["p1"] = pool(a["s1"])
    a["a2"] = relu(conv3(a["p1"], W["e2a"]))
    a["s2"] = relu(conv3(a["a2"], W["e2b"]))
    a["p2"] = pool(a["s2"])
    a["a3"] = relu(conv3(a["p2"], W["e3a"]))
    a["b3"] = relu(conv3(a["a3"], W["e3b"]))
    a["c2"] = np.concatenate([up(a["b3"]), a["s2"]], axis=3)
    a["d2a"] = relu(conv3(a["c2"], W["d2a"]))
    a["d2"] = relu(conv3(a["d2a"], W["d2b"]))
    a["c1"] = np.concatenate([up(a["d2"]), a["s1"]], axis=3)
    a["d1a"] = relu(conv3(a["c1"], W["d1a"]))
    a["d1"] = relu(conv3(a["d1a"], W["d1b"]))
    a["c0"] = np.concatenate([up(a["d1"]), a["s0"]], axis=3)
    a["d0a"] = relu(conv3(a["c0"], W["d0a"]))
    a["d0"] = relu(conv3(a["d0a"], W["d0b"]))
    y = a["d0"] @ P["head.w"] + P["head.b"][0]
    return y, a


def backward(P, x, a, dy):
    """gradients of sum(dy * y) w.r.t. every parameter"""
    W = {c[0]: P[c[0] + ".w"] for c in CONVS}
    G = {}
    m = lambda t: (t > 0).astype(np.float64)  # noqa: E731
    G["head.w"] = np.einsum("ijkc,ijk->c", a["d0"], dy)
    G["head.b"] = np.array([dy.sum()])
    g = dy[..., None] * P["head.w"] * m(a["d0"])

    def cb(name, inp, dz):
        G[name + ".w"] = conv3_wgrad(inp, dz)
        return conv3_dgrad(dz, W[name])

    g = cb("d0b", a["d0a"], g) * m(a["d0a"])
    gc0 = cb("d0a", a["c0"], g)
    g = sumpool(gc0[..., :32]) * m(a["d1"])
    g = cb("d1b", a["d1a"], g) * m(a["d1a"])
    gc1 = cb("d1a", a["c1"], g)
    g = sumpool(gc1[..., :64]) * m(a["d2"])
    g = cb("d2b", a["d2a"], g) * m(a["d2a"])
    gc2 = cb("d2a", a["c2"], g)
    g = sumpool(gc2[..., :64]) * m(a["b3"])
    g = cb("e3b", a["a3"], g) * m(a["a3"])
    gp = cb("e3a", a["p2"], g)
    g = (gc2[..., 64:] + up(gp) / 8) * m(a["s2"])
    g = cb("e2b", a["a2"], g) * m(a["a2"])
    gp = cb("e2a", a["p1"], g)
    g = (gc1[..., 64:] + up(gp) / 8) * m(a["s1"])
    g = cb("e1b", a["a1"], g) * m(a["a1"])
    gp = cb("e1a", a["p0"], g)
    g = (gc0[..., 32:] + up(gp) / 8) * m(a["s0"])
    g = cb("e0b", a["a0"], g) * m(a["a0"])
    G["in.w"] = conv3_wgrad(x[..., None], g)[:, 0, :]
    G["in.b"] = g.sum(axis=(0, 1, 2))
    return G


def flat(G):
    layout, n = param_layout()
    out = np.zeros(n)
    for name, shape, off in layout:
        out[off:off + int(np.prod(shape))] = G[name].ravel()
    return out


def bf16(a):
    """round to bfloat16 (nearest even), returned as float64"""
    a32 = np.ascontiguousarray(a, dtype=np.float32)
    u = a32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)
