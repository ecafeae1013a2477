"""3-D U-Net that gives the multigrid solve a learned initial guess.

Every layer runs on the kernels of ``libbunet.so`` (include/bunet.h):
tensor-core (tcgen05) implicit-GEMM 3x3x3 convolutions for the forward
pass, the data gradients and the weight gradients, CUDA-core kernels for the
one-channel input and output layers, pooling, the loss and Adam.  PyTorch
only allocates the device buffers and provides the stream.

Architecture (4 levels, 16-32-64-64 channels, BF16 activations, FP32
accumulation and master weights):

    a0 = relu(conv(x) + b)      1 -> 16        (CUDA cores)
    s0 = relu(conv(a0))         16 -> 16
    a1, s1 on pool(s0)          16 -> 32 -> 32
    a2, s2 on pool(s1)          32 -> 64 -> 64
    a3, b3 on pool(s2)          64 -> 64 -> 64
    d2 = two convs on [up(b3), s2]   128 -> 64 -> 64
    d1 = two convs on [up(d2), s1]    96 -> 32 -> 32
    d0 = two convs on [up(d1), s0]    48 -> 16 -> 16
    y  = w . d0 + b             16 -> 1        (CUDA cores)

The network maps the normalised source f / rms(f) of a Poisson problem to the
normalised solution x / rms(f); the solution is linear in f, so the guess for
any right-hand side is rms(f) * y.
"""
from __future__ import annotations

import ctypes
import math
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libbunet.so")

CH = (16, 32, 64, 64)

# (name, level, c0, up0, c1, cout): input channels [0, c0) from the first
# source (upsampled from level+1 when up0), then c1 channels of the skip
CONVS = (
    ("e0b", 0, 16, 0, 0, 16),
    ("e1a", 1, 16, 0, 0, 32), ("e1b", 1, 32, 0, 0, 32),
    ("e2a", 2, 32, 0, 0, 64), ("e2b", 2, 64, 0, 0, 64),
    ("e3a", 3, 64, 0, 0, 64), ("e3b", 3, 64, 0, 0, 64),
    ("d2a", 2, 64, 1, 64, 64), ("d2b", 2, 64, 0, 0, 64),
    ("d1a", 1, 64, 1, 32, 32), ("d1b", 1, 32, 0, 0, 32),
    ("d0a", 0, 32, 1, 16, 16), ("d0b", 0, 16, 0, 0, 16),
)


class UNetError(RuntimeError):
    pass


_lib = None


def load(path: str = LIB_PATH):
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise UNetError(f"{path} missing: build it with briscola_b200.build.build_unet()")
    L = ctypes.CDLL(path)
    vp, i, l, f, d = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_float, ctypes.c_double
    sig = {
        "bun_conv3": [i, i, i, vp, i, i, vp, i, vp, i, i, vp, i, vp, vp, vp, vp],
        "bun_conv3_wgrad": [i, i, i, vp, i, i, vp, i, vp, i, i, vp, vp, vp, vp],
        "bun_pack_weights": [vp, i, i, i, i, vp, vp],
        "bun_conv_in": [i, i, i, vp, vp, vp, vp, vp],
        "bun_conv_in_wgrad": [i, i, i, vp, vp, i, vp, vp, vp],
        "bun_head": [l, vp, vp, vp, vp, vp],
        "bun_head_grad": [l, vp, vp, vp, vp, i, vp, vp, vp],
        "bun_pool": [i, i, i, i, vp, vp, vp],
        "bun_unpool_grad": [i, i, i, i, i, vp, vp, vp, vp],
        "bun_skip_grad": [i, i, i, i, i, i, vp, vp, vp, vp, vp],
        "bun_mse": [l, vp, vp, vp, i, vp, vp, vp],
        "bun_adam": [l, vp, vp, vp, vp, f, f, f, f, i, vp],
        "bun_scale_to_float": [l, vp, d, vp, vp],
        "bun_scale_to_double": [l, vp, d, vp, vp],
        "bun_sumsq": [l, vp, i, vp, vp, vp],
        "bun_rms_normalise": [l, vp, f, i, vp, vp, vp, vp],
        "bun_rms_restore": [l, vp, d, vp, vp, vp],
        "bun_laplace_residual": [i, i, i, vp, vp, f, vp, vp],
        "bun_laplace_add": [i, i, i, vp, f, vp, vp],
        "bun_conv3_stage_width": [i, i, i, i],
    }
    for name, args in sig.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = i
    L.bun_wgrad_part_floats.argtypes = [i, i, i]
    L.bun_wgrad_part_floats.restype = ctypes.c_size_t
    _lib = L
    return L


EXPORTED = ("bun_conv3", "bun_conv3_wgrad", "bun_wgrad_part_floats", "bun_pack_weights", "bun_conv_in",
            "bun_conv_in_wgrad", "bun_head", "bun_head_grad", "bun_pool", "bun_unpool_grad", "bun_skip_grad",
            "bun_mse", "bun_adam", "bun_scale_to_float", "bun_scale_to_double", "bun_sumsq",
            "bun_rms_normalise", "bun_rms_restore",
            "bun_laplace_residual", "bun_laplace_add", "bun_conv3_stage_width")


def _check(rc, what):
    if rc != 0:
        raise UNetError(f"{what} failed with status {rc}")


def param_layout():
    """(name, shape, offset) of every parameter in the flat FP32 vector"""
    out, off = [], 0

    def add(name, shape):
        nonlocal off
        out.append((name, shape, off))
        off += int(np.prod(shape))

    add("in.w", (27, 16))
    add("in.b", (16,))
    for name, lev, c0, up0, c1, cout in CONVS:
        add(name + ".w", (27, c0 + c1, cout))
    add("head.w", (16,))
    add("head.b", (1,))
    return out, off


def forward_flops(shape) -> float:
    """algorithmic FLOPs of one forward pass: 2 * 27 * cin * cout per voxel
    and 3x3x3 convolution, 2 * 16 per voxel for the head"""
    nvox = [int(np.prod([s >> l for s in shape])) for l in range(4)]
    f = 2.0 * 27 * 1 * 16 * nvox[0] + 2.0 * 16 * nvox[0]
    for name, lev, c0, up0, c1, cout in CONVS:
        f += 2.0 * 27 * (c0 + c1) * cout * nvox[lev]
    return f


def init_params(seed: int = 0) -> np.ndarray:
    """He-normal weights, zero biases (FP32)."""
    layout, n = param_layout()
    rng = np.random.default_rng(seed)
    p = np.zeros(n, dtype=np.float32)
    for name, shape, off in layout:
        size = int(np.prod(shape))
        if name.endswith(".b"):
            continue
        fan_in = 27 * shape[1] if len(shape) == 3 else (27 if name == "in.w" else shape[0])
        p[off:off + size] = (rng.standard_normal(size) * math.sqrt(2.0 / fan_in)).astype(np.float32)
    return p


# ---------------------------------------------------------------------------
# checkpoint file: magic, version, JSON header, then FP32 arrays
# ---------------------------------------------------------------------------
MAGIC = b"BUNETCK1"
VERSION = 1


def save_state(path: str, params, m=None, v=None, step: int = 0, meta: dict | None = None) -> None:
    """Write parameters (and Adam moments) as a versioned binary file:
    8-byte magic, uint32 header length, UTF-8 JSON header (version, layout,
    step, caller metadata such as the target scale), then the FP32 arrays
    params, m, v back to back."""
    import json

    layout, n = param_layout()
    arrays = [np.asarray(a, dtype=np.float32).ravel() for a in (params, m, v) if a is not None]
    if any(a.size != n for a in arrays):
        raise UNetError("parameter arrays of the wrong length")
    header = {"version": VERSION, "nparam": n, "layout": [[nm, list(sh), off] for nm, sh, off in layout],
              "step": int(step), "has_moments": m is not None and v is not None, "meta": meta or {}}
    blob = json.dumps(header).encode()
    with open(path, "wb") as f:
        f.write(MAGIC)
        f.write(np.uint32(len(blob)).tobytes())
        f.write(blob)
        for a in arrays:
            f.write(a.tobytes())


def load_state(path: str):
    """(params, m, v, step, meta) from save_state's file; m and v are None
    when the file holds no moments.  Rejects other files and layouts."""
    import json

    with open(path, "rb") as f:
        if f.read(8) != MAGIC:
            raise UNetError(f"{path}: not a U-Net checkpoint")
        hlen = int(np.frombuffer(f.read(4), dtype=np.uint32)[0])
        header = json.loads(f.read(hlen).decode())
        if header.get("version") != VERSION:
            raise UNetError(f"{path}: checkpoint version {header.get('version')} (expected {VERSION})")
        layout, n = param_layout()
        if header["nparam"] != n or header["layout"] != [[nm, list(sh), off] for nm, sh, off in layout]:
            raise UNetError(f"{path}: parameter layout differs from this network")
        data = np.frombuffer(f.read(), dtype=np.float32)
    count = 3 if header["has_moments"] else 1
    if data.size != count * n:
        raise UNetError(f"{path}: truncated checkpoint")
    p = data[:n].copy()
    m = data[n:2 * n].copy() if count == 3 else None
    v = data[2 * n:].copy() if count == 3 else None
    return p, m, v, header["step"], header["meta"]


class UNet:
    """The network on one grid shape (each extent divisible by 8), its
    activations, gradients and optimiser state on the current CUDA device."""

    def __init__(self, shape, params: np.ndarray | None = None, seed: int = 0):
        import torch

        self.torch = torch
        self.L = load()
        self.shape = tuple(int(s) for s in shape)
        if any(s % 8 or s < 8 for s in self.shape):
            raise UNetError("every grid extent must be a multiple of 8")
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        self.layout, self.nparam = param_layout()
        p = init_params(seed) if params is None else np.asarray(params, dtype=np.float32)
        if p.size != self.nparam:
            raise UNetError("parameter vector of the wrong length")
        self.p = torch.from_numpy(p.copy()).to(dev)
        self.g = torch.zeros_like(self.p)
        self.m = torch.zeros_like(self.p)
        self.v = torch.zeros_like(self.p)
        self.step = 0
        self.views = {name: (off, shape) for name, shape, off in self.layout}
        self.dims = [tuple(s >> l for s in self.shape) for l in range(4)]
        self.nvox = [int(np.prod(d)) for d in self.dims]
        bf = torch.bfloat16
        z = lambda l, c: torch.zeros(self.nvox[l] * c, dtype=bf, device=dev)  # noqa: E731
        # activations
        self.a = {"a0": z(0, 16), "s0": z(0, 16), "p0": z(1, 16), "a1": z(1, 32), "s1": z(1, 32), "p1": z(2, 32),
                  "a2": z(2, 64), "s2": z(2, 64), "p2": z(3, 64), "a3": z(3, 64), "b3": z(3, 64),
                  "d2a": z(2, 64), "d2": z(2, 64), "d1a": z(1, 32), "d1": z(1, 32), "d0a": z(0, 16),
                  "d0": z(0, 16)}
        # gradients (pre-activation unless noted)
        self.d = {"d0": z(0, 16), "d0a": z(0, 16), "cat0": z(0, 48), "d1": z(1, 32), "d1a": z(1, 32),
                  "cat1": z(1, 96), "d2": z(2, 64), "d2a": z(2, 64), "cat2": z(2, 128), "b3": z(3, 64),
                  "a3": z(3, 64), "p2": z(3, 64), "s2": z(2, 64), "a2": z(2, 64), "p1": z(2, 32),
                  "s1": z(1, 32), "a1": z(1, 32), "p0": z(1, 16), "s0": z(0, 16), "a0": z(0, 16)}
        f32 = torch.float32
        self.x = torch.zeros(self.nvox[0], dtype=f32, device=dev)
        self.y = torch.zeros(self.nvox[0], dtype=f32, device=dev)
        self.dy = torch.zeros(self.nvox[0], dtype=f32, device=dev)
        self.loss = torch.zeros(1, dtype=f32, device=dev)
        self.rloss = torch.zeros(1, dtype=f32, device=dev)
        self.r = torch.zeros(self.nvox[0], dtype=f32, device=dev)
        self.dr = torch.zeros(self.nvox[0], dtype=f32, device=dev)
        self.zero = torch.zeros(self.nvox[0], dtype=f32, device=dev)
        self.err = torch.zeros(1, dtype=torch.int32, device=dev)
        # packed BF16 weights: forward and data-gradient layouts, for the
        # stage width the library picks for each layer's grid
        self.wf, self.wd, self.kcf, self.kcd = {}, {}, {}, {}
        for name, lev, c0, up0, c1, cout in CONVS:
            n = 27 * (c0 + c1) * cout
            n2 = self.dims[lev][2]
            self.kcf[name] = self.L.bun_conv3_stage_width(c0, c1, cout, n2)
            self.kcd[name] = self.L.bun_conv3_stage_width(cout, 0, c0 + c1, n2)
            if not (self.kcf[name] and self.kcd[name]):
                raise UNetError(f"no convolution kernel for layer {name}")
            self.wf[name] = torch.zeros(n, dtype=bf, device=dev)
            self.wd[name] = torch.zeros(n, dtype=bf, device=dev)
        # scratch for the reductions
        self.nsplit = {}
        part = 0
        for name, lev, c0, up0, c1, cout in CONVS:
            nblk = -(-self.nvox[lev] // 128)
            ns = max(1, min(nblk, 512 // max(1, -(-(27 * (c0 + c1)) // 128))))
            self.nsplit[name] = ns
            part = max(part, self.L.bun_wgrad_part_floats(c0 + c1, cout, ns))
        self.red_blocks = 256
        part = max(part, self.red_blocks * 28 * 16, self.red_blocks * 17, self.red_blocks)
        self.part = torch.zeros(part, dtype=f32, device=dev)
        self.dpart = torch.zeros(self.red_blocks, dtype=torch.float64, device=dev)
        self.dsum = torch.zeros(1, dtype=torch.float64, device=dev)
        self.rms = torch.zeros(1, dtype=torch.float64, device=dev)  # input scale kept on the device
        self.stream = None  # a cudaStream_t (int) to queue on instead of torch's current stream
        self.pack()

    # -- helpers -------------------------------------------------------------
    def _s(self):
        if self.stream is not None:
            return ctypes.c_void_p(self.stream)
        return ctypes.c_void_p(self.torch.cuda.current_stream().cuda_stream)

    def _w(self, name, buf=None):
        off, shape = self.views[name]
        t = self.p if buf is None else buf
        return t[off:off + int(np.prod(shape))]

    def pack(self):
        """refresh the BF16 tile layouts from the FP32 master weights"""
        s = self._s()
        for name, lev, c0, up0, c1, cout in CONVS:
            w = self._w(name + ".w")
            _check(self.L.bun_pack_weights(w.data_ptr(), c0 + c1, cout, self.kcf[name], 0,
                                           self.wf[name].data_ptr(), s), "pack")
            _check(self.L.bun_pack_weights(w.data_ptr(), c0 + c1, cout, self.kcd[name], 1,
                                           self.wd[name].data_ptr(), s), "pack")

    def _inputs(self, name):
        a = self.a
        return {"e0b": (a["a0"], None), "e1a": (a["p0"], None), "e1b": (a["a1"], None), "e2a": (a["p1"], None),
                "e2b": (a["a2"], None), "e3a": (a["p2"], None), "e3b": (a["a3"], None),
                "d2a": (a["b3"], a["s2"]), "d2b": (a["d2a"], None), "d1a": (a["d2"], a["s1"]),
                "d1b": (a["d1a"], None), "d0a": (a["d1"], a["s0"]), "d0b": (a["d0a"], None)}[name]

    _OUT = {"e0b": "s0", "e1a": "a1", "e1b": "s1", "e2a": "a2", "e2b": "s2", "e3a": "a3", "e3b": "b3",
            "d2a": "d2a", "d2b": "d2", "d1a": "d1a", "d1b": "d1", "d0a": "d0a", "d0b": "d0"}

    def _conv(self, spec, src0, src1, wpack, kc, cout, relu, mask, out, dims):
        name, lev, c0, up0, c1, _ = spec
        s = self._s()
        n0, n1, n2 = dims
        _check(self.L.bun_conv3(n0, n1, n2, src0.data_ptr(), c0, up0, src1.data_ptr() if src1 is not None else None,
                                c1, wpack.data_ptr(), kc, cout, None, relu,
                                mask.data_ptr() if mask is not None else None, out.data_ptr(),
                                self.err.data_ptr(), s), f"conv {name}")

    # -- forward -------------------------------------------------------------
    def forward(self, x=None):
        """y = net(x); x: FP32 device tensor of the grid's cells (or the
        internal input buffer when None).  Returns the FP32 output buffer."""
        L, s = self.L, self._s()
        if x is not None:
            self.x.copy_(x.reshape(-1))
        n0, n1, n2 = self.dims[0]
        _check(L.bun_conv_in(n0, n1, n2, self.x.data_ptr(), self._w("in.w").data_ptr(), self._w("in.b").data_ptr(),
                             self.a["a0"].data_ptr(), s), "conv_in")
        for spec in CONVS:
            name, lev, c0, up0, c1, cout = spec
            if name in ("e1a", "e2a", "e3a"):
                src, dst, c = {"e1a": ("s0", "p0", 16), "e2a": ("s1", "p1", 32), "e3a": ("s2", "p2", 64)}[name]
                m0, m1, m2 = self.dims[lev - 1]
                _check(L.bun_pool(m0, m1, m2, c, self.a[src].data_ptr(), self.a[dst].data_ptr(), s), "pool")
            src0, src1 = self._inputs(name)
            self._conv(spec, src0, src1, self.wf[name], self.kcf[name], cout, 1, None, self.a[self._OUT[name]],
                       self.dims[lev])
        _check(L.bun_head(self.nvox[0], self.a["d0"].data_ptr(), self._w("head.w").data_ptr(),
                          self._w("head.b").data_ptr(), self.y.data_ptr(), s), "head")
        return self.y

    # -- backward ------------------------------------------------------------
    def _wgrad(self, spec, dz):
        name, lev, c0, up0, c1, cout = spec
        src0, src1 = self._inputs(name)
        n0, n1, n2 = self.dims[lev]
        g = self._w(name + ".w", self.g)
        _check(self.L.bun_conv3_wgrad(n0, n1, n2, src0.data_ptr(), c0, up0,
                                      src1.data_ptr() if src1 is not None else None, c1, dz.data_ptr(), cout,
                                      self.nsplit[name], self.part.data_ptr(), g.data_ptr(), self.err.data_ptr(),
                                      self._s()), f"wgrad {name}")

    def _dgrad(self, spec, dz, out, mask):
        name, lev, c0, up0, c1, cout = spec
        n0, n1, n2 = self.dims[lev]
        _check(self.L.bun_conv3(n0, n1, n2, dz.data_ptr(), cout, 0, None, 0, self.wd[name].data_ptr(),
                                self.kcd[name], c0 + c1, None, 0, mask.data_ptr() if mask is not None else None,
                                out.data_ptr(), self.err.data_ptr(), self._s()), f"dgrad {name}")

    def backward(self):
        """gradients of the loss whose dL/dy is in self.dy, into self.g"""
        L, s, a, d = self.L, self._s(), self.a, self.d
        spec = {c[0]: c for c in CONVS}
        _check(L.bun_head_grad(self.nvox[0], a["d0"].data_ptr(), self.dy.data_ptr(), self._w("head.w").data_ptr(),
                               d["d0"].data_ptr(), self.red_blocks, self.part.data_ptr(),
                               self._w("head.w", self.g).data_ptr(), s), "head_grad")

        def conv_back(name, dz, dst, mask):
            self._wgrad(spec[name], dz)
            self._dgrad(spec[name], dz, dst, mask)

        def up_back(lev, ccat, c0, dcat, act, dst):
            n0, n1, n2 = self.dims[lev]
            _check(L.bun_unpool_grad(n0, n1, n2, ccat, c0, dcat.data_ptr(), act.data_ptr(), dst.data_ptr(), s),
                   "unpool_grad")

        def skip_back(lev, ccat, c0, c, dcat, dp, src, dst):
            n0, n1, n2 = self.dims[lev]
            _check(L.bun_skip_grad(n0, n1, n2, ccat, c0, c, dcat.data_ptr(), dp.data_ptr(), src.data_ptr(),
                                   dst.data_ptr(), s), "skip_grad")

        conv_back("d0b", d["d0"], d["d0a"], a["d0a"])
        conv_back("d0a", d["d0a"], d["cat0"], None)
        up_back(0, 48, 32, d["cat0"], a["d1"], d["d1"])
        conv_back("d1b", d["d1"], d["d1a"], a["d1a"])
        conv_back("d1a", d["d1a"], d["cat1"], None)
        up_back(1, 96, 64, d["cat1"], a["d2"], d["d2"])
        conv_back("d2b", d["d2"], d["d2a"], a["d2a"])
        conv_back("d2a", d["d2a"], d["cat2"], None)
        up_back(2, 128, 64, d["cat2"], a["b3"], d["b3"])
        conv_back("e3b", d["b3"], d["a3"], a["a3"])
        conv_back("e3a", d["a3"], d["p2"], None)
        skip_back(2, 128, 64, 64, d["cat2"], d["p2"], a["s2"], d["s2"])
        conv_back("e2b", d["s2"], d["a2"], a["a2"])
        conv_back("e2a", d["a2"], d["p1"], None)
        skip_back(1, 96, 64, 32, d["cat1"], d["p1"], a["s1"], d["s1"])
        conv_back("e1b", d["s1"], d["a1"], a["a1"])
        conv_back("e1a", d["a1"], d["p0"], None)
        skip_back(0, 48, 32, 16, d["cat0"], d["p0"], a["s0"], d["s0"])
        conv_back("e0b", d["s0"], d["a0"], a["a0"])
        n0, n1, n2 = self.dims[0]
        _check(L.bun_conv_in_wgrad(n0, n1, n2, self.x.data_ptr(), d["a0"].data_ptr(), self.red_blocks,
                                   self.part.data_ptr(), self._w("in.w", self.g).data_ptr(), s), "conv_in_wgrad")

    def mse(self, target):
        """loss = mean (y - target)^2 into self.loss, dL/dy into self.dy"""
        _check(self.L.bun_mse(self.nvox[0], self.y.data_ptr(), target.data_ptr(), self.dy.data_ptr(),
                              self.red_blocks, self.part.data_ptr(), self.loss.data_ptr(), self._s()), "mse")
        return self.loss

    def residual_loss(self, c: float, weight: float):
        """add weight * mean(r^2), r = h^2 A'y + c x (the operator residual
        of the output for the current input), to the loss and to dL/dy"""
        n0, n1, n2 = self.dims[0]
        s = self._s()
        _check(self.L.bun_laplace_residual(n0, n1, n2, self.y.data_ptr(), self.x.data_ptr(), c, self.r.data_ptr(),
                                           s), "laplace_residual")
        _check(self.L.bun_mse(self.nvox[0], self.r.data_ptr(), self.zero.data_ptr(), self.dr.data_ptr(),
                              self.red_blocks, self.part.data_ptr(), self.rloss.data_ptr(), s), "mse")
        _check(self.L.bun_laplace_add(n0, n1, n2, self.dr.data_ptr(), weight, self.dy.data_ptr(), s),
               "laplace_add")
        return self.rloss

    def adam(self, lr=1e-3, b1=0.9, b2=0.999, eps=1e-8):
        self.step += 1
        _check(self.L.bun_adam(self.nparam, self.p.data_ptr(), self.g.data_ptr(), self.m.data_ptr(),
                               self.v.data_ptr(), lr, b1, b2, eps, self.step, self._s()), "adam")
        self.pack()

    def train_step(self, x, target, lr=1e-3, res_c: float = 0.0, res_weight: float = 0.0):
        """one Adam step on mean (y - target)^2 (+ res_weight * the operator
        residual term of residual_loss with c = res_c)"""
        self.forward(x)
        self.mse(target)
        if res_weight > 0:
            self.residual_loss(res_c, res_weight)
        self.backward()
        self.adam(lr)
        return self.loss

    def check_errors(self):
        if int(self.err.item()) != 0:
            raise UNetError("a U-Net kernel gave up waiting on a barrier")

    def params(self) -> np.ndarray:
        return self.p.detach().cpu().numpy().copy()

    def save(self, path: str, meta: dict | None = None) -> None:
        """parameters and Adam state to a checkpoint file"""
        save_state(path, self.params(), self.m.cpu().numpy(), self.v.cpu().numpy(), self.step, meta)

    @classmethod
    def from_file(cls, path: str, shape):
        """a network on grid `shape` from a checkpoint (any training grid:
        the layers are convolutions), with its optimiser state; returns
        (net, meta)"""
        p, m, v, step, meta = load_state(path)
        net = cls(shape, params=p)
        if m is not None:
            net.m.copy_(net.torch.from_numpy(m))
            net.v.copy_(net.torch.from_numpy(v))
        net.step = step
        return net, meta

    # -- the solver's view ---------------------------------------------------
    def solve_level(self, stream: int, rhs: int, x: int, scale: float) -> None:
        """The network as a level's solver (bmg_set_level_solver): rhs and x
        are device pointers to the level's FP32 interior cells, rhs the
        row-scaled right-hand side b/V = -f.  The input is f / rms(f) and
        x = scale * rms(f) * output, with rms(f) kept on the device, so every
        kernel is queued on `stream` and nothing returns to the host (the
        calls may be captured into the solver's graph)."""
        L = self.L
        n = self.nvox[0]
        self.stream = stream
        try:
            _check(L.bun_rms_normalise(n, ctypes.c_void_p(rhs), -1.0, self.red_blocks, self.dpart.data_ptr(),
                                       self.rms.data_ptr(), self.x.data_ptr(), self._s()), "rms_normalise")
            self.forward()
            _check(L.bun_rms_restore(n, self.y.data_ptr(), scale, self.rms.data_ptr(), ctypes.c_void_p(x),
                                     self._s()), "rms_restore")
        finally:
            self.stream = None

    def guess(self, b, V: float, x0, scale: float = 1.0):
        """Initial guess x0 (FP64 device) for the system right-hand side b
        (FP64 device, b = -V f on a uniform grid of cell volume V); scale:
        the factor the training targets were divided by."""
        L, s = self.L, self._s()
        n = self.nvox[0]
        _check(L.bun_sumsq(n, b.data_ptr(), self.red_blocks, self.dpart.data_ptr(), self.dsum.data_ptr(), s), "sumsq")
        rms_b = math.sqrt(float(self.dsum.item()) / n)
        if rms_b == 0.0:
            x0.zero_()
            return x0
        # f = -b / V; input f / rms(f) = -b / rms(b)
        _check(L.bun_scale_to_float(n, b.data_ptr(), -1.0 / rms_b, self.x.data_ptr(), s), "scale")
        self.forward()
        _check(L.bun_scale_to_double(n, self.y.data_ptr(), scale * rms_b / V, x0.data_ptr(), s), "scale")
        return x0
