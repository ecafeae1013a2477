"""The allocation-free residual norm (bmg_residual_norm_noalloc) against the
residual of the regular context-based entry point (bmg_op_residual).

It serves callers that must not call cudaMalloc when they need a residual:
their device memory belongs to their own pool, or an allocation's implicit
synchronisation would stall them, or they are reporting on a solve that
already ran out of memory.  This file is collected last so a failure here
stops a -x run only after every other test has run; it also passes on its
own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import _native as NA
from briscola_b200 import workloads

pytestmark = pytest.mark.gpu


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _dirichlet_mesh(N):
    from briscola_b200.mesh import Brick, Mesh, geometric_points, uniform_points

    br = Brick([uniform_points(N), uniform_points(N), geometric_points(N, 2.0)],
               ("Dirichlet", "Neumann", "periodic", "periodic", "Dirichlet", "Dirichlet"))
    return Mesh([br]), np.random.default_rng(5).standard_normal(N ** 3), None


_BC = {"periodic": NA.BC_PERIODIC, "Neumann": NA.BC_NEUMANN, "Dirichlet": NA.BC_DIRICHLET}


def _long_box():
    # 2304 rows (more than one pass of the row grid) and rows of 384 cells
    # (more than one pass of the 256 threads along k); walls all round, so
    # that the reference context coarsens it (odd periodic extents would not)
    from briscola_b200.mesh import Brick, Mesh, tanh_points, uniform_points

    br = Brick([uniform_points(48), tanh_points(48, 2.0), uniform_points(384)])
    return Mesh([br]), np.random.default_rng(6).standard_normal(48 * 48 * 384), None


@pytest.mark.parametrize("name,N", [("channel", 32), ("cavity", 24), ("dirichlet", 16), ("long_box", 0)])
def test_noalloc_norm_matches_context_residual(native, name, N):
    import torch

    if name == "dirichlet":
        mesh, b, _ = _dirichlet_mesh(N)
    elif name == "long_box":
        mesh, b, _ = _long_box()
    else:
        mesh, b, _ = workloads.CONFIGS[name](N)
    br = mesh.bricks[0]
    rng = np.random.default_rng(17)
    x = rng.standard_normal(b.size)
    # existing entry point: residual field of level 0 through a context
    ctx = bb.Context(mesh, bb.make_options({}))
    ctx.upload(0, "x", x.reshape(br.N))
    ctx.upload(0, "b", b.reshape(br.N))
    ref = float(np.linalg.norm(ctx.residual(0)))
    ctx.close()

    dev = torch.device("cuda", 0)
    xd = torch.from_numpy(x).to(dev)
    bd = torch.from_numpy(b).to(dev)
    pts = [torch.from_numpy(np.ascontiguousarray(p)).to(dev) for p in br.points]
    out = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    n = (ctypes.c_int * 3)(*br.N)
    bc = (ctypes.c_int * 6)(*[_BC[f] for f in br.bc])
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    for call in range(2):  # the static scratch is reused by the second call
        out.fill_(-1.0)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        rc = native.bmg_residual_norm_noalloc(_ptr(xd), _ptr(bd), n, *[_ptr(p) for p in pts], bc, _ptr(out),
                                              stream)
        torch.cuda.synchronize()
        assert rc == NA.OK, (call, rc)
        if call == 1:  # the first call may load the module; the second allocates nothing
            assert torch.cuda.mem_get_info(dev)[0] == free0
        got = float(out.item())
        assert abs(got - ref) <= 1e-12 * ref, (call, got, ref)
    if name == "channel":
        # independent check: the residual of the CPU oracle
        from oracle.pyoracle import Oracle

        o = Oracle(br.points, periodic=br.periodic, nthreads=2)
        o.assemble(n_pre=2, n_post=2, cycle_type="V", coarse_level=1)
        ro = float(np.linalg.norm(o.residual(0, x.reshape(br.N), b.reshape(br.N))))
        assert abs(float(out.item()) - ro) <= 1e-12 * ro


def test_noalloc_rejects_sizes_beyond_scratch(native):
    import torch

    dev = torch.device("cuda", 0)
    dummy = torch.zeros(8, dtype=torch.float64, device=dev)
    n = (ctypes.c_int * 3)(300, 300, 2)  # 90000 rows > BMG_NOALLOC_MAX_ROWS
    bc = (ctypes.c_int * 6)(*([NA.BC_NEUMANN] * 6))
    rc = native.bmg_residual_norm_noalloc(_ptr(dummy), _ptr(dummy), n, _ptr(dummy), _ptr(dummy), _ptr(dummy),
                                          bc, _ptr(dummy), None)
    assert rc == NA.BAD_ARG
