"""Reference-shaped host interface of the B200 multigrid solver.

Mirrors Briscola's linear-solver plugin API for the multigrid path:

* ``solver.New(dict, mesh)`` looks the ``type`` keyword up in a runtime
  table and fails with the list of valid types on a miss
  (src/briscolaFiniteVolume/solvers/solver/solver.C:130-182);
* ``GPUMG`` registers itself under ``"GPUMG"`` the way ``MG`` does
  (src/briscolaFiniteVolume/solvers/MG/MGSolvers.C:13-21) and reads the same
  dictionary keys with the same defaults (MG.C:257-305, solver.C:115-123);
* ``solve(sys, constMatrix)`` updates ``sys.x`` in place
  (src/briscolaFiniteVolume/solvers/solver/solver.H:280-284) and prints the
  reference's statistics line (solver.C:97-112).

Every solve goes through the C ABI of ``libbmg.so``; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import re

import numpy as np

from . import _native as N
from .mesh import Mesh


class FatalError(RuntimeError):
    """Raised where the reference calls FatalErrorInFunction ... abort."""


# ---------------------------------------------------------------------------
# A small subset of the OpenFOAM dictionary syntax: ``key value;``,
# ``key { ... }`` and // or /* */ comments.
# ---------------------------------------------------------------------------
class Dictionary(dict):
    def lookup(self, key):
        if key not in self:
            raise FatalError(f"keyword {key} is undefined in dictionary")
        return self[key]

    def lookupOrDefault(self, key, default):
        return self.get(key, default)

    def subDict(self, key) -> "Dictionary":
        v = self.lookup(key)
        if not isinstance(v, Dictionary):
            raise FatalError(f"keyword {key} is not a sub-dictionary")
        return v

    def found(self, key) -> bool:
        return key in self

    @classmethod
    def parse(cls, text: str) -> "Dictionary":
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        toks = re.findall(r"[{};]|[^\s{};]+", text)
        pos = 0

        def block() -> Dictionary:
            nonlocal pos
            d = cls()
            while pos < len(toks):
                t = toks[pos]
                if t == "}":
                    pos += 1
                    return d
                if t == ";":
                    pos += 1
                    continue
                key = t
                pos += 1
                if pos < len(toks) and toks[pos] == "{":
                    pos += 1
                    d[key] = block()
                    continue
                vals = []
                while pos < len(toks) and toks[pos] != ";":
                    if toks[pos] in "{}":
                        raise FatalError(f"malformed entry {key}")
                    vals.append(toks[pos])
                    pos += 1
                pos += 1
                d[key] = vals[0] if len(vals) == 1 else " ".join(vals)
            return d

        return block()


def _scalar(v) -> float:
    return float(v)


def _label(v) -> int:
    return int(v)


def _switch(v) -> bool:
    if isinstance(v, bool):
        return v
    s = str(v).lower()
    if s in ("on", "yes", "true", "1"):
        return True
    if s in ("off", "no", "false", "0"):
        return False
    raise FatalError(f"bad switch value {v}")


class LinearSystem:
    """The reference's ``linearSystem`` for the Poisson path: unknown x
    (updated in place), system right-hand side b and, for a variable
    coefficient, the face field lambda (three arrays of face values).

    The operator itself is the Laplacian of the mesh (linearGaussLaplacianScheme
    .C:59-94), rebuilt on every level the way the reference rediscretises it.
    x and b are float64 arrays of the mesh's cell count (numpy on the host, or
    torch CUDA tensors for device-resident solves)."""

    def __init__(self, mesh: Mesh, x, b, lam=None, zero_guess: bool = False):
        self.mesh = mesh
        self.x = x
        self.b = b
        self.lam = lam
        # start from x = 0 instead of the incoming x (no host->device copy of x)
        self.zero_guess = zero_guess

    @classmethod
    def poisson(cls, mesh: Mesh, x, source: np.ndarray, lam=None) -> "LinearSystem":
        """``sys = im::laplacian(lambda, x) + source`` (defaultPoissonSolver.C:86-89):
        the system right-hand side is b = -V * source (linearSystem.C:547-556)."""
        if len(mesh.bricks) != 1:
            raise FatalError("poisson() assembles single-brick systems")
        V = mesh.bricks[0].cell_volumes()
        return cls(mesh, x, -V * np.asarray(source, dtype=np.float64).reshape(V.shape), lam)


class solver:
    """Runtime-selection base (solver.H:240-251)."""

    _table: dict = {}
    typeName = "solver"

    def __init_subclass__(cls, **kw):
        super().__init_subclass__(**kw)
        if cls.typeName != "solver":
            solver._table[cls.typeName] = cls

    def __init__(self, dict_: Dictionary, mesh: Mesh):
        self.dict_ = dict_
        self.mesh = mesh
        self.relTol = _scalar(dict_.lookup("relTol"))
        self.tolerance = _scalar(dict_.lookup("tolerance"))
        self.minIter = _label(dict_.lookupOrDefault("minIter", 0))
        self.maxIter = _label(dict_.lookupOrDefault("maxIter", 999))

    @classmethod
    def New(cls, dict_: Dictionary, mesh: Mesh) -> "solver":
        t = dict_.lookup("type")
        if t not in solver._table:
            raise FatalError(f"Unknown solver {t}\n\nValid solvers are:\n{sorted(solver._table)}")
        return solver._table[t](dict_, mesh)

    def solve(self, sys: LinearSystem, constMatrix: bool = False):
        raise NotImplementedError


_BC = {"Neumann": N.BC_NEUMANN, "periodic": N.BC_PERIODIC, "Dirichlet": N.BC_DIRICHLET}


def _mesh_desc(mesh: Mesh):
    bricks = (N.Brick * len(mesh.bricks))()
    keep = []
    for q, br in enumerate(mesh.bricks):
        for d in range(3):
            bricks[q].n[d] = br.N[d]
            p = np.ascontiguousarray(br.points[d], dtype=np.float64)
            keep.append(p)
            bricks[q].points[d] = p.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            bricks[q].origin[d] = int(br.origin[d])
        for f in range(6):
            if br.bc[f] not in _BC:
                raise FatalError(f"Incompatible boundary condition {br.bc[f]} for the GPU multigrid")
            bricks[q].bc[f] = _BC[br.bc[f]]
            bricks[q].value[f] = float(br.values[f])
        for d in range(3):
            bricks[q].transform[d] = int(br.transform[d])
    desc = N.MeshDesc(len(mesh.bricks), bricks)
    return desc, (bricks, keep)


class Context:
    """Owner of one native solver context (``bmg_ctx``)."""

    def __init__(self, mesh: Mesh, opts: N.Options):
        L = N.load()
        self._lib = L
        desc, self._keep = _mesh_desc(mesh)
        h = ctypes.c_void_p()
        rc = L.bmg_create(ctypes.byref(h), ctypes.byref(desc), ctypes.byref(opts))
        if rc != N.OK:
            raise FatalError(f"bmg_create failed: {N.status_string(rc)}")
        self.h = h
        self.opts = opts
        self.n_cells = L.bmg_num_cells(h)
        self.n_bricks = len(mesh.bricks)

    def close(self):
        if getattr(self, "h", None):
            self._lib.bmg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def check(self, rc: int, what: str):
        if rc not in (N.OK, N.NOT_CONVERGED):
            msg = self._lib.bmg_last_error(self.h).decode() if self.h else ""
            raise FatalError(f"{what}: {N.status_string(rc)} {msg}".strip())
        return rc

    def set_options(self, opts: N.Options):
        self.check(self._lib.bmg_set_options(self.h, ctypes.byref(opts)), "bmg_set_options")
        self.opts = opts

    def set_coefficients(self, lam):
        if lam is None:
            rc = self._lib.bmg_set_coefficients(self.h, None, None, None)
        else:
            self._lam = [np.ascontiguousarray(a, dtype=np.float64) for a in lam]
            ptrs = [a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) for a in self._lam]
            rc = self._lib.bmg_set_coefficients(self.h, *ptrs)
        self.check(rc, "bmg_set_coefficients")

    def project_rhs(self, u, c_dt: float, out, per_volume: bool = False):
        """out <- the pressure right-hand side coloDiv(U) / (-c_dt) of a
        staggered projection step (system form -V times it unless
        per_volume); u: three CUDA face arrays, out: CUDA cells."""
        self._follow(out)
        flags = N.PER_VOLUME if per_volume else 0
        self.check(self._lib.bmg_project_rhs(self.h, *(a.data_ptr() for a in u), float(c_dt), out.data_ptr(), flags),
                   "bmg_project_rhs")
        return out

    def project_correct(self, u, p, c_dt: float, lam=None):
        """u <- u - c_dt lambda grad(p) on the faces (stagReconstruct of the
        Poisson flux); CUDA arrays."""
        self._follow(p)
        lp = [None, None, None] if lam is None else [a.data_ptr() for a in lam]
        self.check(self._lib.bmg_project_correct(self.h, *(a.data_ptr() for a in u), p.data_ptr(), *lp,
                                                 float(c_dt)), "bmg_project_correct")
        return u

    def _follow(self, t):
        import torch

        cur = torch.cuda.current_stream(t.device).cuda_stream
        if getattr(self, "_stream", None) != cur:
            self.set_stream(cur)

    def set_level_solver(self, level: int, fn=None, mode: str = "replace"):
        """fn(stream, rhs_ptr, x_ptr, n) -> None in place of the FP32 cycle's
        recursion below `level` (mode "replace"), or as the start of the
        level's usual cycle (mode "guess"); bmg_set_level_solver.  None
        removes it.  fn queues its work on `stream` (an int cudaStream_t)
        and must neither synchronise nor allocate inside a graphed solve."""
        if fn is None:
            self.check(self._lib.bmg_set_level_solver(self.h, level, N.LEVEL_SOLVER(), None, 0),
                       "bmg_set_level_solver")
            self._hook = None
            return

        def call(user, stream, rhs, x, n):
            try:
                fn(stream or 0, rhs, x, (n[0], n[1], n[2]))
                return 0
            except Exception as e:  # reported through the solve's status
                self._hook_error = e
                return 1

        hook = N.LEVEL_SOLVER(call)
        self._hook_error = None
        self.check(self._lib.bmg_set_level_solver(self.h, level, hook, None, N.LEVEL_MODE[mode]),
                   "bmg_set_level_solver")
        self._hook = hook  # kept alive with the context

    def set_stream(self, stream_ptr: int):
        self.check(self._lib.bmg_set_stream(self.h, ctypes.c_void_p(stream_ptr)), "bmg_set_stream")
        self._stream = stream_ptr

    def solve_ptr(self, b_ptr: int, x_ptr: int, flags: int) -> N.Report:
        rep = N.Report()
        rc = self._lib.bmg_solve(self.h, ctypes.c_void_p(b_ptr), ctypes.c_void_p(x_ptr), flags,
                                 ctypes.byref(rep))
        err = getattr(self, "_hook_error", None)
        if err is not None:  # the level solver raised: report its own exception
            self._hook_error = None
            raise FatalError(f"bmg_solve: the level solver raised {err!r}") from err
        if rc in (N.BAD_ARG, N.CUDA_ERROR, N.UNSUPPORTED, N.NO_DEVICE):
            self.check(rc, "bmg_solve")
        rep.status = rc
        return rep

    def solve(self, b, x, zero_guess: bool = False) -> N.Report:
        """b, x: float64 numpy arrays (host) or torch CUDA tensors (device)."""
        flags = N.ZERO_GUESS if zero_guess else 0
        if hasattr(b, "is_cuda") and b.is_cuda:
            if not (x.is_contiguous() and b.is_contiguous()):
                raise FatalError("device arrays must be contiguous")
            # queue the solve behind the work that produced b and x: on the
            # caller's current stream
            import torch

            cur = torch.cuda.current_stream(b.device).cuda_stream
            if getattr(self, "_stream", None) != cur:
                self.set_stream(cur)
            return self.solve_ptr(b.data_ptr(), x.data_ptr(), flags | N.DEVICE_PTRS)
        if not (isinstance(b, np.ndarray) and b.dtype == np.float64 and b.flags["C_CONTIGUOUS"]):
            raise FatalError("b must be a contiguous float64 array")
        if not (isinstance(x, np.ndarray) and x.dtype == np.float64 and x.flags["C_CONTIGUOUS"]):
            raise FatalError("x must be a contiguous float64 array")
        if b.size != self.n_cells or x.size != self.n_cells:
            raise FatalError(f"arrays must hold {self.n_cells} cells")
        return self.solve_ptr(b.ctypes.data, x.ctypes.data, flags)

    # building blocks (per-kernel parity)
    def upload(self, level: int, field: str, arr: np.ndarray, precision: int = 0):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        rc = self._lib.bmg_level_upload(self.h, level, {"x": 0, "b": 1}[field], precision,
                                        a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        self.check(rc, "bmg_level_upload")

    def _level_array(self, level: int) -> np.ndarray:
        # one brick: (n0, n1, n2); several: the bricks' cells one after another
        if self.n_bricks == 1:
            return np.zeros(self.shape(level))
        return np.zeros(sum(int(np.prod(s)) for s in self.shapes(level)))

    def download(self, level: int, field: str, precision: int = 0) -> np.ndarray:
        out = self._level_array(level)
        rc = self._lib.bmg_level_download(self.h, level, {"x": 0, "b": 1}[field], precision,
                                          out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        self.check(rc, "bmg_level_download")
        return out

    def shape(self, level: int, brick: int = 0):
        n = (ctypes.c_int * 3)()
        self.check(self._lib.bmg_level_shape(self.h, level, brick, n), "bmg_level_shape")
        return tuple(n)

    def shapes(self, level: int):
        return [self.shape(level, q) for q in range(self.n_bricks)]

    @property
    def num_levels(self) -> int:
        return self._lib.bmg_num_levels(self.h)

    @property
    def coarse_level_index(self) -> int:
        return self._lib.bmg_coarse_level_index(self.h)

    def tuning(self, level: int, precision: int = 0):
        """(colour stages per fused launch, planes per chunk) on a level."""
        s, t = ctypes.c_int(), ctypes.c_int()
        self.check(self._lib.bmg_level_tuning(self.h, level, precision, ctypes.byref(s), ctypes.byref(t)),
                   "bmg_level_tuning")
        return s.value, t.value

    def set_tuning(self, level: int, precision: int, stages: int, chunk: int = 64):
        """Pin a level's smoother launch shape (stages 0: pass by pass)."""
        self.check(self._lib.bmg_set_level_tuning(self.h, level, precision, stages, chunk),
                   "bmg_set_level_tuning")

    def colour_pass(self, level, colour, precision=0):
        self.check(self._lib.bmg_op_colour_pass(self.h, level, colour, precision), "colour_pass")

    def smooth(self, level, sweeps, precision=0):
        self.check(self._lib.bmg_op_smooth(self.h, level, sweeps, precision), "smooth")

    def residual(self, level, precision=0) -> np.ndarray:
        out = self._level_array(level)
        rc = self._lib.bmg_op_residual(self.h, level, precision,
                                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        self.check(rc, "residual")
        return out

    def residual_restrict(self, level, precision=0):
        self.check(self._lib.bmg_op_residual_restrict(self.h, level, precision), "residual_restrict")

    def prolong_correct(self, level, precision=0):
        self.check(self._lib.bmg_op_prolong_correct(self.h, level, precision), "prolong_correct")

    def coarse_solve(self, precision=0):
        self.check(self._lib.bmg_op_coarse_solve(self.h, precision), "coarse_solve")


def make_options(d: Dictionary | dict | None = None, **over) -> N.Options:
    """bmg_options from the reference dictionary keys (MG.C:257-305)."""
    d = Dictionary(d or {})
    d.update(over)
    o = N.Options()
    N.load().bmg_default_options(ctypes.byref(o))
    if "relTol" in d:
        o.rel_tol = _scalar(d["relTol"])
    if "tolerance" in d:
        o.abs_tol = _scalar(d["tolerance"])
    o.min_iter = _label(d.get("minIter", 0))
    o.max_iter = _label(d.get("maxIter", 999))
    o.n_pre = _label(d.get("nSweepsPre", 0))
    o.n_post = _label(d.get("nSweepsPost", 2))
    ct = str(d.get("cycleType", "F"))
    if ct not in N.CYCLE:
        raise FatalError(f"unknown cycleType {ct}")
    o.cycle_type = N.CYCLE[ct]
    o.coarse_level = _label(d.get("coarseLevel", 0))
    sm = str(d.get("smoother", "rbgs"))
    if sm not in N.SMOOTHER:
        raise FatalError("Unsupported smoother type")
    o.smoother = N.SMOOTHER[sm]
    pr = str(d.get("precision", "fp64"))
    if pr not in N.PRECISION:
        raise FatalError(f"unknown precision {pr}")
    o.precision = N.PRECISION[pr]
    o.use_graph = int(_switch(d.get("graph", "on")))
    o.remove_mean = int(_switch(d.get("removeMean", "on")))
    fused = d.get("fused", "on")
    try:
        o.fused = max(0, min(3, int(fused)))
    except (TypeError, ValueError):
        o.fused = 3 if _switch(fused) else 0
    o.autotune = int(_switch(d.get("autotune", "on")))
    o.fused_chunk = int(_scalar(d.get("fusedChunk", 64)))
    o.fuse_coarse = int(_switch(d.get("fuseCoarse", "on")))
    o.device = _label(d.get("device", 0))
    o.timeout_ms = _scalar(d.get("timeoutMs", 0))
    kr = str(d.get("krylov", "none"))
    if kr not in N.KRYLOV:
        raise FatalError(f"unknown krylov {kr}")
    o.krylov = N.KRYLOV[kr]
    cr = str(d.get("criterion", "initial"))
    if cr not in N.CRITERION:
        raise FatalError(f"unknown criterion {cr}")
    o.criterion = N.CRITERION[cr]
    # MG.C:277-287 (MGCoarseModeNames)
    cm = str(d.get("coarseMode", "direct"))
    if cm not in N.COARSE_MODE:
        raise FatalError(f"unknown coarseMode {cm}")
    o.coarse_mode = N.COARSE_MODE[cm]
    # restriction and prolongation schemes (MG.C:289-305)
    for key, table, field in (("restrict", N.RESTRICT, "restrict_scheme"), ("prolong", N.PROLONG, "prolong_scheme")):
        v = str(d.get(key, "linear"))
        if v not in table:
            raise FatalError(f"GPUMG {key} scheme must be one of {sorted(table)}, not {v}")
        setattr(o, field, table[v])
    rl = str(d.get("rowLayout", "split"))
    if rl not in N.ROW_LAYOUT:
        raise FatalError(f"unknown rowLayout {rl}")
    o.row_layout = N.ROW_LAYOUT[rl]
    o.fuse_first = int(_switch(d.get("fuseFirstPass", "on")))
    return o


class GPUMG(solver):
    """Geometric multigrid on the GPU, selected by ``type GPUMG;``."""

    typeName = "GPUMG"

    def __init__(self, dict_: Dictionary, mesh: Mesh):
        super().__init__(dict_, mesh)
        if dict_.found("coarseSolver"):
            cs = dict_.subDict("coarseSolver")
            if str(cs.lookupOrDefault("type", "APLU")) != "APLU":
                raise FatalError("GPUMG coarse solver is the on-device direct solve (APLU)")
        self.options = make_options(dict_)
        # learned initial guess: "learned guess;" with "learnedWeights <file>;"
        # (a U-Net checkpoint); the stopping test then measures against ||b||
        self.learned = str(dict_.lookupOrDefault("learned", "off"))
        if self.learned not in ("off", "guess"):
            raise FatalError(f"unknown learned mode {self.learned} (off or guess)")
        if self.learned == "guess":
            self.options.criterion = N.CRITERION["rhs"]
        self.context = Context(mesh, self.options)
        self._lam_id = None
        self.last_report = None
        self._guess = None
        if self.learned == "guess":
            self._guess = self._make_guess(dict_, mesh)

    def _make_guess(self, dict_, mesh):
        from . import learned, unet

        if not dict_.found("learnedWeights"):
            raise FatalError("learned guess needs learnedWeights <checkpoint file>")
        if len(mesh.bricks) != 1:
            raise FatalError("learned guess: one brick only")
        br = mesh.bricks[0]
        n = br.N
        if any(v % 8 for v in n):
            raise FatalError("learned guess: every extent a multiple of 8")
        for d in range(3):
            h = np.diff(br.points[d])
            if np.max(np.abs(h - h[0])) > 1e-12 * h[0] or abs(h[0] - br.cell_sizes(0)[0]) > 1e-12 * h[0]:
                raise FatalError("learned guess: uniform cubic cells only")
        net, meta = unet.UNet.from_file(str(dict_.lookup("learnedWeights")), n)
        if "target_scale" not in meta or "training_grid" not in meta:
            raise FatalError("learned guess: the checkpoint has no target scale or training grid")
        h = float(br.cell_sizes(0)[0])
        return learned.LearnedGuess(net, self.context, float(meta["target_scale"]), h=h,
                                    h_train=1.0 / float(meta["training_grid"]))

    def solve(self, sys: LinearSystem, constMatrix: bool = False):
        lam_key = None if sys.lam is None else tuple(id(a) for a in sys.lam)
        if (not constMatrix) or lam_key != self._lam_id:
            if sys.lam is not None or self._lam_id is not None:
                self.context.set_coefficients(sys.lam)
            self._lam_id = lam_key
        if self._guess is not None:
            rep = self._learned_solve(sys)
        else:
            rep = self.context.solve(sys.b, sys.x, zero_guess=sys.zero_guess)
        self.last_report = rep
        print(f"{self.typeName}: Solving for colocated x, initial residual = {rep.initial_residual:g}, "
              f"final residual = {rep.final_residual:g}, nIter = {rep.cycles}")
        if rep.status == N.NAN_DETECTED:
            raise FatalError("GPUMG: residual became NaN or Inf")
        if rep.status == N.TIMEOUT:
            raise FatalError("GPUMG: solve exceeded its time budget")
        return rep

    def _learned_solve(self, sys: LinearSystem):
        """the network's guess for b, then the multigrid solve from it"""
        import torch

        dev = self._guess.net.dev
        on_dev = hasattr(sys.b, "is_cuda") and sys.b.is_cuda
        b = sys.b if on_dev else torch.from_numpy(np.ascontiguousarray(sys.b)).to(dev)
        x = sys.x if on_dev else torch.empty_like(b)
        rep = self._guess.solve(b, x)
        if not on_dev:
            sys.x[...] = x.cpu().numpy().reshape(sys.x.shape)
        return rep
