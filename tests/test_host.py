"""Host-side logic that runs without a GPU: the C ABI library loads and
exports every function of include/bmg.h, the reference-shaped solver API
(dictionary, runtime table, option mapping), mesh generators and workloads."""
import ctypes
import os
import re

import numpy as np
import pytest

import briscola_b200 as bb
from briscola_b200 import _native as NA
from briscola_b200 import workloads
from briscola_b200.build import build_native
from briscola_b200.mesh import geometric_points, tanh_points

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    txt = open(os.path.join(ROOT, "include", "bmg.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(bmg_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_header_function():
    path = build_native()
    lib = ctypes.CDLL(path)
    fns = header_functions()
    assert len(fns) >= 20
    missing = [f for f in fns if not hasattr(lib, f)]
    assert not missing, missing
    assert set(fns) == set(NA.EXPORTED)


def test_status_strings_and_defaults():
    L = NA.load(build_native())
    assert L.bmg_status_string(0) == b"ok"
    assert b"maxIter" in L.bmg_status_string(1)
    o = NA.Options()
    L.bmg_default_options(ctypes.byref(o))
    # MG.C:264-302 and solver.C:121-122 defaults
    assert (o.n_pre, o.n_post, o.cycle_type, o.coarse_level, o.max_iter, o.min_iter) == (0, 2, 2, 0, 999, 0)


def test_create_without_device_fails_loudly():
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except ImportError:
        pass
    mesh, b, _ = workloads.cavity(8)
    with pytest.raises(bb.FatalError, match="no usable|bmg_create"):
        bb.Context(mesh, bb.make_options({}))


def test_dictionary_parser():
    d = bb.Dictionary.parse("""
        // comment
        p { type GPUMG; relTol 0.01; tolerance 1e-8; /* block */ cycleType V;
            coarseSolver { type APLU; } }
        T { type MG; relTol 0; tolerance 1e-10; }""")
    p = d.subDict("p")
    assert p.lookup("type") == "GPUMG" and float(p["relTol"]) == 0.01
    assert p.subDict("coarseSolver").lookup("type") == "APLU"
    assert d.subDict("T").lookupOrDefault("nSweepsPost", 2) == 2
    with pytest.raises(bb.FatalError):
        p.lookup("missing")


def test_runtime_table_and_unknown_type():
    mesh, _, _ = workloads.cavity(8)
    with pytest.raises(bb.FatalError, match="Valid solvers are"):
        bb.solver.New(bb.Dictionary(type="NoSuchSolver", relTol=0, tolerance=0), mesh)
    assert "GPUMG" in bb.solver._table
    with pytest.raises(bb.FatalError, match="keyword relTol"):
        bb.solver.New(bb.Dictionary(type="GPUMG", tolerance=0), mesh)


def test_make_options_maps_reference_keys():
    o = bb.make_options({"relTol": "1e-6", "tolerance": "1e-9", "nSweepsPre": "2", "cycleType": "W",
                         "coarseLevel": 1, "smoother": "jac", "precision": "mixed", "graph": "off",
                         "maxIter": 50})
    assert o.rel_tol == 1e-6 and o.abs_tol == 1e-9 and o.n_pre == 2 and o.n_post == 2
    assert o.cycle_type == NA.CYCLE["W"] and o.coarse_level == 1 and o.smoother == 1
    assert o.precision == 1 and o.use_graph == 0 and o.max_iter == 50
    with pytest.raises(bb.FatalError):
        bb.make_options({"smoother": "lexgs"})
    with pytest.raises(bb.FatalError):
        bb.make_options({"cycleType": "X"})
    assert bb.make_options({}).krylov == 0 and bb.make_options({"krylov": "fcg"}).krylov == 1
    with pytest.raises(bb.FatalError):
        bb.make_options({"krylov": "gmres"})
    assert bb.make_options({}).criterion == 0 and bb.make_options({"criterion": "rhs"}).criterion == 1
    with pytest.raises(bb.FatalError):
        bb.make_options({"criterion": "x"})
    # MG.C:277-305: coarseMode, restrict, prolong
    d = bb.make_options({})
    assert (d.coarse_mode, d.restrict_scheme, d.prolong_scheme) == (0, 0, 0)
    o = bb.make_options({"coarseMode": "smooth", "restrict": "average", "prolong": "injection"})
    assert (o.coarse_mode, o.restrict_scheme, o.prolong_scheme) == (1, 1, 1)
    for bad in ({"coarseMode": "amg"}, {"restrict": "volumeWeighted"}, {"prolong": "cubic"}):
        with pytest.raises(bb.FatalError):
            bb.make_options(bad)


def _fft_desc():
    from briscola_b200 import fft

    return fft.Desc


@pytest.mark.parametrize("header,name,mirror", [("bmg.h", "bmg_options", lambda: NA.Options),
                                                ("bmg.h", "bmg_brick", lambda: NA.Brick),
                                                ("bmg.h", "bmg_report", lambda: NA.Report),
                                                ("bfft.h", "bfft_desc", _fft_desc)])
def test_structs_match_the_header(header, name, mirror):
    """The ctypes mirrors of the C ABI's structs list the header's fields in
    order (a field missing from a mirror would shift every later one)."""
    mirror = mirror()
    txt = open(os.path.join(ROOT, "include", header)).read()
    body = txt[txt.index(f"typedef struct {name} {{"):txt.index(f"}} {name};")]
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    fields = re.findall(r"\b(?:const\s+)?(?:int|double|float|long)\s*\*?\s+(\w+)\s*(?:\[\d+\])?\s*;", body)
    assert fields == [f for f, _ in mirror._fields_]


def test_geometric_grading_ratio():
    p = geometric_points(16, 2.0)
    h = np.diff(p)
    assert abs(p[0]) < 1e-15 and abs(p[-1] - 1) < 1e-14
    # geometricGrading.C:60-67 evaluates g^(f(n-1)) at f = i/n: sizes grow
    # monotonically, ending near (not exactly at) the nominal ratio
    assert np.all(np.diff(h) > 0) and 1.5 < h[-1] / h[0] < 2.5
    assert np.allclose(geometric_points(8, 1.0), np.linspace(0, 1, 9))


def test_tanh_points_cluster_at_walls():
    p = tanh_points(64, 2.0)
    h = np.diff(p)
    assert p[0] == 0 and p[-1] == 1 and np.all(h > 0)
    assert h[0] < h[32] / 3 and abs(h[0] - h[-1]) < 1e-14


@pytest.mark.parametrize("name", ["cavity", "channel", "sphere"])
def test_workloads_are_compatible(name):
    mesh, b, lam = workloads.CONFIGS[name](16)
    # Neumann/periodic Poisson: the system RHS must sum to zero
    assert abs(b.sum()) <= 1e-12 * np.abs(b).sum()
    assert b.dtype == np.float64 and b.flags["C_CONTIGUOUS"] and b.size == 16 ** 3
    if name == "sphere":
        assert all(np.all(a > 0) for a in lam)
        assert lam[0].min() < 2e-3 and lam[0].max() == 1.0


def test_workload_seeds_are_reproducible():
    _, b1, _ = workloads.channel(16, seed=5)
    _, b2, _ = workloads.channel(16, seed=5)
    _, b3, _ = workloads.channel(16, seed=6)
    assert np.array_equal(b1, b2) and not np.array_equal(b1, b3)
