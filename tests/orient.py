"""Brick orientations for tests: a brick of the mesh's frame described in
its own frame (include/bmg.h bmg_brick.transform), and fields moved between
the two frames."""
import numpy as np

from briscola_b200.mesh import Brick


def _axes(t):
    return [abs(v) - 1 for v in t], [v < 0 for v in t]


def orient(br: Brick, t) -> Brick:
    """The brick ``br`` (mesh frame) with transform ``t``: local axis d runs
    along mesh axis |t[d]| - 1, reversed when t[d] < 0."""
    if tuple(t) == (0, 0, 0):
        return br
    tax, tfl = _axes(t)
    pts, bc, vals = [], [None] * 6, [0.0] * 6
    for d in range(3):
        a = tax[d]
        pts.append(np.ascontiguousarray(br.points[a][::-1] if tfl[d] else br.points[a]))
        for side in (0, 1):
            gs = 1 - side if tfl[d] else side
            bc[2 * d + side] = br.bc[2 * a + gs]
            vals[2 * d + side] = br.values[2 * a + gs]
    return Brick(pts, tuple(bc), br.origin, tuple(vals), tuple(t))


def to_local(arr, t):
    """cell or face array of the mesh frame -> the brick's frame (a face
    array of mesh face direction |t[ld]| - 1 becomes local direction ld)"""
    if tuple(t) == (0, 0, 0):
        return arr
    tax, tfl = _axes(t)
    out = np.transpose(arr, tax)
    for d in range(3):
        if tfl[d]:
            out = np.flip(out, d)
    return np.ascontiguousarray(out)


def to_mesh(arr, t):
    """inverse of to_local"""
    if tuple(t) == (0, 0, 0):
        return arr
    tax, tfl = _axes(t)
    out = arr
    for d in range(3):
        if tfl[d]:
            out = np.flip(out, d)
    return np.ascontiguousarray(np.transpose(out, np.argsort(tax)))


def lambda_to_local(lam, t):
    """three face arrays of the mesh frame -> the brick's three local ones"""
    if tuple(t) == (0, 0, 0):
        return lam
    tax, _ = _axes(t)
    return [to_local(lam[tax[ld]], t) for ld in range(3)]
