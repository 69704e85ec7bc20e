"""Pins the oracle's tricubic interpolation (oracle/fsc.py) to the reference's own
Catmull-Rom interpolator, src/main/gte/TricubicInterpolation.hpp, compiled from
its source by oracle/build_ref.py (needs the reference tree; skipped without it).
Points inside the box, on its faces and outside it (the interpolator clamps) on
random data; agreement to rounding."""
import ctypes
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))


@pytest.fixture(scope="module")
def ref():
    import build_ref
    path = build_ref.build()
    if path is None:
        pytest.skip("reference tree not present")
    lib = ctypes.CDLL(path)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ref_tricubic.argtypes = [ctypes.c_int] * 3 + [ctypes.c_double] * 3 + [
        dp, ctypes.c_int, dp, dp]
    lib.ref_tricubic.restype = None
    return lib


@pytest.mark.parametrize("dims,origin", [((7, 6, 5), (-3.0, -2.0, -2.0)),
                                         ((4, 4, 4), (0.0, -1.0, -3.0)),
                                         ((9, 5, 8), (-4.0, -2.0, -4.0))])
def test_tricubic_matches_reference_interpolator(ref, dims, origin):
    from oracle import fsc
    rng = np.random.default_rng(sum(dims))
    F = rng.standard_normal(int(np.prod(dims)))
    lo = np.array(origin) - 1.5
    hi = np.array(origin) + np.array(dims) + 0.5
    pts = lo + (hi - lo) * rng.random((400, 3))
    # lattice points and faces exactly
    pts[:8] = np.array(origin) + np.array([[0, 0, 0], [1, 2, 1], [dims[0] - 1, 0, 0],
                                           [0, dims[1] - 1, dims[2] - 1], [2, 1, 0],
                                           [dims[0] - 1, dims[1] - 1, dims[2] - 1],
                                           [0.5, 0.25, 0.75], [1, 1, 1]], dtype=float)
    out = np.empty(len(pts))
    dp = ctypes.POINTER(ctypes.c_double)
    P = np.ascontiguousarray(pts)
    ref.ref_tricubic(dims[0], dims[1], dims[2], origin[0], origin[1], origin[2],
                     F.ctypes.data_as(dp), len(pts), P.ctypes.data_as(dp),
                     out.ctypes.data_as(dp))
    mine = np.array([fsc.tricubic(F, dims, origin, x) for x in pts])
    many = fsc.tricubic_many(F, dims, origin, pts)
    scale = np.abs(out).max()
    assert np.abs(mine - out).max() < 1e-14 * scale
    assert np.abs(many - out).max() < 1e-14 * scale
