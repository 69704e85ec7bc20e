"""Schedule::ein, the labelled-contraction helper of the device schedules (used by the
cT intermediates of the (T) step), through a test-only entry of the emulation library
(tests/emu/ein_probe.cpp) against numpy's einsum: label fusion, host loops over index
groups wider than the contraction's two levels, batch labels, scalars, the planar complex
path with conjugated operands, and the rejected forms."""
import ctypes
import os
import sys
import zlib

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))


@pytest.fixture(scope="module")
def lib():
    import build_emu
    lib = ctypes.CDLL(build_emu.build())
    P = ctypes.POINTER
    lib.emu_ein.argtypes = [
        ctypes.c_double, ctypes.c_char_p, P(ctypes.c_int64), P(ctypes.c_double), ctypes.c_int64,
        ctypes.c_int, ctypes.c_char_p, P(ctypes.c_int64), P(ctypes.c_double), ctypes.c_int64,
        ctypes.c_int, ctypes.c_double, ctypes.c_char_p, P(ctypes.c_int64), P(ctypes.c_double),
        ctypes.c_int64, P(ctypes.c_int64), ctypes.c_char_p, ctypes.c_int]
    lib.emu_ein.restype = ctypes.c_int
    return lib


def _run(lib, alpha, la, A, lb, B, beta, lc, C, cplx=False, conjA=False, conjB=False):
    """Planar operands: shape (planes, *dims); returns (C after the call, launches)."""
    def args(labels, X):
        dims = (ctypes.c_int64 * max(1, len(labels)))(*X.shape[1:])
        im = int(np.prod(X.shape[1:])) if X.shape[0] == 2 else 0
        return labels.encode(), dims, X.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), im
    la_, da, pa, ia = args(la, A)
    lb_, db, pb, ib = args(lb, B)
    lc_, dc, pc, ic = args(lc, C)
    n = ctypes.c_int64(0)
    err = ctypes.create_string_buffer(256)
    st = lib.emu_ein(alpha, la_, da, pa, ia, int(conjA), lb_, db, pb, ib, int(conjB), beta, lc_,
                     dc, pc, ic, ctypes.byref(n), err, 256)
    if st:
        raise ValueError(err.value.decode())
    return C, n.value


def _planar(rng, shape, cplx):
    return np.ascontiguousarray(rng.standard_normal((2 if cplx else 1,) + tuple(shape)))


def _value(X, conj=False):
    v = X[0] + 1j * X[1] if X.shape[0] == 2 else X[0]
    return np.conj(v) if conj else v


EXT = dict(a=5, b=4, c=3, d=6, e=2, f=3, g=2, h=3, i=4, j=2, k=3, l=4, m=2, n=3, x=3, y=2, z=2)

CASES = [
    ("ik", "kj", "ij"),              # plain matrix product
    ("ijfa", "fk", "ijka"),          # (i, j) fused in the rows
    ("bl", "lcek", "bcke"),          # three column labels that do not fuse: a host loop
    ("blef", "ckfl", "bcke"),        # two-level K, (c, k) fused
    ("blfe", "fclk", "bcek"),        # K labels in opposite orders in A and B
    ("gab", "gbc", "gac"),           # a batch label
    ("ghab", "hgbc", "ghac"),        # two batch labels
    ("ghiab", "ghibc", "ghiac"),     # three batch labels: a host loop
    ("abcd", "cdef", "abef"),        # everything fuses to one matrix product
    ("abcd", "dcef", "feab"),        # nothing fuses
    ("ik", "k", "i"),                # matrix times vector
    ("k", "k", ""),                  # a scalar
    ("xyz", "zyx", ""),              # a full contraction to a scalar
    ("ai", "bj", "abij"),            # an outer product (empty K)
]


@pytest.mark.parametrize("case", CASES)
@pytest.mark.parametrize("cplx", [False, True])
def test_ein_matches_einsum(lib, case, cplx):
    la, lb, lc = case
    rng = np.random.default_rng(zlib.crc32((",".join(case) + str(cplx)).encode()))
    A = _planar(rng, [EXT[c] for c in la], cplx)
    B = _planar(rng, [EXT[c] for c in lb], cplx)
    C = _planar(rng, [EXT[c] for c in lc], cplx)
    C0 = _value(C).copy()
    alpha, beta = 0.7, -1.3
    conjA = cplx and len(la) % 2 == 0
    got, launches = _run(lib, alpha, la, A, lb, B, beta, lc, C, cplx, conjA=conjA)
    ref = alpha * np.einsum("%s,%s->%s" % (la, lb, lc), _value(A, conjA), _value(B)) + beta * C0
    np.testing.assert_allclose(_value(got), ref, rtol=1e-12, atol=1e-12)
    assert launches >= 1


def test_ein_loops_only_where_needed(lib):
    """Fusable labels cost no host loop; a third non-fusable column label costs one
    loop over its extent (the smallest of the group)."""
    rng = np.random.default_rng(0)
    A, B = _planar(rng, (5, 4, 3, 6), False), _planar(rng, (3, 6, 2, 3), False)
    C = np.zeros((1, 5, 4, 2, 3))
    _, n = _run(lib, 1.0, "abcd", A, "cdef", B, 0.0, "abef", C)
    assert n == 1
    A, B = _planar(rng, (4, 4), False), _planar(rng, (4, 3, 2, 3), False)
    C = np.zeros((1, 4, 3, 3, 2))
    _, n = _run(lib, 1.0, "bl", A, "lcek", B, 0.0, "bcke", C)
    assert n == 2  # looped over e (extent 2), the smallest of (c, e, k)


@pytest.mark.parametrize("la,lb,lc,msg", [
    ("ii", "ij", "j", "repeated"),
    ("ik", "kj", "ijq", "one operand"),
    ("ik", "kj", "ij", "differ"),
])
def test_ein_rejects(lib, la, lb, lc, msg):
    rng = np.random.default_rng(1)
    dims = dict(i=3, j=2, k=4, q=2)
    A = _planar(rng, [dims[c] for c in la], False)
    B = _planar(rng, [dims[c] + (1 if msg == "differ" and c == "k" else 0) for c in lb], False)
    C = _planar(rng, [dims[c] for c in lc], False)
    with pytest.raises(ValueError, match=msg):
        _run(lib, 1.0, la, A, lb, B, 0.0, lc, C)
