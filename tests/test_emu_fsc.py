"""The product's finite-size correction (Schedule::structure_factor_pw and the
interpolation kernels of cc4s_b200/csrc/ops_cuda.cu, through
cc4s_cc_finite_size_correction) linked against the plain-loop CPU emulation of
the device operations and checked against the oracle's restatement of
FiniteSizeCorrection (structure factor with singular vectors and Coulomb
potential, Catmull-Rom tricubic interpolation, both energy sums)."""
import os
import sys
import warnings

import numpy as np
import pytest

from oracle import fsc, inputs

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))
warnings.simplefilter("ignore")


@pytest.fixture(scope="module")
def emu_lib():
    import build_emu
    return build_emu.build()


def lattice(n=4, seed=0):
    """Reciprocal basis (slightly skewed) and the n^3 grid vectors around 0."""
    rng = np.random.default_rng(seed)
    B = 2 * np.pi / 5.0 * (np.eye(3) + 0.1 * rng.standard_normal((3, 3)))
    r = np.arange(n) - n // 2
    idx = np.array([(a, b, c) for c in r for b in r for a in r], dtype=float)
    return B, idx @ B


def _amps(rng, No, Nv, cplx):
    T1 = rng.standard_normal((Nv, No)) * 0.05
    T2 = rng.standard_normal((Nv, Nv, No, No)) * 0.03
    if cplx:
        T1 = T1 + 1j * rng.standard_normal((Nv, No)) * 0.05
        T2 = T2 + 1j * rng.standard_normal((Nv, Nv, No, No)) * 0.03
    return T1, T2 + T2.transpose(1, 0, 3, 2)


@pytest.mark.parametrize("case", ["real", "real_stacked", "complex"])
@pytest.mark.parametrize("identity", [False, True])
def test_fsc_matches_oracle(emu_lib, case, identity):
    from cc4s_b200.coupled_cluster import Solver
    No, Nv = 2, 5
    B, grid = lattice(4, seed=1)
    NGG = grid.shape[0]
    NF = NGG if identity else 9
    cplx_vertex = case != "real"
    s = inputs.synthetic_system(No, Nv, NF, complex=cplx_vertex, seed=3)
    half_grid = case != "complex"
    rng = np.random.default_rng(5)
    T1, T2 = _amps(rng, No, Nv, cplx=case == "complex")
    U = None if identity else (rng.standard_normal((NGG, NF)) + 1j * rng.standard_normal((NGG, NF))) / 3
    V = 0.5 + rng.random(NGG)
    g = np.asarray(s.gamma)
    S_ref = fsc.transition_structure_factor(T1, T2, g[:, No:, :No], g[:, :No, No:], U, V)
    E_ref = fsc.interpolation(S_ref, grid, B, N=2, unit_factor=0.7)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=half_grid)
        sol.set_initial_amplitudes(T1, T2)
        e, S = sol.finite_size_correction(grid, B, U, V, grid_size=2, unit_factor=0.7)
    finally:
        sol.close()
    assert np.abs(S - S_ref).max() < 1e-12 * np.abs(S_ref).max()
    for k in ("correction", "uncorrected", "corrected"):
        assert abs(e[k] - E_ref[k]) < 1e-11 * max(1e-300, abs(E_ref["corrected"])), (k, e[k], E_ref[k])
    assert e["box"] == [4, 4, 4]


def test_fsc_rejects_bad_inputs(emu_lib):
    from cc4s_b200 import _abi
    from cc4s_b200.coupled_cluster import CoupledClusterError, Solver
    s = inputs.synthetic_system(2, 5, 8, seed=1)
    B, grid = lattice(4)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        with pytest.raises(CoupledClusterError) as e:   # no amplitudes yet
            sol.finite_size_correction(grid, B)
        assert e.value.status == _abi.ERR_STATE
        sol.set_initial_amplitudes(*_amps(np.random.default_rng(0), 2, 5, False))
        with pytest.raises(CoupledClusterError) as e:   # identity needs NGG == NG
            sol.finite_size_correction(grid, B)
        assert e.value.status == _abi.ERR_BAD_SHAPE
        U = np.ones((64, 8), complex)
        with pytest.raises(CoupledClusterError) as e:   # box of 3 points per direction
            sol.finite_size_correction(grid[:27] * 0 + lattice(3)[1], B, U[:27])
        assert e.value.status == _abi.ERR_BAD_SHAPE
        with pytest.raises(CoupledClusterError) as e:   # degenerate basis
            sol.finite_size_correction(grid, np.zeros((3, 3)), U)
        assert e.value.status == _abi.ERR_INVALID_ARGUMENT
    finally:
        sol.close()


def test_tricubic_interpolates_data_and_linear_functions():
    """Catmull-Rom: the data at grid points, linear functions exactly inside."""
    rng = np.random.default_rng(0)
    dims = np.array([5, 6, 7])
    origin = np.array([-2.0, -3.0, -3.0])
    F = rng.standard_normal(dims.prod())
    for _ in range(5):
        i = np.array([rng.integers(0, d) for d in dims])
        v = fsc.tricubic(F, dims, origin, origin + i)
        assert abs(v - F[i[0] + dims[0] * (i[1] + dims[1] * i[2])]) < 1e-14
    c = np.array([0.3, -1.2, 0.7])
    X, Y, Z = np.meshgrid(*[origin[d] + np.arange(dims[d]) for d in range(3)], indexing="ij")
    Fl = (c[0] * X + c[1] * Y + c[2] * Z + 0.5).transpose(2, 1, 0).reshape(-1)
    for _ in range(5):
        x = origin + 1 + rng.random(3) * (dims - 3)
        assert abs(fsc.tricubic(Fl, dims, origin, x) - (c @ x + 0.5)) < 1e-12


def test_structure_factor_with_identity_is_the_backward_one():
    """U = 1, V = 1: the FiniteSizeCorrection structure factor equals the
    frozen-amplitude one of the adjoint form (oracle.properties)."""
    from oracle import properties
    s = inputs.synthetic_system(3, 7, 11, complex=True, seed=2)
    rng = np.random.default_rng(1)
    T1, T2 = _amps(rng, 3, 7, True)
    g = np.asarray(s.gamma)
    a = fsc.transition_structure_factor(T1, T2, g[:, 3:, :3], g[:, :3, 3:])
    b = properties.structure_factor(s, (T1, T2))
    assert np.abs(a - b).max() < 1e-13 * np.abs(b).max()


@pytest.mark.parametrize("N,NF", [(1, 80), (3, 5)])
def test_fsc_grid_sizes_and_default_potential(emu_lib, N, NF):
    """interpolationGridSize 1 and 3, more vertex rows than plane waves (NF = 80 >
    NGG = 64) and fewer (NF = 5), V(G) = 1 when no potential is given."""
    from cc4s_b200.coupled_cluster import Solver
    No, Nv = 2, 4
    B, grid = lattice(4, seed=3)
    NGG = grid.shape[0]
    s = inputs.synthetic_system(No, Nv, NF, seed=9)
    rng = np.random.default_rng(2)
    T1, T2 = _amps(rng, No, Nv, False)
    U = (rng.standard_normal((NGG, NF)) + 1j * rng.standard_normal((NGG, NF))) / 4
    g = np.asarray(s.gamma)
    S_ref = fsc.transition_structure_factor(T1, T2, g[:, No:, :No], g[:, :No, No:], U, None)
    E_ref = fsc.interpolation(S_ref, grid, B, N=N)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        sol.set_initial_amplitudes(T1, T2)
        e, S = sol.finite_size_correction(grid, B, U, None, grid_size=N)
    finally:
        sol.close()
    assert np.abs(S - S_ref).max() < 1e-12 * np.abs(S_ref).max()
    assert abs(e["correction"] - E_ref["correction"]) < 1e-11 * abs(E_ref["corrected"])


def test_vectorised_tricubic_equals_the_scalar_one():
    rng = np.random.default_rng(4)
    dims = np.array([6, 5, 7])
    origin = np.array([-3.0, -2.0, -3.0])
    F = rng.standard_normal(dims.prod())
    X = origin + rng.random((200, 3)) * (dims + 2) - 1.0   # inside, near and beyond the edges
    a = fsc.tricubic_many(F, dims, origin, X)
    b = np.array([fsc.tricubic(F, dims, origin, x) for x in X])
    assert np.abs(a - b).max() < 1e-13 * np.abs(b).max()
