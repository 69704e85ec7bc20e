"""Parity of the device finite-size correction (cc4s_cc_finite_size_correction)
with the oracle's restatement of FiniteSizeCorrection on a B200."""
import warnings

import numpy as np
import pytest

from oracle import fsc, inputs

pytestmark = pytest.mark.gpu
warnings.simplefilter("ignore")


def lattice(n, seed=0):
    rng = np.random.default_rng(seed)
    B = 2 * np.pi / 5.0 * (np.eye(3) + 0.1 * rng.standard_normal((3, 3)))
    r = np.arange(n) - n // 2
    idx = np.array([(a, b, c) for c in r for b in r for a in r], dtype=float)
    return B, idx @ B


@pytest.mark.parametrize("case", ["real", "real_stacked", "complex"])
def test_fsc_matches_oracle(case):
    from cc4s_b200 import Solver
    No, Nv, NF = 4, 14, 30
    B, grid = lattice(6, seed=2)
    NGG = grid.shape[0]
    s = inputs.synthetic_system(No, Nv, NF, complex=case != "real", seed=4)
    rng = np.random.default_rng(6)
    T1 = rng.standard_normal((Nv, No)) * 0.05
    T2 = rng.standard_normal((Nv, Nv, No, No)) * 0.03
    if case == "complex":
        T1 = T1 + 1j * rng.standard_normal((Nv, No)) * 0.05
        T2 = T2 + 1j * rng.standard_normal((Nv, Nv, No, No)) * 0.03
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    U = (rng.standard_normal((NGG, NF)) + 1j * rng.standard_normal((NGG, NF))) / 5
    V = 0.5 + rng.random(NGG)
    g = np.asarray(s.gamma)
    S_ref = fsc.transition_structure_factor(T1, T2, g[:, No:, :No], g[:, :No, No:], U, V)
    E_ref = fsc.interpolation(S_ref, grid, B, N=3)
    sol = Solver({})
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=case != "complex")
        sol.set_initial_amplitudes(T1, T2)
        e, S = sol.finite_size_correction(grid, B, U, V, grid_size=3)
    finally:
        sol.close()
    assert np.abs(S - S_ref).max() < 1e-11 * np.abs(S_ref).max()
    for k in ("correction", "uncorrected", "corrected"):
        assert abs(e[k] - E_ref[k]) < 1e-10 * abs(E_ref["corrected"]), (k, e[k], E_ref[k])


def test_fsc_operator_after_ccsd():
    """CCSD on the device, then the FiniteSizeCorrection step on its amplitudes
    with identity singular vectors: S(G) sums to the correlation energy."""
    from cc4s_b200 import FiniteSizeCorrection, Solver
    B, grid = lattice(5, seed=1)
    NG = grid.shape[0]
    s = inputs.synthetic_system(4, 20, NG, seed=3)
    opts = dict(maxIterations=30, energyConvergence=1e-10, amplitudesConvergence=1e-8)
    sol = Solver(opts)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        r = sol.run()
        T1, T2 = sol.amplitudes()
    finally:
        sol.close()
    out = FiniteSizeCorrection().run({
        "slicedEigenEnergies": {"h": s.eps_h, "p": s.eps_p}, "coulombVertex": s.gamma,
        "halfGrid": True, "amplitudes": {"ph": T1, "pphh": T2}, "gridVectors": grid,
        "reciprocalBasis": B, "interpolationGridSize": 2})
    S = out["transitionStructureFactor"]
    assert abs(S.sum() - r["correlation"]) < 1e-9 * abs(r["correlation"])
    assert set(out["energy"]) == {"correction", "uncorrected", "corrected", "unit"}
    assert np.isfinite(out["energy"]["correction"])
