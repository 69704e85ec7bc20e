"""Drccd (direct-ring CCD, Drccd.cxx:31-104): the product schedule on the CPU
emulation and, with -m gpu, on the B200, against the oracle and against the
reference's expected UEG Drccd energies."""
import json
import os
import sys
import warnings

import numpy as np
import pytest

from oracle import drccd, inputs

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))
warnings.simplefilter("ignore")
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _case(cplx, rng, No=3, Nv=8, NG=6):
    g = rng.standard_normal((NG, No + Nv, No + Nv)) * 0.1
    if cplx:
        g = g + 1j * rng.standard_normal(g.shape) * 0.1
    s = inputs.System(np.sort(rng.uniform(-1.5, -.5, No)), np.sort(rng.uniform(.2, 3, Nv)), g, not cplx)
    T2 = rng.standard_normal((Nv, Nv, No, No)) * 0.05
    if cplx:
        T2 = T2 + 1j * rng.standard_normal((Nv, Nv, No, No)) * 0.05
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    return s, (np.zeros((Nv, No), dtype=T2.dtype), T2)


def _check_residuals(lib, shape=(3, 8, 6)):
    from cc4s_b200 import Solver
    rng = np.random.default_rng(11)
    for cplx in (False, True):
        s, T = _case(cplx, rng, *shape)
        for lin in (False, True):
            for ape in (False, True):
                sol = Solver({"method": "Drccd", "linearized": lin, "adjacentPairsExchange": ape}, lib=lib)
                sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
                R1, R2 = sol.residual(T)
                Q1, Q2 = drccd.residuum(T, drccd.DrccdInputs(s), linearized=lin,
                                        adjacent_pairs_exchange=ape)
                assert _rel(R2, Q2) < 1e-12
                assert np.abs(R1).max() == 0.0


def _check_ueg(lib, tol):
    from cc4s_b200 import Solver
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    sol = Solver(g["drccd"]["options"], lib=lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    r = sol.run()
    assert r["converged"]
    for k, ref in g["drccd"]["energy"].items():
        assert abs(r[k] - ref) < tol, (k, r[k], ref)


def test_emu_drccd_residuals():
    import build_emu
    _check_residuals(build_emu.build())


def test_emu_drccd_ueg_reference_energies():
    import build_emu
    _check_ueg(build_emu.build(), 1e-10)


@pytest.mark.gpu
def test_gpu_drccd_residuals():
    _check_residuals(None, shape=(6, 40, 50))


@pytest.mark.gpu
def test_gpu_drccd_ueg_reference_energies():
    _check_ueg(None, 1e-9)
