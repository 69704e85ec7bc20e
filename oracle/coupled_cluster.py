"""Restated CoupledCluster driver (src/main/algorithms/CoupledCluster.cxx:56-317).

Test infrastructure (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import numpy as np

from . import ccsd as ccsd_mod
from . import ccsd_reference
from .inputs import System
from .mixers import make_mixer

DEFAULTS = dict(
    method="Ccsd",
    maxIterations=16,            # CoupledCluster.hpp:45
    energyConvergence=1e-7,      # CoupledCluster.hpp:46
    amplitudesConvergence=1e-6,  # CoupledCluster.hpp:47
    levelShift=0.0,              # CoupledCluster.hpp:49
    ppl=True,
    integralsSliceSize=None,
    mixer=None,
)


def energy_differences(sys: System, level):
    """calculateEnergyDifferences, CoupledCluster.cxx:286-317."""
    eh, ep = sys.eps_h, sys.eps_p
    if level == 1:
        return ep[:, None] - eh[None, :]
    return (ep[:, None, None, None] + ep[None, :, None, None]
            - eh[None, None, :, None] - eh[None, None, None, :])


def residuum_to_amplitudes(R, T, sys: System, level_shift):
    """CoupledCluster.cxx:256-283: R <- -(R - s T) / (D + s)."""
    R1, R2 = R
    if T is not None and level_shift != 0.0:
        R1 = R1 - level_shift * T[0]
        R2 = R2 - level_shift * T[1]
    D1 = energy_differences(sys, 1)
    D2 = energy_differences(sys, 2)
    return R1 * (-1.0 / (D1 + level_shift)), R2 * (-1.0 / (D2 + level_shift))


def get_energy(T, Vpphh):
    """getEnergy, CoupledCluster.cxx:195-253.

    direct = 2 sum (T_abij + T_ai T_bj) V_ijab, exchange = -sum (...) V_ijba,
    with V_ijab = conj(V_abij).
    """
    T1, T2 = T
    Vijab = np.conj(Vpphh).transpose(2, 3, 0, 1)  # Vijab[i,j,a,b]
    deg = 2.0
    D = 0.5 * deg * deg * np.einsum("abij,ijab->", T2, Vijab, optimize=True)
    D += 0.5 * deg * deg * np.einsum("ai,bj,ijab->", T1, T1, Vijab, optimize=True)
    X = -0.5 * deg * np.einsum("abij,ijba->", T2, Vijab, optimize=True)
    X += -0.5 * deg * np.einsum("ai,bj,ijba->", T1, T1, Vijab, optimize=True)
    return D + X, D, X


class Result(dict):
    pass


def iterations(sys: System, initial_amplitudes=None, **opts):
    """The loop body of CoupledCluster::run<F,TE> (CoupledCluster.cxx:129-175) as a
    generator: each next() performs one iteration (residuum, Jacobi update, mixer,
    energy) and yields (T, history entry, second_order_flag, converged_flag)."""
    o = dict(DEFAULTS)
    o.update(opts)
    method = o["method"]
    inp = ccsd_mod.CcsdInputs(sys)
    if method == "Ccsd" or method == "Ccd":
        kw = dict(ppl=bool(o["ppl"]), slice_size=o["integralsSliceSize"], ccd=(method == "Ccd"))
        res_fn = lambda T: ccsd_mod.residuum(T, inp, **kw)
    elif method == "Drccd":
        from . import drccd
        dr_inp = drccd.DrccdInputs(sys)
        res_fn = lambda T: drccd.residuum(T, dr_inp, linearized=bool(o.get("linearized", False)),
                                          adjacent_pairs_exchange=bool(o.get("adjacentPairsExchange", False)))
    elif method == "CcsdReference":
        ref_inp = ccsd_reference.ReferenceInputs(sys)
        res_fn = lambda T: ccsd_reference.residuum(T, ref_inp)
    else:
        raise ValueError("Unknown method: '%s'" % method)
    mixer = make_mixer(o["mixer"])
    e_conv = float(o["energyConvergence"])
    a_conv = float(o["amplitudesConvergence"])
    shift = float(o["levelShift"])
    T = initial_amplitudes
    previousE = 0.0
    while True:
        R = res_fn(T)
        R = residuum_to_amplitudes(R, T, sys, shift)
        if T is not None:
            dT = (R[0] - T[0], R[1] - T[1])
            second = False
        else:
            dT = (R[0].copy(), R[1].copy())
            second = True
        mixer.append(R, dT)
        T = mixer.get()
        norm = mixer.getResiduumNorm()
        e, D, X = get_energy(T, inp.V["pphh"])
        h = dict(energy=float(np.real(e)), dE=float(np.real(e - previousE)), dR=norm)
        converged = abs(e - previousE) < e_conv and norm < a_conv
        previousE = e
        yield T, h, second, converged, inp


def run(sys: System, initial_amplitudes=None, **opts):
    """CoupledCluster::run<F,TE>, CoupledCluster.cxx:56-191.

    Returns a dict with 'energy' (correlation, direct, exchange,
    secondOrder), 'convergenceReached', 'amplitudes' (T1, T2), 'iterations'
    and the per-iteration history (energy, dE, residuum norm).
    """
    o = dict(DEFAULTS)
    o.update(opts)
    maxIt = int(o["maxIterations"])
    T = initial_amplitudes
    energy = {}
    history = []
    i = 0
    inp = None
    if maxIt > 0:
        for T, h, second, converged, inp in iterations(sys, initial_amplitudes, **opts):
            history.append(h)
            if second:
                energy["secondOrder"] = h["energy"]
            if converged:
                break
            i += 1
            if i >= maxIt:
                break
    if inp is None:
        inp = ccsd_mod.CcsdInputs(sys)
    e, D, X = get_energy(T, inp.V["pphh"])
    energy.update(correlation=float(np.real(e)), direct=float(np.real(D)),
                  exchange=float(np.real(X)), unit=1.0)
    return Result(energy=energy, convergenceReached=i < maxIt, amplitudes=T,
                  iterations=len(history), history=history)
