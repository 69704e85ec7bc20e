"""Restated direct-ring CCD residual (cc4s ``Drccd::getResiduum``).

Test infrastructure (see ``oracle/__init__.py``).  Follows
src/main/algorithms/coupledcluster/Drccd.cxx:31-104.
"""
from __future__ import annotations

import numpy as np

from .inputs import System, coulomb_integrals


class DrccdInputs:
    def __init__(self, sys: System):
        self.sys = sys
        self.V = coulomb_integrals(sys, ["pphh", "phhp", "hhpp"])


def residuum(T, inp: DrccdInputs, linearized=False, adjacent_pairs_exchange=False):
    V = inp.V
    Vpphh, Vphhp, Vhhpp = V["pphh"], V["phhp"], V["hhpp"]
    No, Nv = inp.sys.No, inp.sys.Nv
    R1 = np.zeros((Nv, No), dtype=Vpphh.dtype)
    if T is None:  # Drccd.cxx:61-66
        return R1, Vpphh.copy()
    T1, T2 = T
    deg = 2.0
    # Drccd.cxx:76-98
    R2 = deg * np.einsum("akic,cbkj->abij", Vphhp, T2, optimize=True)
    R2 = R2 + R2.transpose(1, 0, 3, 2)
    R2 = R2 + Vpphh
    if not linearized:
        W = deg * Vhhpp
        if adjacent_pairs_exchange:
            W = W - Vhhpp.transpose(1, 0, 2, 3)
        R2 = R2 + deg * np.einsum("klcd,acik,dblj->abij", W, T2, T2, optimize=True)
    return R1, R2
