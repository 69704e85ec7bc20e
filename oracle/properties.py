"""MP2 and the transition structure factor S(G).

Test infrastructure (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import numpy as np

from .inputs import System, coulomb_integrals, slice_vertex


def mp2(sys: System):
    """SecondOrderPerturbationTheory.cxx:98-128 for a canonical (f_ph = 0) system.

    Returns (correlation, direct, exchange).
    """
    Vpphh = coulomb_integrals(sys, ["pphh"])["pphh"]
    eh, ep = sys.eps_h, sys.eps_p
    D = (ep[:, None, None, None] + ep[None, :, None, None]
         - eh[None, None, :, None] - eh[None, None, None, :])
    Dpphh = np.conj(Vpphh) * (1.0 / D)
    deg = 2.0
    direct = -0.5 * deg * deg * np.einsum("abij,abij->", Vpphh, Dpphh)
    exchange = 0.5 * deg * np.einsum("abji,abij->", Vpphh, Dpphh)
    return float(np.real(direct + exchange)), float(np.real(direct)), float(np.real(exchange))


def structure_factor(sys: System, T, coulomb_potential=None):
    """Transition structure factor S(G), FiniteSizeCorrection.cxx:50-133.

    With the singular vectors U = identity and V(G) = ``coulomb_potential``
    (default 1):  C_hp = Gamma_hp / sqrt(V), cTC_hp[G,i,a] = conj(Gamma_ph[G,a,i]) / sqrt(V),
    S(G) = Re[ 2 cTC[G,i,a] C[G,j,b] Tt_abij - cTC[G,j,a] C[G,i,b] Tt_abij ],
    Tt = T2 + T1 T1.
    """
    g = slice_vertex(sys)
    NG = sys.NG
    VofG = np.ones(NG) if coulomb_potential is None else np.asarray(coulomb_potential, dtype=float)
    inv = 1.0 / np.sqrt(VofG.astype(np.complex128))
    C = g["hp"].astype(np.complex128) * inv[:, None, None]
    cTC = np.conj(g["ph"]).transpose(0, 2, 1) * inv[:, None, None]
    T1, T2 = T
    Tt = T2.astype(np.complex128) + np.einsum("ai,bj->abij", T1, T1)
    S = 2.0 * np.einsum("Gia,Gjb,abij->G", cTC, C, Tt, optimize=True)
    S += -1.0 * np.einsum("Gja,Gib,abij->G", cTC, C, Tt, optimize=True)
    return S.real
