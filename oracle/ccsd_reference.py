"""Restated textbook CCSD from full integral slices (cc4s ``CcsdReference``).

Test infrastructure (see ``oracle/__init__.py``).  Follows
src/main/algorithms/coupledcluster/CcsdReference.cxx:87-237, including the
V_pppp ladder, and serves as an independent cross-check of the
vertex-factorised residual in ``oracle/ccsd.py``.
"""
from __future__ import annotations

import numpy as np

from .inputs import System, coulomb_integrals


def es(subs, *ops):
    return np.einsum(subs, *ops, optimize=True)


class ReferenceInputs:
    NAMES = ["pphh", "pppp", "phph", "hhhh", "hhhp", "ppph", "hhpp", "pphp",
             "phhh", "hphp", "phhp", "phpp", "hhph", "hppp"]

    def __init__(self, sys: System):
        self.sys = sys
        self.V = coulomb_integrals(sys, self.NAMES)


def residuum(T, inp: ReferenceInputs):
    V = inp.V
    No, Nv = inp.sys.No, inp.sys.Nv
    dt = V["pphh"].dtype
    if T is None:
        return np.zeros((Nv, No), dtype=dt), V["pphh"].copy()
    T1, T2 = T
    Vpppp, Vphph, Vhhhh, Vhhhp = V["pppp"], V["phph"], V["hhhh"], V["hhhp"]
    Vhhpp, Vpphp, Vphhh = V["hhpp"], V["pphp"], V["phhh"]
    Vhphp, Vphhp, Vphpp, Vhhph, Vhppp = V["hphp"], V["phhp"], V["phpp"], V["hhph"], V["hppp"]
    Vpphh = V["pphh"]
    Kac = -2.0 * es("klcd,adkl->ac", Vhhpp, T2)
    Kac += 1.0 * es("kldc,adkl->ac", Vhhpp, T2)
    Kac += -2.0 * es("klcd,ak,dl->ac", Vhhpp, T1, T1)
    Kac += 1.0 * es("kldc,ak,dl->ac", Vhhpp, T1, T1)
    Lac = Kac.copy()
    Lac += 2.0 * es("akcd,dk->ac", Vphpp, T1)
    Lac += -1.0 * es("akdc,dk->ac", Vphpp, T1)
    Kki = 2.0 * es("klcd,cdil->ki", Vhhpp, T2)
    Kki += -1.0 * es("kldc,cdil->ki", Vhhpp, T2)
    Kki += 2.0 * es("klcd,ci,dl->ki", Vhhpp, T1, T1)
    Kki += -1.0 * es("kldc,ci,dl->ki", Vhhpp, T1, T1)
    Lki = Kki.copy()
    Lki += 2.0 * es("klic,cl->ki", Vhhhp, T1)
    Lki += -1.0 * es("klci,cl->ki", Vhhph, T1)
    R2 = 1.0 * es("ac,cbij->abij", Lac, T2)
    R2 += -1.0 * es("ki,abkj->abij", Lki, T2)
    R2 += 1.0 * es("abic,cj->abij", Vpphp, T1)
    R2 += -1.0 * es("kbic,ak,cj->abij", Vhphp, T1, T1)
    R2 += -1.0 * es("akij,bk->abij", Vphhh, T1)
    R2 += -1.0 * es("akic,cj,bk->abij", Vphhp, T1, T1)
    Xakic = Vphhp.copy()
    Xakic += -1.0 * es("lkic,al->akic", Vhhhp, T1)
    Xakic += 1.0 * es("akdc,di->akic", Vphpp, T1)
    Xakic += -0.5 * es("lkdc,dail->akic", Vhhpp, T2)
    Xakic += -1.0 * es("lkdc,di,al->akic", Vhhpp, T1, T1)
    Xakic += 1.0 * es("lkdc,adil->akic", Vhhpp, T2)
    Xakic += -0.5 * es("lkcd,adil->akic", Vhhpp, T2)
    R2 += 2.0 * es("akic,cbkj->abij", Xakic, T2)
    R2 += -1.0 * es("akic,bckj->abij", Xakic, T2)
    Xakci = Vphph.copy()
    Xakci += -1.0 * es("lkci,al->akci", Vhhph, T1)
    Xakci += 1.0 * es("akcd,di->akci", Vphpp, T1)
    Xakci += -0.5 * es("lkcd,dail->akci", Vhhpp, T2)
    Xakci += -1.0 * es("lkcd,di,al->akci", Vhhpp, T1, T1)
    R2 += -1.0 * es("akci,cbkj->abij", Xakci, T2)
    R2 += -1.0 * es("bkci,ackj->abij", Xakci, T2)
    R2 = R2 + R2.transpose(1, 0, 3, 2)
    R2 += Vpphh
    Xklij = Vhhhh.copy()
    Xklij += es("klic,cj->klij", Vhhhp, T1)
    Xklij += es("klcj,ci->klij", Vhhph, T1)
    Xklij += es("klcd,cdij->klij", Vhhpp, T2)
    Xklij += es("klcd,ci,dj->klij", Vhhpp, T1, T1)
    R2 += es("klij,abkl->abij", Xklij, T2)
    R2 += es("klij,ak,bl->abij", Xklij, T1, T1)
    Xabcd = Vpppp.copy()
    Xabcd += -1.0 * es("akcd,bk->abcd", Vphpp, T1)
    Xabcd += -1.0 * es("kbcd,ak->abcd", Vhppp, T1)
    R2 += es("abcd,cdij->abij", Xabcd, T2)
    R2 += es("abcd,ci,dj->abij", Xabcd, T1, T1)
    R1 = 1.0 * es("ac,ci->ai", Kac, T1)
    R1 += -1.0 * es("ki,ak->ai", Kki, T1)
    Kck = 2.0 * es("klcd,dl->ck", Vhhpp, T1)
    Kck += -1.0 * es("kldc,dl->ck", Vhhpp, T1)
    R1 += 2.0 * es("ck,caki->ai", Kck, T2)
    R1 += -1.0 * es("ck,caik->ai", Kck, T2)
    R1 += 1.0 * es("ck,ci,ak->ai", Kck, T1, T1)
    R1 += 2.0 * es("akic,ck->ai", Vphhp, T1)
    R1 += -1.0 * es("akci,ck->ai", Vphph, T1)
    R1 += 2.0 * es("akcd,cdik->ai", Vphpp, T2)
    R1 += -1.0 * es("akdc,cdik->ai", Vphpp, T2)
    R1 += 2.0 * es("akcd,ci,dk->ai", Vphpp, T1, T1)
    R1 += -1.0 * es("akdc,ci,dk->ai", Vphpp, T1, T1)
    R1 += -2.0 * es("klic,ackl->ai", Vhhhp, T2)
    R1 += 1.0 * es("klci,ackl->ai", Vhhph, T2)
    R1 += -2.0 * es("klic,ak,cl->ai", Vhhhp, T1, T1)
    R1 += 1.0 * es("klci,ak,cl->ai", Vhhph, T1, T1)
    return R1, R2
