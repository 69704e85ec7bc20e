"""Restated CCSD / CCD residuals (cc4s ``Ccsd::getResiduum``).

Test infrastructure (see ``oracle/__init__.py``).  Every statement below
follows one statement of src/main/algorithms/coupledcluster/Ccsd.cxx, in the
same order; the line numbers are given beside each block.
"""
from __future__ import annotations

import math

import numpy as np

from .inputs import System, coulomb_integrals, slice_vertex


def es(subs, *ops):
    return np.einsum(subs, *ops, optimize=True)


class CcsdInputs:
    """Vertex slices and integral slices used by the residual.

    Built once per system, like the reference's lazily evaluated recipes.
    """

    def __init__(self, sys: System):
        self.sys = sys
        self.g = slice_vertex(sys)
        names = ["pphh", "hhhh", "hhhp"]
        if not sys.half_grid:
            names += ["phhp", "hhpp", "phph", "phhh"]
        self.V = coulomb_integrals(sys, names)


def _ppl_slices(R2, Xcdij, dG_first, dG_second, No, Nv, slice_size):
    """Particle-particle ladder from vertex slices, Ccsd.cxx:283-333 / 549-601.

    dG_first[k] and dG_second[k] are lists of (left, right) factor pairs of
    V_xycd = sum_G left[G,x,c] * right[G,y,d] (summed over the list).
    """
    n_slices = int(math.ceil(1.0 * Nv / slice_size))
    for m in range(n_slices):
        for n in range(m, n_slices):
            a = n * slice_size
            b = m * slice_size
            xs = slice(a, min(a + slice_size, Nv))
            ys = slice(b, min(b + slice_size, Nv))
            V = 0
            for left, right in zip(dG_first, dG_second):
                V = V + es("Gxc,Gyd->xycd", left[:, xs, :], right[:, ys, :])
            Rxy = es("xycd,cdij->xyij", V, Xcdij)
            R2[xs, ys] += Rxy
            if a > b:
                R2[ys, xs] += Rxy.transpose(1, 0, 3, 2)


def residuum_real(T, inp: CcsdInputs, ppl=True, slice_size=None, ccd=False):
    """Ccsd<Real>::getResiduum (Ccsd.cxx:77-378).  T is None or (T1, T2)."""
    V = inp.V
    Vpphh = V["pphh"]
    No, Nv = inp.sys.No, inp.sys.Nv
    if T is None:  # Ccsd.cxx:97-102
        return np.zeros((Nv, No)), Vpphh.copy()
    T1, T2 = T
    if ccd:
        T1 = np.zeros_like(T1)
    Vhhhh, Vhhhp = V["hhhh"], V["hhhp"]
    # Ccsd.cxx:122-136: real and imaginary parts of the vertex
    parts = [(inp.g["pp"].real, inp.g["ph"].real, inp.g["hh"].real)]
    if np.iscomplexobj(inp.g["pp"]):
        parts.append((inp.g["pp"].imag, inp.g["ph"].imag, inp.g["hh"].imag))
    # Ccsd.cxx:169-197
    X = T2 + es("ai,bj->abij", T1, T1)
    Kki = 2.0 * es("cdkl,cdil->ki", Vpphh, X)
    Kki += -1.0 * es("dckl,cdil->ki", Vpphh, X)
    Lki = Kki.copy()
    Kac = -2.0 * es("cdkl,adkl->ac", Vpphh, X)
    Kac += 1.0 * es("dckl,adkl->ac", Vpphh, X)
    Lac = Kac.copy()
    for Gpp, Gph, Ghh in parts:
        Lac += 2.0 * es("Gca,Gdk,dk->ac", Gpp, Gph, T1)
    for Gpp, Gph, Ghh in parts:
        Lac += -1.0 * es("Gck,Gda,dk->ac", Gph, Gpp, T1)
    Lki += 2.0 * es("klic,cl->ki", Vhhhp, T1)
    Lki += -1.0 * es("lkic,cl->ki", Vhhhp, T1)
    R2 = 1.0 * es("ac,cbij->abij", Lac, T2)
    R2 += -1.0 * es("ki,abkj->abij", Lki, T2)
    # Ccsd.cxx:201-210
    dGph = [Gph - es("Gki,ak->Gai", Ghh, T1) for Gpp, Gph, Ghh in parts]
    for (Gpp, Gph, Ghh), d in zip(parts, dGph):
        R2 += es("Gai,Gbc,cj->abij", d, Gpp, T1)
    R2 += -1.0 * es("jika,bk->abij", Vhhhp, T1)
    R2 += -1.0 * es("bk,acik,cj->abij", T1, Vpphh, T1)
    # Ccsd.cxx:215-229: ring Xakic, with X = T2 + 2 T1 T1
    X = X + es("ai,bj->abij", T1, T1)
    Xakic = -0.5 * es("dclk,dail->akic", Vpphh, X)
    Xakic += 1.0 * es("dclk,adil->akic", Vpphh, T2)
    Xakic += -0.5 * es("cdlk,adil->akic", Vpphh, T2)
    dGph = [d + es("Gad,di->Gai", Gpp, T1) for (Gpp, Gph, Ghh), d in zip(parts, dGph)]
    for (Gpp, Gph, Ghh), d in zip(parts, dGph):
        Xakic += es("Gai,Gck->akic", d, Gph)
    Y = 2.0 * T2 - T2.transpose(1, 0, 2, 3)  # Y_cbkj = 2 T_cbkj - T_bckj
    R2 += 1.0 * es("akic,cbkj->abij", Xakic, Y)
    # Ccsd.cxx:233-257: crossed ring Xakci and the P(ab,ij) symmetrisation
    Xakci = -0.5 * es("cdlk,dail->akci", Vpphh, T2)
    dGpp = [Gpp - es("Gcl,al->Gac", Gph, T1) for Gpp, Gph, Ghh in parts]
    dGhh = [Ghh + es("Gdk,di->Gki", Gph, T1) for Gpp, Gph, Ghh in parts]
    for p, h in zip(dGpp, dGhh):
        Xakci += es("Gac,Gki->akci", p, h)
    R2 += -1.0 * es("akci,cbkj->abij", Xakci, T2)
    R2 += -1.0 * es("bkci,ackj->abij", Xakci, T2)
    R2 = R2 + R2.transpose(1, 0, 3, 2)
    # Ccsd.cxx:262-281: +V, hole-hole ladder
    R2 += Vpphh
    X = T2 + es("ai,bj->abij", T1, T1)
    Xklij = Vhhhh.copy()
    Xklij += es("klic,cj->klij", Vhhhp, T1)
    Xklij += es("lkjc,ci->klij", Vhhhp, T1)
    R2 += es("klij,abkl->abij", Xklij, X)
    Xklij = es("cdkl,cdij->klij", Vpphh, X)
    R2 += es("klij,abkl->abij", Xklij, T2 if ppl else X)
    # Ccsd.cxx:283-333: particle-particle ladder from dressed vertex slices
    if ppl:
        s = slice_size if slice_size else No
        _ppl_slices(R2, X, dGpp, dGpp, No, Nv, s)
    if ccd:
        return np.zeros((Nv, No)), R2
    # Ccsd.cxx:339-375: singles
    R1 = 1.0 * es("ac,ci->ai", Kac, T1)
    R1 += -1.0 * es("ki,ak->ai", Kki, T1)
    Kck = 2.0 * es("cdkl,dl->ck", Vpphh, T1)
    Kck += -1.0 * es("dckl,dl->ck", Vpphh, T1)
    R1 += 2.0 * es("ck,caki->ai", Kck, T2)
    R1 += -1.0 * es("ck,caik->ai", Kck, T2)
    R1 += 1.0 * es("ak,ck,ci->ai", T1, Kck, T1)
    R1 += 2.0 * es("acik,ck->ai", Vpphh, T1)
    for Gpp, Gph, Ghh in parts:
        R1 += -1.0 * es("Gca,Gik,ck->ai", Gpp, Ghh, T1)
    for Gpp, Gph, Ghh in parts:
        R1 += 2.0 * es("Gca,Gdk,cdik->ai", Gpp, Gph, X)
    for Gpp, Gph, Ghh in parts:
        R1 += -1.0 * es("Gda,Gck,cdik->ai", Gpp, Gph, X)
    R1 += -2.0 * es("klic,ackl->ai", Vhhhp, X)
    R1 += 1.0 * es("lkic,ackl->ai", Vhhhp, X)
    return R1, R2


def residuum_complex(T, inp: CcsdInputs, ppl=True, slice_size=None, ccd=False):
    """Ccsd<Complex>::getResiduum (Ccsd.cxx:382-633).  T is None or (T1, T2)."""
    V = inp.V
    Vpphh = V["pphh"]
    No, Nv = inp.sys.No, inp.sys.Nv
    if T is None:  # Ccsd.cxx:404-409
        return np.zeros((Nv, No), dtype=np.complex128), Vpphh.copy()
    T1, T2 = T
    if ccd:
        T1 = np.zeros_like(T1)
    g = inp.g
    Gpp, Gph, Ghp, Ghh = g["pp"], g["ph"], g["hp"], g["hh"]
    # Ccsd.cxx:431-436
    cTpp = np.conj(Gpp).transpose(0, 2, 1)  # cT[G,a,b] = conj(G[G,b,a])
    cThp = np.conj(Gph).transpose(0, 2, 1)  # [G,i,a]
    cTph = np.conj(Ghp).transpose(0, 2, 1)  # [G,a,i]
    cThh = np.conj(Ghh).transpose(0, 2, 1)
    Vphhp, Vhhpp, Vphph = V["phhp"], V["hhpp"], V["phph"]
    Vhhhh, Vhhhp, Vphhh = V["hhhh"], V["hhhp"], V["phhh"]
    # Ccsd.cxx:460-502
    X = T2 + es("ai,bj->abij", T1, T1)
    Y = T2 + 2.0 * es("ai,bj->abij", T1, T1)
    Kac = -2.0 * es("klcd,adkl->ac", Vhhpp, X)
    Kac += 1.0 * es("kldc,adkl->ac", Vhhpp, X)
    Lac = Kac.copy()
    Lac += 2.0 * es("Gac,Gkd,dk->ac", cTpp, Ghp, T1)
    Lac += -1.0 * es("Gad,Gkc,dk->ac", cTpp, Ghp, T1)
    Kki = 2.0 * es("klcd,cdil->ki", Vhhpp, X)
    Kki += -1.0 * es("kldc,cdil->ki", Vhhpp, X)
    Lki = Kki.copy()
    Lki += 2.0 * es("klic,cl->ki", Vhhhp, T1)
    Lki += -1.0 * es("lkic,cl->ki", Vhhhp, T1)
    R2 = 1.0 * es("ac,cbij->abij", Lac, T2)
    R2 += -1.0 * es("ki,abkj->abij", Lki, T2)
    cTdGph = cTph - es("Gki,ak->Gai", cThh, T1)
    R2 += es("Gai,Gbc,cj->abij", cTdGph, Gpp, T1)
    R2 += -1.0 * es("akij,bk->abij", Vphhh, T1)
    R2 += -1.0 * es("akic,cj,bk->abij", Vphhp, T1, T1)
    cTdGph = cTdGph + es("Gad,di->Gai", cTpp, T1)
    cTdGph = cTdGph - 0.5 * es("Gld,dail->Gai", cThp, Y)
    Xakic = es("Gai,Gkc->akic", cTdGph, Ghp)
    Yd = 1.0 * es("lkdc->dclk", Vhhpp) - 0.5 * es("lkcd->dclk", Vhhpp)
    Xakic += es("dclk,adil->akic", Yd, T2)
    Yc = 2.0 * T2 - T2.transpose(1, 0, 2, 3)
    R2 += es("akic,cbkj->abij", Xakic, Yc)
    # Ccsd.cxx:507-521
    cTdGpp = cTpp - es("Glc,al->Gac", cThp, T1)
    dGhh = Ghh + es("Gkd,di->Gki", Ghp, T1)
    Xakci = es("Gac,Gki->akci", cTdGpp, dGhh)
    Xakci += -0.5 * es("lkcd,dail->akci", Vhhpp, T2)
    R2 += -1.0 * es("akci,cbkj->abij", Xakci, T2)
    R2 += -1.0 * es("bkci,ackj->abij", Xakci, T2)
    R2 = R2 + R2.transpose(1, 0, 3, 2)
    # Ccsd.cxx:528-547
    R2 += Vpphh
    Xklij = Vhhhh.copy()
    Xklij += es("klic,cj->klij", Vhhhp, T1)
    Xklij += es("lkjc,ci->klij", Vhhhp, T1)
    R2 += es("klij,abkl->abij", Xklij, X)
    Xklij = es("klcd,cdij->klij", Vhhpp, X)
    R2 += es("klij,abkl->abij", Xklij, T2 if ppl else X)
    # Ccsd.cxx:549-601
    if ppl:
        dGpp = Gpp - es("Gkb,ak->Gab", Ghp, T1)
        s = slice_size if slice_size else No
        _ppl_slices(R2, X, [cTdGpp], [dGpp], No, Nv, s)
    if ccd:
        return np.zeros((Nv, No), dtype=np.complex128), R2
    # Ccsd.cxx:607-629
    R1 = 1.0 * es("ac,ci->ai", Kac, T1)
    R1 += -1.0 * es("ki,ak->ai", Kki, T1)
    Kck = 2.0 * es("klcd,dl->ck", Vhhpp, T1)
    Kck += -1.0 * es("kldc,dl->ck", Vhhpp, T1)
    R1 += 2.0 * es("ck,caki->ai", Kck, T2)
    R1 += -1.0 * es("ck,caik->ai", Kck, T2)
    R1 += 1.0 * es("ck,ci,ak->ai", Kck, T1, T1)
    R1 += 2.0 * es("akic,ck->ai", Vphhp, T1)
    R1 += -1.0 * es("akci,ck->ai", Vphph, T1)
    R1 += 2.0 * es("Gac,Gkd,cdik->ai", cTpp, Ghp, X)
    R1 += -1.0 * es("Gad,Gkc,cdik->ai", cTpp, Ghp, X)
    R1 += -2.0 * es("klic,ackl->ai", Vhhhp, X)
    R1 += 1.0 * es("lkic,ackl->ai", Vhhhp, X)
    return R1, R2


def residuum(T, inp: CcsdInputs, **kw):
    if inp.sys.half_grid:
        return residuum_real(T, inp, **kw)
    return residuum_complex(T, inp, **kw)
