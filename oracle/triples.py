"""Restated perturbative triples (T) energy (cc4s ``PerturbativeTriples``).

Test infrastructure (see ``oracle/__init__.py``): the checker of the device
(T) path, never part of it.

Two restatements of the same energy, used against each other:

* ``triples_reference`` follows ``PerturbativeTriplesReference::run``
  (src/main/algorithms/PerturbativeTriplesReference.cxx:92-179, both branches;
  the cT branch with ``complete_triples_intermediates``, CompleteTriples.cxx:11-118)
  statement by statement on full [a,b,c,i,j,k] arrays (small systems only);
* ``triples_atrip`` follows the tuple loop of the distributed implementation
  that ``PerturbativeTriples`` runs (perturbative-triples/src/atrip/Atrip.cxx:
  447-525 and 640; perturbative-triples/include/atrip/Equations.hpp:
  ``getEnergyDistinct``, ``getEnergySame``, ``singlesContribution`` and the
  GEMM form of ``doublesContribution``): tuples a <= b <= c without a == b == c
  (Tuples.hpp:158-185), for each one the connected triples W[i,j,k], the
  singles-augmented Z[i,j,k] and the energy over i >= j >= k.

Integral slices follow VertexCoulombIntegrals.cxx:87-121 (real) and :143-190
(complex) through ``oracle.inputs.coulomb_integrals``: V_pqsr with names
pphh, ppph, hhhp.
"""
from __future__ import annotations

import numpy as np

from .inputs import System, coulomb_integrals


def es(subs, *ops):
    return np.einsum(subs, *ops, optimize=True)


def triples_integrals(sys: System):
    """The three integral slices the (T) energy reads."""
    return coulomb_integrals(sys, ["pphh", "ppph", "hhhp"])


COMPLETE_TRIPLES_SLICES = ["pppp", "phph", "hhhh", "hhhp", "ppph", "hhpp", "pphp", "phhh",
                           "hphp", "phhp", "phpp", "hhph", "hppp", "hpph", "hphh"]


def complete_triples_intermediates(sys: System, T1, T2):
    """ct::getCompleteTriples (src/main/algorithms/CompleteTriples.cxx:11-118): the
    doubly primed intermediates I_bcek ("ppph") and I_mcjk ("hphh") of the cT
    branch, statement by statement on full arrays (small systems only)."""
    V = coulomb_integrals(sys, COMPLETE_TRIPLES_SLICES)
    t, T = T1, T2
    # :53-55  Xijka = Vhhhp + T_fk Vhhpp_ijfa
    Xijka = V["hhhp"] + es("fk,ijfa->ijka", t, V["hhpp"])
    # :57-59  pXaibc = Vphpp - 1/2 T_al Vhhpp_libc
    pXaibc = V["phpp"] - 0.5 * es("al,libc->aibc", t, V["hhpp"])
    # :61-63  Iia = 2 Vhhpp_ilaf T_fl - Vhhpp_ilfa T_fl
    Iia = 2.0 * es("ilaf,fl->ia", V["hhpp"], t) - es("ilfa,fl->ia", V["hhpp"], t)
    # :66-69  pXiajb = Vhphp - 1/2 Vhhhp_iljb T_al + T_fj pXaibc_aibf
    pXiajb = (V["hphp"] - 0.5 * es("iljb,al->iajb", V["hhhp"], t)
              + es("fj,aibf->iajb", t, pXaibc))
    # :71-74  pXiabj = Vhpph - 1/2 Vhhph_ilbj T_al + pXaibc_aifb T_fj
    pXiabj = (V["hpph"] - 0.5 * es("ilbj,al->iabj", V["hhph"], t)
              + es("aifb,fj->iabj", pXaibc, t))
    # :76-78  Xaibc = pXaibc - 1/2 T_al Vhhpp_libc
    Xaibc = pXaibc - 0.5 * es("al,libc->aibc", t, V["hhpp"])
    # :80-83  dpXiajb = Vhphp - Vhhhp_iljb T_al + 1/2 T_fj Xaibc_aibf
    dpXiajb = (V["hphp"] - es("iljb,al->iajb", V["hhhp"], t)
               + 0.5 * es("fj,aibf->iajb", t, Xaibc))
    # :85-88  dpXiabj = Vhpph - Vhhph_ilbj T_al + 1/2 Xaibc_aifb T_fj
    dpXiabj = (V["hpph"] - es("ilbj,al->iabj", V["hhph"], t)
               + 0.5 * es("aifb,fj->iabj", Xaibc, t))
    # :90-101  dpIbcek
    dpI = (V["ppph"] + es("bcef,fk->bcek", V["pppp"], t)
           - es("lbke,cl->bcek", pXiajb, t) - es("bl,lcek->bcek", t, pXiabj)
           - es("le,bclk->bcek", Iia, T)
           + 2.0 * es("blef,cfkl->bcek", Xaibc, T) - es("blef,fckl->bcek", Xaibc, T)
           - es("blfe,fclk->bcek", Xaibc, T) - es("fbkl,clfe->bcek", T, Xaibc)
           + es("cbln,lnke->bcek", T, Xijka))
    # :103-113  dpImcjk
    dpM = (V["hphh"] - es("mljk,cl->mcjk", V["hhhh"], t)
           + es("mcjf,fk->mcjk", dpXiajb, t) + es("fj,mcfk->mcjk", t, dpXiabj)
           + 2.0 * es("mljf,cfkl->mcjk", Xijka, T) - es("mljf,fckl->mcjk", Xijka, T)
           - es("lmjf,fclk->mcjk", Xijka, T) - es("cflj,lmkf->mcjk", T, Xijka)
           + es("dfkj,cmdf->mcjk", T, Xaibc))
    return {"ppph": dpI, "hphh": dpM}


def triples_reference(T1, T2, V, eps_h, eps_p, complete=None):
    """PerturbativeTriplesReference.cxx:107-175; returns the real part of E.
    complete: the intermediates of complete_triples_intermediates for the cT branch
    (:92-109, :178-179): M = I_bcdk T_adij - conj(I_lcjk) T_abil summed over the six
    simultaneous permutations, and E = sum M Z instead of sum T Z D."""
    Vpphh, Vppph, Vhhhp = V["pphh"], V["ppph"], V["hhhp"]
    cplx = np.iscomplexobj(T2) or np.iscomplexobj(Vppph)
    cj = np.conj if cplx else (lambda x: x)
    # :107-108  T = Vppph_bcdk T_adij - conj(Vhhhp_jklc) T_abil
    T = es("bcdk,adij->abcijk", Vppph, T2)
    T = T - es("jklc,abil->abcijk", cj(Vhhhp), T2)
    # :109-116  Z = sum over the six simultaneous permutations of (ai)(bj)(ck)
    Z = (T + es("bacjik->abcijk", T) + es("acbikj->abcijk", T) + es("cbakji->abcijk", T)
         + es("cabkij->abcijk", T) + es("bcajki->abcijk", T))
    W = Z
    # :118-121  S = W + T1 Vpphh (three terms)
    S = (W + es("ai,bcjk->abcijk", T1, Vpphh) + es("bj,acik->abcijk", T1, Vpphh)
         + es("ck,abij->abcijk", T1, Vpphh))
    # :123-125  Z = 4/3 S_abcijk - 2 S_acbijk + 2/3 S_bcaijk
    Zs = (4.0 / 3.0) * S - 2.0 * es("acbijk->abcijk", S) + (2.0 / 3.0) * es("bcaijk->abcijk", S)
    # :128-134  D = eps_i + eps_j + eps_k - eps_a - eps_b - eps_c
    eh = np.asarray(eps_h, dtype=float)
    ep = np.asarray(eps_p, dtype=float)
    D = (eh[None, None, None, :, None, None] + eh[None, None, None, None, :, None]
         + eh[None, None, None, None, None, :] - ep[:, None, None, None, None, None]
         - ep[None, :, None, None, None, None] - ep[None, None, :, None, None, None])
    # :136-140  Z <- conj(Z) / D, T <- conj(T) / D;  :173  E = T Z D
    if complete is None:
        E = np.sum(cj(W) / D * cj(Zs) / D * D)
        return float(np.real(E))
    # cT (:94-109): M from the intermediates, symmetrised like W;  :178-179  E = M Z
    M = es("bcdk,adij->abcijk", complete["ppph"], T2)
    M = M - es("lcjk,abil->abcijk", cj(complete["hphh"]), T2)
    M = (M + es("bacjik->abcijk", M) + es("acbikj->abcijk", M) + es("cbakji->abcijk", M)
         + es("cabkij->abcijk", M) + es("bcajki->abcijk", M))
    return float(np.real(np.sum(M * cj(Zs) / D)))


def cr_triples_denominator(T1, T2, V, eps_h, eps_p):
    """ct::getDenominator (src/main/algorithms/CompleteTriples.cxx:120-165) as the cT
    branch calls it (PerturbativeTriplesReference.cxx:187-195), with tabcijk the
    reference's T after :139 (conj(W)/D) and zabcijk its S after :155 (the singles'
    4/3, -2, 2/3 combination, conjugated, over D).  The CR-(T) energy the reference
    prints is the cT energy over this value."""
    Vpphh, Vppph, Vhhhp = V["pphh"], V["ppph"], V["hhhp"]
    cplx = np.iscomplexobj(T2) or np.iscomplexobj(Vppph)
    cj = np.conj if cplx else (lambda x: x)
    X = es("bcdk,adij->abcijk", Vppph, T2) - es("jklc,abil->abcijk", cj(Vhhhp), T2)
    W = (X + es("bacjik->abcijk", X) + es("acbikj->abcijk", X) + es("cbakji->abcijk", X)
         + es("cabkij->abcijk", X) + es("bcajki->abcijk", X))
    eh = np.asarray(eps_h, dtype=float)
    ep = np.asarray(eps_p, dtype=float)
    D = (eh[None, None, None, :, None, None] + eh[None, None, None, None, :, None]
         + eh[None, None, None, None, None, :] - ep[:, None, None, None, None, None]
         - ep[None, :, None, None, None, None] - ep[None, None, :, None, None, None])
    tT = cj(W) / D
    # :148-156  R = T1 Vpphh (three terms), S = conj(4/3 R - 2 R_acb + 2/3 R_bca) / D
    R = (es("ai,bcjk->abcijk", T1, Vpphh) + es("bj,acik->abcijk", T1, Vpphh)
         + es("ck,abij->abcijk", T1, Vpphh))
    Sz = cj((4.0 / 3.0) * R - 2.0 * es("acbijk->abcijk", R)
            + (2.0 / 3.0) * es("bcaijk->abcijk", R)) / D
    # CompleteTriples.cxx:138-162
    y = (es("ai,bj,ck->abcijk", T1, T1, T1) + es("ai,bcjk->abcijk", T1, T2)
         + es("bj,acik->abcijk", T1, T2) + es("ck,abij->abcijk", T1, T2))
    bt = (4.0 / 3.0) * tT - 2.0 * es("acbijk->abcijk", tT) + (2.0 / 3.0) * es("bcaijk->abcijk", tT)
    C = T2 + es("ai,bj->abij", T1, T1)
    Wd = 2.0 * T2 - es("baij->abij", T2)
    Dn = (2.0 * np.sum(T1 * T1) + np.sum(Wd * C) + np.sum(y * bt) + np.sum(y * Sz))
    return float(np.real(Dn)) + 1.0


def _atrip_doubles(a, b, c, T2, Vppph, Vhhhp, cplx):
    """Connected triples W[i,j,k] of one tuple: Equations.hpp, doublesContribution
    (GEMM branch: the hole integrals enter conjugated, MAYBE_CONJ)."""
    cj = np.conj if cplx else (lambda x: x)
    Vh = cj(Vhhhp)
    W = np.zeros((T2.shape[2],) * 3, dtype=np.result_type(T2, Vppph))
    # holes
    W -= es("lj,ikl->ijk", T2[a, b], Vh[:, :, :, c])   # t[abLj] V[ikLc]
    W -= es("il,jkl->ijk", T2[a, b], Vh[:, :, :, c])   # t[abiL] V[jkLc]
    W -= es("lk,ijl->ijk", T2[a, c], Vh[:, :, :, b])   # t[acLk] V[ijLb]
    W -= es("il,kjl->ijk", T2[a, c], Vh[:, :, :, b])   # t[aciL] V[kjLb]
    W -= es("lk,jil->ijk", T2[b, c], Vh[:, :, :, a])   # t[bcLk] V[jiLa]
    W -= es("jl,kil->ijk", T2[b, c], Vh[:, :, :, a])   # t[bcjL] V[kiLa]
    # particles
    W += es("eij,ek->ijk", T2[a, :, :, :], Vppph[b, c])  # t[aEij] V[bcEk]
    W += es("eik,ej->ijk", T2[a, :, :, :], Vppph[c, b])  # t[aEik] V[cbEj]
    W += es("eki,ej->ijk", T2[c, :, :, :], Vppph[a, b])  # t[cEki] V[abEj]
    W += es("ekj,ei->ijk", T2[c, :, :, :], Vppph[b, a])  # t[cEkj] V[baEi]
    W += es("eji,ek->ijk", T2[b, :, :, :], Vppph[a, c])  # t[bEji] V[acEk]
    W += es("ejk,ei->ijk", T2[b, :, :, :], Vppph[c, a])  # t[bEjk] V[caEi]
    return W


def tuple_energy(a, b, c, T1, T2, V, eps_h, eps_p):
    """Contribution of one tuple a <= b <= c (not all equal) to the sum of
    Atrip.cxx:500-525 (getEnergyDistinct / getEnergySame), before the final sign."""
    Vpphh, Vppph, Vhhhp = V["pphh"], V["ppph"], V["hhhp"]
    cplx = np.iscomplexobj(T2) or np.iscomplexobj(Vppph)
    cj = np.conj if cplx else (lambda x: x)
    No = T1.shape[1]
    eh = np.asarray(eps_h, dtype=float)
    ep = np.asarray(eps_p, dtype=float)
    i, j, k = np.meshgrid(np.arange(No), np.arange(No), np.arange(No), indexing="ij")
    keep = (i >= j) & (j >= k)
    i, j, k = i[keep], j[keep], k[keep]
    fac = np.where(i == j, 0.5, 1.0) * np.where(j == k, 0.5, 1.0)
    eijk = eh[i] + eh[j] + eh[k]
    Wt = _atrip_doubles(a, b, c, T2, Vppph, Vhhhp, cplx)
    Zt = (Wt + es("i,jk->ijk", T1[a], Vpphh[b, c]) + es("j,ik->ijk", T1[b], Vpphh[a, c])
          + es("k,ij->ijk", T1[c], Vpphh[a, b]))
    den = ep[a] + ep[b] + ep[c] - eijk
    if a != b and b != c:
        U, Vv, Ww, X, Y, Z = (Zt[i, j, k], Zt[i, k, j], Zt[j, i, k], Zt[j, k, i],
                               Zt[k, i, j], Zt[k, j, i])
        A, B, C, Dd, E, F = (cj(Wt[i, j, k]), cj(Wt[i, k, j]), cj(Wt[j, i, k]),
                             cj(Wt[j, k, i]), cj(Wt[k, i, j]), cj(Wt[k, j, i]))
        value = (3.0 * (A * U + B * Vv + C * Ww + Dd * X + E * Y + F * Z)
                 + ((U + X + Y) - 2.0 * (Vv + Ww + Z)) * (A + Dd + E)
                 + ((Vv + Ww + Z) - 2.0 * (U + X + Y)) * (B + C + F))
    else:
        # getEnergySame: U, V, W = Z[ijk], Z[jki], Z[kij]
        U3, V3, W3 = Zt[i, j, k], Zt[j, k, i], Zt[k, i, j]
        A3, B3, C3 = cj(Wt[i, j, k]), cj(Wt[j, k, i]), cj(Wt[k, i, j])
        value = 3.0 * (A3 * U3 + B3 * V3 + C3 * W3) - (A3 + B3 + C3) * (U3 + V3 + W3)
    return float(np.real(np.sum(2.0 * value / den * fac)))


def tuples(Nv):
    """The tuples of Tuples.hpp:158-185: a <= b <= c < Nv without a == b == c."""
    return [(a, b, c) for a in range(Nv) for b in range(a, Nv) for c in range(b, Nv)
            if not a == b == c]


def triples_atrip(T1, T2, V, eps_h, eps_p):
    """Atrip.cxx:447-525, 640: -sum over tuples of getEnergyDistinct / getEnergySame."""
    return -sum(tuple_energy(a, b, c, T1, T2, V, eps_h, eps_p) for a, b, c in tuples(T1.shape[0]))


def triples_flops(No, Nv):
    """Doubles flops of the tuple loop as the reference counts them
    (PerturbativeTriples.cxx, atripDryRun: No^3 Nv^3 (No + Nv) * 2)."""
    return 2.0 * No ** 3 * Nv ** 3 * (No + Nv)


def triples_star(Vpphh, eps_h, eps_p, mp2_pair_energies_cbs, triples_energy):
    """(T*) correction, computeCssdPtStar (PerturbativeTriplesStar.hpp:34-108):
    M_abij = conj(V_abij) / (e_i + e_j - e_a - e_b), basis pair energies
    2 M_abij V_abij - M_abij V_abji summed to E_MP2; returns
    (sum of the CBS pair energies) / Re E_MP2 * E_(T) and E_MP2."""
    D = (eps_h[None, None, :, None] + eps_h[None, None, None, :]
         - eps_p[:, None, None, None] - eps_p[None, :, None, None])
    M = np.conj(Vpphh) / D
    pairs = 2.0 * np.einsum("abij,abij->ij", M, Vpphh) - np.einsum("abij,abji->ij", M, Vpphh)
    e_mp2 = float(np.real(pairs.sum()))
    cbs = float(np.real(np.sum(mp2_pair_energies_cbs)))
    return cbs / e_mp2 * triples_energy, e_mp2
