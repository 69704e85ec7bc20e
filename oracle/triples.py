"""Restated perturbative triples (T) energy (cc4s ``PerturbativeTriples``).

Test infrastructure (see ``oracle/__init__.py``): the checker of the device
(T) path, never part of it.

Two restatements of the same energy, used against each other:

* ``triples_reference`` follows ``PerturbativeTriplesReference::run`` (the
  non-cT branch, src/main/algorithms/PerturbativeTriplesReference.cxx:107-175)
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


def triples_reference(T1, T2, V, eps_h, eps_p):
    """PerturbativeTriplesReference.cxx:107-175 (cT = 0); returns the real part of E."""
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
    E = np.sum(cj(W) / D * cj(Zs) / D * D)
    return float(np.real(E))


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
