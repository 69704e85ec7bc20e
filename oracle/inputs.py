"""Inputs of the CoupledCluster step: synthetic systems, the UEG vertex, slicing.

Test infrastructure (see ``oracle/__init__.py``).
"""
from __future__ import annotations

import itertools
import math
from dataclasses import dataclass

import numpy as np

# Synthetic systems.  Sizes (No, Nv, NG, complex) of the workloads this
# project measures: a CPU-sized case, the FP64 parity case, the large
# precision-form case, the complex case and the adjoint case.
CONFIGS = {
    "c0": dict(No=8, Nv=40, NG=200, complex=False),
    "c1": dict(No=32, Nv=256, NG=1024, complex=False),
    "c2": dict(No=64, Nv=640, NG=2560, complex=False),
    "c3": dict(No=48, Nv=480, NG=3000, complex=True),
    "c4": dict(No=32, Nv=320, NG=1600, complex=False),
}


@dataclass
class System:
    """Orbital energies and Coulomb vertex of one closed-shell system.

    ``gamma`` is Gamma[G, p, q] over all Np = No + Nv states (holes first),
    complex128 or float64.  ``half_grid`` selects the reference's real
    integral path (VertexCoulombIntegrals.cxx:45-52): V = Re*Re + Im*Im.
    """
    eps_h: np.ndarray
    eps_p: np.ndarray
    gamma: np.ndarray
    half_grid: bool

    @property
    def No(self):
        return self.eps_h.shape[0]

    @property
    def Nv(self):
        return self.eps_p.shape[0]

    @property
    def NG(self):
        return self.gamma.shape[0]

    @property
    def is_complex_path(self):
        return not self.half_grid


def synthetic_system(No, Nv, NG, complex=False, seed=0):
    """Seeded synthetic system with the distributions of the measured workloads.

    Occupied energies U[-1.5,-0.5] Eh, virtual U[0.2,3.0] Eh (sorted).  The
    vertex has i.i.d. N(0, s^2) entries with s = 0.1 NG^(-1/4), drawn for p<=q
    and symmetrised (Gamma_qp = Gamma_pq, real path) or made Hermitian
    (Gamma_qp = conj(Gamma_pq), complex path, real and imaginary parts each
    N(0, s^2/2)).
    """
    # The input generator is shared with the benchmark (inputs only; it
    # computes nothing that is checked).
    from cc4s_b200.synthetic import synthetic
    eps_h, eps_p, g, half_grid = synthetic(No, Nv, NG, complex=complex, seed=seed)
    return System(eps_h, eps_p, g, half_grid=half_grid)


def config_system(name, seed=0):
    c = CONFIGS[name]
    return synthetic_system(c["No"], c["Nv"], c["NG"], c["complex"], seed=seed)


# ---------------------------------------------------------------------------
# Uniform electron gas (src/main/algorithms/UegVertexGenerator.cxx:27-297)
# ---------------------------------------------------------------------------

def ueg_madelung(v):
    """Ewald sum of the Madelung constant, UegVertexGenerator.cxx:27-46."""
    kappa = v ** (-1.0 / 3.0)
    term2 = math.pi / (kappa * kappa * v)
    term4 = 2.0 * kappa / math.sqrt(math.pi)
    box = 1.0 / kappa
    recipsum = 0.0
    realsum = 0.0
    for l1 in range(-6, 7):
        for l2 in range(-6, 7):
            for l3 in range(-6, 7):
                n2 = l1 * l1 + l2 * l2 + l3 * l3
                if n2 > 0:
                    modr = box * math.sqrt(n2)
                    k2 = kappa * kappa * n2
                    recipsum -= 1.0 / (math.pi * k2) * math.exp(-math.pi * math.pi * k2 / kappa / kappa) / v
                    realsum -= math.erfc(kappa * modr) / modr
    return realsum + term2 + term4 + recipsum


def ueg_system(No, Nv, rs, NF=0, half_grid=False):
    """Hartree-Fock UEG eigenenergies and Coulomb vertex.

    Follows UegVertexGenerator.cxx:81-297: plane waves sorted by |k|^2, HF
    energies including the Madelung self-exchange, Gamma[G,q,p] =
    sqrt(4 pi / (V b^2 |k_q - k_p|^2)) at the momentum-transfer index G, and
    sqrt(Madelung) for zero transfer.  Energy ordering within a degenerate
    shell may differ from the reference's (std::sort is not stable); energies
    and amplitudes are invariant under it for closed shells.
    """
    Np = No + Nv
    maxG = int(math.pow(5.0 * Np, 1.0 / 3.0))
    grid = [g for g in itertools.product(range(-maxG, maxG + 1), repeat=3)]
    grid.sort(key=lambda a: a[0] * a[0] + a[1] * a[1] + a[2] * a[2])
    sl = lambda a: a[0] * a[0] + a[1] * a[1] + a[2] * a[2]
    if len(grid) < Np:
        raise ValueError("grid too small")
    if sl(grid[No]) == sl(grid[No - 1]):
        raise ValueError("occupied orbitals do not form a closed shell")
    grid = grid[:Np]
    v = rs ** 3 / 3.0 * 4.0 * math.pi * No * 2
    a = v ** (1.0 / 3.0)
    b = 2.0 * math.pi / a
    madelung = ueg_madelung(v)
    dgrid = [(b * i[0], b * i[1], b * i[2]) for i in grid]

    def vijji(p, q):
        d = (p[0] - q[0], p[1] - q[1], p[2] - q[2])
        s = d[0] * d[0] + d[1] * d[1] + d[2] * d[2]
        if s < 1e-8:
            return madelung
        return 4.0 * math.pi / v / s

    energies = np.empty(Np)
    for n, d in enumerate(dgrid):
        e = 0.5 * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2])
        e -= sum(vijji(d, dgrid[o]) for o in range(No))
        energies[n] = e
    fermi = 0.5 * (energies[No] + energies[No - 1])
    # momentum-transfer grid
    maxmom = (0, 0, 0)
    for p in range(Np):
        for q in range(Np):
            d = tuple(grid[p][k] - grid[q][k] for k in range(3))
            if sl(d) > sl(maxmom):
                maxmom = d
    maxR = sl(maxmom)
    mg = max(abs(x) for x in maxmom)
    mommap = {}
    idx = 0
    for t in itertools.product(range(-mg, mg + 1), repeat=3):
        if sl(t) > maxR:
            continue
        mommap[t] = idx
        idx += 1
    if NF == 0:
        NF = len(mommap)
    fac = 4.0 * math.pi / v
    gamma = np.zeros((NF, Np, Np), dtype=np.complex128)
    for p in range(Np):
        for q in range(Np):
            d = tuple(grid[q][k] - grid[p][k] for k in range(3))
            ii = mommap[d] % NF
            s = sl(d)
            res = fac / (b * b * s) if s else madelung
            gamma[ii, q, p] = math.sqrt(res)
    # DefineHolesAndParticles.cxx:42-95
    No_found = 0
    while No_found < Np and energies[No_found] < fermi:
        No_found += 1
    assert No_found == No
    return System(energies[:No].copy(), energies[No:].copy(), gamma, half_grid=half_grid)


# ---------------------------------------------------------------------------
# SliceOperator (SliceOperator.cxx:95-131) and VertexCoulombIntegrals
# ---------------------------------------------------------------------------

def slice_vertex(sys: System):
    """Gamma slices 'hh','hp','ph','pp' of Gamma[G,p,q] (holes first)."""
    No = sys.No
    g = sys.gamma
    return {
        "hh": g[:, :No, :No],
        "hp": g[:, :No, No:],
        "ph": g[:, No:, :No],
        "pp": g[:, No:, No:],
    }


def coulomb_integrals(sys: System, names):
    """Coulomb integral slices V[pqsr], VertexCoulombIntegrals.cxx:55-197.

    Real path (halfGrid): V_pqsr = sum_G Re G^{LO LI}_{ps} Re G^{RO RI}_{qr}
    + Im * Im.  Complex path: V_pqsr = sum_G conj(G^{LI LO}_{sp}) G^{RO RI}_{qr}.
    A slice name is LO RO LI RI, e.g. 'pphh'.
    """
    sl = slice_vertex(sys)
    out = {}
    for name in names:
        LO, RO, LI, RI = name
        if sys.half_grid:
            A = sl[LO + LI]
            B = sl[RO + RI]
            V = np.einsum("Gps,Gqr->pqsr", A.real, B.real, optimize=True)
            V += np.einsum("Gps,Gqr->pqsr", A.imag, B.imag, optimize=True)
        else:
            conjT = np.conj(sl[LI + LO]).transpose(0, 2, 1)  # [G, LO, LI]
            V = np.einsum("Gps,Gqr->pqsr", conjT, sl[RO + RI], optimize=True)
        out[name] = V
    return out
