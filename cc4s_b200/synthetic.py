"""Seeded synthetic CoupledCluster inputs (orbital energies and Coulomb vertex).

Occupied energies U[-1.5,-0.5] Eh, virtual U[0.2,3.0] Eh (sorted).  The vertex
Gamma[G,p,q] has i.i.d. N(0, s^2) entries, s = 0.1 NG^(-1/4), drawn for p <= q
and symmetrised (real, half-grid integral path) or made Hermitian (complex,
real and imaginary parts each N(0, s^2/2)); it is returned column-major.
"""
import math

import numpy as np

CONFIGS = {
    "c0": dict(No=8, Nv=40, NG=200, complex=False),
    "c1": dict(No=32, Nv=256, NG=1024, complex=False),
    "c2": dict(No=64, Nv=640, NG=2560, complex=False),
    "c3": dict(No=48, Nv=480, NG=3000, complex=True),
    "c4": dict(No=32, Nv=320, NG=1600, complex=False),
}


def synthetic(No, Nv, NG, complex=False, seed=0):
    """Returns (eps_h, eps_p, gamma, half_grid)."""
    rng = np.random.default_rng(seed)
    eps_h = np.sort(rng.uniform(-1.5, -0.5, No))
    eps_p = np.sort(rng.uniform(0.2, 3.0, Nv))
    Np = No + Nv
    s = 0.1 * NG ** (-0.25)
    iu = np.triu_indices(Np)
    # column-major (G fastest), the layout in which cc4s holds the vertex and the
    # C ABI takes it, so handing it to the library needs no copy
    if not complex:
        g = np.zeros((NG, Np, Np), order="F")
        vals = rng.standard_normal((NG, iu[0].size)) * s
        g[:, iu[0], iu[1]] = vals
        g[:, iu[1], iu[0]] = vals
        return eps_h, eps_p, g, True
    g = np.zeros((NG, Np, Np), dtype=np.complex128, order="F")
    re = rng.standard_normal((NG, iu[0].size)) * (s / math.sqrt(2.0))
    im = rng.standard_normal((NG, iu[0].size)) * (s / math.sqrt(2.0))
    vals = re + 1j * im
    diag = iu[0] == iu[1]
    vals[:, diag] = vals[:, diag].real
    g[:, iu[0], iu[1]] = vals
    g[:, iu[1], iu[0]] = np.conj(vals)
    return eps_h, eps_p, g, False


def config(name, seed=0):
    c = CONFIGS[name]
    return synthetic(c["No"], c["Nv"], c["NG"], c["complex"], seed=seed)
