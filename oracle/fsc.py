"""Restated finite-size correction (cc4s ``FiniteSizeCorrection``).

Test infrastructure (see ``oracle/__init__.py``): the checker of the device
finite-size-correction path, never part of it.

* ``transition_structure_factor`` follows
  ``FiniteSizeCorrection::calculateTransitionStructureFactor``
  (src/main/algorithms/FiniteSizeCorrection.cxx:50-133): the vertex is taken
  to plane waves G by the singular vectors, Gamma_G = sum_F Gamma_F U_GF, the
  codensities C = Gamma / sqrt(V(G)), and
  S(G) = Re[2 conj(C_Gai) C_Gjb Tt_abij - conj(C_Gaj) C_Gib Tt_abij],
  Tt = T2 + T1 T1.
* ``tricubic`` is the Catmull-Rom tricubic interpolation the reference takes
  from the Geometric Tools Engine (src/main/gte/TricubicInterpolation.hpp,
  IntpTricubic3 with catmullRom = true): index = (x - min) / spacing truncated
  toward zero and clamped to the grid, the 4 x 4 x 4 neighbourhood starting one
  point below it (indices clamped), weights from the Catmull-Rom blend matrix
  applied to the powers (1, t, t^2, t^3) of the offset in each direction.
* ``interpolation`` follows ``FiniteSizeCorrection::interpolation``
  (:135-310): S(G) is placed on the box of integer lattice coordinates of the
  grid (coordinates A.G with A the inverse of the reciprocal basis B; the box
  always contains the origin), interpolated on the (2N)^3-fold refined grid
  G_i + (a B_0 + b B_1 + c B_2) / 2N, a, b, c in [-N, N), and
    uncorrected = sum_{G != 0} f S(G) / |G|^2,
    corrected   = (sum over the refined points != 0 of f S_int / |g|^2) / (8 N^3),
    correction  = corrected - uncorrected,
  with f = Omega / (2 pi^2) times the unit factors.  The reference distributes
  the refined points over MPI ranks by (a + b + c) mod ranks; on one rank every
  point counts, and that is what is restated.
"""
from __future__ import annotations

import numpy as np

# Catmull-Rom blend matrix: P[row] = sum_col BLEND[row][col] t^col
CATMULL_ROM = np.array([[0.0, -0.5, 1.0, -0.5],
                        [1.0, 0.0, -2.5, 1.5],
                        [0.0, 0.5, 2.0, -1.5],
                        [0.0, 0.0, -0.5, 0.5]])


def es(subs, *ops):
    return np.einsum(subs, *ops, optimize=True)


def transition_structure_factor(T1, T2, gamma_ph, gamma_hp, U=None, V=None):
    """S(G) of FiniteSizeCorrection.cxx:50-133.  gamma_ph [F,a,i], gamma_hp [F,i,a]
    (slicedCoulombVertex "ph", "hp"); U [G,F] (coulombVertexSingularVectors,
    identity if None); V [G] (coulombPotential, ones if None)."""
    gph = np.asarray(gamma_ph, dtype=complex)
    ghp = np.asarray(gamma_hp, dtype=complex)
    if U is not None:
        gph = es("Fai,GF->Gai", gph, U)
        ghp = es("Fia,GF->Gia", ghp, U)
    G = gph.shape[0]
    Vg = np.ones(G) if V is None else np.asarray(V, dtype=float)
    inv = 1.0 / np.sqrt(Vg.astype(complex))
    C = ghp * inv[:, None, None]                                   # CGhp[G,j,b]
    cT = np.conj(gph).transpose(0, 2, 1) * inv[:, None, None]      # cTCGhp[G,i,a]
    Tt = np.asarray(T2, dtype=complex) + es("ai,bj->abij", T1, T1)
    S = 2.0 * es("Gia,Gjb,abij->G", cT, C, Tt) - es("Gja,Gib,abij->G", cT, C, Tt)
    return S.real


def tricubic(F, bounds, origin, x):
    """Catmull-Rom tricubic value at the point x (3 coordinates) of the data
    F[ix + nx (iy + ny iz)] on the grid origin + integer spacing 1."""
    nb = [int(b) for b in bounds]
    idx, powers = [], []
    for d in range(3):
        t = x[d] - origin[d]
        i = int(t)                      # truncation toward zero
        i = min(max(i, 0), nb[d] - 1)
        u = t - i
        idx.append(i - 1)
        powers.append(CATMULL_ROM @ np.array([1.0, u, u * u, u * u * u]))
    total = 0.0
    for s in range(4):
        z = min(max(idx[2] + s, 0), nb[2] - 1)
        for r in range(4):
            y = min(max(idx[1] + r, 0), nb[1] - 1)
            for c in range(4):
                xx = min(max(idx[0] + c, 0), nb[0] - 1)
                total += powers[0][c] * powers[1][r] * powers[2][s] * F[xx + nb[0] * (y + nb[1] * z)]
    return total


def tricubic_many(F, bounds, origin, X):
    """``tricubic`` at many points at once (X [n, 3]), the same arithmetic vectorised."""
    nb = np.asarray(bounds, dtype=np.int64)
    X = np.asarray(X, dtype=float)
    idx, w = [], []
    for d in range(3):
        t = X[:, d] - origin[d]
        i = np.clip(np.trunc(t).astype(np.int64), 0, nb[d] - 1)
        u = t - i
        pw = np.stack([np.ones_like(u), u, u * u, u * u * u], axis=1)   # [n, 4]
        w.append(pw @ CATMULL_ROM.T)                                     # [n, 4]
        idx.append(i - 1)
    total = np.zeros(X.shape[0])
    for s in range(4):
        z = np.clip(idx[2] + s, 0, nb[2] - 1)
        for r in range(4):
            y = np.clip(idx[1] + r, 0, nb[1] - 1)
            for c in range(4):
                x = np.clip(idx[0] + c, 0, nb[0] - 1)
                total += w[0][:, c] * w[1][:, r] * w[2][:, s] * F[x + nb[0] * (y + nb[1] * z)]
    return total


def box_of(grid, B):
    """Inverse basis A, box dimensions, origin and the S(G) placement indices."""
    B = np.asarray(B, dtype=float)
    omega = abs(np.dot(np.cross(B[0], B[1]), B[2]))
    A = np.array([np.cross(B[1], B[2]), np.cross(B[2], B[0]), np.cross(B[0], B[1])]) / omega
    direct = grid @ A.T                                           # [NG, 3]
    dmin = np.minimum(direct.min(axis=0), 0.0)
    dmax = np.maximum(direct.max(axis=0), 0.0)
    dims = np.floor(dmax - dmin + 1.5).astype(int)
    origin = np.floor(dmin + 0.5)
    return A, omega, dims, origin, direct


def interpolation(S, grid, B, N=20, unit_factor=1.0):
    """FiniteSizeCorrection.cxx:135-310 on one rank.  grid [NG, 3] cartesian G
    vectors (gridVectors), B [3, 3] rows Gi, Gj, Gk (gridVectors metaData),
    unit_factor = toCoulombVertexUnits * (grid unit / Gamma unit^2).  Returns
    dict(correction, uncorrected, corrected)."""
    grid = np.asarray(grid, dtype=float)
    A, omega, dims, origin, direct = box_of(grid, B)
    f = unit_factor * omega / 2.0 / np.pi / np.pi
    box = np.zeros(int(np.prod(dims)))
    for g in range(grid.shape[0]):
        i = np.floor(direct[g] + 0.5).astype(int) - origin.astype(int)
        box[i[0] + dims[0] * (i[1] + dims[1] * i[2])] = S[g]
    norms = (grid ** 2).sum(axis=1)
    keep = np.sqrt(norms) >= 1e-8
    sum3d = float(np.sum(f * S[keep] / norms[keep]))
    inter = 0.0
    B = np.asarray(B, dtype=float)
    for a in range(-N, N):
        for b in range(-N, N):
            for c in range(-N, N):
                shift = (B[0] * a + B[1] * b + B[2] * c) / (2.0 * N)
                for i in range(grid.shape[0]):
                    gv = grid[i] + shift
                    n2 = float(gv @ gv)
                    if np.sqrt(n2) < 1e-8:
                        continue
                    inter += f * tricubic(box, dims, origin, A @ gv) / n2
    corrected = inter / N / N / N / 8.0
    return {"correction": corrected - sum3d, "uncorrected": sum3d, "corrected": corrected}
