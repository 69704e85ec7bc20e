"""Algorithmic flop count of one CCSD iteration in the reference's formulation.

Counts every contraction of Ccsd<Real>::getResiduum
(src/main/algorithms/coupledcluster/Ccsd.cxx:77-378) once, in its cheapest
pairwise order, at 2 flops per multiply-add (the rule of the reference's own
counter, src/main/tcc/Contraction.hpp:393-398).  The zero imaginary parts of a
real vertex are not counted.  Complex systems count 8 real flops per complex
multiply-add (x4).  This is the "reference-equivalent" work used for the
TFLOP/s figures: the same number for every implementation of the step, so
ratios of TFLOP/s are ratios of speed.
"""


def reference_macs(o, v, G, s=None):
    s = s or o
    macs = 0.0
    macs += 2 * o**3 * v**2            # Kki
    macs += 2 * v**3 * o**2            # Kac
    macs += 2 * (G * v * o + G * v**2)  # Lac: 2 Gamma Gamma T1 via Gamma.T1 first
    macs += 2 * G * v**2 * o           # Lac: Gamma_ck Gamma_da T_dk
    macs += 2 * o**3 * v               # Lki
    macs += v**3 * o**2 + v**2 * o**3  # Lac T2, Lki T2
    macs += G * v * o**2               # dressing Gamma_ph
    macs += G * v**2 * o + G * v**2 * o**2  # dGamma Gamma T1
    macs += v**2 * o**3 + 2 * v**2 * o**3   # V_jika T_bk, T V T
    macs += 3 * v**3 * o**3            # Xakic V.T terms
    macs += G * v**2 * o + G * v**2 * o**2  # Xakic vertex part
    macs += v**3 * o**3                # Xakic . (2T - T)
    macs += v**3 * o**3                # Xakci V.T
    macs += G * v**2 * o + G * o**2 * v + G * v**2 * o**2  # Xakci dressings and vertex part
    macs += 2 * v**3 * o**3            # Xakci . T (two terms)
    macs += 2 * o**4 * v + 3 * v**2 * o**4  # hole-hole ladder
    pairs = 0.0
    nb = (v + s - 1) // s
    for m in range(nb):
        for n in range(m, nb):
            pairs += min(s, v - n * s) * min(s, v - m * s)
    macs += pairs * v**2 * (G + o**2)  # particle-particle ladder from slices
    # singles
    macs += v**2 * o + o**2 * v + 2 * v**2 * o**2 + 2 * v**2 * o**2 + 2 * v * o**2 + v**2 * o**2
    macs += G * v * o**2 + G * v**2 * o
    macs += 2 * (G * v**2 * o**2 + G * v**2 * o)
    macs += 2 * o**3 * v**2
    return macs


def reference_flops(o, v, G, s=None, complex=False):
    return 2.0 * reference_macs(o, v, G, s) * (4.0 if complex else 1.0)
