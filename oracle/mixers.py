"""Restated amplitude mixers (src/main/mixers/).

Test infrastructure (see ``oracle/__init__.py``).  An amplitude "TensorSet"
is a tuple (T1, T2); ``dot`` is sum(conj(a) * b) over both components
(src/main/TensorSet.hpp:209-224).
"""
from __future__ import annotations

import warnings

import numpy as np
import scipy.linalg


def ts_dot(a, b):
    return sum(np.vdot(x, y) for x, y in zip(a, b))


def ts_axpy_list(coeffs, vecs):
    out = [np.zeros_like(v) for v in vecs[0]]
    for c, v in zip(coeffs, vecs):
        for o, x in zip(out, v):
            o += c * x
    return tuple(out)


class DiisMixer:
    """DiisMixer.cxx:28-146.

    Ring buffer of N (amplitudes, change) pairs; bordered overlap matrix
    B with -1 borders and B[0,0] = 0; the upper-left (count+1)^2 corner is
    solved with ?sysv for right-hand side (-1, 0, ...); slot i takes the
    coefficient column[i+1].
    """

    def __init__(self, maxResidua=4):
        self.N = int(maxResidua)
        self.amplitudes = [None] * self.N
        self.residua = [None] * self.N
        self.nextIndex = 0
        self.count = 0
        M = self.N + 1
        self.B = np.zeros((M, M))
        self.B[0, 1:] = -1.0
        self.B[1:, 0] = -1.0
        self.last_coefficients = None

    def append(self, A, R):
        N = self.N
        self.amplitudes[self.nextIndex] = A
        self.residua[self.nextIndex] = R
        for i in range(N):
            if self.residua[i] is not None:
                overlap = 2.0 * ts_dot(self.residua[i], R).real
                self.B[i + 1, self.nextIndex + 1] = overlap
                self.B[self.nextIndex + 1, i + 1] = overlap
        if self.count < N:
            self.count += 1
        dim = self.count + 1
        matrix = self.B[:dim, :dim].copy()
        rhs = np.zeros(dim)
        rhs[0] = -1.0
        with warnings.catch_warnings():
            # near convergence the bordered matrix is ill-conditioned, as in the reference
            warnings.simplefilter("ignore", scipy.linalg.LinAlgWarning)
            column = scipy.linalg.solve(matrix, rhs, assume_a="sym")
        coeffs, amps, ress = [], [], []
        for j in range(self.count):
            i = (self.nextIndex + N - j) % N
            coeffs.append(column[i + 1])
            amps.append(self.amplitudes[i])
            ress.append(self.residua[i])
        self.last_coefficients = column
        self.next = ts_axpy_list(coeffs, amps)
        self.nextResiduum = ts_axpy_list(coeffs, ress)
        self.nextIndex = (self.nextIndex + 1) % N
        self.residuumNorm = float(np.sqrt(ts_dot(self.nextResiduum, self.nextResiduum).real))

    def get(self):
        return self.next

    def getResiduumNorm(self):
        return self.residuumNorm


class LinearMixer:
    """LinearMixer.cxx:27-70: T <- ratio*T_new + (1-ratio)*T_last."""

    def __init__(self, ratio=1.0):
        self.ratio = float(ratio)
        self.last = None
        self.lastResiduum = None

    def append(self, nxt, nxtR):
        if self.last is not None:
            r = self.ratio
            nxt = tuple(r * n + (1.0 - r) * l for n, l in zip(nxt, self.last))
            nxtR = tuple(r * n + (1.0 - r) * l for n, l in zip(nxtR, self.lastResiduum))
        self.last = nxt
        self.lastResiduum = nxtR
        self.residuumNorm = float(np.sqrt(ts_dot(nxtR, nxtR).real))

    def get(self):
        return self.last

    def getResiduumNorm(self):
        return self.residuumNorm


def make_mixer(mixer_opts):
    mixer_opts = mixer_opts or {}
    kind = mixer_opts.get("type", "DiisMixer")
    if kind == "DiisMixer":
        return DiisMixer(mixer_opts.get("maxResidua", 4))
    if kind == "LinearMixer":
        return LinearMixer(mixer_opts.get("ratio", 1.0))
    raise ValueError("Unknown mixer type: '%s'" % kind)
