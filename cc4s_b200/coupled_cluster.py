"""Host-side mirror of cc4s's ``CoupledCluster`` algorithm step.

``CoupledCluster().run(arguments)`` takes the same keys as the reference's YAML
step (src/main/algorithms/CoupledCluster.cxx:56-191) and returns the same
output map; all work goes through the C ABI of the CUDA library
(include/cc4s_cc.h).  ``Solver`` is the thin handle wrapper underneath.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi


class CoupledClusterError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("status %d: %s" % (status, message))
        self.status = status


def _options(lib, arguments):
    o = _abi.Options()
    lib.cc4s_cc_default_options(ctypes.byref(o))
    method = arguments.get("method", "Ccsd")
    if method not in _abi.METHODS:
        raise CoupledClusterError(_abi.ERR_INVALID_ARGUMENT, "Unknown method: '%s'" % method)
    o.method = _abi.METHODS[method]
    mixer = arguments.get("mixer") or {}
    mtype = mixer.get("type", "DiisMixer")
    if mtype not in _abi.MIXERS:
        raise CoupledClusterError(_abi.ERR_INVALID_ARGUMENT, "Unknown mixer type: '%s'" % mtype)
    o.mixer = _abi.MIXERS[mtype]
    o.max_residua = int(mixer.get("maxResidua", 4))
    o.ratio = float(mixer.get("ratio", 1.0))
    o.max_iterations = int(arguments.get("maxIterations", 16))
    o.energy_convergence = float(arguments.get("energyConvergence", 1e-7))
    o.amplitudes_convergence = float(arguments.get("amplitudesConvergence", 1e-6))
    o.level_shift = float(arguments.get("levelShift", 0.0))
    o.integrals_slice_size = int(arguments.get("integralsSliceSize", 0) or 0)
    o.ppl = 1 if arguments.get("ppl", True) else 0
    o.precision = _abi.PRECISIONS[arguments.get("precision", "fp64")]
    o.device = int(arguments.get("device", 0))
    o.profile = 1 if arguments.get("profile", False) else 0
    o.linearized = 1 if arguments.get("linearized", False) else 0
    o.adjacent_pairs_exchange = 1 if arguments.get("adjacentPairsExchange", False) else 0
    o.precision_refinement = float(arguments.get("precisionRefinement", 0.0))
    return o


class Solver:
    """One library handle: inputs resident on the device, residual and run entries."""

    def __init__(self, arguments=None, lib=None):
        self.lib = _abi.load(lib)
        self.h = ctypes.c_void_p()
        self.opts = _options(self.lib, arguments or {})
        st = self.lib.cc4s_cc_create(ctypes.byref(self.opts), ctypes.byref(self.h))
        if st:
            raise CoupledClusterError(st, self.lib.cc4s_cc_last_error(None).decode())
        self.No = self.Nv = self.NG = None
        self.cplx = False

    def _check(self, st, ok=(0,)):
        if st not in ok:
            raise CoupledClusterError(st, self.lib.cc4s_cc_last_error(self.h).decode())
        return st

    def close(self):
        if self.h:
            self.lib.cc4s_cc_destroy(self.h)
            self.h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_inputs(self, eps_h, eps_p, gamma, half_grid=True):
        eps_h = np.ascontiguousarray(eps_h, dtype=np.float64)
        eps_p = np.ascontiguousarray(eps_p, dtype=np.float64)
        gamma = np.asarray(gamma)
        NG, Np, Np2 = gamma.shape
        No, Nv = eps_h.size, eps_p.size
        if Np != No + Nv or Np2 != Np:
            raise CoupledClusterError(_abi.ERR_BAD_SHAPE, "vertex shape %s vs No=%d Nv=%d" % (gamma.shape, No, Nv))
        cplx = np.iscomplexobj(gamma)
        g = _abi.as_f64(gamma)
        self._check(self.lib.cc4s_cc_set_inputs(self.h, _abi.ptr(eps_h), No, _abi.ptr(eps_p), Nv,
                                                _abi.ptr(g), NG, int(cplx), int(bool(half_grid))))
        self.No, self.Nv, self.NG = No, Nv, NG
        self.cplx = cplx and not half_grid
        self.in_complex_input = cplx

    def _dtype(self):
        return np.complex128 if self.cplx else np.float64

    def set_initial_amplitudes(self, T1, T2):
        t1 = _abi.as_f64(np.asarray(T1, dtype=self._dtype()))
        t2 = _abi.as_f64(np.asarray(T2, dtype=self._dtype()))
        self._check(self.lib.cc4s_cc_set_initial_amplitudes(self.h, _abi.ptr(t1), _abi.ptr(t2)))

    def _alloc_amps(self):
        k = 2 if self.cplx else 1
        return (np.zeros(self.Nv * self.No * k), np.zeros((self.Nv * self.No) ** 2 * k))

    def _unpack(self, b1, b2):
        No, Nv = self.No, self.Nv
        if self.cplx:
            b1, b2 = b1.view(np.complex128), b2.view(np.complex128)
        return b1.reshape((Nv, No), order="F"), b2.reshape((Nv, Nv, No, No), order="F")

    def residual(self, T=None):
        """One residual evaluation, Ccsd::getResiduum; T is None or (T1, T2)."""
        r1, r2 = self._alloc_amps()
        if T is None:
            self._check(self.lib.cc4s_cc_residual(self.h, None, None, _abi.ptr(r1), _abi.ptr(r2)))
        else:
            t1 = _abi.as_f64(np.asarray(T[0], dtype=self._dtype()))
            t2 = _abi.as_f64(np.asarray(T[1], dtype=self._dtype()))
            self._check(self.lib.cc4s_cc_residual(self.h, _abi.ptr(t1), _abi.ptr(t2),
                                                  _abi.ptr(r1), _abi.ptr(r2)))
        return self._unpack(r1, r2)

    def run(self):
        res = _abi.Result()
        st = self._check(self.lib.cc4s_cc_run(self.h, ctypes.byref(res)),
                         ok=(0, _abi.WARN_NOT_CONVERGED))
        n = res.history_len
        hist = [dict(energy=res.energy[k], dE=res.delta_energy[k], dR=res.residuum_norm[k],
                     seconds=res.seconds[k]) for k in range(n)]
        return dict(status=st, correlation=res.correlation, direct=res.direct,
                    exchange=res.exchange, secondOrder=res.second_order,
                    correlation_imag=res.correlation_imag, iterations=res.iterations,
                    converged=bool(res.converged), history=hist,
                    flops_per_iteration=res.flops_per_iteration, refined_from=res.refined_from)

    def amplitudes(self):
        t1, t2 = self._alloc_amps()
        self._check(self.lib.cc4s_cc_get_amplitudes(self.h, _abi.ptr(t1), _abi.ptr(t2)))
        return self._unpack(t1, t2)

    def backward(self, gradient=False):
        """Adjoint at the current amplitudes: S(G) = dE/dV(G) and, on the real
        path, dE/dGamma in the caller's vertex layout (cc4s_cc_backward)."""
        S = np.zeros(self.NG)
        g = None
        if gradient:
            k = 2 if self.in_complex_input else 1
            g = np.zeros(self.NG * (self.No + self.Nv) ** 2 * k)
        self._check(self.lib.cc4s_cc_backward(self.h, _abi.ptr(S), _abi.ptr(g)))
        if g is not None:
            Np = self.No + self.Nv
            if self.in_complex_input:
                g = g.view(np.complex128)
            g = g.reshape((self.NG, Np, Np), order="F")
        return S, g

    def _vertex_grad_buffer(self):
        k = 2 if self.in_complex_input else 1
        return np.zeros(self.NG * (self.No + self.Nv) ** 2 * k)

    def _vertex_grad(self, g):
        Np = self.No + self.Nv
        if self.in_complex_input:
            g = g.view(np.complex128)
        return g.reshape((self.NG, Np, Np), order="F")

    def residual_vjp(self, T, Rbar, gradient=True):
        """Transposed-Jacobian product of the residual at amplitudes T = (T1, T2):
        returns (T1bar, T2bar) = Rbar^T dR/dT and, if asked, Rbar^T dR/dGamma in the
        vertex layout (cc4s_cc_residual_vjp).  On the complex path every adjoint is
        d/dRe + i d/dIm of the real-valued <Rbar, R> pairing Re sum conj(Rbar) R."""
        dt = self._dtype()
        t1 = _abi.as_f64(np.asarray(T[0], dtype=dt))
        t2 = _abi.as_f64(np.asarray(T[1], dtype=dt))
        r1 = _abi.as_f64(np.asarray(Rbar[0], dtype=dt))
        r2 = _abi.as_f64(np.asarray(Rbar[1], dtype=dt))
        b1, b2 = self._alloc_amps()
        g = self._vertex_grad_buffer() if gradient else None
        self._check(self.lib.cc4s_cc_residual_vjp(self.h, _abi.ptr(t1), _abi.ptr(t2), _abi.ptr(r1),
                                                  _abi.ptr(r2), _abi.ptr(b1), _abi.ptr(b2),
                                                  _abi.ptr(g)))
        T1b, T2b = self._unpack(b1, b2)
        return (T1b, T2b), (self._vertex_grad(g) if gradient else None)

    def relaxed_gradient(self, max_iterations=100, convergence=1e-10):
        """dE_c/dGamma of the converged energy (Lambda equations solved on the device;
        cc4s_cc_relaxed_gradient).  Returns (gradient in the vertex layout, info)."""
        g = self._vertex_grad_buffer()
        res = _abi.LambdaResult()
        st = self._check(self.lib.cc4s_cc_relaxed_gradient(self.h, int(max_iterations),
                                                           float(convergence), _abi.ptr(g),
                                                           ctypes.byref(res)),
                         ok=(0, _abi.WARN_NOT_CONVERGED))
        info = dict(status=st, iterations=res.iterations, converged=bool(res.converged),
                    residuum_norm=res.residuum_norm, prepare_seconds=res.prepare_seconds,
                    vjp_seconds=res.vjp_seconds, gradient_seconds=res.gradient_seconds)
        return self._vertex_grad(g), info

    def perturbative_triples(self, block_size=0, reference_form=False, cT=False):
        """(T) energy at the current amplitudes (cc4s_cc_perturbative_triples);
        reference_form: the conjugation of PerturbativeTriplesReference (complex path);
        cT: its completely renormalised branch (PerturbativeTriplesReference.cxx:92-109)."""
        o = _abi.TriplesOptions()
        self.lib.cc4s_cc_triples_default_options(ctypes.byref(o))
        o.block_size = int(block_size)
        o.formulation = 1 if reference_form else 0
        o.cT = 1 if cT else 0
        r = _abi.TriplesResult()
        self._check(self.lib.cc4s_cc_perturbative_triples(self.h, ctypes.byref(o),
                                                          ctypes.byref(r)))
        return dict(correlation=r.correlation, seconds=r.seconds,
                    setup_seconds=r.setup_seconds, flops=r.flops,
                    executed_flops=r.executed_flops, block_size=r.block_size,
                    block_triples=r.block_triples, mp2_energy=r.mp2_energy,
                    cr_denominator=r.cr_denominator,
                    cr_correlation=(r.correlation / r.cr_denominator
                                    if r.cr_denominator != 0.0 else None),
                    phase_seconds=dict(zip(("singles", "particle", "hole", "energy"),
                                           list(r.phase_seconds))))

    def finite_size_correction(self, grid, reciprocal_basis, singular_vectors=None,
                               coulomb_potential=None, grid_size=20, unit_factor=1.0):
        """FiniteSizeCorrection at the current amplitudes (cc4s_cc_finite_size_correction).
        grid [NGG, 3] cartesian G vectors; reciprocal_basis [3, 3] rows Gi, Gj, Gk;
        singular_vectors U [NGG, NG] (None: identity); coulomb_potential V [NGG].
        Returns (energy dict, S(G))."""
        grid = np.ascontiguousarray(grid, dtype=np.float64)
        NGG = grid.shape[0]
        B = np.ascontiguousarray(reciprocal_basis, dtype=np.float64).reshape(9)
        U = None
        if singular_vectors is not None:
            U = np.asarray(singular_vectors, dtype=np.complex128).reshape(-1, order="F").view(np.float64)
        V = None if coulomb_potential is None else np.ascontiguousarray(coulomb_potential, dtype=np.float64)
        o = _abi.FscOptions()
        self.lib.cc4s_cc_fsc_default_options(ctypes.byref(o))
        o.interpolation_grid_size = int(grid_size)
        o.unit_factor = float(unit_factor)
        S = np.empty(NGG)
        r = _abi.FscResult()
        self._check(self.lib.cc4s_cc_finite_size_correction(
            self.h, _abi.ptr(U), NGG, _abi.ptr(V), _abi.ptr(grid), _abi.ptr(B), ctypes.byref(o),
            _abi.ptr(S), ctypes.byref(r)))
        return (dict(correction=r.correction, uncorrected=r.uncorrected, corrected=r.corrected,
                     seconds=r.seconds, box=list(r.box)), S)

    def stats(self):
        s = _abi.Stats()
        self._check(self.lib.cc4s_cc_get_stats(self.h, ctypes.byref(s)))
        return dict(gemm_launches=s.gemm_launches, other_launches=s.other_launches,
                    device_bytes=s.device_bytes, flops_per_residual=s.flops_per_residual,
                    gemm_seconds=s.gemm_seconds, gemm_flops=s.gemm_flops,
                    top_seconds=s.top_seconds, top_flops=s.top_flops,
                    gemm_profiled_launches=s.gemm_profiled_launches,
                    split_seconds=s.split_seconds, split_flops=s.split_flops,
                    split_launches=s.split_launches)


def _full_vertex(arguments):
    if "coulombVertex" in arguments:
        return np.asarray(arguments["coulombVertex"])
    sl = arguments["slicedCoulombVertex"]
    hh, hp, ph, pp = (np.asarray(sl[k]) for k in ("hh", "hp", "ph", "pp"))
    NG, No, Nv = hh.shape[0], hh.shape[1], pp.shape[1]
    dt = np.result_type(hh, hp, ph, pp)
    g = np.zeros((NG, No + Nv, No + Nv), dtype=dt)
    g[:, :No, :No], g[:, :No, No:], g[:, No:, :No], g[:, No:, No:] = hh, hp, ph, pp
    return g


class CoupledCluster:
    """The cc4s ``CoupledCluster`` step (methods Ccsd and Ccd).

    ``arguments`` holds the reference's input keys: slicedEigenEnergies
    ({'h': eps_h, 'p': eps_p}), slicedCoulombVertex ({'hh','hp','ph','pp'}
    slices of Gamma[G,p,q]) or coulombVertex (the full Gamma), halfGrid (the
    vertex metadata that selects the real integral path), coulombIntegrals
    (accepted and not needed), method, mixer, maxIterations,
    energyConvergence, amplitudesConvergence, levelShift, initialAmplitudes
    ({'ph': T1, 'pphh': T2}), integralsSliceSize and ppl.
    """

    def __init__(self, lib=None):
        self.lib = lib

    def run(self, arguments):
        eps = arguments["slicedEigenEnergies"]
        gamma = _full_vertex(arguments)
        half_grid = bool(arguments.get("halfGrid", not np.iscomplexobj(gamma)))
        s = Solver(arguments, lib=self.lib)
        try:
            s.set_inputs(eps["h"], eps["p"], gamma, half_grid=half_grid)
            init = arguments.get("initialAmplitudes")
            if init is not None:
                s.set_initial_amplitudes(init["ph"], init["pphh"])
            r = s.run()
            T1, T2 = s.amplitudes()
        finally:
            s.close()
        energy = dict(correlation=r["correlation"], direct=r["direct"], exchange=r["exchange"],
                      unit=1.0)
        if not np.isnan(r["secondOrder"]):
            energy["secondOrder"] = r["secondOrder"]
        return {"energy": energy, "convergenceReached": r["converged"],
                "amplitudes": {"ph": T1, "pphh": T2}, "iterations": r["iterations"],
                "history": r["history"]}


class PerturbativeTriples:
    """The cc4s ``PerturbativeTriples`` / ``PerturbativeTriplesReference`` step.

    ``arguments`` holds the reference's input keys (PerturbativeTriples.cxx:27-255,
    PerturbativeTriplesReference.cxx:56-222): amplitudes ({'ph': T1,
    'pphh': T2}), slicedEigenEnergies, slicedCoulombVertex or coulombVertex
    (the integral slices are formed on the device, so coulombIntegrals is not
    needed), halfGrid; plus precision ('fp64' or 'split3'), blockSize and
    referenceForm (the complex-path conjugation of PerturbativeTriplesReference;
    the pipeline sets it for that step name), cT (that step's completely
    renormalised branch, PerturbativeTriplesReference.cxx:70-71; 0 or 1), and optionally mp2PairEnergies
    (the complete-basis-set estimates of the MP2 pair energies, any shape).
    Returns {'energy': {'correlation', 'unit'}} like the reference, with
    'starCorrection' = (sum of mp2PairEnergies) / E_MP2 * correlation when
    mp2PairEnergies is given (the (T*) correction, PerturbativeTriplesStar.hpp:34-108,
    E_MP2 the second-order energy of the integrals, computed on the device).
    """

    def __init__(self, lib=None):
        self.lib = lib

    def run(self, arguments):
        eps = arguments["slicedEigenEnergies"]
        gamma = _full_vertex(arguments)
        half_grid = bool(arguments.get("halfGrid", not np.iscomplexobj(gamma)))
        amps = arguments["amplitudes"]
        s = Solver(arguments, lib=self.lib)
        try:
            s.set_inputs(eps["h"], eps["p"], gamma, half_grid=half_grid)
            s.set_initial_amplitudes(amps["ph"], amps["pphh"])
            r = s.perturbative_triples(int(arguments.get("blockSize", 0) or 0),
                                       reference_form=bool(arguments.get("referenceForm", False)),
                                       cT=int(arguments.get("cT", 0) or 0) == 1)
        finally:
            s.close()
        energy = {"correlation": r["correlation"], "unit": 1.0}
        if arguments.get("mp2PairEnergies") is not None:
            cbs = float(np.real(np.sum(np.asarray(arguments["mp2PairEnergies"]))))
            energy["starCorrection"] = cbs / r["mp2_energy"] * r["correlation"]
        return {"energy": energy, "stats": r}


class FiniteSizeCorrection:
    """The cc4s ``FiniteSizeCorrection`` step (FiniteSizeCorrection.cxx:28-310).

    ``arguments``: amplitudes ({'ph', 'pphh'}), slicedEigenEnergies,
    slicedCoulombVertex or coulombVertex, halfGrid, coulombVertexSingularVectors
    (U [G, F]; optional here, identity if absent), coulombPotential (V [G];
    optional, 1), gridVectors ([G, 3] cartesian), reciprocalBasis ([3, 3], the
    rows Gi, Gj, Gk of the gridVectors metaData), interpolationGridSize (20),
    unitFactor (1).  Returns {'energy': {correction, uncorrected, corrected,
    unit}, 'transitionStructureFactor': S(G)}.
    """

    def __init__(self, lib=None):
        self.lib = lib

    def run(self, arguments):
        eps = arguments["slicedEigenEnergies"]
        gamma = _full_vertex(arguments)
        half_grid = bool(arguments.get("halfGrid", not np.iscomplexobj(gamma)))
        amps = arguments["amplitudes"]
        s = Solver(arguments, lib=self.lib)
        try:
            s.set_inputs(eps["h"], eps["p"], gamma, half_grid=half_grid)
            s.set_initial_amplitudes(amps["ph"], amps["pphh"])
            e, S = s.finite_size_correction(
                arguments["gridVectors"], arguments["reciprocalBasis"],
                arguments.get("coulombVertexSingularVectors"), arguments.get("coulombPotential"),
                int(arguments.get("interpolationGridSize", 20)),
                float(arguments.get("unitFactor", 1.0)))
        finally:
            s.close()
        return {"energy": {"correction": e["correction"], "uncorrected": e["uncorrected"],
                           "corrected": e["corrected"], "unit": 1.0},
                "transitionStructureFactor": S, "stats": e}
