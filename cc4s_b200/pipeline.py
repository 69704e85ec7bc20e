"""Runs the steps of a cc4s input file that lead to and include CoupledCluster.

A cc4s input is a YAML list of steps ``{name, in, out}`` evaluated in order
(src/main/Cc4s.cxx:131-150).  This runner restates the steps of the
CoupledCluster input chain (e.g. test/tests/h2o/dz/cc4s.in):

* ``Read``: a cc4s tensor file (cc4s_b200.tensor_io; TensorIo.cxx);
* ``DefineHolesAndParticles``: the eigen energies below ``metaData.fermiEnergy``
  are holes, the rest particles (DefineHolesAndParticles.cxx:42-95);
* ``SliceOperator``: every dimension of type ``State`` is cut into its hole
  (first No) and particle (last Nv) parts, giving the slices "hh", "hp", ...
  (SliceOperator.cxx:95-131);
* ``VertexCoulombIntegrals``: recorded only; the integrals are formed on the
  device from the vertex slices by the CoupledCluster step;
* ``CoupledCluster``: the B200 step (cc4s_b200.CoupledCluster);
* ``PerturbativeTriples`` / ``PerturbativeTriplesReference``: the B200 (T)
  step (cc4s_b200.PerturbativeTriples) on the amplitudes of a CoupledCluster
  step (e.g. test/tests/h2o/dz/cc4s.in:49-55);
* ``FiniteSizeCorrection``: the B200 structure factor and interpolation
  (cc4s_b200.FiniteSizeCorrection); gridVectors is a [3, NG] tensor whose
  metaData holds the reciprocal basis Gi, Gj, Gk (FiniteSizeCorrection.cxx:143-183);
* ``Write``: a tensor to a cc4s tensor file, anything else to YAML.

Any other step name raises ValueError: it is not part of this library.
"""
from __future__ import annotations

import os

import numpy as np
import yaml

from . import tensor_io
from .coupled_cluster import CoupledCluster, FiniteSizeCorrection, PerturbativeTriples


def _define_holes_and_particles(eps):
    md = eps.meta_data or {}
    energies = md.get("energies")
    if isinstance(energies, dict):
        energies = [energies[k] for k in sorted(energies, key=int)]
    fermi = md.get("fermiEnergy")
    if energies is None or fermi is None:
        raise ValueError("DefineHolesAndParticles: eigen energies need metaData.energies and "
                         "metaData.fermiEnergy")
    No = 0
    while No < len(energies) and float(energies[No]) < float(fermi):
        No += 1
    if No == 0:
        raise ValueError("Fermi energy below all eigen energies.")
    if No >= len(energies):
        raise ValueError("Fermi energy above all eigen energies.")
    vals = np.asarray(eps.values).reshape(-1)
    mk = lambda v: tensor_io.Tensor(values=v, dimension_types=list(eps.dimension_types),
                                    unit=eps.unit, meta_data=md)
    return {"h": mk(vals[:No].copy()), "p": mk(vals[No:].copy())}


def _slice_operator(op, sliced_eps):
    No = sliced_eps["h"].values.size
    Nv = sliced_eps["p"].values.size
    dims = [d for d, t in enumerate(op.dimension_types) if t == "State"]
    out = {}

    def rec(parts):
        if len(parts) < len(dims):
            rec(parts + "h")
            rec(parts + "p")
            return
        idx = [slice(None)] * op.values.ndim
        for k, d in enumerate(dims):
            n = op.values.shape[d]
            idx[d] = slice(0, No) if parts[k] == "h" else slice(n - Nv, n)
        out[parts] = tensor_io.Tensor(values=np.ascontiguousarray(op.values[tuple(idx)]),
                                      dimension_types=list(op.dimension_types), unit=op.unit,
                                      meta_data=op.meta_data)
    rec("")
    return out


def run_steps(steps, workdir=".", lib=None, symbols=None):
    """Evaluates the steps in order; returns the symbol table."""
    sym = {} if symbols is None else symbols

    def arg(a, key, default=None):
        v = a.get(key, default)
        return sym.get(v, v) if isinstance(v, str) else v

    for step in steps:
        name = step.get("name")
        a = step.get("in") or {}
        out = step.get("out") or {}
        if name == "Read":
            sym[out["destination"]] = tensor_io.read(os.path.join(workdir, a["fileName"]))
        elif name == "DefineHolesAndParticles":
            sym[out["slicedEigenEnergies"]] = _define_holes_and_particles(arg(a, "eigenEnergies"))
        elif name == "SliceOperator":
            sym[out["slicedOperator"]] = _slice_operator(arg(a, "operator"),
                                                          arg(a, "slicedEigenEnergies"))
        elif name == "VertexCoulombIntegrals":
            sym[out["coulombIntegrals"]] = {"slicedCoulombVertex": arg(a, "slicedCoulombVertex")}
        elif name == "CoupledCluster":
            eps = arg(a, "slicedEigenEnergies")
            vertex = arg(a, "slicedCoulombVertex")
            if vertex is None:
                vertex = (arg(a, "coulombIntegrals") or {}).get("slicedCoulombVertex")
            md = vertex["hh"].meta_data or {}
            args = {k: v for k, v in a.items()
                    if k not in ("slicedEigenEnergies", "slicedCoulombVertex", "coulombIntegrals",
                                 "initialAmplitudes")}
            args["slicedEigenEnergies"] = {"h": eps["h"].values, "p": eps["p"].values}
            args["slicedCoulombVertex"] = {k: t.values for k, t in vertex.items()}
            args["halfGrid"] = bool(int(md.get("halfGrid", 0)))
            init = arg(a, "initialAmplitudes")
            if init is not None:
                args["initialAmplitudes"] = {k: getattr(t, "values", t) for k, t in init.items()}
            res = CoupledCluster(lib=lib).run(args)
            if "energy" in out:
                sym[out["energy"]] = res["energy"]
            if "amplitudes" in out:
                sym[out["amplitudes"]] = {
                    k: tensor_io.Tensor(values=v, dimension_types=["State"] * v.ndim)
                    for k, v in res["amplitudes"].items()}
            if "convergenceReached" in out:
                sym[out["convergenceReached"]] = res["convergenceReached"]
        elif name in ("PerturbativeTriples", "PerturbativeTriplesReference"):
            eps = arg(a, "slicedEigenEnergies")
            vertex = arg(a, "slicedCoulombVertex")
            if vertex is None:
                vertex = (arg(a, "coulombIntegrals") or {}).get("slicedCoulombVertex")
            if vertex is None:
                raise ValueError("%s: the integrals must come from a VertexCoulombIntegrals "
                                 "step (the vertex is needed on the device)" % name)
            md = vertex["hh"].meta_data or {}
            amps = arg(a, "amplitudes")
            pairs = arg(a, "mp2PairEnergies") if "mp2PairEnergies" in a else None
            res = PerturbativeTriples(lib=lib).run({
                "slicedEigenEnergies": {"h": eps["h"].values, "p": eps["p"].values},
                "slicedCoulombVertex": {k: t.values for k, t in vertex.items()},
                "halfGrid": bool(int(md.get("halfGrid", 0))),
                "amplitudes": {k: getattr(t, "values", t) for k, t in amps.items()},
                "precision": a.get("precision", "fp64"),
                "blockSize": a.get("blockSize", 0),
                "referenceForm": name == "PerturbativeTriplesReference",
                "cT": int(a.get("cT", 0) or 0) if name == "PerturbativeTriplesReference" else 0,
                "mp2PairEnergies": getattr(pairs, "values", pairs)})
            sym[out.get("energy", name + "Energy")] = res["energy"]
        elif name == "FiniteSizeCorrection":
            eps = arg(a, "slicedEigenEnergies")
            vertex = arg(a, "slicedCoulombVertex")
            md = vertex["hh"].meta_data or {}
            amps = arg(a, "amplitudes")
            grid = arg(a, "gridVectors")
            gmd = grid.meta_data or {}
            basis = np.array([[float(x) for x in gmd[k]] for k in ("Gi", "Gj", "Gk")])
            U = arg(a, "coulombVertexSingularVectors")
            V = arg(a, "coulombPotential")
            res = FiniteSizeCorrection(lib=lib).run({
                "slicedEigenEnergies": {"h": eps["h"].values, "p": eps["p"].values},
                "slicedCoulombVertex": {k: t.values for k, t in vertex.items()},
                "halfGrid": bool(int(md.get("halfGrid", 0))),
                "amplitudes": {k: getattr(t, "values", t) for k, t in amps.items()},
                "gridVectors": np.asarray(grid.values).T, "reciprocalBasis": basis,
                "coulombVertexSingularVectors": None if U is None else U.values,
                "coulombPotential": None if V is None else V.values,
                "interpolationGridSize": int(a.get("interpolationGridSize", 20))})
            sym[out.get("energy", "FiniteSizeEnergy")] = res["energy"]
            if "transitionStructureFactor" in out:
                sym[out["transitionStructureFactor"]] = tensor_io.Tensor(
                    values=res["transitionStructureFactor"], dimension_types=["Momentum"])
        elif name == "Write":
            src = arg(a, "source")
            path = os.path.join(workdir, a.get("fileName", "%s.yaml" % a.get("source")))
            if isinstance(src, tensor_io.Tensor):
                tensor_io.write(path, src, binary=bool(a.get("binary", True)))
            else:
                with open(path, "w") as f:
                    yaml.safe_dump(_plain(src), f, sort_keys=False)
        else:
            raise ValueError("step %r is not part of the CoupledCluster input chain this "
                             "library runs" % name)
    return sym


def _plain(x):
    if isinstance(x, dict):
        return {k: _plain(v) for k, v in x.items()}
    if isinstance(x, (np.floating, np.integer)):
        return x.item()
    if isinstance(x, np.ndarray):
        return x.tolist()
    return x


def run_file(path, lib=None):
    """Runs a cc4s input file (YAML list of steps) relative to its directory."""
    with open(path) as f:
        steps = yaml.safe_load(f)
    return run_steps(steps, workdir=os.path.dirname(os.path.abspath(path)), lib=lib)
