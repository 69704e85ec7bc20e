"""cc4s tensor files (cc4s_b200.tensor_io) and the CoupledCluster input chain
(cc4s_b200.pipeline): every chain test runs on the CPU emulation of the device
operations and, marked gpu, on the CUDA library itself (the c0 system there)."""
import os
import sys
import warnings

import numpy as np
import pytest

from oracle import coupled_cluster, inputs

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))
warnings.simplefilter("ignore")


@pytest.fixture(scope="module", params=["emulated", pytest.param("device", marks=pytest.mark.gpu)])
def emu_lib(request):
    """The library the chain calls: the CPU emulation build, or (gpu) None, i.e.
    the in-tree CUDA library."""
    if request.param == "device":
        return None
    import build_emu
    return build_emu.build()


@pytest.mark.parametrize("binary", [True, False])
@pytest.mark.parametrize("cplx", [False, True])
def test_tensor_file_round_trip(tmp_path, binary, cplx):
    from cc4s_b200 import tensor_io
    rng = np.random.default_rng(0)
    v = rng.standard_normal((3, 4, 5))
    if cplx:
        v = v + 1j * rng.standard_normal(v.shape)
    t = tensor_io.Tensor(values=v, dimension_types=["AuxiliaryField", "State", "State"],
                         unit=0.5, meta_data={"halfGrid": 1})
    path = tensor_io.write(str(tmp_path / "V.yaml"), t, binary=binary)
    r = tensor_io.read(path)
    assert r.values.dtype == v.dtype and r.values.shape == v.shape
    assert np.array_equal(r.values, v)
    assert r.dimension_types == t.dimension_types and r.unit == 0.5
    assert r.meta_data["halfGrid"] == 1
    # first index fastest on disk
    if binary:
        raw = np.fromfile(str(tmp_path / "V.elements"), dtype=v.dtype)
        assert np.array_equal(raw, v.reshape(-1, order="F"))


def _write_system(tmp_path, s, half_grid, binary):
    from cc4s_b200 import tensor_io
    eps = np.concatenate([s.eps_h, s.eps_p])
    fermi = 0.5 * (s.eps_h.max() + s.eps_p.min())
    tensor_io.write(str(tmp_path / "EigenEnergies.yaml"),
                    tensor_io.Tensor(values=eps, dimension_types=["State"],
                                     meta_data={"fermiEnergy": float(fermi),
                                                "energies": [float(e) for e in eps]}),
                    binary=binary)
    g = np.asarray(s.gamma, dtype=np.complex128)
    tensor_io.write(str(tmp_path / "CoulombVertex.yaml"),
                    tensor_io.Tensor(values=g, dimension_types=["AuxiliaryField", "State", "State"],
                                     meta_data={"halfGrid": int(half_grid)}),
                    binary=binary)


STEPS = [
    {"name": "Read", "in": {"fileName": "EigenEnergies.yaml"}, "out": {"destination": "EigenEnergies"}},
    {"name": "Read", "in": {"fileName": "CoulombVertex.yaml"}, "out": {"destination": "CoulombVertex"}},
    {"name": "DefineHolesAndParticles", "in": {"eigenEnergies": "EigenEnergies"},
     "out": {"slicedEigenEnergies": "EigenEnergies"}},
    {"name": "SliceOperator", "in": {"slicedEigenEnergies": "EigenEnergies", "operator": "CoulombVertex"},
     "out": {"slicedOperator": "CoulombVertex"}},
    {"name": "VertexCoulombIntegrals", "in": {"slicedCoulombVertex": "CoulombVertex"},
     "out": {"coulombIntegrals": "CoulombIntegrals"}},
    {"name": "CoupledCluster",
     "in": {"method": "Ccsd", "slicedEigenEnergies": "EigenEnergies",
            "coulombIntegrals": "CoulombIntegrals", "slicedCoulombVertex": "CoulombVertex",
            "maxIterations": 40, "energyConvergence": 1.0e-10, "amplitudesConvergence": 1.0e-8,
            "mixer": {"type": "DiisMixer", "maxResidua": 4}},
     "out": {"energy": "CcsdEnergy", "amplitudes": "Amplitudes"}},
    {"name": "Write", "in": {"source": "CcsdEnergy", "fileName": "CcsdEnergy.yaml"}, "out": {}},
]


@pytest.mark.parametrize("half_grid,binary", [(True, True), (False, False), (True, False),
                                             (False, True)])
def test_input_chain_runs_coupled_cluster(tmp_path, emu_lib, half_grid, binary):
    """Read -> DefineHolesAndParticles -> SliceOperator -> VertexCoulombIntegrals ->
    CoupledCluster -> Write, from files in the reference's tensor format; the energy
    equals the oracle's on the same inputs (real half-grid path and complex path)."""
    import yaml
    from cc4s_b200 import pipeline
    if emu_lib is None:   # the device library: the c0 system (No=8, Nv=40, NG=200)
        c = inputs.CONFIGS["c0"]
        s = inputs.synthetic_system(c["No"], c["Nv"], c["NG"], complex=not half_grid, seed=0)
    else:
        s = inputs.synthetic_system(4, 12, 20, complex=not half_grid, seed=6)
    _write_system(tmp_path, s, half_grid, binary)
    with open(tmp_path / "cc4s.in", "w") as f:
        yaml.safe_dump(STEPS, f, sort_keys=False)
    sym = pipeline.run_file(str(tmp_path / "cc4s.in"), lib=emu_lib)
    ref = coupled_cluster.run(s, maxIterations=40, energyConvergence=1e-10,
                              amplitudesConvergence=1e-8,
                              mixer=dict(type="DiisMixer", maxResidua=4))
    assert abs(sym["CcsdEnergy"]["correlation"] - ref["energy"]["correlation"]) < 1e-10
    T2 = sym["Amplitudes"]["pphh"].values
    assert np.abs(T2 - ref["amplitudes"][1]).max() < 1e-9 * np.abs(ref["amplitudes"][1]).max()
    written = yaml.safe_load(open(tmp_path / "CcsdEnergy.yaml"))
    assert abs(written["correlation"] - ref["energy"]["correlation"]) < 1e-10


def test_unknown_step_is_rejected(tmp_path):
    from cc4s_b200 import pipeline
    with pytest.raises(ValueError, match="not part of"):
        pipeline.run_steps([{"name": "UegVertexGenerator", "in": {}, "out": {}}], str(tmp_path))


def test_input_chain_runs_perturbative_triples(tmp_path, emu_lib):
    """... -> CoupledCluster -> PerturbativeTriples (test/tests/h2o/dz/cc4s.in:32-55):
    the (T) energy on the chain's CCSD amplitudes equals the oracle's."""
    import yaml
    from cc4s_b200 import pipeline
    from oracle import triples
    s = inputs.synthetic_system(3, 9, 20, seed=2)
    _write_system(tmp_path, s, True, True)
    steps = STEPS[:-1] + [
        {"name": "PerturbativeTriples",
         "in": {"coulombIntegrals": "CoulombIntegrals", "amplitudes": "Amplitudes",
                "slicedEigenEnergies": "EigenEnergies"},
         "out": {"energy": "TriplesEnergy"}}]
    with open(tmp_path / "cc4s.in", "w") as f:
        yaml.safe_dump(steps, f, sort_keys=False)
    sym = pipeline.run_file(str(tmp_path / "cc4s.in"), lib=emu_lib)
    ref = coupled_cluster.run(s, maxIterations=40, energyConvergence=1e-10,
                              amplitudesConvergence=1e-8,
                              mixer=dict(type="DiisMixer", maxResidua=4))
    T1, T2 = ref["amplitudes"]
    e = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    assert abs(sym["TriplesEnergy"]["correlation"] - e) < 1e-9 * max(1.0, abs(e))


def test_input_chain_runs_finite_size_correction(tmp_path, emu_lib):
    """... -> CoupledCluster -> FiniteSizeCorrection with grid vectors, Coulomb
    potential and singular vectors read from tensor files: S(G) and the energies
    equal the oracle's on the chain's CCSD amplitudes."""
    import yaml
    from cc4s_b200 import pipeline, tensor_io
    from oracle import fsc
    No, Nv, NF = 2, 6, 10
    s = inputs.synthetic_system(No, Nv, NF, seed=8)
    _write_system(tmp_path, s, True, True)
    rng = np.random.default_rng(3)
    B = 2 * np.pi / 4.0 * np.eye(3)
    r = np.arange(4) - 2
    grid = np.array([(a, b, c) for c in r for b in r for a in r], dtype=float) @ B
    NGG = grid.shape[0]
    U = (rng.standard_normal((NGG, NF)) + 1j * rng.standard_normal((NGG, NF))) / 4
    V = 0.5 + rng.random(NGG)
    tensor_io.write(str(tmp_path / "GridVectors.yaml"), tensor_io.Tensor(
        values=grid.T.copy(), dimension_types=["Vector", "Momentum"],
        meta_data={"Gi": B[0].tolist(), "Gj": B[1].tolist(), "Gk": B[2].tolist()}))
    tensor_io.write(str(tmp_path / "CoulombPotential.yaml"),
                    tensor_io.Tensor(values=V, dimension_types=["Momentum"]))
    tensor_io.write(str(tmp_path / "CoulombVertexSingularVectors.yaml"),
                    tensor_io.Tensor(values=U, dimension_types=["Momentum", "AuxiliaryField"]))
    steps = STEPS[:-1] + [
        {"name": "Read", "in": {"fileName": f + ".yaml"}, "out": {"destination": f}}
        for f in ("GridVectors", "CoulombPotential", "CoulombVertexSingularVectors")] + [
        {"name": "FiniteSizeCorrection",
         "in": {"amplitudes": "Amplitudes", "slicedCoulombVertex": "CoulombVertex",
                "slicedEigenEnergies": "EigenEnergies", "gridVectors": "GridVectors",
                "coulombPotential": "CoulombPotential",
                "coulombVertexSingularVectors": "CoulombVertexSingularVectors",
                "interpolationGridSize": 2},
         "out": {"energy": "FscEnergy", "transitionStructureFactor": "SofG"}}]
    with open(tmp_path / "cc4s.in", "w") as f:
        yaml.safe_dump(steps, f, sort_keys=False)
    sym = pipeline.run_file(str(tmp_path / "cc4s.in"), lib=emu_lib)
    ref = coupled_cluster.run(s, maxIterations=40, energyConvergence=1e-10,
                              amplitudesConvergence=1e-8,
                              mixer=dict(type="DiisMixer", maxResidua=4))
    T1, T2 = ref["amplitudes"]
    g = np.asarray(s.gamma)
    S_ref = fsc.transition_structure_factor(T1, T2, g[:, No:, :No], g[:, :No, No:], U, V)
    E_ref = fsc.interpolation(S_ref, grid, B, N=2)
    S = sym["SofG"].values
    assert np.abs(S - S_ref).max() < 1e-8 * np.abs(S_ref).max()
    assert abs(sym["FscEnergy"]["correction"] - E_ref["correction"]) < 1e-8 * abs(E_ref["corrected"])


def test_tensor_file_rejections(tmp_path):
    """TensorIo header checks (TensorIo.cxx:142-247): version, scalar type,
    block-sparse files, element count, elements type."""
    import yaml
    from cc4s_b200 import tensor_io
    base = {"type": "Tensor", "scalarType": "Real64", "version": 100,
            "dimensions": {0: {"length": 3, "type": "State"}},
            "elements": {"type": "TextFile"}, "unit": 1.0}
    (tmp_path / "T.elements").write_text("1\n2\n3\n")

    def write_header(h):
        with open(tmp_path / "T.yaml", "w") as f:
            yaml.safe_dump(h, f)

    write_header(base)
    assert np.array_equal(tensor_io.read(str(tmp_path / "T.yaml")).values, [1.0, 2.0, 3.0])
    for bad, msg in [(dict(base, version=99), "version"), (dict(base, scalarType="Real32"), "scalarType"),
                     (dict(base, nonZeroCondition={"all": []}), "block-sparse"),
                     (dict(base, elements={"type": "Hdf5"}), "elements type"),
                     (dict(base, dimensions={0: {"length": 4}}), "elements, expecting")]:
        write_header(bad)
        with pytest.raises(ValueError, match=msg):
            tensor_io.read(str(tmp_path / "T.yaml"))


def test_tensor_file_text_complex(tmp_path):
    """Complex text elements are (re,im) per line, first index fastest."""
    from cc4s_b200 import tensor_io
    v = np.array([[1 + 2j, 3 - 1j], [0.5j, -2.0]])
    tensor_io.write(str(tmp_path / "C.yaml"), tensor_io.Tensor(values=v), binary=False)
    lines = (tmp_path / "C.elements").read_text().split()
    assert lines[0] == "(1,2)" and lines[1] == "(0,0.5)"   # column-major: v[0,0], v[1,0]
    assert np.array_equal(tensor_io.read(str(tmp_path / "C.yaml")).values, v)


@pytest.mark.parametrize("step", ["PerturbativeTriples", "PerturbativeTriplesReference"])
def test_input_chain_complex_triples_step_names(tmp_path, emu_lib, step):
    """Complex chain: the step name selects the conjugation of the (T) energy
    (atrip's Re conj(W) Z or the array form's Re conj(W) conj(Z))."""
    import yaml
    from cc4s_b200 import pipeline
    from oracle import triples
    s = inputs.synthetic_system(2, 6, 12, complex=True, seed=5)
    _write_system(tmp_path, s, False, True)
    steps = STEPS[:-1] + [
        {"name": step,
         "in": {"coulombIntegrals": "CoulombIntegrals", "amplitudes": "Amplitudes",
                "slicedEigenEnergies": "EigenEnergies"},
         "out": {"energy": "TriplesEnergy"}}]
    with open(tmp_path / "cc4s.in", "w") as f:
        yaml.safe_dump(steps, f, sort_keys=False)
    sym = pipeline.run_file(str(tmp_path / "cc4s.in"), lib=emu_lib)
    T1 = sym["Amplitudes"]["ph"].values
    T2 = sym["Amplitudes"]["pphh"].values
    V = triples.triples_integrals(s)
    f = triples.triples_reference if step.endswith("Reference") else triples.triples_atrip
    e = f(T1, T2, V, s.eps_h, s.eps_p)
    assert abs(sym["TriplesEnergy"]["correlation"] - e) < 1e-11 * max(1.0, abs(e))


@pytest.mark.parametrize("half_grid", [True, False])
def test_input_chain_triples_reference_with_cT(tmp_path, emu_lib, half_grid):
    """The (T) step of test/tests/hf/cc4s.in:49-56: PerturbativeTriplesReference with
    cT: 1 after the CCSD step; the energy is the completely renormalised one
    (CompleteTriples.cxx:11-118), against the oracle on the chain's amplitudes."""
    import yaml
    from cc4s_b200 import pipeline
    from oracle import triples
    s = inputs.synthetic_system(2, 6, 12, complex=not half_grid, seed=5)
    _write_system(tmp_path, s, half_grid, True)
    steps = STEPS[:-1] + [
        {"name": "PerturbativeTriplesReference",
         "in": {"coulombIntegrals": "CoulombIntegrals", "cT": 1, "amplitudes": "Amplitudes",
                "slicedEigenEnergies": "EigenEnergies"},
         "out": {"energy": "TriplesEnergy"}}]
    with open(tmp_path / "cc4s.in", "w") as f:
        yaml.safe_dump(steps, f, sort_keys=False)
    sym = pipeline.run_file(str(tmp_path / "cc4s.in"), lib=emu_lib)
    T1 = sym["Amplitudes"]["ph"].values
    T2 = sym["Amplitudes"]["pphh"].values
    J = triples.complete_triples_intermediates(s, T1, T2)
    e = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p,
                                  complete=J)
    assert abs(sym["TriplesEnergy"]["correlation"] - e) < 1e-11 * max(1.0, abs(e))
