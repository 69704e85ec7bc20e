"""cc4s tensor files (cc4s_b200.tensor_io) and the CoupledCluster input chain
(cc4s_b200.pipeline) on the CPU emulation of the device operations."""
import os
import sys
import warnings

import numpy as np
import pytest

from oracle import coupled_cluster, inputs

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))
warnings.simplefilter("ignore")


@pytest.fixture(scope="module")
def emu_lib():
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


@pytest.mark.parametrize("half_grid,binary", [(True, True), (False, False)])
def test_input_chain_runs_coupled_cluster(tmp_path, emu_lib, half_grid, binary):
    """Read -> DefineHolesAndParticles -> SliceOperator -> VertexCoulombIntegrals ->
    CoupledCluster -> Write, from files in the reference's tensor format; the energy
    equals the oracle's on the same inputs (real half-grid path and complex path)."""
    import yaml
    from cc4s_b200 import pipeline
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
        pipeline.run_steps([{"name": "PerturbativeTriples", "in": {}, "out": {}}], str(tmp_path))
