"""Parity of the device (T) energy (cc4s_cc_perturbative_triples) with the
oracle's restatement of PerturbativeTriplesReference on a B200."""
import json
import os
import warnings

import numpy as np
import pytest

from oracle import inputs, triples

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
warnings.simplefilter("ignore")

# FP64: the block sums differ from the oracle's order of summation only by
# rounding (1e-11 relative).  Split form: 28 bits of every operand in the
# particle contractions give ~1e-8 relative in the energy (tolerance 1e-6).
TOL_FP64 = 1e-11
TOL_SPLIT = 1e-6


def _rand_T(rng, Nv, No, scale=0.03):
    T1 = rng.standard_normal((Nv, No)) * scale
    T2 = rng.standard_normal((Nv, Nv, No, No)) * scale
    return T1, T2 + T2.transpose(1, 0, 3, 2)


def _triples(s, T1, T2, block=0, precision="fp64"):
    from cc4s_b200 import Solver
    sol = Solver({"precision": precision})
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        sol.set_initial_amplitudes(T1, T2)
        return sol.perturbative_triples(block)
    finally:
        sol.close()


@pytest.mark.parametrize("shape", [(4, 24, 48), (6, 30, 90), (3, 17, 40)])
@pytest.mark.parametrize("block", [1, 5, 0])
def test_triples_matches_oracle(shape, block):
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, seed=No * Nv)
    rng = np.random.default_rng(NG)
    T1, T2 = _rand_T(rng, Nv, No)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    r = _triples(s, T1, T2, block)
    assert abs(r["correlation"] - ref) < TOL_FP64 * abs(ref), (r["correlation"], ref)


def test_triples_split_precision_matches_oracle():
    s = inputs.synthetic_system(6, 30, 90, seed=5)
    rng = np.random.default_rng(9)
    T1, T2 = _rand_T(rng, 30, 6)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    r = _triples(s, T1, T2, 4, precision="split3")
    assert abs(r["correlation"] - ref) < TOL_SPLIT * abs(ref), (r["correlation"], ref)


def test_triples_block_invariance_and_split_at_size():
    """No=16, Nv=128 (beyond the oracle's array form): every block length and
    the split form give the same energy; the loop covers v^3/6 ordered triples."""
    s = inputs.synthetic_system(16, 128, 256, seed=3)
    rng = np.random.default_rng(4)
    T1, T2 = _rand_T(rng, 128, 16, scale=0.01)
    a = _triples(s, T1, T2, 0)
    b = _triples(s, T1, T2, 9)
    c = _triples(s, T1, T2, 0, precision="split3")
    assert abs(a["correlation"] - b["correlation"]) < TOL_FP64 * abs(a["correlation"])
    assert abs(c["correlation"] - a["correlation"]) < TOL_SPLIT * abs(a["correlation"])
    assert a["flops"] == 2.0 * 16 ** 3 * 128 ** 3 * (16 + 128)
    assert a["seconds"] > 0


def test_c0_triples_golden_after_ccsd():
    """CCSD on the device, then (T) on the handle's amplitudes: the committed
    c0 golden (oracle CCSD + tuple-loop (T))."""
    from cc4s_b200 import Solver
    g = json.load(open(os.path.join(GOLDEN, "c0_seed0.json")))
    s = inputs.config_system("c0", seed=g["seed"])
    sol = Solver(g["options"])
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        r = sol.run()
        assert r["converged"]
        t = sol.perturbative_triples()
    finally:
        sol.close()
    assert abs(t["correlation"] - g["triples"]["correlation"]) < 1e-8, t


def test_perturbative_triples_operator():
    """The operator mirror of the reference step: amplitudes in, energy map out."""
    from cc4s_b200 import PerturbativeTriples
    s = inputs.synthetic_system(4, 24, 48, seed=2)
    rng = np.random.default_rng(1)
    T1, T2 = _rand_T(rng, 24, 4)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    out = PerturbativeTriples().run({
        "slicedEigenEnergies": {"h": s.eps_h, "p": s.eps_p}, "coulombVertex": s.gamma,
        "halfGrid": True, "amplitudes": {"ph": T1, "pphh": T2}})
    assert set(out["energy"]) == {"correlation", "unit"}
    assert abs(out["energy"]["correlation"] - ref) < TOL_FP64 * abs(ref)


@pytest.mark.parametrize("reference_form", [False, True])
def test_triples_complex_matches_oracle(reference_form):
    """Complex path, both conjugations: the atrip tuple loop (formulation 0) and the
    array form of PerturbativeTriplesReference (formulation 1)."""
    from cc4s_b200 import Solver
    No, Nv = 4, 20
    c = inputs.synthetic_system(No, Nv, 40, complex=True, seed=6)
    rng = np.random.default_rng(3)
    T1 = (rng.standard_normal((Nv, No)) + 1j * rng.standard_normal((Nv, No))) * 0.03
    T2 = (rng.standard_normal((Nv, Nv, No, No)) + 1j * rng.standard_normal((Nv, Nv, No, No))) * 0.02
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    V = triples.triples_integrals(c)
    f = triples.triples_reference if reference_form else triples.triples_atrip
    ref = f(T1, T2, V, c.eps_h, c.eps_p)
    sol = Solver({})
    try:
        sol.set_inputs(c.eps_h, c.eps_p, c.gamma, half_grid=False)
        sol.set_initial_amplitudes(T1, T2)
        e = sol.perturbative_triples(3, reference_form=reference_form)["correlation"]
    finally:
        sol.close()
    assert abs(e - ref) < TOL_FP64 * abs(ref), (e, ref)


def test_ueg_triples_after_ccsd_matches_reference_expected_output():
    """The reference's UEG regression test (complex path): CCSD on the device,
    then PerturbativeTriplesReference's (T) on the handle's amplitudes, against
    the expected output in test/tests/ueg/rs1.0-7occ-26virt/correct.out.yaml."""
    from cc4s_b200 import Solver
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    sol = Solver(g["ccsd"]["options"])
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
        r = sol.run()
        assert r["converged"]
        a = sol.perturbative_triples(reference_form=True)["correlation"]
        b = sol.perturbative_triples()["correlation"]
    finally:
        sol.close()
    ref = g["triples"]["energy"]["correlation"]
    assert abs(a - ref) < 1e-9, (a, ref)
    assert abs(b - ref) < 1e-9, (b, ref)


@pytest.mark.parametrize("cplx", [False, True])
def test_triples_star_correction_on_device(cplx):
    """(T*) on the B200: starCorrection = (sum of the CBS pair energies) / E_MP2 *
    E_(T) with the basis MP2 energy reduced on the device, against the oracle's
    restatement of PerturbativeTriplesStar.hpp:34-108 (1e-11 relative)."""
    from cc4s_b200 import PerturbativeTriples
    s = inputs.synthetic_system(6, 30, 90, complex=cplx, seed=3)
    rng = np.random.default_rng(9)
    T1, T2 = _rand_T(rng, 30, 6)
    if cplx:
        T1 = T1 + 1j * _rand_T(rng, 30, 6)[0]
        T2 = T2 + 1j * _rand_T(rng, 30, 6)[1]
    pairs = -0.01 * rng.random((6, 6))
    r = PerturbativeTriples().run({
        "slicedEigenEnergies": {"h": s.eps_h, "p": s.eps_p}, "coulombVertex": s.gamma,
        "halfGrid": not cplx, "amplitudes": {"ph": T1, "pphh": T2}, "mp2PairEnergies": pairs})
    V = inputs.coulomb_integrals(s, ["pphh"])["pphh"]
    star, e_mp2 = triples.triples_star(V, s.eps_h, s.eps_p, pairs, r["energy"]["correlation"])
    assert abs(r["stats"]["mp2_energy"] - e_mp2) < TOL_FP64 * abs(e_mp2)
    assert abs(r["energy"]["starCorrection"] - star) < TOL_FP64 * abs(star)


@pytest.mark.parametrize("cplx,block,precision", [(False, 0, "fp64"), (False, 4, "fp64"),
                                                  (True, 3, "fp64"), (False, 4, "split3")])
def test_triples_complete_matches_oracle(cplx, block, precision):
    """cT = 1 on the B200: the ct::getCompleteTriples intermediates (CompleteTriples.cxx:
    11-118) formed on the device, the second block array M and E = sum M Z
    (PerturbativeTriplesReference.cxx:92-109, :178-179), against the oracle."""
    from cc4s_b200 import Solver
    No, Nv = 4, 20
    s = inputs.synthetic_system(No, Nv, 40, complex=cplx, seed=6)
    rng = np.random.default_rng(3)
    T1, T2 = _rand_T(rng, Nv, No)
    if cplx:
        U1, U2 = _rand_T(rng, Nv, No)
        T1, T2 = T1 + 1j * U1, T2 + 1j * U2
    J = triples.complete_triples_intermediates(s, T1, T2)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p,
                                    complete=J)
    sol = Solver({"precision": precision})
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
        sol.set_initial_amplitudes(T1, T2)
        e = sol.perturbative_triples(block, reference_form=True, cT=True)["correlation"]
    finally:
        sol.close()
    tol = TOL_FP64 if precision == "fp64" else TOL_SPLIT
    assert abs(e - ref) < tol * abs(ref), (e, ref)


@pytest.mark.parametrize("cplx,cT", [(True, False), (False, True)])
def test_triples_split_sliced_operands_match_fp64(cplx, cT):
    """The split form with both operands of the block contractions sliced once per
    evaluation (K = v + o = 66, blocks of 11 with a ragged last block) against the
    device FP64 energy, on the complex path (atrip's conjugation) and for cT = 1."""
    from cc4s_b200 import Solver
    No, Nv = 6, 60
    s = inputs.synthetic_system(No, Nv, 80, complex=cplx, seed=5)
    rng = np.random.default_rng(6)
    T1, T2 = _rand_T(rng, Nv, No, scale=0.01)
    if cplx:
        U1, U2 = _rand_T(rng, Nv, No, scale=0.01)
        T1, T2 = T1 + 1j * U1, T2 + 1j * U2
    e = {}
    for p in ("fp64", "split3"):
        sol = Solver({"precision": p})
        try:
            sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
            sol.set_initial_amplitudes(T1, T2)
            e[p] = sol.perturbative_triples(11, reference_form=cT, cT=cT)["correlation"]
        finally:
            sol.close()
    assert abs(e["split3"] - e["fp64"]) < TOL_SPLIT * abs(e["fp64"]), e
    assert e["split3"] != e["fp64"]  # the split form ran


@pytest.mark.parametrize("cplx", [False, True])
def test_triples_cr_denominator_matches_oracle(cplx):
    """cT = 1: the denominator of the CR-(T) energy the reference prints
    (PerturbativeTriplesReference.cxx:187-195, ct::getDenominator in
    CompleteTriples.cxx:120-165), formed on the device beside the energy."""
    from cc4s_b200 import Solver
    No, Nv = 4, 20
    s = inputs.synthetic_system(No, Nv, 40, complex=cplx, seed=6)
    rng = np.random.default_rng(3)
    T1, T2 = _rand_T(rng, Nv, No)
    if cplx:
        U1, U2 = _rand_T(rng, Nv, No)
        T1, T2 = T1 + 1j * U1, T2 + 1j * U2
    den = triples.cr_triples_denominator(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    sol = Solver({})
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
        sol.set_initial_amplitudes(T1, T2)
        r = sol.perturbative_triples(3, reference_form=True, cT=True)
    finally:
        sol.close()
    assert abs(r["cr_denominator"] - den) < TOL_FP64 * abs(den), (r["cr_denominator"], den)
    assert abs(r["cr_correlation"] - r["correlation"] / den) < TOL_FP64 * abs(r["cr_correlation"])
