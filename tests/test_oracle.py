"""The CPU oracle against the reference's own expected output and against
independent formulations (CPU only)."""
import json
import os
import warnings

import numpy as np
import pytest

from oracle import ccsd, ccsd_reference, coupled_cluster, inputs, mixers, properties, triples

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
warnings.simplefilter("ignore")


def _rand_T(rng, Nv, No, cplx=False, scale=0.01):
    T1 = rng.standard_normal((Nv, No)) * scale
    T2 = rng.standard_normal((Nv, Nv, No, No)) * scale
    if cplx:
        T1 = T1 + 1j * rng.standard_normal((Nv, No)) * scale
        T2 = T2 + 1j * rng.standard_normal((Nv, Nv, No, No)) * scale
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    return T1, T2


def test_ueg_pinned_to_reference_expected_output():
    """Restated UEG vertex + complex CCSD reproduce cc4s's own expected energies."""
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    r = coupled_cluster.run(s, **g["ccsd"]["options"])
    assert r["convergenceReached"]
    for k, ref in g["ccsd"]["energy"].items():
        assert abs(r["energy"][k] - ref) < 1e-10, (k, r["energy"][k], ref)


def test_ueg_drccd_pinned_to_reference_expected_output():
    """Restated Drccd reproduces the reference's expected UEG Drccd energies."""
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    r = coupled_cluster.run(s, **g["drccd"]["options"])
    assert r["convergenceReached"]
    for k, ref in g["drccd"]["energy"].items():
        assert abs(r["energy"][k] - ref) < 1e-10, (k, r["energy"][k], ref)


def test_ueg_mp2_matches_second_order():
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    e, d, x = properties.mp2(s)
    assert abs(e - g["ccsd"]["energy"]["secondOrder"]) < 1e-12


@pytest.mark.parametrize("slice_size", [None, 3, 7, 40])
def test_real_ccsd_equals_textbook(slice_size):
    s = inputs.config_system("c0", seed=1)
    rng = np.random.default_rng(5)
    T = _rand_T(rng, s.Nv, s.No)
    R1, R2 = ccsd.residuum(T, ccsd.CcsdInputs(s), slice_size=slice_size)
    Q1, Q2 = ccsd_reference.residuum(T, ccsd_reference.ReferenceInputs(s))
    assert np.abs(R1 - Q1).max() < 1e-12 * np.abs(Q1).max()
    assert np.abs(R2 - Q2).max() < 1e-12 * np.abs(Q2).max()


def test_complex_ccsd_equals_textbook():
    s = inputs.synthetic_system(6, 20, 50, complex=True, seed=3)
    rng = np.random.default_rng(7)
    T = _rand_T(rng, 20, 6, cplx=True)
    R1, R2 = ccsd.residuum(T, ccsd.CcsdInputs(s), slice_size=7)
    Q1, Q2 = ccsd_reference.residuum(T, ccsd_reference.ReferenceInputs(s))
    assert np.abs(R1 - Q1).max() < 1e-12 * np.abs(Q1).max()
    assert np.abs(R2 - Q2).max() < 1e-12 * np.abs(Q2).max()


def test_residual_pair_symmetry():
    s = inputs.config_system("c0", seed=2)
    rng = np.random.default_rng(1)
    T = _rand_T(rng, s.Nv, s.No)
    R1, R2 = ccsd.residuum(T, ccsd.CcsdInputs(s))
    assert np.abs(R2 - R2.transpose(1, 0, 3, 2)).max() < 1e-14 * np.abs(R2).max()


def test_first_iteration_is_mp2():
    s = inputs.config_system("c0", seed=0)
    r = coupled_cluster.run(s, maxIterations=1)
    assert abs(r["energy"]["secondOrder"] - properties.mp2(s)[0]) < 1e-12


def test_structure_factor_sums_to_energy():
    s = inputs.synthetic_system(4, 12, 30, seed=4)
    r = coupled_cluster.run(s, maxIterations=40, energyConvergence=1e-10)
    S = properties.structure_factor(s, r["amplitudes"])
    assert abs(S.sum() - r["energy"]["correlation"]) < 1e-12


def test_ccd_has_no_singles():
    s = inputs.synthetic_system(4, 12, 30, seed=4)
    r = coupled_cluster.run(s, method="Ccd", maxIterations=30, energyConvergence=1e-10)
    assert np.abs(r["amplitudes"][0]).max() == 0.0
    assert r["convergenceReached"]


def test_c0_golden_trajectory():
    g = json.load(open(os.path.join(GOLDEN, "c0_seed0.json")))
    s = inputs.config_system("c0", seed=g["seed"])
    r = coupled_cluster.run(s, **g["options"])
    assert r["iterations"] == g["iterations"]
    for h, e in zip(r["history"], g["history_energy"]):
        assert abs(h["energy"] - e) < 1e-11
    assert abs(r["energy"]["correlation"] - g["energy"]["correlation"]) < 1e-11


def test_diis_two_vectors():
    """Bordered 2x2 DIIS: coefficients (c1, c2) minimise |c1 r1 + c2 r2|, sum c = 1."""
    m = mixers.DiisMixer(4)
    r1 = (np.array([1.0, 0.0]), np.zeros((1,)))
    r2 = (np.array([0.0, 2.0]), np.zeros((1,)))
    a1 = (np.array([10.0, 0.0]), np.zeros((1,)))
    a2 = (np.array([0.0, 10.0]), np.zeros((1,)))
    m.append(a1, r1)
    m.append(a2, r2)
    # minimiser of c1^2 + 4 c2^2 with c1 + c2 = 1: c1 = 0.8, c2 = 0.2
    T = m.get()
    assert np.allclose(T[0], [8.0, 2.0])
    assert abs(m.getResiduumNorm() - np.sqrt(0.8 ** 2 + (0.4) ** 2)) < 1e-14


def test_diis_ring_buffer_slot_order():
    rng = np.random.default_rng(3)
    m = mixers.DiisMixer(3)
    vecs = [(rng.standard_normal(5), rng.standard_normal(2)) for _ in range(5)]
    for k in range(5):
        m.append(vecs[k], vecs[k])
    # after 5 appends the ring holds appends 3, 4, 2 in slots 0, 1, 2
    assert m.count == 3 and m.nextIndex == 2
    assert m.amplitudes[0] is vecs[3] and m.amplitudes[1] is vecs[4] and m.amplitudes[2] is vecs[2]


def test_linear_mixer():
    m = mixers.LinearMixer(0.5)
    m.append((np.ones(2), np.ones(1)), (np.ones(2), np.ones(1)))
    m.append((3 * np.ones(2), np.ones(1)), (np.zeros(2), np.zeros(1)))
    assert np.allclose(m.get()[0], 2.0)
    assert abs(m.getResiduumNorm() - np.sqrt(0.75)) < 1e-15


def test_ueg_triples_pinned_to_reference_expected_output():
    """Both (T) restatements, at the restated CCSD amplitudes of the UEG test,
    reproduce the reference's expected PerturbativeTriplesReference energy
    (complex path)."""
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    r = coupled_cluster.run(s, **g["ccsd"]["options"])
    T1, T2 = r["amplitudes"]
    V = triples.triples_integrals(s)
    ref = g["triples"]["energy"]["correlation"]
    e_ctf = triples.triples_reference(T1, T2, V, s.eps_h, s.eps_p)
    e_atrip = triples.triples_atrip(T1, T2, V, s.eps_h, s.eps_p)
    assert abs(e_ctf - ref) < 1e-12, (e_ctf, ref)
    assert abs(e_atrip - ref) < 1e-12, (e_atrip, ref)


@pytest.mark.parametrize("shape", [(3, 8, 12), (4, 11, 20)])
def test_triples_restatements_agree_real(shape):
    """The array form (PerturbativeTriplesReference) and the tuple loop (atrip)
    give the same real-path energy on arbitrary symmetric amplitudes."""
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, seed=Nv)
    rng = np.random.default_rng(No)
    T1, T2 = _rand_T(rng, Nv, No, scale=0.03)
    V = triples.triples_integrals(s)
    a = triples.triples_reference(T1, T2, V, s.eps_h, s.eps_p)
    b = triples.triples_atrip(T1, T2, V, s.eps_h, s.eps_p)
    assert abs(a - b) < 1e-13 * max(1.0, abs(a)), (a, b)


def test_c0_triples_golden():
    """The committed c0 (T) energy (self-made golden) from the converged oracle amplitudes."""
    g = json.load(open(os.path.join(GOLDEN, "c0_seed0.json")))
    s = inputs.config_system("c0", seed=0)
    r = coupled_cluster.run(s, **g["options"])
    T1, T2 = r["amplitudes"]
    e = triples.triples_atrip(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    assert abs(e - g["triples"]["correlation"]) < 1e-10


def test_real_path_equals_pinned_complex_path():
    """The real (half-grid) path pinned through the complex path: for a real
    symmetric vertex the complex path's integrals V_pqsr = sum conj(G_sp) G_qr
    (VertexCoulombIntegrals.cxx:143-190) equal the real path's sum G_ps G_qr, so a
    converged CCSD run on the complex path (pinned to cc4s's expected UEG
    energies by test_ueg_pinned_to_reference_expected_output) and on the real
    path give the same energies and amplitudes."""
    s = inputs.synthetic_system(5, 18, 40, seed=12)
    sc = inputs.System(s.eps_h, s.eps_p, np.asarray(s.gamma, dtype=complex), half_grid=False)
    opts = dict(maxIterations=60, energyConvergence=1e-12, amplitudesConvergence=1e-10,
                mixer=dict(type="DiisMixer", maxResidua=5))
    r = coupled_cluster.run(s, **opts)
    c = coupled_cluster.run(sc, **opts)
    assert r["iterations"] == c["iterations"]
    for k in ("correlation", "direct", "exchange", "secondOrder"):
        assert abs(r["energy"][k] - c["energy"][k]) < 1e-12 * abs(r["energy"][k])
    assert np.abs(r["amplitudes"][1] - c["amplitudes"][1].real).max() < 1e-12
    assert np.abs(c["amplitudes"][1].imag).max() < 1e-14


@pytest.mark.parametrize("cplx", [False, True])
def test_cr_denominator_decomposition(cplx):
    """The CR-(T) denominator restated from ct::getDenominator (CompleteTriples.cxx:
    120-165) equals the form the device evaluates: 1 + 2 sum t t + sum (2T - T^x)(T + t t)
    + sum y conj(Z) / D with Z the energy's 4/3, -2, 2/3 combination of S = W + singles
    (the t-bar and z arrays of the reference sum to conj(Z) / D)."""
    from oracle.triples import es
    s = inputs.synthetic_system(3, 7, 14, complex=cplx, seed=11)
    rng = np.random.default_rng(2)
    T1 = rng.standard_normal((7, 3)) * 0.05
    T2 = rng.standard_normal((7, 7, 3, 3)) * 0.03
    if cplx:
        T1 = T1 + 0.05j * rng.standard_normal((7, 3))
        T2 = T2 + 0.03j * rng.standard_normal((7, 7, 3, 3))
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    V = triples.triples_integrals(s)
    den = triples.cr_triples_denominator(T1, T2, V, s.eps_h, s.eps_p)
    cj = np.conj if cplx else (lambda x: x)
    X = es("bcdk,adij->abcijk", V["ppph"], T2) - es("jklc,abil->abcijk", cj(V["hhhp"]), T2)
    W = sum(es(p + "->abcijk", X) for p in
            ("abcijk", "bacjik", "acbikj", "cbakji", "cabkij", "bcajki"))
    S = W + (es("ai,bcjk->abcijk", T1, V["pphh"]) + es("bj,acik->abcijk", T1, V["pphh"])
             + es("ck,abij->abcijk", T1, V["pphh"]))
    Z = (4 / 3) * S - 2 * es("acbijk->abcijk", S) + (2 / 3) * es("bcaijk->abcijk", S)
    eh, ep = s.eps_h, s.eps_p
    D = (eh[None, None, None, :, None, None] + eh[None, None, None, None, :, None]
         + eh[None, None, None, None, None, :] - ep[:, None, None, None, None, None]
         - ep[None, :, None, None, None, None] - ep[None, None, :, None, None, None])
    y = (es("ai,bj,ck->abcijk", T1, T1, T1) + es("ai,bcjk->abcijk", T1, T2)
         + es("bj,acik->abcijk", T1, T2) + es("ck,abij->abcijk", T1, T2))
    small = np.real(2 * np.sum(T1 * T1) + np.sum((2 * T2 - T2.transpose(1, 0, 2, 3))
                                                  * (T2 + es("ai,bj->abij", T1, T1))))
    assert abs(den - (1 + small + np.sum(np.real(y * np.conj(Z)) / D))) < 1e-13 * abs(den)
