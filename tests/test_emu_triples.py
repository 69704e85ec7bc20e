"""The product's (T) schedule (cc4s_b200/csrc/triples.cpp) and its C-ABI entry,
linked against the plain-loop CPU emulation of the device operations
(tests/emu/ops_emu.cpp, test-only) and checked against the oracle's
restatement of PerturbativeTriplesReference.  This pins the strides of the
twelve block contractions, the singles, the hole-permutation weights of every
kind of block triple and the block bookkeeping without a GPU."""
import os
import sys
import warnings

import numpy as np
import pytest

from oracle import inputs, triples

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))
warnings.simplefilter("ignore")


@pytest.fixture(scope="module")
def emu_lib():
    import build_emu
    return build_emu.build()


def _rand_T(rng, Nv, No):
    T1 = rng.standard_normal((Nv, No)) * 0.05
    T2 = rng.standard_normal((Nv, Nv, No, No)) * 0.03
    return T1, T2 + T2.transpose(1, 0, 3, 2)


def _triples(lib, s, T1, T2, block, precision="fp64"):
    from cc4s_b200.coupled_cluster import Solver
    sol = Solver({"precision": precision}, lib=lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        sol.set_initial_amplitudes(T1, T2)
        return sol.perturbative_triples(block)
    finally:
        sol.close()


@pytest.mark.parametrize("shape", [(3, 10, 16), (2, 7, 9), (4, 6, 20)])
@pytest.mark.parametrize("block", [1, 2, 3, 4, 0])
def test_triples_matches_oracle(emu_lib, shape, block):
    """Every block length, ragged last blocks included, gives the oracle's energy."""
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, seed=No + Nv)
    rng = np.random.default_rng(NG)
    T1, T2 = _rand_T(rng, Nv, No)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    r = _triples(emu_lib, s, T1, T2, block)
    assert abs(r["correlation"] - ref) < 1e-12 * max(1.0, abs(ref)), (r["correlation"], ref)
    nb = r["block_size"]
    nbk = -(-Nv // nb)
    assert r["block_triples"] == nbk * (nbk + 1) * (nbk + 2) // 6
    assert r["flops"] == 2.0 * No ** 3 * Nv ** 3 * (No + Nv)
    assert r["executed_flops"] >= r["flops"] * (1 - 1e-12)


def test_triples_split_precision(emu_lib):
    """The split form of the particle contractions stays within 1e-7 of the energy."""
    s = inputs.synthetic_system(3, 10, 80, seed=4)
    rng = np.random.default_rng(8)
    T1, T2 = _rand_T(rng, 10, 3)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    r = _triples(emu_lib, s, T1, T2, 4, precision="split3")
    assert abs(r["correlation"] - ref) < 1e-7 * abs(ref)


def test_triples_requires_amplitudes(emu_lib):
    from cc4s_b200 import _abi
    from cc4s_b200.coupled_cluster import CoupledClusterError, Solver
    s = inputs.synthetic_system(2, 5, 8, seed=1)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        with pytest.raises(CoupledClusterError) as e:
            sol.perturbative_triples()
        assert e.value.status == _abi.ERR_STATE
        sol.set_initial_amplitudes(*_rand_T(np.random.default_rng(0), 5, 2))
        with pytest.raises(CoupledClusterError) as e:
            sol.perturbative_triples(-1)
        assert e.value.status == _abi.ERR_INVALID_ARGUMENT
    finally:
        sol.close()


@pytest.mark.parametrize("block", [1, 3, 0])
def test_triples_complex_both_formulations(emu_lib, block):
    """Complex path: formulation 0 is the atrip tuple loop (Re conj(W) Z),
    formulation 1 the array form of PerturbativeTriplesReference
    (Re conj(W) conj(Z)); on arbitrary complex amplitudes they differ."""
    from cc4s_b200.coupled_cluster import Solver
    No, Nv = 3, 8
    c = inputs.synthetic_system(No, Nv, 14, complex=True, seed=3)
    rng = np.random.default_rng(2)
    T1 = (rng.standard_normal((Nv, No)) + 1j * rng.standard_normal((Nv, No))) * 0.05
    T2 = (rng.standard_normal((Nv, Nv, No, No)) + 1j * rng.standard_normal((Nv, Nv, No, No))) * 0.03
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    V = triples.triples_integrals(c)
    e_atrip = triples.triples_atrip(T1, T2, V, c.eps_h, c.eps_p)
    e_ref = triples.triples_reference(T1, T2, V, c.eps_h, c.eps_p)
    assert abs(e_atrip - e_ref) > 1e-6  # the two conjugations are distinguishable here
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(c.eps_h, c.eps_p, c.gamma, half_grid=False)
        sol.set_initial_amplitudes(T1, T2)
        a = sol.perturbative_triples(block)["correlation"]
        b = sol.perturbative_triples(block, reference_form=True)["correlation"]
    finally:
        sol.close()
    assert abs(a - e_atrip) < 1e-12 * max(1.0, abs(e_atrip)), (a, e_atrip)
    assert abs(b - e_ref) < 1e-12 * max(1.0, abs(e_ref)), (b, e_ref)


def test_block_weights_cover_every_ordering():
    """The hole-permutation weights of a block triple: the blocked sum over
    A <= B <= C equals the full sum for symmetric W, S (checked in numpy with
    the same weights the C++ schedule uses, restated here)."""
    PERMS = [(0, 1, 2), (0, 2, 1), (1, 0, 2), (1, 2, 0), (2, 0, 1), (2, 1, 0)]

    def comp(a, b):
        return tuple(a[b[m]] for m in range(3))

    def inv(a):
        r = [0, 0, 0]
        for m in range(3):
            r[a[m]] = m
        return tuple(r)

    def coefs(blk):
        seen, c = set(), np.zeros(6)
        for sg in PERMS:
            key = tuple(blk[sg[m]] for m in range(3))
            if key in seen:
                continue
            seen.add(key)
            c[0] += 4 / 3
            c[PERMS.index(comp(comp(sg, (0, 2, 1)), inv(sg)))] -= 2
            c[PERMS.index(comp(comp(sg, (2, 0, 1)), inv(sg)))] += 2 / 3
        return c

    assert np.allclose(coefs((0, 1, 2)), [8, -4, -4, 2, 2, -4])
    assert np.allclose(coefs((0, 0, 0)), [4 / 3, -2, 0, 0, 2 / 3, 0])
    # the weights of each kind of triple sum to zero: a fully symmetric S adds nothing
    for blk in [(0, 0, 0), (0, 0, 1), (0, 1, 1), (0, 1, 2)]:
        assert abs(coefs(blk).sum()) < 1e-12


@pytest.mark.parametrize("shape,block", [((1, 4, 6), 0), ((1, 5, 7), 2), ((3, 1, 5), 0),
                                         ((2, 3, 4), 5)])
def test_triples_edge_shapes(emu_lib, shape, block):
    """One hole (all hole permutations coincide), one virtual (every triple has
    a = b = c: the energy vanishes), a block longer than Nv."""
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, seed=7)
    rng = np.random.default_rng(11)
    T1, T2 = _rand_T(rng, Nv, No)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    r = _triples(emu_lib, s, T1, T2, block)
    if Nv == 1:
        assert abs(ref) < 1e-15 and abs(r["correlation"]) < 1e-15
    else:
        assert abs(r["correlation"] - ref) < 1e-12 * max(1.0, abs(ref)), (r["correlation"], ref)
    assert r["block_size"] == (min(block, Nv) if block > 0 else r["block_size"])


@pytest.mark.parametrize("cplx", [False, True])
def test_triples_star_correction(emu_lib, cplx):
    """mp2PairEnergies given: starCorrection = (sum of the CBS pair energies) / E_MP2
    * E_(T), E_MP2 the basis second-order energy formed on the device
    (PerturbativeTriplesStar.hpp:34-108), against the oracle's restatement."""
    from cc4s_b200 import PerturbativeTriples
    s = inputs.synthetic_system(3, 8, 14, complex=cplx, seed=3)
    rng = np.random.default_rng(9)
    T1, T2 = _rand_T(rng, 8, 3)
    if cplx:
        T1 = T1 + 1j * _rand_T(rng, 8, 3)[0]
        T2 = T2 + 1j * _rand_T(rng, 8, 3)[1]
    pairs = -0.01 * rng.random((3, 3))
    r = PerturbativeTriples(lib=emu_lib).run({
        "slicedEigenEnergies": {"h": s.eps_h, "p": s.eps_p}, "coulombVertex": s.gamma,
        "halfGrid": not cplx, "amplitudes": {"ph": T1, "pphh": T2}, "mp2PairEnergies": pairs})
    V = inputs.coulomb_integrals(s, ["pphh"])["pphh"]
    e_t = r["energy"]["correlation"]
    star, e_mp2 = triples.triples_star(V, s.eps_h, s.eps_p, pairs, e_t)
    assert abs(r["stats"]["mp2_energy"] - e_mp2) < 1e-12 * abs(e_mp2)
    assert abs(r["energy"]["starCorrection"] - star) < 1e-12 * abs(star)
    from oracle import properties
    assert abs(e_mp2 - properties.mp2(s)[0]) < 1e-12 * abs(e_mp2)


def _amplitudes(rng, Nv, No, cplx):
    T1, T2 = _rand_T(rng, Nv, No)
    if cplx:
        U1, U2 = _rand_T(rng, Nv, No)
        T1, T2 = T1 + 1j * U1, T2 + 1j * U2
    return T1, T2


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape,block", [((3, 8, 14), 0), ((2, 7, 9), 3), ((3, 10, 16), 4),
                                         ((1, 5, 7), 2)])
def test_triples_complete_matches_oracle(emu_lib, cplx, shape, block):
    """cT = 1 (PerturbativeTriplesReference.cxx:92-109, :178-179): the intermediates of
    ct::getCompleteTriples formed on the device from the vertex (every statement of
    CompleteTriples.cxx:51-114 as a labelled contraction) and E = sum M Z, against the
    oracle's statement-by-statement restatement on full arrays."""
    from cc4s_b200.coupled_cluster import Solver
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, complex=cplx, seed=No + Nv)
    T1, T2 = _amplitudes(np.random.default_rng(NG), Nv, No, cplx)
    J = triples.complete_triples_intermediates(s, T1, T2)
    ref = triples.triples_reference(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p,
                                    complete=J)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
        sol.set_initial_amplitudes(T1, T2)
        r = sol.perturbative_triples(block, reference_form=True, cT=True)
        plain = sol.perturbative_triples(block, reference_form=True)["correlation"]
    finally:
        sol.close()
    assert abs(r["correlation"] - ref) < 1e-12 * max(1.0, abs(ref)), (r["correlation"], ref)
    assert abs(r["correlation"] - plain) > 1e-8 * abs(plain)  # the branches differ here
    # the M contractions double the executed flops of the block loop
    assert r["executed_flops"] >= 2 * r["flops"] * (1 - 1e-12)


def test_triples_complete_rejects_invalid_flag(emu_lib):
    import ctypes
    from cc4s_b200 import _abi
    from cc4s_b200.coupled_cluster import Solver
    s = inputs.synthetic_system(2, 5, 8, seed=1)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        sol.set_initial_amplitudes(*_rand_T(np.random.default_rng(0), 5, 2))
        o = _abi.TriplesOptions()
        sol.lib.cc4s_cc_triples_default_options(ctypes.byref(o))
        assert o.cT == 0
        o.cT = 2
        r = _abi.TriplesResult()
        st = sol.lib.cc4s_cc_perturbative_triples(sol.h, ctypes.byref(o), ctypes.byref(r))
        assert st == _abi.ERR_INVALID_ARGUMENT
    finally:
        sol.close()


def test_complete_intermediates_reduce_to_integrals_at_zero_amplitudes():
    """Oracle check: at T = 0 every correction term of CompleteTriples.cxx:90-113
    vanishes, I_bcek = V_bcek and I_mcjk = V_mcjk; and the cT energy then equals
    the plain energy with W in place of M (both vanish with T)."""
    s = inputs.synthetic_system(2, 5, 8, seed=3)
    z1, z2 = np.zeros((5, 2)), np.zeros((5, 5, 2, 2))
    J = triples.complete_triples_intermediates(s, z1, z2)
    V = inputs.coulomb_integrals(s, ["ppph", "hphh"])
    assert np.array_equal(J["ppph"], V["ppph"]) and np.array_equal(J["hphh"], V["hphh"])


@pytest.mark.parametrize("cplx", [False, True])
def test_triples_split_sliced_operands(emu_lib, cplx):
    """The split form once K = v + o >= 64: both concatenated operands sliced once per
    evaluation, every block contraction reading its rows through runs (the p = 2 terms
    from the (hole, pair) slicing, the columns from runs of one block of pairs; on the
    complex path four real products per contraction), against the FP64 form of the same
    schedule; the slicing happens outside the block loop."""
    from cc4s_b200.coupled_cluster import Solver
    No, Nv = 4, 64
    s = inputs.synthetic_system(No, Nv, 60, complex=cplx, seed=4)
    T1, T2 = _amplitudes(np.random.default_rng(8), Nv, No, cplx)
    e, st = {}, {}
    for p in ("fp64", "split3"):
        sol = Solver({"precision": p}, lib=emu_lib)
        try:
            sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
            sol.set_initial_amplitudes(T1, T2)
            s0 = sol.stats()
            e[p] = sol.perturbative_triples(8)["correlation"]
            s1 = sol.stats()
            st[p] = s1["gemm_launches"] - s0["gemm_launches"]
        finally:
            sol.close()
    assert abs(e["split3"] - e["fp64"]) < 1e-7 * abs(e["fp64"]), e
    assert e["split3"] != e["fp64"]
    # 120 block triples x 6 contractions (x 4 real products on the complex path), plus
    # 3 x 2 slicing launches per plane and the integral builds (FP64): far fewer than 5
    # launches per split product
    assert st["split3"] < 2 * 120 * 6 * (4 if cplx else 1), st


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("shape,block", [((3, 8, 14), 0), ((2, 7, 9), 3)])
def test_triples_cr_denominator(emu_lib, cplx, shape, block):
    """cT = 1: the CR-(T) denominator (ct::getDenominator, CompleteTriples.cxx:120-165, as
    PerturbativeTriplesReference.cxx:187-195 calls it) from the block loop (the sum of y
    with the triples' Z over D, folded over block orderings like the energy) and the
    amplitude-only terms, against the oracle; 0 without cT."""
    from cc4s_b200.coupled_cluster import Solver
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, complex=cplx, seed=No + Nv)
    T1, T2 = _amplitudes(np.random.default_rng(NG), Nv, No, cplx)
    den = triples.cr_triples_denominator(T1, T2, triples.triples_integrals(s), s.eps_h, s.eps_p)
    sol = Solver({}, lib=emu_lib)
    try:
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
        sol.set_initial_amplitudes(T1, T2)
        r = sol.perturbative_triples(block, reference_form=True, cT=True)
        r0 = sol.perturbative_triples(block, reference_form=True)
    finally:
        sol.close()
    assert abs(r["cr_denominator"] - den) < 1e-12 * abs(den), (r["cr_denominator"], den)
    assert r["cr_correlation"] == r["correlation"] / r["cr_denominator"]
    assert r0["cr_denominator"] == 0.0 and r0["cr_correlation"] is None
