"""Parity of the CUDA library (through its C ABI) with the oracle on a B200."""
import json
import os
import warnings

import numpy as np
import pytest

from oracle import ccsd, coupled_cluster, inputs, properties

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
warnings.simplefilter("ignore")

# FP64 parity bar: 1e-9 Eh in energies and 1e-9 relative in amplitudes; single
# residual evaluations agree to rounding (1e-12 relative to the largest element).
TOL_E = 1e-9
TOL_AMP = 1e-9
TOL_RES = 1e-12


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _rand_T(rng, Nv, No, scale=0.02):
    T1 = rng.standard_normal((Nv, No)) * scale
    T2 = rng.standard_normal((Nv, Nv, No, No)) * scale
    return T1, T2 + T2.transpose(1, 0, 3, 2)


@pytest.fixture(scope="module")
def Solver():
    from cc4s_b200 import Solver as S
    return S


@pytest.mark.parametrize("shape,cplx", [((3, 7, 5), True), ((8, 40, 200), False),
                                        ((5, 33, 70), True), ((16, 128, 256), False)])
@pytest.mark.parametrize("method", ["Ccsd", "Ccd"])
def test_residual_parity(Solver, shape, cplx, method):
    No, Nv, NG = shape
    rng = np.random.default_rng(No * 1000 + Nv)
    g = rng.standard_normal((NG, No + Nv, No + Nv)) * 0.1 * NG ** -0.25
    if cplx:
        g = g + 1j * rng.standard_normal(g.shape) * 0.1 * NG ** -0.25
    s = inputs.System(np.sort(rng.uniform(-1.5, -.5, No)), np.sort(rng.uniform(.2, 3, Nv)), g, True)
    T = _rand_T(rng, Nv, No)
    sol = Solver({"method": method})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
    R1, R2 = sol.residual(T)
    Q1, Q2 = ccsd.residuum(T, ccsd.CcsdInputs(s), ccd=(method == "Ccd"))
    assert _rel(R2, Q2) < TOL_RES
    if method == "Ccsd":
        assert _rel(R1, Q1) < TOL_RES
    F1, F2 = sol.residual(None)
    assert _rel(F2, Q2 * 0 + ccsd.residuum(None, ccsd.CcsdInputs(s))[1]) < TOL_RES
    sol.close()


def test_c0_golden_trajectory(Solver):
    g = json.load(open(os.path.join(GOLDEN, "c0_seed0.json")))
    s = inputs.config_system("c0", seed=g["seed"])
    sol = Solver(g["options"])
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
    r = sol.run()
    assert r["iterations"] == g["iterations"]
    assert r["converged"] == g["converged"]
    for h, e in zip(r["history"], g["history_energy"]):
        assert abs(h["energy"] - e) < TOL_E
    assert abs(r["correlation"] - g["energy"]["correlation"]) < TOL_E
    assert abs(r["secondOrder"] - g["energy"]["secondOrder"]) < TOL_E
    T1, T2 = sol.amplitudes()
    ref = coupled_cluster.run(s, **g["options"])
    assert _rel(T2, ref["amplitudes"][1]) < TOL_AMP
    assert _rel(T1, ref["amplitudes"][0]) < TOL_AMP


@pytest.mark.parametrize("opts", [
    dict(method="Ccd", mixer=dict(type="DiisMixer", maxResidua=4)),
    dict(method="Ccsd", mixer=dict(type="LinearMixer", ratio=0.8), levelShift=0.2),
    dict(method="Ccsd", ppl=False, mixer=dict(type="DiisMixer", maxResidua=3)),
])
def test_run_variants(Solver, opts):
    s = inputs.synthetic_system(6, 30, 60, seed=11)
    o = dict(maxIterations=40, energyConvergence=1e-10, amplitudesConvergence=1e-8)
    o.update(opts)
    ref = coupled_cluster.run(s, **o)
    sol = Solver(o)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    r = sol.run()
    assert r["iterations"] == ref["iterations"]
    assert abs(r["correlation"] - ref["energy"]["correlation"]) < TOL_E
    T1, T2 = sol.amplitudes()
    assert _rel(T2, ref["amplitudes"][1]) < TOL_AMP


def test_c1_size_independent_properties(Solver):
    """At the FP64 parity size (No=32, Nv=256, NG=1024): the first iteration gives
    the MP2 energy, and the amplitudes keep the pair symmetry T_abij = T_baji."""
    s = inputs.config_system("c1", seed=0)
    sol = Solver(dict(maxIterations=3, energyConvergence=0.0))
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    r = sol.run()
    assert abs(r["secondOrder"] - properties.mp2(s)[0]) < TOL_E
    T1, T2 = sol.amplitudes()
    assert _rel(T2.transpose(1, 0, 3, 2), T2) < 1e-12
    assert all(np.isfinite(h["energy"]) for h in r["history"])


def _summary_check(A, g, arrays, name, seed, tol):
    """A against the fixture's norm, seeded weighted checksum and element sample
    (tests/golden/make_large_golden.py): every difference relative to the
    fixture's largest element (sample) or norm (norm, checksum)."""
    flat = np.asarray(A).reshape(-1, order="F")
    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(flat.size, size=arrays[name + "_idx"].size, replace=False))
    assert np.array_equal(idx, arrays[name + "_idx"])
    w = rng.standard_normal(flat.size)
    assert np.abs(flat[idx] - arrays[name + "_val"]).max() < tol * g[name + "_max"]
    assert abs(np.sqrt((flat * flat).sum()) - g[name + "_norm"]) < tol * g[name + "_norm"]
    assert abs(w @ flat - g[name + "_checksum"]) < tol * g[name + "_norm"]


def test_c1_parity_trajectory(Solver):
    """The FP64 parity configuration (No=32, Nv=256, NG=1024, seed 0, unscaled
    generator): four iterations from T = 0 with DIIS depth 5 against the oracle's
    committed fixture -- every iteration's energy within 1e-9 Eh, the final
    direct/exchange energies likewise, and the final amplitudes within 1e-9
    relative (element sample, norm and a seeded weighted checksum of all elements)."""
    g = json.load(open(os.path.join(GOLDEN, "c1_seed0_4it.json")))
    arrays = np.load(os.path.join(GOLDEN, "c1_seed0_4it.npz"))
    s = inputs.config_system("c1", seed=g["seed"])
    sol = Solver(g["options"])
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    r = sol.run()
    assert r["iterations"] == g["iterations"]
    for h, e, dr in zip(r["history"], g["history_energy"], g["history_dR"]):
        assert abs(h["energy"] - e) < TOL_E
        assert abs(h["dR"] - dr) < TOL_AMP * dr
    for k in ("correlation", "direct", "exchange", "secondOrder"):
        assert abs(r[k] - g["energy"][k]) < TOL_E
    T1, T2 = sol.amplitudes()
    sol.close()
    _summary_check(T1, g, arrays, "T1", g["sample_seeds"]["T1"], TOL_AMP)
    _summary_check(T2, g, arrays, "T2", g["sample_seeds"]["T2"], TOL_AMP)


def test_c4_residual_parity(Solver):
    """One residual at the c4 shape (No=32, Nv=320, NG=1600, seed 0) at seeded
    random amplitudes against the oracle's committed fixture, to 1e-12 relative."""
    g = json.load(open(os.path.join(GOLDEN, "c4_seed0_residual.json")))
    arrays = np.load(os.path.join(GOLDEN, "c4_seed0_residual.npz"))
    s = inputs.config_system("c4", seed=g["seed"])
    T = _rand_T(np.random.default_rng(4), s.Nv, s.No)
    sol = Solver({})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    R1, R2 = sol.residual(T)
    sol.close()
    _summary_check(R1, g, arrays, "R1", g["sample_seeds"]["R1"], TOL_RES)
    _summary_check(R2, g, arrays, "R2", g["sample_seeds"]["R2"], TOL_RES)


def test_ueg_reference_energies(Solver):
    """cc4s's own expected CCSD energies of its UEG regression test
    (test/tests/ueg/rs1.0-7occ-26virt), reproduced on the GPU."""
    g = json.load(open(os.path.join(GOLDEN, "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    sol = Solver(g["ccsd"]["options"])
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    r = sol.run()
    assert r["converged"]
    for k, ref in g["ccsd"]["energy"].items():
        assert abs(r[k] - ref) < TOL_E, (k, r[k], ref)


@pytest.mark.parametrize("shape,hermitian", [((3, 7, 5), False), ((6, 30, 40), True),
                                             ((10, 64, 90), True)])
def test_complex_residual_parity(Solver, shape, hermitian):
    No, Nv, NG = shape
    rng = np.random.default_rng(7 * No + Nv)
    if hermitian:
        s = inputs.synthetic_system(No, Nv, NG, complex=True, seed=No)
    else:
        g = (rng.standard_normal((NG, No + Nv, No + Nv)) + 1j * rng.standard_normal((NG, No + Nv, No + Nv))) * 0.1
        s = inputs.System(np.sort(rng.uniform(-1.5, -.5, No)), np.sort(rng.uniform(.2, 3, Nv)), g, False)
    T1 = (rng.standard_normal((Nv, No)) + 1j * rng.standard_normal((Nv, No))) * 0.02
    T2 = (rng.standard_normal((Nv, Nv, No, No)) + 1j * rng.standard_normal((Nv, Nv, No, No))) * 0.02
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    sol = Solver({})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    R1, R2 = sol.residual((T1, T2))
    Q1, Q2 = ccsd.residuum((T1, T2), ccsd.CcsdInputs(s))
    assert _rel(R1, Q1) < TOL_RES and _rel(R2, Q2) < TOL_RES


def test_split_precision_residual(Solver):
    """Three-slice tensor-core form of the residual vs the FP64 oracle: the split
    products carry 28 bits of each operand row/column, so the residual agrees to
    ~1e-7 of its largest element (tolerance 1e-5)."""
    s = inputs.synthetic_system(16, 128, 256, seed=2)
    rng = np.random.default_rng(3)
    T = _rand_T(rng, 128, 16)
    sol = Solver({"precision": "split3"})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    R1, R2 = sol.residual(T)
    Q1, Q2 = ccsd.residuum(T, ccsd.CcsdInputs(s))
    assert _rel(R2, Q2) < 1e-5 and _rel(R1, Q1) < 1e-5
    assert _rel(R2, Q2) > 1e-14  # the tensor-core path really ran


@pytest.mark.parametrize("precision,tol", [("fp64", TOL_RES), ("split3", 1e-5)])
def test_ladder_blocks_and_c_panels(Solver, monkeypatch, precision, tol):
    """Ladder on ragged virtual blocks (48, 48, 32) and four panels of c."""
    monkeypatch.setenv("CC4S_PPL_SLAB_DOUBLES", str(48 * 48 * 128 * 40))
    s = inputs.synthetic_system(16, 128, 256, seed=2)
    T = _rand_T(np.random.default_rng(3), 128, 16)
    sol = Solver({"precision": precision, "integralsSliceSize": 48})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    R1, R2 = sol.residual(T)
    sol.close()
    Q1, Q2 = ccsd.residuum(T, ccsd.CcsdInputs(s))
    assert _rel(R2, Q2) < tol and _rel(R1, Q1) < tol


def test_split_precision_k_panels(Solver, monkeypatch):
    """With the packed-slice scratch limited to 1 MiB every split contraction is
    cut into K panels (one-level, whole inner runs and inside inner runs) that
    accumulate into C; the residual still agrees with the oracle to 1e-5 and
    with the single-panel split result to 1e-6."""
    s = inputs.synthetic_system(16, 128, 256, seed=2)
    rng = np.random.default_rng(3)
    T = _rand_T(rng, 128, 16)
    one = Solver({"precision": "split3"})
    one.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    P1, P2 = one.residual(T)
    one.close()
    monkeypatch.setenv("CC4S_SPLIT_PANEL_BYTES", str(1 << 20))
    sol = Solver({"precision": "split3"})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    R1, R2 = sol.residual(T)
    sol.close()
    Q1, Q2 = ccsd.residuum(T, ccsd.CcsdInputs(s))
    assert _rel(R2, Q2) < 1e-5 and _rel(R1, Q1) < 1e-5
    assert _rel(R2, P2) < 1e-6 and _rel(R1, P1) < 1e-6


def test_split_precision_refinement_reaches_fp64_energy(Solver):
    """precisionRefinement: split iterations until the residuum norm is below
    1e-5, FP64 after; the converged energy equals the FP64 form's to 1e-9 Eh."""
    s = inputs.synthetic_system(10, 64, 150, seed=0)
    o = dict(maxIterations=80, energyConvergence=1e-11, amplitudesConvergence=1e-9,
             mixer=dict(type="DiisMixer", maxResidua=5))
    runs = {}
    for name, extra in (("fp64", {}), ("refined", dict(precision="split3", precisionRefinement=1e-5))):
        sol = Solver(dict(o, **extra))
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
        runs[name] = sol.run()
        sol.close()
        assert runs[name]["converged"]
    assert runs["refined"]["refined_from"] > 1
    assert abs(runs["refined"]["correlation"] - runs["fp64"]["correlation"]) < TOL_E


def test_split_precision_complex(Solver):
    """Complex path in the split form: residual within 1e-5 of the oracle, and the
    converged energy within 1 uEh of the FP64 form."""
    s = inputs.synthetic_system(8, 64, 120, complex=True, seed=6)
    rng = np.random.default_rng(4)
    T1 = (rng.standard_normal((64, 8)) + 1j * rng.standard_normal((64, 8))) * 0.02
    T2 = (rng.standard_normal((64, 64, 8, 8)) + 1j * rng.standard_normal((64, 64, 8, 8))) * 0.02
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    sol = Solver({"precision": "split3"})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    R1, R2 = sol.residual((T1, T2))
    sol.close()
    Q1, Q2 = ccsd.residuum((T1, T2), ccsd.CcsdInputs(s))
    assert _rel(R2, Q2) < 1e-5 and _rel(R1, Q1) < 1e-5
    assert _rel(R2, Q2) > 1e-14
    o = dict(maxIterations=60, energyConvergence=1e-10, amplitudesConvergence=1e-7)
    a = Solver(o)
    a.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    ra = a.run()
    b = Solver(dict(o, precision="split3"))
    b.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    rb = b.run()
    assert ra["converged"] and rb["converged"]
    assert abs(ra["correlation"] - rb["correlation"]) < 1e-6


@pytest.mark.parametrize("shape", [(8, 40, 200), (10, 64, 150)])
def test_split_precision_energy_within_1ueh(Solver, shape):
    """Converged CCSD energy of the split-precision form within 1 uEh of FP64."""
    No, Nv, NG = shape
    s = inputs.synthetic_system(No, Nv, NG, seed=0)
    o = dict(maxIterations=80, energyConvergence=1e-10, amplitudesConvergence=1e-7,
             mixer=dict(type="DiisMixer", maxResidua=5))
    a = Solver(o)
    a.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    ra = a.run()
    b = Solver(dict(o, precision="split3"))
    b.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    rb = b.run()
    assert ra["converged"] and rb["converged"]
    assert abs(ra["correlation"] - rb["correlation"]) < 1e-6


@pytest.mark.parametrize("cfg", ["c0", "complex"])
def test_backward_structure_factor(Solver, cfg):
    """S(G) = dE_c/dV(G) at frozen amplitudes: equals the restated reference
    structure factor (FiniteSizeCorrection.cxx:113-125) and central finite
    differences in V(G) (Gamma_G scaled by sqrt(V(G))) to 1e-6 relative."""
    from oracle.inputs import coulomb_integrals
    if cfg == "c0":
        s = inputs.config_system("c0", seed=0)
    else:
        s = inputs.synthetic_system(6, 30, 40, complex=True, seed=4)
    cplx = cfg != "c0"
    sol = Solver(dict(maxIterations=40, energyConvergence=1e-10))
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
    r = sol.run()
    T = sol.amplitudes()
    S, g = sol.backward(gradient=not cplx)
    S0 = properties.structure_factor(s, T)
    assert _rel(S, S0) < 1e-11
    assert abs(S.sum() - r["correlation"]) < TOL_E

    def energy_of(gm):  # E_c at the frozen amplitudes for vertex gm
        ss = inputs.System(s.eps_h, s.eps_p, gm, s.half_grid)
        return np.real(coupled_cluster.get_energy(T, coulomb_integrals(ss, ["pphh"])["pphh"])[0])

    h = 1e-5
    for G in (0, s.NG // 2, s.NG - 1):
        up, dn = np.ones(s.NG), np.ones(s.NG)
        up[G] += h
        dn[G] -= h
        fd = (energy_of(s.gamma * np.sqrt(up)[:, None, None]) -
              energy_of(s.gamma * np.sqrt(dn)[:, None, None])) / (2 * h)
        assert abs(S[G] - fd) < 1e-6 * max(abs(fd), 1e-12)
    if not cplx:
        d = np.random.default_rng(0).standard_normal(s.gamma.shape)
        fd = (energy_of(s.gamma + h * d) - energy_of(s.gamma - h * d)) / (2 * h)
        assert abs((g * d).sum() - fd) < 1e-6 * abs(fd)


def test_complex_run(Solver):
    s = inputs.synthetic_system(6, 30, 60, complex=True, seed=5)
    o = dict(maxIterations=30, energyConvergence=1e-10, amplitudesConvergence=1e-8)
    ref = coupled_cluster.run(s, **o)
    sol = Solver(o)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    r = sol.run()
    assert r["iterations"] == ref["iterations"]
    assert abs(r["correlation"] - ref["energy"]["correlation"]) < TOL_E
    T1, T2 = sol.amplitudes()
    assert _rel(T2, ref["amplitudes"][1]) < TOL_AMP


def test_residual_vjp_on_device(Solver):
    """Transposed-Jacobian product of the residual on the B200 against central
    differences of <Rbar, R(T)> in T and in the vertex."""
    No, Nv, NG = 6, 30, 40
    s = inputs.synthetic_system(No, Nv, NG, seed=3)
    rng = np.random.default_rng(1)
    T = _rand_T(rng, Nv, No, scale=0.05)
    Rb = (rng.standard_normal((Nv, No)), rng.standard_normal((Nv, Nv, No, No)))
    sol = Solver({})
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    (T1b, T2b), Gb = sol.residual_vjp(T, Rb)

    def f(TT, gm=None):
        so = sol
        if gm is not None:
            so = Solver({})
            so.set_inputs(s.eps_h, s.eps_p, gm, True)
        return sum((a * b).sum() for a, b in zip(Rb, so.residual(TT)))
    d = _rand_T(rng, Nv, No, scale=1.0)
    h = 1e-5
    fd = (f((T[0] + h * d[0], T[1] + h * d[1])) - f((T[0] - h * d[0], T[1] - h * d[1]))) / (2 * h)
    assert abs(fd - ((T1b * d[0]).sum() + (T2b * d[1]).sum())) < 1e-6 * abs(fd)
    dg = rng.standard_normal(s.gamma.shape)
    fdg = (f(T, s.gamma + h * dg) - f(T, s.gamma - h * dg)) / (2 * h)
    assert abs(fdg - (Gb * dg).sum()) < 1e-6 * abs(fdg)


def test_relaxed_gradient_on_device(Solver):
    """Lambda equations on the B200: dE_c/dGamma of the converged CCSD energy
    against central differences of re-converged energies (step 1e-5, four
    random directions) to 1e-6 relative."""
    s = inputs.synthetic_system(8, 40, 100, seed=2)
    opts = dict(maxIterations=100, energyConvergence=1e-14, amplitudesConvergence=1e-11)

    def energy(gm):
        so = Solver(opts)
        so.set_inputs(s.eps_h, s.eps_p, gm, True)
        e = so.run()["correlation"]
        return so, e
    sol, _ = energy(s.gamma)
    g, info = sol.relaxed_gradient(max_iterations=100, convergence=1e-11)
    assert info["converged"]
    rng = np.random.default_rng(5)
    h = 1e-5
    for _ in range(4):
        d = rng.standard_normal(s.gamma.shape)
        fd = (energy(s.gamma + h * d)[1] - energy(s.gamma - h * d)[1]) / (2 * h)
        assert abs(fd - (g * d).sum()) < 1e-6 * abs(fd)


def test_relaxed_gradient_split_precision_on_device(Solver):
    """The split-precision variant of the backward on the B200: the recorded
    residual and the large contractions of the transposed-Jacobian products run
    on the tcgen05 split kernel; the relaxed gradient agrees with the FP64 one to
    1e-6 relative (largest element) and with central differences of FP64
    re-converged energies to 1e-5 relative (the split rounding of the residual and
    of its transposed Jacobian leaves ~1e-6 in a projected derivative; the FP64
    gradient meets 1e-6, test_relaxed_gradient_on_device)."""
    s = inputs.synthetic_system(8, 72, 100, seed=2)
    # the split form's residual carries ~1e-9 relative rounding, so its forward and
    # Lambda iterations stop at looser thresholds than the FP64 ones
    conv = {"fp64": (dict(energyConvergence=1e-14, amplitudesConvergence=1e-11), 1e-11),
            "split3": (dict(energyConvergence=1e-10, amplitudesConvergence=1e-8), 1e-8)}

    def solve(gm, precision="fp64"):
        so = Solver(dict(conv[precision][0], maxIterations=100, precision=precision))
        so.set_inputs(s.eps_h, s.eps_p, gm, True)
        return so, so.run()["correlation"]
    grads = {}
    for p in ("fp64", "split3"):
        sol, _ = solve(s.gamma, p)
        grads[p], info = sol.relaxed_gradient(max_iterations=100, convergence=conv[p][1])
        sol.close()
        assert info["converged"]
    g64, gs = grads["fp64"], grads["split3"]
    assert 0.0 < np.abs(gs - g64).max() < 1e-6 * np.abs(g64).max()
    rng = np.random.default_rng(5)
    h = 1e-5
    for _ in range(3):
        d = rng.standard_normal(s.gamma.shape)
        fd = (solve(s.gamma + h * d)[1] - solve(s.gamma - h * d)[1]) / (2 * h)
        assert abs(fd - (gs * d).sum()) < 1e-5 * abs(fd)


def test_real_path_equals_complex_path_on_device(Solver):
    """On the B200: a real symmetric vertex run through the complex path (the path
    pinned to cc4s's expected UEG energies) and through the real half-grid path
    gives the same converged energies and amplitudes (to 1e-10 relative)."""
    s = inputs.synthetic_system(12, 96, 200, seed=12)
    opts = dict(maxIterations=60, energyConvergence=1e-12, amplitudesConvergence=1e-10)
    out = {}
    for hg, g in ((True, s.gamma), (False, np.asarray(s.gamma, dtype=complex))):
        sol = Solver(opts)
        sol.set_inputs(s.eps_h, s.eps_p, g, half_grid=hg)
        r = sol.run()
        out[hg] = (r, sol.amplitudes())
        sol.close()
    (rr, Tr), (rc, Tc) = out[True], out[False]
    assert rr["iterations"] == rc["iterations"]
    for k in ("correlation", "direct", "exchange", "secondOrder"):
        assert abs(rr[k] - rc[k]) < 1e-10 * abs(rr[k])
    assert _rel(Tc[1].real, Tr[1]) < 1e-10 and np.abs(Tc[1].imag).max() < 1e-12


def test_complex_relaxed_gradient_on_device(Solver):
    """Complex path on the B200: the relaxed dE_c/dGamma (Lambda equations, d/dRe +
    i d/dIm) against central differences of re-converged energies along Hermitian
    vertex directions (Richardson-extrapolated from steps 1e-5 and 5e-6), 1e-6
    relative."""
    s = inputs.synthetic_system(6, 36, 80, complex=True, seed=2)
    opts = dict(maxIterations=100, energyConvergence=1e-14, amplitudesConvergence=1e-11)

    def energy(gm):
        so = Solver(opts)
        so.set_inputs(s.eps_h, s.eps_p, gm, half_grid=False)
        return so, so.run()["correlation"]
    sol, _ = energy(s.gamma)
    g, info = sol.relaxed_gradient(max_iterations=100, convergence=1e-11)
    sol.close()
    assert info["converged"]
    rng = np.random.default_rng(5)
    h = 1e-5
    for _ in range(3):
        d = rng.standard_normal(s.gamma.shape) + 1j * rng.standard_normal(s.gamma.shape)
        d = d + np.conj(d.transpose(0, 2, 1))

        def cd(step):
            return (energy(s.gamma + step * d)[1] - energy(s.gamma - step * d)[1]) / (2 * step)
        fd = (4.0 * cd(h / 2) - cd(h)) / 3.0
        assert abs(fd - np.real(np.conj(g) * d).sum()) < 1e-6 * abs(fd)
