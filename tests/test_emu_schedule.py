"""The product's CCSD schedule and driver (C++ sources of cc4s_b200/csrc)
linked against a plain-loop CPU emulation of the device operations
(tests/emu/ops_emu.cpp, test-only) and checked against the oracle.  This pins
every stride of every contraction without a GPU."""
import os
import sys
import warnings

import numpy as np
import pytest

from oracle import ccsd, coupled_cluster, inputs

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))
warnings.simplefilter("ignore")


@pytest.fixture(scope="module")
def emu_lib():
    import build_emu
    return build_emu.build()


def _rel(a, b):
    return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)


def _rand_T(rng, Nv, No):
    T1 = rng.standard_normal((Nv, No)) * 0.05
    T2 = rng.standard_normal((Nv, Nv, No, No)) * 0.05
    return T1, T2 + T2.transpose(1, 0, 3, 2)


@pytest.mark.parametrize("shape", [(3, 7, 5), (4, 10, 12), (2, 5, 3)])
@pytest.mark.parametrize("method", ["Ccsd", "Ccd"])
def test_residual_matches_oracle(emu_lib, shape, method):
    from cc4s_b200 import Solver
    No, Nv, NG = shape
    rng = np.random.default_rng(sum(shape))
    g = (rng.standard_normal((NG, No + Nv, No + Nv)) + 1j * rng.standard_normal((NG, No + Nv, No + Nv))) * 0.1
    s = inputs.System(np.sort(rng.uniform(-1.5, -.5, No)), np.sort(rng.uniform(.2, 3, Nv)), g, half_grid=True)
    T = _rand_T(rng, Nv, No)
    for ppl in (True, False):
        sol = Solver({"method": method, "ppl": ppl}, lib=emu_lib)
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=True)
        R1, R2 = sol.residual(T)
        Q1, Q2 = ccsd.residuum(T, ccsd.CcsdInputs(s), ppl=ppl, ccd=(method == "Ccd"))
        assert _rel(R2, Q2) < 1e-13
        if method == "Ccsd":
            assert _rel(R1, Q1) < 1e-13
        else:
            assert np.abs(R1).max() == 0.0


@pytest.mark.parametrize("cplx", [False, True])
@pytest.mark.parametrize("slice_size,budget", [(4, 528), (5, 300), (11, 0)])
def test_ladder_blocks_and_c_panels(emu_lib, monkeypatch, slice_size, budget, cplx):
    """Ladder on several virtual blocks (integralsSliceSize) and several panels of
    c (slab budget CC4S_PPL_SLAB_DOUBLES), ragged edges included; the complex case
    uses a Hermitian vertex, for which the reference's slicing is exact."""
    from cc4s_b200 import Solver
    if budget:
        monkeypatch.setenv("CC4S_PPL_SLAB_DOUBLES", str(budget))
    s = inputs.synthetic_system(4, 11, 12, complex=cplx, seed=5)
    T = _rand_T(np.random.default_rng(8), 11, 4)
    if cplx:
        rng = np.random.default_rng(9)
        T = (T[0] + 0.05j * rng.standard_normal(T[0].shape),
             T[1] + 0.05j * (lambda x: x + x.transpose(1, 0, 3, 2))(rng.standard_normal(T[1].shape)))
    sol = Solver({"integralsSliceSize": slice_size}, lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
    R1, R2 = sol.residual(T)
    Q1, Q2 = ccsd.residuum(T, ccsd.CcsdInputs(s))
    assert _rel(R2, Q2) < 1e-13 and _rel(R1, Q1) < 1e-13


@pytest.mark.parametrize("mixer", [dict(type="DiisMixer", maxResidua=5),
                                   dict(type="DiisMixer", maxResidua=2),
                                   dict(type="LinearMixer", ratio=0.7)])
def test_run_matches_oracle(emu_lib, mixer):
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(4, 12, 20, seed=3)
    opts = dict(maxIterations=30, energyConvergence=1e-10, amplitudesConvergence=1e-8, mixer=mixer,
                levelShift=0.1 if mixer["type"] == "LinearMixer" else 0.0)
    r0 = coupled_cluster.run(s, **opts)
    sol = Solver(opts, lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    r = sol.run()
    T1, T2 = sol.amplitudes()
    assert r["iterations"] == r0["iterations"]
    assert abs(r["correlation"] - r0["energy"]["correlation"]) < 1e-12
    assert abs(r["secondOrder"] - r0["energy"]["secondOrder"]) < 1e-12
    assert _rel(T2, r0["amplitudes"][1]) < 1e-12


def test_split_precision_form_accuracy(emu_lib):
    """Three-slice split products (exact model of the tensor-core scheme) on the
    ladder/ring/vertex contractions: the converged energy stays far inside 1 uEh."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(6, 30, 60, seed=0)  # large enough for the split path (>= 64)
    o = dict(maxIterations=40, energyConvergence=1e-10, amplitudesConvergence=1e-7)
    a = Solver(o, lib=emu_lib)
    a.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    ra = a.run()
    b = Solver(dict(o, precision="split3"), lib=emu_lib)
    b.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    rb = b.run()
    assert ra["converged"] and rb["converged"]
    assert abs(ra["correlation"] - rb["correlation"]) < 1e-8
    assert ra["correlation"] != rb["correlation"]  # the split path really ran


def test_split_precision_refinement_reaches_fp64_fixed_point(emu_lib):
    """precisionRefinement: split iterations until the residuum norm is below the
    threshold, FP64 after; the converged energy is the FP64 one to the convergence
    threshold, while the pure split form differs at the split-precision level."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(6, 30, 60, seed=0)
    o = dict(maxIterations=60, energyConvergence=1e-13, amplitudesConvergence=1e-10)
    runs = {}
    for name, extra in (("fp64", {}), ("split", dict(precision="split3")),
                        ("refined", dict(precision="split3", precisionRefinement=1e-5))):
        sol = Solver(dict(o, **extra), lib=emu_lib)
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
        runs[name] = sol.run()
        assert runs[name]["converged"]
    assert runs["refined"]["refined_from"] > 1
    assert abs(runs["refined"]["correlation"] - runs["fp64"]["correlation"]) < 1e-12
    assert abs(runs["split"]["correlation"] - runs["fp64"]["correlation"]) > 1e-14


def test_split_precision_complex_path(emu_lib):
    """Complex path: the large contractions run as split products (exact model of
    the tensor-core scheme); the converged energy stays far inside 1 uEh."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(6, 30, 60, complex=True, seed=1)
    o = dict(maxIterations=40, energyConvergence=1e-10, amplitudesConvergence=1e-7)
    a = Solver(o, lib=emu_lib)
    a.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    ra = a.run()
    b = Solver(dict(o, precision="split3"), lib=emu_lib)
    b.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    rb = b.run()
    assert ra["converged"] and rb["converged"]
    assert abs(ra["correlation"] - rb["correlation"]) < 1e-8
    assert ra["correlation"] != rb["correlation"]  # the split path really ran


@pytest.mark.parametrize("cplx", [False, True])
def test_backward_structure_factor_and_gradient(emu_lib, cplx):
    """Adjoint entry: S(G) equals the restated FiniteSizeCorrection structure
    factor, sums to E_c, and dE/dGamma (real path) matches central differences."""
    from cc4s_b200 import Solver
    from oracle import properties
    from oracle.inputs import coulomb_integrals
    s = inputs.synthetic_system(4, 12, 20, complex=cplx, seed=2)
    sol = Solver(dict(maxIterations=30, energyConvergence=1e-10, amplitudesConvergence=1e-8),
                 lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
    r = sol.run()
    T = sol.amplitudes()
    S, g = sol.backward(gradient=not cplx)
    S0 = properties.structure_factor(s, T)
    assert _rel(S, S0) < 1e-12
    assert abs(S.sum() - r["correlation"]) < 1e-12
    if not cplx:
        d = np.random.default_rng(0).standard_normal(s.gamma.shape)

        def E(gm):
            ss = inputs.System(s.eps_h, s.eps_p, gm, True)
            return coupled_cluster.get_energy(T, coulomb_integrals(ss, ["pphh"])["pphh"])[0]
        h = 1e-5
        fd = (E(s.gamma + h * d) - E(s.gamma - h * d)) / (2 * h)
        assert abs((g * d).sum() - fd) < 1e-6 * abs(fd)


def test_errors_are_reported(emu_lib):
    from cc4s_b200 import CoupledClusterError, Solver
    sol = Solver({}, lib=emu_lib)
    with pytest.raises(CoupledClusterError) as e:
        sol.run()
    assert e.value.status == 8  # inputs not set
    s = inputs.synthetic_system(2, 5, 3, seed=1)
    g = s.gamma.copy()
    g[0, 0, 0] = np.nan
    with pytest.raises(CoupledClusterError) as e:
        sol.set_inputs(s.eps_h, s.eps_p, g, True)
    assert e.value.status == 9  # non-finite input
    with pytest.raises(CoupledClusterError) as e:
        Solver({"method": "Ccsdt"}, lib=emu_lib)
    assert e.value.status == 1


@pytest.mark.parametrize("shape", [(3, 7, 5), (4, 9, 11)])
@pytest.mark.parametrize("method", ["Ccsd", "Ccd"])
def test_complex_residual_matches_oracle(emu_lib, shape, method):
    """Complex integral path with a non-Hermitian vertex."""
    from cc4s_b200 import Solver
    No, Nv, NG = shape
    rng = np.random.default_rng(100 + sum(shape))
    g = (rng.standard_normal((NG, No + Nv, No + Nv)) + 1j * rng.standard_normal((NG, No + Nv, No + Nv))) * 0.1
    s = inputs.System(np.sort(rng.uniform(-1.5, -.5, No)), np.sort(rng.uniform(.2, 3, Nv)), g, half_grid=False)
    T1 = (rng.standard_normal((Nv, No)) + 1j * rng.standard_normal((Nv, No))) * 0.05
    T2 = (rng.standard_normal((Nv, Nv, No, No)) + 1j * rng.standard_normal((Nv, Nv, No, No))) * 0.05
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    sol = Solver({"method": method}, lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    R1, R2 = sol.residual((T1, T2))
    Q1, Q2 = ccsd.residuum((T1, T2), ccsd.CcsdInputs(s), ccd=(method == "Ccd"))
    assert _rel(R2, Q2) < 1e-13
    if method == "Ccsd":
        assert _rel(R1, Q1) < 1e-13


def test_ueg_reference_energies_through_product_schedule(emu_lib):
    """The product's complex schedule and driver reproduce cc4s's own expected
    UEG (rs=1, No=7, Nv=26) CCSD energies."""
    import json
    from cc4s_b200 import Solver
    g = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "ueg_rs1.0_7occ_26virt.json")))
    s = inputs.ueg_system(7, 26, 1.0)
    sol = Solver(g["ccsd"]["options"], lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    r = sol.run()
    assert r["converged"]
    for k, ref in g["ccsd"]["energy"].items():
        assert abs(r[k] - ref) < 1e-10, (k, r[k], ref)


@pytest.mark.parametrize("method,ppl", [("Ccsd", True), ("Ccsd", False), ("Ccd", True)])
def test_residual_vjp_matches_finite_differences(emu_lib, method, ppl):
    """Transposed-Jacobian product of the residual (reverse replay of the
    recorded schedule) against central differences of <Rbar, R(T)> in T and in
    the vertex."""
    from cc4s_b200 import Solver
    No, Nv, NG = 3, 8, 6
    s = inputs.synthetic_system(No, Nv, NG, seed=3)
    rng = np.random.default_rng(1)

    def sym(x):
        return x + x.transpose(1, 0, 3, 2)
    T = (rng.standard_normal((Nv, No)) * 0.1, sym(rng.standard_normal((Nv, Nv, No, No))) * 0.05)
    Rb = (rng.standard_normal((Nv, No)), rng.standard_normal((Nv, Nv, No, No)))
    opts = {"method": method, "ppl": ppl}
    sol = Solver(opts, lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
    (T1b, T2b), Gb = sol.residual_vjp(T, Rb)

    def f(TT, gm=None):
        so = sol
        if gm is not None:
            so = Solver(opts, lib=emu_lib)
            so.set_inputs(s.eps_h, s.eps_p, gm, True)
        return sum((a * b).sum() for a, b in zip(Rb, so.residual(TT)))
    d = (rng.standard_normal((Nv, No)) * (method == "Ccsd"), sym(rng.standard_normal((Nv, Nv, No, No))))
    h = 1e-5
    fd = (f((T[0] + h * d[0], T[1] + h * d[1])) - f((T[0] - h * d[0], T[1] - h * d[1]))) / (2 * h)
    assert abs(fd - ((T1b * d[0]).sum() + (T2b * d[1]).sum())) < 1e-7 * abs(fd)
    dg = rng.standard_normal(s.gamma.shape)
    fdg = (f(T, s.gamma + h * dg) - f(T, s.gamma - h * dg)) / (2 * h)
    assert abs(fdg - (Gb * dg).sum()) < 1e-8 * abs(fdg)


@pytest.mark.parametrize("method", ["Ccsd", "Ccd"])
def test_relaxed_gradient_matches_finite_differences(emu_lib, method):
    """Lambda equations solved with transposed-Jacobian products: dE_c/dGamma of
    the converged energy against central differences of re-converged energies
    (step 1e-5, three random directions) to 1e-6 relative."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(4, 12, 20, seed=2)
    opts = dict(method=method, maxIterations=80, energyConvergence=1e-14,
                amplitudesConvergence=1e-12)

    def energy(gm):
        so = Solver(opts, lib=emu_lib)
        so.set_inputs(s.eps_h, s.eps_p, gm, True)
        return so, so.run()["correlation"]
    sol, _ = energy(s.gamma)
    g, info = sol.relaxed_gradient(max_iterations=100, convergence=1e-12)
    assert info["converged"]
    rng = np.random.default_rng(5)
    h = 1e-5
    for _ in range(3):
        d = rng.standard_normal(s.gamma.shape)
        fd = (energy(s.gamma + h * d)[1] - energy(s.gamma - h * d)[1]) / (2 * h)
        assert abs(fd - (g * d).sum()) < 1e-6 * abs(fd)


def test_relaxed_gradient_split_precision(emu_lib):
    """The split-precision variant of the backward: the recorded residual and the
    large contractions of every transposed-Jacobian product in split precision
    (emulated slicing); the relaxed gradient agrees with the FP64 one to 1e-6
    relative and with central differences of FP64 re-converged energies to 1e-6."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(2, 32, 40, seed=2)
    opts = dict(maxIterations=80, energyConvergence=1e-14, amplitudesConvergence=1e-12)

    def solve(gm, precision="fp64"):
        so = Solver(dict(opts, precision=precision), lib=emu_lib)
        so.set_inputs(s.eps_h, s.eps_p, gm, True)
        return so, so.run()["correlation"]
    grads = {}
    for p in ("fp64", "split3"):
        sol, _ = solve(s.gamma, p)
        grads[p], info = sol.relaxed_gradient(max_iterations=100, convergence=1e-12)
        sol.close()
        assert info["converged"]
    g64, gs = grads["fp64"], grads["split3"]
    assert np.abs(gs - g64).max() < 1e-6 * np.abs(g64).max()
    assert np.abs(gs - g64).max() > 0.0     # the split path really ran
    rng = np.random.default_rng(5)
    h = 1e-5
    for _ in range(2):
        d = rng.standard_normal(s.gamma.shape)
        fd = (solve(s.gamma + h * d)[1] - solve(s.gamma - h * d)[1]) / (2 * h)
        assert abs(fd - (gs * d).sum()) < 1e-6 * abs(fd)


def test_split_ladder_prepacked_x_panel(emu_lib):
    """Split form with several ladder blocks (integralsSliceSize 8 at Nv = 24): the
    X panel is sliced once per c range and shared by the block pairs; the residual
    equals the one-block split residual (no shared panel) and the oracle's to the
    split precision."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(8, 24, 30, seed=3)
    rng = np.random.default_rng(5)
    T1 = rng.standard_normal((24, 8)) * 0.02
    T2 = rng.standard_normal((24, 24, 8, 8)) * 0.02
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    out = {}
    for sl in (8, 24):
        sol = Solver({"precision": "split3", "integralsSliceSize": sl}, lib=emu_lib)
        sol.set_inputs(s.eps_h, s.eps_p, s.gamma, True)
        out[sl] = sol.residual((T1, T2))
        sol.close()
    Q1, Q2 = ccsd.residuum((T1, T2), ccsd.CcsdInputs(s))
    for R1, R2 in out.values():
        assert np.abs(R2 - Q2).max() < 1e-6 * np.abs(Q2).max()
        assert np.abs(R1 - Q1).max() < 1e-6 * np.abs(Q1).max()
    assert np.abs(out[8][1] - out[24][1]).max() < 1e-12 * np.abs(Q2).max()


@pytest.mark.parametrize("method,ppl", [("Ccsd", True), ("Ccd", True), ("Ccsd", False)])
def test_complex_residual_vjp_matches_finite_differences(emu_lib, method, ppl):
    """Complex path: the transposed-Jacobian product of the residual (reverse
    replay of the recorded planar schedule) against central differences of
    Re sum conj(Rbar) R(T) along complex directions in T and in the vertex; the
    adjoints are d/dRe + i d/dIm."""
    from cc4s_b200 import Solver
    No, Nv, NG = 3, 8, 6
    s = inputs.synthetic_system(No, Nv, NG, complex=True, seed=3)
    rng = np.random.default_rng(1)

    def c(shape):
        return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)

    def sym(x):
        return x + x.transpose(1, 0, 3, 2)
    T = (c((Nv, No)) * 0.1, sym(c((Nv, Nv, No, No))) * 0.05)
    Rb = (c((Nv, No)), c((Nv, Nv, No, No)))
    opts = {"method": method, "ppl": ppl}
    sol = Solver(opts, lib=emu_lib)
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=False)
    (T1b, T2b), Gb = sol.residual_vjp(T, Rb)

    def f(TT, gm=None):
        so = sol
        if gm is not None:
            so = Solver(opts, lib=emu_lib)
            so.set_inputs(s.eps_h, s.eps_p, gm, half_grid=False)
        return sum(np.real(np.conj(a) * b).sum() for a, b in zip(Rb, so.residual(TT)))
    d = (c((Nv, No)) * (method == "Ccsd"), sym(c((Nv, Nv, No, No))))
    h = 1e-5
    fd = (f((T[0] + h * d[0], T[1] + h * d[1])) - f((T[0] - h * d[0], T[1] - h * d[1]))) / (2 * h)
    an = np.real(np.conj(T1b) * d[0]).sum() + np.real(np.conj(T2b) * d[1]).sum()
    assert abs(fd - an) < 1e-7 * abs(fd)
    dg = c(s.gamma.shape)
    fdg = (f(T, s.gamma + h * dg) - f(T, s.gamma - h * dg)) / (2 * h)
    assert abs(fdg - np.real(np.conj(Gb) * dg).sum()) < 1e-8 * abs(fdg)


@pytest.mark.parametrize("method", ["Ccsd", "Ccd"])
def test_complex_relaxed_gradient_matches_finite_differences(emu_lib, method):
    """Complex path: Lambda equations by transposed-Jacobian products, relaxed
    dE_c/dGamma (d/dRe + i d/dIm) against central differences of re-converged
    energies, to 1e-6 relative.  The directions keep the vertex Hermitian
    (Gamma_qp = conj(Gamma_pq)), the symmetry under which the integrals are pair
    symmetric (V_abij = V_baji) and the amplitude iteration keeps T_abij = T_baji.
    The differences are Richardson-extrapolated from steps 1e-5 and 5e-6 (these
    Hermitian directions are long enough for an O(h^2) error of a few 1e-6)."""
    from cc4s_b200 import Solver
    s = inputs.synthetic_system(3, 10, 16, complex=True, seed=2)
    opts = dict(method=method, maxIterations=80, energyConvergence=1e-14,
                amplitudesConvergence=1e-12)

    def energy(gm):
        so = Solver(opts, lib=emu_lib)
        so.set_inputs(s.eps_h, s.eps_p, gm, half_grid=False)
        return so, so.run()["correlation"]
    sol, _ = energy(s.gamma)
    g, info = sol.relaxed_gradient(max_iterations=100, convergence=1e-12)
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
