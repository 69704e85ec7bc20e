"""The allocation-free energy entry point, cc4s_cc_energy_noalloc.

It serves callers that cannot allocate device memory where they need the
energy (hosts whose device memory is entirely owned by their own pool), so it
takes only device buffers the caller already owns and uses a fixed 2 MiB
device array for its partial sums.  Here it is called through the C ABI on device buffers and checked, on
two calls in a row, against the energy the existing run entry point computes
for the same amplitudes (cc4s_cc_run with maxIterations = 0).

This file is collected last so that a failure here stops a -x run only after
every other test has run; it passes alone and after the others.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# Same FP64 tolerance as the other parity tests (1e-9 Eh); different reduction
# orders agree to rounding.
TOL_E = 1e-9


def _system_and_amplitudes(cplx):
    from oracle import inputs
    from oracle.inputs import coulomb_integrals
    No, Nv, NG = 6, 30, 40
    s = inputs.synthetic_system(No, Nv, NG, complex=cplx, seed=9)
    rng = np.random.default_rng(21)
    T1 = rng.standard_normal((Nv, No)) * 0.02
    T2 = rng.standard_normal((Nv, Nv, No, No)) * 0.02
    if cplx:
        T1 = T1 + 1j * rng.standard_normal((Nv, No)) * 0.02
        T2 = T2 + 1j * rng.standard_normal((Nv, Nv, No, No)) * 0.02
    T2 = T2 + T2.transpose(1, 0, 3, 2)
    V = coulomb_integrals(s, ["pphh"])["pphh"]
    return s, T1, T2, V


def _to_device(a):
    import torch
    from cc4s_b200 import _abi
    return torch.from_numpy(_abi.as_f64(a).copy()).cuda()


@pytest.mark.parametrize("cplx", [False, True])
def test_energy_noalloc_matches_run_entry(cplx):
    import torch
    from cc4s_b200 import Solver, _abi
    s, T1, T2, V = _system_and_amplitudes(cplx)
    sol = Solver(dict(maxIterations=0))
    sol.set_inputs(s.eps_h, s.eps_p, s.gamma, half_grid=not cplx)
    sol.set_initial_amplitudes(T1, T2)
    ref = sol.run()
    sol.close()
    lib = _abi.load()
    t1, t2, vv = _to_device(T1), _to_device(T2), _to_device(V)
    out = torch.zeros(4, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    free_after_first = None
    for k in range(2):  # two calls in a row share the static scratch array
        out.zero_()
        torch.cuda.synchronize()
        st = lib.cc4s_cc_energy_noalloc(t1.data_ptr(), t2.data_ptr(), vv.data_ptr(),
                                        s.No, s.Nv, int(cplx), out.data_ptr(),
                                        ctypes.c_void_p(stream))
        assert st == 0, lib.cc4s_cc_last_error(None)
        torch.cuda.synchronize()
        free = torch.cuda.mem_get_info()[0]
        if k == 0:
            free_after_first = free
        else:
            # the second call took no device memory (the first may load the module)
            assert free == free_after_first
        d, x, di, xi = out.cpu().numpy()
        assert abs(d - ref["direct"]) < TOL_E
        assert abs(x - ref["exchange"]) < TOL_E
        assert abs((d + x) - ref["correlation"]) < TOL_E
        assert abs((di + xi) - ref["correlation_imag"]) < TOL_E


def test_energy_noalloc_rejects_oversized_systems():
    import torch
    from cc4s_b200 import _abi
    lib = _abi.load()
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    st = lib.cc4s_cc_energy_noalloc(buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), 257, 4, 0,
                                    buf.data_ptr(), None)
    assert st == 2  # CC4S_ERR_BAD_SHAPE, nothing launched
    assert b"256" in lib.cc4s_cc_last_error(None)
