"""The C-ABI library builds for sm_100a, loads without a GPU and exports every
symbol that include/cc4s_cc.h declares (no compute calls)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "cc4s_cc.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(cc4s_cc_[a-z_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib_path():
    from cc4s_b200 import build
    return build.build()


def test_header_declarations_match_binding():
    from cc4s_b200 import _abi
    assert declared_symbols() == sorted(_abi.EXPORTS)


def test_library_loads_and_exports(lib_path):
    lib = ctypes.CDLL(lib_path)
    for name in declared_symbols():
        assert hasattr(lib, name), name


def test_default_options_without_gpu(lib_path):
    from cc4s_b200 import _abi
    lib = _abi.load(lib_path)
    o = _abi.Options()
    lib.cc4s_cc_default_options(ctypes.byref(o))
    assert (o.method, o.mixer, o.max_residua, o.max_iterations) == (0, 0, 4, 16)
    assert o.energy_convergence == 1e-7 and o.amplitudes_convergence == 1e-6
    assert o.ppl == 1 and o.level_shift == 0.0


def test_missing_library_fails_loudly(tmp_path):
    from cc4s_b200 import _abi
    with pytest.raises(RuntimeError):
        _abi.load(str(tmp_path / "nonexistent.so"))
