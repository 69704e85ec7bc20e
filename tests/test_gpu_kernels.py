"""Kernel-level check of the split-precision contraction on a B200: gemm_split
against the FP64 DMMA gemm on plain operands (tests/kernels/split_check.cu), on
the small shapes (ragged edges, transposed operands)."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "kernels"))


@pytest.mark.parametrize("shape", [0, 1, 2, 3])
def test_split_kernel_against_fp64(shape):
    import build as kbuild
    exe = kbuild.build()
    r = subprocess.run([exe, str(shape)], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "errflag=0" in r.stdout
