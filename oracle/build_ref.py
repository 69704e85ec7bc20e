"""Builds oracle/_ref/libref_tricubic.so: the reference's tricubic interpolator
(src/main/gte/TricubicInterpolation.hpp and the cc4s headers it includes,
compiled where they lie under the reference tree) behind oracle/ref_tricubic.cpp.

Test infrastructure: only the tests use the library, as the checker of the
oracle's restatement.  The reference tree must be present (it is not on the GPU
hosts); the rest of the reference's FiniteSizeCorrection needs CTF and MPI and
is not built.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE = os.environ.get("CC4S_REFERENCE_TREE", "/root/reference")
OUT = os.path.join(HERE, "_ref", "libref_tricubic.so")


def available():
    return os.path.exists(os.path.join(REFERENCE, "src", "main", "gte",
                                       "TricubicInterpolation.hpp"))


def build():
    """Compiles the library if the reference tree is present; returns its path or None."""
    if not available():
        return None
    src = os.path.join(HERE, "ref_tricubic.cpp")
    hdr = os.path.join(REFERENCE, "src", "main", "gte", "TricubicInterpolation.hpp")
    if os.path.exists(OUT) and os.path.getmtime(OUT) > max(os.path.getmtime(src),
                                                          os.path.getmtime(hdr)):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    subprocess.run(["g++", "-O2", "-std=c++17", "-fPIC", "-shared",
                    "-I", os.path.join(REFERENCE, "src", "main"), src, "-o", OUT], check=True)
    return OUT


if __name__ == "__main__":
    print(build() or "reference tree not present")
    sys.exit(0)
