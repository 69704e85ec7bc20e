"""Builds the test-only CPU emulation library (see ops_emu.cpp)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "cc4s_b200", "csrc")
OUT = os.path.join(HERE, "_build", "libcc4s_emu.so")
SCHEDULE_SOURCES = ("schedule.cpp", "ccsd_real.cpp", "ccsd_complex.cpp", "drccd.cpp",
                    "driver.cpp", "abi.cpp", "triples.cpp")


def build():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    srcs = ([os.path.join(HERE, "ops_emu.cpp"), os.path.join(HERE, "ein_probe.cpp")] +
            [os.path.join(CSRC, f) for f in SCHEDULE_SOURCES])
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    deps.append(os.path.join(ROOT, "include", "cc4s_cc.h"))
    if os.path.exists(OUT) and os.path.getmtime(OUT) > max(os.path.getmtime(d) for d in deps):
        return OUT
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-Wall", "-I/usr/local/cuda/include",
           "-o", OUT] + srcs
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build())
