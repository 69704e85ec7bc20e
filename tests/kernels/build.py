"""Builds tests/kernels/_build/split_check (test infrastructure: kernel-level check
and timing of the split-precision contraction against the FP64 one)."""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
CSRC = os.path.join(ROOT, "cc4s_b200", "csrc")
OUT = os.path.join(HERE, "_build", "split_check")


def build():
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    srcs = [os.path.join(HERE, "split_check.cu"), os.path.join(CSRC, "split_gemm.cu"),
            os.path.join(CSRC, "gemm_f64.cu")]
    deps = srcs + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    if os.path.exists(OUT) and os.path.getmtime(OUT) > max(os.path.getmtime(d) for d in deps):
        return OUT
    nvcc = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17",
                    "-lineinfo", "-o", OUT] + srcs + ["-lcuda"], check=True)
    return OUT


if __name__ == "__main__":
    print(build())
