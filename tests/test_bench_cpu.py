"""The JSON lines of bench.py's secondary modes (--triples, --fsc) and of the
reference arm, produced on the host: the library calls go to the CPU emulation
library (tests/emu), the device-only calls are stood in for, and the emulated
device times (0 s) are floored.  This checks the keys of each line, not numbers."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))

SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.environ["REPO_ROOT"])
from cc4s_b200 import _abi
_abi.DEFAULT_LIB = os.environ["EMU_LIB"]   # the CPU emulation build of the same ABI
import torch
torch.cuda.set_device = lambda *a, **k: None
torch.cuda.synchronize = lambda *a, **k: None
import bench
_median = bench.statistics.median
bench.statistics.median = lambda xs: max(_median(list(xs)), 1e-3)
bench.dgemm_peak = lambda local: 35.0
from cc4s_b200 import coupled_cluster as ccm
_stats = ccm.Solver.stats
def _floored_stats(self):
    d = _stats(self)
    for k in ("gemm_seconds", "split_seconds", "top_seconds"):
        d[k] = max(d[k], 1e-3)
    return d
ccm.Solver.stats = _floored_stats
_all_max = bench.all_max
bench.all_max = lambda x, world: max(_all_max(x, world), 1e-3)
sys.argv = ["bench.py"] + json.loads(os.environ["BENCH_ARGS"])
if __name__ == "__main__":
    bench.main()
"""

COMMON = {"metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
          "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config", "e2e"}


def _line(lib, args):
    env = dict(os.environ, EMU_LIB=lib, REPO_ROOT=ROOT, BENCH_ARGS=json.dumps(args))
    out = subprocess.run([sys.executable, "-c", SCRIPT], env=env, capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stdout[-2000:] + out.stderr[-2000:]
    return json.loads(out.stdout.strip().splitlines()[-1])


def test_triples_line():
    import build_emu
    line = _line(build_emu.build(), ["--triples", "--shape", "2,6,10", "--warmup", "1",
                                      "--steps", "1"])
    assert COMMON <= set(line)
    assert {"roofline", "cpu_baseline", "gpu_launches", "clocks"} <= set(line)
    assert set(line["config"]["forms"]) == {"fp64", "split3"}
    assert line["cpu_baseline"]["kind"] == "port" and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] > 0


def test_triples_cT_line():
    """--cT: the completely renormalised branch; device and operator energies agree."""
    import build_emu
    line = _line(build_emu.build(), ["--triples", "--cT", "--shape", "2,6,10", "--warmup", "0",
                                      "--steps", "1", "--precision", "fp64",
                                      "--no-cpu-baseline"])
    assert "cT=1" in line["config"]["workload"]
    e = line["config"]["forms"]["fp64"]["energy"]
    assert abs(line["e2e"]["energy"] - e) < 1e-12 * max(1.0, abs(e))


def test_fsc_line():
    import build_emu
    line = _line(build_emu.build(), ["--fsc", "--shape", "2,6,10", "--fsc-grid", "4",
                                      "--fsc-n", "2", "--warmup", "1", "--steps", "1"])
    assert COMMON <= set(line)
    assert line["config"]["points"] == (2 * 2) ** 3 * 64
    assert line["config"]["box"] == [4, 4, 4]
    assert {"cpu_baseline", "gpu_launches"} <= set(line)


def test_reference_line():
    import build_emu
    line = _line(build_emu.build(), ["--impl", "reference", "--config", "c0", "--warmup", "1",
                                      "--steps", "1"])
    assert line["impl"] == "reference"
    assert COMMON <= set(line)
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["value"] == line["value"]


def test_ccsd_line():
    """The default line (both forms at one GPU) on a small custom shape."""
    import build_emu
    line = _line(build_emu.build(), ["--shape", "3,9,14", "--warmup", "3", "--steps", "1"])
    assert COMMON <= set(line)
    assert {"roofline", "cpu_baseline", "gpu_launches", "clocks"} <= set(line)
    assert {"bound", "achieved", "peak", "unit", "frac", "traffic"} <= set(line["roofline"])
    assert {"value", "unit", "cores", "kind", "sample"} <= set(line["cpu_baseline"])
    assert {"value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"} <= set(line["e2e"])
    assert "split_speedup_vs_fp64" in line["config"] and line["n_gpus"] == 1
    assert line["warmup"] == 3 and line["steps"] == 1


def test_default_benchmark_command_fits_its_limit():
    """`bench.py --gpus 1 --steps 20 --warmup 5` at c2 (the measured seconds per
    iteration of both forms) projects well inside the 1800 s limit of a bench
    step, and the FP64 comparison is not skipped by the default 1500 s budget."""
    import bench
    legs = bench.projected_seconds(5, 20)
    total = sum(legs.values())
    assert total < 1200, legs
    before_fp64 = total - legs["fp64"] - legs["dgemm_peak"] - legs["cpu_baseline"]
    projected_fp64 = ((2 - 1 + 2) * bench.FP64_OVER_SPLIT_BOUND * bench.MEASURED_C2["split3"]
                      + 60.0)
    assert before_fp64 + projected_fp64 < 1500


def test_adjoint_line():
    """--adjoint: both backward forms, their finite-difference checks and timings."""
    import build_emu
    line = _line(build_emu.build(), ["--adjoint", "--shape", "2,32,40", "--fd-directions", "1"])
    assert set(line["forms"]) == {"fp64", "split3"}
    for f in line["forms"].values():
        assert f["lambda_converged"] and len(f["fd_directions"]) == 1
        assert f["fd_max_rel_err"] < 1e-5
    assert "max_abs_diff_vs_fp64_over_max" in line["forms"]["split3"]


def test_converge_line():
    """--converge: split form, FP64 from the split amplitudes, FP64 from T = 0."""
    import build_emu
    line = _line(build_emu.build(), ["--converge", "--shape", "2,32,40",
                                      "--converge-energy", "1e-10"])
    forms = line["forms"]
    assert set(forms) == {"split3", "fp64_from_split", "fp64"}
    assert line["value"] == forms["split3"]["abs_dE_vs_fp64"] < 1e-6
    assert forms["fp64"]["abs_dE_vs_fp64_from_split"] < 1e-9
    assert forms["fp64_from_split"]["iterations"] < forms["fp64"]["iterations"]
    assert len(forms["split3"]["history_residuum_norm"]) == forms["split3"]["iterations"]
