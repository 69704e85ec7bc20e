"""The multi-rank path of bench.py (one replica of the workload per rank, device
time reduced as the maximum over ranks) run as two gloo ranks on the host, each
rank's library calls going to the CPU emulation library (tests/emu)."""
import json
import os
import socket
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "emu"))

RANK_SCRIPT = r"""
import json, os, sys
sys.path.insert(0, os.environ["REPO_ROOT"])
from cc4s_b200 import _abi
_abi.DEFAULT_LIB = os.environ["EMU_LIB"]   # the CPU emulation build of the same ABI
import torch.distributed as dist
dist.init_process_group("gloo", init_method="env://")
rank, world = dist.get_rank(), dist.get_world_size()
import bench
from cc4s_b200.synthetic import synthetic
inputs = synthetic(3, 9, 14, complex=False, seed=4)
opts = dict(maxIterations=3, energyConvergence=-1.0, amplitudesConvergence=-1.0,
            mixer=dict(type="DiisMixer", maxResidua=5))
r = bench.timed_run(opts, inputs, 1, 2, world, 0, keep_amplitudes=False)
out = {"rank": rank, "t": r["t"], "energy": r["r"]["correlation"],
       "max": bench.all_max(1.5 + rank, world), "launches": r["launches"]}
bench.barrier(world)
json.dump(out, open(os.environ["OUT_PREFIX"] + str(rank) + ".json", "w"))
dist.destroy_process_group()
"""


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_gloo_replicas(tmp_path):
    import build_emu
    from oracle import coupled_cluster, inputs
    lib = build_emu.build()
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                   RANK=str(rank), LOCAL_RANK="0", EMU_LIB=lib, REPO_ROOT=ROOT,
                   OUT_PREFIX=str(tmp_path / "rank"))
        procs.append(subprocess.Popen([sys.executable, "-c", RANK_SCRIPT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    for p in procs:
        out, _ = p.communicate(timeout=240)
        assert p.returncode == 0, out.decode()[-2000:]
    res = [json.load(open(tmp_path / ("rank%d.json" % r))) for r in range(2)]
    # the device-time reduction is the maximum over ranks
    assert res[0]["max"] == res[1]["max"] == 2.5
    assert res[0]["t"] == res[1]["t"]
    # every replica runs the same workload to the same energy, the oracle's
    s = inputs.synthetic_system(3, 9, 14, seed=4)
    ref = coupled_cluster.run(s, maxIterations=3, energyConvergence=-1.0,
                              amplitudesConvergence=-1.0, mixer=dict(type="DiisMixer", maxResidua=5))
    for r in res:
        assert abs(r["energy"] - ref["energy"]["correlation"]) < 1e-10 * max(1.0, abs(r["energy"]))
        assert r["launches"] > 0


RUN_OURS_SCRIPT = r"""
import json, os, sys, argparse
sys.path.insert(0, os.environ["REPO_ROOT"])
from cc4s_b200 import _abi
_abi.DEFAULT_LIB = os.environ["EMU_LIB"]   # the CPU emulation build of the same ABI
import torch, torch.distributed as dist
dist.init_process_group("gloo", init_method="env://")
torch.cuda.set_device = lambda *a, **k: None     # host-only stand-ins for the device calls
torch.cuda.synchronize = lambda *a, **k: None
import bench
from cc4s_b200 import coupled_cluster as ccm
_stats = ccm.Solver.stats
def _floored_stats(self):                        # emulated events read 0 s
    d = _stats(self)
    for k in ("gemm_seconds", "split_seconds", "top_seconds"):
        d[k] = max(d[k], 1e-3)
    return d
ccm.Solver.stats = _floored_stats
bench.dgemm_peak = lambda local: 35.0
_all_max = bench.all_max
bench.all_max = lambda x, world: max(_all_max(x, world), 1e-3)  # emulated events read 0 s
bench.CONFIG_SHAPES["custom"] = (3, 9, 14)
args = argparse.Namespace(config="custom", steps=1, warmup=1, precision="both", vertex_scale=None,
                          time_budget=1500.0, e2e_iterations=2, fp64_steps=2, fp64_warmup=2)
line = bench.run_ours(args, dist.get_world_size(), dist.get_rank(), 0)
json.dump(line, open(os.environ["OUT_PREFIX"] + str(dist.get_rank()) + ".json", "w"))
dist.destroy_process_group()
"""


def test_two_gloo_ranks_run_the_bench_replica_line(tmp_path):
    """The whole replica line of bench.py at world size 2: both ranks take the same
    collective steps, only the headline split form is timed, n_gpus and the
    aggregate value count both replicas."""
    import build_emu
    lib = build_emu.build()
    port = _free_port()
    procs = []
    for rank in range(2):
        env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2",
                   RANK=str(rank), LOCAL_RANK="0", EMU_LIB=lib, REPO_ROOT=ROOT,
                   OUT_PREFIX=str(tmp_path / "line"))
        procs.append(subprocess.Popen([sys.executable, "-c", RUN_OURS_SCRIPT], env=env,
                                      stdout=subprocess.PIPE, stderr=subprocess.STDOUT))
    for p in procs:
        out, _ = p.communicate(timeout=300)
        assert p.returncode == 0, out.decode()[-3000:]
    lines = [json.load(open(tmp_path / ("line%d.json" % r))) for r in range(2)]
    for line in lines:
        assert line["n_gpus"] == 2
        assert line["config"]["parallelism"] == "replicas"
        assert line["config"]["precision"] == "split3"
        assert "fp64_s_per_iter" not in line["config"]
    assert lines[0]["value"] == lines[1]["value"]
