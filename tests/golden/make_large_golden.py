"""Regenerates the oracle fixtures at the FP64 parity sizes (self-made goldens).

Run from the repository root:  python tests/golden/make_large_golden.py [c1] [c4]

c1 (No=32, Nv=256, NG=1024, seed 0): the first four CoupledCluster iterations
from T = 0 with DIIS depth 5 (CoupledCluster.cxx:56-191, Ccsd.cxx:77-378,
DiisMixer.cxx:28-146): the energy and residuum norm of every iteration, the
final correlation/direct/exchange energies, and the final amplitudes as norms,
seeded weighted checksums and seeded element samples (the full T2 is 0.5 GB).

c4 (No=32, Nv=320, NG=1600, seed 0): one residual evaluation at seeded random
amplitudes (the same draw as tests/test_gpu_ccsd.py's _rand_T), stored the same
way.

The arrays go to <name>.npz, the scalars to <name>.json.  A full oracle
iteration at these sizes takes minutes on a CPU; that is why the results are
committed instead of recomputed by the GPU tests.
"""
import json
import os
import sys
import time
import warnings

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
warnings.simplefilter("ignore")

from oracle import ccsd, coupled_cluster, inputs  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
N_SAMPLE_T1 = 4096
N_SAMPLE_T2 = 16384


def summary(prefix, A, seed):
    """Norm, weighted checksum (weights N(0,1) from `seed`) and an element sample."""
    rng = np.random.default_rng(seed)
    flat = A.reshape(-1, order="F")
    n = N_SAMPLE_T1 if A.ndim == 2 else N_SAMPLE_T2
    idx = np.sort(rng.choice(flat.size, size=min(n, flat.size), replace=False))
    w = rng.standard_normal(flat.size)
    scal = {prefix + "_norm": float(np.sqrt((flat * flat).sum())),
            prefix + "_checksum": float(w @ flat), prefix + "_max": float(np.abs(flat).max())}
    return scal, {prefix + "_idx": idx, prefix + "_val": flat[idx]}


def c1():
    opts = dict(method="Ccsd", maxIterations=4, energyConvergence=1e-10,
                amplitudesConvergence=1e-6, mixer=dict(type="DiisMixer", maxResidua=5))
    s = inputs.config_system("c1", seed=0)
    t0 = time.perf_counter()
    r = coupled_cluster.run(s, **opts)
    T1, T2 = r["amplitudes"]
    out = dict(source="oracle (self-made golden), tests/golden/make_large_golden.py", config="c1",
               seed=0, options=opts, iterations=r["iterations"], energy=r["energy"],
               history_energy=[h["energy"] for h in r["history"]],
               history_dR=[h["dR"] for h in r["history"]],
               oracle_seconds=time.perf_counter() - t0)
    arrays = {}
    for name, A, seed in (("T1", T1, 101), ("T2", T2, 102)):
        sc, ar = summary(name, A, seed)
        out.update(sc)
        arrays.update(ar)
    out.update(sample_seeds={"T1": 101, "T2": 102})
    json.dump(out, open(os.path.join(HERE, "c1_seed0_4it.json"), "w"), indent=1)
    np.savez_compressed(os.path.join(HERE, "c1_seed0_4it.npz"), **arrays)


def rand_T(rng, Nv, No, scale=0.02):
    T1 = rng.standard_normal((Nv, No)) * scale
    T2 = rng.standard_normal((Nv, Nv, No, No)) * scale
    return T1, T2 + T2.transpose(1, 0, 3, 2)


def c4():
    s = inputs.config_system("c4", seed=0)
    rng = np.random.default_rng(4)
    T = rand_T(rng, s.Nv, s.No)
    t0 = time.perf_counter()
    R1, R2 = ccsd.residuum(T, ccsd.CcsdInputs(s))
    out = dict(source="oracle (self-made golden), tests/golden/make_large_golden.py", config="c4",
               seed=0, amplitudes="rand_T(default_rng(4), Nv, No, 0.02)",
               oracle_seconds=time.perf_counter() - t0)
    arrays = {}
    for name, A, seed in (("R1", R1, 201), ("R2", R2, 202)):
        sc, ar = summary(name, A, seed)
        out.update(sc)
        arrays.update(ar)
    out.update(sample_seeds={"R1": 201, "R2": 202})
    json.dump(out, open(os.path.join(HERE, "c4_seed0_residual.json"), "w"), indent=1)
    np.savez_compressed(os.path.join(HERE, "c4_seed0_residual.npz"), **arrays)


if __name__ == "__main__":
    which = sys.argv[1:] or ["c1", "c4"]
    for name in which:
        {"c1": c1, "c4": c4}[name]()
        print(name, "done", flush=True)
