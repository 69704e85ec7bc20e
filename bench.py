"""Benchmark of the CoupledCluster (CCSD) step on B200.

A "step" is one CCSD iteration (residual, Jacobi update, DIIS, energy) on a
seeded synthetic system.  Default workload: No=64, Nv=640, NG=2560, real
(T2 13.4 GB), both the split-precision tensor-core form (headline) and the
FP64 form, W warm-up and K timed iterations each.  T2 and the vertex are far
larger than L2, so no flush is needed between iterations.

value: reference-equivalent TFLOP/s = F_ref / (s per iteration), with F_ref
the flop count of the reference's formulation (cc4s_b200.flops), timed with
CUDA events on the library's stream inside the library, max over ranks.
e2e: the same metric through the C ABI from host buffers: set_inputs (vertex
upload and integral build) + the first (MP2) iteration + K full iterations +
amplitude download, wall clock; only the K full iterations' flops count.

Multi-GPU: every rank runs its own replica of the workload (weak scaling, no
collective on the data path); value is the sum over ranks.

--impl reference: the CPU restatement of the reference (the oracle; the
reference itself needs MPI and the Cyclops Tensor Framework, which are not
installed) timed on this host's cores on a bounded sample of the same
workload.
--adjoint: relaxed-gradient (Lambda equations) timing and finite-difference
check; --converge: converged energies of the FP64, split and refined forms;
--triples: the perturbative triples (T) step after CCSD; --fsc: the
FiniteSizeCorrection step.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
import warnings

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
warnings.simplefilter("ignore")

CONFIG_SHAPES = {
    "c0": (8, 40, 200), "c1": (32, 256, 1024), "c2": (64, 640, 2560), "c3": (48, 480, 3000),
    "c4": (32, 320, 1600),
}
COMPLEX_CONFIGS = {"c3"}  # complex vertex: 8 real flops per complex multiply-add
METRIC = "CCSD s/iter & TFLOP/s: TC split-precision vs FP64 on 1 B200 at |ΔEc|≤1µEh"


def peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.stop = threading.Event()

    def _run(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits"], capture_output=True,
                                     text=True, timeout=5).stdout.strip()
                if out:
                    self.rows.append([x.strip() for x in out.split(",")])
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        self.t = threading.Thread(target=self._run, daemon=True)
        self.t.start()
        return self

    def __exit__(self, *a):
        self.stop.set()
        self.t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4)
                          if len(r) > 5 + k and r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def dgemm_peak(device):
    """FP64 tensor peak measured here: cuBLAS DGEMM 8192^3, best of 5 (CUDA events)."""
    import torch
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    best = 1e30
    for k in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        if k:
            best = min(best, s.elapsed_time(e) * 1e-3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


def cpu_sample(cfg, target=2e12):
    """CPU rate of the oracle on the workload's dominant contractions (bounded sample).

    Times, with the oracle's numpy/BLAS restatement on all host cores, a block of
    the (vo)^3 ring contraction (virtual indices a, b restricted to n values) and
    one particle-particle-ladder slice pair (sl x sl virtual pairs, occupied pairs
    restricted to m x m), each sized to about `target` flops, on random operands
    of the workload's shapes; the measured rate converts the reference
    formulation's flops into seconds per iteration.
    """
    import numpy as np
    from oracle import ccsd as occ
    from cc4s_b200.flops import reference_flops
    o, v, G = CONFIG_SHAPES[cfg]
    rng = np.random.default_rng(0)
    n = int(min(v, max(1, (target / (2.0 * v * o ** 3)) ** 0.5)))
    Y = rng.standard_normal((n, o, o, v))
    X = rng.standard_normal((v, n, o, o))
    m = min(o, 16)
    sl = int(min(o, max(1, (target / (2.0 * v * v * (G + m * m))) ** 0.5)))
    dG = rng.standard_normal((G, 2 * sl, v)) * 0.1 * G ** -0.25
    Xl = rng.standard_normal((v, v, m, m))
    t0 = time.perf_counter()
    occ.es("akic,cbkj->abij", Y, X)
    V = occ.es("Gxc,Gyd->xycd", dG[:, :sl, :], dG[:, sl:, :])
    occ.es("xycd,cdij->xyij", V, Xl)
    t1 = time.perf_counter()
    flops = 2.0 * n * n * v * o ** 3 + 2.0 * sl * sl * v * v * (G + m * m)
    rate = flops / (t1 - t0)
    s_iter = reference_flops(o, v, G, complex=cfg in COMPLEX_CONFIGS) / rate
    return dict(s_per_iter=s_iter, rate_tflops=rate / 1e12, sample_seconds=t1 - t0,
                cores=os.cpu_count(),
                sample="oracle numpy/BLAS on %s: ring block a,b < %d of akic,cbkj->abij and one "
                       "ladder slice pair (%d x %d virtuals, %d x %d occupied pairs), %.2g flops; "
                       "s/iter = reference flops / measured rate" % (cfg, n, sl, sl, m, m, flops))


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def all_max(x, world):
    """Maximum of x over the ranks (NCCL on the GPUs; gloo ranks on the host use CPU tensors)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    import torch
    if torch.cuda.is_available():
        torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def timed_run(opts, inputs, W, K, world, local, keep_amplitudes=True):
    """W + K iterations; the last K are timed (CUDA events on the library stream)."""
    from cc4s_b200 import Solver
    eh, ep, g, hg = inputs
    sol = Solver(opts)
    sol.set_inputs(eh, ep, g, half_grid=hg)
    st0 = sol.stats()
    barrier(world)
    with ClockSampler(local) as clk:
        r = sol.run()
    barrier(world)
    st1 = sol.stats()
    secs = [h["seconds"] for h in r["history"]]
    t = all_max(sum(secs[W:W + K]), world)
    launches = ((st1["gemm_launches"] - st0["gemm_launches"]) +
                (st1["other_launches"] - st0["other_launches"])) / (W + K)
    T = sol.amplitudes() if keep_amplitudes else None
    sol.close()
    return dict(t=t, r=r, launches=launches, T=T, clocks=clk.summary())


def run_ours(args, world, rank, local):
    import torch
    from cc4s_b200 import Solver, reference_flops
    from cc4s_b200.synthetic import config
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    if cfg == "custom":
        from cc4s_b200.synthetic import synthetic
        inputs = synthetic(o, v, G, complex=False, seed=0)
    else:
        inputs = config(cfg, seed=0)
    eh, ep, g, hg = inputs
    if args.vertex_scale is not None:
        g *= args.vertex_scale
    F = reference_flops(o, v, G, complex=cfg in COMPLEX_CONFIGS)
    K, W = args.steps, args.warmup
    base = dict(maxIterations=W + K, energyConvergence=-1.0, amplitudesConvergence=-1.0,
                mixer=dict(type="DiisMixer", maxResidua=5), device=local)
    # the FP64 form is the single-GPU comparison of the two forms; replicas under
    # torchrun time the headline form only, so the GPUs are held for less time
    if args.precision == "both":
        forms = ["fp64", "split3"] if world == 1 else ["split3"]
    else:
        forms = [args.precision]
    head = "split3" if "split3" in forms else "fp64"
    runs = {p: timed_run(dict(base, precision=p), inputs, W, K, world, local,
                         keep_amplitudes=(p == head)) for p in forms}
    hr = runs[head]
    t = hr["t"]
    # dominant kernel: per-launch CUDA events around every contraction of one
    # residual, evaluated at the amplitudes the timed run ended with
    prof = Solver(dict(base, precision=head, profile=True, maxIterations=1))
    prof.set_inputs(eh, ep, g, half_grid=hg)
    prof.set_initial_amplitudes(*hr["T"])
    hr["T"] = None
    prof.run()
    ps = prof.stats()
    prof.close()
    pk = peaks()
    dpeak = dgemm_peak(local)
    if head == "split3":
        # executed FP16 tensor work: six slice products per FP64-equivalent multiply-add
        achieved = 6.0 * ps["split_flops"] / ps["split_seconds"] / 1e12
        peak = pk.get("bf16_tflops_sustained", 1405.3)
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": "split_kernel (tcgen05.mma kind::f16, TMEM, TMA) incl. operand slicing, "
                          "%d launches of one residual" % ps["split_launches"],
                "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)",
                "fp64_equivalent_tflops": ps["split_flops"] / ps["split_seconds"] / 1e12}
    else:
        achieved = ps["gemm_flops"] / ps["gemm_seconds"] / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": dpeak, "unit": "TFLOP/s",
                "frac": achieved / dpeak, "traffic": None,
                "kernel": "gemm_f64_kernel (mma.sync m16n8k16 f64), all %d contraction launches "
                          "of one residual" % ps["gemm_profiled_launches"],
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured; no FP64 "
                               "entry in MEASURED_PEAKS.json)",
                "top_launch_tflops": ps["top_flops"] / ps["top_seconds"] / 1e12}
    # end to end through the C ABI from host buffers
    barrier(world)
    t0 = time.perf_counter()
    # the first iteration is the cheap one (R = V, the MP2 step); K full
    # iterations follow it, and only their flops are counted
    e2e = Solver(dict(base, precision=head, maxIterations=K + 1))
    e2e.set_inputs(eh, ep, g, half_grid=hg)
    re = e2e.run()
    A1, A2 = e2e.amplitudes()
    torch.cuda.synchronize()
    t_e2e = all_max(time.perf_counter() - t0, world)
    e2e.close()
    h2d = (g.nbytes + eh.nbytes + ep.nbytes) / K
    d2h = (A1.nbytes + A2.nbytes) / K + 5 * 8 + 8
    kind = "complex" if cfg in COMPLEX_CONFIGS else "real"
    conf = {"workload": "CCSD %s: No=%d Nv=%d NG=%d %s, DIIS 5, %s" % (cfg, o, v, G, kind, head),
            "precision": head, "s_per_iter": t / K,
            "flops_per_iter_reference_formulation": F,
            "flops_per_iter_executed": hr["r"]["flops_per_iteration"],
            "l2": "inputs larger than L2 (T2 %.2f GB)" % ((v * o) ** 2 * 8 / 1e9),
            "parallelism": "replicas" if world > 1 else "single GPU",
            "energy_after_steps": hr["r"]["correlation"],
            "fp64_dgemm_peak_tflops": dpeak}
    if "fp64" in runs and "split3" in runs:
        t64 = runs["fp64"]["t"]
        conf.update({"fp64_s_per_iter": t64 / K, "fp64_tflops": world * F / (t64 / K) / 1e12,
                     "split_speedup_vs_fp64": t64 / t,
                     "abs_dE_after_steps_split_vs_fp64":
                         abs(runs["split3"]["r"]["correlation"] - runs["fp64"]["r"]["correlation"])})
    line = {
        "metric": METRIC, "value": world * F / (t / K) / 1e12, "unit": "TFLOP/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": 1e3 * t / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the workload's distributions)",
        "config": conf,
        "e2e": {"value": world * F * K / t_e2e / 1e12, "unit": "TFLOP/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "seconds": t_e2e, "iterations": re["iterations"]},
        "gpu_launches": int(round(hr["launches"] * K)),
        "roofline": roof,
        "clocks": hr["clocks"],
    }
    return line


def run_adjoint(args, local):
    """Adjoint form at the workload: converged FP64 CCSD, Lambda equations by
    transposed-Jacobian products, relaxed dE_c/dGamma; times each against one
    forward iteration and checks the gradient against central differences of
    re-converged energies (step 1e-5) on a few random vertex directions."""
    import numpy as np
    import torch
    from cc4s_b200 import Solver
    from cc4s_b200.synthetic import config
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    eh, ep, g, hg = config(cfg, seed=0)
    scale = args.vertex_scale if args.vertex_scale is not None else 0.3
    g *= scale
    # tight enough for 1e-6 differences at step 1e-5, loose enough that the DIIS
    # changes do not vanish (a singular DIIS system ends the reference's run too)
    opts = dict(maxIterations=100, energyConvergence=1e-11, amplitudesConvergence=1e-9,
                mixer=dict(type="DiisMixer", maxResidua=5), device=local)

    def solve(gm):
        so = Solver(opts)
        so.set_inputs(eh, ep, gm, half_grid=hg)
        return so, so.run()
    sol, r = solve(g)
    fwd = statistics.median(h["seconds"] for h in r["history"][2:]) if r["iterations"] > 3 else \
        r["history"][-1]["seconds"]
    t0 = time.perf_counter()
    grad, info = sol.relaxed_gradient(max_iterations=100, convergence=1e-9)
    t_back = time.perf_counter() - t0
    sol.close()
    rng = np.random.default_rng(7)
    h = 1e-5
    checks = []
    for _ in range(args.fd_directions):
        d = rng.standard_normal(g.shape)
        ep_ = solve(g + h * d)[1]["correlation"]
        em_ = solve(g - h * d)[1]["correlation"]
        fd = (ep_ - em_) / (2 * h)
        an = float((grad * d).sum())
        checks.append({"fd": fd, "adjoint": an, "rel_err": abs(fd - an) / abs(fd)})
    return {"metric": "CCSD adjoint: relaxed dE_c/dGamma (Lambda equations) vs one forward iteration",
            "value": (info["vjp_seconds"] / fwd) if fwd else None, "unit": "x forward iteration",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "CCSD %s: No=%d Nv=%d NG=%d real, DIIS 5, FP64" % (cfg, o, v, G),
                       "vertex_scale": scale,
                       "forward_iterations": r["iterations"], "forward_s_per_iter": fwd,
                       "energy": r["correlation"],
                       "lambda_iterations": info["iterations"], "lambda_converged": info["converged"],
                       "lambda_residuum_norm": info["residuum_norm"],
                       "prepare_seconds": info["prepare_seconds"],
                       "lambda_s_per_iter": info["vjp_seconds"],
                       "gradient_seconds": info["gradient_seconds"],
                       "backward_total_seconds": t_back,
                       "backward_total_vs_forward_iteration": t_back / fwd if fwd else None},
            "fd_check": {"step": h, "directions": checks,
                         "max_rel_err": max((c["rel_err"] for c in checks), default=None)}}


def run_converge(args, local):
    """Accuracy of the split form at convergence: FP64, pure split and split with
    FP64 refinement, each to energyConvergence 1e-10 (DIIS 5, at most 80
    iterations); reports |E_split - E_fp64|, iterations and time to solution.
    The synthetic vertex is scaled (default 0.3): unscaled, CCSD diverges at
    these sizes."""
    import torch
    from cc4s_b200 import Solver
    from cc4s_b200.synthetic import config
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    eh, ep, g, hg = config(cfg, seed=0)
    scale = args.vertex_scale if args.vertex_scale is not None else 0.3
    g *= scale
    base = dict(maxIterations=80, energyConvergence=1e-10, amplitudesConvergence=1e-8,
                mixer=dict(type="DiisMixer", maxResidua=5), device=local)
    forms = {"fp64": {}, "split3": dict(precision="split3"),
             "split3_refined": dict(precision="split3", precisionRefinement=args.refine)}
    out = {}
    for name, extra in forms.items():
        so = Solver(dict(base, **extra))
        so.set_inputs(eh, ep, g, half_grid=hg)
        r = so.run()
        so.close()
        out[name] = {"energy": r["correlation"], "iterations": r["iterations"],
                     "converged": r["converged"], "seconds": sum(h["seconds"] for h in r["history"]),
                     "refined_from": r["refined_from"],
                     "s_per_iter": [h["seconds"] for h in r["history"]]}
    e64 = out["fp64"]["energy"]
    for name in ("split3", "split3_refined"):
        out[name]["abs_dE_vs_fp64"] = abs(out[name]["energy"] - e64)
    kind = "complex" if cfg in COMPLEX_CONFIGS else "real"
    return {"metric": "CCSD converged |dE_c| split-precision vs FP64 (bound 1e-6 Eh)",
            "value": out["split3_refined"]["abs_dE_vs_fp64"], "unit": "Eh",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "CCSD %s: No=%d Nv=%d NG=%d %s, DIIS 5, energyConvergence 1e-10"
                                   % (cfg, o, v, G, kind),
                       "precision_refinement": args.refine, "vertex_scale": scale},
            "forms": out}


_TRIPLES_SAMPLE = {}


def _triples_worker_init(arrays):
    _TRIPLES_SAMPLE.update(arrays)


def _triples_worker(chunk):
    from oracle import triples as otr
    d = _TRIPLES_SAMPLE
    return sum(otr.tuple_energy(a, b, c, d["T1"], d["T2"], d["V"], d["eh"], d["ep"])
               for a, b, c in chunk)


def cpu_triples_sample(cfg, n=32):
    """CPU rate of the oracle's (T) tuple loop (the atrip formulation: per tuple
    twelve o^2 x o x (v or o) contractions, singles and energy), tuples spread
    over all host cores like atrip spreads them over ranks (one process per core,
    one BLAS thread each; spawned, so safe after GPU work), timed on the tuples
    a <= b <= c < n of the workload's shapes with random operands; the
    reference's flop count per tuple converts the rate to seconds."""
    import multiprocessing as mp
    import numpy as np
    from oracle import triples as otr
    o, v, G = CONFIG_SHAPES[cfg]
    n = min(n, v)
    rng = np.random.default_rng(0)
    arrays = {"T1": rng.standard_normal((n, o)) * 0.01,
              "T2": rng.standard_normal((n, v, o, o)) * 0.01,
              "V": {"pphh": rng.standard_normal((n, n, o, o)),
                    "ppph": rng.standard_normal((n, n, v, o)),
                    "hhhp": rng.standard_normal((o, o, o, n))},
              "eh": -1.0 - rng.random(o), "ep": 1.0 + rng.random(n)}
    work = otr.tuples(n)
    cores = os.cpu_count() or 1
    chunks = [work[k::cores] for k in range(cores)]
    old = os.environ.get("OPENBLAS_NUM_THREADS")
    os.environ["OPENBLAS_NUM_THREADS"] = "1"
    try:
        with mp.get_context("spawn").Pool(cores, _triples_worker_init, (arrays,)) as pool:
            pool.map(_triples_worker, [c[:2] for c in chunks])   # start-up, imports
            t0 = time.perf_counter()
            pool.map(_triples_worker, chunks)
            dt = time.perf_counter() - t0
    finally:
        if old is None:
            os.environ.pop("OPENBLAS_NUM_THREADS", None)
        else:
            os.environ["OPENBLAS_NUM_THREADS"] = old
    all_tuples = v * (v + 1) * (v + 2) // 6 - v
    per_tuple = otr.triples_flops(o, v) / all_tuples
    rate = len(work) * per_tuple / dt
    return dict(seconds=otr.triples_flops(o, v) / rate, rate_tflops=rate / 1e12, cores=cores,
                sample="oracle tuple loop (numpy, one BLAS thread per process) on %d of the %d "
                       "tuples of %s (a<=b<=c<%d) spread over %d processes, %.1f s; seconds = "
                       "reference flops / measured rate" % (len(work), all_tuples, cfg, n, cores, dt))


def run_triples(args, local):
    """(T) after CCSD: two FP64 CCSD iterations give amplitudes with singles; the
    (T) energy of those amplitudes, device-resident, in the FP64 and the split
    form (CUDA events inside the library); e2e through the PerturbativeTriples
    operator from host buffers (vertex and amplitude upload, integral slices,
    block loop), wall clock."""
    import numpy as np
    import torch
    from cc4s_b200 import PerturbativeTriples, Solver
    from cc4s_b200.synthetic import config
    from oracle.triples import triples_flops
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    if cfg in COMPLEX_CONFIGS:
        raise SystemExit("--triples: real configurations only")
    if cfg == "custom":
        from cc4s_b200.synthetic import synthetic
        eh, ep, g, hg = synthetic(o, v, G, complex=False, seed=0)
    else:
        eh, ep, g, hg = config(cfg, seed=0)
    if args.vertex_scale is not None:
        g *= args.vertex_scale
    F = triples_flops(o, v)
    forms = ["fp64", "split3"] if args.precision == "both" else [args.precision]
    out = {}
    so = Solver(dict(maxIterations=2, energyConvergence=-1.0, amplitudesConvergence=-1.0,
                     mixer=dict(type="DiisMixer", maxResidua=5), device=local))
    so.set_inputs(eh, ep, g, half_grid=hg)
    so.run()
    T = so.amplitudes()
    so.close()
    for p in forms:
        so = Solver(dict(device=local, precision=p, profile=args.profile))
        so.set_inputs(eh, ep, g, half_grid=hg)
        so.set_initial_amplitudes(*T)
        runs = []
        st0 = so.stats()
        for k in range(args.warmup + args.steps):
            with ClockSampler(local) as clk:
                r = so.perturbative_triples(args.triples_block)
            runs.append((r, clk.summary()))
        st1 = so.stats()
        so.close()
        timed = runs[args.warmup:]
        secs = statistics.median(x[0]["seconds"] for x in timed)
        out[p] = {"seconds": secs, "tflops": F / secs / 1e12, "energy": timed[-1][0]["correlation"],
                  "setup_seconds": timed[-1][0]["setup_seconds"],
                  "executed_flops": timed[-1][0]["executed_flops"],
                  "block_size": timed[-1][0]["block_size"],
                  "block_triples": timed[-1][0]["block_triples"], "clocks": timed[-1][1],
                  "phase_seconds": timed[-1][0]["phase_seconds"] if args.profile else None,
                  "launches": ((st1["gemm_launches"] - st0["gemm_launches"]) +
                               (st1["other_launches"] - st0["other_launches"])) /
                              (args.warmup + args.steps)}
    head = "split3" if "split3" in out else "fp64"
    hr = out[head]
    # end to end: host amplitudes and vertex through the operator
    t0 = time.perf_counter()
    e = PerturbativeTriples().run({"slicedEigenEnergies": {"h": eh, "p": ep}, "coulombVertex": g,
                                   "halfGrid": hg, "amplitudes": {"ph": T[0], "pphh": T[1]},
                                   "precision": head, "blockSize": args.triples_block,
                                   "device": local})
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    pk = peaks()
    dpeak = dgemm_peak(local)
    if head == "split3":
        achieved = 6.0 * hr["executed_flops"] / hr["seconds"] / 1e12
        peak = pk.get("bf16_tflops", 1686.1)
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": "whole (T) block loop: split_kernel particle contractions, FP64 hole "
                          "contractions, singles and energy kernels (six FP16 slice products per "
                          "executed FP64 multiply-add)",
                "peak_source": "MEASURED_PEAKS.json bf16_tflops (of measured)"}
    else:
        achieved = hr["executed_flops"] / hr["seconds"] / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": dpeak, "unit": "TFLOP/s",
                "frac": achieved / dpeak, "traffic": None,
                "kernel": "whole (T) block loop (gemm_f64_kernel contractions + bandwidth kernels)",
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured)"}
    line = {"metric": "(T) perturbative triples energy TFLOP/s (reference flop count) on 1 B200",
            "value": F / hr["seconds"] / 1e12, "unit": "TFLOP/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * hr["seconds"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator; amplitudes after two CCSD iterations)",
            "config": {"workload": "(T) %s: No=%d Nv=%d NG=%d real, %s" % (cfg, o, v, G, head),
                       "flops_reference": F, "forms": out, "fp64_dgemm_peak_tflops": dpeak,
                       "abs_dE_split_vs_fp64": abs(out["split3"]["energy"] - out["fp64"]["energy"])
                       if len(out) == 2 else None,
                       "split_speedup_vs_fp64": out["fp64"]["seconds"] / out["split3"]["seconds"]
                       if len(out) == 2 else None},
            "e2e": {"value": F / t_e2e / 1e12, "unit": "TFLOP/s",
                    "h2d_bytes_per_step": int(g.nbytes + eh.nbytes + ep.nbytes + T[0].nbytes +
                                              T[1].nbytes),
                    "d2h_bytes_per_step": 8, "seconds": t_e2e,
                    "energy": e["energy"]["correlation"]},
            "roofline": roof, "clocks": hr["clocks"], "gpu_launches": int(round(hr["launches"]))}
    if not args.no_cpu_baseline:
        c = cpu_triples_sample(cfg)
        line["cpu_baseline"] = {"value": F / c["seconds"] / 1e12, "unit": "TFLOP/s",
                                "cores": c["cores"], "kind": "port", "sample": c["sample"]}
    return line


def run_fsc(args, local):
    """FiniteSizeCorrection after CCSD: two FP64 CCSD iterations give the
    amplitudes; plane-wave grid of n^3 vectors (n = 16 by default) of a skewed reciprocal
    lattice, random complex singular vectors U [NGG, NG] and potential V(G);
    device time of the step (uploads, structure factor, interpolation over
    (2N)^3 NGG points); e2e through the operator from host buffers; CPU: the
    oracle's interpolation on a bounded sample of the refined points."""
    import numpy as np
    import torch
    from cc4s_b200 import FiniteSizeCorrection, Solver
    from cc4s_b200.synthetic import config
    from oracle import fsc as ofsc
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    if cfg in COMPLEX_CONFIGS:
        raise SystemExit("--fsc: real configurations only")
    if cfg == "custom":
        from cc4s_b200.synthetic import synthetic
        eh, ep, g, hg = synthetic(o, v, G, complex=False, seed=0)
    else:
        eh, ep, g, hg = config(cfg, seed=0)
    rng = np.random.default_rng(0)
    n = args.fsc_grid
    B = 2 * np.pi / 6.0 * (np.eye(3) + 0.05 * rng.standard_normal((3, 3)))
    r = np.arange(n) - n // 2
    grid = np.array([(a, b, c) for c in r for b in r for a in r], dtype=float) @ B
    NGG = grid.shape[0]
    U = (rng.standard_normal((NGG, G)) + 1j * rng.standard_normal((NGG, G))) / np.sqrt(G)
    V = 0.5 + rng.random(NGG)
    N = args.fsc_n
    so = Solver(dict(maxIterations=2, energyConvergence=-1.0, amplitudesConvergence=-1.0,
                     mixer=dict(type="DiisMixer", maxResidua=5), device=local))
    so.set_inputs(eh, ep, g, half_grid=hg)
    so.run()
    T = so.amplitudes()
    st0 = so.stats()
    secs = []
    for k in range(args.warmup + args.steps):
        e, S = so.finite_size_correction(grid, B, U, V, grid_size=N)
        secs.append(e["seconds"])
    st1 = so.stats()
    so.close()
    t = statistics.median(secs[args.warmup:])
    points = (2 * N) ** 3 * NGG
    launches = ((st1["gemm_launches"] - st0["gemm_launches"]) +
                (st1["other_launches"] - st0["other_launches"])) / (args.warmup + args.steps)
    t0 = time.perf_counter()
    out = FiniteSizeCorrection().run({
        "slicedEigenEnergies": {"h": eh, "p": ep}, "coulombVertex": g, "halfGrid": hg,
        "amplitudes": {"ph": T[0], "pphh": T[1]}, "gridVectors": grid, "reciprocalBasis": B,
        "coulombVertexSingularVectors": U, "coulombPotential": V, "interpolationGridSize": N,
        "device": local})
    torch.cuda.synchronize()
    t_e2e = time.perf_counter() - t0
    line = {"metric": "FiniteSizeCorrection: interpolated points per second (tricubic, (2N)^3 NGG)",
            "value": points / t, "unit": "points/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded grid, singular vectors, potential; amplitudes after two "
                    "CCSD iterations)",
            "config": {"workload": "FSC %s: No=%d Nv=%d NG=%d, NGG=%d plane waves, N=%d" % (
                cfg, o, v, G, NGG, N), "points": points, "box": e["box"],
                       "correction": e["correction"], "uncorrected": e["uncorrected"]},
            "gpu_launches": int(round(launches)),
            "e2e": {"value": points / t_e2e, "unit": "points/s",
                    "h2d_bytes_per_step": int(g.nbytes + T[0].nbytes + T[1].nbytes + U.nbytes +
                                              V.nbytes + grid.nbytes),
                    "d2h_bytes_per_step": int(S.nbytes + 24), "seconds": t_e2e}}
    if not args.no_cpu_baseline:
        # oracle interpolation on a sample of the refined points (same box and S)
        A, omega, dims, origin, direct = ofsc.box_of(grid, B)
        box = np.zeros(int(np.prod(dims)))
        for i in range(NGG):
            idx = np.floor(direct[i] + 0.5).astype(int) - origin.astype(int)
            box[idx[0] + dims[0] * (idx[1] + dims[1] * idx[2])] = S[i]
        # refined points g = G_i + (a B0 + b B1 + c B2) / 2N for a slab of (a, b, c)
        rows = []
        for a_ in (-N,):
            for b_ in range(-N, min(N, -N + 4)):
                for c_ in range(-N, N):
                    rows.append(grid + (B[0] * a_ + B[1] * b_ + B[2] * c_) / (2.0 * N))
        pts = np.concatenate(rows)
        n2 = (pts * pts).sum(axis=1)
        t0 = time.perf_counter()
        keep = np.sqrt(n2) >= 1e-8
        val = ofsc.tricubic_many(box, dims, origin, pts[keep] @ A.T)
        _ = float(np.sum(val / n2[keep]))
        dt = time.perf_counter() - t0
        line["cpu_baseline"] = {"value": pts.shape[0] / dt, "unit": "points/s", "cores": 1,
                                "kind": "port",
                                "sample": "oracle tricubic interpolation (numpy, vectorised, one "
                                          "thread) on %d refined points (a = -N, b in [-N, -N+4)), %.1f s"
                                          % (pts.shape[0], dt)}
    return line


def run_reference(args, world, rank):
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    from cc4s_b200.flops import reference_flops
    F = reference_flops(o, v, G, complex=cfg in COMPLEX_CONFIGS)
    for _ in range(args.warmup):
        cpu_sample(cfg)
    samples = [cpu_sample(cfg) for _ in range(max(1, args.steps))]
    s_iter = statistics.median(x["s_per_iter"] for x in samples)
    c = samples[0]
    val = F / s_iter / 1e12
    return {"impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * s_iter, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "CCSD FP64 %s: No=%d Nv=%d NG=%d %s" % (
                cfg, o, v, G, "complex" if cfg in COMPLEX_CONFIGS else "real"),
                       "implementation": "CPU restatement of the reference (oracle, numpy/BLAS); "
                                         "the reference build needs MPI + CTF, not installed"},
            "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": c["cores"],
                             "kind": "port", "sample": c["sample"]},
            "e2e": {"value": val, "unit": "TFLOP/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="c2", choices=sorted(CONFIG_SHAPES))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--precision", default="both", choices=["both", "fp64", "split3"])
    ap.add_argument("--adjoint", action="store_true",
                    help="time and check the adjoint form (relaxed gradient) instead")
    ap.add_argument("--fd-directions", type=int, default=2)
    ap.add_argument("--converge", action="store_true",
                    help="converge FP64, split and refined split forms and compare energies")
    ap.add_argument("--refine", type=float, default=1e-5,
                    help="residuum norm below which the refined split form switches to FP64")
    ap.add_argument("--triples", action="store_true",
                    help="time the perturbative triples (T) step instead (real configurations)")
    ap.add_argument("--fsc", action="store_true",
                    help="time the FiniteSizeCorrection step instead (real configurations)")
    ap.add_argument("--fsc-grid", type=int, default=16,
                    help="--fsc: plane-wave grid of n^3 vectors")
    ap.add_argument("--fsc-n", type=int, default=20, help="--fsc: interpolationGridSize")
    ap.add_argument("--triples-block", type=int, default=0,
                    help="virtual indices per (T) block (0: automatic)")
    ap.add_argument("--shape", default=None,
                    help="No,Nv,NG of a real synthetic system instead of --config (profiling of "
                         "small cases)")
    ap.add_argument("--profile", action="store_true",
                    help="--triples: device time of each phase of the block loop")
    ap.add_argument("--vertex-scale", type=float, default=None,
                    help="scale of the synthetic vertex (default 1; 0.3 for --converge and "
                         "--adjoint: CCSD on the unscaled synthetic vertex diverges at these "
                         "sizes, strongly correlated)")
    args = ap.parse_args()
    if args.shape:
        o_, v_, g_ = (int(x) for x in args.shape.split(","))
        CONFIG_SHAPES["custom"] = (o_, v_, g_)
        args.config = "custom"
    if args.impl == "reference":
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        if rank != 0:
            return
        print(json.dumps(run_reference(args, world, rank)), flush=True)
        return
    world, rank, local = dist_setup()
    if args.adjoint or args.converge or args.triples or args.fsc:
        if rank == 0:
            if args.fsc:
                line = run_fsc(args, local)
            elif args.triples:
                line = run_triples(args, local)
            else:
                line = run_adjoint(args, local) if args.adjoint else run_converge(args, local)
            print(json.dumps(line), flush=True)
        return
    line = run_ours(args, world, rank, local)
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            c = cpu_sample(args.config)
            from cc4s_b200.flops import reference_flops
            o, v, G = CONFIG_SHAPES[args.config]
            cfg = args.config
            line["cpu_baseline"] = {"value": reference_flops(o, v, G, complex=cfg in COMPLEX_CONFIGS) / c["s_per_iter"] / 1e12,
                                    "unit": "TFLOP/s", "cores": c["cores"], "kind": "port",
                                    "sample": c["sample"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
