"""Benchmark of the CoupledCluster (CCSD) step on B200.

A "step" is one CCSD iteration (residual, Jacobi update, DIIS, energy) on a
seeded synthetic system.  Default workload: No=64, Nv=640, NG=2560, real
(T2 13.4 GB), vertex scaled by 0.2 (CCSD diverges on the unscaled synthetic
vertex; the cost of an iteration does not depend on the scale).  T2 and the
vertex are far larger than L2, so no flush is needed between iterations.

Order of the CCSD line (single GPU):
 1. the headline split-precision form: W warm-up + K timed iterations (the
    first warm-up is the cheap R = V iteration), with CUDA events around every
    contraction launch on the library stream for the roofline;
 2. e2e: the same metric through the C ABI from host buffers: set_inputs
    (vertex upload and integral build) + the first iteration + a bounded
    number of full iterations (--e2e-iterations) + amplitude download, wall
    clock; only the full iterations' flops count;
 3. the FP64 form for the speed-up, a bounded number of iterations
    (--fp64-warmup, --fp64-steps), skipped if it would pass --time-budget;
 4. the CPU baseline: one full oracle iteration of a quarter-size system.

value: reference-equivalent TFLOP/s = F_ref / (s per iteration), with F_ref
the flop count of the reference's formulation (cc4s_b200.flops), timed with
CUDA events on the library's stream inside the library, max over ranks.

Multi-GPU: every rank runs its own replica of the workload (weak scaling, no
collective on the data path); value is the sum over ranks.

--impl reference: the CPU restatement of the reference (the oracle; the
reference itself needs MPI and the Cyclops Tensor Framework, which are not
installed), one full iteration of a quarter-size system per step, on all host
cores.
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


def cores_available():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def sample_shape(cfg):
    """The CPU sample system: the workload's generator at a quarter of each
    dimension (c2: No=16, Nv=160, NG=640), so that one full oracle iteration
    takes seconds instead of hours."""
    o, v, G = CONFIG_SHAPES[cfg]
    return max(2, o // 4), max(4, v // 4), max(8, G // 4)


class OracleSteps:
    """One CoupledCluster iteration per step of the oracle (the CPU restatement
    of CoupledCluster.cxx:129-175 with the Ccsd residual of Ccsd.cxx:77-378 and
    the DIIS mixer of DiisMixer.cxx), numpy/BLAS on all host cores, on the
    sample system of `cfg` (same seeded generator and vertex scale).  The first
    step is the cheap first iteration (R = V); every later one is a full
    iteration."""

    def __init__(self, cfg, vertex_scale):
        from oracle import coupled_cluster, inputs
        from cc4s_b200.flops import reference_flops
        from cc4s_b200.synthetic import synthetic
        self.cfg = cfg
        self.shape = sample_shape(cfg)
        o, v, G = self.shape
        cplx = cfg in COMPLEX_CONFIGS
        eh, ep, g, hg = synthetic(o, v, G, complex=cplx, seed=0)
        g *= vertex_scale
        self.system = inputs.System(eh, ep, g, half_grid=hg)
        self.flops = reference_flops(o, v, G, complex=cplx)
        self.it = coupled_cluster.iterations(self.system, None, method="Ccsd",
                                             mixer=dict(type="DiisMixer", maxResidua=5),
                                             energyConvergence=-1.0, amplitudesConvergence=-1.0)
        self.steps = 0

    def step(self):
        t0 = time.perf_counter()
        next(self.it)
        dt = time.perf_counter() - t0
        self.steps += 1
        return dt

    def describe(self, seconds):
        o, v, G = self.shape
        return ("oracle (numpy/BLAS, %d threads): full CoupledCluster iterations (Ccsd residual, "
                "Jacobi, DIIS 5, energy) of the %s generator at a quarter of each dimension "
                "(No=%d Nv=%d NG=%d, %.3g reference flops per iteration), %.2f s per iteration"
                % (cores_available(), self.cfg, o, v, G, self.flops, seconds))


def cpu_sample(cfg, vertex_scale, full_iterations=1):
    """Bounded CPU baseline: the first (cheap) iteration and `full_iterations`
    full iterations of OracleSteps; the rate of the full ones in TFLOP/s of the
    reference formulation."""
    run = OracleSteps(cfg, vertex_scale)
    run.step()
    secs = [run.step() for _ in range(full_iterations)]
    s = statistics.median(secs)
    return dict(rate_tflops=run.flops / s / 1e12, seconds=s, cores=cores_available(),
                sample=run.describe(s))


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


def timed_run(opts, inputs, W, K, world, local, keep_amplitudes=False):
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
    return dict(t=t, r=r, launches=launches, T=T, clocks=clk.summary(), stats=st1,
                secs=secs)


# Default vertex scale of the CCSD line: the synthetic systems of c1, c2 and c4
# are strongly correlated and CCSD from T = 0 diverges on the unscaled vertex
# (E_c of about -3200 Eh after four iterations at c2; at scale 0.3 c1 and c4
# converge but c2 still diverges after ~80 iterations); at 0.2 all converge.  The
# cost of an iteration does not depend on the scale.
DEFAULT_VERTEX_SCALE = 0.2
# Upper bound of the FP64 form's time per iteration relative to the split form,
# used only to decide whether the FP64 comparison still fits the time budget
# (measured at c2: 3.3).
FP64_OVER_SPLIT_BOUND = 4.5


# DRAM traffic of the split contraction kernel at c2, from one ncu capture of the 851
# split launches of one iteration (dram__bytes_read.sum + dram__bytes_write.sum with
# -k regex:split_kernel -c 851 around `bench.py --config c2 --precision split3 --steps 1
# --warmup 1 --no-cpu-baseline`): 15.09 TB in all, 17.73 GB per launch, 3.6x the
# algorithmic bytes (packed slices of both operands read once, the output read and
# written once).
SPLIT_TRAFFIC_C2 = {"bytes_per_launch": 17.73e9, "algorithmic_bytes_per_launch": 4.9e9,
                    "launches": 851}
# Measured on one B200 at c2 (No=64, Nv=640, NG=2560, real): seconds per full
# iteration of each form (CUDA events), and wall seconds of the host-side input
# generation, of one handle's set-up (vertex upload, integral build) and of the
# CPU baseline leg.  projected_seconds() uses them to check that the default
# benchmark command (--steps 20 --warmup 5) fits a 1800 s limit.
MEASURED_C2 = {"split3": 12.0, "fp64": 69.7, "inputs": 60.0, "setup": 30.0, "cpu": 40.0,
               "download": 15.0}


def projected_seconds(W, K, e2e_iterations=2, fp64_warmup=2, fp64_steps=2, m=MEASURED_C2):
    """Projected wall seconds of each leg of the c2 CCSD line."""
    s, s64 = m["split3"], m["fp64"]
    n_e2e = max(1, min(K, e2e_iterations))
    return {"inputs": m["inputs"],
            "headline": m["setup"] + (W - 1 + K) * s + 0.1 * s,
            "e2e": m["setup"] + n_e2e * s + 0.1 * s + m["download"],
            "fp64": m["setup"] + (max(1, fp64_warmup) - 1 + fp64_steps) * s64 + 0.1 * s64,
            "dgemm_peak": 5.0, "cpu_baseline": m["cpu"]}


def run_ours(args, world, rank, local):
    """The CCSD line: headline form first (W warm-up + K timed iterations, the
    contractions' per-launch CUDA events recorded inside the timed region),
    then an e2e leg of a bounded number of iterations from host buffers, then
    the FP64 comparison (1 warm-up + a bounded number of timed iterations) if
    it fits the remaining time budget."""
    import torch
    from cc4s_b200 import Solver, reference_flops
    from cc4s_b200.synthetic import config
    t_begin = time.perf_counter()
    deadline = t_begin + args.time_budget
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    if cfg == "custom":
        from cc4s_b200.synthetic import synthetic
        inputs = synthetic(o, v, G, complex=False, seed=0)
    else:
        inputs = config(cfg, seed=0)
    eh, ep, g, hg = inputs
    scale = DEFAULT_VERTEX_SCALE if args.vertex_scale is None else args.vertex_scale
    if scale != 1.0:
        g *= scale
    F = reference_flops(o, v, G, complex=cfg in COMPLEX_CONFIGS)
    K, W = args.steps, args.warmup
    base = dict(energyConvergence=-1.0, amplitudesConvergence=-1.0,
                mixer=dict(type="DiisMixer", maxResidua=5), device=local)
    head = "fp64" if args.precision == "fp64" else "split3"
    # 1. headline form, with per-launch events on the library stream
    hr = timed_run(dict(base, precision=head, maxIterations=W + K, profile=True), inputs, W, K,
                   world, local)
    t = hr["t"]
    ps = hr["stats"]
    pk = peaks()
    # 2. end to end through the C ABI from host buffers: vertex upload and
    # integral build, the cheap first iteration, n_e2e full iterations and the
    # amplitude download; only the full iterations' flops are counted
    n_e2e = max(1, min(K, args.e2e_iterations))
    barrier(world)
    t0 = time.perf_counter()
    e2e = Solver(dict(base, precision=head, maxIterations=n_e2e + 1))
    e2e.set_inputs(eh, ep, g, half_grid=hg)
    re = e2e.run()
    A1, A2 = e2e.amplitudes()
    torch.cuda.synchronize()
    t_e2e = all_max(time.perf_counter() - t0, world)
    e2e.close()
    h2d = (g.nbytes + eh.nbytes + ep.nbytes) / n_e2e
    d2h = (A1.nbytes + A2.nbytes) / n_e2e + 5 * 8 + 8
    del A1, A2
    # 3. FP64 comparison (single GPU): args.fp64_warmup warm-up iterations (the
    # first one is the cheap R = V iteration) and args.fp64_steps timed full
    # iterations, if the projection fits the budget
    runs = {head: hr}
    fp64_note = None
    W64 = max(1, args.fp64_warmup)
    if world == 1 and args.precision == "both":
        s_split = t / K
        projected = ((W64 - 1 + args.fp64_steps) * FP64_OVER_SPLIT_BOUND * s_split +
                     max(0.0, t_e2e - (n_e2e + 1) * s_split) + 60.0)
        if time.perf_counter() + projected < deadline:
            runs["fp64"] = timed_run(dict(base, precision="fp64",
                                          maxIterations=W64 + args.fp64_steps),
                                     inputs, W64, args.fp64_steps, world, local)
        else:
            fp64_note = ("skipped: projected %.0f s would pass the %.0f s time budget"
                         % (projected, args.time_budget))
    dpeak = dgemm_peak(local)
    if head == "split3":
        # executed FP16 tensor work: six slice products per FP64-equivalent multiply-add
        achieved = 6.0 * ps["split_flops"] / ps["split_seconds"] / 1e12
        peak = pk.get("bf16_tflops_sustained", 1405.3)
        roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved / peak, "traffic": None,
                "kernel": "split_kernel_persistent (tcgen05.mma kind::f16, TMEM, TMA) incl. operand "
                          "slicing: %d launches of the last timed iteration, CUDA events on the "
                          "library stream" % ps["split_launches"],
                "peak_source": "MEASURED_PEAKS.json bf16_tflops_sustained (of measured)",
                "fp64_equivalent_tflops": ps["split_flops"] / ps["split_seconds"] / 1e12}
        if cfg == "c2":
            roof["traffic"] = SPLIT_TRAFFIC_C2["bytes_per_launch"]
            roof["traffic_note"] = (
                "bytes per launch, mean over the %d split launches of one iteration (one ncu "
                "capture); algorithmic %.2g bytes per launch" %
                (SPLIT_TRAFFIC_C2["launches"], SPLIT_TRAFFIC_C2["algorithmic_bytes_per_launch"]))
    else:
        achieved = ps["gemm_flops"] / ps["gemm_seconds"] / 1e12
        roof = {"bound": "tensor", "achieved": achieved, "peak": dpeak, "unit": "TFLOP/s",
                "frac": achieved / dpeak, "traffic": None,
                "kernel": "gemm_f64_kernel (mma.sync m16n8k16 f64): all %d contraction launches "
                          "of the last timed iteration" % ps["gemm_profiled_launches"],
                "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured; no FP64 "
                               "entry in MEASURED_PEAKS.json)",
                "top_launch_tflops": ps["top_flops"] / ps["top_seconds"] / 1e12}
    kind = "complex" if cfg in COMPLEX_CONFIGS else "real"
    conf = {"workload": "CCSD %s: No=%d Nv=%d NG=%d %s, DIIS 5, %s" % (cfg, o, v, G, kind, head),
            "precision": head, "s_per_iter": t / K, "vertex_scale": scale,
            "s_per_iter_all": hr["secs"][W:W + K],
            "flops_per_iter_reference_formulation": F,
            "flops_per_iter_executed": hr["r"]["flops_per_iteration"],
            "l2": "inputs larger than L2 (T2 %.2f GB), no flush" % ((v * o) ** 2 * 8 / 1e9),
            "parallelism": "replicas" if world > 1 else "single GPU",
            "energy_after_steps": hr["r"]["correlation"],
            "residuum_norm_after_steps": hr["r"]["history"][-1]["dR"],
            "fp64_dgemm_peak_tflops": dpeak, "e2e_iterations": n_e2e,
            "time_budget_s": args.time_budget}
    if "fp64" in runs:
        t64 = runs["fp64"]["t"]
        s64 = t64 / args.fp64_steps
        conf.update({"fp64_s_per_iter": s64, "fp64_tflops": F / s64 / 1e12,
                     "fp64_timed_iterations": args.fp64_steps, "fp64_warmup": W64,
                     "split_speedup_vs_fp64": s64 / (t / K)})
    elif fp64_note:
        conf["fp64"] = fp64_note
    line = {
        "metric": METRIC, "value": world * F / (t / K) / 1e12, "unit": "TFLOP/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": 1e3 * t / K,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator of the workload's distributions, vertex x%g)" % scale,
        "config": conf,
        "e2e": {"value": world * F * n_e2e / t_e2e / 1e12, "unit": "TFLOP/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "seconds": t_e2e, "iterations": re["iterations"],
                "counted_iterations": n_e2e},
        "gpu_launches": int(round(hr["launches"] * K)),
        "roofline": roof,
        "clocks": hr["clocks"],
    }
    line["config"]["wall_seconds_to_line"] = time.perf_counter() - t_begin
    return line


def run_adjoint(args, local):
    """Adjoint form at the workload: converged FP64 CCSD, Lambda equations by
    transposed-Jacobian products, relaxed dE_c/dGamma; the same with the split
    form's backward (forward and reverse contractions on the split kernel); the
    time of each against one forward iteration, and both gradients against
    central differences of re-converged FP64 energies (steps 1e-5 and 5e-6,
    Richardson-extrapolated) on --fd-directions random vertex directions (each
    perturbed solve starts from the converged amplitudes and reaches the FP64
    fixed point)."""
    import numpy as np
    import torch
    from cc4s_b200 import Solver
    from cc4s_b200.synthetic import config
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    if cfg == "custom":
        from cc4s_b200.synthetic import synthetic
        eh, ep, g, hg = synthetic(o, v, G, complex=False, seed=0)
    else:
        eh, ep, g, hg = config(cfg, seed=0)
    scale = args.vertex_scale if args.vertex_scale is not None else DEFAULT_VERTEX_SCALE
    g *= scale
    # energies converged far below the 1e-5 step times the 1e-6 bound on the
    # derivative; the split form's rounding (~1e-9 relative in the residual) sets
    # its own floor
    tight = dict(energyConvergence=1e-13, amplitudesConvergence=1e-11)
    loose = dict(energyConvergence=1e-10, amplitudesConvergence=1e-8)
    base = dict(maxIterations=200, mixer=dict(type="DiisMixer", maxResidua=5), device=local)

    def solve(gm, precision="fp64", start=None):
        so = Solver(dict(base, precision=precision, **(tight if precision == "fp64" else loose)))
        so.set_inputs(eh, ep, gm, half_grid=hg)
        if start is not None:
            so.set_initial_amplitudes(*start)
        return so, so.run()

    forms = {}
    T0 = None
    for prec in (["fp64", "split3"] if args.precision == "both" else [args.precision]):
        sol, r = solve(g, prec)
        if prec == "fp64":
            T0 = sol.amplitudes()
        fwd = statistics.median(h["seconds"] for h in r["history"][2:]) if r["iterations"] > 3 \
            else r["history"][-1]["seconds"]
        t0 = time.perf_counter()
        grad, info = sol.relaxed_gradient(max_iterations=200,
                                          convergence=1e-10 if prec == "fp64" else 1e-8)
        t_back = time.perf_counter() - t0
        sol.close()
        forms[prec] = dict(grad=grad, info=info, fwd=fwd, t_back=t_back, r=r)
    if T0 is None:
        so, _ = solve(g)
        T0 = so.amplitudes()
        so.close()
    rng = np.random.default_rng(7)
    h = 1e-5
    checks = {p: [] for p in forms}

    def fd_energy(gm):
        # the FP64 fixed point from the converged amplitudes: split iterations until
        # the residuum norm is below 1e-7, FP64 iterations to energyConvergence 1e-13
        so = Solver(dict(base, precision="split3", precisionRefinement=1e-7, **tight))
        so.set_inputs(eh, ep, gm, half_grid=hg)
        so.set_initial_amplitudes(*T0)
        r = so.run()
        so.close()
        return r

    def central(d, step):
        rp, rm_ = fd_energy(g + step * d), fd_energy(g - step * d)
        return (rp["correlation"] - rm_["correlation"]) / (2 * step), [rp["iterations"],
                                                                        rm_["iterations"]]
    for _ in range(args.fd_directions):
        d = rng.standard_normal(g.shape)
        # Richardson: the O(h^2) error of a central difference along these long
        # directions (|d| ~ sqrt(#entries)) is ~1e-5 relative at h = 1e-5
        c1, it1 = central(d, h)
        c2, it2 = central(d, h / 2)
        fd = (4.0 * c2 - c1) / 3.0
        for p, f in forms.items():
            an = float((f["grad"] * d).sum())
            checks[p].append({"fd": fd, "fd_h": c1, "fd_h2": c2, "adjoint": an,
                              "rel_err": abs(fd - an) / abs(fd),
                              "rel_err_plain_central": abs(c1 - an) / abs(c1),
                              "fd_iterations": it1 + it2})
    head = "fp64" if "fp64" in forms else args.precision
    out = {}
    for p, f in forms.items():
        info = f["info"]
        out[p] = {"forward_iterations": f["r"]["iterations"], "forward_s_per_iter": f["fwd"],
                  "energy": f["r"]["correlation"],
                  "lambda_iterations": info["iterations"], "lambda_converged": info["converged"],
                  "lambda_residuum_norm": info["residuum_norm"],
                  "prepare_seconds": info["prepare_seconds"],
                  "lambda_s_per_iter": info["vjp_seconds"],
                  "gradient_seconds": info["gradient_seconds"],
                  "backward_total_seconds": f["t_back"],
                  "backward_total_vs_forward_iteration": f["t_back"] / f["fwd"] if f["fwd"] else None,
                  "lambda_iteration_vs_forward_iteration":
                      info["vjp_seconds"] / f["fwd"] if f["fwd"] else None,
                  "fd_max_rel_err": max((c["rel_err"] for c in checks[p]), default=None),
                  "fd_directions": checks[p]}
    if len(forms) == 2:
        g64, gs = forms["fp64"]["grad"], forms["split3"]["grad"]
        out["split3"]["max_abs_diff_vs_fp64_over_max"] = float(np.abs(gs - g64).max() /
                                                             np.abs(g64).max())
        out["split3"]["backward_speedup_vs_fp64"] = forms["fp64"]["t_back"] / forms["split3"]["t_back"]
    return {"metric": "CCSD adjoint: relaxed dE_c/dGamma (Lambda equations) vs one forward iteration",
            "value": out[head]["backward_total_vs_forward_iteration"],
            "unit": "x forward iteration", "higher_is_better": False, "n_gpus": 1, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": "CCSD %s: No=%d Nv=%d NG=%d real, DIIS 5" % (cfg, o, v, G),
                       "vertex_scale": scale, "fd_steps": [h, h / 2], "fd_directions": args.fd_directions,
                       "fd": "central differences at h and h/2, Richardson-extrapolated "
                             "(4 D(h/2) - D(h)) / 3"},
            "forms": out}


def run_converge(args, local):
    """Accuracy of the split form at convergence.  Forms, each to
    energyConvergence --converge-energy (DIIS 5, at most 100 iterations):
      split3          the split form from T = 0;
      fp64_from_split FP64 iterations started from the split form's converged
                      amplitudes (converges to the FP64 fixed point);
      fp64            the FP64 form from T = 0 (skipped with --converge-skip-fp64).
    Reports |E_split - E_fp64|, the per-iteration energies and residuum norms,
    the final amplitudes' difference (max and norm, relative), iterations and
    time to solution.  The synthetic vertex is scaled (default 0.2): unscaled,
    CCSD diverges at these sizes."""
    import numpy as np
    import torch
    from cc4s_b200 import Solver
    from cc4s_b200.synthetic import config
    torch.cuda.set_device(local)
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    if cfg == "custom":
        from cc4s_b200.synthetic import synthetic
        eh, ep, g, hg = synthetic(o, v, G, complex=False, seed=0)
    else:
        eh, ep, g, hg = config(cfg, seed=0)
    scale = args.vertex_scale if args.vertex_scale is not None else DEFAULT_VERTEX_SCALE
    g *= scale
    base = dict(maxIterations=100, energyConvergence=args.converge_energy,
                amplitudesConvergence=1e-7, mixer=dict(type="DiisMixer", maxResidua=5),
                device=local)

    def solve(precision, start=None):
        so = Solver(dict(base, precision=precision))
        so.set_inputs(eh, ep, g, half_grid=hg)
        if start is not None:
            so.set_initial_amplitudes(*start)
        r = so.run()
        T = so.amplitudes()
        so.close()
        return r, T

    def summary(r):
        return {"energy": r["correlation"], "iterations": r["iterations"],
                "converged": r["converged"], "seconds": sum(h["seconds"] for h in r["history"]),
                "history_energy": [h["energy"] for h in r["history"]],
                "history_residuum_norm": [h["dR"] for h in r["history"]],
                "s_per_iter": [h["seconds"] for h in r["history"]]}

    out = {}
    rs, Ts = solve("split3")
    out["split3"] = summary(rs)
    rf, Tf = solve("fp64", start=Ts)
    out["fp64_from_split"] = summary(rf)
    T64, r64 = Tf, rf
    if not args.converge_skip_fp64:
        r0, T0 = solve("fp64")
        out["fp64"] = summary(r0)
        out["fp64"]["abs_dE_vs_fp64_from_split"] = abs(r0["correlation"] - rf["correlation"])
        T64, r64 = T0, r0
    e64 = r64["correlation"]
    for name, T in (("split3", Ts), ("fp64_from_split", Tf)):
        if name == "fp64_from_split" and T is T64:
            continue
        out[name]["abs_dE_vs_fp64"] = abs(out[name]["energy"] - e64)
        for k, (A, B) in enumerate(zip(T, T64)):
            d = np.abs(A - B).max() / np.abs(B).max()
            n = float(np.linalg.norm((A - B).ravel()) / np.linalg.norm(B.ravel()))
            out[name]["T%d_max_rel_diff" % (k + 1)] = float(d)
            out[name]["T%d_norm_rel_diff" % (k + 1)] = n
    kind = "complex" if cfg in COMPLEX_CONFIGS else "real"
    ref = "fp64" if "fp64" in out else "fp64_from_split"
    conf = {"workload": "CCSD %s: No=%d Nv=%d NG=%d %s, DIIS 5, energyConvergence %g"
                        % (cfg, o, v, G, kind, args.converge_energy),
            "vertex_scale": scale, "fp64_reference": ref}
    if ref == "fp64" and out["fp64"]["seconds"] > 0:
        conf["split_time_to_solution_vs_fp64"] = out["split3"]["seconds"] / out["fp64"]["seconds"]
    else:
        # the FP64 leg started from the split form's amplitudes: an FP64 solve from
        # T = 0 is estimated as the split form's iteration count at the FP64 leg's
        # median seconds per iteration (the DIIS trajectories of the two forms agree
        # to the split rounding)
        fp_it = statistics.median(out[ref]["s_per_iter"]) if out[ref]["s_per_iter"] else 0.0
        est = out["split3"]["iterations"] * fp_it
        conf["fp64_from_zero_seconds_estimated"] = est
        conf["split_time_to_solution_vs_fp64_estimated"] = (
            out["split3"]["seconds"] / est if est > 0 else None)
    return {"metric": "CCSD converged |dE_c| split-precision vs FP64 (bound 1e-6 Eh)",
            "value": out["split3"]["abs_dE_vs_fp64"], "unit": "Eh",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f64", "data": "synthetic",
            "config": conf, "forms": out}


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
                r = so.perturbative_triples(args.triples_block, reference_form=args.cT,
                                            cT=args.cT)
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
                                   "referenceForm": args.cT, "cT": int(args.cT),
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
                "kernel": "whole (T) block loop: split_kernel contractions (particle and hole "
                          "halves over K = v + o), singles and energy kernels (six FP16 slice "
                          "products per executed FP64 multiply-add)",
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
            "config": {"workload": "(T)%s %s: No=%d Nv=%d NG=%d real, %s" % (
                           " cT=1" if args.cT else "", cfg, o, v, G, head),
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
    """The reference arm: the reference's algorithm on the host cores.  The
    reference itself (CTF + MPI + yaml-cpp) cannot be built here, so its CPU
    restatement (the oracle, numpy/BLAS on all host threads) runs instead: each
    step is one full CoupledCluster iteration of the workload's generator at a
    quarter of each dimension (OracleSteps), and value is the reference
    formulation's flops of that iteration per second.  ms_per_step and steps
    describe those iterations; the c2 time per iteration at that rate is
    reported under config as an extrapolation."""
    cfg = args.config
    o, v, G = CONFIG_SHAPES[cfg]
    from cc4s_b200.flops import reference_flops
    scale = DEFAULT_VERTEX_SCALE if args.vertex_scale is None else args.vertex_scale
    F = reference_flops(o, v, G, complex=cfg in COMPLEX_CONFIGS)
    run = OracleSteps(cfg, scale)
    run.step()                      # the first, cheap iteration (R = V) is not a full one
    for _ in range(max(0, args.warmup - 1)):
        run.step()
    secs = [run.step() for _ in range(max(1, args.steps))]
    total = sum(secs)
    s_iter = total / len(secs)
    val = run.flops / s_iter / 1e12
    kind = "complex" if cfg in COMPLEX_CONFIGS else "real"
    sample = run.describe(s_iter)
    return {"impl": "reference", "metric": METRIC, "value": val, "unit": "TFLOP/s",
            "n_gpus": world, "steps": len(secs), "warmup": max(1, args.warmup),
            "ms_per_step": 1e3 * s_iter, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded generator of the workload's distributions, vertex x%g)" % scale,
            "config": {"workload": "CCSD %s: No=%d Nv=%d NG=%d %s, DIIS 5" % (cfg, o, v, G, kind),
                       "implementation": "CPU restatement of the reference (oracle, numpy/BLAS); "
                                         "the reference build needs MPI + CTF, not installed",
                       "sample_shape": list(run.shape), "sample_flops_per_iter": run.flops,
                       "sample_s_per_iter_all": secs,
                       "extrapolated_s_per_iter_at_workload": F / (val * 1e12),
                       "extrapolation": "reference flops of the workload / the sample's measured "
                                        "rate (CPU rates grow with size, so this is an estimate)"},
            "cpu_baseline": {"value": val, "unit": "TFLOP/s", "cores": cores_available(),
                             "kind": "port", "sample": sample},
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
    ap.add_argument("--time-budget", type=float, default=1500.0,
                    help="CCSD line: seconds after which optional legs (the FP64 comparison) "
                         "are skipped")
    ap.add_argument("--e2e-iterations", type=int, default=2,
                    help="CCSD line: full iterations of the e2e leg (at most --steps)")
    ap.add_argument("--fp64-steps", type=int, default=2,
                    help="CCSD line: timed iterations of the FP64 comparison")
    ap.add_argument("--fp64-warmup", type=int, default=2,
                    help="CCSD line: warm-up iterations of the FP64 comparison (the first is "
                         "the cheap R = V iteration)")
    ap.add_argument("--adjoint", action="store_true",
                    help="time and check the adjoint form (relaxed gradient) instead")
    ap.add_argument("--fd-directions", type=int, default=8)
    ap.add_argument("--converge", action="store_true",
                    help="converge FP64, split and refined split forms and compare energies")
    ap.add_argument("--converge-energy", type=float, default=1e-9,
                    help="--converge: energyConvergence of every form")
    ap.add_argument("--converge-skip-fp64", action="store_true",
                    help="--converge: no FP64 solve from T = 0 (the FP64 reference is then the "
                         "FP64 iteration started from the split form's amplitudes)")
    ap.add_argument("--triples", action="store_true",
                    help="time the perturbative triples (T) step instead (real configurations)")
    ap.add_argument("--fsc", action="store_true",
                    help="time the FiniteSizeCorrection step instead (real configurations)")
    ap.add_argument("--fsc-grid", type=int, default=16,
                    help="--fsc: plane-wave grid of n^3 vectors")
    ap.add_argument("--fsc-n", type=int, default=20, help="--fsc: interpolationGridSize")
    ap.add_argument("--triples-block", type=int, default=0,
                    help="virtual indices per (T) block (0: automatic)")
    ap.add_argument("--cT", action="store_true",
                    help="--triples: the completely renormalised branch (cT = 1) of "
                         "PerturbativeTriplesReference")
    ap.add_argument("--shape", default=None,
                    help="No,Nv,NG of a real synthetic system instead of --config (profiling of "
                         "small cases)")
    ap.add_argument("--profile", action="store_true",
                    help="--triples: device time of each phase of the block loop")
    ap.add_argument("--vertex-scale", type=float, default=None,
                    help="scale of the synthetic vertex (default 0.2 for the CCSD line, the "
                         "reference arm, --converge and --adjoint: CCSD on the unscaled "
                         "synthetic vertex diverges at these sizes, strongly correlated; 1 for "
                         "--triples and --fsc)")
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
            scale = line["config"]["vertex_scale"]
            c = cpu_sample(args.config, scale)
            line["cpu_baseline"] = {"value": c["rate_tflops"], "unit": "TFLOP/s",
                                    "cores": c["cores"], "kind": "port", "sample": c["sample"]}
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
