"""Benchmark of the B200 APT solver.

Workload (default, one GPU): the 2D batched configuration — 256 independent
FP64 APT problems on sin-wavy meshes with sides drawn from U{64..512}, wave
amplitude U(0, 0.08), κ = Tⁿ with n ∈ {0, 1, 2.5, 3}, Gaussian centre
U(0.3, 0.7)² and width U(0.05, 0.2) from seed 20261203; every problem solves
each time step to rel ≤ 1e-8 or max|r|/√N ≤ 1e-8.  One bench step is one time
step (dt = 1e-5) of the whole batch.  Inputs are synthetic (seeded), there is
no dataset.

Metric: Gcell-iter/s = Σ_p (domain cells_p × pseudo-iterations_p) / time,
aggregated over all ranks.  With N GPUs the job is N seeded batches of 256
problems (seeds 20261203 .. +N-1, weak scaling) split over the ranks by the
library's sharded batch (longest-processing-time-first assignment by cells);
no field data crosses ranks, only each step's per-problem statistics.

CPU arms: `--impl reference` times the reference's CPU algorithm (the oracle
restatement, OpenMP on every host core) on a size-stratified quarter of the
256-problem batch (every 4th problem in order of size, 64 problems), each bench
step one time step of every sampled problem after the warm-up steps; the
`cpu_baseline` of our line is one post-warm-up time step of the same sample.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batch|gaussian128|gaussian2048|mms4096|mms1024|multigauss1024|
                              gauss3d256|gauss3d128]
                  [--precision fp64|fp64_exact|mixed] [--tuning V,H,K]
  python bench.py --compare [--workload W]     seconds per time step, FP64 vs mixed (vs learned)
  python bench.py --net-timing N               guess network: training step and N^2 prediction
  python bench.py --implicit N                 the implicit comparator, s/timestep on the N^2 multi-Gaussian
  python bench.py --implicit3d N               the same on the N^3 Gaussian pulse

Without --tuning the kernel variant, strip height and iteration block are
chosen by the library's autotuner before the warm-up (outside the timed
region); the choice is reported in `config`.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BYTES_PER_CELL_ITER = {2: 120, 3: 184}  # canonical algorithmic bytes, FP64 sweep
BYTES_PER_CELL_ITER_FP32 = {2: 60, 3: 92}  # FP32 correction sweep (mixed precision)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="batch",
                    choices=["batch", "gaussian128", "gaussian2048", "mms4096", "mms1024", "multigauss1024",
                             "gauss3d256", "gauss3d128"])
    ap.add_argument("--nprob", type=int, default=256)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "fp64_exact", "mixed"])
    ap.add_argument("--compare", action="store_true", help="single-problem s/timestep: fp64 vs mixed (vs learned)")
    ap.add_argument("--learned-steps", type=int, default=2000, help="APT steps of guess-network training data")
    ap.add_argument("--train-steps", type=int, default=3000, help="optimisation steps of the guess network")
    ap.add_argument("--smooth", type=int, default=8, help="smoothing passes of the predicted correction")
    ap.add_argument("--net-timing", type=int, default=0, metavar="N",
                    help="time the guess network: one training step on 16 x 128^2 crops, one N^2 prediction")
    ap.add_argument("--tuning", default="", metavar="V,H,K",
                    help="kernel variant, strip height, iteration block (skips the autotuner)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-compare", action="store_true",
                    help="skip the per-time-step FP64 / mixed / learned comparison of the default line")
    ap.add_argument("--compare-steps", type=int, default=3)
    ap.add_argument("--implicit", type=int, default=0, metavar="N",
                    help="time the implicit comparator on the N^2 multi-Gaussian problem (--steps, --warmup)")
    ap.add_argument("--implicit3d", type=int, default=0, metavar="N",
                    help="the same on the N^3 Gaussian pulse (kappa = T^2.5)")
    return ap.parse_args()


# ----------------------------------------------------------------- distributed
def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import torch.distributed as dist
        import datetime
        backend = "nccl" if args.impl == "ours" else "gloo"
        if args.impl == "ours":
            import torch
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
    return ws, rank, local


def barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def allreduce_max(x, ws, device=None):
    """Maximum over ranks (curvilineardiffusionmanuscript_b200.sharding.reduce_max)."""
    from curvilineardiffusionmanuscript_b200.sharding import reduce_max
    return reduce_max(x) if ws > 1 else x


def allreduce_sum(x, ws, device=None):
    """Sum over ranks (curvilineardiffusionmanuscript_b200.sharding.reduce_sum)."""
    from curvilineardiffusionmanuscript_b200.sharding import reduce_sum
    return reduce_sum(x) if ws > 1 else x


# -------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index=0):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ------------------------------------------------------------------- workloads
SINGLE = {
    "gaussian128": (lambda P, d: P.gaussian_2d(128, device=d), 130 * 130,
                    {"workload": "gaussian2d_128_fp64", "kappa": "T^3"}),
    "gaussian2048": (lambda P, d: P.gaussian_2d(2048, device=d), 2050 * 2050,
                     {"workload": "gaussian2d_2048_fp64", "kappa": "T^3"}),
    "gauss3d128": (lambda P, d: P.gaussian_3d(128, device=d), 130 ** 3,
                   {"workload": "gaussian3d_128_fp64", "kappa": "T^2.5"}),
    "gauss3d256": (lambda P, d: P.gaussian_3d(256, device=d), 258 ** 3,
                   {"workload": "gaussian3d_256_fp64", "kappa": "T^2.5"}),
    "mms4096": (lambda P, d: P.mms_2d(4096, device=d), 4098 * 4098, {"workload": "mms2d_4096", "kappa": "T^2.5"}),
    "mms1024": (lambda P, d: P.mms_2d(1024, device=d), 1026 * 1026, {"workload": "mms2d_1024", "kappa": "T^2.5"}),
    "multigauss1024": (lambda P, d: P.multi_gaussian_2d(1024, seed=12345, device=d), 1026 * 1026,
                       {"workload": "multigauss2d_1024", "kappa": "T^3"}),
}


def build_single(name, device):
    """The one problem of a single-problem workload, built on `device`."""
    from curvilineardiffusionmanuscript_b200 import problems as P
    return [SINGLE[name][0](P, device)]


def workload(name, nprob, ws):
    """(costs, build, cfg) of the whole job on ws ranks: one cost per problem
    (cells), build(indices, device) -> those problems, and the config record,
    which is the same for every arm of the benchmark."""
    from curvilineardiffusionmanuscript_b200 import problems as P
    if name == "batch":
        params = [q for r in range(ws) for q in P.batch_2d_params(nprob, seed=P.BATCH_SEED + r)]
        costs = [float(q["n"] ** 2) for q in params]
        build = lambda idx, device: [P.batch_problem(params[i], device=device) for i in idx]
        full = sum((q["n"] + 2) ** 2 for q in params)
        cfg = {"workload": "batch2d_256_fp64", "nprob": len(params), "sides": "U{64..512}",
               "seed": P.BATCH_SEED if ws == 1 else f"{P.BATCH_SEED}..{P.BATCH_SEED + ws - 1}", "dt": 1e-5,
               "tol": "rel <= 1e-8 or max|r|/sqrt(N) <= 1e-8", "bcs": "Neumann x4", "mean": "harmonic",
               "parallelism": f"dp{ws} (sharded batch, LPT by cells x expected iterations)"}
    else:
        make, full1, cfg = SINGLE[name]
        cfg = dict(cfg, dt=1e-5, tol="rel <= 1e-8 or max|r|/sqrt(N) <= 1e-8",
                   parallelism=f"dp{ws} (one replica per rank)")
        costs = [1.0] * ws
        build = lambda idx, device: [make(P, device) for _ in idx]
        full = full1 * ws
    cfg["l2"] = "inputs larger than L2 (working set %.1f GB per job)" % (full * 8 * 16 / 1e9)
    return costs, build, cfg


# ---------------------------------------------------------------- reference arm
def oracle_steps(probs, nsteps, states=None):
    """One time step of every problem per round with the oracle (the reference's
    CPU algorithm, OpenMP over every host core); returns per-round seconds and
    cell-iterations, and the solver states to continue from."""
    from oracle.oracle import OracleSolver
    if states is None:
        # host copies of every input are made here, outside the timed rounds
        states = []
        for p in probs:
            o = OracleSolver(p.mesh.to("cpu"), p.bcs)
            if p.source is not None:
                o.set_source(p.source.cpu().numpy())
            states.append((o, p.T0.cpu().numpy().copy(), p.rho.cpu().numpy().copy()))
    rounds = []
    for _ in range(nsteps):
        t0 = time.perf_counter()
        ci = 0
        for p, (o, T, rho) in zip(probs, states):
            st, _ = o.step(T, rho, p.cp, p.kappa.k0, p.kappa.n, p.dt, rtol=p.rtol, atol=p.atol, max_iter=100000)
            ci += p.mesh.ncells * st["niter"]
        rounds.append((time.perf_counter() - t0, ci))
    return rounds, states


def cpu_sample(costs, ws):
    """Problems the CPU arms time: a size-stratified quarter of the first
    256-problem batch (every 4th problem in order of cells, from the second), or
    the single problem of a one-problem workload."""
    n_one = len(costs) // ws
    if n_one == 1:
        return [0], "the workload's problem"
    order = sorted(range(n_one), key=lambda i: (costs[i], i))
    idx = sorted(order[1::4])
    return idx, (f"{len(idx)} of the batch's {n_one} problems, every 4th in order of size "
                 f"(cells {sum(costs[i] for i in idx) / sum(costs[:n_one]):.3f} of the batch)")


def run_reference(args, ws, rank):
    """The reference's CPU algorithm (the oracle restatement: the Julia reference
    cannot run here) on the host cores: every bench step is one time step of
    every problem of the stratified sample (rank 0 alone)."""
    if rank != 0:
        return
    from oracle.oracle import num_threads, set_threads
    set_threads(len(os.sched_getaffinity(0)))  # every host core this process may use
    costs, build, cfg = workload(args.workload, args.nprob, ws)
    idx, what = cpu_sample(costs, ws)
    probs = build(idx, "cpu")
    _, states = oracle_steps(probs, args.warmup)
    rounds, _ = oracle_steps(probs, args.steps, states)
    tot_t = sum(t for t, _ in rounds)
    v = sum(c for _, c in rounds) / tot_t / 1e9
    line = {"metric": "Gcell-iter/s", "value": v, "unit": "Gcell-iter/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "Gcell-iter/s", "cores": num_threads(), "kind": "port",
                             "sample": f"{what}, one time step each per bench step, after {args.warmup} "
                                       f"warm-up steps"},
            "e2e": {"value": v, "unit": "Gcell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(probs, what):
    """The oracle (OpenMP, all host threads) on a bounded sample of the workload:
    one untimed time step of every sampled problem (the first step checks the
    residual at every iteration), then one timed step."""
    from oracle.oracle import num_threads, set_threads
    set_threads(len(os.sched_getaffinity(0)))  # every host core this process may use
    _, states = oracle_steps(probs, 1)
    ((tt, ci),), _ = oracle_steps(probs, 1, states)
    return {"value": ci / tt / 1e9, "unit": "Gcell-iter/s", "cores": num_threads(), "kind": "port",
            "sample": f"{what}, the second time step of each"}


# ---------------------------------------------------------------------- ours
def run_ours(args, ws, rank, local):
    import torch
    from curvilineardiffusionmanuscript_b200.sharding import ShardedBatch
    from curvilineardiffusionmanuscript_b200.solver import PseudoTransientBatch
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    costs, build, cfg = workload(args.workload, args.nprob, ws)
    stream = torch.cuda.current_stream(dev)
    mixed = args.precision == "mixed"
    local_probs = {}

    def build_local(idx):
        for i, pr in zip(idx, build(idx, dev)):
            local_probs[i] = pr
        return [local_probs[i].mesh for i in idx], [local_probs[i].bcs for i in idx]

    # the library's multi-GPU path: every rank builds and steps its LPT share, the
    # batch's problems weighted by cells x expected iterations (the counts differ by
    # 30x over the batch: by cells alone 8 ranks would carry up to 9 % unequal work)
    weights = costs
    if args.workload == "batch":
        from curvilineardiffusionmanuscript_b200 import problems as P
        params = [q for r in range(ws) for q in P.batch_2d_params(args.nprob, seed=P.BATCH_SEED + r)]
        weights = [c * P.batch_expected_iterations(q) for c, q in zip(costs, params)]
    sb = ShardedBatch.from_factory(weights, build_local, make_batch=PseudoTransientBatch, stream=stream.cuda_stream,
                                   precision=args.precision)
    mine = sb.local
    probs = [local_probs[i] for i in mine]
    nd = probs[0].mesh.ndim
    for k, pr in enumerate(probs):
        if pr.source is not None:
            sb.batch.set_source(k, pr.source)
    n = sb.n

    def full(local_list):  # global-order list with this rank's entries
        out = [None] * n
        for i, x in zip(mine, local_list):
            out[i] = x
        return out

    Ts = [pr.T0.clone() for pr in probs]
    rhos = [pr.rho for pr in probs]
    cps, kaps, dts = full([pr.cp for pr in probs]), full([pr.kappa for pr in probs]), full([pr.dt for pr in probs])
    kw = dict(rtol=probs[0].rtol, atol=probs[0].atol, max_iter=100000)

    def one_step(T_list, R_list):
        st, _ = sb.step(full(T_list), full(R_list), cps, kaps, dts, **kw)
        return st, sb.batch.profile()

    # kernel variant, strip height and iteration block timed on this rank's batch
    # (set-up, outside the timed region), from the state after one time step:
    # the first step of a problem checks its residual at every iteration
    # (PseudoTransientSolver.jl:206-208, last_err_check = 0), the later ones on
    # the schedule its previous step sets
    one_step(Ts, rhos)
    if args.tuning:
        sb.batch.set_tuning(*[int(v) for v in args.tuning.split(",")])
        tuning = sb.batch.tuning()
    else:
        cand = sb.batch.autotune(Ts, rhos, [pr.cp for pr in probs], [pr.kappa for pr in probs],
                                 [pr.dt for pr in probs], **kw)
        tuning = dict(candidate=cand, **sb.batch.tuning())

    for _ in range(args.warmup):
        one_step(Ts, rhos)
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ci, sweep_ms, launches, sweep_launches, iters, last = 0, 0.0, 0, 0, [], None
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("bench_timed")
        e0.record(stream)
        for _ in range(args.steps):
            st, pf = one_step(Ts, rhos)
            ci += pf["cell_iters"]
            sweep_ms += pf["sweep_ms"]
            launches += pf["sweep_launches"] + pf["other_launches"]
            sweep_launches += pf["sweep_launches"]
            iters.append(sum(x["niter"] for x in st))
            last = st
        e1.record(stream)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    ms = e0.elapsed_time(e1)
    barrier(ws)
    ms_max = allreduce_max(ms, ws, dev)
    ci_tot = allreduce_sum(float(ci), ws, dev)
    value = ci_tot / (ms_max / 1e3) / 1e9
    peak, peak_kind = measured_peak()
    bpc = (BYTES_PER_CELL_ITER_FP32 if mixed else BYTES_PER_CELL_ITER)[nd]
    achieved = ci * bpc / (sweep_ms / 1e3) / 1e9 if sweep_ms > 0 else 0.0
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": None, "kernel": f"sweep{nd}d_{'fp32' if mixed else 'fp64'}", "peak_kind": peak_kind,
            "bytes_per_cell_iter": bpc}
    tb = traffic_per_cell_iter(nd, args.workload, mixed)
    if tb is not None:
        # DRAM bytes per cell-iteration of one ncu capture, times the cells one sweep launch updates
        roof["traffic"] = tb[0] * ci / max(1, sweep_launches)
        roof["traffic_source"] = tb[1]
    # the residual each problem stopped at in the last timed step (rule: rel <= 1e-8 or abs <= 1e-8)
    absr = sorted(x["abs_err"] for x in last)
    final = {"abs_err_max": absr[-1], "abs_err_median": absr[len(absr) // 2],
             "stopped_by_rel": sum(1 for x in last if x["abs_err"] > kw["atol"]), "problems": len(last),
             "niter_min": min(x["niter"] for x in last), "niter_max": max(x["niter"] for x in last)}
    e2e = None
    if not args.no_e2e:
        # end to end through the public API with host (pinned) buffers
        Th = [t.cpu().pin_memory() for t in Ts]
        Rh = [r.cpu().pin_memory() for r in rhos]
        one_step(Th, Rh)  # warm the host path
        barrier(ws)
        torch.cuda.synchronize()
        ci2 = 0
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            _, pf = one_step(Th, Rh)
            ci2 += pf["cell_iters"]
        f1.record(stream)
        torch.cuda.synchronize()
        ms2 = max(f0.elapsed_time(f1), 1e3 * (time.perf_counter() - t0))
        ms2 = allreduce_max(ms2, ws, dev)
        ci2 = allreduce_sum(float(ci2), ws, dev)
        nbytes = allreduce_sum(float(sum(t.numel() for t in Ts) * 8), ws, dev)
        e2e = {"value": ci2 / (ms2 / 1e3) / 1e9, "unit": "Gcell-iter/s", "h2d_bytes_per_step": int(2 * nbytes),
               "d2h_bytes_per_step": int(nbytes)}
    cpu = None
    if ws == 1 and not args.no_cpu:
        idx, what = cpu_sample(costs, ws)
        cpu = cpu_baseline([local_probs[i] for i in idx], what)
    sb.close()
    compare = None
    if ws == 1 and not args.no_compare and args.workload == "batch" and args.precision == "fp64":
        del Ts, rhos, local_probs, probs
        torch.cuda.empty_cache()
        compare = compare_block(args, stream)
    if rank != 0:
        return
    line = {"metric": "Gcell-iter/s", "value": value, "unit": "Gcell-iter/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": cfg, "tuning": tuning,
            "s_per_timestep": ms_max / args.steps / 1e3, "pseudo_iters_per_step": statistics.mean(iters),
            "final_residual": final, "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary(), "compare_s_per_timestep": compare}
    print(json.dumps(line), flush=True)


def traffic_per_cell_iter(nd, workload, mixed):
    """DRAM bytes per cell-iteration of the sweep kernel from profiles/traffic.json
    (one ncu capture per entry, its command recorded beside it): the entry of this
    workload where one exists, else the kernel's default entry."""
    f = ROOT / "profiles" / "traffic.json"
    if not f.exists():
        return None
    data = json.loads(f.read_text())
    kern = f"sweep{nd}d_{'fp32' if mixed else 'fp64'}"
    for key in (f"{kern}/{workload}", kern):
        if key in data:
            return float(data[key]["dram_bytes_per_cell_iter"]), f"profiles/traffic.json:{key}"
    return None


def time_single(pr, precision, steps, warmup, stream, net=None, rtol=None, max_iter=100000, extrapolate=False):
    """Seconds per time step of one problem (CUDA events on the solver's stream).
    With a guess network the steps after the first start from its prediction,
    with `extrapolate` from 2Tⁿ − Tⁿ⁻¹; the guess and the plain-start probe are
    inside the timed step.  `rtol` replaces the workload's relative tolerance
    (0: the absolute test alone)."""
    import torch
    from curvilineardiffusionmanuscript_b200 import _lib, learned, problems
    from curvilineardiffusionmanuscript_b200.solver import PseudoTransientSolver, step
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision=precision, stream=stream.cuda_stream)
    guess = _lib.CDM_GUESS_EXTRAPOLATE if extrapolate else _lib.CDM_GUESS_PREV
    if net is not None:
        learned.attach(g, net)
        guess = _lib.CDM_GUESS_LEARNED
    try:
        T = pr.T0.clone()
        t = 0.0
        mms = pr.name == "mms_2d"
        times, iters, restarts, absr, initr = [], [], [], [], []
        for k in range(warmup + steps):
            if mms:
                g.set_source(problems.mms_source(pr, t + pr.dt))
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, _ = step(g, pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt, rtol=pr.rtol if rtol is None else rtol,
                         atol=pr.atol, max_iter=max_iter, guess=guess)
            e1.record(stream)
            torch.cuda.synchronize()
            t += pr.dt
            if k >= warmup:
                times.append(e0.elapsed_time(e1) / 1e3)
                iters.append(st["niter"])
                restarts.append(st["n_restarts"])
                absr.append(st["abs_err"])
                # the residual the relative test divides by: that of the first iteration
                if st["rel_err"] > 0:
                    initr.append(st["abs_err"] / st["rel_err"])
        out = {"s_per_step": statistics.median(times), "iters": statistics.mean(iters),
               "restarts": statistics.mean(restarts), "final_abs_err": statistics.mean(absr),
               "first_residual": statistics.mean(initr) if initr else None}
        if mms:
            out["err_vs_exact"] = problems.mms_error(pr, T, t)
    finally:
        g.close()
    return out


# algorithmic bytes per row of one BiCGSTAB iteration of the implicit solve: the
# stored stencil entries twice (two products with A; 9 in 2D, 19 in 3D) and the
# 25 vector reads and writes of its five kernels (p, p̂, v, s, ŝ, t, x, r, r̂, D⁻¹)
IMPLICIT_BYTES_PER_ROW_ITER = {2: (2 * 9 + 25) * 8, 3: (2 * 19 + 25) * 8}


def time_implicit(pr, steps, warmup, stream):
    """Seconds per time step of the reference's implicit comparator (backward
    Euler, Krylov solve to atol = rtol = 1e-9 as _iterative_solve! defaults)
    on one problem, CUDA events around each step's library call."""
    import torch
    from curvilineardiffusionmanuscript_b200.solver import ImplicitScheme
    g = ImplicitScheme(pr.mesh, pr.bcs, stream=stream.cuda_stream)
    try:
        T = pr.T0.clone()
        times, iters, res, gbs = [], [], [], []
        for k in range(warmup + steps):
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st, _ = g.step(pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt)
            e1.record(stream)
            torch.cuda.synchronize()
            if k >= warmup:
                pf = g.profile()
                times.append(e0.elapsed_time(e1) / 1e3)
                iters.append(st["niter"])
                res.append(st["abs_err"])
                if pf["solve_ms"] > 0:
                    gbs.append(IMPLICIT_BYTES_PER_ROW_ITER[pr.mesh.ndim] * pf["rows"] * st["niter"]
                               / (pf["solve_ms"] / 1e3) / 1e9)
        return {"s_per_step": statistics.median(times), "krylov_iters": statistics.mean(iters),
                "final_residual_2norm": statistics.mean(res), "tol": "atol = rtol = 1e-9 (2-norm)",
                "solver": "BiCGSTAB, Jacobi preconditioner on the right",
                "solve_GBs": statistics.mean(gbs) if gbs else None,
                "bytes_per_row_iter": IMPLICIT_BYTES_PER_ROW_ITER[pr.mesh.ndim]}
    finally:
        g.close()


def train_guess(n, nseeds, nsteps, train_steps):
    """Guess network trained on APT trajectories of the multi-Gaussian problem
    (seeds disjoint from the timed problem's)."""
    from curvilineardiffusionmanuscript_b200.train_guess import train_multigauss
    return train_multigauss(n, nseeds, nsteps, train_steps)


def compare_block(args, stream):
    """Seconds per time step to the workloads' stopping rule (rel <= 1e-8 or
    abs <= 1e-8), one GPU, CUDA events around each step's library call:
    the 4096^2 manufactured solution in FP64 and in mixed precision (with each
    one's error against the exact solution), and the 1024^2 multi-Gaussian in
    FP64, mixed precision and learned guess + mixed precision, the network
    loaded from the checkpoint the project's trainer wrote
    (python -m curvilineardiffusionmanuscript_b200.train_guess); the same after
    20 warm-up steps, with the extrapolated start 2Tⁿ − Tⁿ⁻¹ beside them; and the
    reference's implicit scheme on the same problem."""
    import torch
    from curvilineardiffusionmanuscript_b200 import learned
    from curvilineardiffusionmanuscript_b200.train_guess import DEFAULT_CHECKPOINT
    dev = torch.device("cuda", torch.cuda.current_device())
    out = {"steps": args.compare_steps, "warmup": 2, "timing": "median of the timed steps"}
    w = {}
    for prec in ("fp64", "mixed"):
        w[prec] = time_single(build_single("mms4096", dev)[0], prec, args.compare_steps, 2, stream)
    w["speedup_mixed_vs_fp64"] = w["fp64"]["s_per_step"] / w["mixed"]["s_per_step"]
    out["mms2d_4096"] = w
    w = {}
    for prec in ("fp64", "mixed"):
        w[prec] = time_single(build_single("multigauss1024", dev)[0], prec, args.compare_steps, 2, stream)
    w["speedup_mixed_vs_fp64"] = w["fp64"]["s_per_step"] / w["mixed"]["s_per_step"]
    # the manuscript's comparison: the reference's implicit scheme on the same problem
    w["implicit_krylov"] = time_implicit(build_single("multigauss1024", dev)[0], args.compare_steps, 2, stream)
    w["implicit_s_per_step_over_fp64"] = w["implicit_krylov"]["s_per_step"] / w["fp64"]["s_per_step"]
    if DEFAULT_CHECKPOINT.exists():
        net = learned.GuessNet(seed=0)
        net.load(DEFAULT_CHECKPOINT)
        for prec in ("fp64", "mixed"):
            w["learned_" + prec] = time_single(build_single("multigauss1024", dev)[0], prec, args.compare_steps, 2,
                                               stream, net=net)
        w["speedup_learned_mixed_vs_fp64"] = w["fp64"]["s_per_step"] / w["learned_mixed"]["s_per_step"]
        # the absolute test alone (max|r|/sqrt(N) <= 1e-8, rtol = 0): there a start
        # closer to the solution saves the decades of residual it removes
        a = {}
        for key, prec, nn in (("fp64", "fp64", None), ("learned_fp64", "fp64", net), ("mixed", "mixed", None),
                              ("learned_mixed", "mixed", net)):
            try:
                a[key] = time_single(build_single("multigauss1024", dev)[0], prec, args.compare_steps, 2, stream,
                                     net=nn, rtol=0.0, max_iter=20000)
            except RuntimeError as err:  # a step that does not reach the absolute test is reported, not fatal
                a[key] = {"unavailable": str(err)[:200]}
        if "s_per_step" in a["fp64"] and "s_per_step" in a["learned_mixed"]:
            a["speedup_learned_mixed_vs_fp64"] = a["fp64"]["s_per_step"] / a["learned_mixed"]["s_per_step"]
        w["absolute_test_only"] = a
        # after 20 steps: the reference's check schedule (the first check at 0.9 x the
        # previous step's count, PseudoTransientSolver.jl:206-208) has come down to
        # where the residual converges, so a start's gain shows in the count
        st = {"warmup_steps": 20}
        for key, prec, nn, ex in (("fp64", "fp64", None, False), ("mixed", "mixed", None, False),
                                  ("extrapolated_fp64", "fp64", None, True),
                                  ("extrapolated_mixed", "mixed", None, True),
                                  ("learned_mixed", "mixed", net, False)):
            st[key] = time_single(build_single("multigauss1024", dev)[0], prec, args.compare_steps, 20, stream,
                                  net=nn, extrapolate=ex)
        for key in ("mixed", "extrapolated_fp64", "extrapolated_mixed", "learned_mixed"):
            st["speedup_" + key + "_vs_fp64"] = st["fp64"]["s_per_step"] / st[key]["s_per_step"]
        w["after_20_steps"] = st
        w["checkpoint"] = str(DEFAULT_CHECKPOINT.relative_to(ROOT))
        net.close()
    else:
        w["learned_mixed"] = {"unavailable": "no checkpoint at " + str(DEFAULT_CHECKPOINT.relative_to(ROOT))}
    out["multigauss2d_1024"] = w
    return out


def run_compare(args):
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    res = {}
    for wl in (["mms4096", "multigauss1024"] if args.workload == "batch" else [args.workload]):
        r = {}
        for prec in ("fp64", "mixed"):
            probs = build_single(wl, dev)
            r[prec] = time_single(probs[0], prec, args.steps, args.warmup, stream)
        r["speedup_mixed_vs_fp64"] = r["fp64"]["s_per_step"] / r["mixed"]["s_per_step"]
        if wl.startswith("multigauss") and args.learned_steps > 0:
            n = probs[0].mesh.ni
            net, info = train_guess(n, args.learned_steps // 8, 8, args.train_steps)
            net.set_smoothing(args.smooth)
            info["smoothing_passes"] = args.smooth
            r["training"] = info
            for prec in ("fp64", "mixed"):
                probs = build_single(wl, dev)
                r["learned_" + prec] = time_single(probs[0], prec, args.steps, args.warmup, stream, net=net)
            r["speedup_learned_fp64_vs_fp64"] = r["fp64"]["s_per_step"] / r["learned_fp64"]["s_per_step"]
            r["speedup_learned_mixed_vs_fp64"] = r["fp64"]["s_per_step"] / r["learned_mixed"]["s_per_step"]
            net.close()
        res[wl] = r
    print(json.dumps({"compare": res}), flush=True)


def run_net_timing(args):
    """Milliseconds per guess-network training step (16 crops of 128², Adam
    included) and per N² prediction, CUDA events on the current stream, after
    `--warmup` untimed repetitions; trained on 2 seeds × 3 APT steps."""
    import torch
    from curvilineardiffusionmanuscript_b200 import learned, problems
    n = args.net_timing
    make = lambda seed: problems.multi_gaussian_2d(n, seed=seed, device="cuda")
    pr = make(1)
    trajs = learned.generate_trajectories(make, seeds=[1, 2], nsteps=3)
    net = learned.GuessNet(seed=0)
    ljm = learned.log_jmean(pr.mesh)
    stream = torch.cuda.current_stream()

    def timed(fn, reps):
        fn(args.warmup)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn(reps)
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def train(k):
        learned.train(net, trajs, pr.mesh, pr.kappa.k0, pr.kappa.n, steps=k, batch=16, crop=128)

    def predict(k):
        for _ in range(k):
            net.predict(trajs[0][0], trajs[0][1], pr.mesh, pr.kappa.k0, pr.kappa.n, ljm)

    out = {"net_timing": {"train_step_ms": timed(train, args.steps), "predict_ms": timed(predict, args.steps),
                          "n": n, "batch": 16, "crop": 128, "params": net.nparams}}
    net.close()
    print(json.dumps(out), flush=True)


def run_implicit(args):
    """Seconds per time step of the implicit comparator on the N² multi-Gaussian
    problem (κ = T³, seed 0) or the N³ Gaussian pulse (κ = T^2.5), one JSON line."""
    import torch
    from curvilineardiffusionmanuscript_b200 import problems
    dev = torch.device("cuda", 0)
    if args.implicit3d:
        n, nd = args.implicit3d, 3
        pr = problems.gaussian_3d(n, device=dev)
    else:
        n, nd = args.implicit, 2
        pr = problems.multi_gaussian_2d(n, seed=0, device=dev)
    r = time_implicit(pr, args.steps, args.warmup, torch.cuda.current_stream(dev))
    r.update(n=n, ndim=nd, rows=(n + 2) ** nd)
    peak, kind = measured_peak()
    if r["solve_GBs"]:
        r["roofline"] = {"bound": "hbm", "achieved": r["solve_GBs"], "peak": peak, "unit": "GB/s",
                         "frac": r["solve_GBs"] / peak, "peak_kind": kind}
    print(json.dumps({"implicit": r}), flush=True)


def main():
    args = parse()
    if args.implicit or args.implicit3d:
        run_implicit(args)
        return
    if args.net_timing:
        run_net_timing(args)
        return
    if args.compare:
        run_compare(args)
        return
    ws, rank, local = dist_setup(args)
    try:
        if args.impl == "reference":
            run_reference(args, ws, rank)
        else:
            run_ours(args, ws, rank, local)
    finally:
        if ws > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
