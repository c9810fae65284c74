"""Benchmark of the B200 APT solver.

Workload (default, one GPU): the 2D batched configuration — 256 independent
FP64 APT problems on sin-wavy meshes with sides drawn from U{64..512}, wave
amplitude U(0, 0.08), κ = Tⁿ with n ∈ {0, 1, 2.5, 3}, Gaussian centre
U(0.3, 0.7)² and width U(0.05, 0.2) from seed 20261203; every problem solves
each time step to rel ≤ 1e-8 or max|r|/√N ≤ 1e-8.  One bench step is one time
step (dt = 1e-5) of the whole batch.  Inputs are synthetic (seeded), there is
no dataset.

Metric: Gcell-iter/s = Σ_p (domain cells_p × pseudo-iterations_p) / time,
aggregated over all ranks (each rank solves its own seeded batch: weak
scaling, no collective in the data path).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload batch|gaussian128|gaussian2048|mms4096|mms1024|multigauss1024|
                              gauss3d256|gauss3d128]
                  [--precision fp64|fp64_exact|mixed] [--tuning V,H,K]
  python bench.py --compare [--workload W]     seconds per time step, FP64 vs mixed (vs learned)
  python bench.py --net-timing N               guess network: training step and N^2 prediction

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
def make_workload(name, nprob, rank, device):
    from curvilineardiffusionmanuscript_b200 import problems
    if name == "batch":
        probs = problems.batch_2d(nprob=nprob, seed=problems.BATCH_SEED + rank, device=device)
        cfg = {"workload": "batch2d_256_fp64", "nprob": nprob, "sides": "U{64..512}", "seed": problems.BATCH_SEED,
               "dt": 1e-5, "tol": "rel <= 1e-8 or max|r|/sqrt(N) <= 1e-8", "bcs": "Neumann x4", "mean": "harmonic"}
    elif name == "gaussian128":
        probs = [problems.gaussian_2d(128, device=device)]
        cfg = {"workload": "gaussian2d_128_fp64", "kappa": "T^3", "dt": 1e-5, "tol": 1e-8}
    elif name == "gaussian2048":
        probs = [problems.gaussian_2d(2048, device=device)]
        cfg = {"workload": "gaussian2d_2048_fp64", "kappa": "T^3", "dt": 1e-5, "tol": 1e-8}
    elif name == "gauss3d128":
        probs = [problems.gaussian_3d(128, device=device)]
        cfg = {"workload": "gaussian3d_128_fp64", "kappa": "T^2.5", "dt": 1e-5, "tol": 1e-8}
    elif name == "mms4096":
        probs = [problems.mms_2d(4096, device=device)]
        cfg = {"workload": "mms2d_4096", "kappa": "T^2.5", "dt": 1e-5, "tol": 1e-8}
    elif name == "mms1024":
        probs = [problems.mms_2d(1024, device=device)]
        cfg = {"workload": "mms2d_1024", "kappa": "T^2.5", "dt": 1e-5, "tol": 1e-8}
    elif name == "multigauss1024":
        probs = [problems.multi_gaussian_2d(1024, seed=12345, device=device)]
        cfg = {"workload": "multigauss2d_1024", "kappa": "T^3", "dt": 1e-5, "tol": 1e-8}
    else:
        probs = [problems.gaussian_3d(256, device=device)]
        cfg = {"workload": "gaussian3d_256_fp64", "kappa": "T^2.5", "dt": 1e-5, "tol": 1e-8}
    return probs, cfg


# ---------------------------------------------------------------- reference arm
def run_reference(args, ws, rank):
    """The reference's CPU algorithm (the oracle restatement: the Julia reference
    cannot run here) on the host cores, each step a bounded sample."""
    if rank != 0:
        return
    import torch
    from oracle.oracle import OracleSolver, num_threads, set_threads
    set_threads(len(os.sched_getaffinity(0)))  # every host core this process may use
    probs, cfg = make_workload(args.workload, args.nprob, 0, "cpu")
    sample = probs[: min(len(probs), 6)] if args.workload == "batch" else probs
    solvers = [OracleSolver(p.mesh, p.bcs) for p in sample]
    Ts = [p.T0.numpy().copy() for p in sample]
    for p, o in zip(sample, solvers):
        if p.source is not None:
            o.set_source(p.source.numpy())
    tot_ci, tot_t = 0, 0.0
    for s in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        ci = 0
        for p, o, T in zip(sample, solvers, Ts):
            st, _ = o.step(T, p.rho.numpy(), p.cp, p.kappa.k0, p.kappa.n, p.dt, rtol=p.rtol, atol=p.atol,
                           max_iter=100000)
            ci += p.mesh.ncells * st["niter"]
        dt = time.perf_counter() - t0
        if s >= args.warmup:
            tot_ci += ci
            tot_t += dt
    v = tot_ci / tot_t / 1e9
    cores = num_threads()
    line = {"metric": "Gcell-iter/s", "value": v, "unit": "Gcell-iter/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg, "impl": "reference",
            "cpu_baseline": {"value": v, "unit": "Gcell-iter/s", "cores": cores, "kind": "port",
                             "sample": f"first {len(sample)} problems of the workload, one time step each per bench step"},
            "e2e": {"value": v, "unit": "Gcell-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(probs, budget_s=15.0):
    """Oracle (OpenMP, all host threads) on a bounded sample of the workload."""
    from oracle.oracle import OracleSolver, num_threads, set_threads
    set_threads(len(os.sched_getaffinity(0)))  # every host core this process may use
    t_start = time.perf_counter()
    ci, tt, used = 0, 0.0, 0
    for p in probs:
        o = OracleSolver(p.mesh.to("cpu"), p.bcs)
        T = p.T0.cpu().numpy().copy()
        if p.source is not None:
            o.set_source(p.source.cpu().numpy())
        t0 = time.perf_counter()
        st, _ = o.step(T, p.rho.cpu().numpy(), p.cp, p.kappa.k0, p.kappa.n, p.dt, rtol=p.rtol, atol=p.atol,
                       max_iter=100000)
        tt += time.perf_counter() - t0
        ci += p.mesh.ncells * st["niter"]
        used += 1
        if time.perf_counter() - t_start > budget_s:
            break
    return {"value": ci / tt / 1e9, "unit": "Gcell-iter/s", "cores": num_threads(), "kind": "port",
            "sample": f"first time step of {used} problem(s) of the workload"}


# ---------------------------------------------------------------------- ours
def run_ours(args, ws, rank, local):
    import torch
    from curvilineardiffusionmanuscript_b200.solver import PseudoTransientBatch, PseudoTransientSolver, step
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    probs, cfg = make_workload(args.workload, args.nprob, rank, dev)
    nd = probs[0].mesh.ndim
    stream = torch.cuda.current_stream(dev)
    mixed = args.precision == "mixed"
    batch = PseudoTransientBatch([p.mesh for p in probs], [p.bcs for p in probs], stream=stream.cuda_stream,
                                 precision=args.precision)
    for i, p in enumerate(probs):
        if p.source is not None:
            batch.set_source(i, p.source)
    Ts = [p.T0.clone() for p in probs]
    rhos = [p.rho for p in probs]
    cps = [p.cp for p in probs]
    kaps = [p.kappa for p in probs]
    dts = [p.dt for p in probs]
    kw = dict(rtol=probs[0].rtol, atol=probs[0].atol, max_iter=100000)
    # strip height and iteration-block length timed on this batch (set-up, outside the timed region)
    if args.tuning:
        batch.set_tuning(*[int(v) for v in args.tuning.split(",")])
        cfg["tuning"] = batch.tuning()
    else:
        tuned = batch.autotune(Ts, rhos, cps, kaps, dts, **kw)
        cfg["autotune"] = dict(candidate=tuned, **batch.tuning())

    def one_step():
        st, _ = batch.step(Ts, rhos, cps, kaps, dts, **kw)
        return st, batch.profile()

    for _ in range(args.warmup):
        one_step()
    barrier(ws)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ci, sweep_ms, launches, sweep_launches, iters = 0, 0.0, 0, 0, []
    with ClockSampler(local) as clk:
        torch.cuda.nvtx.range_push("bench_timed")
        e0.record(stream)
        for _ in range(args.steps):
            st, pf = one_step()
            ci += pf["cell_iters"]
            sweep_ms += pf["sweep_ms"]
            launches += pf["sweep_launches"] + pf["other_launches"]
            sweep_launches += pf["sweep_launches"]
            iters.append(sum(s["niter"] for s in st))
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
    tb, tsrc = traffic_per_cell_iter(nd, args.workload) if not mixed else (None, None)
    if tb is not None:
        # DRAM bytes per cell-iteration from one ncu capture, times the cells one sweep updates
        roof["traffic"] = tb * ci / max(1, sweep_launches)
        roof["traffic_source"] = tsrc
    e2e = None
    if not args.no_e2e:
        # end to end through the public API with host (pinned) buffers
        Th = [t.cpu().pin_memory() for t in Ts]
        Rh = [r.cpu().pin_memory() for r in rhos]
        st, _ = batch.step(Th, Rh, cps, kaps, dts, **kw)  # warm the host path
        barrier(ws)
        torch.cuda.synchronize()
        ci2 = 0
        t0 = time.perf_counter()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        for _ in range(args.steps):
            st, _ = batch.step(Th, Rh, cps, kaps, dts, **kw)
            ci2 += batch.profile()["cell_iters"]
        f1.record(stream)
        torch.cuda.synchronize()
        ms2 = max(f0.elapsed_time(f1), 1e3 * (time.perf_counter() - t0))
        ms2 = allreduce_max(ms2, ws, dev)
        ci2 = allreduce_sum(float(ci2), ws, dev)
        nbytes = sum(t.numel() for t in Ts) * 8
        e2e = {"value": ci2 / (ms2 / 1e3) / 1e9, "unit": "Gcell-iter/s", "h2d_bytes_per_step": 2 * nbytes,
               "d2h_bytes_per_step": nbytes}
    if rank != 0:
        return
    cpu = None
    if ws == 1 and not args.no_cpu:
        cpu = cpu_baseline(probs[:64])
    cfg.update({"l2": "inputs larger than L2 (working set %.1f GB)" % (
        sum(p.mesh.ncells_full for p in probs) * 8 * 16 / 1e9), "parallelism": f"dp{ws} (independent batches)"})
    line = {"metric": "Gcell-iter/s", "value": value, "unit": "Gcell-iter/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64" if mixed else "f64", "data": "synthetic",
            "config": cfg,
            "s_per_timestep": ms_max / args.steps / 1e3, "pseudo_iters_per_step": statistics.mean(iters),
            "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    batch.close()


TRAFFIC_SUMMARY = {2: {"batch": "sweep2d_fp64_batch.md"}, 3: {}}
TRAFFIC_DEFAULT = {2: "sweep2d_fp64_gaussian2048.md", 3: "sweep3d_fp64_gauss3d.md"}


def traffic_per_cell_iter(nd, workload):
    """DRAM bytes per cell-iteration of the sweep, read from the committed ncu summary
    (line `dram_bytes_per_cell_iter: X`): the capture of this workload where one
    exists, else the 2048^2 (2D) / 3D capture, scaled by the cells a sweep updates."""
    import re
    for name in (TRAFFIC_SUMMARY[nd].get(workload), TRAFFIC_DEFAULT[nd]):
        if not name:
            continue
        f = ROOT / "profiles" / name
        if f.exists():
            m = re.search(r"^dram_bytes_per_cell_iter:\s*([0-9.]+)", f.read_text(), re.M)
            if m:
                return float(m.group(1)), "profiles/" + name
    return None, None


def time_single(pr, precision, steps, warmup, stream, net=None):
    """Seconds per time step of one problem (CUDA events on the solver's stream).
    With a guess network the steps after the first start from its prediction;
    the prediction and the plain-start probe are inside the timed step."""
    import torch
    from curvilineardiffusionmanuscript_b200 import _lib, learned, problems
    from curvilineardiffusionmanuscript_b200.solver import PseudoTransientSolver, step
    g = PseudoTransientSolver(pr.mesh, pr.bcs, precision=precision, stream=stream.cuda_stream)
    guess = _lib.CDM_GUESS_PREV
    if net is not None:
        learned.attach(g, net)
        guess = _lib.CDM_GUESS_LEARNED
    T = pr.T0.clone()
    t = 0.0
    mms = pr.name == "mms_2d"
    times, iters, restarts = [], [], []
    for k in range(warmup + steps):
        if mms:
            g.set_source(problems.mms_source(pr, t + pr.dt))
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st, _ = step(g, pr.mesh, T, pr.rho, pr.cp, pr.kappa, pr.dt, rtol=pr.rtol, atol=pr.atol, max_iter=100000,
                     guess=guess)
        e1.record(stream)
        torch.cuda.synchronize()
        t += pr.dt
        if k >= warmup:
            times.append(e0.elapsed_time(e1) / 1e3)
            iters.append(st["niter"])
            restarts.append(st["n_restarts"])
    out = {"s_per_step": statistics.median(times), "iters": statistics.mean(iters),
           "restarts": statistics.mean(restarts)}
    if mms:
        out["err_vs_exact"] = problems.mms_error(pr, T, t)
    g.close()
    return out


def train_guess(n, nseeds, nsteps, train_steps):
    """Guess network trained on APT trajectories of the multi-Gaussian problem
    (seeds disjoint from the timed problem's)."""
    import time as _t
    import torch
    from curvilineardiffusionmanuscript_b200 import learned, problems
    make = lambda seed: problems.multi_gaussian_2d(n, seed=seed, device="cuda")
    t0 = _t.time()
    skipped = []
    trajs = learned.generate_trajectories(make, seeds=list(range(1000, 1000 + nseeds)), nsteps=nsteps,
                                          skipped=skipped)
    t1 = _t.time()
    net = learned.GuessNet(seed=1)
    pr0 = make(1000)
    losses = learned.train(net, trajs, pr0.mesh, pr0.kappa.k0, pr0.kappa.n, steps=train_steps, batch=16, crop=128,
                           lr=2e-3)
    torch.cuda.synchronize()
    info = {"apt_steps": len(trajs) * nsteps, "seeds_diverged": len(skipped), "data_s": round(t1 - t0, 1), "train_s": round(_t.time() - t1, 1),
            "train_steps": train_steps, "loss_first": float(sum(losses[:10]) / 10),
            "loss_last": float(sum(losses[-50:]) / 50)}
    del trajs
    torch.cuda.empty_cache()
    return net, info


def run_compare(args):
    import torch
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    res = {}
    for wl in (["mms4096", "multigauss1024"] if args.workload == "batch" else [args.workload]):
        r = {}
        for prec in ("fp64", "mixed"):
            probs, cfg = make_workload(wl, 1, 0, dev)
            r[prec] = time_single(probs[0], prec, args.steps, args.warmup, stream)
        r["speedup_mixed_vs_fp64"] = r["fp64"]["s_per_step"] / r["mixed"]["s_per_step"]
        if wl.startswith("multigauss") and args.learned_steps > 0:
            n = probs[0].mesh.ni
            net, info = train_guess(n, args.learned_steps // 8, 8, args.train_steps)
            net.set_smoothing(args.smooth)
            info["smoothing_passes"] = args.smooth
            r["training"] = info
            for prec in ("fp64", "mixed"):
                probs, cfg = make_workload(wl, 1, 0, dev)
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


def main():
    args = parse()
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
