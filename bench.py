#!/usr/bin/env python
"""Benchmark of the B200 SDOT solver on the plain large single instance.

Workload: N = 65,536 sites (256x256 jittered grid, Gaussian-beam masses,
sigma 0.35), 1024x1024 Gaussian-mixture target (K = 16, floor 1e-3), cold
start w = 0, L-BFGS with memory 10 and a strong-Wolfe line search, stopped at
max_i |mu_i - nu_i| / nu_i <= 1e-4.  One step = one complete solve.

Metric: cell-evals/s = N x objective evaluations (every line-search trial
counts) / solve time; the solve time itself is reported as solve_ms.

  value  -- device-resident inputs, CUDA events on the launching stream
  e2e    -- through the public API with host buffers: problem upload, the
            solve, and the weights read back, every step
  roofline -- the fused cell kernel: algorithmic bytes per evaluation
            (8*H*W density + 48*N per-site) / its average launch time
  cpu_baseline -- the CPU oracle (restated reference algorithm) on a bounded
            sample of the same solve, on this machine's host cores

With --gpus N (torchrun) every rank solves its own replica (the solver does
not shard: replicas only), time = max over ranks.
--impl reference times the CPU restatement of the reference's algorithm on
this host (rank 0 only).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "OT solve ms @1e-4 mass err: learned warm-start vs plain L-BFGS; cell-evals/s"
UNIT = "cell-evals/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--tol", type=float, default=1e-4)
    ap.add_argument("--history", type=int, default=10)
    ap.add_argument("--cpu-sample-evals", type=int, default=6,
                    help="oracle evaluations per CPU sample (about 1 s each at the default size)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--cells-per-warp", type=int, default=0, help="1 or 2 (0: the library default)")
    ap.add_argument("--bucket-size", type=int, default=0, help="sites per neighbour bucket (0: the library default)")
    ap.add_argument("--multilevel", action="store_true",
                    help="cold against multilevel warm-started solves (config 2, 4 or 5)")
    ap.add_argument("--instances", type=int, default=0,
                    help="instances of a --multilevel run (0: 1 at config 2, 64 at config 4, 16 at config 5)")
    ap.add_argument("--no-warm-start", action="store_true",
                    help="skip the warm-started arms of the default run")
    ap.add_argument("--warm-steps", type=int, default=0,
                    help="timed solves of each warm-started arm (0: --steps)")
    ap.add_argument("--no-config5", action="store_true",
                    help="skip the combined configuration's arms (16 x 262,144 sites, 2048^2)")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched configuration's sub-object of the default run")
    return ap.parse_args()


def workload(config):
    from caustic_b200 import problems

    p = problems.make(config)
    return p, {"workload": f"sdot_config{config}_cold_lbfgs_wolfe", "n_sites": p.n, "image": list(p.size),
               "target": "gaussian_mixture_floor1e-3", "masses": "beam_sigma0.35" if config in (2, 5) else "uniform",
               "stop": "max_rel_mass_err<=1e-4", "lbfgs_memory": 10, "line_search": "strong_wolfe"}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def committed_figure(key):
    """A per-launch figure of the cell kernels from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "k_cells_config2.md")
    try:
        with open(path) as f:
            for line in f:
                if line.strip().startswith(key + ":"):
                    return float(line.split(":", 1)[1].strip().split()[0])
    except Exception:
        pass
    return None


def committed_traffic():
    """Per-launch DRAM bytes of the cell kernels from the committed ncu summary."""
    return committed_figure("traffic_bytes_per_launch")


class Clocks:
    """nvidia-smi sampling while the timed region runs."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        try:
            with open(self.path) as f:
                for line in f:
                    c = [x.strip() for x in line.split(",")]
                    if len(c) < 9:
                        continue
                    try:
                        sm.append(float(c[1]))
                        mx = float(c[2])
                    except ValueError:
                        continue
                    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
                    for nm, v in zip(names, c[5:9]):
                        if v.lower() == "active":
                            reasons.add(nm)
            os.unlink(self.path)
        except Exception:
            pass
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2], "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def cpu_baseline(p, evals, tol, history):
    """Oracle (CPU restatement) on the first `evals` evaluations of the solve."""
    import numpy as np

    from oracle import oracle as O

    prob = O.Problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
    t = time.perf_counter()
    _, st = O.lbfgs_wolfe(prob, np.zeros(p.n), tol=tol, m=history, max_evals=evals)
    dt = time.perf_counter() - t
    return p.n * st.evaluations / dt, st.evaluations, dt


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import numpy as np  # noqa: F401

    p, cfg = workload(args.config)
    vals = []
    tot_e = 0
    tot_t = 0.0
    for k in range(args.warmup + args.steps):
        v, e, dt = cpu_baseline(p, args.cpu_sample_evals, args.tol, args.history)
        if k >= args.warmup:
            vals.append(v)
            tot_e += e
            tot_t += dt
    value = p.n * tot_e / tot_t
    cores = os.cpu_count()
    sample = (f"first {args.cpu_sample_evals} objective evaluations of the cold-start L-BFGS per step, "
              f"same problem; Qhull regular triangulation (1 thread) + C integration (OpenMP {cores} threads)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * tot_t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64, same generator as the GPU arm)", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "the reference's own solver needs CGAL 5.5/Eigen/Boost, absent here; this is the oracle port"}
    print(json.dumps(line), flush=True)
    return 0


NET_C2 = os.path.join(ROOT, "caustic_b200", "data", "warmstart_c2_64.npz")
NET_C2_LEVEL = 4096    # sites of the level the network predicts (64^2 sites, 256^2 image at config 2);
                       # its prediction is averaged down to the coarsest level (1,024 sites)


def warm_start_arms(args, p, cold_solve_ms, cold_e2e_ms, local):
    """The metric's first half: warm-started solves of the same workload to
    the same tolerance, each through warm.WarmSolver with the plain L-BFGS as
    the judge at the end.  Every step is one whole solve from the host arrays
    (coarsening, uploads, inference and the judge inside the timed region,
    host wall clock with the device synchronised), compared with the cold
    L-BFGS's device solve time (``value``'s solves) and its end-to-end time
    (``e2e``'s solves)."""
    import numpy as np
    import torch

    from caustic_b200.warm import WarmSolver

    arms = {"multilevel": dict(start="multilevel")}
    if os.path.exists(NET_C2):
        from caustic_b200 import warmstart

        net = warmstart.CNet.from_npz(NET_C2, device=local)   # inference through the C ABI
        arms["learned"] = dict(start="learned", net=net, net_level_sites=NET_C2_LEVEL)
    out = {"cold_solve_ms": cold_solve_ms, "cold_e2e_ms": cold_e2e_ms,
           "timing": "host wall clock per whole solve (host arrays in, weights out), device synchronised; "
                     "device_ms sums the solves' CUDA-event times",
           "learned": None if "learned" not in arms else {},
           "learned_note": None if "learned" in arms else f"no trained network at {os.path.relpath(NET_C2, ROOT)}"}
    steps = args.warm_steps or args.steps
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for name, kw in arms.items():
        with WarmSolver(device=local, tol=args.tol, history=args.history, **kw) as ws:
            for _ in range(args.warmup):
                ws.solve(p)
            walls, devs, infer, errs, conv, judge_it, levels = [], [], [], [], [], [], None
            for k in range(steps):
                flush.fill_(k & 255)
                torch.cuda.synchronize()
                w, st = ws.solve(p)
                torch.cuda.synchronize()
                walls.append(st.wall_ms)
                devs.append(st.device_ms)
                infer.append(st.infer_ms)
                errs.append(st.max_rel_err)
                conv.append(st.converged)
                judge_it.append(st.judge.iterations)
                levels = st.levels
        wall = float(np.mean(walls))
        dev = float(np.mean(devs))
        out[name] = {"wall_ms": wall, "device_ms": dev, "infer_ms": float(np.mean(infer)),
                     "speedup_wall_vs_cold_e2e": (cold_e2e_ms / wall) if cold_e2e_ms else None,
                     "speedup_device_vs_cold": cold_solve_ms / dev,
                     "max_rel_err": float(max(errs)), "converged": bool(all(conv)),
                     "judge_iterations_max": int(max(judge_it)), "steps": steps,
                     "levels": [{"n_sites": n, "newton_iterations": x.newton_iterations,
                                 "lbfgs_iterations": x.lbfgs_iterations, "evaluations": x.evaluations,
                                 "cg_iterations": x.cg_iterations, "fallback": x.fallback, "ms": x.ms}
                                for n, x in levels]}
    return out


def batched_arms(args, local, stream):
    """The batched configuration beside the headline: its 64 seeded instances
    (N log-uniform in [1,024, 32,768], 512^2 targets) solved to the same
    tolerance (i) by the plain L-BFGS in one graph launch after the
    autotuner picked the cell kernel's shape (cells per warp {1, 2, 4} x
    sites per bucket {4, 8, 16}), (ii) one after another (the sequential
    pass), and (iii) by the warm-start pipeline instance by instance (host
    arrays in, weights out, host wall clock).  One run of each."""
    import numpy as np
    import torch

    from caustic_b200 import batch
    from caustic_b200.warm import WarmSolver

    probs = batch.instances(64)
    opts = dict(tol=args.tol, history=args.history, max_iter=100000)
    tune = batch.autotune(probs, stream=stream.cuda_stream, tol=args.tol, history=args.history)
    kw = dict(cells_per_warp=tune.cells_per_warp, bucket_size=tune.bucket_size, stream=stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    batch.solve(probs[:8], **kw, **opts)          # warm-up
    flush.fill_(1)
    torch.cuda.synchronize()
    _, st, sec = batch.solve(probs, **kw, **opts)
    flush.fill_(2)
    torch.cuda.synchronize()
    _, sq, sq_sec = batch.solve_sequential(probs, **kw, **opts)
    with WarmSolver(device=local, tol=args.tol, history=args.history) as ws:
        ws.solve(probs[0])                          # warm-up
        flush.fill_(3)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        wst = [ws.solve(p)[1] for p in probs]
        torch.cuda.synchronize()
        warm_sec = time.perf_counter() - t0
    ibig = int(np.argmax([p.n for p in probs]))
    big = probs[ibig]
    return {"instances": 64, "n_range": [min(p.n for p in probs), max(p.n for p in probs)], "image": [512, 512],
            "batched_solves_per_s": 64 / sec, "batched_converged": all(x.converged for x in st),
            "batched_max_rel_err": max(x.max_rel_err for x in st),
            "batched_cell_evals_per_s": sum(p.n * x.evaluations for p, x in zip(probs, st)) / sec,
            "sequential_solves_per_s": 64 / sq_sec, "batched_over_sequential": sq_sec / sec,
            # the slowest instance solved alone bounds any batch of these
            # solves from below (its iterations run one after another)
            "longest_single_solve_s": max(x.ms for x in sq) * 1e-3,
            "batched_over_longest_single": sec / (max(x.ms for x in sq) * 1e-3),
            # the largest instance alone fills the GPU best of all: a batch
            # that evaluates cells faster than it keeps every SM busy
            "largest_alone_cell_evals_per_s": big.n * sq[ibig].evaluations / (sq[ibig].ms * 1e-3),
            "warm_pipeline_solves_per_s": 64 / warm_sec, "warm_over_batched": sec / warm_sec,
            "warm_converged": all(x.converged for x in wst), "warm_max_rel_err": max(x.max_rel_err for x in wst),
            "timing": "batched and sequential: device time of the solves; warm: host wall clock of the 64 pipelines",
            "autotune": {"cells_per_warp": tune.cells_per_warp, "bucket_size": tune.bucket_size,
                         "table": [{"cells_per_warp": c, "bucket_size": b, "cell_evals_per_s": r}
                                   for c, b, r in tune.table]}}


def config5_arms(args, local, workers=8, count=16):
    """The combined configuration at scale: 16 seeded instances of N = 262,144
    sites on 2048^2 targets (beam masses), each solved from the host arrays
    to the same tolerance (i) by the warm pipeline, one instance after
    another, (ii) by WORKERS warm pipelines side by side (warm.WarmPool: one
    stream and host thread each), and (iii) cold: the plain L-BFGS from zero
    on the first instance only (one cold solve takes tens of seconds at this
    size).  Host wall clock with the device synchronised; the cold solve
    adds its device time."""
    from concurrent.futures import ThreadPoolExecutor

    import numpy as np
    import torch

    from caustic_b200 import capi, problems
    from caustic_b200.warm import WarmPool, WarmSolver

    with ThreadPoolExecutor(8) as ex:
        probs = list(ex.map(lambda i: problems.make(5, i), range(count)))
    kw = dict(device=local, tol=args.tol, history=args.history)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    with WarmSolver(**kw) as ws:
        ws.solve(probs[0])                       # warm-up: the handles' buffers
        flush.fill_(1)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        seq = [ws.solve(p)[1] for p in probs]
        torch.cuda.synchronize()
        seq_s = time.perf_counter() - t0
    with WarmPool(workers, **kw) as pool:
        pool.solve_all(probs[:workers])          # warm-up: every pipeline's buffers
        flush.fill_(2)
        torch.cuda.synchronize()
        res, con_s = pool.solve_all(probs)
        torch.cuda.synchronize()
    con = [x[1] for x in res]
    p = probs[0]
    flush.fill_(3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    with capi.Solver(device=local) as s:
        s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
        _, cst = s.solve(np.zeros(p.n), tol=args.tol, history=args.history, max_iter=100000)
    cold_wall = time.perf_counter() - t0
    return {"instances": count, "n_sites": p.n, "image": list(p.size), "masses": "beam_sigma0.35",
            "warm_sequential_ms_per_solve": 1e3 * seq_s / count,
            "warm_concurrent_ms_per_solve": 1e3 * con_s / count, "warm_workers": workers,
            "concurrent_over_sequential": seq_s / con_s,
            "warm_device_ms_per_solve": float(np.mean([x.device_ms for x in seq])),
            "warm_converged": all(x.converged for x in seq + con),
            "warm_max_rel_err": max(x.max_rel_err for x in seq + con),
            "cold_wall_ms": 1e3 * cold_wall, "cold_device_ms": cst.ms, "cold_iterations": cst.iterations,
            "cold_evaluations": cst.evaluations, "cold_converged": bool(cst.converged),
            "cold_max_rel_err": cst.max_rel_err,
            "cold_cell_evals_per_s": p.n * cst.evaluations / (cst.ms * 1e-3),
            "speedup_concurrent_wall_vs_cold": cold_wall / (con_s / count),
            "speedup_sequential_wall_vs_cold": cold_wall / (seq_s / count),
            "timing": "host wall clock, host arrays in and weights out, device synchronised; the cold arm one "
                      "instance (the first)"}


def run_ours(args):
    import numpy as np
    import torch

    from caustic_b200 import capi

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    p, cfg = workload(args.config)
    dev = torch.device("cuda", local)
    # a stream of our own: the legacy default stream cannot be captured, and
    # the solve runs its trial loop as one CUDA graph
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    kw = dict(cells_per_warp=args.cells_per_warp, bucket_size=args.bucket_size)
    solver = capi.Solver(device=local, **kw)
    solver.set_stream(stream.cuda_stream)
    xy_d = torch.from_numpy(p.xy.reshape(-1)).to(dev)
    nu_d = torch.from_numpy(p.nu).to(dev)
    pic_d = torch.from_numpy(p.picture).to(dev)
    solver.set_problem(xy_d, nu_d, pic_d, p.size, p.proj_domain)
    w0 = torch.zeros(p.n, dtype=torch.float64, device=dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    def solve():
        return solver.solve(w0, mode=capi.SOLVE_WOLFE, history=args.history, max_iter=100000, tol=args.tol)

    for _ in range(args.warmup):
        flush.fill_(1)
        w, st = solve()
    torch.cuda.synchronize()
    solver.kernel_stats(reset=True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stats = []
    with Clocks(local) as clk:
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        for k in range(args.steps):
            flush.fill_(k & 255)  # evict L2 between solves
            evs[k][0].record(stream)
            w, st = solve()
            evs[k][1].record(stream)
            stats.append(st)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
    ks = solver.kernel_stats(reset=True)
    step_ms = [a.elapsed_time(b) for a, b in evs]
    tot_ms = sum(step_ms)
    evals = sum(s.evaluations for s in stats)
    conv = all(s.converged for s in stats)
    cell_evals = float(p.n) * evals
    if dist is not None:
        t = torch.tensor([tot_ms], device=dev, dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        tot_ms = float(t.item())
        c = torch.tensor([cell_evals], device=dev, dtype=torch.float64)
        dist.all_reduce(c, op=dist.ReduceOp.SUM)
        cell_evals = float(c.item())
    value = cell_evals / (tot_ms * 1e-3)

    # roofline of the cell kernels (ring construction, certificate and
    # integration, timed together per evaluation): CUDA events around every launch need
    # the host-driven trial loop (graph-captured launches carry no per-launch
    # events), so one more solve of the same workload runs that way, on the
    # same stream, right after the timed region
    prof = capi.Solver(device=local, profile=True, **kw)
    prof.set_stream(stream.cuda_stream)
    prof.set_problem(xy_d, nu_d, pic_d, p.size, p.proj_domain)
    flush.fill_(7)
    prof.solve(w0, mode=capi.SOLVE_WOLFE, history=args.history, max_iter=100000, tol=args.tol, use_graph=-1)
    kp = prof.kernel_stats(reset=True)
    prof.close()
    hbm, peak_kind = peaks()
    H, W = p.size[1], p.size[0]
    alg_bytes = 8.0 * H * W + 48.0 * p.n
    avg_ms = kp["cell_ms"] / max(kp["cell_launches"], 1)
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9 if avg_ms > 0 else None
    traffic = committed_traffic()
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": (achieved / hbm) if achieved else None, "traffic": traffic,
            "kernel": "k_cells_first + k_bucket_walk + k_cells_walk + k_cells_heavy + k_integrate (power-cell rings, the bucket lists, their certificate, the overflowed certificates a block each, their integration; timed together)",
            "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms, "launches": kp["cell_launches"],
            "timing": "CUDA events around each launch, one host-driven solve of the same workload",
            "peak_kind": f"{peak_kind} hbm_gbs (burst copy)"}

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        xy_h = torch.from_numpy(p.xy.reshape(-1)).pin_memory()
        nu_h = torch.from_numpy(p.nu).pin_memory()
        pic_h = torch.from_numpy(p.picture).pin_memory()
        w_h = torch.zeros(p.n, dtype=torch.float64).pin_memory()
        s2 = capi.Solver(device=local, **kw)
        s2.set_stream(stream.cuda_stream)
        # warm the handle once
        s2.set_problem(xy_h.numpy(), nu_h.numpy(), pic_h.numpy(), p.size, p.proj_domain)
        s2.solve(w_h.numpy(), mode=capi.SOLVE_WOLFE, history=args.history, max_iter=100000, tol=args.tol)
        torch.cuda.synchronize()
        e_ev = 0
        t_ms = 0.0
        for k in range(args.steps):
            flush.fill_(k & 255)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            s2.set_problem(xy_h.numpy(), nu_h.numpy(), pic_h.numpy(), p.size, p.proj_domain)
            wout, st2 = s2.solve(w_h.numpy(), mode=capi.SOLVE_WOLFE, history=args.history, max_iter=100000,
                                 tol=args.tol)
            b.record(stream)
            b.synchronize()
            t_ms += a.elapsed_time(b)
            e_ev += st2.evaluations
        s2.close()
        ce = float(p.n) * e_ev
        if dist is not None:
            t = torch.tensor([t_ms], device=dev, dtype=torch.float64)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            t_ms = float(t.item())
            c = torch.tensor([ce], device=dev, dtype=torch.float64)
            dist.all_reduce(c, op=dist.ReduceOp.SUM)
            ce = float(c.item())
        h2d = p.xy.nbytes + p.nu.nbytes + p.picture.nbytes + 8 * p.n
        e2e = {"value": ce / (t_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(8 * p.n), "ms_per_step": t_ms / args.steps}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, e, dt = cpu_baseline(p, args.cpu_sample_evals, args.tol, args.history)
        cpu = {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"first {e} objective evaluations of the same cold-start solve ({dt:.1f} s)"}

    if rank == 0:
        cfg = dict(cfg)
        cfg["parallelism"] = f"replicas{world}"
        cfg["l2"] = "256 MiB buffer written between timed solves"
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": tot_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded PCG64 jittered sites + Gaussian-mixture target)", "config": cfg,
                "solve_ms": tot_ms / args.steps, "evaluations_per_solve": evals / args.steps,
                "iterations_per_solve": sum(s.iterations for s in stats) / args.steps,
                "max_rel_err": max(s.max_rel_err for s in stats), "converged": conv,
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "clocks": clk.summary(),
                "gpu_launches": ks["launches"]}
        # the bound that does hold: warp-instruction issue (4 schedulers per
        # SM, one warp instruction per cycle each, at the sampled SM clock)
        insts = committed_figure("warp_instructions_per_launch")
        ck = line["clocks"]
        mhz = ck.get("sm_mhz") or ck.get("sm_max_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(local).multi_processor_count
        issue_peak = sms * 4 * mhz * 1e6
        if insts and avg_ms > 0:
            ach = insts / (avg_ms * 1e-3)
            line["roofline_issue"] = {"bound": "issue", "achieved": ach, "peak": issue_peak, "unit": "warp-inst/s",
                                      "frac": ach / issue_peak, "insts_per_launch": insts,
                                      "peak_kind": f"{sms} SMs x 4 schedulers x 1 warp-inst/cycle at {mhz:.0f} MHz",
                                      "insts_source": "smsp__inst_executed.sum, committed ncu summary"}
        if world == 1 and not args.no_warm_start:
            line["warm_start"] = warm_start_arms(args, p, tot_ms / args.steps,
                                                 e2e["ms_per_step"] if e2e else None, local)
        if world == 1 and not args.no_batched:
            line["batched_config3"] = batched_arms(args, local, stream)
        if world == 1 and not args.no_config5:
            line["config5"] = config5_arms(args, local)
        print(json.dumps(line), flush=True)
    solver.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_batch(args):
    """The batched configuration: 64 seeded instances of uneven N (1,024 to
    32,768 sites, 512^2 targets) solved from w = 0 to max-rel 1e-4 in one
    graph launch per batch, after the autotuner picked the cell kernel's
    shape; one sequential pass of the same 64 solves is timed beside it."""
    import torch

    from caustic_b200 import batch

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    stream = torch.cuda.Stream(device=dev)
    torch.cuda.set_stream(stream)
    probs = batch.instances(64)
    opts = dict(tol=args.tol, history=args.history, max_iter=100000)
    tune = batch.autotune(probs, stream=stream.cuda_stream, tol=args.tol, history=args.history)
    kw = dict(cells_per_warp=tune.cells_per_warp, bucket_size=tune.bucket_size, stream=stream.cuda_stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        batch.solve(probs, **kw, **opts)
    secs, evals, conv, maxrel = [], 0, True, 0.0
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            _, st, sec = batch.solve(probs, **kw, **opts)
            secs.append(sec)
            evals += sum(p.n * x.evaluations for p, x in zip(probs, st))
            conv = conv and all(x.converged for x in st)
            maxrel = max(maxrel, max(x.max_rel_err for x in st))
    tot = sum(secs)
    _, sq, sq_sec = batch.solve_sequential(probs, **kw, **opts)
    if rank == 0:
        line = {"metric": "batched OT solves @1e-4 mass err (64 uneven instances, one graph launch)", "impl": "ours",
                "value": 64 * args.steps / tot, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * tot / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64",
                "data": "synthetic (seeded PCG64, 64 instances of the batched configuration)",
                "config": {"workload": "sdot_config3_batch64", "n_range": [min(p.n for p in probs), max(p.n for p in probs)],
                           "image": [512, 512], "stop": "max_rel_mass_err<=1e-4", "lbfgs_memory": args.history,
                           "l2": "256 MiB buffer written between timed batches"},
                "cell_evals_per_s": evals / tot, "converged": conv, "max_rel_err": maxrel,
                "sequential": {"solves_per_s": 64 / sq_sec, "seconds": sq_sec,
                               "converged": all(x.converged for x in sq)},
                "batched_over_sequential": (64 * args.steps / tot) / (64 / sq_sec),
                "autotune": {"cells_per_warp": tune.cells_per_warp, "bucket_size": tune.bucket_size,
                             "table": [{"cells_per_warp": c, "bucket_size": b, "cell_evals_per_s": r}
                                       for c, b, r in tune.table]},
                "clocks": clk.summary()}
        print(json.dumps(line), flush=True)
    return 0


def run_warmstart(args):
    """The learned warm start: the network trained on 2,000 solver-made
    pairs (caustic_b200/data/warmstart_c4.npz, made by
    `python -m caustic_b200.warmstart`) starts the solves of held-out seeds
    of the configuration (128^2 jittered sites, 256^2 targets, K in 2..16);
    the same solves from w = 0 run beside them.  Both arms run to max-rel
    1e-4 as batched solves of 64; a step is one chunk of 64 instances."""
    import numpy as np
    import torch

    from caustic_b200 import problems, warmstart

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    path = os.path.join(ROOT, "caustic_b200", "data", "warmstart_c4.npz")
    if not os.path.exists(path):
        print(json.dumps({"impl": "ours", "unavailable": f"no trained network at {os.path.relpath(path, ROOT)}"}))
        return 0
    net = warmstart.WarmStartNet.from_file(path)
    warm = [problems.make(4, 200000 + i) for i in range(8)]
    for _ in range(args.warmup):
        warmstart.compare(net, warm, tol=args.tol, history=args.history)
    probs = [problems.make(4, 100000 + i) for i in range(64 * args.steps)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    res = {}
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            r = warmstart.compare(net, probs[64 * k:64 * (k + 1)], tol=args.tol, history=args.history)
            for key, v in r.items():
                res[key] = res.get(key, 0.0 if not isinstance(v, list) else []) + v
    n = len(probs)
    line = {"metric": "OT solve ms @1e-4 mass err: learned warm-start vs plain L-BFGS", "impl": "ours",
            "value": 1e3 * res["warm_s"] / n, "unit": "ms/solve", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64 solve, bf16 network", "data": "synthetic (seeded held-out instances of the warm-start configuration)",
            "config": {"workload": "sdot_config4_warmstart", "n_sites": probs[0].n, "image": list(probs[0].size),
                       "held_out": n, "train_pairs": 2000, "stop": "max_rel_mass_err<=1e-4",
                       "batched": 64, "l2": "256 MiB buffer written between chunks"},
            "cold_ms_per_solve": 1e3 * res["cold_s"] / n, "warm_ms_per_solve": 1e3 * res["warm_s"] / n,
            "inference_ms_per_solve": 1e3 * res["infer_s"] / n,
            "speedup": res["cold_s"] / res["warm_s"],
            "cold_iterations_mean": float(np.mean(res["cold_iters"])),
            "warm_iterations_mean": float(np.mean(res["warm_iters"])),
            "cold_max_rel_err": float(max(res["cold_err"])), "warm_max_rel_err": float(max(res["warm_err"])),
            "clocks": clk.summary()}
    line["pipelines"] = config4_pipelines(args, probs[:32], path, local)
    print(json.dumps(line), flush=True)
    return 0


def config4_pipelines(args, probs, net_path, local):
    """The same held-out seeds through the warm pipeline (warm.WarmSolver:
    multilevel damped Newton levels and the plain L-BFGS as the judge), one
    instance after another, with and without the network's prediction
    averaged down to the coarsest level as its start, and through the plain
    L-BFGS from zero one after another (its device time).  Host wall clock
    per whole solve, host arrays in and weights out."""
    import numpy as np
    import torch

    from caustic_b200 import capi, warmstart
    from caustic_b200.warm import WarmSolver

    out = {"instances": len(probs), "timing": "warm arms: host wall clock per solve; cold: device time per solve"}
    cold, it = [], []
    with capi.Solver(device=local) as s:
        for p in probs:
            s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
            _, st = s.solve(np.zeros(p.n), tol=args.tol, history=args.history, max_iter=100000)
            cold.append(st.ms)
            it.append(st.iterations)
    out["cold_ms_per_solve"] = float(np.mean(cold))
    out["cold_iterations_mean"] = float(np.mean(it))
    net = warmstart.CNet.from_npz(net_path, device=local)   # inference through the C ABI
    arms = {"multilevel": dict(start="multilevel"),
            "learned": dict(start="learned", net=net, net_level_sites=probs[0].n, learned_at="coarsest")}
    for name, kw in arms.items():
        with WarmSolver(device=local, tol=args.tol, history=args.history, **kw) as ws:
            ws.solve(probs[0])
            torch.cuda.synchronize()
            sts = [ws.solve(p)[1] for p in probs]
        out[name] = {"wall_ms_per_solve": float(np.mean([x.wall_ms for x in sts])),
                     "device_ms_per_solve": float(np.mean([x.device_ms for x in sts])),
                     "converged": all(x.converged for x in sts), "max_rel_err": max(x.max_rel_err for x in sts)}
    out["learned_over_multilevel"] = out["multilevel"]["wall_ms_per_solve"] / out["learned"]["wall_ms_per_solve"]
    out["learned_over_cold"] = out["cold_ms_per_solve"] / out["learned"]["wall_ms_per_solve"]
    return out


def run_multilevel(args):
    """Cold solves against multilevel warm-started solves
    (caustic_b200/multilevel.py) of the same seeded instances to max-rel
    1e-4, each arm as one batched solve per level.  A step solves every
    instance once in each arm; the reported value is the multilevel arm's
    device time per solve (all levels).  Wall times add the host work
    (problem uploads, coarsening, interpolation)."""
    import time

    import numpy as np
    import torch

    from caustic_b200 import capi, multilevel, problems

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    cfg = args.config if args.config in (2, 4, 5) else 2
    count = args.instances or {2: 1, 4: 64, 5: 16}[cfg]
    # config 4: the learned warm start's held-out seeds
    first = 100000 if cfg == 4 else 0
    probs = [problems.make(cfg, first + i) for i in range(count)]

    def cold_arm(ps):
        t0 = time.perf_counter()
        sols = []
        for p in ps:
            s = capi.Solver()
            s.set_problem(p.xy, p.nu, p.picture, p.size, p.proj_domain)
            sols.append(s)
        _, st = capi.solve_batch(sols, [np.zeros(p.n) for p in ps], tol=args.tol, history=args.history,
                                 max_iter=100000)
        for s in sols:
            s.close()
        return st, st[0].ms, time.perf_counter() - t0

    def ml_arm(ps):
        t0 = time.perf_counter()
        _, levels = multilevel.solve(ps, tol=args.tol, history=args.history)
        return levels, sum(lv.ms for lv in levels), time.perf_counter() - t0

    small = [problems.make(cfg, 900 + i, g=64, res=256) for i in range(2)]
    for _ in range(args.warmup):
        cold_arm(small)
        ml_arm(small)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    tot = {"cold_ms": 0.0, "ml_ms": 0.0, "cold_wall": 0.0, "ml_wall": 0.0}
    cold_st, ml_lv = [], None
    with Clocks(local) as clk:
        for k in range(args.steps):
            flush.fill_(k & 255)
            torch.cuda.synchronize()
            st, ms, wall = cold_arm(probs)
            tot["cold_ms"] += ms
            tot["cold_wall"] += wall
            cold_st += st
            flush.fill_((k + 1) & 255)
            torch.cuda.synchronize()
            lv, ms, wall = ml_arm(probs)
            tot["ml_ms"] += ms
            tot["ml_wall"] += wall
            ml_lv = lv
    n = count * args.steps
    line = {"metric": "OT solve ms @1e-4 mass err: multilevel warm start vs plain L-BFGS", "impl": "ours",
            "value": tot["ml_ms"] / n, "unit": "ms/solve", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded PCG64 jittered sites + Gaussian-mixture targets)",
            "config": {"workload": f"sdot_config{cfg}_multilevel_vs_cold", "n_sites": probs[0].n,
                       "image": list(probs[0].size), "instances": count, "batched": count > 1,
                       "stop": "max_rel_mass_err<=1e-4", "coarse_stop": "max_rel_mass_err<=1e-3",
                       "l2": "256 MiB buffer written before each arm"},
            "cold_ms_per_solve": tot["cold_ms"] / n, "multilevel_ms_per_solve": tot["ml_ms"] / n,
            "speedup": tot["cold_ms"] / tot["ml_ms"],
            "cold_wall_ms_per_solve": 1e3 * tot["cold_wall"] / n,
            "multilevel_wall_ms_per_solve": 1e3 * tot["ml_wall"] / n,
            "wall_speedup": tot["cold_wall"] / tot["ml_wall"],
            "cold_iterations_mean": float(np.mean([s.iterations for s in cold_st])),
            "cold_max_rel_err": float(max(s.max_rel_err for s in cold_st)),
            "cold_converged": all(s.converged and s.max_rel_err <= args.tol for s in cold_st),
            "multilevel_converged": all(s.converged and s.max_rel_err <= args.tol for s in ml_lv[-1].stats),
            "levels": [{"n_sites": lv.n, "image": list(lv.image), "tol": lv.tol, "ms": lv.ms,
                        "iterations_mean": float(np.mean([s.iterations for s in lv.stats])),
                        "max_rel_err": float(max(s.max_rel_err for s in lv.stats))} for lv in ml_lv],
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.multilevel:
        return run_multilevel(args)
    if args.config == 3:
        return run_batch(args)
    if args.config == 4:
        return run_warmstart(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
