#!/usr/bin/env python
"""Benchmark of the SPHERA per-step particle path on B200.

Workload: the 3D dam break (tank 1.6 x 0.6 x 0.6 m, block 0.6 x 0.3 x 0.6 m,
dx = 0.005 m, 864,000 particles, seeded +-0.01 dx jitter, SA-SPH fixe
walls), synthetic state generated in-repo.  A step is one whole leapfrog
step of time_step_loop.f90 (momentum + leapfrog, cell sort, SA-SPH boundary
data, continuity + EoS, time step), replayed from a CUDA graph.

  value       particle-steps/s over all ranks, state resident on the device
              (device time, CUDA events on the library's stream, max over
              ranks): the median of repeated windows of --steps graph
              replays, repeated until at least --min-seconds are timed
  e2e         the same metric through the C ABI with the state in pinned host
              memory: every step uploads pg(:), advances and downloads it
              (both forms; the top-level e2e is the headline form's)
  roofline    dominant kernel (momentum pass) against the larger of its two
              roofs: the measured HBM copy bandwidth and the FMA rate of its
              arithmetic (FP32 for the FP32c form, FP64 for the FP64 form),
              measured in the run with its clocks recorded
  cpu_baseline  the oracle (FP64 OpenMP restatement) on the host cores

`--impl reference` times the oracle alone (the reference is Fortran and
cannot be built here) on the same workload.  `--gpus N` runs N ranks, one
per GPU: under torchrun it reads the ranks from the environment, otherwise
it starts them itself through torch.distributed.run.  Each rank advances
an independent replica (no data-path collective: weak scaling).
`--dry-run` exercises the rank plumbing without a GPU.
"""
import argparse
import json
import math
import os
import socket
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "particle-steps/s FP32c vs FP64 at ≤1e-3 rel L2; ensemble p50/p99 time-to-result"
UNIT = "particle-steps/s"
# launches of one FP32c step graph (3D, sph_api.cu step_sequence): momentum
# pair sums and finish, 8 sort, 3 boundary, lists, continuity pair sums and
# finish, finalize; the FP64 graph has one momentum and one continuity kernel
KERNELS_PER_STEP = 17
KERNELS_PER_STEP_FP64 = 15
# algorithmic bytes of the fused FP32c momentum pass (k_momentum_f32 pair
# sums + k_momentum_f32_finish): per particle, each record read once -- X 32,
# V 32, RP 16, XF 16, VF 16, RM 8 (the neighbours' XF/VF/RM are these same
# records), L 1, I 4, ncount 4, bdt_count 4 -- and written once -- X2 32,
# V2 32, P2 8, I2 4, L2 1 -- plus 4 B per neighbour-list entry and 168 B per
# boundary entry.  The nine pair sums that a particle with close faces hands
# from the pair launch to the finishing one (72 B each way) are the split's
# own traffic, not the algorithm's, and are left out.  The FP64 pass (one
# launch) reads X, V, RP, L, I, ncount, bdt_count and the neighbours' X, V,
# RP and writes the same record: 218 B per particle.
MOM_BYTES_PER_PARTICLE = 210
MOM_BYTES_PER_PARTICLE_FP64 = 218
LIST_ENTRY_BYTES = 4
BDT_ENTRY_BYTES = 168
# Operations per accepted non-self pair: 107 in the momentum pass, 34 in the
# continuity pass (sqrt and divide counted as one); 9 per candidate test of
# the neighbour-list pass
FLOP_CAND, FLOP_MOM_PAIR, FLOP_CONT_PAIR = 9, 107, 34


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _spawn_ranks(nranks):
    """`bench.py --gpus N` started without torchrun: run the same command
    line as N ranks of torch.distributed.run (one per GPU) and return its
    exit status."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={nranks}",
           "--master-addr=127.0.0.1", f"--master-port={_free_port()}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if ws > 1:
        import datetime
        import torch.distributed as dist
        # gloo carries only scalars here (timings, work counts); a rank that
        # never arrives ends the others' next collective with an error
        dist.init_process_group("gloo", init_method="env://", timeout=datetime.timedelta(seconds=600))
    return ws, rank, local


def _barrier(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()


def _max_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _sum_over_ranks(ws, v):
    if ws == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())


def _finish_dist(ws):
    if ws > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        # nvidia-smi's first query can stall the driver for seconds on a box
        # without persistence mode: wait for its first sample before timing
        t0 = time.time()
        while self.p is not None and time.time() - t0 < 10.0:
            if os.path.getsize(self.f.name) > 0:
                break
            time.sleep(0.05)

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [t.strip() for t in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None,
                "reasons": sorted(reasons), "samples": len(rows)}


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            pk = json.load(f)
        return float(pk["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _traffic(workload):
    """DRAM bytes per momentum launch from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            t = json.load(f)
        return t.get(workload)
    except (OSError, ValueError):
        return None


def cpu_oracle_rate(case, steps, threads):
    from oracle.pyoracle import Oracle
    o = Oracle(case, nthreads=threads)
    o.prepare()
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    n = o.n
    o.close()
    return n * steps / dt, dt


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    from sphera_b200 import cases
    threads = os.cpu_count() or 1
    case = cases.dam_break_3d()
    steps = max(1, min(args.steps, 20))
    from oracle.pyoracle import Oracle
    o = Oracle(case, nthreads=threads)
    o.prepare()
    o.step(max(0, min(args.warmup, 3)))
    t0 = time.perf_counter()
    o.step(steps)
    el = time.perf_counter() - t0
    v = case.n * steps / el
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
        "steps": steps, "warmup": min(args.warmup, 3), "ms_per_step": el / steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded 3D dam break generated in-repo)",
        "config": {"workload": "dam_break_3d: tank 1.6x0.6x0.6 m, block 0.6x0.3x0.6 m, dx 0.005 m, "
                               "864000 particles, SA-SPH walls, FP64", "particles": case.n},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{steps} leapfrog steps of the full 864000-particle state after the IC "
                                   f"(timed steps capped at 20 so the run stays within minutes)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference is Fortran 90 and no Fortran compiler exists on these machines; "
                "timed: the oracle's C++ OpenMP restatement of the same subroutines",
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ensemble(args, ws, rank, emit=True):
    """256 independent 2D dam breaks (column width U[0.5, 2.0] m, height
    U[0.5, 2.5] m, dx 0.01 m) advanced together in the same launches and
    CUDA graph, FP32-compensated form, each to t_end; all requests are
    present at t = 0.  Reports the aggregate particle-steps/s and the
    p50/p99 time-to-result over the simulations."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from sphera_b200 import Batch, abi, cases
    cs = cases.ensemble_2d(n_sims=args.n_sims, dx=0.01, seed=0xC3 + rank, precision=abi.SPH_PREC_FP32C)
    b = Batch(cs)
    b.upload()
    if getattr(args, "shape", None) and len(args.shape.split(",")) == 7:
        # a fixed launch configuration instead of the autotuner's choice
        grids = dict(zip(__import__("sphera_b200")._SHAPE_KEYS, (int(t) for t in args.shape.split(","))))
        b.set_launch_shape(grids)
    else:
        grids = b.autotune(reps=2)
    for i in range(len(cs)):
        b.set_end_time(i, args.t_end)
    n_total = sum(c.n for c in cs)
    chunk = 25
    done_at = np.full(len(cs), np.nan)
    _barrier(ws)
    t0 = time.perf_counter()
    while True:
        b.step_async(chunk)
        fr, tt, st, _ = b.status()
        now = time.perf_counter() - t0
        newly = fr & np.isnan(done_at)
        done_at[newly] = now
        if fr.all():
            break
    elapsed = time.perf_counter() - t0
    fr, tt, st, _ = b.status()
    psteps = float(sum(c.n * int(k) for c, k in zip(cs, st)))
    elapsed = _max_over_ranks(ws, elapsed)
    line = {
        "metric": METRIC, "workload": "ensemble_2d", "value": ws * psteps / elapsed, "unit": UNIT,
        "n_gpus": ws, "higher_is_better": True, "scaling": "weak", "dtype": "fp32c",
        "config": {"workload": f"{len(cs)} 2D dam breaks, width U[0.5,2.0] m, height U[0.5,2.5] m, dx 0.01 m, "
                               f"to t = {args.t_end} s, one batch per GPU",
                   "particles": n_total, "min_particles": min(c.n for c in cs),
                   "max_particles": max(c.n for c in cs), "autotuned_grids": grids},
        "time_to_result_s": {"p50": float(np.percentile(done_at, 50)), "p99": float(np.percentile(done_at, 99)),
                             "max": float(np.max(done_at)), "poll_steps": chunk},
        "steps": {"min": int(st.min()), "max": int(st.max())},
        "elapsed_s": elapsed,
    }
    b.close()
    if not emit:
        return line
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def run_serving(args, ws, rank, emit=True):
    """A seeded Poisson stream (mean 20 requests/s) of 3D dam-break and
    sloshing-tank requests (dx log-uniform in [0.005, 0.0125] m, 55k-1M
    particles, FP32-compensated form, each run to t = 0.3 s) served in real
    time: admission by HBM budget, grouped batches on their own streams,
    state resident on the device, each result downloaded when its request
    finishes.  Reports p50/p99 time-to-result (arrival to result on the
    host) and the aggregate particle-steps/s over the run's wall time."""
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    from sphera_b200 import abi, cases
    from sphera_b200.serve import Server, summarize
    reqs = cases.serving_requests(n_requests=args.requests, rate=20.0, seed=0xC4 + rank, t_end=args.t_end,
                                  precision=abi.SPH_PREC_FP32C)
    budget = int(args.hbm_budget_gib * (1 << 30))
    srv = Server(budget, chunk=32)
    _barrier(ws)
    res = srv.run(reqs)
    summ = summarize(res, srv.wall)
    wall = _max_over_ranks(ws, srv.wall)
    total_work = _sum_over_ranks(ws, summ["particle_steps"])
    d2h = sum(r.n * (3 + 3 + 1 + 1 + 1) * 8 for r in res.values() if not r.rejected)
    line = {
        "metric": METRIC, "workload": "serving", "value": total_work / wall, "unit": UNIT,
        "n_gpus": ws, "higher_is_better": True, "scaling": "weak", "dtype": "fp32c",
        "config": {"workload": f"{len(reqs)} requests, Poisson 20/s, 3D dam break and sloshing tank "
                               "(1.0x0.5x0.5 m half filled, A 0.02 m, T U[0.8,1.6] s), dx log-uniform "
                               f"[0.005,0.0125] m, each to t = {args.t_end} s, FP32c",
                   "hbm_budget_bytes": budget, "particles": [r.case.n for r in reqs],
                   "kinds": [r.case.name for r in reqs]},
        "time_to_result_s": {"p50": summ["p50_s"], "p99": summ["p99_s"],
                             "mean_queue": summ["mean_queue_s"]},
        "completed": summ["completed"], "rejected": summ["rejected"],
        "peak_resident_bytes": srv.peak_used, "groups": srv.groups_formed,
        "max_concurrent_requests": srv.max_concurrent, "result_d2h_bytes": d2h,
        "elapsed_s": wall,
    }
    if not emit:
        return line
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


def _quick_rate(case, steps=5, min_seconds=1.0):
    """particle-steps/s of graph replays of `case` after the autotuner,
    timed with CUDA events on the library's stream (median of windows of
    `steps` replays, repeated to at least min_seconds), and its phase times."""
    import torch
    from sphera_b200 import Simulation
    sim = Simulation(case)
    sim.upload(case.state)
    tuned = sim.autotune(reps=2)
    sim.step(3)
    stream = torch.cuda.ExternalStream(sim.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    wins = []
    while not wins or sum(wins) < min_seconds * 1e3:
        sim.sync()
        e0.record(stream)
        sim.step_async(steps)
        e1.record(stream)
        e1.synchronize()
        sim.sync()
        wins.append(e0.elapsed_time(e1))
    ms = statistics.median(wins) / steps
    sim.counters(reset=True)
    ph = sim.profile_phases(3)
    cnt = sim.counters()
    sim.close()
    return {"value": case.n / (ms * 1e-3), "ms_per_step": ms, "windows": len(wins), "autotuned": tuned,
            "phases_ms_per_step": {k: v / 3 for k, v in ph.items()},
            "pairs_per_particle": cnt["pairs"] / 3 / case.n, "candidates_per_particle": cnt["candidates"] / 3 / case.n}


def run_extras(ws, rank):
    """The other workloads of the metric, one GPU: the neighbour-search and
    pair-loop microbenchmark (16M-particle random box, one whole step, both
    forms), the 256-simulation 2D ensemble to 0.5 s and the serving stream
    (8 Poisson requests to 0.3 s)."""
    import types
    from sphera_b200 import abi, cases
    out = {}
    rb = {}
    for name, prec in (("fp32c", abi.SPH_PREC_FP32C), ("fp64", abi.SPH_PREC_FP64)):
        rb[name] = _quick_rate(cases.random_box(n=16_000_000, precision=prec))
    rb["workload"] = ("random_box: 16000000 particles uniform in a 2.52 m cube (mean spacing 0.01 m), "
                      "rho = 1000 (1 + N(0, 1e-3)), v ~ N(0, 0.1) m/s, no walls; whole steps replayed from the graph")
    rb["speedup_fp32c_vs_fp64"] = rb["fp32c"]["value"] / rb["fp64"]["value"]
    out["random_box_16m"] = rb
    ens = types.SimpleNamespace(n_sims=256, t_end=0.5)
    out["ensemble_256"] = run_ensemble(ens, ws, rank, emit=False)
    srv = types.SimpleNamespace(requests=8, t_end=0.3, hbm_budget_gib=4.0)
    out["serving"] = run_serving(srv, ws, rank, emit=False)
    return out


def _fp_summary(r, n, fp_peak, flop_pair):
    if r is None:
        return None
    c, nprof = r["cnt"], r["nprof"]
    mom_ms = r["phases"]["momentum"]
    flops = (c["pairs"] - n * nprof) * flop_pair / nprof
    return {"value": r["value"], "ms_per_step": r["ms_step"], "ms_per_step_spread": r["spread"],
            "windows": r["windows"], "phases_ms_per_step": r["phases"], "clocks": r["clocks"],
            "momentum_tflops": flops / (mom_ms * 1e-3) / 1e12, "fma_peak_tflops": fp_peak,
            "e2e": r["e2e"], "autotuned_grids": r["grids"]}


def _measure_peak(fp32, gpu_id):
    """Dense FMA rate of the device (FP32 or FP64), the best of repeated
    probes over about half a second, with the clocks seen meanwhile."""
    from sphera_b200 import measure_fp32_peak, measure_fp64_peak
    f = measure_fp32_peak if fp32 else measure_fp64_peak
    f()
    sampler = ClockSampler(gpu_id)
    best, t0 = 0.0, time.perf_counter()
    while time.perf_counter() - t0 < 0.6:
        best = max(best, f())
    return best, sampler.stop()


def run_dry(args, ws, rank):
    """The rank plumbing of a multi-GPU run without a GPU: each rank reports
    one unit of work and its rank; rank 0 prints the line the real run
    would print, with n_gpus taken from the ranks that reported."""
    ranks = _sum_over_ranks(ws, 1.0)
    ids = _sum_over_ranks(ws, float(rank))
    wall = _max_over_ranks(ws, 1.0 + rank)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "dry_run": True, "n_gpus": ws, "ranks_reporting": int(ranks),
                          "rank_id_sum": int(ids), "max_over_ranks": wall, "unit": UNIT,
                          "scaling": "weak"}), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--min-seconds", type=float, default=2.0,
                    help="repeat the timed window of --steps replays until this much device time is timed")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=30)
    ap.add_argument("--cpu-steps", type=int, default=3)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the random-box, ensemble and serving workloads of the default run")
    ap.add_argument("--dry-run", action="store_true", help="rank plumbing only, no GPU work")
    ap.add_argument("--workload", default="dam_break_3d", choices=["dam_break_3d", "random_box", "ensemble", "serving"])
    ap.add_argument("--n", type=int, default=16_000_000, help="particles of the random-box workload")
    ap.add_argument("--n-sims", type=int, default=256)
    ap.add_argument("--t-end", type=float, default=None)
    ap.add_argument("--requests", type=int, default=8)
    ap.add_argument("--hbm-budget-gib", type=float, default=4.0)
    ap.add_argument("--dx", type=float, default=0.005,
                    help="lattice spacing of the 3D dam break (0.005: the 864000-particle workload)")
    ap.add_argument("--forms", default="both", choices=["both", "fp32c", "fp64"])
    ap.add_argument("--autotune", type=int, default=1, help="size the persistent grids on the live state first")
    ap.add_argument("--shape", default=None,
                    help="force the FP32c momentum,continuity pair-loop shapes, e.g. 1,1 (0 lean, 1 batched "
                         "loads, 2 batched with paired FP32 arithmetic), or all seven values sph_autotune chooses")
    ap.add_argument("--teta", type=float, default=0.0,
                    help="partial smoothing coefficient TetaP = TetaV of the dam-break workload (0: off)")
    ap.add_argument("--c1", action="store_true",
                    help="dam break with the 1st-order consistency renormalisation (C1_BE and C1_divu, "
                         "invB_det_thresh 1e-3), in the forms --forms names")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.t_end is None:
        args.t_end = 0.3 if args.workload == "serving" else 0.5
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return _spawn_ranks(args.gpus)
    ws, rank, local = _dist()
    if ws != args.gpus:
        sys.stderr.write(f"bench.py: --gpus {args.gpus} but {ws} ranks were started\n")
        _finish_dist(ws)
        return 2
    if args.dry_run:
        rc = run_dry(args, ws, rank)
    elif args.impl == "reference":
        rc = run_reference(args, ws, rank)
    elif args.workload == "ensemble":
        rc = run_ensemble(args, ws, rank)
    elif args.workload == "serving":
        rc = run_serving(args, ws, rank)
    else:
        rc = run_step_bench(args, ws, rank, local)
    _finish_dist(ws)
    return rc


def run_step_bench(args, ws, rank, local):
    import ctypes as C

    import torch
    torch.cuda.set_device(local)
    from sphera_b200 import Simulation, abi, cases

    try:
        gpu_id = "GPU-" + str(torch.cuda.get_device_properties(local).uuid)
    except Exception:
        gpu_id = str(local)
    fp64_peak, fp64_peak_clocks = _measure_peak(False, gpu_id)
    fp32_peak, fp32_peak_clocks = _measure_peak(True, gpu_id)

    def make_case(precision, n=None):
        if args.workload == "random_box":
            return cases.random_box(n=n or args.n, precision=precision)
        c = cases.dam_break_3d(dx=args.dx, precision=precision)
        c.params.teta_p = args.teta
        c.params.teta_v = args.teta
        if args.c1:
            # the C1 settings of the reference's own tutorials with C1_BE
            # (water shipping, WSI WAVESAX: invB_det_thresh = 0.614); its input
            # template warns that C1_BE is unstable when the threshold is too
            # small, and at 1e-3 this dam break blows up within 0.02 s (dt
            # falls below 1e-10), in the oracle as on the device
            c.params.c1_be = 1
            c.params.c1_divu = 1
            c.params.invb_det_thresh = 0.614
        return c

    def timed_window(sim, stream, e0, e1):
        _barrier(ws)
        torch.cuda.synchronize()
        sim.sync()
        e0.record(stream)
        sim.step_async(args.steps)
        e1.record(stream)
        e1.synchronize()
        sim.sync()
        torch.cuda.synchronize()
        _barrier(ws)
        return _max_over_ranks(ws, e0.elapsed_time(e1))

    def e2e_leg(sim, case, stream, e0, e1):
        """Every step through the C ABI from pinned host memory: sph_upload
        (the IC part included) and sph_step_download(1).  The state is the
        one the timed windows left: particles that left the domain during
        them are gone, as in the reference, so its count may be below the
        case's."""
        st0 = sim.download()
        n = st0.n
        pin = {k: torch.empty(sh, dtype=torch.float64, pin_memory=True)
               for k, sh in (("x", (n, 3)), ("v", (n, 3)), ("rho", (n,)), ("p", (n,)), ("m", (n,)))}
        for k in pin:
            pin[k].numpy()[...] = getattr(st0, k)
        hs = abi.SphState()
        hs.n = n
        for k in pin:
            setattr(hs, k, C.cast(pin[k].data_ptr(), C.POINTER(C.c_double)))
        lib = __import__("sphera_b200").lib()
        _barrier(ws)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(stream)
        for _ in range(args.e2e_steps):
            hs.n = n
            if lib.sph_upload(sim._h, C.byref(hs)) != 0:
                raise RuntimeError("sph_upload failed")
            if lib.sph_step_download(sim._h, 1, C.byref(hs)) != 0:
                raise RuntimeError("sph_step_download failed")
        e1.record(stream)
        e1.synchronize()
        wall = time.perf_counter() - t0
        ms = _max_over_ranks(ws, max(e0.elapsed_time(e1), wall * 1e3))
        state_bytes = n * (3 + 3 + 1 + 1 + 1) * 8
        return {"value": ws * n * args.e2e_steps / (ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": state_bytes,
                "d2h_bytes_per_step": state_bytes, "steps": args.e2e_steps,
                "path": "sph_upload + sph_step_download(1) per step, pinned host buffers"}

    def run_form(precision, keep):
        case = make_case(precision)
        n = case.n
        sim = Simulation(case)
        sim.upload(case.state)
        grids = sim.autotune(reps=3) if args.autotune else None
        if args.shape is not None:
            # a fixed launch configuration (profiling the same kernels
            # without the autotuner's sweeps): "m,c" sets the pair-loop
            # shapes on the default grids; seven values set everything
            # sph_autotune chooses (lists, momentum, continuity, boundary,
            # integrals grids, momentum and continuity shapes)
            v = [int(t) for t in args.shape.split(",")]
            if len(v) == 7:
                grids = dict(zip(__import__("sphera_b200")._SHAPE_KEYS, v))
            elif len(v) == 2:
                grids = dict(grids or {}, momentum_shape=v[0], continuity_shape=v[1])
            else:
                raise SystemExit("--shape takes m,c or the seven values of sph_autotune")
            sim.set_launch_shape(grids)
        sim.step(args.warmup)
        stream = torch.cuda.ExternalStream(sim.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        sampler = ClockSampler(gpu_id)
        wins = [timed_window(sim, stream, e0, e1)]
        # the same window count on every rank: it follows from the first
        # window's time, which is already the max over ranks
        nwin = max(1, math.ceil(args.min_seconds * 1e3 / wins[0]))
        for _ in range(nwin - 1):
            wins.append(timed_window(sim, stream, e0, e1))
        clocks = sampler.stop()
        ms = statistics.median(wins)
        # particles that leave the domain are removed, as in the reference:
        # the count after the windows makes the rate a lower bound
        n = sim.download().n
        value = ws * n * args.steps / (ms * 1e-3)
        # phase times and counters of the same workload (un-graphed steps)
        sim.counters(reset=True)
        nprof = 10
        phases = sim.profile_phases(nprof)
        cnt = sim.counters(reset=True)
        diag = sim.diagnostics()
        e2e = e2e_leg(sim, case, stream, e0, e1)
        r = dict(case=case, n=n, value=value, ms=ms, ms_step=ms / args.steps,
                 spread=[min(wins) / args.steps, max(wins) / args.steps], windows=len(wins),
                 clocks=clocks, grids=grids, phases={k: v / nprof for k, v in phases.items()},
                 nprof=nprof, cnt=cnt, diag=diag, e2e=e2e)
        if keep:
            r["sim"] = sim
        else:
            sim.close()
        return r

    r64 = r32 = None
    if args.forms in ("both", "fp64"):
        r64 = run_form(abi.SPH_PREC_FP64, keep=args.forms == "fp64")
    if args.forms in ("both", "fp32c"):
        r32 = run_form(abi.SPH_PREC_FP32C, keep=True)
    fp32c = r32 is not None
    head = r32 if fp32c else r64
    case, n, sim = head["case"], head["n"], head["sim"]
    cnt, diag, nprof = head["cnt"], head["diag"], head["nprof"]
    mom_ms = head["phases"]["momentum"]
    list_entries = cnt["pairs"] / nprof - n          # accepted pairs less the particle itself
    per_particle = MOM_BYTES_PER_PARTICLE if fp32c else MOM_BYTES_PER_PARTICLE_FP64
    alg_bytes = n * per_particle + list_entries * LIST_ENTRY_BYTES + diag.bdt_entries * BDT_ENTRY_BYTES
    hbm_peak, peak_kind = _peaks()
    achieved_gbs = alg_bytes / (mom_ms * 1e-3) / 1e9
    mom_flops = (cnt["pairs"] - n * nprof) * FLOP_MOM_PAIR / nprof
    mom_tflops = mom_flops / (mom_ms * 1e-3) / 1e12
    fp_peak = fp32_peak if fp32c else fp64_peak
    fp_clocks = fp32_peak_clocks if fp32c else fp64_peak_clocks
    if args.workload == "random_box":
        workload = f"random_box_{n}"
        desc = (f"random_box: {n} particles uniform in a cube at mean spacing 0.01 m, rho = 1000 (1 + N(0, 1e-3)), "
                f"v ~ N(0, 0.1) m/s, h = 0.013 m, no walls; one whole step (sort, lists, both pair passes)")
    else:
        workload = "dam_break_3d" if args.dx == 0.005 else f"dam_break_3d_dx{args.dx:g}"
        desc = (f"dam_break_3d: tank 1.6x0.6x0.6 m, block 0.6x0.3x0.6 m, dx {args.dx:g} m, "
                f"{n} particles per GPU, SA-SPH walls"
                + (f", partial smoothing TetaP = TetaV = {args.teta:g}" if args.teta > 0 else "")
                + (", C1 renormalisation (C1_BE, C1_divu)" if args.c1 else ""))
    traffic = _traffic(workload) if fp32c else None
    roof_hbm = {"achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s", "frac": achieved_gbs / hbm_peak,
                "peak_kind": f"{peak_kind} HBM copy bandwidth", "algorithmic_bytes": alg_bytes}
    roof_fp = {"achieved": mom_tflops, "peak": fp_peak, "unit": "TFLOP/s", "frac": mom_tflops / fp_peak,
               "peak_kind": ("measured FP32" if fp32c else "measured FP64") + " FMA rate (in-run probe)",
               "peak_clocks": fp_clocks, "flops_per_pair": FLOP_MOM_PAIR}
    fp_bound = roof_fp["frac"] > roof_hbm["frac"]
    main_roof = roof_fp if fp_bound else roof_hbm
    roofline = {"bound": ("fp32" if fp32c else "fp64") if fp_bound else "hbm",
                "achieved": main_roof["achieved"], "peak": main_roof["peak"], "unit": main_roof["unit"],
                "frac": main_roof["frac"], "traffic": traffic,
                "kernel": ("k_momentum_f32<3> + k_momentum_f32_finish<3,true> (momentum pair sums; wall terms, "
                           "leapfrog)" if fp32c else "k_momentum<3,true> (FP64 momentum, wall terms, leapfrog)"),
                "hbm": roof_hbm, "fp": roof_fp}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        threads = os.cpu_count() or 1
        if args.workload == "random_box":
            # the oracle keeps the reference's lists (17 kB per particle):
            # time it on a 250,000-particle box of the same density
            cc = make_case(abi.SPH_PREC_FP64, n=250_000)
            rate, el = cpu_oracle_rate(cc, args.cpu_steps, threads)
            sample = (f"{args.cpu_steps} leapfrog steps of a 250000-particle random box of the same density "
                      f"after its IC ({el:.1f} s), FP64 oracle, OpenMP on all host threads")
        else:
            rate, el = cpu_oracle_rate(case, args.cpu_steps, threads)
            sample = (f"{args.cpu_steps} leapfrog steps of the full {n}-particle 3D dam break after "
                      f"its IC ({el:.1f} s), FP64 oracle, OpenMP on all host threads")
        cpu = {"value": rate, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample}

    e2e = dict(head["e2e"])
    e2e["path"] += ", " + ("fp32c" if fp32c else "fp64") + " form"
    line = {
        "metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": head["ms_step"], "ms_per_step_spread": head["spread"],
        "timed_windows": head["windows"], "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None,
        "dtype": ("fp32c (f32 pair sums, compensated; f64 positions/integration/boundary terms)"
                  if fp32c else "f64"),
        "data": f"synthetic (seeded {args.workload} generated in-repo)",
        "config": {"workload": desc,
                   "particles_per_gpu": n, "form": "fp32c" if fp32c else "fp64",
                   "autotuned_grids": head["grids"],
                   "l2": "state and scratch (~250 MB per step) exceed the 126 MB L2; no flush",
                   "timing": f"median of {head['windows']} windows of {args.steps} graph replays "
                             f"(at least {args.min_seconds:g} s of device time), each bracketed by a barrier "
                             f"and synchronisation, max over ranks",
                   "parallelism": f"replicas x{ws} (independent simulations, no collective)"},
        "fp64": _fp_summary(r64, n, fp64_peak, FLOP_MOM_PAIR),
        "fp32c": _fp_summary(r32, n, fp32_peak, FLOP_MOM_PAIR),
        "speedup_fp32c_vs_fp64": r32["value"] / r64["value"] if (r32 and r64) else None,
        "e2e": e2e,
        "roofline": roofline,
        "phases_ms_per_step": head["phases"],
        "pairs_per_particle": cnt["pairs"] / nprof / n,
        "candidates_per_particle": cnt["candidates"] / nprof / n,
        # + 2 launches each for the velocity and the pressure smoothing
        # passes, + 1 for the renormalisation matrices
        "gpu_launches": ((KERNELS_PER_STEP if fp32c else KERNELS_PER_STEP_FP64)
                         + (4 if args.teta > 0 else 0) + (1 if args.c1 else 0)) * args.steps,
        # the line's figures are one window's (the median); every window launches as many
        "gpu_launches_all_windows": ((KERNELS_PER_STEP if fp32c else KERNELS_PER_STEP_FP64)
                                     + (4 if args.teta > 0 else 0) + (1 if args.c1 else 0))
                                    * args.steps * head["windows"],
        "clocks": head["clocks"],
        "cpu_baseline": cpu,
    }
    sim.close()
    if ws == 1 and not args.no_extras and args.workload == "dam_break_3d" and args.dx == 0.005 \
            and not args.c1 and args.teta == 0.0:
        line["workloads"] = run_extras(ws, rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
