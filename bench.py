"""Benchmark of the mgkmc mechanical-equilibrium hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): 2D small-strain Lippmann-Schwinger equilibrium solves on
a 256x256 periodic plane-strain grid with the heterogeneous material of the
KMC/AQS benchmark (mu ~ mu0 (1 + 0.1 N(0,1)) clipped, K = 100 GPa, 5 % pure
shear eigenstrains of magnitude 0.1, eps_xx = 0.01), solved to an update norm
of 1e-8 in FP64.  One step = one batch of ``--batch`` solves on distinct
seeded problems; value = solves/s over all ranks (replicas only: each rank
solves its own problems, no collective; scaling "weak").

``--impl reference`` times the CPU restatement of the reference algorithm
(oracle, numpy FFT) on the host cores, one process per core, on the same
problems, and prints the same JSON line.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX = NY = 256
TOL = 1e-8
METRIC = "equilibrium solves/s (2D LS 256^2, FP64, update norm 1e-8)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--grid", type=int, default=256, help="grid side (2^a 3^b); the headline workload is 256")
    a = ap.parse_args()
    global NX, NY
    NX = NY = a.grid
    return a


def _rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


# ------------------------------------------------------------- CPU legs ----
def _cpu_worker(args):
    seed, deadline = args
    from oracle import ls as OL
    from mgkmc_b200 import workloads as W
    E, nu, ep, eb = W.ls2d_problem(NX, NY, seed)
    n = 0
    t0 = time.perf_counter()
    while True:
        OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=TOL)
        n += 1
        if time.perf_counter() >= deadline:
            break
    return n, time.perf_counter() - t0


def cpu_baseline(seconds, procs):
    """Oracle restatement of the reference LS solve on host cores (bounded sample)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    deadline = time.perf_counter() + seconds
    t0 = time.perf_counter()
    if procs == 1:
        res = [_cpu_worker((0, deadline))]
    else:
        with ctx.Pool(procs) as pool:
            # perf_counter is per-process monotonic; pass a relative deadline
            res = pool.map(_cpu_worker_rel, [(s, seconds) for s in range(procs)])
    wall = time.perf_counter() - t0
    solves = sum(r[0] for r in res)
    return solves / wall, solves, wall


def _cpu_worker_rel(args):
    seed, seconds = args
    return _cpu_worker((seed, time.perf_counter() + seconds))


def run_reference(a):
    rank, world, _ = _rank()
    if rank != 0:
        return
    cores = os.cpu_count() or 1
    v, solves, wall = cpu_baseline(a.cpu_seconds, cores)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * a.batch / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, survey config)",
            "config": {"workload": "ls2d_256_fp64", "batch": a.batch, "grid": [NX, NY], "tol": TOL},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port",
                             "sample": f"{solves} oracle solves in {wall:.1f} s, one process per core"},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------- clocks ------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, nm in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


# ------------------------------------------------------------- GPU leg -----
def run_ours(a):
    import torch
    rank, world, local = _rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from mgkmc_b200 import _lib as L
    from mgkmc_b200 import linear_elastic_simulator as les
    from mgkmc_b200 import workloads as W

    B = a.batch
    probs = [W.ls2d_problem(NX, NY, seed=1000 * rank + b) for b in range(B)]
    solvers, eps, sig = [], [], []
    for (E, nu, ep, eb) in probs:
        s = les.Ls2dSolver(NX, NY)
        s.set_material(torch.from_numpy(E).to(dev), torch.from_numpy(nu).to(dev), torch.from_numpy(ep).to(dev))
        solvers.append(s)
        eps.append(torch.empty((NX, NY, 2, 2), dtype=torch.float64, device=dev))
        sig.append(torch.empty_like(eps[-1]))
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    stream = torch.cuda.current_stream()

    def step():
        for b in range(B):
            solvers[b].solve(probs[b][3], eps[b], sig[b], max_iter=500, tol=TOL, sync=False)

    for _ in range(a.warmup):
        step()
    torch.cuda.synchronize()
    # iterations per solve (device-decided) for the launch count and roofline
    iters = []
    for b in range(B):
        info = solvers[b].solve(probs[b][3], eps[b], sig[b], max_iter=500, tol=TOL, sync=True)
        iters.append(info.iterations)
    # equilibrium residual of the returned field: one LS iteration from it
    chk = solvers[0].solve(probs[0][3], torch.empty_like(eps[0]), torch.empty_like(sig[0]), eps_init=eps[0],
                           max_iter=1, tol=0.0, sync=True)
    residual = chk.final_diff

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(a.steps)]
    for k in range(a.steps):
        flush.zero_()  # L2 flush between timed steps (outside the timed events)
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = sum(e0.elapsed_time(e1) for e0, e1 in ev)
    if world > 1:
        t = torch.tensor([ms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = float(t.item())
    solves = B * a.steps * world
    value = solves / (ms / 1e3)

    # per-kernel timing of one LS iteration (row and column kernels) on solver 0
    kt = solvers[0].profile_kernels(probs[0][3], reps=50)

    # end-to-end through the reference-facing API with host numpy buffers
    e2e_n = 0
    h2d = d2h = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(max(1, a.steps // 2)):
        for b in range(min(B, 8)):
            E, nu, ep, eb = probs[b]
            les.spectral_solver_2d(E, nu, eb, ep, max_iter=500, tol=TOL)
            e2e_n += 1
    e2e_s = time.perf_counter() - t0
    h2d = (E.nbytes + nu.nbytes + ep.nbytes)
    d2h = 2 * ep.nbytes
    e2e_val = e2e_n / e2e_s * world

    launches_per_solve = [4 + 2 * i for i in iters]  # begin, row0, (col,row) x iters, output, finalize
    gpu_launches = int(sum(launches_per_solve) * a.steps)

    if rank != 0:
        return
    N = NX * NY
    roof = None
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    peak_kind = "measured" if os.path.exists(peaks_path) else "fallback"
    if kt is not None:
        row_ms, col_ms = kt
        row_bytes = 136.0 * N
        achieved = row_bytes / (row_ms * 1e-3) / 1e9
        roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": None, "kernel": "ls2d_row_kernel<double,true>", "peak_kind": peak_kind,
                "row_us": row_ms * 1e3, "col_us": col_ms * 1e3}
    cpu = None
    if world == 1 and a.cpu_seconds > 0:
        v, nsol, wall = cpu_baseline(a.cpu_seconds, 1)
        cpu = {"value": v, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"{nsol} oracle solves of the same {NX}^2 problem in {wall:.1f} s (numpy FFT, 1 thread)"}
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, survey config)",
            "config": {"workload": f"ls2d_{NX}_fp64_plain", "batch": B, "grid": [NX, NY], "tol": TOL,
                       "l2": "flushed between steps (256 MB write)", "iters_mean": float(np.mean(iters)),
                       "residual": residual, "parallelism": f"replicas x{world}"},
            "e2e": {"value": e2e_val, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "api": "mgkmc_b200.linear_elastic_simulator.spectral_solver_2d"},
            "gpu_launches": gpu_launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
