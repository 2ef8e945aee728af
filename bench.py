"""Benchmark of the mgkmc mechanical-equilibrium hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (default): 2D small-strain Lippmann-Schwinger equilibrium solves on
a 256x256 periodic plane-strain grid with the heterogeneous material of the
KMC/AQS benchmark (mu ~ mu0 (1 + 0.1 N(0,1)) clipped, K = 100 GPa, 5 % pure
shear eigenstrains of magnitude 0.1, eps_xx = 0.01), solved to an update norm
of 1e-8.  One step = one batch of ``--batch`` solves on distinct seeded
problems, in three forms: plain FP64 (one solve after another), batched FP64
(one launch per stage for the batch) and batched mixed precision (FP32 bulk,
FP64 finish; the headline value).  value = solves/s over all ranks (replicas
only: each rank solves its own problems, no collective; scaling "weak").

Finite-strain block (N = 1, ``--fs-grid``, default 128^3): the 10-step
Neo-Hookean ramp of the finite-strain workload in the plain FP64 form and the
mixed form (FP32 Krylov matvecs), device-timed, with the mixed form's field
error and the per-kernel times of one Krylov iteration.

Ensemble block (``--ensemble 96``, off by default: about a minute): the
batched KMC ensemble, events/s and replica-solves/s.

Serving block (N = 1, ``--serve-window`` seconds of the serving stream): the
continuous-batching server in mixed precision against the plain FP64 form
served one request at a time, both on this GPU with arrivals replayed in real
time; solves/s and p50/p99 request latency of each, and their ratios.

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
METRIC = ("equilibrium solves/s (2D LS 256^2, update norm 1e-8, field err <= 1e-6 vs FP64); "
          "serving block: served mixed precision vs plain FP64 sequential, solves/s and p50/p99 latency")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--grid", type=int, default=256, help="grid side (2^a 3^b); the headline workload is 256")
    ap.add_argument("--forms", default="plain_fp64,batched_fp64,batched_mixed",
                    help="comma list of forms to time (the headline is batched_mixed)")
    ap.add_argument("--fs-grid", type=int, default=128,
                    help="side of the finite-strain block (Neo-Hookean + F_p, 10 load steps); 0 skips it")
    ap.add_argument("--ensemble", type=int, default=96,
                    help="replicas of the batched KMC ensemble block (96 = the ensemble workload, ~1 min); 0 skips it")
    ap.add_argument("--ensemble-ragged", type=int, default=1,
                    help="1: also run the ensemble with every replica in one ragged plan; 0 skips it")
    ap.add_argument("--kmc-events", type=int, default=2000,
                    help="events of the 256^2 x 8 KMC/AQS block (2000 = the KMC workload); 0 skips it")
    ap.add_argument("--landau", type=int, default=1, help="1: the Landau 2D block (256^2, Anderson depth 5); 0 skips it")
    ap.add_argument("--serve-window", type=float, default=0.25,
                    help="seconds of the serving stream (Poisson 200 req/s, seed 3) replayed in the serving block; "
                         "0 skips it")
    ap.add_argument("--serve-plain", type=int, default=0,
                    help="0: the plain FP64 form's service time is measured for every request of the window; n > 0: "
                         "for a seeded subsample of n (the others get a measured time of their class: an estimate)")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving block (a long window: --serve-window 10 --serve-plain 150)")
    ap.add_argument("--cpu-kmc-seconds", type=float, default=12.0,
                    help="seconds of the oracle's per-event KMC loop at 256^2 x 8 on one host core; 0 skips it")
    ap.add_argument("--cpu-fs-grid", type=int, default=32,
                    help="side of the oracle's finite-strain load step on one host core; 0 skips it")
    ap.add_argument("--profile-case", default="", choices=["", "ls3d", "fs3d", "kmc", "landau"],
                    help="run one kernel-profiling workload instead of the benchmark (for ncu captures): ls3d = "
                         "LS 3D solves at --profile-n^3 (tol 1e-8, three solves), fs3d = one finite-strain load "
                         "step at --profile-n^3 (Neo-Hookean + 2 %% F_p, F_xx = 1.005), kmc = three rounds of "
                         "barrier, exact rates/total and selection at --profile-n^2 x 8 modes, landau = three Landau "
                         "LS 2D solves at --profile-n^2 (Anderson depth 5, tol 1e-8)")
    ap.add_argument("--profile-n", type=int, default=128)
    ap.add_argument("--profile-precision", default="fp64", choices=["fp64", "mixed"])
    a = ap.parse_args()
    global NX, NY
    NX = NY = a.grid
    return a


def _rank():
    return int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), int(os.environ.get("LOCAL_RANK", "0"))


def _max_over_ranks(values, device=None):
    """Element-wise maximum of per-rank values over the job's ranks (a job's
    time is its slowest rank's); the values themselves on one process."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return [float(v) for v in values]
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def _job_rates(ms, per_rank_items, steps, world):
    """Whole-job throughput: every rank's items over the slowest rank's time
    (ms: {form: max-over-ranks milliseconds for `steps` steps})."""
    return {k: per_rank_items * steps * world / (v / 1e3) for k, v in ms.items()}


# ------------------------------------------------------------- CPU legs ----
_THREAD_VARS = ("OMP_NUM_THREADS", "OPENBLAS_NUM_THREADS", "MKL_NUM_THREADS", "NUMEXPR_NUM_THREADS",
                "VECLIB_MAXIMUM_THREADS")


def _single_thread_env():
    """One BLAS/OpenMP thread per process: spawned CPU workers inherit this
    environment before numpy loads, so P processes use P cores, not P^2
    threads."""
    for k in _THREAD_VARS:
        os.environ[k] = "1"


def host_cpu():
    """Host cores this process may use: the affinity mask, capped by a cgroup
    CPU quota when one is set (a container can see many cores and be allowed
    a fraction of them), and the CPU model."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    try:
        aff = len(os.sched_getaffinity(0))
    except AttributeError:
        aff = os.cpu_count() or 1
    quota = None
    for path in ("/sys/fs/cgroup/cpu.max",):
        try:
            q, p = open(path).read().split()[:2]
            if q != "max":
                quota = float(q) / float(p)
        except (OSError, ValueError):
            pass
    if quota is None:
        try:
            q = float(open("/sys/fs/cgroup/cpu/cpu.cfs_quota_us").read())
            p = float(open("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read())
            if q > 0:
                quota = q / p
        except (OSError, ValueError):
            pass
    usable = aff if quota is None else max(1, min(aff, int(quota + 1e-9)))
    return {"model": model, "cpu_count": os.cpu_count(), "affinity": aff, "cgroup_quota_cores": quota,
            "usable": usable}


def _ls_worker(widx, share, warm_steps, steps, grid, tol, start, ready, results):
    """Reference-arm worker: its share of every step's LS solves, after its
    warm-up steps; reports when its timed steps end (perf_counter is the
    system-wide monotonic clock on Linux, comparable across processes)."""
    from oracle import ls as OL
    from mgkmc_b200 import workloads as W
    E, nu, ep, eb = W.ls2d_problem(grid, grid, widx)
    OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=tol)  # first call: imports, FFT plans
    for _ in range(warm_steps * share):
        OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=tol)
    ready.put(widx)
    start.wait()
    n = 0
    for _ in range(steps * share):
        OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=tol)
        n += 1
    results.put((widx, time.perf_counter(), n))


def cpu_ls_steps(procs, per_step, warm_steps, steps, grid, tol):
    """Times `steps` steps of `per_step` oracle LS solves spread over `procs`
    single-threaded spawn-started processes; the clock starts once every
    worker has finished its warm-up.  Returns (solves/s, wall s, solves)."""
    import multiprocessing as mp
    _single_thread_env()
    ctx = mp.get_context("spawn")
    start, ready, results = ctx.Event(), ctx.Queue(), ctx.Queue()
    shares = [per_step // procs + (1 if i < per_step % procs else 0) for i in range(procs)]
    ws = [ctx.Process(target=_ls_worker, args=(i, shares[i], warm_steps, steps, grid, tol, start, ready, results))
          for i in range(procs) if shares[i] > 0]
    for w in ws:
        w.start()
    try:
        for _ in ws:
            ready.get(timeout=900)
        t0 = time.perf_counter()
        start.set()
        ends = [results.get(timeout=1800) for _ in ws]
    finally:
        for w in ws:
            w.join(timeout=60)
    wall = max(e[1] for e in ends) - t0
    solves = sum(e[2] for e in ends)
    return solves / wall, wall, solves


def cpu_ls_baseline(seconds):
    """One host core, oracle LS solves of the headline problem for about
    `seconds` (bounded sample); returns (solves/s, solves, wall s)."""
    from oracle import ls as OL
    from mgkmc_b200 import workloads as W
    E, nu, ep, eb = W.ls2d_problem(NX, NY, 0)
    OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=TOL)
    n, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < seconds:
        OL.spectral_solver(E, nu, eb, ep, max_iter=500, tol=TOL)
        n += 1
    wall = time.perf_counter() - t0
    return n / wall, n, wall


def cpu_kmc_sample(seconds, n=256, M=8, strain=0.024):
    """One host core, the oracle's per-event loop of the 256^2 x 8 KMC/AQS
    workload (kmc_simulator.py:871-1101): barriers, rates with the sequential
    total, selection, flip with redraws and a cold LS re-solve (tol 1e-6),
    from a state pre-strained to `strain` (where the workload's events
    happen), for about `seconds`.  Returns seconds per LS solve and per rate
    step (barriers + rates), and events done."""
    from oracle import kmc as OK
    from oracle import ls as OL
    from oracle.kmc_driver import pure_shear_modes
    from mgkmc_b200 import workloads as W
    rng = np.random.default_rng(1)
    E, nu = W.ls2d_material(n, n, rng)
    cat, Q0 = W.kmc2d_state(n, n, M, rng)
    eps_p = np.zeros((n, n, 2, 2))
    soft, t_last = np.zeros((n, n, 2)), np.full((n, n), -np.inf)
    prev, Q = np.zeros((n, n, 2, 2)), np.zeros((n, n, M))
    eb = np.zeros((2, 2))
    eb[0, 0], eb[1, 1] = strain, -0.4 * strain
    t_solve, t_rate, events = [], [], 0
    t = time.perf_counter()
    _, sig, _, _ = OL.spectral_solver(E, nu, eb, eps_p, max_iter=200, tol=1e-6)
    t_solve.append(time.perf_counter() - t)
    t_end = time.perf_counter() + seconds
    tau = 1.0 / (1e13 * np.exp(-0.37 / (OK.KB * 300.0)))
    while time.perf_counter() < t_end:
        t = time.perf_counter()
        OK.compute_barrier(Q, Q0, sig, cat, 1.0, soft, t_last, 0.0, prev, 2.0, 0, tau)
        rates, idx, total = OK.compute_rates(Q, 1.0, 300.0, 1e13, cascade_mode=False)
        k = OK.select_event(rates, total, rng.random())
        t_rate.append(time.perf_counter() - t)
        x, y, m = OK.decode_index_2d(int(idx[k]), n, M)
        OK.apply_flip_2d(eps_p, soft, t_last, cat, x, y, m, 0.0, 0.0, 0.0, 2.0, 0.0)
        prev[x, y] = cat[x, y, m]
        cat[x, y] = pure_shear_modes(rng.uniform(0.0, np.pi, M), 0.1)
        Q0[x, y] = np.clip(rng.normal(1.0, 0.15, M), 0.3, None)
        t = time.perf_counter()
        _, sig, _, _ = OL.spectral_solver(E, nu, eb, eps_p, max_iter=200, tol=1e-6)
        t_solve.append(time.perf_counter() - t)
        events += 1
    return float(np.mean(t_solve)), float(np.mean(t_rate)), events, len(t_solve)


def cpu_fs_sample(n=32):
    """One host core, the oracle's first load step of the finite-strain
    workload (Neo-Hookean + 2 % F_p, F_xx = 1.005, lateral stresses zero,
    Newton 1e-8, CG 1e-6) at n^3.  Returns (seconds, Newton, Krylov)."""
    from oracle import fs as OF
    from mgkmc_b200 import workloads as W
    E, nu, Fp = W.fs3d_material(n, n, n, np.random.default_rng(2))
    Fp = OF.to_spatial(Fp)
    F = np.broadcast_to(np.eye(3), (n, n, n, 3, 3)).copy()
    Fb, _, Pt, Pm = OF.build_bc_3d((0, 0), 0.005, {(1, 1): 0.0, (2, 2): 0.0})
    t0 = time.perf_counter()
    OF.solver_step_3d(F, Fb, E, nu, Fp, (0, 0), Pt, Pm, tol_NW=1e-8, tol_CG=1e-6, model="neo_hookean",
                      krylov="cg")
    return time.perf_counter() - t0


def headline_config(a, world=1):
    """The workload description both arms print (identical dicts)."""
    return {"workload": f"ls2d_{NX}_batched_mixed", "problems_per_step": a.batch, "grid": [NX, NY], "tol": TOL,
            "material": "mu ~ mu0 (1 + 0.1 N(0,1)) clipped [0.7,1.3] mu0, K = 100 GPa, 5 % pure-shear "
                        "eigenstrains gamma0 = 0.1, eps_xx = 0.01, plane strain",
            "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{world}"}


def run_reference(a):
    """The reference's CPU path (the oracle restatement of spectral_solver_2d:
    the reference is Python and does not travel to the GPU host) on this
    host's usable cores: one single-threaded process per core, each step a
    bounded sample of the headline workload's solves."""
    rank, world, _ = _rank()
    if rank != 0:
        return
    info = host_cpu()
    P = info["usable"]
    per_step = min(a.batch, 2 * P)
    v, wall, solves = cpu_ls_steps(P, per_step, max(1, a.warmup), a.steps, NX, TOL)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": a.gpus,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1e3 * wall / a.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; the benchmark material and sizes, no dataset)",
            "config": headline_config(a, world),
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": P, "kind": "port",
                             "sample": f"{a.steps} steps x {per_step} solves of the {NX}^2 problem (tol {TOL:g}), "
                                       f"{P} single-threaded processes, clock started after every process had "
                                       f"solved {max(1, a.warmup)} warm-up steps; {solves} solves in {wall:.2f} s",
                             "host": info},
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


# ------------------------------------------------------------- serving -----
def _fifo(arrivals, services):
    """Latencies of a single sequential server taking requests in arrival
    order: start = max(arrival, previous finish), finish = start + service."""
    lat, finish = [], 0.0
    for a, s in zip(arrivals, services):
        finish = max(a, finish) + s
        lat.append(finish - a)
    return np.array(lat)


def run_serving(window, n_plain=0, progress=None):
    """The serving stream's first `window` seconds of arrivals served by the
    continuous-batching server (mixed precision, arrivals replayed in real
    time, latency = completion - arrival on the host clock), against the plain
    FP64 form served sequentially.  The sequential form runs one request at a
    time, so a request's service time does not depend on the others: each is
    measured running alone (back to back), and the sequential latencies of
    the same arrivals follow exactly from the FIFO recursion.  n_plain = 0
    measures every request's service time; n_plain > 0 measures a seeded
    subsample and gives each other request the measured service time of a
    subsampled request of its class (kind, dimension, side) -- an estimate,
    labelled as such.  Solves/s: served = solves over the makespan; plain =
    solves over the measured busy time.  progress: seconds between progress
    lines on stderr, and the served summary printed there as soon as it is
    known (None: quiet)."""
    from mgkmc_b200.serving import Server, request_stream, summarize
    reqs = [r for r in request_stream(rate=200.0, duration=60.0, seed=3) if r.t_arrival <= window]
    out = {"workload": (f"serving stream (Poisson 200 req/s, seed 3; 60 % equilibrium solves, 40 % 100-event KMC "
                        f"trajectories; 70 % 2D sides 64..1024, 30 % 3D sides 64..128): the {len(reqs)} arrivals of "
                        f"its first {window:g} s"),
           "classes": {}}
    for r in reqs:
        k = f"{r.dim}d_{r.kind}_{r.n}"
        out["classes"][k] = out["classes"].get(k, 0) + 1
    srv = Server(mode="served")
    srv.progress = progress
    srv.prepare(reqs)
    res = srv.run(reqs, realtime=True)
    out["served_mixed"] = summarize(res)
    if progress is not None:
        print(json.dumps({"served_mixed": out["served_mixed"]}), file=sys.stderr, flush=True)
    del srv
    if n_plain and n_plain < len(reqs):
        rng = np.random.default_rng(4)
        sub = [reqs[i] for i in sorted(rng.choice(len(reqs), size=n_plain, replace=False))]
    else:
        sub = reqs
    srv = Server(mode="sequential")
    srv.progress = progress
    srv.prepare(sub)
    res_p = srv.run(sub, realtime=False)
    ok = [r for r in res_p if not r.error]
    svc = {r.rid: r.t_done - r.t_admit for r in ok}
    solves = sum(r.solves for r in ok)
    busy = sum(svc.values())
    plain = {"measured_requests": len(ok), "errors": len(res_p) - len(ok), "solves": solves, "busy_s": busy,
             "solves_per_busy_s": solves / max(busy, 1e-9),
             "service_p50_s": float(np.percentile(list(svc.values()), 50)),
             "service_p99_s": float(np.percentile(list(svc.values()), 99))}
    cls = {}
    for r in sub:
        if r.rid in svc:
            cls.setdefault((r.kind, r.dim, r.n), []).append(svc[r.rid])
    services, estimated = [], 0
    rng = np.random.default_rng(5)
    for r in reqs:
        if r.rid in svc:
            services.append(svc[r.rid])
        else:
            pool = cls.get((r.kind, r.dim, r.n)) or [v for (k, d, _), vs in cls.items() if (k, d) == (r.kind, r.dim)
                                                      for v in vs]
            services.append(float(rng.choice(pool)))
            estimated += 1
    lat = _fifo([r.t_arrival for r in reqs], services)
    # the whole window's plain busy time and solves: measured where measured;
    # elsewhere the class's service time and the served run's solve count of
    # the request (both forms run the same macro-loop solves)
    plain_solves = {r.rid: r.solves for r in ok}
    served_solves = {r.rid: r.solves for r in res}
    win_solves = sum(plain_solves.get(r.rid, served_solves.get(r.rid, 0)) for r in reqs)
    win_busy = float(np.sum(services))
    plain.update(window_solves=int(win_solves), window_busy_s=win_busy,
                 window_solves_per_busy_s=win_solves / max(win_busy, 1e-9),
                 latency_p50_s=float(np.percentile(lat, 50)), latency_p99_s=float(np.percentile(lat, 99)),
                 makespan_s=float(reqs[-1].t_arrival + lat[-1] - reqs[0].t_arrival) if len(lat) else 0.0,
                 service_times="measured for every request" if estimated == 0 else
                 f"measured for {len(reqs) - estimated}, drawn from the measured times of the same class for "
                 f"{estimated} (estimate)")
    out["plain_fp64_sequential"] = plain
    from mgkmc_b200 import serving as SV
    out["autotuned_ls_families"] = {f"{k[0]}^2 x{k[1]} {k[2]}": {"family": v[0], "ms_per_iteration": v[1]}
                                    for k, v in SV._TUNED.items() if isinstance(k[0], int)}
    a = out["served_mixed"]
    if a.get("completed"):
        out["solves_per_s_ratio"] = a["solves_per_s"] / plain["solves_per_busy_s"]
        out["solves_per_s_ratio_window"] = a["solves_per_s"] / plain["window_solves_per_busy_s"]
        out["p50_ratio"] = plain["latency_p50_s"] / a["p50_s"]
        out["p99_ratio"] = plain["latency_p99_s"] / a["p99_s"]
    return out


# ------------------------------------------------------------- KMC/AQS -----
def run_kmc(n_events, n=256, M=8):
    """The 256^2 x 8 KMC/AQS workload (heterogeneous medium, Q0 ~ N(1.0,
    0.15) eV clipped at 0.3, T = 300 K, AQS steps of 1e-5 at a strain rate of
    1e7/s, lateral mean stress driven to zero) for `n_events` events, in the
    plain form (FP64 cold LS re-solves at tol 1e-6, the bit-exact sequential
    rate total: the reference's arithmetic) and the served form (mixed
    precision, warm starts, the fused rate pass).  Device-driven trajectory;
    timed with CUDA events and the host clock."""
    import torch
    from mgkmc_b200.kmc import Kmc2D
    from mgkmc_b200 import workloads as W
    rng0 = np.random.default_rng(1)
    E, nu = W.ls2d_material(n, n, rng0)
    cat, Q0 = W.kmc2d_state(n, n, M, rng0)
    out = {"workload": f"KMC/AQS {n}^2 x {M} modes, {n_events} events, seed 1"}
    for name, kw in (("plain_fp64_exact", dict(selection="exact", ls_start="cold", precision="fp64")),
                     ("served_mixed_fast", dict(selection="fast", ls_start="warm", precision="mixed"))):
        k = Kmc2D(E, nu, cat, Q0, **kw)
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        e0.record(st)
        r = k.run(np.random.default_rng(1), 10 ** 9, max_events=n_events)
        e1.record(st)
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        out[name] = {"seconds": wall, "device_span_s": e0.elapsed_time(e1) / 1e3, "events": len(r["events"]),
                     "aqs_steps": int(r["steps"]), "solves": int(r["solves"]),
                     "events_per_s": len(r["events"]) / wall, "final_strain_xx": float(r["eps_macro"][0, 0]),
                     "sim_time_s": float(r["time"])}
        del k
    return out


# the Landau coefficients (v1, v2, v3, g1, g2, g3, g4) in Pa of the
# reference's Landau tests
LANDAU_COEFF = (-199.7e9, -75.4e9, -23.1e9, 1432.0e9, 311.0e9, 145.0e9, -273.0e9)


def _landau_device(n, m, reps=5, tol=1e-8):
    """Device time of one Landau LS solve at n^2 with Anderson depth m (CUDA
    events, device-resident fields), its iterations, and the per-iteration
    time from the difference with a solve capped at 2 iterations."""
    import torch
    from mgkmc_b200 import linear_elastic_simulator as les
    from mgkmc_b200 import workloads as W
    E, nu, ep, _ = W.ls2d_problem(n, n, seed=13)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    eb = np.array([[0.008, 0.002], [0.002, -0.003]])
    dev = torch.device("cuda", torch.cuda.current_device())
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    p = les.Ls2dBatch([(n, n)])
    p.set_landau(LANDAU_COEFF)
    p.set_anderson(m)
    p.set_lame(0, t(lam), t(mu), t(ep))
    eps = torch.empty((n, n, 2, 2), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    ms, its = {}, {}
    for cap in (2, 400):
        its[cap] = p.solve([0], [eb], [eps], [sig], max_iter=cap, tol=tol)[0].iterations
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record()
        for _ in range(reps):
            p.solve([0], [eb], [eps], [sig], max_iter=cap, tol=tol, sync=False)
        e1.record()
        torch.cuda.synchronize()
        ms[cap] = e0.elapsed_time(e1) / reps
    return ms[400], int(its[400]), (ms[400] - ms[2]) / max(1, its[400] - 2) * 1e3


def run_landau(n=256, m=5, reps=5):
    """The Landau 2D LS solve (plane strain, Anderson depth m) at n^2 on the
    benchmark material and eigenstrains with a sheared macro strain, tol 1e-8:
    the numpy-in, numpy-out drop-in (host clock) and the device-resident
    solve (CUDA events); per-iteration device times (tol 1e-12, so that the
    loops run long enough) at depths 0, 1 and m, at n^2 and 1024^2."""
    import torch
    from mgkmc_b200 import linear_elastic_simulator as les
    from mgkmc_b200 import workloads as W
    E, nu, ep, _ = W.ls2d_problem(n, n, seed=13)
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    eb = np.array([[0.008, 0.002], [0.002, -0.003]])
    kw = dict(zip(("v1", "v2", "v3", "g1", "g2", "g3", "g4"), LANDAU_COEFF))
    les.spectral_solver_landau_2d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, tol=1e-8, anderson_m=m)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(reps):
        les.spectral_solver_landau_2d(lam, mu, **kw, eps_bar=eb, eps_plastic=ep, tol=1e-8, anderson_m=m)
    dropin_ms = (time.perf_counter() - t0) / reps * 1e3
    solve_ms, iters, _ = _landau_device(n, m, reps)
    per_it = {}
    for side in (n, 1024):
        for depth in (0, 1, m):
            per_it[f"{side}^2 depth {depth}"] = _landau_device(side, depth, reps, tol=1e-12)[2]
    return {"workload": f"Landau LS 2D {n}^2 plane strain, Anderson depth {m}, tol 1e-8, benchmark material "
                        f"and eigenstrains, eps_bar = [[0.008, 0.002], [0.002, -0.003]]",
            "dropin_ms": dropin_ms, "device_solve_ms": solve_ms, "iterations": iters,
            "device_us_per_iteration": per_it}


# ------------------------------------------------------- finite strain -----
def run_finite_strain(n, peak):
    """3D finite-strain ramp (Neo-Hookean, 2 % F_p, F_xx to 1.05 in 10 load
    steps, lateral stresses zero, Newton 1e-8, CG 1e-6) in the plain FP64 form
    and the mixed form (FP32 Krylov matvecs), device-timed; the mixed form's
    field error against FP64; per-kernel times of one Krylov iteration."""
    import torch
    from mgkmc_b200 import workloads as W
    from mgkmc_b200.finite_strain_simulator import Fs3dSolver, simulate_3d
    E, nu, Fp = W.fs3d_material(n, n, n, np.random.default_rng(2))
    out = {"workload": f"finite strain {n}^3, Neo-Hookean + 2 % F_p, F_xx 1 -> 1.05 in 10 load steps, "
                       f"lateral stresses zero, Newton tol 1e-8, CG tol 1e-6"}
    fields = {}
    N = n ** 3
    for prec in ("fp64", "mixed"):
        solver = Fs3dSolver(n, n, n, model="neo_hookean", precision=prec)
        st = torch.cuda.current_stream()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(st)
        s, steps = simulate_3d(E, nu, Fp, 0.05, 10, mixed_targets={(1, 1): 0.0, (2, 2): 0.0}, model="neo_hookean",
                               tol_NW=1e-8, tol_CG=1e-6, solver=solver)
        e1.record(st)
        torch.cuda.synchronize()
        sec = e0.elapsed_time(e1) / 1e3
        F = torch.empty((3, 3, n, n, n), dtype=torch.float64, device="cuda")
        P = torch.empty_like(F)
        s.get(F, P)
        fields[prec] = (F, P)
        ms = s.profile_kernels(fp32=(prec == "mixed"), reps=10)
        w = 8.0 if prec == "fp64" else 4.0
        it_bytes = 110.0 * w * N  # algorithmic bytes of one Krylov iteration
        out[prec] = {"seconds": sec, "load_steps_per_s": 11 / sec,
                     "krylov": int(sum(x[1]["krylov"] for x in steps)),
                     "newton": int(sum(x[1]["newton"] for x in steps)),
                     "macro": int(sum(x[1]["macro"] for x in steps)),
                     "kernels_us": dict(zip(["z_fwd_Kp", "y", "x_G", "y_inv", "z_inv_pq", "cg_update"],
                                            [round(1e3 * v, 1) for v in ms])),
                     "krylov_iteration_gbs": it_bytes / (sum(ms) * 1e-3) / 1e9,
                     "krylov_iteration_frac_of_measured_hbm": it_bytes / (sum(ms) * 1e-3) / 1e9 / peak}
        del s, solver
    (Fa, Pa), (Fb, Pb) = fields["mixed"], fields["fp64"]
    out["mixed_speedup"] = out["fp64"]["seconds"] / out["mixed"]["seconds"]
    out["mixed_field_err_vs_fp64"] = {"F": float((Fa - Fb).abs().max() / Fb.abs().max()),
                                      "P": float((Pa - Pb).abs().max() / Pb.abs().max())}
    return out


# ------------------------------------------------------------- GPU leg -----
def _time_steps(step, steps, flush, stream):
    """Device time (ms) of `steps` calls of step(), L2 flushed between them."""
    import torch
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
    for k in range(steps):
        flush.zero_()  # > L2 write between timed steps, outside the events
        ev[k][0].record(stream)
        step()
        ev[k][1].record(stream)
    torch.cuda.synchronize()
    return sum(e0.elapsed_time(e1) for e0, e1 in ev)


def run_ours(a):
    import torch
    rank, world, local = _rank()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    from mgkmc_b200 import linear_elastic_simulator as les
    from mgkmc_b200 import workloads as W

    B = a.batch
    probs = [W.ls2d_problem(NX, NY, seed=1000 * rank + b) for b in range(B)]
    dE = [torch.from_numpy(p[0]).to(dev) for p in probs]
    dnu = [torch.from_numpy(p[1]).to(dev) for p in probs]
    dep = [torch.from_numpy(p[2]).to(dev) for p in probs]
    ebs = [p[3] for p in probs]
    eps = [torch.empty((NX, NY, 2, 2), dtype=torch.float64, device=dev) for _ in range(B)]
    sig = [torch.empty_like(e) for e in eps]
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > L2 (126 MB)
    stream = torch.cuda.current_stream()
    reps = list(range(B))

    # form 1: plain FP64, one plan per problem, one solve after another
    plain = []
    for b in range(B):
        s = les.Ls2dSolver(NX, NY)
        s.set_material(dE[b], dnu[b], dep[b])
        plain.append(s)

    def step_plain():
        for b in range(B):
            plain[b].solve(ebs[b], eps[b], sig[b], max_iter=500, tol=TOL, sync=False)

    # forms 2 and 3: one launch per stage for the whole batch
    batches = {}
    for prec in ("fp64", "mixed"):
        bt = les.Ls2dBatch([(NX, NY)] * B, precision=prec)
        for b in range(B):
            bt.set_material(b, dE[b], dnu[b], dep[b])
        batches[prec] = bt

    def step_batch(prec):
        batches[prec].solve(reps, ebs, eps, sig, max_iter=500, tol=TOL, sync=False)

    forms = {"plain_fp64": step_plain, "batched_fp64": lambda: step_batch("fp64"),
             "batched_mixed": lambda: step_batch("mixed")}
    keep = [f for f in a.forms.split(",") if f]
    forms = {k: v for k, v in forms.items() if k in keep}
    iters = {}
    for name, fn in forms.items():
        for _ in range(a.warmup):
            fn()
    torch.cuda.synchronize()
    iters["plain_fp64"] = [plain[b].solve(ebs[b], eps[b], sig[b], max_iter=500, tol=TOL).iterations for b in range(B)]
    ref_eps = [e.clone() for e in eps]
    for prec in ("fp64", "mixed"):
        inf = batches[prec].solve(reps, ebs, eps, sig, max_iter=500, tol=TOL, sync=True)
        iters["batched_" + prec] = [i.iterations for i in inf]
    # mixed-form field error against the FP64 result, and its equilibrium
    # residual: one FP64 LS iteration started from the mixed field
    err_mixed = max(float((eps[b] - ref_eps[b]).abs().max() / ref_eps[b].abs().max()) for b in range(B))
    chk = plain[0].solve(ebs[0], torch.empty_like(eps[0]), torch.empty_like(sig[0]), eps_init=eps[0].clone(),
                         max_iter=1, tol=0.0, sync=True)
    residual = chk.final_diff

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    clk.start()
    ms = {name: _time_steps(fn, a.steps, flush, stream) for name, fn in forms.items()}
    clocks = clk.stop()
    ms = dict(zip(forms, _max_over_ranks([ms[k] for k in forms], dev)))
    rate = _job_rates(ms, B, a.steps, world)
    head = "batched_mixed" if "batched_mixed" in forms else list(forms)[-1]

    # per-kernel timing (CUDA events on the launching stream) over the batch
    row64, col64 = batches["fp64"].profile_kernels(reps, ebs, fp32=False, n=20)
    row32, col32 = batches["mixed"].profile_kernels(reps, ebs, fp32=True, n=20)

    # end to end through the batch API with pinned host buffers: every step
    # copies its problems' E, nu, eps_p host -> device, sets the materials,
    # solves (mixed form) and copies eps and sig device -> host.  The batch's
    # fields sit in contiguous (B, ...) buffers (one copy per field and
    # direction; the API gets per-replica views), and three plans on three
    # streams take steps in turn, so one step's input copies, another's solve
    # and a third's result copies overlap, the way a caller pipelines batches
    # through the API.
    hE = torch.from_numpy(np.stack([p[0] for p in probs])).pin_memory()
    hnu = torch.from_numpy(np.stack([p[1] for p in probs])).pin_memory()
    hep = torch.from_numpy(np.stack([p[2] for p in probs])).pin_memory()

    def e2e_slot(bt):
        shp = (B, NX, NY, 2, 2)
        return dict(bt=bt, s=torch.cuda.Stream(), dE=torch.empty_like(hE, device=dev),
                    dnu=torch.empty_like(hnu, device=dev), dep=torch.empty_like(hep, device=dev),
                    eps=torch.empty(shp, dtype=torch.float64, device=dev),
                    sig=torch.empty(shp, dtype=torch.float64, device=dev),
                    heps=torch.empty(shp, dtype=torch.float64).pin_memory(),
                    hsig=torch.empty(shp, dtype=torch.float64).pin_memory())

    slots = [e2e_slot(batches["mixed"])] + [e2e_slot(les.Ls2dBatch([(NX, NY)] * B, precision="mixed"))
                                            for _ in range(2)]

    def e2e_step(k):
        sl = slots[k % len(slots)]
        with torch.cuda.stream(sl["s"]):
            sl["dE"].copy_(hE, non_blocking=True)
            sl["dnu"].copy_(hnu, non_blocking=True)
            sl["dep"].copy_(hep, non_blocking=True)
            for b in range(B):
                sl["bt"].set_material(b, sl["dE"][b], sl["dnu"][b], sl["dep"][b])
            sl["bt"].solve(reps, ebs, list(sl["eps"].unbind(0)), list(sl["sig"].unbind(0)), max_iter=500, tol=TOL,
                           sync=False)
            sl["heps"].copy_(sl["eps"], non_blocking=True)
            sl["hsig"].copy_(sl["sig"], non_blocking=True)

    torch.cuda.synchronize()
    for k in range(len(slots)):
        e2e_step(k)
    torch.cuda.synchronize()
    n_e2e = max(6, a.steps)
    t0 = time.perf_counter()
    for k in range(n_e2e):
        e2e_step(k)
    torch.cuda.synchronize()
    e2e_s = time.perf_counter() - t0
    # the host copy of the results against the device-resident batched solve
    e2e_err = max(float((slots[1]["heps"][b] - eps[b].cpu()).abs().max() / eps[b].abs().max().cpu())
                  for b in range(B))
    h2d = hE.nbytes + hnu.nbytes + hep.nbytes
    d2h = slots[0]["heps"].nbytes + slots[0]["hsig"].nbytes
    e2e_val = B * n_e2e / e2e_s * world

    it_head = iters[head]
    gpu_launches = int(a.steps * (7 + 2 * max(it_head) + 3))  # begin, row0, 2/iter, promote+phase2+row0, output, finalize

    if rank != 0:
        return
    N = NX * NY
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(peaks_path))["hbm_gbs"] if os.path.exists(peaks_path) else 6650.0
    peak_kind = "measured" if os.path.exists(peaks_path) else "fallback"
    row_bytes = 136.0 * N * B
    achieved = row_bytes / (row64 * 1e-3) / 1e9
    # DRAM read+write bytes of one launch of this kernel on this workload (32 x
    # 256^2, FP64), from the ncu capture summarised in
    # profiles/ls2d_warp_kernels_256x32_fp64.md; scaled by voxels for other
    # batch sizes or grids (the traffic per voxel does not depend on them)
    traffic = 242.4e6 * (N * B) / (32 * 256 * 256)
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "traffic_source": "ncu capture, profiles/ls2d_warp_kernels_256x32_fp64.md",
            "kernel": "ls2d_row_fast_kernel<double,256,true,true> (C2R + update + tau + R2C along y) over the batch",
            "peak_kind": peak_kind, "bytes_per_launch": row_bytes,
            "kernels_us": {"row_fp64": row64 * 1e3, "col_fp64": col64 * 1e3, "row_fp32": row32 * 1e3,
                           "col_fp32": col32 * 1e3},
            "col_fp64_frac": 48.0 * N * B / (col64 * 1e-3) / 1e9 / peak,
            "row_fp32_frac": 68.0 * N * B / (row32 * 1e-3) / 1e9 / peak}
    finite_strain = None
    if world == 1 and a.fs_grid > 0:
        finite_strain = run_finite_strain(a.fs_grid, peak)
    kmc = None
    if world == 1 and a.kmc_events > 0:
        kmc = run_kmc(a.kmc_events)
    landau = run_landau() if world == 1 and a.landau else None
    ensemble = None
    if world == 1 and a.ensemble > 0:
        from mgkmc_b200.serving import ensemble_requests, run_ensemble
        reqs = ensemble_requests(n_replicas=a.ensemble, n_events=500)
        _, ensemble = run_ensemble(reqs)
        ensemble["workload"] = (f"{a.ensemble} 2D KMC/AQS replicas, sides uniform in {{128,192,256,384,512}}, "
                                f"T uniform in [200, 400] K, seeds 0..{a.ensemble - 1}, 500 events each, mixed form, "
                                f"one batched solve launch per size per round, the sizes on their own streams")
        if a.ensemble_ragged:
            _, rag = run_ensemble(reqs, ragged=True)
            rag["workload"] = "the same replicas in one ragged plan: one launch per solver stage for all replicas"
            ensemble["ragged"] = rag
    serving = None
    if world == 1 and a.serve_window > 0:
        serving = run_serving(a.serve_window, a.serve_plain)
    cpu = None
    cpu_other = None
    if world == 1:
        from threadpoolctl import threadpool_limits
        host = host_cpu()
        with threadpool_limits(1):
            if a.cpu_seconds > 0:
                v, nsol, wall = cpu_ls_baseline(a.cpu_seconds)
                cpu = {"value": v, "unit": "solves/s", "cores": 1, "kind": "port",
                       "sample": f"{nsol} oracle solves of the {NX}^2 problem (tol {TOL:g}) in {wall:.1f} s, "
                                 f"numpy FFT, one thread", "host": host}
            cpu_other = {}
            if a.cpu_kmc_seconds > 0:
                ts, tr, nev, nsol = cpu_kmc_sample(a.cpu_kmc_seconds)
                d = {"kind": "port", "cores": 1, "s_per_ls_solve": ts, "s_per_rate_step": tr,
                     "sample": f"{nev} events of the oracle's per-event loop at 256^2 x 8 (barriers, rates with the "
                               f"sequential total, selection, flip with redraws, cold LS re-solve at tol 1e-6) "
                               f"from a state pre-strained to 2.4 %, {nsol} LS solves"}
                if kmc is not None:
                    # the same trajectory's solve and rate-step counts at the CPU's per-unit costs
                    pk = kmc["plain_fp64_exact"]
                    cpu_s = pk["solves"] * ts + (pk["aqs_steps"] + pk["events"]) * tr
                    d["events_per_s_estimate"] = pk["events"] / cpu_s
                    d["estimate"] = (f"{pk['solves']} LS solves x {ts:.3f} s + {pk['aqs_steps'] + pk['events']} "
                                     f"rate steps x {tr:.4f} s (the GPU trajectory's counts)")
                cpu_other["kmc_256x256x8"] = d
            if a.cpu_fs_grid > 0:
                n = a.cpu_fs_grid
                s = cpu_fs_sample(n)
                scale = (128.0 / n) ** 3 * np.log(128.0 ** 3) / np.log(float(n) ** 3)
                cpu_other["finite_strain_128"] = {
                    "kind": "port", "cores": 1, "seconds_per_load_step_sample": s,
                    "seconds_per_load_step_128_estimate": s * scale,
                    "sample": f"the first load step (F_xx = 1.005) at {n}^3, Neo-Hookean + 2 % F_p, Newton 1e-8, "
                              f"CG 1e-6; scaled to 128^3 by N log N ({scale:.1f}x)"}
    line = {"metric": METRIC, "value": rate[head], "unit": "solves/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms[head] / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "mixed fp32/fp64 (FP32 bulk iterations, FP64 finish, norms and sums)",
            "data": "synthetic (seeded; the benchmark material and sizes, no dataset)", "config": headline_config(a, world),
            "forms": {"solves_per_s": rate,
                      "speedup_vs_plain_fp64": rate[head] / rate["plain_fp64"] if "plain_fp64" in rate else None,
                      "iters_mean": {k: float(np.mean(v)) for k, v in iters.items()},
                      "mixed_field_err_vs_fp64": err_mixed, "mixed_residual": residual},
            "e2e": {"value": e2e_val, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "api": "mgkmc_b200.linear_elastic_simulator.Ls2dBatch",
                    "pipelining": "three plans on three streams, steps in turn", "host_result_err": e2e_err},
            "gpu_launches": gpu_launches, "roofline": roof, "cpu_baseline": cpu, "cpu_baselines_other": cpu_other,
            "clocks": clocks, "finite_strain": finite_strain, "kmc": kmc, "landau": landau, "serving": serving,
            "ensemble": ensemble}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_profile_case(a):
    """One workload whose kernels an ncu capture looks at; prints one line."""
    import torch
    from mgkmc_b200 import workloads as W
    n, prec = a.profile_n, a.profile_precision
    dev = torch.device("cuda", 0)
    if a.profile_case == "landau":
        for _ in range(3):
            solve_ms, iters, _ = _landau_device(n, 5, reps=1)
        print(f"landau {n}^2 depth 5: {iters} iterations, {solve_ms:.3f} ms", flush=True)
    elif a.profile_case == "ls3d":
        from mgkmc_b200.linear_elastic_simulator import Ls3dBatch
        rng = np.random.default_rng(21)
        E, nu = W.ls3d_material(n, n, n, rng)
        ep = W.pure_shear_eigenstrain_3d(n, n, n, rng)
        t = lambda x: torch.from_numpy(np.ascontiguousarray(x)).to(dev)
        eb = np.zeros((3, 3))
        eb[0, 0], eb[1, 2] = 0.01, 0.002
        B = Ls3dBatch([(n, n, n)], precision=prec)
        B.set_material(0, t(E), t(nu), t(ep))
        o = torch.empty((n, n, n, 3, 3), dtype=torch.float64, device=dev)
        s = torch.empty_like(o)
        for _ in range(3):
            info = B.solve([0], [eb], [o], [s], max_iter=300, tol=1e-8)
        print(f"ls3d {n}^3 {prec}: {info[0].iterations} iterations", flush=True)
    elif a.profile_case == "fs3d":
        from mgkmc_b200.finite_strain_simulator import Fs3dSolver
        lam, mu, Fp = W.fs3d_material_dev(n, n, n, 2, dev)
        S = Fs3dSolver(n, n, n, model="neo_hookean", precision=prec)
        S.set_material(lam, mu, Fp)
        S.set_F(torch.eye(3, dtype=torch.float64, device=dev).reshape(3, 3, 1, 1, 1).expand(3, 3, n, n, n).contiguous())
        Fb = np.eye(3)
        Fb[0, 0] = 1.005
        Pm = np.zeros((3, 3), bool)
        Pm[1, 1] = Pm[2, 2] = True
        _, info = S.step(Fb, (0, 0), np.zeros((3, 3)), Pm, 90e9, 0.35, 1e-8, 1e-6, 50, 1e6, 20)
        print(f"fs3d {n}^3 {prec}: {info.newton_iterations} Newton, {info.krylov_iterations} Krylov", flush=True)
    else:
        from mgkmc_b200 import kmc_simulator_functions as K
        rng = np.random.default_rng(1)
        cat, Q0 = W.kmc2d_state(n, n, 8, rng)
        sig = 1e8 * rng.standard_normal((n, n, 2, 2))
        Q = np.zeros((n, n, 8))
        soft, tl, prev = np.zeros((n, n, 2)), np.full((n, n), -np.inf), np.zeros((n, n, 2, 2))
        for _ in range(3):
            K.compute_barrier_2d(Q, Q0, sig, cat, 1.0, soft, tl, 0.0, prev, 2.0, 0, np.inf)
            r, idx, total = K.compute_rates_2d(Q, 1.0, 300.0, 1e13, cascade_mode=False)
            e = K.select_event_2d_u(r, total, 0.37)
        print(f"kmc {n}^2 x 8: total rate {total:.6e}, event {e}", flush=True)
    torch.cuda.synchronize()


def main():
    a = parse()
    if a.profile_case:
        run_profile_case(a)
        return
    if a.serve_only:
        # one serving-block line (no headline): for long windows of the stream
        import torch
        torch.cuda.set_device(0)
        clk = ClockSampler(0)
        clk.start()
        out = run_serving(a.serve_window, a.serve_plain, progress=30.0)
        out["clocks"] = clk.stop()
        print(json.dumps({"serving": out}), flush=True)
        return
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
