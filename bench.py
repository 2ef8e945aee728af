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
    ap.add_argument("--ensemble", type=int, default=0,
                    help="replicas of the batched KMC ensemble block (96 = the ensemble workload, ~1 min); 0 skips it")
    ap.add_argument("--serve-window", type=float, default=0.1,
                    help="seconds of the serving stream (Poisson 200 req/s, seed 3) replayed in the serving block; "
                         "0 skips it")
    ap.add_argument("--profile-case", default="", choices=["", "ls3d", "fs3d", "kmc"],
                    help="run one kernel-profiling workload instead of the benchmark (for ncu captures): ls3d = "
                         "LS 3D solves at --profile-n^3 (tol 1e-8, three solves), fs3d = one finite-strain load "
                         "step at --profile-n^3 (Neo-Hookean + 2 %% F_p, F_xx = 1.005), kmc = three rounds of "
                         "barrier, exact rates/total and selection at --profile-n^2 x 8 modes")
    ap.add_argument("--profile-n", type=int, default=128)
    ap.add_argument("--profile-precision", default="fp64", choices=["fp64", "mixed"])
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
            "config": {"workload": f"ls2d_{NX}_batched_mixed", "batch": a.batch, "grid": [NX, NY], "tol": TOL},
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


# ------------------------------------------------------------- serving -----
def run_serving(window):
    """The serving stream's first `window` seconds of arrivals, served by the
    continuous-batching server (mixed precision) and by the plain FP64 form one
    request at a time; arrivals replayed in real time."""
    from mgkmc_b200.serving import Server, request_stream, summarize
    reqs = [r for r in request_stream(rate=200.0, duration=60.0, seed=3) if r.t_arrival <= window]
    out = {"workload": (f"serving stream (Poisson 200 req/s, seed 3; 60 % equilibrium solves, 40 % 100-event KMC "
                        f"trajectories; 70 % 2D sides 64..1024, 30 % 3D finite-strain 64..128): the "
                        f"{len(reqs)} arrivals of its first {window:g} s, replayed in real time"),
           "requests": [[r.kind, r.dim, r.n] for r in reqs]}
    for name, mode in (("served_mixed", "served"), ("plain_fp64_sequential", "sequential")):
        srv = Server(mode=mode)
        srv.prepare(reqs)
        res = srv.run(reqs, realtime=True)
        out[name] = summarize(res)
    from mgkmc_b200 import serving as SV
    out["autotuned_ls_families"] = {f"{k[0]}^2 x{k[1]} {k[2]}": {"family": v[0], "ms_per_iteration": v[1]}
                                    for k, v in SV._TUNED.items()}
    a, b = out["served_mixed"], out["plain_fp64_sequential"]
    if a.get("completed") and b.get("completed"):
        out["solves_per_s_ratio"] = a["solves_per_s"] / b["solves_per_s"]
        out["p50_ratio"] = b["p50_s"] / a["p50_s"]
        out["p99_ratio"] = b["p99_s"] / a["p99_s"]
    return out


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
    if world > 1:
        t = torch.tensor([ms[k] for k in forms], device=dev)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        ms = {k: float(v) for k, v in zip(forms, t.tolist())}
    rate = {k: B * a.steps * world / (ms[k] / 1e3) for k in forms}
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
    ensemble = None
    if world == 1 and a.ensemble > 0:
        from mgkmc_b200.serving import ensemble_requests, run_ensemble
        _, ensemble = run_ensemble(ensemble_requests(n_replicas=a.ensemble, n_events=500))
        ensemble["workload"] = (f"{a.ensemble} 2D KMC/AQS replicas, sides uniform in {{128,192,256,384,512}}, "
                                f"T uniform in [200, 400] K, seeds 0..{a.ensemble - 1}, 500 events each, mixed form, "
                                f"one batched solve launch per size per round")
    serving = None
    if world == 1 and a.serve_window > 0:
        serving = run_serving(a.serve_window)
    cpu = None
    if world == 1 and a.cpu_seconds > 0:
        v, nsol, wall = cpu_baseline(a.cpu_seconds, 1)
        cpu = {"value": v, "unit": "solves/s", "cores": 1, "kind": "port",
               "sample": f"{nsol} oracle solves of the same {NX}^2 problem in {wall:.1f} s (numpy FFT, 1 thread)"}
    line = {"metric": METRIC, "value": rate[head], "unit": "solves/s", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms[head] / a.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, survey config)",
            "config": {"workload": f"ls2d_{NX}_batched_mixed", "batch": B, "grid": [NX, NY], "tol": TOL,
                       "l2": "flushed between steps (256 MB write)", "parallelism": f"replicas x{world}",
                       "forms_solves_per_s": rate,
                       "speedup_vs_plain_fp64": rate[head] / rate["plain_fp64"] if "plain_fp64" in rate else None,
                       "iters_mean": {k: float(np.mean(v)) for k, v in iters.items()},
                       "mixed_field_err_vs_fp64": err_mixed, "mixed_residual": residual},
            "e2e": {"value": e2e_val, "unit": "solves/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "api": "mgkmc_b200.linear_elastic_simulator.Ls2dBatch",
                    "pipelining": "three plans on three streams, steps in turn", "host_result_err": e2e_err},
            "gpu_launches": gpu_launches, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "finite_strain": finite_strain, "serving": serving, "ensemble": ensemble}
    print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def run_profile_case(a):
    """One workload whose kernels an ncu capture looks at; prints one line."""
    import torch
    from mgkmc_b200 import workloads as W
    n, prec = a.profile_n, a.profile_precision
    dev = torch.device("cuda", 0)
    if a.profile_case == "ls3d":
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
    if a.impl == "reference":
        run_reference(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
