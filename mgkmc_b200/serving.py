"""Continuous-batching server for mechanical-equilibrium work on one GPU.

A request is one of
  * a 2D small-strain equilibrium solve: the mixed-BC macro loop of
    mgkmc/linear_elastic_simulator.py:176-197 (eps_xx prescribed, the other
    mean stresses driven to zero) around LS solves, on a grid with the
    heterogeneous medium and pure-shear eigenstrains of the benchmark's first
    workload;
  * a 2D KMC/AQS trajectory of ``n_events`` STZ events (the driver of
    mgkmc/kmc_simulator.py:796-1157 as run by ``Kmc2D``), material and barrier
    model of the 256^2 KMC workload;
  * a 3D finite-strain load step (the Newton-Krylov step of
    mgkmc/finite_strain_simulator.py:2967-3168, Neo-Hookean with eigen-
    deformations, F_xx = 1 + ``fs_strain`` prescribed, lateral stresses zero);
  * a 3D KMC/AQS trajectory of ``n_events`` events (the small-strain path of
    ThermalSimulation.run_simulation, mgkmc/aqs.py:682-1201, as run by
    ``Kmc3D``): the 2D trajectory's medium, catalog and barrier model in 3D.
    A finite-strain trajectory would need thousands of Newton load steps per
    request (one per AQS step, aqs.py:1097, plus the sub-stepped flips), so
    3D trajectories use the small-strain solver, the reference's default
    strain assumption.

Each request's inputs are generated on the GPU from its seed.

Served form (``Server(mode="served")``): requests are admitted as they arrive
while a slot of their grid size is free and the device-memory footprint of
the admitted work stays under ``hbm_budget``; 2D work sits in per-size plans
(``Ls2dBatch`` slots, one CUDA stream each) and advances in rounds: every
round resumes each admitted request until it needs a device result (a solve
or a synchronisation), then runs all the solves of that size in ONE batched
call (one launch per stage, loop on the device) and records an event; a
size's next round starts as soon as its event completes, independently of the
other sizes, so the work of different sizes overlaps on the device.  Solves
use the mixed-precision form and warm starts from the device-resident fields
(the previous macro iterate, or the trajectory's previous field).  Single
solves and trajectories of a size have separate plans, the solves' on
high-priority streams, so that a solve's kernels are scheduled ahead of the
long trajectory work at kernel boundaries.  3D finite-strain steps run on one
worker thread per size with its own high-priority stream; 3D trajectories on
one worker thread per size that advances them in rounds over a batched 3D LS
plan (one solve launch per stage for every admitted trajectory of the size);
all of it overlaps with the 2D work.

Sequential form (``mode="sequential"``): the plain FP64 form of the same
requests one at a time in arrival order, cold LS starts and the exact
sequential rate sum (the reference's arithmetic).

Latency = completion time - arrival time on the host clock (perf_counter),
with arrivals replayed in real time; a request that arrives while the server
is busy waits, and that wait is part of its latency.
"""
import collections
import queue
import sys
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import workloads as W

SIZES_2D = (64, 128, 256, 512, 768, 1024)
_TUNED = {}  # (side, slots, precision) -> (kernel family, ms per iteration) chosen by the LS autotuner
SIZES_3D = (64, 96, 128)


@dataclass
class Request:
    rid: int
    t_arrival: float  # seconds from the start of the stream
    kind: str         # "solve" | "trajectory"
    dim: int          # 2 | 3
    n: int            # grid side
    seed: int
    T: float = None   # KMC temperature (K); None: the server's
    n_events: int = None  # events of a trajectory; None: the server's


def request_stream(rate=200.0, duration=60.0, seed=3, p_traj=0.4, p_3d=0.3, sizes_2d=SIZES_2D,
                   sizes_3d=SIZES_3D):
    """Poisson arrivals (exponential gaps of mean 1/rate) over ``duration``
    seconds; per request: kind (trajectory with probability p_traj), dimension
    (3D with probability p_3d), a side drawn uniformly from the sizes, and a
    seed."""
    rng = np.random.default_rng(seed)
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t > duration:
            return out
        kind = "trajectory" if rng.random() < p_traj else "solve"
        dim = 3 if rng.random() < p_3d else 2
        n = int(rng.choice(sizes_3d if dim == 3 else sizes_2d))
        out.append(Request(len(out), t, kind, dim, n, int(rng.integers(0, 2 ** 31 - 1))))


@dataclass
class Result:
    rid: int
    kind: str
    dim: int
    n: int
    t_arrival: float
    t_admit: float = 0.0
    t_done: float = 0.0
    solves: int = 0
    ls_iterations: int = 0
    error: str = ""
    out: dict = field(default_factory=dict)

    @property
    def latency(self):
        return self.t_done - self.t_arrival


def footprint_bytes(req, n_modes=8):
    """Device bytes a request holds while admitted (its own tensors; the
    per-size plan slots are allocated once)."""
    if req.dim == 3 and req.kind == "trajectory":
        return req.n ** 3 * 8 * (2 + 9 * n_modes + 4 * n_modes + 9 + 4 + 1 + 9 + 27)
    if req.dim == 3:
        return req.n ** 3 * 8 * (83 + 9 + 2 + 27)
    N = req.n * req.n
    if req.kind == "solve":
        return N * 8 * (2 + 4 + 4 + 4)
    return N * 8 * (2 + 4 * n_modes + 3 * n_modes + 4 + 2 + 1 + 4 + 12 + 3 * n_modes)


class _Task:
    __slots__ = ("req", "res", "gen", "send", "need", "slot", "bytes")

    def __init__(self, req, res, gen, slot, nbytes):
        self.req, self.res, self.gen, self.slot, self.bytes = req, res, gen, slot, nbytes
        self.send = None
        self.need = None


class _Bucket:
    """A batched 2D LS plan with a stream: ``slots`` replicas of side n, or
    one replica per entry of ``sizes`` (a ragged bucket: replicas of several
    sides advance in one launch per solver stage)."""

    def __init__(self, torch, n, slots, precision, sizes=None, priority=0):
        from .linear_elastic_simulator import Ls2dBatch
        self.n = n
        self.sizes = list(sizes) if sizes is not None else [n] * slots
        self.stream = torch.cuda.Stream(priority=priority)
        self.plan = Ls2dBatch([(m, m) for m in self.sizes], precision=precision)
        self.free_by = {}
        for idx in range(len(self.sizes) - 1, -1, -1):
            self.free_by.setdefault(self.sizes[idx], []).append(idx)
        self.tasks = []        # admitted tasks
        self.waiting = collections.deque()
        self.inflight = None   # tasks of the running round
        self.solving = []
        self.event = torch.cuda.Event()

    def has_free(self, n):
        return bool(self.free_by.get(n))

    def take(self, n):
        return self.free_by[n].pop()

    def give(self, slot):
        self.free_by[self.sizes[slot]].append(slot)

    def nfree(self, n):
        return len(self.free_by.get(n, ()))


class _Bucket3:
    """One 3D grid size of trajectories: a batched 3D LS plan and a stream."""

    def __init__(self, torch, n, slots, precision):
        from .linear_elastic_simulator import Ls3dBatch
        self.n = n
        self.stream = torch.cuda.Stream()
        self.plan = Ls3dBatch([(n, n, n)] * slots, precision=precision)
        self.free = list(range(slots))[::-1]
        self.tasks = []


def _by_tol(tasks):
    """[(tol, tasks solved at tol)] in first-seen order."""
    groups = {}
    for t in tasks:
        groups.setdefault(t.need[5], []).append(t)
    return list(groups.items())


class Server:
    def __init__(self, mode="served", hbm_budget=None, slots=None, ls_tol=1e-8, ls_max_iter=500,
                 macro_tol=1e4, macro_max_iter=20, n_events=100, n_modes=8, q_mean=1.0, kmc_T=300.0,
                 fs_strain=0.005, fs_tol_nw=1e-8, fs_tol_cg=1e-6, selection=None, device=None, traj_ls_tol=1e-6,
                 ragged=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
        self.torch = torch
        self.mode = mode
        self.served = mode == "served"
        self.dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.precision = "mixed" if self.served else "fp64"
        self.ls_start = "warm" if self.served else "cold"
        self.selection = selection or ("fast" if self.served else "exact")
        # single solves at ls_tol; a trajectory's re-solves at the KMC driver's
        # spectral_solver_2d default tolerance (kmc_simulator.py:134, :517 pass
        # no tol; linear_elastic_simulator.py:13)
        self.ls_tol, self.ls_max_iter, self.traj_ls_tol = ls_tol, ls_max_iter, traj_ls_tol
        self.macro_tol, self.macro_max_iter = macro_tol, macro_max_iter
        self.n_events, self.n_modes, self.q_mean, self.kmc_T = n_events, n_modes, q_mean, kmc_T
        self.fs_strain, self.fs_tol_nw, self.fs_tol_cg = fs_strain, fs_tol_nw, fs_tol_cg
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.dev)
            hbm_budget = int(0.5 * free)
        self.hbm_budget = hbm_budget
        self.slots = dict(slots) if slots else {64: 32, 128: 32, 256: 32, 512: 16, 768: 8, 1024: 8}
        self.slots3 = {64: 8, 96: 4, 128: 2}
        # ragged: sides of the slots of one bucket shared by every 2D request
        # (None: one bucket per side)
        self.ragged = list(ragged) if ragged is not None else None
        self.buckets = {}
        self.buckets3 = {}
        self.fs_plans = {}
        self.used = 0
        self.lock = threading.Lock()
        self.progress = None  # seconds between progress lines on stderr (None: quiet)
        self._last_report = 0.0

    def _report(self, tag):
        if self.progress is None:
            return
        now = self._now()
        if now - self._last_report < self.progress:
            return
        self._last_report = now
        done = sum(1 for r in self.results.values() if r.t_done > 0)
        print(f"[{tag}] t = {now:.0f} s: {done} / {len(self.results)} requests done", file=sys.stderr, flush=True)

    # ------------------------------------------------------------ helpers ---
    def _now(self):
        return time.perf_counter() - self._t0

    def _prepare_ragged(self):
        """The ragged bucket: the kernel family picked by timing one replica
        of each side, then one solve of those (graph set-up)."""
        torch = self.torch
        b = self._bucket(None)
        with torch.cuda.stream(b.stream):
            reps, ebs, outs = [], [], []
            for n in sorted(set(b.sizes)):
                r = b.sizes.index(n)
                E, nu, ep, eb = W.ls2d_problem_dev(n, n, 0, self.dev)
                b.plan.set_material(r, E, nu, ep, stream=b.stream)
                reps.append(r)
                ebs.append(eb)
                outs.append(torch.empty((n, n, 2, 2), dtype=torch.float64, device=self.dev))
            key = ("ragged", tuple(b.sizes), self.precision)
            if key not in _TUNED:
                _TUNED[key] = b.plan.autotune(reps, ebs, stream=b.stream)
            else:
                b.plan.set_family(_TUNED[key][0])
            b.plan.solve(reps, ebs, outs, [None] * len(reps), max_iter=self.ls_max_iter, tol=self.ls_tol,
                         sync=True, stream=b.stream)

    def _bucket(self, n, kind="trajectory"):
        """The 2D bucket of side n: in the served form single solves and
        trajectories have separate buckets, the solves' on a high-priority
        stream (a solve's few kernels are scheduled ahead of the long
        trajectory and 3D work at kernel boundaries); one bucket per side in
        the sequential form."""
        if self.ragged is not None:  # one bucket for every 2D request
            b = self.buckets.get("ragged")
            if b is None:
                b = self.buckets["ragged"] = _Bucket(self.torch, 0, 0, self.precision, sizes=self.ragged)
            return b
        key = (n, kind) if self.served else n
        b = self.buckets.get(key)
        if b is None:
            k = self.slots.get(n, 4) if self.served else 1
            prio = -1 if self.served and kind == "solve" else 0
            b = self.buckets[key] = _Bucket(self.torch, n, k, self.precision, priority=prio)
        return b

    def _finish(self, res, out=None, error=""):
        res.t_done = self._now()
        res.error = error
        if out:
            res.out.update(out)

    # ----------------------------------------------------------- 2D tasks ---
    def _solve_task(self, b, slot, req, res):
        """Mixed-BC macro loop of one equilibrium solve (generator)."""
        torch = self.torch
        n = req.n
        E, nu, ep, eb = W.ls2d_problem_dev(n, n, req.seed, self.dev)
        b.plan.set_material(slot, E, nu, ep, stream=b.stream)
        eps = torch.empty((n, n, 2, 2), dtype=torch.float64, device=self.dev)
        sig = torch.empty_like(eps)
        strain_mask = np.array([[True, False], [False, False]])
        stress_mask = ~strain_mask
        target = np.zeros((2, 2))
        target[0, 0] = eb[0, 0]
        # means for the macro update, copied without a synchronisation; read
        # after the first solve has completed
        means = torch.empty(2, dtype=torch.float64).pin_memory()
        means.copy_(torch.stack([E.mean(), nu.mean()]), non_blocking=True)
        E_avg = nu_avg = None
        eps_bar = np.zeros((2, 2))
        warm = False
        sigM = None
        for _ in range(self.macro_max_iter):
            eps_bar[strain_mask] = target[strain_mask]
            info = yield ("solve", eps_bar.copy(), eps, sig, eps if warm else None, self.ls_tol)
            warm = self.ls_start == "warm"
            res.solves += 1
            res.ls_iterations += info.iterations
            sigM = np.array(info.sig_mean).reshape(2, 2)
            if E_avg is None:
                E_avg, nu_avg = float(means[0]), float(means[1])
            err = np.zeros((2, 2))
            err[stress_mask] = target[stress_mask] - sigM[stress_mask]
            if np.max(np.abs(err[stress_mask])) < self.macro_tol:
                break
            d_eps = (err - nu_avg * np.trace(err) * np.eye(2)) / E_avg
            eps_bar[stress_mask] += d_eps[stress_mask]
        return dict(eps=eps, sig=sig, eps_bar=eps_bar.copy(), sig_mean=sigM, E=E, nu=nu, ep=ep)

    def _traj_task(self, b, slot, req, res):
        """A KMC/AQS trajectory of n_events events (generator)."""
        from .kmc import Kmc2D
        n, M = req.n, self.n_modes
        E, nu, _, _ = W.ls2d_problem_dev(n, n, req.seed, self.dev)
        cat, Q0 = W.kmc2d_state_dev(n, n, M, req.seed, self.dev, q_mean=self.q_mean)
        k = Kmc2D(E, nu, cat, Q0, T=self.kmc_T if req.T is None else req.T, q_mean=self.q_mean, ls_tol=self.traj_ls_tol,
                  ls_max_iter=self.ls_max_iter, selection=self.selection, ls_start=self.ls_start,
                  precision=self.precision, ls=b.plan, rep=slot, stream=b.stream)
        rng = np.random.default_rng(req.seed)
        gen = k.trajectory(rng, 10 ** 9, max_events=self.n_events if req.n_events is None else req.n_events)
        send = None
        while True:
            try:
                need = gen.send(send)
            except StopIteration as stop:
                out = stop.value
                res.solves = k.n_solves
                return dict(events=out["events"], eps_macro=out["eps_macro"], eps=k.eps, sig=k.sig,
                            eps_p=k.eps_p, time=out["time"], steps=out["steps"])
            if need[0] == "solve":
                _, _, eb, eo, so, init = k.solve_args()
                info = yield ("solve", eb, eo, so, init, self.traj_ls_tol)
                res.ls_iterations += info.iterations
                send = info
            else:
                yield ("sync",)
                send = None

    # ----------------------------------------------------- 3D trajectories ---
    def _bucket3(self, n):
        b = self.buckets3.get(n)
        if b is None:
            k = self.slots3.get(n, 1) if self.served else 1
            b = self.buckets3[n] = _Bucket3(self.torch, n, k, self.precision)
        return b

    def _traj3_task(self, b, slot, req, res):
        """A 3D KMC/AQS trajectory of n_events events (generator, as _traj_task)."""
        from .kmc3d import Kmc3D
        n, M = req.n, self.n_modes
        E, nu = W.ls3d_material_dev(n, n, n, req.seed, self.dev)
        cat, Q0 = W.kmc3d_state_dev(n, n, n, M, req.seed, self.dev, q_mean=self.q_mean)
        k = Kmc3D(E, nu, cat, Q0, T=self.kmc_T if req.T is None else req.T, q_mean=self.q_mean,
                  ls_tol=self.traj_ls_tol,
                  ls_max_iter=self.ls_max_iter, selection=self.selection, ls_start=self.ls_start,
                  precision=self.precision, ls=b.plan, rep=slot, stream=b.stream)
        k.host_result = False
        del E, nu, cat, Q0
        gen = k.trajectory(np.random.default_rng(req.seed), 10 ** 9,
                           max_events=self.n_events if req.n_events is None else req.n_events)
        send = None
        while True:
            try:
                need = gen.send(send)
            except StopIteration as stop:
                out = stop.value
                res.solves = k.n_solves
                return dict(events=out["events"], eps_macro=out["eps_macro"], eps=k.eps, sig=k.sig,
                            eps_p=k.eps_p, time=out["time"], steps=out["steps"])
            if need[0] == "solve":
                _, _, eb, eo, so, init = k.solve_args()
                info = yield ("solve", eb, eo, so, init, self.traj_ls_tol)
                res.ls_iterations += info.iterations
                send = info
            else:
                yield ("sync",)
                send = None

    def _round3(self, b):
        """One round of a 3D bucket: resume every trajectory until it needs a
        device result, then one batched solve of all of them."""
        torch = self.torch
        solving, syncing, alive = [], [], []
        with torch.cuda.stream(b.stream):
            for t in b.tasks:
                try:
                    t.need = t.gen.send(t.send)
                except StopIteration as stop:
                    self._finish(t.res, stop.value)
                    b.free.append(t.slot)
                    continue
                except ValueError as e:
                    self._finish(t.res, error=str(e))
                    b.free.append(t.slot)
                    continue
                alive.append(t)
                (solving if t.need[0] == "solve" else syncing).append(t)
        b.tasks = alive
        for tol, group in _by_tol(solving):
            infos = b.plan.solve([t.slot for t in group], [t.need[1] for t in group],
                                 [t.need[2] for t in group], [t.need[3] for t in group],
                                 eps_init=[t.need[4] for t in group], max_iter=self.ls_max_iter, tol=tol,
                                 sync=True, stream=b.stream)
            for t, info in zip(group, infos):
                t.send = info
        if syncing:
            b.stream.synchronize()
            for t in syncing:
                t.send = None

    def _traj3_worker(self, q):
        """Admits the 3D trajectories of its queue into free slots of their
        size and advances the admitted ones in rounds until the queue is
        closed and all are done.  A worker advances only the buckets its own
        requests went to."""
        waiting = collections.deque()
        mine = []
        closed = False
        while True:
            try:
                while True:
                    r = q.get_nowait()
                    if r is None:
                        closed = True
                    else:
                        waiting.append(r)
            except queue.Empty:
                pass
            still = collections.deque()
            for r in waiting:
                b = self._bucket3(r.n)
                if b not in mine:
                    mine.append(b)
                if b.free:
                    res = self.results[r.rid]
                    res.t_admit = self._now()
                    slot = b.free.pop()
                    with self.torch.cuda.stream(b.stream):
                        gen = self._traj3_task(b, slot, r, res)
                    b.tasks.append(_Task(r, res, gen, slot, 0))
                else:
                    still.append(r)
            waiting = still
            active = [b for b in mine if b.tasks]
            if not active:
                if closed and not waiting:
                    return
                r = q.get()
                if r is None:
                    closed = True
                else:
                    waiting.append(r)
                continue
            for b in active:
                self._round3(b)

    def _admit(self, b, req):
        res = self.results[req.rid]
        nbytes = footprint_bytes(req, self.n_modes)
        slot = b.take(req.n)
        self.used += nbytes
        res.t_admit = self._now()
        with self.torch.cuda.stream(b.stream):
            gen = (self._solve_task if req.kind == "solve" else self._traj_task)(b, slot, req, res)
        b.tasks.append(_Task(req, res, gen, slot, nbytes))

    def _release(self, b, t):
        b.give(t.slot)
        self.used -= t.bytes

    def _start_round(self, b):
        torch = self.torch
        solving, alive = [], []
        with torch.cuda.stream(b.stream):
            for t in b.tasks:
                try:
                    t.need = t.gen.send(t.send)
                except StopIteration as stop:
                    self._finish(t.res, stop.value)
                    self._release(b, t)
                    continue
                except ValueError as e:
                    self._finish(t.res, error=str(e))
                    self._release(b, t)
                    continue
                alive.append(t)
                if t.need[0] == "solve":
                    solving.append(t)
        b.tasks = alive
        for tol, group in _by_tol(solving):  # one launch per tolerance in use
            b.plan.solve([t.slot for t in group], [t.need[1] for t in group], [t.need[2] for t in group],
                         [t.need[3] for t in group], eps_init=[t.need[4] for t in group],
                         max_iter=self.ls_max_iter, tol=tol, sync=False, stream=b.stream)
        b.solving = solving
        b.inflight = list(alive)  # tasks admitted during the round join the next one
        b.event.record(b.stream)

    def _complete_round(self, b):
        if b.solving:
            infos = b.plan.collect([t.slot for t in b.solving], stream=b.stream)
            for t, info in zip(b.solving, infos):
                t.send = info
        for t in b.inflight:
            if t.need[0] == "sync":
                t.send = None
        b.inflight = None
        b.solving = []

    # ----------------------------------------------------------- 3D tasks ---
    def _fs_plan(self, n):
        from .finite_strain_simulator import Fs3dSolver
        s = self.fs_plans.get(n)
        if s is None:
            s = self.fs_plans[n] = Fs3dSolver(n, n, n, model="neo_hookean", precision=self.precision)
        return s

    def _fs_run(self, req, stream):
        """One finite-strain load step; returns the result dict."""
        from .finite_strain_simulator import build_finite_strain_bc_3d
        torch = self.torch
        n = req.n
        s = self._fs_plan(n)
        with torch.cuda.stream(stream):
            lam, mu, Fp = W.fs3d_material_dev(n, n, n, req.seed, self.dev)
            E = mu * (3 * lam + 2 * mu) / (lam + mu)
            nu = lam / (2 * (lam + mu))
            F0 = torch.zeros((3, 3, n, n, n), dtype=torch.float64, device=self.dev)
            for i in range(3):
                F0[i, i] = 1.0
            s.set_material(lam, mu, Fp, stream=stream)
            s.set_F(F0, stream=stream)
            Fb, _, Pt, Pm = build_finite_strain_bc_3d((0, 0), self.fs_strain, {(1, 1): 0.0, (2, 2): 0.0})
            Fbo, info = s.step(Fb, (0, 0), Pt, Pm, float(E.mean()), float(nu.mean()), self.fs_tol_nw,
                               self.fs_tol_cg, 50, 1e6, 20, stream=stream)
            Fo = torch.empty_like(F0)
            Po = torch.empty_like(F0)
            s.get(Fo, Po, None, stream=stream)
            stream.synchronize()
        return dict(F=Fo, P=Po, F_bar=Fbo, sig_mean=np.array(info.sig_mean).reshape(3, 3),
                    newton=info.newton_iterations, krylov=info.krylov_iterations)

    def _fs_worker(self, q, stream):
        while True:
            req = q.get()
            if req is None:
                return
            res = self.results[req.rid]
            res.t_admit = self._now()
            try:
                out = self._fs_run(req, stream)
                res.solves = 1
                self._finish(res, out)
            except (ValueError, RuntimeError) as e:
                self._finish(res, error=str(e))

    # ---------------------------------------------------------------- run ---
    def prepare(self, requests):
        """Creates the plans the requests will use and runs one solve on each,
        so that plan set-up and graph instantiation happen before the first
        arrival (a server is started before its traffic)."""
        torch = self.torch
        if self.ragged is not None:
            self._prepare_ragged()
        for n, kind in sorted({(r.n, r.kind) for r in requests if r.dim == 2} if self.ragged is None else ()):
            b = self._bucket(n, kind)
            with torch.cuda.stream(b.stream):
                E, nu, ep, eb = W.ls2d_problem_dev(n, n, 0, self.dev)
                eps = torch.empty((n, n, 2, 2), dtype=torch.float64, device=self.dev)
                nf = b.nfree(n)
                for k in range(min(4, nf)):
                    b.plan.set_material(k, E, nu, ep, stream=b.stream)
                k = min(4, nf)
                if self.served:
                    # kernel family picked by measurement, once per (side, slots, precision)
                    key = (n, nf, self.precision)
                    if key not in _TUNED:
                        _TUNED[key] = b.plan.autotune(list(range(k)), [eb] * k, stream=b.stream)
                    else:
                        b.plan.set_family(_TUNED[key][0])
                for k in range(1, min(4, nf) + 1):
                    b.plan.solve(list(range(k)), [eb] * k, [eps] * k, [None] * k, max_iter=self.ls_max_iter,
                                 tol=self.ls_tol, sync=True, stream=b.stream)
        for n in sorted({r.n for r in requests if r.dim == 3 and r.kind == "solve"}):
            self._fs_plan(n)
        for n in sorted({r.n for r in requests if r.dim == 3 and r.kind == "trajectory"}):
            b = self._bucket3(n)
            with torch.cuda.stream(b.stream):
                E, nu = W.ls3d_material_dev(n, n, n, 0, self.dev)
                eps = torch.empty((n, n, n, 3, 3), dtype=torch.float64, device=self.dev)
                eb = np.zeros((3, 3))
                eb[0, 0] = 0.01
                k = min(2, len(b.free))
                for r in range(k):
                    b.plan.set_material(r, E, nu, None, stream=b.stream)
                for r in range(1, k + 1):
                    b.plan.solve(list(range(r)), [eb] * r, [eps] * r, [None] * r, max_iter=self.ls_max_iter,
                                 tol=self.ls_tol, sync=True, stream=b.stream)
        torch.cuda.synchronize()

    def run(self, requests, realtime=True, keep_outputs=False):
        """Serve ``requests`` (arrival times relative to the start); returns
        the list of Results in request order."""
        self.results = {r.rid: Result(r.rid, r.kind, r.dim, r.n, r.t_arrival) for r in requests}
        order = sorted(requests, key=lambda r: r.t_arrival)
        if self.served:
            self._run_served(order, realtime)
        else:
            self._run_sequential(order, realtime)
        out = [self.results[r.rid] for r in requests]
        if not keep_outputs:
            for r in out:
                r.out = {k: v for k, v in r.out.items() if not hasattr(v, "data_ptr")}
        return out

    def _run_served(self, order, realtime):
        torch = self.torch
        pending = collections.deque(order)
        # one finite-strain worker per side, each with its plan and stream:
        # load steps of different sides overlap on the device
        fs_qs = {n: queue.Queue() for n in sorted({r.n for r in order if r.dim == 3 and r.kind == "solve"})}
        workers_fs = [threading.Thread(target=self._fs_worker, args=(q, torch.cuda.Stream(priority=-1)), daemon=True)
                      for q in fs_qs.values()]
        # one 3D-trajectory worker per side: a side's rounds (synchronous
        # batched solves) do not wait behind another side's
        t3_qs = {n: queue.Queue() for n in sorted({r.n for r in order if r.dim == 3 and r.kind == "trajectory"})}
        workers3 = [threading.Thread(target=self._traj3_worker, args=(q,), daemon=True) for q in t3_qs.values()]
        n3d = sum(1 for r in order if r.dim == 3)
        self._t0 = time.perf_counter()
        for w in workers_fs + workers3:
            w.start()
        done3d = lambda: sum(1 for r in self.results.values() if r.dim == 3 and r.t_done > 0)
        try:
            while True:
                now = self._now()
                while pending and (not realtime or pending[0].t_arrival <= now):
                    r = pending.popleft()
                    if not realtime:
                        self.results[r.rid].t_arrival = now
                    if r.dim == 3:
                        (t3_qs if r.kind == "trajectory" else fs_qs)[r.n].put(r)
                    else:
                        self._bucket(r.n, r.kind).waiting.append(r)
                progressed = False
                for b in self.buckets.values():
                    while b.waiting and b.has_free(b.waiting[0].n) and (self.used + footprint_bytes(b.waiting[0], self.n_modes)
                                                    <= self.hbm_budget or not b.tasks):
                        self._admit(b, b.waiting.popleft())
                    if b.inflight is not None and b.event.query():
                        self._complete_round(b)
                        progressed = True
                    if b.inflight is None and b.tasks:
                        self._start_round(b)
                        progressed = True
                self._report("served")
                busy = any(b.tasks or b.waiting or b.inflight for b in self.buckets.values())
                if not pending and not busy and done3d() == n3d:
                    break
                if not progressed:
                    if not busy and pending and realtime:
                        time.sleep(max(0.0, min(0.002, pending[0].t_arrival - self._now())))
                    else:
                        time.sleep(2e-5)
        finally:
            for q in list(fs_qs.values()) + list(t3_qs.values()):
                q.put(None)
            for w in workers_fs + workers3:
                w.join()

    def _run_sequential(self, order, realtime):
        torch = self.torch
        self._t0 = time.perf_counter()
        stream = torch.cuda.current_stream()
        for r in order:
            now = self._now()
            if realtime and r.t_arrival > now:
                time.sleep(r.t_arrival - now)
            res = self.results[r.rid]
            self._report("sequential")
            if not realtime:
                res.t_arrival = self._now()
            res.t_admit = self._now()
            try:
                if r.dim == 3 and r.kind == "solve":
                    out = self._fs_run(r, stream)
                    res.solves = 1
                else:
                    b = self._bucket(r.n) if r.dim == 2 else self._bucket3(r.n)
                    if r.dim == 3:
                        task = self._traj3_task
                    else:
                        task = self._solve_task if r.kind == "solve" else self._traj_task
                    gen = task(b, 0, r, res)
                    send = None
                    while True:
                        try:
                            # the request's own work (inputs, KMC kernels) on the plan's stream
                            with torch.cuda.stream(b.stream):
                                need = gen.send(send)
                        except StopIteration as stop:
                            out = stop.value
                            break
                        if need[0] == "solve":
                            send = b.plan.solve([0], [need[1]], [need[2]], [need[3]],
                                                eps_init=[need[4]], max_iter=self.ls_max_iter, tol=need[5],
                                                sync=True, stream=b.stream)[0]
                        else:
                            b.stream.synchronize()
                            send = None
                self._finish(res, out)
            except ValueError as e:
                self._finish(res, error=str(e))


def ensemble_requests(n_replicas=96, sizes=(128, 192, 256, 384, 512), T_range=(200.0, 400.0), n_events=500,
                      seed=0):
    """The batched KMC ensemble: replica k has seed k, a side drawn uniformly
    from `sizes` and a temperature uniform in `T_range`, all arriving at once."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_replicas):
        n = int(rng.choice(sizes))
        T = float(rng.uniform(*T_range))
        out.append(Request(k, 0.0, "trajectory", 2, n, k, T=T, n_events=n_events))
    return out


def run_ensemble(requests, slots=None, ragged=False, **server_kw):
    """Runs an ensemble through the served form (every replica admitted at
    once when slots allow) and returns (results, summary with events/s).
    ragged=False: one bucket per side, one batched solve launch per side per
    round, the sides' buckets on their own streams; True: one ragged bucket
    with a slot per replica, one launch per solver stage for all replicas of
    a round."""
    from collections import Counter
    cnt = Counter(r.n for r in requests)
    if ragged:
        server_kw["ragged"] = sorted(r.n for r in requests)
    srv = Server(mode="served", slots=slots or {n: c for n, c in cnt.items()}, **server_kw)
    srv.prepare(requests)
    t0 = time.perf_counter()
    res = srv.run(requests, realtime=False, keep_outputs=False)
    wall = time.perf_counter() - t0
    ok = [r for r in res if not r.error]
    events = sum(len(r.out.get("events", ())) for r in ok)
    solves = sum(r.solves for r in ok)
    return res, {"replicas": len(requests), "completed": len(ok), "events": events, "solves": solves,
                 "seconds": wall, "events_per_s": events / wall, "solves_per_s": solves / wall}


def summarize(results, window=None):
    """solves/s over the makespan, request latencies p50/p99 (seconds), by
    request class too."""
    ok = [r for r in results if not r.error and r.t_done > 0]
    if not ok:
        return dict(requests=len(results), completed=0)
    t_end = max(r.t_done for r in ok)
    t_start = min(r.t_arrival for r in results)
    solves = sum(r.solves for r in ok)
    lat = np.array([r.latency for r in ok])
    out = dict(requests=len(results), completed=len(ok), errors=len(results) - len(ok), solves=solves,
               makespan_s=t_end - t_start, solves_per_s=solves / max(t_end - t_start, 1e-9),
               requests_per_s=len(ok) / max(t_end - t_start, 1e-9),
               p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)))
    by = {}
    for key in sorted({(r.dim, r.kind) for r in ok}):
        l = np.array([r.latency for r in ok if (r.dim, r.kind) == key])
        by[f"{key[0]}d_{key[1]}"] = dict(n=int(l.size), p50_s=float(np.percentile(l, 50)),
                                         p99_s=float(np.percentile(l, 99)))
    out["by_class"] = by
    return out
