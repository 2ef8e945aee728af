"""Device-resident 2D KMC/AQS driver.

Runs the trajectory of KmcSimulation2D.run_simulation
(mgkmc/kmc_simulator.py:796-1157) on the path the KMC benchmark exercises
(small-strain linear elasticity, KMC mode, optional cascade mode and fast
patching, no thermal conduction, redraw of directions and barriers) with every
field resident on the GPU: barriers, rates, the running rate sum, selection,
the flip bookkeeping and the LS re-solve never leave the device.  The host
keeps the clock, the macro strain and the random draws (one small
device-to-host read of the total rate per attempt, and of the mean stress
per solve).

Draw order (matches oracle/kmc_driver.py): per attempt u_wait; per event
u_sel, then M orientations theta ~ U[0, pi) and M barriers N(q_mean, q_std)
clipped below at q_min.

Selection modes: ``exact`` reproduces the reference's sequential FP64 rate
sum bit for bit (one dependent chain); ``fast`` uses a parallel scan whose
running sums differ by rounding.  LS forms: ``cold`` re-solves from eps_bar
as the reference does (kmc_simulator.py:517 passes no warm start); ``warm``
starts from the previous field.
"""
import numpy as np

from . import _lib as L
from .linear_elastic_simulator import Ls2dBatch

KB = 8.617e-5


def pure_shear_modes(theta, gamma0):
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    cat = np.empty(theta.shape + (2, 2))
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    return cat


class GeneratorDraws:
    """The driver's draws from an explicit numpy Generator, in a fixed order:
    per attempt u_wait; per event u_sel, then M orientations theta ~ U[0, pi)
    (pure-shear modes of amplitude gamma0/2) and M barriers N(q_mean, q_std)
    clipped below at q_min."""

    def __init__(self, rng, gamma0, q_mean, q_std, q_min):
        self.rng, self.gamma0, self.q = rng, gamma0, (q_mean, q_std, q_min)

    def u_wait(self):
        return self.rng.random()

    def u_sel(self):
        return self.rng.random()

    def catalog(self, M):
        return pure_shear_modes(self.rng.uniform(0.0, np.pi, M), self.gamma0)

    def q0(self, M):
        return np.clip(self.rng.normal(self.q[0], self.q[1], M), self.q[2], None)


class ReferenceDraws:
    """The reference simulator's draws, call for call, from a numpy
    RandomState standing for its global stream: t_wait = -ln(rand()) / total
    (kmc_simulator.py:893); the selection threshold uniform(0, total)
    (kmc_simulator_functions.py:62, taken here as u = U with r = u * total);
    the redrawn catalog of stz_catalog_glass_2d (:78-98: per mode
    gxx = 0.5 gamma0 N(0,1), then gxy, pure shear); the redrawn barriers of the
    Gaussian generator (:222-229: normal(mean, std, size=M) clipped)."""

    def __init__(self, rs, gamma0, mean, std, min_cutoff=None, max_cutoff=None):
        self.rs, self.gamma0 = rs, gamma0
        self.mean, self.std, self.lo, self.hi = mean, std, min_cutoff, max_cutoff

    def u_wait(self):
        return self.rs.rand()

    def u_sel(self):
        return self.rs.uniform(0.0, 1.0)

    def catalog(self, M):
        cat = np.zeros((M, 2, 2))
        for i in range(M):
            gxx = 0.5 * self.gamma0 * self.rs.normal()
            gxy = 0.5 * self.gamma0 * self.rs.normal()
            cat[i, 0, 0], cat[i, 1, 1] = gxx, -gxx
            cat[i, 0, 1] = cat[i, 1, 0] = gxy
        return cat

    def q0(self, M):
        b = self.rs.normal(loc=self.mean, scale=self.std, size=(M,))
        if self.lo is not None or self.hi is not None:
            b = np.clip(b, self.lo, self.hi)
        return b


class Kmc2D:
    def __init__(self, E, nu, catalog, Q0, gamma0=0.1, T=300.0, nu0=1e13, strain_rate=1e7, step_size=1e-5,
                 q_act_temp=0.37, jp=0.0, jt=0.0, cap=2.0, jn=0.0, stress_targets=None, mixed_tol=1e4,
                 mixed_max_iter=50, ls_tol=1e-6, ls_max_iter=200, q_mean=1.0, q_std=0.15, q_min=0.3, volume=1.0,
                 selection="exact", ls_start="cold", precision="fp64", ls=None, rep=0, stream=None,
                 cascade_mode=False, stability_threshold=0.0, max_cascade_steps_pct=0.3, fast_patching=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
        self.torch = torch
        d = self.dev = torch.device("cuda", torch.cuda.current_device())
        self.nx, self.ny, self.M = Q0.shape
        nx, ny, M = self.nx, self.ny, self.M
        self.p = dict(gamma0=gamma0, T=T, nu0=nu0, strain_rate=strain_rate, step_size=step_size, jp=jp, jt=jt,
                      cap=cap, jn=jn, mixed_tol=mixed_tol, mixed_max_iter=mixed_max_iter, ls_tol=ls_tol,
                      ls_max_iter=ls_max_iter, q_mean=q_mean, q_std=q_std, q_min=q_min, volume=volume)
        self.stress_targets = {(1, 1): 0.0} if stress_targets is None else dict(stress_targets)
        self.selection = selection
        # cascade mode (kmc_simulator.py:876-889, _run_cascade :577-794): flips of
        # unstable modes in batches; its rates keep only q > 0 modes, which the
        # exact (compacting) rate path provides
        if cascade_mode and selection != "exact":
            raise ValueError("cascade mode uses the exact selection (compacted rates)")
        self.cascade_mode = bool(cascade_mode)
        self.stability_threshold = float(stability_threshold)
        self.max_cascade_limit = int(max_cascade_steps_pct * self.nx * self.ny)
        self.cascade_flips = []
        self.ls_start = ls_start
        self.tau = 1.0 / (nu0 * np.exp(-q_act_temp / (KB * T))) if T > 0 else np.inf
        f64 = torch.float64
        self.stream = stream if stream is not None else torch.cuda.current_stream()

        def t(a):
            if isinstance(a, torch.Tensor):
                return a.to(device=d, dtype=torch.float64).contiguous()
            return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(d)
        self.E, self.nu = t(E), t(nu)
        # medium means for the mixed stress loop, copied without a
        # synchronisation (first read after a solve has completed)
        self._means_h = torch.empty(2, dtype=torch.float64).pin_memory()
        with torch.cuda.stream(self.stream):
            self._means_h.copy_(torch.stack([self.E.mean(), self.nu.mean()]), non_blocking=True)
        self.catalog, self.Q0 = t(catalog), t(Q0)
        self.eps_p = torch.zeros((nx, ny, 2, 2), dtype=f64, device=d)
        self.soft = torch.zeros((nx, ny, 2), dtype=f64, device=d)
        self.t_last = torch.full((nx, ny), -np.inf, dtype=f64, device=d)
        self.prev = torch.zeros((nx, ny, 2, 2), dtype=f64, device=d)
        self.Q = torch.zeros((nx, ny, M), dtype=f64, device=d)
        self.eps = torch.zeros((nx, ny, 2, 2), dtype=f64, device=d)
        self.sig = torch.zeros_like(self.eps)
        self.eps_prev = torch.zeros_like(self.eps)
        n = nx * ny * M
        self.rates = torch.empty(n, dtype=f64, device=d)
        self.indices = torch.empty(n, dtype=torch.int64, device=d)
        self.prefix = torch.empty(n, dtype=f64, device=d)
        self.count = torch.zeros(1, dtype=torch.int64, device=d)
        self.total = torch.zeros(1, dtype=f64, device=d)
        self.total_h = torch.zeros(1, dtype=f64).pin_memory()
        self.total_fast = torch.zeros(1, dtype=f64, device=d)  # fast mode: total of the fused rate pass
        self.sel = torch.zeros(1, dtype=torch.int64, device=d)
        self.xym = torch.zeros(3, dtype=torch.int64, device=d)
        self.xym_h = torch.zeros(3, dtype=torch.int64).pin_memory()
        self.redraw_h = torch.zeros(5 * M, dtype=f64).pin_memory()
        self.redraw = torch.zeros(5 * M, dtype=f64, device=d)
        self.work = torch.empty(max(int(L.lib().mgk_kmc_rates_work_bytes(n)), int(L.lib().mgk_kmc_scan_work_bytes(n))),
                                dtype=torch.uint8, device=d)
        if ls is None:
            self.ls, self.rep = Ls2dBatch([(nx, ny)], precision=precision), 0
        else:
            self.ls, self.rep = ls, int(rep)
        self.ls.set_material(self.rep, self.E, self.nu, self.eps_p, stream=self.stream)
        # fast patching (kmc_simulator.py:76-80, :170-171, :229-261): stress
        # patches and the unit macro-strain response, solved once
        self.fast = bool(fast_patching and fast_patching.get("enabled", False))
        if self.fast:
            self.R = int(fast_patching.get("patch_radius", 5))
            self.sync_interval = int(fast_patching.get("sync_interval", 100))
            self._setup_patches(getattr(self.ls, "precision", precision))
        self.flips_since_sync = 0
        self.unit_ready = False  # the reference computes the unit response at the first KMC flip
        self.eps_macro = np.zeros((2, 2))
        self.time = 0.0
        self.events = []
        self.n_solves = 0
        self.steps_done = 0
        self._resume = False  # set by load_state_dict: the fields are the state, no initial solve

    # ------------------------------------------------------- checkpoints ---
    _FIELDS = ("E", "nu", "eps", "sig", "eps_p", "soft", "Q", "Q0", "catalog", "t_last", "prev")

    def state_dict(self):
        """Host copies of the trajectory state between AQS steps (the fields,
        the clock, the macro strain, the event list and counters)."""
        self.stream.synchronize()
        st = {k: getattr(self, k).cpu().numpy() for k in self._FIELDS}
        st.update(eps_macro=self.eps_macro.copy(), time=self.time, events=list(self.events),
                  n_solves=self.n_solves, steps_done=self.steps_done, unit_ready=self.unit_ready,
                  flips_since_sync=self.flips_since_sync)
        return st

    def load_state_dict(self, st):
        """Restores a state from ``state_dict`` (same grid, modes and
        material); the next ``trajectory`` continues from it without the
        initial re-solve (the stored fields are that solve's result)."""
        torch = self.torch
        with torch.cuda.stream(self.stream):
            for k in self._FIELDS:
                getattr(self, k).copy_(torch.from_numpy(np.ascontiguousarray(st[k], dtype=np.float64)).to(self.dev))
        self.ls.set_eigenstrain(self.rep, self.eps_p, stream=self.stream)
        self.eps_macro = np.array(st["eps_macro"], dtype=np.float64).reshape(2, 2)
        self.time = float(st["time"])
        self.events = [tuple(e) for e in st["events"]]
        self.n_solves = int(st["n_solves"])
        self.steps_done = int(st["steps_done"])
        self.unit_ready = bool(st.get("unit_ready", False))
        self.flips_since_sync = int(st.get("flips_since_sync", 0))
        self._resume = True
        self.stream.synchronize()

    def _setup_patches(self, precision):
        """LS responses to unit eigenstrains [[1,0],[0,-1]] and [[0,1],[1,0]] at
        (nx//2, ny//2) under zero macro strain, and to the unit macro strain
        e_00 without eigenstrain (one batched solve of three replicas), then
        the windows and missing means on the device."""
        torch, d, f64 = self.torch, self.dev, self.torch.float64
        nx, ny = self.nx, self.ny
        with torch.cuda.stream(self.stream):
            ep = torch.zeros((3, nx, ny, 2, 2), dtype=f64, device=d)
            ep[0, nx // 2, ny // 2, 0, 0], ep[0, nx // 2, ny // 2, 1, 1] = 1.0, -1.0
            ep[1, nx // 2, ny // 2, 0, 1], ep[1, nx // 2, ny // 2, 1, 0] = 1.0, 1.0
        tmp = Ls2dBatch([(nx, ny)] * 3, precision=precision)
        for r in range(3):
            tmp.set_material(r, self.E, self.nu, ep[r], stream=self.stream)
        resp = torch.empty((3, nx, ny, 2, 2), dtype=f64, device=d)
        eps = torch.empty_like(resp)
        unit = np.zeros((2, 2))
        unit[0, 0] = 1.0
        infos = tmp.solve([0, 1, 2], [np.zeros((2, 2)), np.zeros((2, 2)), unit], list(eps), list(resp),
                          max_iter=self.p["ls_max_iter"], tol=self.p["ls_tol"], stream=self.stream)
        for info in infos:
            if not np.all(np.isfinite(np.array(info.sig_mean))):
                raise ValueError("fast patching: non-finite patch response")
        W = 2 * self.R + 1
        self.kern = torch.empty((2, W, W, 2, 2), dtype=f64, device=d)
        self.miss = torch.empty((2, 2, 2), dtype=f64, device=d)
        L.check(L.lib().mgk_kmc2d_patch_setup(nx, ny, self.R, L.ptr(resp[0]), L.ptr(resp[1]), L.ptr(self.kern),
                                              L.ptr(self.miss), L.stream_ptr(self.stream)), "mgk_kmc2d_patch_setup")
        with torch.cuda.stream(self.stream):
            self.sig_unit = resp[2].clone()
        self.stream.synchronize()  # the temporary plan and responses are released after this
        del tmp

    def launch_patch(self, sel, indices=None, unit_scale=None):
        """One fast-patching stress update (``mgk_kmc2d_patch``); ``sel`` a
        device pointer to the selection (None: only the macro-strain term)."""
        unit = L.ptr(self.sig_unit) if unit_scale is not None else None
        L.check(L.lib().mgk_kmc2d_patch(self.nx, self.ny, self.M, L.ptr(self.sig), unit,
                                        0.0 if unit_scale is None else float(unit_scale), L.ptr(self.kern),
                                        L.ptr(self.miss), self.R, L.ptr(self.catalog), sel, indices,
                                        L.stream_ptr(self.stream)), "mgk_kmc2d_patch")

    @property
    def E_avg(self):
        return float(self._means_h[0])

    @property
    def nu_avg(self):
        return float(self._means_h[1])

    # ------------------------------------------------------------ stages ---
    def solve_args(self):
        """(plan, replica, eps_bar, eps_out, sig_out, eps_init) of the next LS
        solve with the current eigenstrain (the caller runs it on ``stream``)."""
        init = None
        if self.ls_start == "warm" and self.n_solves > 0:
            with self.torch.cuda.stream(self.stream):
                self.eps_prev.copy_(self.eps)
            init = self.eps_prev
        return self.ls, self.rep, self.eps_macro.copy(), self.eps, self.sig, init

    def after_solve(self, info):
        """Mean stress of a finished solve, with the reference's stability guard
        (kmc_simulator.py:522-524)."""
        self.n_solves += 1
        sigM = np.array(info.sig_mean).reshape(2, 2)
        if not np.all(np.isfinite(sigM)) or np.max(np.abs(sigM)) / 1e9 > 20.0:
            raise ValueError(f"Unstable stress in small-strain elastic_run: {sigM / 1e9} GPa")
        return sigM

    def elastic_run(self):
        """LS solve with the current eigenstrain; returns the mean stress."""
        ls, rep, eb, eo, so, init = self.solve_args()
        info = ls.solve([rep], [eb], [eo], [so], eps_init=None if init is None else [init],
                        max_iter=self.p["ls_max_iter"], tol=self.p["ls_tol"], stream=self.stream)[0]
        return self.after_solve(info)

    def launch_rates(self):
        """Enqueues barriers, rates and the copy of the total rate to the host.
        Exact selection: barriers, then rates with the reference's sequential
        running sum.  Fast selection: one fused pass for barriers and the total
        (rates and running sums are built in ``event`` when a draw needs them)."""
        lib, S, p = L.lib(), L.stream_ptr(self.stream), self.p
        if self.selection == "exact":
            L.check(lib.mgk_kmc2d_barrier(self.nx, self.ny, self.M, L.ptr(self.Q), L.ptr(self.Q0), L.ptr(self.sig),
                                          L.ptr(self.catalog), p["volume"], L.ptr(self.soft), L.ptr(self.t_last),
                                          self.time, L.ptr(self.prev), p["cap"], 0, self.tau, S), "mgk_kmc2d_barrier")
            L.check(lib.mgk_kmc2d_rates(self.nx, self.ny, self.M, L.ptr(self.Q), 1.0, None, p["T"], p["nu0"],
                                        1 if self.cascade_mode else 0, L.ptr(self.rates), L.ptr(self.indices),
                                        L.ptr(self.prefix), L.ptr(self.count), L.ptr(self.total), L.ptr(self.work),
                                        S), "mgk_kmc2d_rates")
            self.total_h.copy_(self.total, non_blocking=True)
        else:
            L.check(lib.mgk_kmc2d_barrier_total(self.nx, self.ny, self.M, L.ptr(self.Q), L.ptr(self.Q0),
                                                L.ptr(self.sig), L.ptr(self.catalog), p["volume"], L.ptr(self.soft),
                                                L.ptr(self.t_last), self.time, L.ptr(self.prev), p["cap"], 0,
                                                self.tau, 1.0, None, p["T"], p["nu0"], L.ptr(self.total_fast),
                                                L.ptr(self.work), S), "mgk_kmc2d_barrier_total")
            self.total_h.copy_(self.total_fast, non_blocking=True)

    def barriers_and_rates(self):
        """Barriers, rates and the total rate (one synchronisation)."""
        self.launch_rates()
        self.stream.synchronize()
        return float(self.total_h[0])

    def event(self, u_sel, new_catalog, q0, t_wait=0.0):
        """One KMC event on the device: selection with the draw u_sel, the flip
        and its bookkeeping, the redraw of the voxel's catalog (new_catalog,
        (M, 2, 2)) and barriers (q0, (M,))."""
        lib, S, p = L.lib(), L.stream_ptr(self.stream), self.p
        M = self.M
        self.redraw_h[:4 * M] = self.torch.from_numpy(np.ascontiguousarray(new_catalog, dtype=np.float64).reshape(-1))
        self.redraw_h[4 * M:] = self.torch.from_numpy(q0)
        self.redraw.copy_(self.redraw_h, non_blocking=True)
        total = self.total
        if self.selection != "exact":
            # rates of the drawn step and their parallel running sums; the draw
            # scales the total the waiting time used (the fused pass's)
            L.check(lib.mgk_kmc2d_rates_only(self.nx, self.ny, M, L.ptr(self.Q), 1.0, None, p["T"], p["nu0"],
                                             L.ptr(self.rates), S), "mgk_kmc2d_rates_only")
            L.check(lib.mgk_kmc_prefix_fast(L.ptr(self.rates), self.nx * self.ny * M, L.ptr(self.prefix),
                                            L.ptr(self.count), L.ptr(self.total), L.ptr(self.work), S),
                    "mgk_kmc_prefix_fast")
            total = self.total_fast
        L.check(lib.mgk_kmc_select(L.ptr(self.prefix), L.ptr(self.count), L.ptr(total), float(u_sel),
                                   L.ptr(self.sel), S), "mgk_kmc_select")
        nc = L.ptr(self.redraw)
        nq = L.c_void_p(self.redraw.data_ptr() + 4 * M * 8)
        # compacted rates (cascade mode) map the selected position to its mode
        ind = L.ptr(self.indices) if self.cascade_mode else None
        if self.fast:
            # the stress patch of the pre-flip direction (kmc_simulator.py:1044-1069)
            self.unit_ready = True
            self.launch_patch(L.ptr(self.sel), ind, p["strain_rate"] * t_wait if t_wait > 0 else None)
        L.check(lib.mgk_kmc2d_event(self.nx, self.ny, M, L.ptr(self.sel), ind, L.ptr(self.eps_p), L.ptr(self.soft),
                                    L.ptr(self.t_last), L.ptr(self.catalog), L.ptr(self.Q0), L.ptr(self.prev), nc, nq,
                                    self.time, p["jp"], p["jt"], p["cap"], p["jn"], L.ptr(self.xym), S),
                "mgk_kmc2d_event")
        L.check(lib.mgk_ls2d_sync_voxel(self.ls._h, self.rep, L.ptr(self.eps_p), L.ptr(self.xym), S),
                "mgk_ls2d_sync_voxel")
        self.xym_h.copy_(self.xym, non_blocking=True)

    # ------------------------------------------------------------ cascade ---
    def launch_barriers(self):
        lib, S, p = L.lib(), L.stream_ptr(self.stream), self.p
        L.check(lib.mgk_kmc2d_barrier(self.nx, self.ny, self.M, L.ptr(self.Q), L.ptr(self.Q0), L.ptr(self.sig),
                                      L.ptr(self.catalog), p["volume"], L.ptr(self.soft), L.ptr(self.t_last),
                                      self.time, L.ptr(self.prev), p["cap"], 0, self.tau, S), "mgk_kmc2d_barrier")

    def unstable_batch(self):
        """The modes of one cascade batch (kmc_simulator.py:578-600,
        find_unstable_2d :162-181): modes with Q < threshold in (x, y, m)
        order, sorted by Q ascending, the first of each voxel.  Reads the
        barriers (call after the stream has completed them)."""
        with self.torch.cuda.stream(self.stream):
            Qf = self.Q.reshape(-1)
            flat = self.torch.nonzero(Qf < self.stability_threshold).flatten()
            q = Qf[flat].cpu().numpy()
            flat = flat.cpu().numpy()
        if flat.size == 0:
            return []
        order = flat[np.argsort(q)]
        seen, batch = set(), []
        for f in order:
            v = int(f) // self.M
            if v not in seen:
                seen.add(v)
                batch.append(int(f))
        return batch

    def cascade_flips_batch(self, batch, draws):
        """Flips the batch's modes in order, each with the bookkeeping and
        redraws of a KMC event (kmc_simulator.py:728-760)."""
        lib, S, p = L.lib(), L.stream_ptr(self.stream), self.p
        M, k = self.M, len(batch)
        torch = self.torch
        sel_h = torch.tensor(batch, dtype=torch.int64).pin_memory()
        red_h = torch.empty((k, 5 * M), dtype=torch.float64).pin_memory()
        for i in range(k):
            red_h[i, :4 * M] = torch.from_numpy(np.ascontiguousarray(draws.catalog(M), dtype=np.float64).reshape(-1))
            red_h[i, 4 * M:] = torch.from_numpy(np.ascontiguousarray(draws.q0(M), dtype=np.float64))
        with torch.cuda.stream(self.stream):
            sel_d = sel_h.to(self.dev, non_blocking=True)
            red_d = red_h.to(self.dev, non_blocking=True)
        self._keep_batch = (sel_h, red_h, sel_d, red_d)  # alive until the stream has used them
        for i in range(k):
            nc = L.c_void_p(red_d.data_ptr() + i * 5 * M * 8)
            nq = L.c_void_p(red_d.data_ptr() + (i * 5 * M + 4 * M) * 8)
            L.check(lib.mgk_kmc2d_event(self.nx, self.ny, M, L.c_void_p(sel_d.data_ptr() + 8 * i), None,
                                        L.ptr(self.eps_p), L.ptr(self.soft), L.ptr(self.t_last),
                                        L.ptr(self.catalog), L.ptr(self.Q0), L.ptr(self.prev), nc, nq, self.time,
                                        p["jp"], p["jt"], p["cap"], p["jn"], L.ptr(self.xym), S), "mgk_kmc2d_event")
            L.check(lib.mgk_ls2d_sync_voxel(self.ls._h, self.rep, L.ptr(self.eps_p), L.ptr(self.xym), S),
                    "mgk_ls2d_sync_voxel")
            if self.fast:
                # the patch of the redrawn direction (kmc_simulator.py:764-774)
                self.launch_patch(L.c_void_p(sel_d.data_ptr() + 8 * i))

    # ---------------------------------------------------------------- run ---
    def trajectory(self, rng, n_steps, max_events=None):
        """The trajectory as a generator of the host-visible results it needs:
        it yields ("solve",) when the next LS solve (``solve_args``) must run and
        be sent back as its LsInfo, and ("sync",) when the work enqueued on
        ``stream`` must complete; it returns the result dict.  A scheduler can
        advance many trajectories and batch their solves; ``run`` drives one."""
        p = self.p
        draws = rng if hasattr(rng, "u_wait") else GeneratorDraws(rng, p["gamma0"], p["q_mean"], p["q_std"],
                                                                  p["q_min"])
        if self._resume:
            # restored between AQS steps: the stored fields are the last solve's
            self._resume = False
        else:
            self.after_solve((yield ("solve",)))
        strain_unit = np.zeros((2, 2))
        strain_unit[0, 0] = 1.0
        dt_step = abs(p["step_size"]) / p["strain_rate"] if p["strain_rate"] > 0 else 1.0
        remaining = 0.0
        steps_done = self.steps_done
        M = self.M
        cascade_count = 0
        n_batches = 0
        while steps_done < n_steps:
            remaining += dt_step
            while remaining > 0:
                if self.cascade_mode:
                    self.launch_barriers()
                    yield ("sync",)
                    batch = self.unstable_batch()
                    if batch:
                        # _run_cascade: batches until no mode is unstable
                        local_step = flips = 0
                        while batch:
                            self.cascade_flips_batch(batch, draws)
                            for f in batch:
                                x, y, m = f // (self.ny * M), (f // M) % self.ny, f % M
                                self.cascade_flips.append((x, y, m, self.time, n_batches))
                            if not self.fast:
                                self.after_solve((yield ("solve",)))
                            n_batches += 1
                            flips += len(batch)
                            local_step += 1
                            if local_step > self.nx * self.ny:
                                break
                            self.launch_barriers()
                            yield ("sync",)
                            batch = self.unstable_batch()
                        if self.fast and flips > 0:
                            # corrector: the final sync (kmc_simulator.py:790-792)
                            self.after_solve((yield ("solve",)))
                        if flips > 0:
                            cascade_count += 1
                        if cascade_count > self.max_cascade_limit:
                            return self.result(steps_done)
                        continue
                    cascade_count = 0
                self.launch_rates()
                yield ("sync",)
                total = float(self.total_h[0])
                if total > 0:
                    u = draws.u_wait()
                    t_wait = -np.log(u) / total
                    if t_wait < remaining:
                        self.time += t_wait
                        self.eps_macro += strain_unit * (p["strain_rate"] * t_wait)
                        remaining -= t_wait
                        u_sel = draws.u_sel()
                        new_cat = draws.catalog(M)
                        q0 = draws.q0(M)
                        self.event(u_sel, new_cat, q0, t_wait)
                        if not self.fast:
                            self.after_solve((yield ("solve",)))
                        else:
                            # a full re-solve every sync_interval KMC flips (:1071-1074)
                            self.flips_since_sync += 1
                            if self.flips_since_sync >= self.sync_interval:
                                self.after_solve((yield ("solve",)))
                                self.flips_since_sync = 0
                            else:
                                yield ("sync",)
                        x, y, m = (int(v) for v in self.xym_h.tolist())
                        self.events.append((x, y, m, self.time))
                        if max_events is not None and len(self.events) >= max_events:
                            return self.result(steps_done)
                        continue
                if self.fast and self.unit_ready:
                    self.launch_patch(None, None, p["strain_rate"] * remaining)  # :1094-1096
                self.eps_macro += strain_unit * (p["strain_rate"] * remaining)
                self.time += remaining
                remaining = 0.0
            prev_e, prev_s = {}, {}
            for _ in range(p["mixed_max_iter"]):
                sigM = self.after_solve((yield ("solve",)))
                err = np.zeros((2, 2))
                err_max = 0.0
                for idx, target in self.stress_targets.items():
                    e = target - sigM[idx]
                    err[idx] = e
                    err_max = max(err_max, abs(e))
                if err_max < p["mixed_tol"]:
                    break
                d_eps = (err - self.nu_avg * np.trace(err) * np.eye(2)) / self.E_avg
                for idx in self.stress_targets:
                    step = d_eps[idx]
                    if idx in prev_e:
                        d_e = self.eps_macro[idx] - prev_e[idx]
                        d_s = sigM[idx] - prev_s[idx]
                        if abs(d_e) > 1e-14 and np.isfinite(d_s):
                            slope = d_s / d_e
                            if np.isfinite(slope) and slope > 0.01 * self.E_avg:
                                step = err[idx] / slope
                    prev_e[idx] = self.eps_macro[idx]
                    prev_s[idx] = sigM[idx]
                    self.eps_macro[idx] += step
            steps_done += 1
            self.steps_done = steps_done
        return self.result(steps_done)

    def run(self, rng, n_steps, max_events=None):
        gen = self.trajectory(rng, n_steps, max_events)
        send = None
        while True:
            try:
                need = gen.send(send)
            except StopIteration as stop:
                return stop.value
            if need[0] == "solve":
                ls, rep, eb, eo, so, init = self.solve_args()
                send = ls.solve([rep], [eb], [eo], [so], eps_init=None if init is None else [init],
                                max_iter=self.p["ls_max_iter"], tol=self.p["ls_tol"], stream=self.stream)[0]
            else:
                self.stream.synchronize()
                send = None

    def result(self, steps):
        self.steps_done = steps
        return dict(events=list(self.events), eps_macro=self.eps_macro.copy(), sig=self.sig.cpu().numpy(),
                    eps_p=self.eps_p.cpu().numpy(), time=self.time, steps=steps, solves=self.n_solves,
                    cascade_flips=list(self.cascade_flips))
