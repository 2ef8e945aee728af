"""Device-resident 3D KMC/AQS driver.

Runs the trajectory of ThermalSimulation.run_simulation (mgkmc/aqs.py:682-1201)
on its small-strain KMC path (no cascade, no fast patching, no thermal
conduction; redraw of the voxel's catalog and barriers after a flip) with
every field resident on the GPU: barriers (mgk_kmc3d_barrier), rates and the
running rate sum (mgk_kmc3d_rates, bit-exact with the reference's sequential
total), selection (mgk_kmc_select), the flip with its bookkeeping and redraws
(mgk_kmc3d_event) and the LS re-solve (update_stress_fft_full, aqs.py:349, on a
3D LS plan) never leave the device.  The host keeps the clock, the macro
strain and the random draws; it reads the total rate once per attempt and
the mean stress once per solve.

Per AQS step (aqs.py:840-1152): attempts until the step's time is used; each
attempt updates the barriers, computes the rates and draws a waiting time;
an event inside the remaining time flips a mode and re-solves; at the end of
the step one solve, then the mixed loop: while the stress-controlled mean
stresses miss their targets by more than mixed_tol, add the isotropic
compliance correction (sigma_err - nu_avg tr I) / E_avg with the driven
component zeroed to eps_macro and re-solve.

Draws (``GeneratorDraws3D`` by default, or ``ReferenceDraws3D`` for the
reference's own RandomState stream): per attempt u_wait; per event u_sel,
then the voxel's M new modes and M new barriers.
"""
import numpy as np

from . import _lib as L
from .kmc import GeneratorDraws, ReferenceDraws
from .linear_elastic_simulator import Ls3dBatch

KB = 8.617e-5


def in_plane_modes(theta, gamma0):
    """(M, 3, 3) in-plane pure-shear modes of amplitude gamma0/2 and
    orientation theta (the glass mode of stz/catalog.py:7-29)."""
    c, s = np.cos(2 * theta), np.sin(2 * theta)
    cat = np.zeros(theta.shape + (3, 3))
    cat[..., 0, 0] = 0.5 * gamma0 * c
    cat[..., 1, 1] = -0.5 * gamma0 * c
    cat[..., 0, 1] = 0.5 * gamma0 * s
    cat[..., 1, 0] = 0.5 * gamma0 * s
    return cat


class GeneratorDraws3D(GeneratorDraws):
    """GeneratorDraws with (M, 3, 3) in-plane modes."""

    def catalog(self, M):
        return in_plane_modes(self.rng.uniform(0.0, np.pi, M), self.gamma0)


class ReferenceDraws3D(ReferenceDraws):
    """The 3D simulator's draws, call for call: t_wait from uniform()
    (aqs.py:880), the selection's uniform(0, total) (stz/kmc.py:84), the
    catalog of stz_catalog_glass (stz/catalog.py:7-40, in-plane), Gaussian
    barriers (stz/barrier_generators.py:24-29)."""

    def u_wait(self):
        return self.rs.uniform()

    def catalog(self, M):
        cat = np.zeros((M, 3, 3))
        cat[:, :2, :2] = super().catalog(M)
        return cat


class Kmc3D:
    def __init__(self, E, nu, catalog, Q0, gamma0=0.1, T=300.0, nu0=1e13, strain_rate=1e7, step_size=1e-5,
                 q_act_temp=0.37, jp=0.0, jt=0.0, cap=2.0, jn=0.0, component=(0, 0), stress_targets=None,
                 mixed_tol=1e4, mixed_max_iter=50, ls_tol=1e-6, ls_max_iter=200, q_mean=1.0, q_std=0.15, q_min=0.3,
                 volume=1.0, selection="exact", ls_start="cold", precision="fp64", ls=None, rep=0, stream=None):
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("mgkmc_b200 needs a CUDA device (no CPU fallback)")
        self.torch = torch
        d = self.dev = torch.device("cuda", torch.cuda.current_device())
        self.nx, self.ny, self.nz, self.M = Q0.shape
        nx, ny, nz, M = self.nx, self.ny, self.nz, self.M
        self.p = dict(gamma0=gamma0, T=T, nu0=nu0, strain_rate=strain_rate, step_size=step_size, jp=jp, jt=jt,
                      cap=cap, jn=jn, mixed_tol=mixed_tol, mixed_max_iter=mixed_max_iter, ls_tol=ls_tol,
                      ls_max_iter=ls_max_iter, q_mean=q_mean, q_std=q_std, q_min=q_min, volume=volume)
        self.component = tuple(component)
        if stress_targets is None:  # aqs.py:715-722
            stress_targets = {(1, 1): 0.0, (2, 2): 0.0} if self.component == (0, 0) else \
                {(0, 0): 0.0, (1, 1): 0.0, (2, 2): 0.0}
        self.stress_targets = dict(stress_targets)
        if selection not in ("exact", "fast"):
            raise ValueError("selection: 'exact' or 'fast'")
        self.selection, self.ls_start = selection, ls_start
        self.tau = 1.0 / (nu0 * np.exp(-q_act_temp / (KB * T))) if T > 0 else np.inf
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        f64 = torch.float64

        def t(a):
            if isinstance(a, torch.Tensor):
                return a.to(device=d, dtype=f64).contiguous()
            return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).to(d)
        self.E, self.nu = t(E), t(nu)
        self._means_h = torch.empty(2, dtype=f64).pin_memory()
        with torch.cuda.stream(self.stream):
            self._means_h.copy_(torch.stack([self.E.mean(), self.nu.mean()]), non_blocking=True)
        self.catalog, self.Q0 = t(catalog), t(Q0)
        self.eps_p = torch.zeros((nx, ny, nz, 3, 3), dtype=f64, device=d)
        self.soft = torch.zeros((nx, ny, nz, 4), dtype=f64, device=d)
        self.t_last = torch.full((nx, ny, nz), -np.inf, dtype=f64, device=d)
        self.prev = torch.zeros((nx, ny, nz, 3, 3), dtype=f64, device=d)
        self.Q = torch.zeros((nx, ny, nz, M), dtype=f64, device=d)
        self.eps = torch.zeros((nx, ny, nz, 3, 3), dtype=f64, device=d)
        self.sig = torch.zeros_like(self.eps)
        self.eps_prev = torch.zeros_like(self.eps)
        n = nx * ny * nz * M
        self.rates = torch.empty(n, dtype=f64, device=d)
        self.indices = torch.empty(n, dtype=torch.int64, device=d)
        self.prefix = torch.empty(n, dtype=f64, device=d)
        self.count = torch.zeros(1, dtype=torch.int64, device=d)
        self.total = torch.zeros(1, dtype=f64, device=d)
        self.total_h = torch.zeros(1, dtype=f64).pin_memory()
        self.sel = torch.zeros(1, dtype=torch.int64, device=d)
        self.xyzm = torch.zeros(4, dtype=torch.int64, device=d)
        self.xyzm_h = torch.zeros(4, dtype=torch.int64).pin_memory()
        self.redraw_h = torch.zeros(10 * M, dtype=f64).pin_memory()
        self.redraw = torch.zeros(10 * M, dtype=f64, device=d)
        self.work = torch.empty(max(int(L.lib().mgk_kmc_rates_work_bytes(n)), int(L.lib().mgk_kmc_scan_work_bytes(n))),
                                dtype=torch.uint8, device=d)
        if ls is None:
            self.ls, self.rep = Ls3dBatch([(nx, ny, nz)], precision=precision), 0
        else:
            self.ls, self.rep = ls, int(rep)
        self.ls.set_material(self.rep, self.E, self.nu, self.eps_p, stream=self.stream)
        self.eps_macro = np.zeros((3, 3))
        self.time = 0.0
        self.events = []
        self.n_solves = 0
        self.steps_done = 0
        self.host_result = True
        self._resume = False

    _FIELDS = ("E", "nu", "eps", "sig", "eps_p", "soft", "Q", "Q0", "catalog", "t_last", "prev")

    def state_dict(self):
        """Host copies of the trajectory state between AQS steps (the fields,
        the clock, the macro strain, the event list and counters)."""
        self.stream.synchronize()
        st = {k: getattr(self, k).cpu().numpy() for k in self._FIELDS}
        st.update(eps_macro=self.eps_macro.copy(), time=self.time, events=list(self.events),
                  n_solves=self.n_solves, steps_done=self.steps_done)
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
        self.eps_macro = np.array(st["eps_macro"], dtype=np.float64).reshape(3, 3)
        self.time = float(st["time"])
        self.events = [tuple(e) for e in st["events"]]
        self.n_solves = int(st["n_solves"])
        self.steps_done = int(st["steps_done"])
        self._resume = True
        self.stream.synchronize()

    @property
    def E_avg(self):
        return float(self._means_h[0])

    @property
    def nu_avg(self):
        return float(self._means_h[1])

    # ------------------------------------------------------------ stages ---
    def solve_args(self):
        init = None
        if self.ls_start == "warm" and self.n_solves > 0:
            with self.torch.cuda.stream(self.stream):
                self.eps_prev.copy_(self.eps)
            init = self.eps_prev
        return self.ls, self.rep, self.eps_macro.copy(), self.eps, self.sig, init

    def after_solve(self, info):
        self.n_solves += 1
        sigM = np.array(info.sig_mean).reshape(3, 3)
        if not np.all(np.isfinite(sigM)):
            raise ValueError(f"Unstable stress in the 3D solve: {sigM / 1e9} GPa")
        return sigM

    def launch_rates(self):
        lib, S, p = L.lib(), L.stream_ptr(self.stream), self.p
        nx, ny, nz, M = self.nx, self.ny, self.nz, self.M
        L.check(lib.mgk_kmc3d_barrier(nx, ny, nz, M, L.ptr(self.Q), L.ptr(self.Q0), L.ptr(self.sig),
                                      L.ptr(self.catalog), p["volume"], L.ptr(self.soft), L.ptr(self.t_last),
                                      self.time, L.ptr(self.prev), p["cap"], 0, self.tau, S), "mgk_kmc3d_barrier")
        if self.selection == "exact":
            L.check(lib.mgk_kmc3d_rates(nx, ny, nz, M, L.ptr(self.Q), 1.0, None, p["T"], p["nu0"], 0,
                                        L.ptr(self.rates), L.ptr(self.indices), L.ptr(self.prefix), L.ptr(self.count),
                                        L.ptr(self.total), L.ptr(self.work), S), "mgk_kmc3d_rates")
        else:
            # KMC-mode rates of the flattened modes (the rate of a mode depends
            # on its barrier and the scalar temperature only) and a parallel scan
            L.check(lib.mgk_kmc2d_rates_only(nx * ny, nz, M, L.ptr(self.Q), 1.0, None, p["T"], p["nu0"],
                                             L.ptr(self.rates), S), "mgk_kmc2d_rates_only")
            L.check(lib.mgk_kmc_prefix_fast(L.ptr(self.rates), nx * ny * nz * M, L.ptr(self.prefix),
                                            L.ptr(self.count), L.ptr(self.total), L.ptr(self.work), S),
                    "mgk_kmc_prefix_fast")
        self.total_h.copy_(self.total, non_blocking=True)

    def event(self, u_sel, new_catalog, q0):
        lib, S, p = L.lib(), L.stream_ptr(self.stream), self.p
        M = self.M
        self.redraw_h[:9 * M] = self.torch.from_numpy(np.ascontiguousarray(new_catalog, dtype=np.float64).reshape(-1))
        self.redraw_h[9 * M:] = self.torch.from_numpy(np.ascontiguousarray(q0, dtype=np.float64))
        self.redraw.copy_(self.redraw_h, non_blocking=True)
        L.check(lib.mgk_kmc_select(L.ptr(self.prefix), L.ptr(self.count), L.ptr(self.total), float(u_sel),
                                   L.ptr(self.sel), S), "mgk_kmc_select")
        nc = L.ptr(self.redraw)
        nq = L.c_void_p(self.redraw.data_ptr() + 9 * M * 8)
        L.check(lib.mgk_kmc3d_event(self.nx, self.ny, self.nz, M, L.ptr(self.sel), None, L.ptr(self.eps_p),
                                    L.ptr(self.soft), L.ptr(self.t_last), L.ptr(self.catalog), L.ptr(self.Q0),
                                    L.ptr(self.prev), nc, nq, self.time, p["jp"], p["jt"], p["cap"], p["jn"],
                                    L.ptr(self.xyzm), S), "mgk_kmc3d_event")
        self.ls.set_eigenstrain(self.rep, self.eps_p, stream=self.stream)
        self.xyzm_h.copy_(self.xyzm, non_blocking=True)

    # ---------------------------------------------------------------- run ---
    def trajectory(self, rng, n_steps, max_events=None):
        """Generator like Kmc2D.trajectory: yields ("solve",) when the next LS
        solve (``solve_args``) must run and be sent back as its info, ("sync",)
        when the work on ``stream`` must complete; returns the result dict."""
        p = self.p
        M = self.M
        draws = rng if hasattr(rng, "u_wait") else GeneratorDraws3D(rng, p["gamma0"], p["q_mean"], p["q_std"],
                                                                    p["q_min"])
        unit = np.zeros((3, 3))
        unit[self.component] = 1.0
        if self._resume:  # the restored fields are the last solve's result
            self._resume = False
        else:
            self.after_solve((yield ("solve",)))
        dt_step = abs(p["step_size"]) / p["strain_rate"] if p["strain_rate"] > 0 else 1.0
        remaining = 0.0
        steps_done = self.steps_done
        while steps_done < n_steps:
            remaining += dt_step
            while remaining > 0:
                self.launch_rates()
                yield ("sync",)
                total = float(self.total_h[0])
                if total > 0:
                    t_wait = -np.log(draws.u_wait()) / total
                    if t_wait < remaining:
                        self.time += t_wait
                        self.eps_macro += unit * (p["strain_rate"] * t_wait)
                        remaining -= t_wait
                        self.event(draws.u_sel(), draws.catalog(M), draws.q0(M))
                        self.after_solve((yield ("solve",)))
                        x, y, z, m = (int(v) for v in self.xyzm_h.tolist())
                        self.events.append((x, y, z, m, self.time))
                        if max_events is not None and len(self.events) >= max_events:
                            return self.result(steps_done)
                        continue
                self.eps_macro += unit * (p["strain_rate"] * remaining)
                self.time += remaining
                remaining = 0.0
            sigM = self.after_solve((yield ("solve",)))
            for _ in range(p["mixed_max_iter"]):
                err = np.zeros((3, 3))
                err_max = 0.0
                for idx, target in self.stress_targets.items():
                    e = target - sigM[idx]
                    err[idx] = e
                    err_max = max(err_max, abs(e))
                if err_max < p["mixed_tol"]:
                    break
                corr = (err - self.nu_avg * np.trace(err) * np.eye(3)) / self.E_avg
                corr[self.component] = 0.0
                self.eps_macro += corr
                sigM = self.after_solve((yield ("solve",)))
            steps_done += 1
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
        """The trajectory's result; with ``host_result`` False the fields stay
        on the device (the caller reads what it needs)."""
        self.steps_done = steps
        out = dict(events=list(self.events), eps_macro=self.eps_macro.copy(), time=self.time, steps=steps,
                   solves=self.n_solves)
        if self.host_result:
            out.update(sig=self.sig.cpu().numpy(), eps_p=self.eps_p.cpu().numpy(), catalog=self.catalog.cpu().numpy(),
                       Q0=self.Q0.cpu().numpy())
        return out
