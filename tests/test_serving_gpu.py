"""Served form: each request's result is the same alone and in the mix.

A small stream of 2D solves, 2D KMC trajectories, 3D finite-strain steps and
a 3D KMC trajectory runs through the continuous-batching server; then every request runs again
alone on a fresh server.  Batching changes which replicas share a launch,
never a replica's arithmetic, so fields, event lists and macro strains must
agree to 1e-12 relative (they agree bit for bit in practice)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a = a.double().cpu().numpy() if hasattr(a, "cpu") else np.asarray(a)
    b = b.double().cpu().numpy() if hasattr(b, "cpu") else np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _mix():
    from mgkmc_b200.serving import Request
    reqs = []
    spec = [("solve", 2, 64), ("trajectory", 2, 64), ("solve", 2, 128), ("solve", 2, 64), ("trajectory", 2, 64),
            ("solve", 3, 32), ("solve", 2, 128), ("trajectory", 2, 128), ("solve", 3, 32), ("trajectory", 3, 64)]
    for i, (kind, dim, n) in enumerate(spec):
        reqs.append(Request(i, 0.002 * i, kind, dim, n, 1000 + 17 * i))
    return reqs


def _server():
    from mgkmc_b200.serving import Server
    return Server(mode="served", n_events=6, q_mean=0.6, slots={64: 4, 128: 4})


def test_served_results_match_alone():
    reqs = _mix()
    mixed = _server().run(reqs, realtime=False, keep_outputs=True)
    assert all(not r.error for r in mixed), [r.error for r in mixed]
    for req, rm in zip(reqs, mixed):
        alone = _server().run([req], realtime=False, keep_outputs=True)[0]
        assert not alone.error
        if req.dim == 3 and req.kind == "trajectory":
            assert len(rm.out["events"]) == 6 and rm.out["events"] == alone.out["events"]
            assert np.allclose(rm.out["eps_macro"], alone.out["eps_macro"], rtol=1e-12, atol=0)
            assert _rel(rm.out["sig"], alone.out["sig"]) < 1e-12
        elif req.dim == 3:
            assert _rel(rm.out["F"], alone.out["F"]) < 1e-12
            assert _rel(rm.out["P"], alone.out["P"]) < 1e-12
        elif req.kind == "solve":
            assert _rel(rm.out["eps"], alone.out["eps"]) < 1e-12
            assert _rel(rm.out["sig"], alone.out["sig"]) < 1e-12
            assert np.allclose(rm.out["eps_bar"], alone.out["eps_bar"], rtol=1e-12, atol=0)
        else:
            assert rm.out["events"] == alone.out["events"]
            assert np.allclose(rm.out["eps_macro"], alone.out["eps_macro"], rtol=1e-12, atol=0)
            assert _rel(rm.out["sig"], alone.out["sig"]) < 1e-12
        assert rm.solves == alone.solves


def test_served_solve_matches_plain_fp64():
    # mixed precision + warm starts against the plain FP64 sequential form:
    # same converged fields within the solver tolerance
    from mgkmc_b200.serving import Request, Server
    reqs = [Request(0, 0.0, "solve", 2, 128, 5), Request(1, 0.0, "solve", 2, 64, 6)]
    a = Server(mode="served").run(reqs, realtime=False, keep_outputs=True)
    b = Server(mode="sequential").run(reqs, realtime=False, keep_outputs=True)
    for ra, rb in zip(a, b):
        assert _rel(ra.out["sig"], rb.out["sig"]) < 1e-6
        assert _rel(ra.out["eps"], rb.out["eps"]) < 1e-6
        assert np.max(np.abs(ra.out["sig_mean"][1, 1])) < 1e4 and np.max(np.abs(rb.out["sig_mean"][1, 1])) < 1e4


def test_summary_fields():
    from mgkmc_b200.serving import Request, Server, summarize
    reqs = [Request(i, 0.001 * i, "solve", 2, 64, i) for i in range(6)]
    s = summarize(Server(mode="served").run(reqs, realtime=True))
    assert s["completed"] == 6 and s["p99_s"] >= s["p50_s"] > 0 and s["solves_per_s"] > 0


def test_ensemble_runs_every_replica_to_its_event_count():
    # a small version of the batched KMC ensemble: mixed sizes and
    # temperatures, every replica admitted at once, one batched solve per size
    # per round; each replica reaches its event count, and a replica's
    # trajectory is the same as when it runs alone
    from mgkmc_b200.serving import Server, ensemble_requests, run_ensemble
    reqs = ensemble_requests(n_replicas=5, sizes=(64, 96), T_range=(300.0, 400.0), n_events=4)
    res, summ = run_ensemble(reqs, q_mean=0.6)
    assert summ["completed"] == 5 and summ["events"] == 20
    assert all(len(r.out["events"]) == 4 for r in res)
    alone = Server(mode="served", n_events=4, q_mean=0.6, slots={64: 1, 96: 1}).run([reqs[2]], realtime=False)[0]
    assert alone.out["events"] == res[2].out["events"]


def test_ragged_ensemble_matches_per_size_buckets():
    # one ragged plan (every replica's solve in one launch per stage) gives
    # each replica the trajectory it has in the per-size buckets (the
    # autotuner may pick another kernel family for the ragged plan, so the
    # fields agree to rounding, the events exactly)
    import numpy as np
    from mgkmc_b200.serving import ensemble_requests, run_ensemble
    reqs = ensemble_requests(n_replicas=6, sizes=(64, 96, 128), T_range=(300.0, 400.0), n_events=4)
    per, _ = run_ensemble(reqs, q_mean=0.6)
    rag, summ = run_ensemble(reqs, ragged=True, q_mean=0.6)
    assert summ["completed"] == 6 and summ["events"] == 24
    for a, b in zip(per, rag):
        assert a.out["events"] == b.out["events"]
        assert np.allclose(a.out["eps_macro"], b.out["eps_macro"], rtol=1e-9, atol=0)
