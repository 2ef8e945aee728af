"""The multi-process path of bench.py on CPU (gloo, world size 2): the
max-over-ranks timing reduction every rank takes, the whole-job rate, and
the reference arm running on rank 0 only.  Replicas only: the ranks share
nothing else."""
import os
import socket
import sys
import types

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import datetime
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = bench._max_over_ranks([10.0 + rank, 20.0 - 5.0 * rank])
        rates = bench._job_rates({"a": ms[0]}, 32, 10, world)
        # the reference arm: rank 0 alone runs it; the others return at once
        a = types.SimpleNamespace(batch=32, warmup=1, steps=1, gpus=world)
        ran = None if rank == 0 else bench.run_reference(a)
        dist.barrier()
        q.put((rank, ms, rates["a"], ran, bench._rank()))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reduce_timings_and_only_rank0_runs_the_reference():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, ms, rate, ran, rk in out:
        assert ms == [11.0, 20.0]                       # element-wise max over the two ranks
        assert abs(rate - 32 * 10 * 2 / 0.011) < 1e-6   # both ranks' items over the slowest time
        assert rk == (rank, 2, rank)
        if rank == 1:
            assert ran is None


def test_single_process_reduction_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench._max_over_ranks([3.0, 4.0]) == [3.0, 4.0]
    assert bench._job_rates({"x": 100.0}, 32, 10, 1) == {"x": 3200.0}
