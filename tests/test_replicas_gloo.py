"""Multi-GPU runs are replicas: every rank solves its own batch, and the
job's figures use the slowest rank's times.  The rank arithmetic of
bench.py runs here on two CPU processes over gloo."""
import os
import socket
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms, e2e = bench.max_over_ranks(dist, 1000.0 + 500.0 * rank, 9.0 - 1.0 * rank, "cpu")
        q.put((rank, ms, e2e, bench.job_values(world, 148, 70, ms, e2e)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_replicas_use_the_slowest_rank():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, ms, e2e, (value, strict, e2e_value) in out:
        assert ms == 1500.0 and e2e == 9.0  # the slower rank's step, the slower rank's end-to-end time
        assert abs(value - 2 * 148 / 1.5) < 1e-9
        assert abs(strict - 2 * 70 / 1.5) < 1e-9
        assert abs(e2e_value - 2 * 148 / 9.0) < 1e-9


def test_one_process_is_the_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(None, 3.0, 4.0, "cpu") == (3.0, 4.0)
    assert bench.job_values(1, 10, 5, 2000.0, 4.0) == (5.0, 2.5, 2.5)


def test_task_histogram_names_every_code():
    """The bench's report of how solves ended: one count per L-BFGS-B task
    code, unknown codes under "other"."""
    sys.path.insert(0, ROOT)
    import bench
    from smili_b200 import _lib
    h = bench.task_histogram([_lib.TASK_TARGET, _lib.TASK_TARGET, _lib.TASK_STOP, _lib.TASK_CONV,
                              _lib.TASK_ABNORMAL, _lib.TASK_ERROR, 99])
    assert h == {"target": 2, "converged": 1, "abnormal": 1, "iteration_limit": 1, "error": 1, "other": 1}
    assert bench.task_histogram([]) == {"target": 0, "converged": 0, "abnormal": 0, "iteration_limit": 0,
                                        "error": 0}
