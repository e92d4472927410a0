"""The N > 1 plumbing of bench.py (replicas, one process per GPU), on CPU with two gloo ranks:
the slowest replica's time is what every rank reports (max over ranks), the barrier joins, and the
job's value is the sum over the replicas (weak scaling)."""
import datetime
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import torch
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, 2, torch.device("cpu"))
    bench.barrier(2)
    value = 2 * bench.sim_days_per_hour(100, ms / 1000.0)
    q.put((rank, ms, value))
    dist.destroy_process_group()


def test_two_gloo_ranks_report_the_slowest_replica():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in (0, 1)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = {r: (ms, v) for r, ms, v in got}
    assert res[0][0] == res[1][0] == 15.0            # both see the slower rank's time
    assert res[0][1] == res[1][1]
    # 100 steps of 600 s in 15 ms (the timed region), two replicas
    want = 2 * (100 * 600.0 / 86400.0) / (0.015 / 3600.0)
    assert abs(res[0][1] - want) < 1e-9 * want
