"""The bench's multi-GPU form is replicas: one independent simulation per
rank, a barrier around the timed region and the max device time over ranks.
This checks that harness with two gloo ranks on the CPU."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(ws),
                      LOCAL_RANK=str(rank))
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import torch.distributed as dist
    w, r, _ = bench.dist_setup("gloo")
    bench.dist_barrier(w)
    # rank r "took" 100 + 50 r ms for 2 simulations of 1000 cells x 10 steps
    value, ms_max = bench.job_throughput(w, 1000.0, 10, 2, 100.0 + 50.0 * r)
    bench.dist_barrier(w)
    q.put((r, value, ms_max))
    dist.destroy_process_group()


def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, value, ms_max in res:
        assert ms_max == 150.0
        assert value == pytest.approx(2 * 1000.0 * 10 * 2 / 0.150 / 1e9)
