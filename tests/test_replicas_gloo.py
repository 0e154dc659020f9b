"""The N>1 path of bench.py: one process per GPU, independent replicas, the
step time reduced as the max over ranks and the value aggregated over ranks.
Runs as two gloo ranks on CPU (no GPU, no collective on the data path)."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank), DDC_BENCH_BACKEND="gloo")
    import bench
    w, r, local, pg = bench._dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench._barrier(pg, "cpu")
    # rank r "measured" (r + 1) * 100 ms for 2 steps: the job time is the max
    ms = bench._max_over_ranks((rank + 1) * 100.0, pg, "cpu")
    value = w * 2 / (ms * 1e-3)
    q.put((rank, ms, value))
    pg.destroy_process_group()


@pytest.mark.timeout(120)
def test_replica_timing_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [200.0, 200.0]
    assert all(abs(r[2] - 20.0) < 1e-9 for r in res)  # 2 replicas x 2 steps / 0.2 s


def test_reference_arm_iteration_counts_parse():
    import bench
    d, a = bench._reference_iters()
    assert d > 0 and a > 0
