"""Multi-rank host logic of the weak-scaling bench on CPU: world_size 2 with gloo."""
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
    import datetime
    import torch.distributed as dist
    from ves3d_b200 import dist as vd
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = 1.0 + rank  # rank 1 is the slow one
    tmax = vd.max_over_ranks(t, world)
    seed = vd.rank_seed(1001, rank)
    dist.barrier()
    dist.destroy_process_group()
    q.put((rank, tmax, seed))


@pytest.mark.timeout(120)
def test_weak_scaling_host_logic_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
    assert [r[1] for r in res] == [2.0, 2.0]        # max over ranks on every rank
    assert res[0][2] != res[1][2]                    # independent suspensions per rank
    from ves3d_b200 import dist as vd
    assert vd.aggregate_throughput(278528, 0.5, 2) == 2 * 278528 / 0.5
