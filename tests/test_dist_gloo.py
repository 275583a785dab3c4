"""Multi-rank host logic of the weak-scaling bench on CPU: world_size 2 with gloo."""
import os
import socket

import numpy as np
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


def _vtk_worker(rank, world, port, base, q):
    import datetime
    import numpy as np
    import torch.distributed as dist
    from ves3d_b200 import vtk
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    p1, nv = 3, rank + 1  # each rank writes its own vesicles
    X1 = np.full(nv * 3 * 2 * p1 * (p1 + 1), float(rank))
    vtk.write_grid(X1, np.zeros(nv * 6), p1, base)  # rank and size from the process group
    dist.barrier()
    dist.destroy_process_group()
    q.put(rank)


@pytest.mark.timeout(120)
def test_vtk_output_from_two_ranks(tmp_path):
    """Each rank writes its piece <base>_<rank>.vtp; rank 0 writes the index naming both."""
    from ves3d_b200 import vtk
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    base = str(tmp_path / "frame")
    procs = [ctx.Process(target=_vtk_worker, args=(r, 2, port, base, q)) for r in range(2)]
    for p in procs:
        p.start()
    assert sorted(q.get(timeout=90) for _ in procs) == [0, 1]
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert vtk.read_pvtp(base + ".pvtp") == ["frame_000000.vtp", "frame_000001.vtp"]
    for r in range(2):
        d = vtk.read_vtp(base + "_%06d.vtp" % r)
        npt = 2 * 3 * 4 + 2
        assert d["points"].shape == ((r + 1) * npt, 3)
        assert np.all(d["points"][: 2 * 3 * 4] == float(r))


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
