"""The multi-GPU form is replicas: one independent solve per rank, no
collective on the data path, whole-job throughput = all ranks' points over
the slowest rank's time.  The rank logic of bench.py runs here on two gloo
ranks on the CPU; the tree each rank builds is checked against a tree built
in the parent for that rank's seed."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import datetime
    import torch.distributed as dist
    import bench
    import __graft_entry__
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    K = __graft_entry__.load_package()
    r, w, _ = bench.dist_env()
    pts = K.generate_points(5000, "uniform", 0, bench.replica_seed(r))
    t = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
    fake_ms = 10.0 + 5.0 * r  # rank 1 is the slow one
    ms = bench.reduce_max(fake_ms, w, "cpu")
    q.put((r, t.desc.num_nodes, int(t.array("src_perm")[:5].sum()), ms,
           bench.aggregate_mpts(5000, w, ms)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_gloo(K):
    import multiprocessing as mp
    import bench
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for r, nodes, psum, ms, mpts in res:
        pts = K.generate_points(5000, "uniform", 0, bench.replica_seed(r))
        t = K.Tree(pts["sx"], pts["sy"], pts["sz"], pts["tx"], pts["ty"], pts["tz"], 32)
        assert nodes == t.desc.num_nodes and psum == int(t.array("src_perm")[:5].sum())
        assert ms == 15.0  # max over ranks
        assert mpts == pytest.approx(2 * 5000 / 15e3)
    assert res[0][2] != res[1][2]  # different problems per rank
