"""The multi-GPU path of bench.py is replicas only: each rank runs its own Fisher
simulations (disjoint seeds, no data-path collective) and the job time is the
slowest rank's.  Checked on CPU with two gloo ranks."""
import os
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    seeds = bench.replica_seeds(rank, 5)
    t = bench.max_over_ranks(10.0 + rank, "cpu")
    out.put((rank, seeds, t))
    dist.destroy_process_group()


def test_replicas_disjoint_seeds_and_max_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    res = dict((r, (s, t)) for r, s, t in res)
    assert not set(res[0][0]) & set(res[1][0])
    assert res[0][1] == res[1][1] == 11.0
