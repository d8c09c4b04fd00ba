"""Multi-rank host logic of bench.py (replicas): two gloo ranks on CPU."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    sys.path.insert(0, os.path.join(root, "pagani-toolkit_b200"))
    import torch.distributed as dist
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    t = bench.reduce_max_ms(10.0 * (rank + 1), "cpu")
    out[rank] = (t, bench.rank_subject_seed(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_max_time_and_distinct_subjects():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][0] == res[1][0] == pytest.approx(20.0)
    assert res[0][1] != res[1][1]


def _env_rank(out):
    import torch.distributed as dist
    import bench
    rank, world = int(os.environ["RANK"]), int(os.environ["WORLD_SIZE"])
    assert int(os.environ["LOCAL_RANK"]) == rank
    dist.init_process_group("gloo")          # env:// rendezvous, as bench.run does
    out[rank] = (world, bench.reduce_max_ms(5.0 + rank, "cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_spawn_without_torchrun_sets_rank_env():
    """bench.py --gpus N started without torchrun spawns its own N ranks with
    the torchrun environment, so init_process_group finds its rendezvous."""
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    for p in (root, os.path.join(root, "pagani-toolkit_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import bench
    with mp.Manager() as m:
        out = m.dict()
        bench.spawn_ranks(2, _env_rank, out)
        res = dict(out)
    assert res == {0: (2, 6.0), 1: (2, 6.0)}
