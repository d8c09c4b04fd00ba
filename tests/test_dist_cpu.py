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
