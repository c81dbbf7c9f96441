"""The multi-GPU form of bench.py on the host: world size 2 over gloo.  Each rank times its own replica
(the single-graph path does not shard) or its own batch of graphs (the batched form shards by graphs, with
no collective on the data path); the job's time is the maximum over ranks."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank: int, world: int, port: int, out: str) -> None:
    import datetime
    import sys

    import torch.distributed as dist

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    from dmolp_b200.batch import random_instances

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    t = bench.max_over_ranks(dist, [1.0 + rank, 5.0 - rank])
    inst = random_instances(3, seed=bench.rank_seed(11, rank), vmin=200, vmax=400, threads=1)
    sig = [int(it.graph.num_arcs) for it in inst] + [it.k for it in inst]
    np.save(os.path.join(out, f"r{rank}.npy"), np.array(t + sig, np.float64))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_max_timing_and_distinct_shards(tmp_path):
    port = _free_port()
    mp.spawn(_rank, args=(2, port, str(tmp_path)), nprocs=2, join=True)
    r0 = np.load(tmp_path / "r0.npy")
    r1 = np.load(tmp_path / "r1.npy")
    assert list(r0[:2]) == [2.0, 5.0] and list(r1[:2]) == [2.0, 5.0]  # max over ranks, on every rank
    assert not np.array_equal(r0[2:], r1[2:])  # each rank partitions its own graphs


def test_single_process_is_identity():
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    assert bench.max_over_ranks(None, [3.0, 4.0]) == [3.0, 4.0]
    assert bench.rank_seed(11, 0) == 11 and bench.rank_seed(11, 1) != 11
