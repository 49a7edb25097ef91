"""Multi-GPU sharding of the Monte Carlo batch, exercised on CPU with two gloo
ranks: every rank gets its own sample ids (the union is contiguous, no
overlap, different input rows) and the step time is the max over ranks --
the only collective of the multi-GPU bench."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import torch.distributed as dist
    from ufem_b200 import meshgen as mg
    from ufem_b200.shard import max_over_ranks, rank_samples
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        first, count = rank_samples(rank, 6, 1 << 20)
        m = mg.warm_beam(4, 1, 1, zones=2)
        rows = mg.warm_samples(m, count, first_sample=first)
        t = max_over_ranks(10.0 + rank)
        np.savez(os.path.join(out_dir, f"r{rank}.npz"), first=first, count=count, rows=rows, t=t)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_disjoint_samples_and_max(tmp_path):
    import torch.multiprocessing as mp
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, join=True, start_method="spawn")
    r = [np.load(tmp_path / f"r{k}.npz") for k in range(2)]
    ids = [set(range(int(z["first"]), int(z["first"]) + int(z["count"]))) for z in r]
    assert not (ids[0] & ids[1]) and len(ids[0] | ids[1]) == 12
    assert min(ids[0] | ids[1]) == 1 << 20 and max(ids[0] | ids[1]) == (1 << 20) + 11
    assert not np.array_equal(r[0]["rows"], r[1]["rows"])
    assert float(r[0]["t"]) == float(r[1]["t"]) == 11.0


def test_single_process_max_is_identity():
    from ufem_b200.shard import max_over_ranks, rank_samples
    assert max_over_ranks(3.5) == 3.5
    assert rank_samples(0, 8) == (0, 8) and rank_samples(3, 8, 100) == (124, 8)
    with pytest.raises(ValueError):
        rank_samples(-1, 8)
