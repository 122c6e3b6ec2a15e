"""Multi-GPU batch sharding, host side: two gloo ranks on CPU split a batch, each computes its
instances (with the CPU oracle standing in for its GPU), and the gathered result equals the
unsharded one. No GPU is used."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from ssblasex_b200.sharding import shard_range


@pytest.mark.parametrize("batch,world", [(0, 2), (1, 2), (7, 2), (32, 4), (5, 8), (512, 3)])
def test_shard_ranges_partition_the_batch(batch, world):
    seen = []
    sizes = []
    for r in range(world):
        s, e = shard_range(batch, world, r)
        assert 0 <= s <= e <= batch
        seen.extend(range(s, e))
        sizes.append(e - s)
    assert seen == list(range(batch))
    assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    import pathlib
    sys.path.insert(0, str(pathlib.Path(__file__).resolve().parents[1]))
    import torch.distributed as dist
    from ssblasex_b200 import workloads as W
    from ssblasex_b200.sharding import run_sharded
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        p = W.make_problem("i8", 1, 0, 33, 20, 70, 7, 3, -2, seed=8)
        C, rng = run_sharded(p, lambda sub: O.restated_gemm(sub)[1], gather=True)
        out[rank] = (rng, bool(np.array_equal(C, O.restated_gemm(p)[1])))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reproduce_the_unsharded_batch():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
        for pr in procs:
            pr.start()
        for pr in procs:
            pr.join(timeout=120)
            assert pr.exitcode == 0
        res = dict(out)
    assert res[0][1] and res[1][1]
