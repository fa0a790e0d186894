"""The N>1 host path on CPU: world_size-2 gloo processes shard instances, commit them (with the
CPU oracle standing in for the device), gather the 32-byte roots, and must reproduce the
single-process roots exactly.  Also covers the bench's max-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

SHAPES = [(8, 9, 5), (10, 11, 17), (7, 9, 3), (9, 10, 40), (6, 7, 1), (11, 12, 2), (8, 10, 9)]


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _roots_for(indices):
    import oracle
    orc = oracle.Oracle()
    out = {}
    for i in indices:
        nb, nbe, nc = SHAPES[i]
        trace = oracle.random_field((1 << nb, nc), 9000 + i)
        out[i] = [int(v) for v in orc.commit(trace, nbe, 4)[0]]
    return out


def _worker(rank, world, port, result_path):
    import sys
    here = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(here, "tests"))
    import datetime

    import torch
    from conftest import load_package

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    pkg = load_package()
    import importlib
    sharding = importlib.import_module("pil2_proofman_b200.sharding")
    mine = sharding.my_instances(SHAPES, world, rank)
    roots = sharding.gather_roots(_roots_for(mine), len(SHAPES), dist)
    # max-over-ranks timing reduction as bench.py does it
    t = torch.tensor([float(rank + 1)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    if rank == 0:
        np.save(result_path, np.array([[int(v) for v in r] for r in roots], dtype=np.uint64))
        with open(result_path + ".max", "w") as f:
            f.write(str(float(t.item())))
    dist.barrier()
    dist.destroy_process_group()
    assert pkg is not None


def test_assignment_balanced(pkg):
    import importlib
    sharding = importlib.import_module("pil2_proofman_b200.sharding")
    owner = sharding.assign_instances(SHAPES, 2)
    loads = [0, 0]
    for i, r in enumerate(owner):
        loads[r] += sharding.commit_cost(*SHAPES[i])
    assert set(owner) == {0, 1}
    assert max(loads) <= sum(loads) * 0.7
    assert sharding.assign_instances(SHAPES, 1) == [0] * len(SHAPES)


def test_two_rank_gloo_roots_match_single(tmp_path, pkg):
    path = str(tmp_path / "roots.npy")
    mp.start_processes(_worker, args=(2, _free_port(), path), nprocs=2, join=True, start_method="spawn")
    got = np.load(path)
    single = _roots_for(range(len(SHAPES)))
    assert (got == np.array([single[i] for i in range(len(SHAPES))], dtype=np.uint64)).all()
    assert float(open(path + ".max").read()) == 2.0
