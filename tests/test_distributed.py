"""Multi-GPU plumbing on the CPU: two gloo ranks shard a batch of independent states, each
evaluates its own (here with the oracle's cheap stationary state as the per-state work) and the
results are gathered on the host. The data path needs no collective; the gather is reporting."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from rcmps_b200.batch import random_state, shard


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, dims, out):
    import sys
    from pathlib import Path
    root = Path(__file__).resolve().parents[1]
    sys.path[:0] = [str(root), str(root / "rcmpscore.jl_b200")]
    from oracle import fg_phi4_oracle as O
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard(dims, rank, world)
    results = {}
    for i in mine:
        r, k = random_state(dims[i], 1000 + i)
        rho = O.stationary_state(O.left_canonical_q(r, k), r)
        results[i] = float(np.trace(rho).real)
    gathered = [None] * world
    dist.all_gather_object(gathered, results)
    if rank == 0:
        merged = {}
        for part in gathered:
            merged.update(part)
        out.put(merged)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_covers_every_state_once_and_balances():
    dims = [16, 32, 48, 64, 96, 128] * 5
    parts = [shard(dims, r, 4) for r in range(4)]
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(dims)))
    loads = [sum(dims[i] ** 3 for i in p) for p in parts]
    assert max(loads) / min(loads) < 1.2
    with pytest.raises(ValueError):
        shard(dims, 4, 4)


def test_two_gloo_ranks_evaluate_disjoint_shards():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    dims = [4, 6, 8, 5, 7, 3]
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, dims, out)) for r in range(2)]
    for p in procs:
        p.start()
    merged = out.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert sorted(merged) == list(range(len(dims)))
    assert all(abs(v - 1.0) < 1e-12 for v in merged.values())
