"""Instance sharding of a batch across ranks (CPU; gloo, world size 2).

The batch path shards independent LPs over ranks with no data-path
collective; only the final results are gathered on rank 0. These tests run
the host logic without a GPU: the device solve is replaced by a fake that
returns a value derived from the instance.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from nirnaya_b200 import batch as B
from nirnaya_b200 import lp as L


def test_shards_cover_every_instance_once_and_balance():
    rng = np.random.default_rng(0)
    work = rng.integers(1, 10_000, size=257).tolist()
    for world in (1, 2, 3, 8):
        shards = B.shard_instances(work, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(work)))
        loads = [sum(work[i] for i in s) for s in shards]
        # LPT bound: max load <= mean + largest item
        assert max(loads) <= sum(work) / world + max(work)
        assert shards == B.shard_instances(work, world)  # deterministic


def test_shards_with_more_ranks_than_instances():
    shards = B.shard_instances([5, 3], 4)
    assert sorted(len(s) for s in shards) == [0, 0, 1, 1]
    with pytest.raises(ValueError):
        B.shard_instances([1], 0)


def _fake_solve(lps):
    return [(float(lp.nnz) + 0.5 * lp.nrow, 0, lp.ncol) for lp in lps]


def _rank_main(rank, world, port, out_path):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        lps = [L.generate(L.RANDOM_EQ, 100 + i, m=20 + 7 * i, n=50 + 11 * i) for i in range(9)]
        got = B.solve_sharded(lps, rank, world, solve_fn=_fake_solve)
        if rank == 0:
            want = {i: v for i, v in enumerate(_fake_solve(lps))}
            ok = got == want
            with open(out_path, "w") as f:
                f.write("ok" if ok else f"mismatch {got} {want}")
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_sharded_solve_gathers_on_rank0(tmp_path):
    out = tmp_path / "result.txt"
    mp.start_processes(_rank_main, args=(2, _free_port(), str(out)), nprocs=2, join=True, start_method="spawn")
    assert out.read_text() == "ok"
