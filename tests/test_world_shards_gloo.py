# SPDX-License-Identifier: Apache-2.0
"""World sharding across ranks (the multi-GPU layout of batched worlds), exercised on CPU with two gloo ranks: each
rank steps only its shard of worlds (the oracle stands in for the GPU step), the only collective is a gather of the
per-world report at the end, and every world's particles match a one-process run of all worlds bit for bit."""

from __future__ import annotations

import os
import pickle
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from alloy_b200.solvers.sph.sharding import shard_worlds, sub_arrays
from alloy_b200.solvers.sph.testing import batched_worlds

STEPS = 8


def _scene():
    return batched_worlds(worlds=6, lo=150, hi=700, seed=5)


def _rank(rank: int, world: int, port: int, out: str):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.pyoracle import Oracle

        sc = _scene()
        arr = sc.model.host()
        ws = arr["world_start"]
        parts = shard_worlds(np.diff(ws), world)
        mine = parts[rank]
        o = Oracle(sub_arrays(arr, mine), sc.config, threads=1)
        for _ in range(STEPS):
            o.step(sc.dt)
        q, _ = o.state()
        sws = np.concatenate([[0], np.cumsum([ws[w + 1] - ws[w] for w in mine])])
        res = {w: (q[sws[k]:sws[k + 1]].tobytes(), int(o.report()["iters_density"][k])) for k, w in enumerate(mine)}
        gathered = [None] * world if rank == 0 else None
        dist.gather_object(res, gathered, dst=0)
        if rank == 0:
            merged = {}
            for g in gathered:
                merged.update(g)
            with open(out, "wb") as f:
                pickle.dump(merged, f)
    finally:
        dist.destroy_process_group()


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.timeout(300)
def test_two_gloo_ranks_step_disjoint_world_shards_bitwise(tmp_path):
    out = str(tmp_path / "merged.pkl")
    mp.start_processes(_rank, args=(2, _free_port(), out), nprocs=2, join=True, start_method="spawn")
    with open(out, "rb") as f:
        merged = pickle.load(f)
    from oracle.pyoracle import Oracle

    sc = _scene()
    arr = sc.model.host()
    o = Oracle(arr, sc.config, threads=1)
    for _ in range(STEPS):
        o.step(sc.dt)
    qa, _ = o.state()
    ws = arr["world_start"]
    assert sorted(merged) == list(range(len(ws) - 1))
    for w in range(len(ws) - 1):
        assert merged[w][0] == qa[ws[w]:ws[w + 1]].tobytes(), w
        assert merged[w][1] == int(o.report()["iters_density"][w])
