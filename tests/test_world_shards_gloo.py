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


def _scene(kind: str = "particles"):
    if kind == "sdf":  # box-tank columns of different heights and a global box every world sees
        from alloy_b200.solvers.sph.build import add_box_tank, add_fluid_block, wall_box
        from alloy_b200.solvers.sph.model import ModelBuilder
        from alloy_b200.solvers.sph.testing import Scene, benchmark_config

        cfg = benchmark_config(0.02)
        b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
        for w in range(5):
            b.begin_world()
            add_box_tank(b, (0.0, 0.0, 0.0), (0.12, 0.12, 0.3), wall=cfg.h)
            add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (6, 6, 4 + w), jitter=0.01, seed=w)
            b.end_world()
        wall_box(b, (0.06, 0.06, 0.0), (0.01, 0.01, 0.01), mu=0.5)
        return Scene(b.finalize("cpu"), cfg, 1.0e-3, STEPS, 0, 0, name="sdf_columns")
    return batched_worlds(worlds=6, lo=150, hi=700, seed=5)


def _rank(rank: int, world: int, port: int, out: str, kind: str = "particles"):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from oracle.pyoracle import Oracle

        sc = _scene(kind)
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
@pytest.mark.parametrize("kind", ["particles", "sdf"])
def test_two_gloo_ranks_step_disjoint_world_shards_bitwise(tmp_path, kind):
    """Particle-wall worlds, and box-tank worlds whose shards carry their own boxes and the global one."""
    out = str(tmp_path / "merged.pkl")
    mp.start_processes(_rank, args=(2, _free_port(), out, kind), nprocs=2, join=True, start_method="spawn")
    with open(out, "rb") as f:
        merged = pickle.load(f)
    from oracle.pyoracle import Oracle

    sc = _scene(kind)
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
