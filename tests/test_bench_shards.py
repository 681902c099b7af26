# SPDX-License-Identifier: Apache-2.0
"""The bench's world shards of the pour (the layout `bench.py --gpus N` steps, one shard per rank), on CPU: every
world lands in exactly one shard, each shard's particles, spouts and moving bowls are its worlds' own, renumbered
consistently, and the shards' liquid adds up to the whole scene's."""

from __future__ import annotations

import numpy as np

import bench
from alloy_b200.solvers.sph.sharding import shard_worlds
from alloy_b200.solvers.sph.testing import pour_bowls


def test_pour_shards_partition_the_worlds():
    sc = pour_bowls(worlds=12, device="cpu")
    full = sc.model.host()
    ws = np.asarray(full["world_start"], np.int64)
    shards = shard_worlds(np.diff(ws), 3)
    assert sorted(w for s in shards for w in s) == list(range(12))
    fluid = 0
    for r, mine in enumerate(shards):
        s = bench.worlds_scene(sc, mine, "cpu", f"shard{r}")
        h = s.model.host()
        sws = np.asarray(h["world_start"], np.int64)
        assert len(sws) == len(mine) + 1
        for k, w in enumerate(mine):  # the world's particles, in order
            np.testing.assert_array_equal(h["q"][sws[k]:sws[k + 1]], full["q"][ws[w]:ws[w + 1]])
            np.testing.assert_array_equal(h["phase"][sws[k]:sws[k + 1]], full["phase"][ws[w]:ws[w + 1]])
        m, fm = s.motion, sc.motion
        for k, w in enumerate(mine):  # the world's bowl particles, renumbered, with its own path
            sel = m.wall_world == k
            np.testing.assert_array_equal(m.wall_index[sel] - sws[k], fm.wall_index[fm.wall_world == w] - ws[w])
            np.testing.assert_array_equal(m.direction[k], fm.direction[w])
            assert m.phase[k] == fm.phase[w]
        assert np.all(np.diff(m.wall_world) >= 0)
        for e in s.emitters:  # each spout's pool inside its (renumbered) world
            pool = np.asarray(e["pool"])
            assert np.all((pool >= sws[e["world"]]) & (pool < sws[e["world"] + 1]))
        assert len(s.emitters) == sum(1 for e in sc.emitters if e["world"] in mine)
        fluid += s.fluid_count
    assert fluid == int(np.sum(full["phase"] >= 1))
