# SPDX-License-Identifier: Apache-2.0
"""The seeded workload scenes: the first k worlds of a multi-world build are the same worlds as a k-world build
(sizes, particles, bowl paths and phases, spouts), which the FP64 check (16 worlds) and the CPU baseline (256 worlds)
of the pour workload rely on."""

from __future__ import annotations

import numpy as np

from alloy_b200.solvers.sph.testing import batched_worlds, pour_bowls


def _prefix_equal(small, big):
    hs, hb = small.model.host(), big.model.host()
    n = int(hs["world_start"][-1])
    for k in ("q", "qd", "mass", "flags", "phase", "world", "radius"):
        np.testing.assert_array_equal(hs[k], hb[k][:n], err_msg=k)
    for es, eb in zip(small.emitters, big.emitters):
        assert es["world"] == eb["world"] and np.array_equal(es["pool"], eb["pool"])


def test_pour_first_worlds_are_the_workloads_worlds():
    small, big = pour_bowls(worlds=5, device="cpu"), pour_bowls(worlds=12, device="cpu")
    _prefix_equal(small, big)
    np.testing.assert_array_equal(small.motion.phase, big.motion.phase[:5])
    np.testing.assert_array_equal(small.motion.direction, big.motion.direction[:5])
    sel = big.motion.wall_world < 5
    np.testing.assert_array_equal(small.motion.wall_index, big.motion.wall_index[sel])
    np.testing.assert_array_equal(small.motion.host_velocities(0.37, 1e-3), big.motion.host_velocities(0.37, 1e-3)
                                  [: len(small.motion.wall_index)])


def test_batched_first_worlds_are_the_workloads_worlds():
    _prefix_equal(batched_worlds(worlds=4, device="cpu"), batched_worlds(worlds=9, device="cpu"))
