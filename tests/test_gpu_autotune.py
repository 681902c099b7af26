# SPDX-License-Identifier: Apache-2.0
"""The autotuner: the tuning step computes exactly an ordinary step (its trials are idempotent or restored), every
tuned kernel reports a measured configuration from the candidate set, and a tuned solver and an untuned one stay
bit-identical over the following graph-replayed steps (the configuration changes launch shapes, never sums)."""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import batched_worlds

pytestmark = pytest.mark.gpu


def test_tuned_and_untuned_solvers_agree_bit_for_bit(cuda):
    runs = []
    for tune in (True, False):
        sc = batched_worlds(worlds=4, lo=1500, hi=6000, seed=5, device=cuda)
        sol = SolverDFSPH(sc.model, sc.config)
        sol.autotune(tune)
        a, b = sc.model.state(), sc.model.state()
        for _ in range(6):
            sol.step(a, b, None, None, sc.dt)
            a, b = b, a
        cfg = sol.tuned_configs()
        r = sol.report()
        runs.append((a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy(), r.iters_density.copy(),
                     r.iters_divergence.copy(), cfg))
    (q0, v0, d0, e0, c0), (q1, v1, d1, e1, c1) = runs
    np.testing.assert_array_equal(q0, q1)
    np.testing.assert_array_equal(v0, v1)
    np.testing.assert_array_equal(d0, d1)
    np.testing.assert_array_equal(e0, e1)
    for name, c in c0.items():
        if name == "lists":
            assert c["block"] == 128 and c["nb"] in (16, 32) and c["ms"] > 0.0, c
        else:
            assert c["block"] in (128, 256) and c["nb"] in (4, 8, 16) and c["ms"] > 0.0, (name, c)
    for name, c in c1.items():
        assert c == ({"block": 128, "nb": 32, "ms": -1.0} if name == "lists" else {"block": 256, "nb": 8, "ms": -1.0})


@pytest.mark.parametrize("ppw", [16, 32])
def test_list_build_rows_equal_the_oracle_at_either_particles_per_warp(cuda, ppw):
    """16 particles per warp (two lanes per particle, merged half-rows) and 32 give the oracle's rows bit for bit, on
    uneven worlds and on a capacity that overflows."""
    from oracle.pyoracle import Oracle

    for sc in (batched_worlds(worlds=4, lo=700, hi=3000, seed=9, device=cuda),
               batched_worlds(worlds=2, lo=500, hi=900, seed=2, device=cuda, neighbor_capacity=24)):
        sol = SolverDFSPH(sc.model, sc.config)
        sol.autotune(False)
        sol.set_tuned_config("lists", 128, ppw)
        orc = Oracle(sc.model.host(), sc.config)
        a, b = sc.model.state(), sc.model.state()
        for k in range(5):
            sol.step(a, b, None, None, sc.dt)
            a, b = b, a
            orc.step(sc.dt)
            rows, cnt = sol.neighbor_rows()
            orows, ocnt = orc.lists()
            np.testing.assert_array_equal(cnt, ocnt, err_msg=f"step {k}")
            np.testing.assert_array_equal(rows, orows, err_msg=f"step {k}")
            np.testing.assert_array_equal(sol.report().neighbor_overflow, orc.report()["neighbor_overflow"])
        q, _ = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q)
