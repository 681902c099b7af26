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
        assert c["block"] in (128, 256) and c["nb"] in (4, 8, 16) and c["ms"] > 0.0, (name, c)
    for c in c1.values():
        assert c == {"block": 256, "nb": 8, "ms": -1.0}
