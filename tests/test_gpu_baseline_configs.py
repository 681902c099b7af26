# SPDX-License-Identifier: Apache-2.0
"""GPU parity on the benchmark configurations themselves, against the CPU oracle, bit for bit.

- The single-world dam break as specified: 20 x 20 x 20 = 8,000 liquid particles at 0.02 m with +-1 % seeded
  jitter in the corner of a 1 x 1 x 1 m box of one layer of boundary particles, Jacobi, tolerances 1e-3, dt 1 ms,
  200 steps. Iteration counts and per-world errors every step, positions and velocities every 10 steps.
- The 1,048,576-particle dam break (128 x 64 x 128 at 0.01 m in a 4 x 2 x 2 m tank): neighbour rows and counts after
  the first build and again after 5 steps. Its world holds more than 65,536 particles (the reference's 24-bit
  offsets, neighbors.py:15-17) and runs the Jacobi path.
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import dam_break, large_dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def test_single_world_dam_break_200_steps_bit_exact(cuda):
    sc = dam_break(device=cuda)
    assert (sc.fluid_count, sc.steps, sc.dt, sc.config.pressure_solver) == (8000, 200, 1.0e-3, "jacobi")
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    for k in range(sc.steps):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        rep, orep = sol.report(), orc.report()
        assert int(rep.iters_density[0]) == orep["iters_density"][0], k
        assert int(rep.iters_divergence[0]) == orep["iters_divergence"][0], k
        assert rep.density_err[0] == orep["density_err"][0], k
        assert rep.divergence_err[0] == orep["divergence_err"][0], k
        if (k + 1) % 10 == 0:
            q, qd = orc.state()
            np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
            np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
    assert int(rep.neighbor_overflow[0]) == 0


def _rows_equal(sol, orc, fluid, when: str):
    rows, cnt = sol.neighbor_rows()
    orows, ocnt = orc.lists()
    np.testing.assert_array_equal(cnt, ocnt, err_msg=f"counts {when}")
    assert cnt[fluid].min() > 0 and cnt[~fluid].max() == 0
    np.testing.assert_array_equal(rows, orows, err_msg=f"rows {when}")


def test_million_particle_rows_bit_exact(cuda):
    sc = large_dam_break(device=cuda)
    assert sc.fluid_count == 1_048_576 and sc.config.pressure_solver == "jacobi"
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    fluid = sc.model.sph.phase.cpu().numpy() >= 1
    a, b = sc.model.state(), sc.model.state()
    sol.density_ratio(a)
    orc.prepare_density()
    _rows_equal(sol, orc, fluid, "first build")
    for k in range(5):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
    q, qd = orc.state()
    np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q)
    np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd)
    sol.density_ratio(a)
    orc.prepare_density()
    _rows_equal(sol, orc, fluid, "after 5 steps")
