# SPDX-License-Identifier: Apache-2.0
"""Verlet-skin reuse of the neighbour rows (neighbors_skin.py, Config.reneighbor_skin) on the GPU. The reference
states its contract as "results bitwise the same" as building every step (config.py:78-80, neighbors_skin.py:14-17):

- a dam break in the box tank with skin 0.1 h against the oracle (which builds every step): rows, counts, state and
  iteration counts bit for bit;
- resting columns in box tanks, primed: the skin solver and a plain solver stepped side by side give the same bits,
  and after the first step most steps rebuild no world;
- superset rows far too small for the fill (every row overfull): each is written as a plain row and its world
  rebuilds the next step, still bit for bit.
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import dam_break, water_column
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _tank(device, skin=0.1, solver="jacobi"):
    return dam_break(counts=(8, 8, 10), box=(0.2, 0.2, 0.24), walls="sdf", open_top=True, device=device,
                     pressure_solver=solver, reneighbor_skin=skin)


def _rows_equal(sol, orc, when):
    rows, cnt = sol.neighbor_rows()
    orows, ocnt = orc.lists()
    np.testing.assert_array_equal(cnt, ocnt, err_msg=f"counts {when}")
    np.testing.assert_array_equal(rows, orows, err_msg=f"rows {when}")


@pytest.mark.parametrize("skin_rows", [None, 8])
def test_skin_dam_break_bit_exact_against_plain_build(cuda, skin_rows):
    sc = _tank(cuda)
    sol = SolverDFSPH(sc.model, sc.config, skin_rows=skin_rows)
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    rebuilt = []
    for k in range(30):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        rebuilt.append(bool(sol.skin_flags()[0]))
        np.testing.assert_array_equal(sol.report().iters_density, orc.report()["iters_density"], err_msg=f"step {k}")
        if k % 5 == 4:
            _rows_equal(sol, orc, f"step {k}")
            q, qd = orc.state()
            np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
            np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
    assert rebuilt[0]  # nothing was built before the first step
    if skin_rows is not None:  # every superset row overflows: a plain row each step and a forced rebuild
        assert all(rebuilt)


def test_skin_resting_columns_reuse_rows(cuda):
    sc = water_column(8, 8, 12, worlds=3, r=2.0e-3, device=cuda, reneighbor_skin=0.1)
    plain_cfg = type(sc.config)(**{**sc.config.__dict__, "reneighbor_skin": None})
    skin, plain = SolverDFSPH(sc.model, sc.config), SolverDFSPH(sc.model, plain_cfg)
    a, b = sc.model.state(), sc.model.state()
    c, d = sc.model.state(), sc.model.state()
    skin.prime(a, sc.dt)
    plain.prime(c, sc.dt)
    flags = []
    for k in range(40):
        skin.step(a, b, None, None, sc.dt)
        plain.step(c, d, None, None, sc.dt)
        a, b, c, d = b, a, d, c
        flags.append(skin.skin_flags())
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), c.particle_q.cpu().numpy(), err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), c.particle_qd.cpu().numpy(), err_msg=f"qd {k}")
    rows, cnt = skin.neighbor_rows()
    prow, pcnt = plain.neighbor_rows()
    np.testing.assert_array_equal(cnt, pcnt)
    np.testing.assert_array_equal(rows, prow)
    flags = np.asarray(flags)  # the prime built every world's rows before the first step
    assert flags.mean() < 0.5, flags.astype(int)  # at rest most steps reuse the rows
