# SPDX-License-Identifier: Apache-2.0
"""Item halos of the Jacobi iterations: the pressure acceleration (pressure.py:264-291) and the Jacobi update
(pressure.py:294-352) gather each 256-particle work item's neighbours from shared memory, through rows rewritten as
16-bit indices into the item's list of distinct neighbours, instead of from the particle arrays.

- bit for bit against the global gathers (positions, velocities, warm starts, per-world iterations and errors every
  step): a dam break in a tank of boundary particles, replayed as CUDA graphs and launched eagerly; uneven batched
  worlds with spouts (items end at world ends, active sets change); a dam break in a box tank (four wall slots);
- bit for bit against the CPU oracle on the dam break with the halos forced on;
- the halo statistics: items staged, none left out at these sizes, at most 1,280 records an item;
- off by default; with -1 the autotuner times both forms and keeps one.
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.solver import layer_offsets
from alloy_b200.solvers.sph.testing import batched_worlds, dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _spouts(sc, sol):
    arr = sc.model.host()
    for e in sc.emitters:
        w = e["world"]
        i0 = int(arr["world_start"][w])
        vol = float(arr["mass"][i0]) / float(arr["rest_density"][i0])
        offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64),
                             sc.config.spacing)
        sol.add_emitter(w, e["centre"], e["half"], len(offs) * vol / (10.0 * sc.dt), e["velocity"], pool=e["pool"])


def _lockstep(make, steps, graphs=True, spouts=False):
    """Staged and global gathers side by side, each solver on its own model."""
    scenes = [make(), make()]
    sc = scenes[0]
    sols = [SolverDFSPH(x.model, x.config) for x in scenes]
    sols[0].halo(1)
    sols[1].halo(0)
    states = [[x.model.state(), x.model.state()] for x in scenes]
    for sol, x in zip(sols, scenes):
        sol.use_graphs(graphs)
        if spouts:
            _spouts(x, sol)
    for k in range(steps):
        for sol, st in zip(sols, states):
            sol.step(st[0], st[1], None, None, sc.dt)
            st.reverse()
        r0, r1 = sols[0].report(), sols[1].report()
        (a, _), (c, _) = states
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), c.particle_q.cpu().numpy(), err_msg=f"q {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), c.particle_qd.cpu().numpy(), err_msg=f"qd {k}")
        for f in ("iters_density", "iters_divergence", "density_err", "divergence_err"):
            np.testing.assert_array_equal(getattr(r0, f), getattr(r1, f), err_msg=f"{f} step {k}")
    s0, s1 = sols[0].alloy_state_arrays(), sols[1].alloy_state_arrays()
    for key in ("sph.kappa_v", "sph.kappa_d"):
        np.testing.assert_array_equal(s0[key].cpu().numpy(), s1[key].cpu().numpy(), err_msg=key)
    stats = sols[0].halo_stats()
    assert stats["accel"] and stats["jacobi"]
    assert not sols[1].halo_stats()["jacobi"]
    return stats


@pytest.mark.parametrize("graphs", [True, False])
def test_halo_dam_break_equals_global_gathers(cuda, graphs):
    st = _lockstep(lambda: dam_break(counts=(16, 12, 18), box=(0.5, 0.4, 0.6), device=cuda), 25, graphs)
    assert st["staged"] >= 14 and st["global"] == 0  # 3,456 liquid particles: 14 items
    assert 256 < st["max_records"] <= 1280


def test_halo_batched_worlds_with_spouts_equal_global_gathers(cuda):
    st = _lockstep(lambda: batched_worlds(worlds=6, lo=400, hi=3000, seed=6, device=cuda), 30, spouts=True)
    assert st["staged"] >= 6 and st["global"] == 0


def test_halo_box_tank_walls_equal_global_gathers(cuda):
    _lockstep(lambda: dam_break(counts=(12, 10, 14), box=(0.4, 0.3, 0.5), walls="sdf", device=cuda), 20)


def test_halo_dam_break_equals_oracle(cuda):
    sc = dam_break(counts=(14, 10, 16), box=(0.5, 0.4, 0.6), device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    sol.halo(1)
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    for k in range(15):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
    assert sol.halo_stats()["staged"] > 0


def test_autotuner_times_both_forms(cuda):
    sc = dam_break(counts=(16, 12, 18), box=(0.5, 0.4, 0.6), device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    assert not sol.halo_stats()["jacobi"]
    sol.halo(-1)
    sol.autotune(True)
    a, b = sc.model.state(), sc.model.state()
    for _ in range(3):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
    st = sol.halo_stats()
    assert isinstance(st["accel"], bool) and isinstance(st["jacobi"], bool)
    if st["accel"] or st["jacobi"]:
        assert st["staged"] > 0
    with pytest.raises(ValueError, match="adf_set_halo"):
        sol.halo(2)
