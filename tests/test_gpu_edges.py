# SPDX-License-Identifier: Apache-2.0
"""Edge cases of the CUDA path against the oracle, bit for bit: worlds without liquid (walls only, spares only) beside
a liquid world, a model without particles, neighbour rows that overflow a small capacity (lowest ids kept, overflow
counted, neighbors.py:131-195), the shared-memory list path of capacities above 64, the Wendland C2 kernel, a sink
emptying liquid into the ledger (then reset restores flags, phase and warm starts of the masked worlds), and walls dense
enough that some liquid particles' wall slots are done by one lane instead of a team of four."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.build import add_fluid_block, add_particle_box, add_spares, add_wall_particles, box_shell_points
from alloy_b200.solvers.sph.model import ModelBuilder
from alloy_b200.solvers.sph.solver import _xform7
from alloy_b200.solvers.sph.testing import benchmark_config, dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _lockstep(model, cfg, dt, steps, setup=None):
    sol = SolverDFSPH(model, cfg)
    orc = Oracle(model.host(), cfg)
    if setup is not None:
        setup(sol, orc)
    a, b = model.state(), model.state()
    for k in range(steps):
        sol.step(a, b, None, None, dt)
        a, b = b, a
        orc.step(dt)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.neighbor_overflow, orep["neighbor_overflow"], err_msg=f"step {k}")
    return sol, orc, a


def test_worlds_without_liquid_beside_a_liquid_world(cuda):
    cfg = benchmark_config(0.02)
    b = ModelBuilder()
    b.begin_world()  # liquid in a box
    add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (6, 5, 7), jitter=0.01, seed=1)
    add_particle_box(b, cfg, (0.0, 0.0, 0.0), (0.3, 0.3, 0.3))
    b.end_world()
    b.begin_world()  # walls only
    add_particle_box(b, cfg, (0.0, 0.0, 0.0), (0.2, 0.2, 0.2))
    b.end_world()
    b.begin_world()  # spares only
    add_spares(b, cfg, 40)
    b.end_world()
    sol, orc, _ = _lockstep(b.finalize(cuda), cfg, 1.0e-3, 10)
    rep = sol.report()
    assert rep.iters_density[0] >= 2 and (rep.iters_density[1:] == 0).all()
    assert (rep.density_err[1:] == 0).all() and (rep.mass_active[1:] == 0).all()


def test_model_without_particles(cuda):
    cfg = benchmark_config(0.02)
    b = ModelBuilder()
    b.begin_world()
    b.end_world()
    model = b.finalize(cuda)
    sol = SolverDFSPH(model, cfg)
    s = model.state()
    sol.step(s, s, None, None, 1.0e-3)  # returns at once (solver.py:218-224)
    with pytest.raises(ValueError):
        sol.step(s, s, None, None, 0.0)


@pytest.mark.parametrize("capacity", [16, 96])
def test_row_capacity_overflow_and_wide_rows_bit_exact(cuda, capacity):
    """16: rows overflow (about 29 neighbours at h = 2 spacings), the lowest ids are kept and the overflow counted;
    96: rows longer than 64 entries are built by the shared-memory list kernel."""
    sc = dam_break(counts=(10, 8, 9), box=(0.4, 0.4, 0.4), device=cuda, neighbor_capacity=capacity)
    sol, orc, _ = _lockstep(sc.model, sc.config, sc.dt, 8)
    rows, cnt = sol.neighbor_rows()
    orows, ocnt = orc.lists()
    np.testing.assert_array_equal(cnt, ocnt)
    np.testing.assert_array_equal(rows, orows)
    ov = sol.report().neighbor_overflow
    assert (ov > 0).all() if capacity == 16 else (ov == 0).all()


def test_wendland_kernel_bit_exact(cuda):
    sc = dam_break(counts=(9, 8, 10), box=(0.4, 0.4, 0.4), device=cuda, kernel="wendland_c2")
    _lockstep(sc.model, sc.config, sc.dt, 12)


def test_sink_ledger_and_reset(cuda):
    sc = dam_break(counts=(8, 8, 10), box=(0.4, 0.4, 0.4), device=cuda)
    region, half = (0.08, 0.08, 0.02, 0.0, 0.0, 0.0, 1.0), (0.1, 0.1, 0.03)

    def sinks(sol, orc):
        sol.add_sink(0, region, half)
        orc.add_sink(0, _xform7(region), np.asarray(half, np.float32))

    sol, orc, a = _lockstep(sc.model, sc.config, sc.dt, 20, sinks)
    led = sol.mass_ledger()
    orep = orc.report()
    assert int(led["out"][0]) > 0
    np.testing.assert_array_equal(led["out"], orep["mass_out"])
    np.testing.assert_array_equal(led["active"] + led["out"], led["initial"] + led["in"])

    def live():
        return int((((sc.model.particle_flags & 1) != 0) & (sc.model.sph.phase >= 1)).sum())

    assert live() < sc.fluid_count  # the sink retired liquid
    sol.reset(a, world_mask=np.array([1], np.uint8))
    torch.cuda.synchronize()
    assert live() == sc.fluid_count
    assert int(sol.mass_ledger()["out"][0]) == 0
    assert (sol.alloy_state_arrays()["sph.kappa_d"] == 0).all()


def test_capability_factory_builds_a_working_solver(cuda):
    """The router's path (plugin.py:36-61): the sph capability's factory from config fields, with the automatic
    escape box, steps like a solver built directly."""
    from alloy_b200.solvers.sph.plugin import CAPABILITY

    sc = dam_break(counts=(6, 6, 6), box=(0.3, 0.3, 0.3), device=cuda)
    sol = CAPABILITY.factory(sc.model, {"particle_radius": 0.01, "pressure_solver": "jacobi", "rest_jitter_speed": None,
                                        "xsph_c": 0.01, "viscosity": "xsph"})
    assert sol.config.world_bounds is not None and sol.escape_box_pad >= 0.25
    a, b = sc.model.state(), sc.model.state()
    for _ in range(3):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
    r = sol.report()
    assert r.iters_density[0] >= 2 and r.escaped[0] == 0


def test_dense_walls_take_the_one_lane_wall_slot_path(cuda):
    """Walls of boundary particles at half the liquid spacing: liquid particles near an edge or corner see more than 48
    wall particles within h, which the four-lane wall-slot teams leave to one lane; both paths agree with the oracle."""
    cfg = benchmark_config(0.02)
    s = cfg.spacing
    b = ModelBuilder()
    b.begin_world()
    add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (6, 6, 6), jitter=0.01, seed=3)
    add_wall_particles(b, cfg, box_shell_points((0.0, 0.0, 0.0), (8 * s, 8 * s, 10 * s), 0.5 * s), spacing=0.5 * s)
    b.end_world()
    model = b.finalize(cuda)
    host = model.host()
    q = host["q"].reshape(-1, 3)
    fl, wl = host["phase"] >= 1, host["phase"] == -1
    d2 = ((q[fl][:, None, :] - q[wl][None, :, :]) ** 2).sum(-1)
    assert ((d2 < cfg.h * cfg.h).sum(1) > 48).any()  # some liquid particle takes the one-lane path
    _lockstep(model, cfg, 1.0e-3, 8)
