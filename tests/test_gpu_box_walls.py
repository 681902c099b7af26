# SPDX-License-Identifier: Apache-2.0
"""Static box walls on the CUDA path against the CPU oracle, bit for bit (boundary.py:190-396 slots from the SDF,
boundary_slots.py insertion with duplicate eviction, integrate.py:212-309 sweep and projection, pressure.py:393-458
lone-particle limit and friction).

- the slots of every liquid particle in the reference's box tank (walls h thick) after the first build: count, wall
  ids in order, Psi, phi, gradient and normal of each of the four slots;
- 25 steps of the box-tank dam break with Jacobi and with CG, state every 5 steps, iteration counts, per-world errors
  and the projection / sweep counters every step;
- the impact scene (liquid thrown into a corner, lone particles at 30 m/s past the CFL step and grazing the walls):
  10 steps, every step;
- two worlds mixing both wall kinds: particle walls with a box obstacle in one, a box tank in the other, and a global
  box seen by both; slots with the particle wall merged among the boxes.
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.build import add_box_tank, add_fluid_block, add_particle_box, wall_box
from alloy_b200.solvers.sph.model import ModelBuilder
from alloy_b200.solvers.sph.testing import Scene, benchmark_config, dam_break, tank_impacts
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _tank(device, solver="jacobi"):
    return dam_break(counts=(8, 8, 10), box=(0.2, 0.2, 0.24), walls="sdf", open_top=True, device=device,
                     pressure_solver=solver)


def _mixed(device):
    cfg = benchmark_config(0.02)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.begin_world()
    add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (8, 8, 8), jitter=0.01, seed=1)
    add_particle_box(b, cfg, (0.0, 0.0, 0.0), (0.2, 0.2, 0.3), open_top=True)
    wall_box(b, (0.1, 0.1, 0.05), (0.03, 0.03, 0.05), mu=0.5)  # an obstacle in the liquid
    b.end_world()
    b.begin_world()
    add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (7, 8, 9), jitter=0.01, seed=2)
    add_box_tank(b, (0.0, 0.0, 0.0), (0.2, 0.2, 0.3), wall=cfg.h, open_top=True, mu=0.3)
    b.end_world()
    wall_box(b, (0.02, 0.02, 0.0), (0.01, 0.01, 0.01), mu=0.8)  # global: every world sees it, after its own
    return Scene(b.finalize(device), cfg, 1.0e-3, 20, 0, 0, name="mixed_walls")


def _compare_slots(sol, orc, fluid, when):
    np.testing.assert_array_equal(sol.debug_field("slot_count")[fluid].astype(np.int32), orc.slot_on()[fluid],
                                  err_msg=f"slot count {when}")
    shapes = orc.slot_shapes()
    for k in range(4):
        np.testing.assert_array_equal(sol.debug_field(f"slot_shape:{k}")[fluid].astype(np.int32), shapes[fluid, k],
                                      err_msg=f"slot {k} walls {when}")
        for name in ("slot_psi", "slot_phi", "slot_g", "slot_n"):
            ours, ref = sol.debug_field(f"{name}:{k}"), orc.field(f"{name}:{k}")
            np.testing.assert_array_equal(ours[fluid], ref[fluid], err_msg=f"{name}:{k} {when}")


def _lockstep(sc, steps, every, cuda_solver=None):
    sol = cuda_solver or SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    for k in range(steps):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.density_err.astype(np.float32), orep["density_err"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.divergence_err.astype(np.float32), orep["divergence_err"],
                                      err_msg=f"step {k}")
        d = sol.diagnostics()
        np.testing.assert_array_equal(d["projected"], orep["projected"], err_msg=f"projected step {k}")
        np.testing.assert_array_equal(d["swept"], orep["swept"], err_msg=f"swept step {k}")
        if (k + 1) % every == 0 or k == steps - 1:
            q, qd = orc.state()
            np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
            np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
    return sol, orc


def test_box_tank_slots_bit_exact(cuda):
    sc = _tank(cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    fluid = sc.model.sph.phase.cpu().numpy() >= 1
    sol.density_ratio(sc.model.state())
    orc.prepare_density()
    _compare_slots(sol, orc, fluid, "first build")
    assert (orc.slot_on()[fluid] >= 2).any()  # corner and edge particles see two or three walls


@pytest.mark.parametrize("solver", ["jacobi", "cg"])
def test_box_tank_lockstep(cuda, solver):
    sc = _tank(cuda, solver)
    _, orc = _lockstep(sc, 25, 5)
    assert orc.report()["projected"][0] >= 0


def test_impacts_lockstep_projection_and_sweep(cuda):
    sc = tank_impacts(device=cuda)
    sol, orc = _lockstep(sc, 10, 1)
    rep = orc.report()
    assert rep["projected"][0] > 0 and rep["swept"][0] > 0  # both wall paths ran


def test_mixed_walls_slots_and_steps(cuda):
    sc = _mixed(cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    fluid = sc.model.sph.phase.cpu().numpy() >= 1
    sol.density_ratio(sc.model.state())
    orc.prepare_density()
    _compare_slots(sol, orc, fluid, "first build")
    shapes = orc.slot_shapes()[fluid]
    S = len(sc.model.host()["shape_type"])
    assert ((shapes == S).any(1) & ((shapes >= 0) & (shapes < S)).any(1)).any()  # particle wall among boxes
    _lockstep(sc, 20, 5)
