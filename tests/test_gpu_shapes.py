# SPDX-License-Identifier: Apache-2.0
"""Static shapes other than axis-aligned boxes on the CUDA path against the CPU oracle, bit for bit: spheres, capsules,
straight cylinders, planes (finite and infinite) and turned boxes, each in its own frame, through newton's
closed-form distances (boundary.py:190-396 slots, integrate.py:98-115 the sampled sweep of non-box shapes and the slab
test of boxes in their frame, integrate.py:212-309 the projection with friction).

- the slots of every liquid particle of the obstacle scene after the first build, with the liquid moved onto the
  shapes: count, wall ids in order, Psi, phi, gradient and normal of each slot;
- 20 steps of the obstacle scene with Jacobi and with CG: a block falling onto a sphere and a capsule on the ground
  plane beside a finite shelf, a turned box and a lying cylinder, and lone particles at 30 m/s swept into them; the
  state, iteration counts, per-world errors and the projection and sweep counters every step.
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import shape_obstacles
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def test_obstacle_slots_bit_exact(cuda):
    sc = shape_obstacles(device=cuda)
    q = sc.model.particle_q.clone()
    fluid = (sc.model.sph.phase.cpu().numpy() >= 1)
    # move the block's particles onto the shapes: rings around the sphere, the capsule, the lying cylinder and the
    # turned box, and a layer on the ground under the shelf
    idx = np.flatnonzero(fluid)[:180]
    k = np.arange(len(idx))
    ang = 2.0 * np.pi * k / 23.0
    pts = np.stack([0.15 + 0.062 * np.cos(ang), 0.15 + 0.062 * np.sin(ang), 0.03 + 0.01 * (k % 9)], 1)
    c, s_ = np.cos(ang), np.sin(ang)
    pts[36:72] = np.stack([0.07 + 0.04 * c[36:72], 0.22 + 0.04 * s_[36:72], 0.02 + 0.012 * (k[36:72] % 13)], 1)
    pts[72:108] = np.stack([0.06 + 0.027 * c[72:108], 0.04 + 0.008 * (k[72:108] % 11),
                            0.03 + 0.027 * np.abs(s_[72:108])], 1)
    pts[108:144] = np.stack([0.24 + 0.045 * c[108:144], 0.22 + 0.045 * s_[108:144], 0.02 + 0.01 * (k[108:144] % 8)], 1)
    pts[144:] = np.stack([0.22 + 0.006 * (k[144:] % 10), 0.04 + 0.006 * (k[144:] // 10 % 4), 0.004 + 0.0 * k[144:]], 1)
    q[idx] = torch_tensor(pts, cuda)
    sc.model.particle_q.copy_(q)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    sol.density_ratio(sc.model.state())
    orc.prepare_density()
    np.testing.assert_array_equal(sol.debug_field("slot_count")[fluid].astype(np.int32), orc.slot_on()[fluid])
    shapes = orc.slot_shapes()
    for s in range(4):
        np.testing.assert_array_equal(sol.debug_field(f"slot_shape:{s}")[fluid].astype(np.int32), shapes[fluid, s],
                                      err_msg=f"slot {s} walls")
        for name in ("slot_psi", "slot_phi", "slot_g", "slot_n"):
            np.testing.assert_array_equal(sol.debug_field(f"{name}:{s}")[fluid], orc.field(f"{name}:{s}")[fluid],
                                          err_msg=f"{name}:{s}")
    seen = set(shapes[fluid].ravel().tolist())
    assert {4, 5, 7, 8, 9} <= seen  # the sphere, the capsule, the turned box, the lying cylinder and the ground


def torch_tensor(a, device):
    import torch

    return torch.as_tensor(np.asarray(a, np.float32), device=device)


@pytest.mark.parametrize("solver", ["jacobi", "cg"])
def test_obstacle_lockstep_with_sweeps(cuda, solver):
    sc = shape_obstacles(device=cuda, pressure_solver=solver)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    swept = projected = 0
    for k in range(sc.steps):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.density_err.astype(np.float32), orep["density_err"], err_msg=f"step {k}")
        d = sol.diagnostics()
        np.testing.assert_array_equal(d["projected"], orep["projected"], err_msg=f"projected step {k}")
        np.testing.assert_array_equal(d["swept"], orep["swept"], err_msg=f"swept step {k}")
        swept += int(orep["swept"].sum())
        projected += int(orep["projected"].sum())
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
    assert swept >= 5 and projected > 0  # the sampled sweeps and the projections both ran
    assert (a.particle_q.cpu().numpy()[:, 2] > 0.0).all()  # nothing went through the ground
