# SPDX-License-Identifier: Apache-2.0
"""The resting-jitter rule (solve_driver.py:1-118) on the CUDA path against the oracle, bit for bit: the per-world
flow sums of the step's start velocity, the head sums of the density warm starts, the tolerance factor and every
stop test that uses it.

- primed resting columns of 8 and 25 layers in box tanks (the reference's scene, tests/solvers/sph/
  test_jitter_rule.py:21-36), the default config (projected CG, run as one persistent launch per solve): 25 steps,
  the reported tolerance, iterations and errors every step, the state every 5;
- the same with relaxed Jacobi and a sideways kick, so that the flow allowance decides the tolerance;
- the reference's dam break of the speed harness at a small size (default config, the rule on, the liquid flowing).
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.build import add_box_tank, add_fluid_block
from alloy_b200.solvers.sph.config import DFSPHConfig
from alloy_b200.solvers.sph.model import ModelBuilder
from alloy_b200.solvers.sph.solver import hydrostatic_guess
from alloy_b200.solvers.sph.testing import tank_dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu

DT = 1.25e-3


def _columns(cfg, device, worlds=(8, 25)):
    s_ = cfg.spacing
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    for nz in worlds:
        b.begin_world()
        add_box_tank(b, (0.0, 0.0, 0.0), (6 * s_, 6 * s_, (nz + 6) * s_), wall=cfg.h)
        add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (6, 6, nz))
        b.end_world()
    return b.finalize(device)


def _lockstep(model, cfg, dt, steps, kick=0.0, prime=True, persistent=False):
    sol = SolverDFSPH(model, cfg)
    sol.persistent(persistent)
    orc = Oracle(model.host(), cfg)
    a, b = model.state(), model.state()
    if prime:
        guess = hydrostatic_guess(sol, a)
        sol.prime(a, dt)
        orc.set_warm(guess * np.float32(dt), orc.warm()[1])
        orc.prime(dt)
    if kick:
        qd = a.particle_qd.clone()
        qd[:, 0] += kick
        a.particle_qd.copy_(qd)
        orc.set_state(a.particle_q.cpu().numpy(), qd.cpu().numpy())
    tols = []
    for k in range(steps):
        sol.step(a, b, None, None, dt)
        a, b = b, a
        orc.step(dt)
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.density_tol, orep["density_tol"], err_msg=f"density_tol step {k}")
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.density_err.astype(np.float32), orep["density_err"], err_msg=f"step {k}")
        if (k + 1) % 5 == 0 or k == steps - 1:
            q, qd = orc.state()
            np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
            np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        tols.append(np.asarray(rep.density_tol, np.float64))
    return np.asarray(tols)


def test_jitter_rule_columns_cg_bit_exact(cuda):
    cfg = DFSPHConfig(particle_radius=2.0e-3)
    assert cfg.rest_jitter_speed and cfg.pressure_solver == "cg"
    tols = _lockstep(_columns(cfg, cuda), cfg, DT, 25, persistent=True)
    assert (tols[5:] < cfg.max_density_error).all()  # at rest the rule tightens every world's tolerance


def test_jitter_rule_flow_allowance_jacobi_bit_exact(cuda):
    cfg = DFSPHConfig(particle_radius=2.0e-3, pressure_solver="jacobi")
    tols = _lockstep(_columns(cfg, cuda), cfg, DT, 10, kick=0.02)
    assert tols[0].min() > cfg.rest_jitter_speed * DT / (25 * cfg.spacing) * 2.0  # the kick loosened it


def test_jitter_rule_harness_dam_break_bit_exact(cuda):
    sc = tank_dam_break(12, 10, 6, 30, r=2.0e-3, device=cuda)
    assert sc.config.rest_jitter_speed
    _lockstep(sc.model, sc.config, sc.dt, 20, prime=False)
