# SPDX-License-Identifier: Apache-2.0
"""Hydrostatic priming (SolverDFSPH.prime, prime.py:52-87): the GPU prime equals the oracle's bit for bit (iteration
count, both warm starts; the state is left unchanged), the steps after it stay bit-exact, and a primed column at rest
has its pressure grow with depth."""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.solver import hydrostatic_guess
from alloy_b200.solvers.sph.testing import dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver", ["jacobi", "cg"])
def test_prime_bit_exact_and_steps_after(cuda, solver):
    sc = dam_break(counts=(8, 8, 16), box=(0.16, 0.16, 0.4), device=cuda, pressure_solver=solver)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    q0 = a.particle_q.cpu().numpy().copy()
    guess = hydrostatic_guess(sol, a)
    assert guess[: sc.fluid_count].max() > 0.0
    it = sol.prime(a, sc.dt)
    kv0, kd0 = orc.warm()
    orc.set_warm(guess * np.float32(sc.dt), kd0)
    it_o = orc.prime(sc.dt)
    assert it == it_o and it > 1
    kv, kd = orc.warm()
    arr = sol.alloy_state_arrays()
    np.testing.assert_array_equal(arr["sph.kappa_v"].cpu().numpy(), kv)
    np.testing.assert_array_equal(arr["sph.kappa_d"].cpu().numpy(), kd)
    assert (kv == 0).all() and kd[: sc.fluid_count].max() > 0.0
    np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q0)  # the state is untouched
    for k in range(8):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")


def test_primed_pressure_grows_with_depth(cuda):
    """The primed density warm start (kappa dt^2) is non-negative and grows with depth below the free surface: the
    divergence solve of one gravity step's velocity, started from the hydrostatic guess, keeps the deepest layers'
    pressure (at the reference's tolerance 1e-6 it does not propagate the full hydrostatic value up the column)."""
    sc = dam_break(counts=(8, 8, 24), box=(0.16, 0.16, 0.6), device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    a = sc.model.state()
    assert sol.prime(a, sc.dt) > 1
    kd = sol.alloy_state_arrays()["sph.kappa_d"].cpu().numpy()[: sc.fluid_count]
    z = a.particle_q.cpu().numpy()[: sc.fluid_count, 2]
    depth = z.max() - z
    deep, shallow = kd[depth > 0.38].mean(), kd[depth < 0.1].mean()
    assert (kd >= 0.0).all() and deep > 5.0 * shallow, (deep, shallow)


def test_primed_resting_columns_bit_exact(cuda):
    """The reference's speed-harness scene (alloy/testing/sph.py:49-73) at a small size: several resting columns in
    box tanks, fast preset with the projected CG solve, primed, then stepped at dt_max beside the oracle."""
    from alloy_b200.solvers.sph.testing import water_column

    sc = water_column(8, 8, 12, worlds=3, r=2.0e-3, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    assert sol.pressure_solver == "cg"
    orc = Oracle(sc.model.host(), sc.config)
    a, b = sc.model.state(), sc.model.state()
    guess = hydrostatic_guess(sol, a)
    it = sol.prime(a, sc.dt)
    orc.set_warm(guess * np.float32(sc.dt), orc.warm()[1])
    assert it == orc.prime(sc.dt)
    for k in range(10):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        np.testing.assert_array_equal(sol.report().iters_density, orc.report()["iters_density"], err_msg=f"step {k}")
