# SPDX-License-Identifier: Apache-2.0
"""The batched pour workload: hemisphere bowls of boundary particles moving on seeded sinusoids (their velocities set
by the caller between steps), liquid resting in them, a spout pouring into each and an escape box retiring what
spills. (1) Against the FP32 oracle the CUDA path agrees bit for bit: positions, velocities, iteration counts and the
mass ledger. (2) Against an FP64 run of the oracle on the first 16 worlds of the workload: every world's density
error stays at the solver's tolerance in both precisions, and the FP32 state's density error measured in FP64 differs
from the FP64 run's by a small fraction of the tolerance."""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.solver import _xform7, layer_offsets
from alloy_b200.solvers.sph.testing import pour_bowls
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _spouts(sc, sol, orc):
    arr = sc.model.host()
    for e in sc.emitters:
        w = e["world"]
        i0 = int(arr["world_start"][w])
        vol = float(arr["mass"][i0]) / float(arr["rest_density"][i0])
        offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64),
                             sc.config.spacing)
        rate = len(offs) * vol / e["layer_every"]
        sol.add_emitter(w, e["centre"], e["half"], rate, e["velocity"], pool=e["pool"])
        orc.add_emitter(w, _xform7(e["centre"]), offs, e["velocity"], float(np.float32(len(offs) * vol / rate)),
                        np.sort(e["pool"]))


def _step_both(sc, sol, orc, a, b, k):
    m = sc.motion
    m.apply(a, k * sc.dt, sc.dt)
    orc.set_velocity(m.wall_index, m.host_velocities(k * sc.dt, sc.dt))
    sol.step(a, b, None, None, sc.dt)
    orc.step(sc.dt)
    return b, a


def test_pour_bowls_bit_exact(cuda):
    sc = pour_bowls(worlds=3, lo=1200, hi=2400, seed=4, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    _spouts(sc, sol, orc)
    a, b = sc.model.state(), sc.model.state()
    for k in range(40):
        a, b = _step_both(sc, sol, orc, a, b, k)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        led = sol.mass_ledger()
        np.testing.assert_array_equal(led["in"], orep["mass_in"])
        np.testing.assert_array_equal(led["active"] + led["out"], led["initial"] + led["in"])
    assert int(sol.mass_ledger()["in"].sum()) > 0
    # the bowls moved with their prescribed velocities
    m = sc.motion
    np.testing.assert_array_equal(a.particle_qd.cpu().numpy()[m.wall_index], m.host_velocities(39 * sc.dt, sc.dt))


def _state_density_error(sc, q, qd) -> np.ndarray:
    """Per world: mean over liquid of max(rho / rho0 - 1, 0) of a state, evaluated by the FP64 oracle."""
    orc = Oracle(sc.model.host(), sc.config, f64=True)
    orc.set_state(q, qd)
    orc.prepare_density()
    ratio, act = orc.field("ratio").astype(np.float64), orc.field("active") > 0
    world = sc.model.host()["world"]
    W = len(sc.model.host()["world_start"]) - 1
    out = np.zeros(W)
    for w in range(W):
        sel = act & (world == w)
        out[w] = np.maximum(ratio[sel] - 1.0, 0.0).mean() if sel.any() else 0.0
    return out


def test_pour_first_16_worlds_against_fp64(cuda):
    sc = pour_bowls(worlds=16, seed=0, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config, f64=True)
    _spouts(sc, sol, orc)
    a, b = sc.model.state(), sc.model.state()
    steps = 30
    for k in range(steps):
        a, b = _step_both(sc, sol, orc, a, b, k)
    tol = sc.config.max_density_error
    rep, orep = sol.report(), orc.report()
    assert (rep.density_err <= tol).all() and (orep["density_err"] <= tol).all()
    q64, v64 = orc.state64()
    e32 = _state_density_error(sc, a.particle_q.cpu().numpy(), a.particle_qd.cpu().numpy())
    e64 = _state_density_error(sc, q64.astype(np.float32), v64.astype(np.float32))
    dq = np.abs(a.particle_q.cpu().numpy().astype(np.float64) - q64).max()
    print(f"16 worlds, {steps} steps: solver density error FP32 max {rep.density_err.max():.3e}, FP64 "
          f"{orep['density_err'].max():.3e}; state compression measured in FP64: FP32 run max {e32.max():.3e}, FP64 "
          f"run max {e64.max():.3e}, largest per-world difference {np.abs(e32 - e64).max():.3e}; max |dq| {dq:.2e} m")
    assert np.abs(e32 - e64).max() < 0.5 * tol
    assert dq < 0.5 * sc.config.spacing
