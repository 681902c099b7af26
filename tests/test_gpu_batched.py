# SPDX-License-Identifier: Apache-2.0
"""GPU parity on batched uneven worlds (the layout of the 256-world spout benchmark, scaled down): several worlds of
different sizes in one model, each in its own open particle box with a spout emitter drawing from its spare pool.
Every step the CUDA path and the oracle agree bit for bit on positions, velocities, per-world iteration counts,
residuals and the exact int64 mass ledger (emitted and active mass)."""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.solver import _xform7, layer_offsets
from alloy_b200.solvers.sph.testing import batched_worlds
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _spouts(sc, sol, orc):
    """One spout per world releasing a layer every 10 steps: rate = layer volume / (10 dt)."""
    arr = sc.model.host()
    cfg = sc.config
    for e in sc.emitters:
        w = e["world"]
        i0 = int(arr["world_start"][w])
        mass, rho0 = float(arr["mass"][i0]), float(arr["rest_density"][i0])
        offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64), cfg.spacing)
        rate = len(offs) * (mass / rho0) / (10.0 * sc.dt)
        sol.add_emitter(w, e["centre"], e["half"], rate, e["velocity"], pool=e["pool"])
        interval = np.float32(len(offs) * (mass / rho0) / rate)
        orc.add_emitter(w, _xform7(e["centre"]), offs, e["velocity"], float(interval), np.sort(e["pool"]))


def test_batched_worlds_with_spouts_bit_exact(cuda):
    sc = batched_worlds(worlds=5, lo=300, hi=1500, seed=3, device=cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    _spouts(sc, sol, orc)
    a, b = sc.model.state(), sc.model.state()
    emitted = 0
    for k in range(60):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.density_err.astype(np.float32), orep["density_err"])
        led = sol.mass_ledger()
        np.testing.assert_array_equal(led["in"], orep["mass_in"], err_msg=f"mass in, step {k}")
        np.testing.assert_array_equal(led["active"] + led["out"], led["initial"] + led["in"])
        emitted = int(led["in"].sum())
    assert emitted > 0  # every spout released layers


def test_world_count_does_not_change_a_world(cuda):
    """A world stepped inside a batch equals the same world stepped alone, bit for bit (per-world groups, grids and
    reductions; test_determinism.py:36-51)."""
    from alloy_b200.solvers.sph.sharding import sub_model

    sc = batched_worlds(worlds=4, lo=300, hi=1200, seed=11, device=cuda)
    full = SolverDFSPH(sc.model, sc.config)
    one = sub_model(sc.model, [2], cuda)
    alone = SolverDFSPH(one, sc.config)
    a, b = sc.model.state(), sc.model.state()
    c, d = one.state(), one.state()
    for _ in range(20):
        full.step(a, b, None, None, sc.dt)
        a, b = b, a
        alone.step(c, d, None, None, sc.dt)
        c, d = d, c
    ws = sc.model.host()["world_start"]
    np.testing.assert_array_equal(a.particle_q.cpu().numpy()[ws[2]:ws[3]], c.particle_q.cpu().numpy())
    assert full.report().iters_density[2] == alone.report().iters_density[0]
