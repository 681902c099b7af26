# SPDX-License-Identifier: Apache-2.0
"""The projected preconditioned CG pressure solve (the reference's default, krylov.py:77-318) against the oracle's
restatement of it: positions, velocities, warm starts, per-world iteration counts and residuals bit for bit, on a
single dam break, on batched uneven worlds with spouts (active-set changes and restarts happen), replayed as a CUDA
graph and launched kernel by kernel; a model whose liquid masses differ falls back to Jacobi, as the reference's
solver does (solver.py:89-91)."""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.solver import _xform7, layer_offsets
from alloy_b200.solvers.sph.testing import batched_worlds, dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _compare(sc, sol, orc, steps, spouts=False):
    if spouts:
        arr = sc.model.host()
        for e in sc.emitters:
            w = e["world"]
            i0 = int(arr["world_start"][w])
            vol = float(arr["mass"][i0]) / float(arr["rest_density"][i0])
            offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64),
                                 sc.config.spacing)
            rate = len(offs) * vol / (10.0 * sc.dt)
            sol.add_emitter(w, e["centre"], e["half"], rate, e["velocity"], pool=e["pool"])
            orc.add_emitter(w, _xform7(e["centre"]), offs, e["velocity"], float(np.float32(len(offs) * vol / rate)),
                            np.sort(e["pool"]))
    a, b = sc.model.state(), sc.model.state()
    its = []
    for k in range(steps):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        rep, orep = sol.report(), orc.report()
        np.testing.assert_array_equal(rep.iters_density, orep["iters_density"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.iters_divergence, orep["iters_divergence"], err_msg=f"step {k}")
        np.testing.assert_array_equal(rep.density_err.astype(np.float32), orep["density_err"], err_msg=f"step {k}")
        its.append(int(rep.iters_density.sum() + rep.iters_divergence.sum()))
    kv, kd = orc.warm()
    np.testing.assert_array_equal(sol.alloy_state_arrays()["sph.kappa_v"].cpu().numpy(), kv)
    np.testing.assert_array_equal(sol.alloy_state_arrays()["sph.kappa_d"].cpu().numpy(), kd)
    return its


def test_cg_dam_break_bit_exact(cuda):
    sc = dam_break(counts=(12, 10, 14), box=(0.5, 0.4, 0.6), device=cuda, pressure_solver="cg")
    sol = SolverDFSPH(sc.model, sc.config)
    assert sol.pressure_solver == "cg"
    orc = Oracle(sc.model.host(), sc.config)
    assert orc.params.cg == 1
    _compare(sc, sol, orc, 25)


def test_cg_batched_worlds_with_spouts_bit_exact(cuda):
    sc = batched_worlds(worlds=5, lo=400, hi=2000, seed=6, device=cuda, pressure_solver="cg")
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    its = _compare(sc, sol, orc, 40, spouts=True)
    assert max(its) > 2 * 2 * 5  # some world needed more than the minimum iterations


def test_cg_graph_equals_kernel_by_kernel(cuda):
    runs = []
    for graphs in (True, False):
        sc = batched_worlds(worlds=3, lo=800, hi=2500, seed=8, device=cuda, pressure_solver="cg")
        sol = SolverDFSPH(sc.model, sc.config)
        sol.use_graphs(graphs)
        a, b = sc.model.state(), sc.model.state()
        for _ in range(12):
            sol.step(a, b, None, None, sc.dt)
            a, b = b, a
        runs.append((a.particle_q.cpu().numpy(), sol.report().iters_density.copy()))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def test_cg_falls_back_to_jacobi_for_unequal_masses(cuda):
    sc = dam_break(counts=(6, 6, 6), box=(0.3, 0.3, 0.3), device=cuda, pressure_solver="cg")
    sc.model.particle_mass[: sc.fluid_count // 2] *= 1.01
    sol = SolverDFSPH(sc.model, sc.config)
    assert sol.pressure_solver == "jacobi"


def test_cg_one_lane_products_in_a_large_model_bit_exact(cuda):
    """Models of more than 131,072 particles take the CG products with one lane per particle (smaller ones by teams of
    four lanes, which every other test here exercises): a 139,776-particle dam break against the oracle."""
    sc = dam_break(counts=(56, 48, 52), box=(0.8, 0.6, 0.8), spacing=0.01, device=cuda, pressure_solver="cg")
    assert sc.model.particle_count > 131072
    sol = SolverDFSPH(sc.model, sc.config)
    orc = Oracle(sc.model.host(), sc.config)
    _compare(sc, sol, orc, 8)
