# SPDX-License-Identifier: Apache-2.0
"""The CUDA step against the reference's OWN kernels (fixtures ``tests/golden/reference_steps_<case>.npz``, made by
``tests/golden/make_step_golden.py`` from alloy/solvers/sph under a float32 warp stand-in).

Anchored steps (each from the reference's start state and warm starts) and a free run from the initial state, through
``SolverDFSPH.step`` and the C ABI, for particle walls and for the box tank of box-shape walls (Jacobi, CG, and the
impact scene's projections and sweeps). Bit for bit: per-solve iteration counts; neighbour rows after the first build;
with box walls, every particle's slot walls in order and the projection and sweep counters of every step.
Within the tolerances of ``tests/test_oracle_reference_steps.py`` (the CUDA path equals the oracle bit for bit, and the
oracle is within them of the reference): velocities 2e-3 of the largest speed, positions 1e-6 m, warm starts 2e-4
(divergence) and 2e-2 (density) of their largest value, per-world mean errors 1e-2 relative plus 1e-7; free running,
velocities 1e-2 of the largest speed.
"""

from __future__ import annotations

import ast
from pathlib import Path

import numpy as np
import pytest
import torch

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import dam_break, tank_impacts

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("dam_break_jacobi", "dam_break_cg", "column_jacobi_tight", "tank_sdf_jacobi", "tank_sdf_cg", "tank_impacts")
SDF_CASES = ("tank_sdf_jacobi", "tank_sdf_cg", "tank_impacts")
TOL = {"kv": 2e-4, "kd": 2e-2, "qd": 2e-3, "q_abs_m": 1e-6, "err_rel": 1e-2, "err_abs": 1e-7, "qd_free": 1e-2}


def load(case: str, device):
    g = np.load(GOLDEN / f"reference_steps_{case}.npz")
    c = ast.literal_eval(str(g["scene"]))
    if c.get("builder") == "tank_impacts":
        return g, c, tank_impacts(device=device, dt=c["scene"]["dt"], **c["config"])
    return g, c, dam_break(device=device, **c["scene"], **c["config"])


def rel(x, y, m) -> float:
    return float(np.max(np.abs(x[m] - y[m])) / (np.max(np.abs(y[m])) + 1e-30))


def host(t) -> np.ndarray:
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("case", CASES)
def test_cuda_rows_match_reference_kernels(cuda, case):
    g, c, sc = load(case, cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    sol.density_ratio(sc.model.state())
    rows, cnt = sol.neighbor_rows()
    fluid = host(sc.model.sph.phase) >= 1
    np.testing.assert_array_equal(cnt[fluid], g["count"][0][fluid])
    for i in np.flatnonzero(fluid):
        np.testing.assert_array_equal(rows[i, :cnt[i]], g["rows"][0][i, :cnt[i]], err_msg=f"row {i}")


@pytest.mark.parametrize("case", CASES)
def test_cuda_anchored_steps_match_reference_kernels(cuda, case):
    g, c, sc = load(case, cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    fluid = host(sc.model.sph.phase) >= 1
    dt = c["scene"]["dt"]
    a, b = sc.model.state(), sc.model.state()
    warm = sol.alloy_state_arrays()
    for s in range(int(g["steps"])):
        a.particle_q.copy_(torch.from_numpy(g["q0"][s]))
        a.particle_qd.copy_(torch.from_numpy(g["qd0"][s]))
        warm["sph.kappa_v"].copy_(torch.from_numpy(g["kv0"][s]))
        warm["sph.kappa_d"].copy_(torch.from_numpy(g["kd0"][s]))
        sol.step(a, b, None, None, dt)
        rep = sol.report()
        assert int(rep.iters_divergence[0]) == g["iters_div"][s][0], (case, s)
        assert int(rep.iters_density[0]) == g["iters_den"][s][0], (case, s)
        assert float(np.max(np.abs(host(b.particle_q) - g["q1"][s])[fluid])) <= TOL["q_abs_m"], (case, s)
        assert rel(host(b.particle_qd), g["qd1"][s], fluid) <= TOL["qd"], (case, s)
        assert rel(host(warm["sph.kappa_v"]), g["kv"][s], fluid) <= TOL["kv"], (case, s)
        assert rel(host(warm["sph.kappa_d"]), g["kd"][s], fluid) <= TOL["kd"], (case, s)
        for ours, ref in ((rep.density_err, "den_err"), (rep.divergence_err, "div_err")):
            r = float(g[ref][s][0])
            assert abs(float(ours[0]) - r) <= TOL["err_rel"] * r + TOL["err_abs"], (case, s, ref)


@pytest.mark.parametrize("case", CASES)
def test_cuda_free_run_matches_reference_kernels(cuda, case):
    g, c, sc = load(case, cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    fluid = host(sc.model.sph.phase) >= 1
    a, b = sc.model.state(), sc.model.state()
    for s in range(int(g["steps"])):
        sol.step(a, b, None, None, c["scene"]["dt"])
        a, b = b, a
        rep = sol.report()
        assert int(rep.iters_divergence[0]) == g["iters_div"][s][0], (case, s)
        assert int(rep.iters_density[0]) == g["iters_den"][s][0], (case, s)
        assert float(np.max(np.abs(host(a.particle_q) - g["q1"][s])[fluid])) <= TOL["q_abs_m"], (case, s)
        assert rel(host(a.particle_qd), g["qd1"][s], fluid) <= TOL["qd_free"], (case, s)


@pytest.mark.parametrize("case", SDF_CASES)
def test_cuda_box_wall_slots_and_counters_match_reference(cuda, case):
    """The walls of every slot in the reference's order, and its projections and sweeps at the same steps."""
    g, c, sc = load(case, cuda)
    sol = SolverDFSPH(sc.model, sc.config)
    fluid = host(sc.model.sph.phase) >= 1
    a, b = sc.model.state(), sc.model.state()
    warm = sol.alloy_state_arrays()
    for s in range(int(g["steps"])):
        a.particle_q.copy_(torch.from_numpy(g["q0"][s]))
        a.particle_qd.copy_(torch.from_numpy(g["qd0"][s]))
        warm["sph.kappa_v"].copy_(torch.from_numpy(g["kv0"][s]))
        warm["sph.kappa_d"].copy_(torch.from_numpy(g["kd0"][s]))
        p0, w0 = sol.diagnostics()["projected"].copy(), sol.diagnostics()["swept"].copy()
        sol.step(a, b, None, None, c["scene"]["dt"])
        shapes = np.stack([sol.debug_field(f"slot_shape:{k}") for k in range(4)], 1).astype(np.int32)
        np.testing.assert_array_equal(shapes[fluid], g["slot_shapes"][s][fluid], err_msg=f"{case} step {s}")
        d = sol.diagnostics()
        assert int(d["projected"][0] - p0[0]) == int(g["projected"][s][0] - (g["projected"][s - 1][0] if s else 0))
        assert int(d["swept"][0] - w0[0]) == int(g["swept"][s][0] - (g["swept"][s - 1][0] if s else 0))
