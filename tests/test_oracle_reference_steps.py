# SPDX-License-Identifier: Apache-2.0
"""The CPU oracle against the reference's OWN kernels at step level.

The fixtures ``tests/golden/reference_steps_<case>.npz`` hold DFSPH steps computed by the reference's Warp kernels and
solve driver (alloy/solvers/sph: neighbors.py:160-195, boundary.py:190-396, particle_walls.py:65-135,
pressure.py:144-480, krylov.py, solve_driver.py:121-186, integrate.py:150-326) run under a float32 warp stand-in
(``tests/golden/make_step_golden.py``, ``tests/golden/refrun.py``). Two comparisons per case:

- anchored: every step starts the oracle from the reference's own start state and warm starts, so each step's
  differences are that step's alone;
- free running: the oracle steps from the initial state on its own, as a user's run would.

Bit for bit: neighbour rows and counts (integer ids), per-solve iteration counts (every step, both comparisons).
Within tolerance (the reference's Warp code generation may contract multiply-adds and its wall-colour sums follow
Warp's hash order, neither pinned; the oracle fixes both orders and spells its fused multiply-adds out), each
relative to the field's largest magnitude over the liquid unless it says otherwise: ``TOL`` below.
"""

from __future__ import annotations

import ast
from pathlib import Path

import numpy as np
import pytest

from alloy_b200.solvers.sph.testing import dam_break
from oracle.pyoracle import Oracle

GOLDEN = Path(__file__).resolve().parent / "golden"
CASES = ("dam_break_jacobi", "dam_break_cg", "column_jacobi_tight", "tank_sdf_jacobi", "tank_sdf_cg", "tank_impacts")
SDF_CASES = ("tank_sdf_jacobi", "tank_sdf_cg", "tank_impacts")
# Largest differences measured over the six cases, for scale: ratio 7.3e-6, alpha 4.3e-5, neff 6.2e-6, reg 1.5e-6,
# slot psi 3.9e-5 (every slot), slot phi 4.9e-7, kv 2.3e-5, kd 6.5e-3 (CG in the box tank), q 8.9e-8 m (6.5e-7 m free
# running), qd 5.9e-4 (box tank; 3.6e-3 free running with CG, which amplifies last-bit differences).
TOL = {"ratio": 1e-4, "alpha": 2e-4, "neff": 1e-4, "reg": 1e-4, "slot_psi": 2e-4, "slot_phi": 1e-5, "kv": 2e-4,
       "kd": 2e-2, "qd": 2e-3, "q_abs_m": 1e-6, "err_rel": 1e-2,
       "err_abs": 1e-7, "qd_free": 1e-2}  # per-world mean errors: 1 % of the value plus 1e-4 of the 1e-3 solver tolerance


def scene(c: dict, device="cpu"):
    if c.get("builder") == "tank_impacts":
        from alloy_b200.solvers.sph.testing import tank_impacts

        return tank_impacts(device=device, dt=c["scene"]["dt"], **c["config"])
    return dam_break(device=device, **c["scene"], **c["config"])


def load(case: str):
    g = np.load(GOLDEN / f"reference_steps_{case}.npz")
    c = ast.literal_eval(str(g["scene"]))
    return g, c, scene(c)


def rel(x, y, m) -> float:
    return float(np.max(np.abs(x[m] - y[m])) / (np.max(np.abs(y[m])) + 1e-30))


@pytest.mark.parametrize("case", CASES)
def test_fixture_matches_scene(case):
    """The fixture was made from the scene the test builds: same start state, same particle count."""
    g, c, sc = load(case)
    a = sc.model.host()
    np.testing.assert_array_equal(g["q0"][0], a["q"])
    np.testing.assert_array_equal(g["qd0"][0], a["qd"])
    assert int(g["steps"]) == c["steps"] >= 10


@pytest.mark.parametrize("case", CASES)
def test_anchored_steps_match_reference_kernels(case):
    g, c, sc = load(case)
    a = sc.model.host()
    fluid = a["phase"] >= 1
    dt = c["scene"]["dt"]
    orc = Oracle(a, sc.config)
    for s in range(int(g["steps"])):
        orc.set_state(g["q0"][s], g["qd0"][s])
        orc.set_warm(g["kv0"][s], g["kd0"][s])
        orc.step(dt)
        rows, cnt = orc.lists()
        np.testing.assert_array_equal(cnt[fluid], g["count"][s][fluid], err_msg=f"{case} step {s} counts")
        for i in np.flatnonzero(fluid):
            np.testing.assert_array_equal(rows[i, :cnt[i]], g["rows"][s][i, :cnt[i]], err_msg=f"{case} step {s} row {i}")
        rep = orc.report()
        assert rep["iters_divergence"][0] == g["iters_div"][s][0], (case, s)
        assert rep["iters_density"][0] == g["iters_den"][s][0], (case, s)
        for name in ("ratio", "alpha", "neff", "reg", "slot_psi"):
            assert rel(orc.field(name), g[name][s], fluid) <= TOL[name], \
                (case, s, name)
        on = fluid & (g["slot_shape"][s] >= 0)
        assert on.any() or s > 0
        if on.any():
            assert rel(orc.field("slot_phi"), g["slot_phi"][s], on) <= TOL["slot_phi"], (case, s)
        if "slot_shapes" in g.files:  # every slot: the same walls in the same order, Psi within tolerance
            np.testing.assert_array_equal(orc.slot_shapes()[fluid], g["slot_shapes"][s][fluid], err_msg=f"{case} {s}")
            psi4 = np.stack([orc.field(f"slot_psi:{k}") for k in range(4)], 1)
            assert rel(psi4, g["slot_psi4"][s], fluid) <= TOL["slot_psi"], (case, s)
        kv, kd = orc.warm()
        assert rel(kv, g["kv"][s], fluid) <= TOL["kv"], (case, s)
        assert rel(kd, g["kd"][s], fluid) <= TOL["kd"], (case, s)
        q, qd = orc.state()
        assert float(np.max(np.abs(q - g["q1"][s])[fluid])) <= TOL["q_abs_m"], (case, s)
        assert rel(qd, g["qd1"][s], fluid) <= TOL["qd"], (case, s)
        for ours, ref in (("density_err", "den_err"), ("divergence_err", "div_err")):
            r = float(g[ref][s][0])
            assert abs(float(rep[ours][0]) - r) <= TOL["err_rel"] * r + TOL["err_abs"], (case, s, ours)


@pytest.mark.parametrize("case", CASES)
def test_free_run_matches_reference_kernels(case):
    g, c, sc = load(case)
    a = sc.model.host()
    fluid = a["phase"] >= 1
    orc = Oracle(a, sc.config)
    for s in range(int(g["steps"])):
        orc.step(c["scene"]["dt"])
        q, qd = orc.state()
        rep = orc.report()
        assert rep["iters_divergence"][0] == g["iters_div"][s][0], (case, s)
        assert rep["iters_density"][0] == g["iters_den"][s][0], (case, s)
        assert float(np.max(np.abs(q - g["q1"][s])[fluid])) <= TOL["q_abs_m"], (case, s)
        assert rel(qd, g["qd1"][s], fluid) <= TOL["qd_free"], (case, s)


@pytest.mark.parametrize("case", SDF_CASES)
def test_wall_counters_match_reference(case):
    """Projections onto walls and sweeps past fast steps happen at the same steps as in the reference."""
    g, c, sc = load(case)
    orc = Oracle(sc.model.host(), sc.config)
    for s in range(int(g["steps"])):
        orc.set_state(g["q0"][s], g["qd0"][s])
        orc.set_warm(g["kv0"][s], g["kd0"][s])
        orc.step(c["scene"]["dt"])
        rep = orc.report()
        assert rep["projected"][0] == g["projected"][s][0] and rep["swept"][0] == g["swept"][s][0], (case, s)


def test_cases_cover_both_solvers_walls_and_the_iteration_cap():
    """The fixtures exercise relaxed Jacobi, projected CG, multi-iteration solves and the 50-iteration cap, particle
    walls and box walls with two and three slots per particle, projections and sweeps."""
    its = {case: (load(case)[0]["iters_div"][:, 0], load(case)[0]["iters_den"][:, 0]) for case in CASES}
    assert load("dam_break_cg")[1]["config"]["pressure_solver"] == "cg"
    div, den = its["column_jacobi_tight"]
    assert div.max() == 50 and den.max() > 2
    g = load("tank_impacts")[0]
    assert ((g["slot_shapes"] >= 0).sum(-1) >= 3).any()
    assert g["projected"][-1][0] > 0 and g["swept"][-1][0] > 0
