# SPDX-License-Identifier: Apache-2.0
"""The persistent CG solve: each projected-CG pressure solve of a model of at most 131,072 particles runs as one
cooperative launch whose phases (the bodies of the multi-launch path's kernels) are separated by grid-wide barriers
with bounded waits (krylov.py:254-297 with the loop of solve_driver.py:121-186).

- bit for bit against the multi-launch path (positions, velocities, warm starts, per-world iterations and errors every
  step) on a dam break in a tank of boundary particles, on uneven batched worlds with spouts (active sets change,
  worlds stop at different iterations), and on primed resting columns in box tanks (four wall slots per
  particle), each replayed as CUDA graphs and launched eagerly; the launches per step drop;
- the bounded waits: a barrier told to wait for one block more than the grid has gives up at every block, the report
  fails with ADF_ERR_STATE instead of returning results, and after the status is cleared the solver steps on and
  equals a fresh solver bit for bit (no GPU fault, no unbounded wait).

The multi-launch path, the default, is the one the tests against the oracle run; test_gpu_jitter_rule.py runs the
persistent one against the oracle as well.
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.solver import layer_offsets
from alloy_b200.solvers.sph.testing import batched_worlds, dam_break, water_column

pytestmark = pytest.mark.gpu


def _spouts(sc, sol):
    arr = sc.model.host()
    for e in sc.emitters:
        w = e["world"]
        i0 = int(arr["world_start"][w])
        vol = float(arr["mass"][i0]) / float(arr["rest_density"][i0])
        offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64),
                             sc.config.spacing)
        sol.add_emitter(w, e["centre"], e["half"], len(offs) * vol / (10.0 * sc.dt), e["velocity"], pool=e["pool"])


def _lockstep(make, steps, graphs, spouts=False, prime=False):
    """Both paths side by side, each on its own model (emission and escape write the model's flags and phases)."""
    scenes = [make(), make()]
    sc = scenes[0]
    sols = [SolverDFSPH(x.model, x.config) for x in scenes]
    sols[0].persistent(True)
    sols[1].persistent(False)
    states = [[x.model.state(), x.model.state()] for x in scenes]
    for sol, st, x in zip(sols, states, scenes):
        sol.use_graphs(graphs)
        if spouts:
            _spouts(x, sol)
        if prime:
            sol.prime(st[0], sc.dt)
    launches = []
    for k in range(steps):
        counts = []
        for sol, st in zip(sols, states):
            l0 = sol.kernel_launches()
            sol.step(st[0], st[1], None, None, sc.dt)
            counts.append(sol.kernel_launches() - l0)
            st.reverse()
        launches.append(counts)
        r0, r1 = sols[0].report(), sols[1].report()  # raises if a barrier wait gave up
        (a, _), (c, _) = states
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), c.particle_q.cpu().numpy(), err_msg=f"q {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), c.particle_qd.cpu().numpy(), err_msg=f"qd {k}")
        for f in ("iters_density", "iters_divergence", "density_err", "divergence_err"):
            np.testing.assert_array_equal(getattr(r0, f), getattr(r1, f), err_msg=f"{f} step {k}")
    s0, s1 = sols[0].alloy_state_arrays(), sols[1].alloy_state_arrays()
    for key in ("sph.kappa_v", "sph.kappa_d"):
        np.testing.assert_array_equal(s0[key].cpu().numpy(), s1[key].cpu().numpy(), err_msg=key)
    return sols[0], np.asarray(launches), r0


@pytest.mark.parametrize("graphs", [True, False])
def test_persistent_dam_break_equals_multi_launch(cuda, graphs):
    sol, launches, rep = _lockstep(
        lambda: dam_break(counts=(12, 10, 14), box=(0.5, 0.4, 0.6), device=cuda, pressure_solver="cg"), 20, graphs)
    assert sol.pressure_solver == "cg"
    if not graphs:  # eager steps count every launch: the persistent solve is one per solve
        assert (launches[:, 0] < launches[:, 1]).all(), launches


@pytest.mark.parametrize("graphs", [True, False])
def test_persistent_batched_worlds_with_spouts_equal_multi_launch(cuda, graphs):
    _lockstep(lambda: batched_worlds(worlds=6, lo=400, hi=3000, seed=6, device=cuda, pressure_solver="cg"), 30,
              graphs, spouts=True)


def test_persistent_primed_columns_in_box_tanks_equal_multi_launch(cuda):
    sol, launches, _ = _lockstep(lambda: water_column(8, 8, 12, worlds=3, r=2.0e-3, device=cuda), 12, True,
                                 prime=True)
    assert sol.pressure_solver == "cg"
    assert (launches[:, 0] <= launches[:, 1]).all()


def test_persistent_barrier_wait_expires_with_status(cuda):
    def make():
        return dam_break(counts=(8, 8, 10), box=(0.3, 0.3, 0.3), device=cuda, pressure_solver="cg")

    sc, sr = make(), make()  # each solver on its own model
    sol, ref = SolverDFSPH(sc.model, sc.config), SolverDFSPH(sr.model, sr.config)
    sol.persistent(True)
    a, b = sc.model.state(), sc.model.state()
    c, d = sr.model.state(), sr.model.state()
    sol.barrier_wait(polls=2000, extra_arrivals=1)  # every barrier waits for a block that does not exist
    sol.step(a, b, None, None, sc.dt)
    with pytest.raises(RuntimeError, match="grid-barrier wait"):
        sol.report()
    sol.clear_status()
    sol.barrier_wait()  # the defaults: the grid's own blocks, about a second per wait
    # the failed step's results are invalid: both solvers go on from the model's state with the same warm starts
    a, b = sc.model.state(), sc.model.state()
    mine, theirs = sol.alloy_state_arrays(), ref.alloy_state_arrays()
    for key in ("sph.kappa_v", "sph.kappa_d", "sph.phase", "particle_flags"):
        mine[key].copy_(theirs[key])
    for _ in range(5):
        sol.step(a, b, None, None, sc.dt)
        ref.step(c, d, None, None, sr.dt)
        a, b, c, d = b, a, d, c
    np.testing.assert_array_equal(a.particle_q.cpu().numpy(), c.particle_q.cpu().numpy())
    np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), c.particle_qd.cpu().numpy())
    np.testing.assert_array_equal(sol.report().iters_density, ref.report().iters_density)
