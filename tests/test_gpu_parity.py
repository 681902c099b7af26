# SPDX-License-Identifier: Apache-2.0
"""GPU parity against the CPU oracle on identical seeded inputs: neighbour rows bit for bit, every field of the step
bit for bit (the kernels and the oracle share one arithmetic contract), per-step iteration counts equal."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import dam_break
from oracle.pyoracle import Oracle

pytestmark = pytest.mark.gpu


def _pair(scene):
    sol = SolverDFSPH(scene.model, scene.config)
    orc = Oracle(scene.model.host(), scene.config)
    return sol, orc


def test_neighbour_rows_bit_exact(cuda):
    sc = dam_break(counts=(12, 10, 14), box=(0.5, 0.4, 0.6), device=cuda)
    sol, orc = _pair(sc)
    s = sc.model.state()
    sol.density_ratio(s)
    orc.prepare_density()
    rows, cnt = sol.neighbor_rows()
    orows, ocnt = orc.lists()
    np.testing.assert_array_equal(cnt, ocnt)
    np.testing.assert_array_equal(rows, orows)
    assert cnt[: sc.fluid_count].min() > 0


def test_density_and_slots_bit_exact(cuda):
    sc = dam_break(counts=(12, 10, 14), box=(0.5, 0.4, 0.6), device=cuda)
    sol, orc = _pair(sc)
    ratio, active = sol.density_ratio(sc.model.state())
    orc.prepare_density()
    np.testing.assert_array_equal(ratio, orc.field("ratio"))
    np.testing.assert_array_equal(active, orc.field("active") > 0)
    act = orc.field("active") > 0
    for name in ("alpha", "neff", "reg"):
        np.testing.assert_array_equal(sol.debug_field(name), np.where(act, orc.field(name), 0), err_msg=name)
    on = orc.slot_on() > 0
    psi = sol.debug_field("slot_psi")  # the kernels mark a particle without a wall slot with psi = -1
    np.testing.assert_array_equal((psi >= 0)[act], on[act])
    assert on.sum() > 0
    np.testing.assert_array_equal(psi[on], orc.field("slot_psi")[on])
    for name in ("slot_phi", "slot_g", "slot_vb", "slot_n"):
        np.testing.assert_array_equal(sol.debug_field(name)[on], orc.field(name)[on], err_msg=name)


@pytest.mark.parametrize("steps", [25])
def test_steps_bit_exact(cuda, steps):
    sc = dam_break(counts=(12, 10, 14), box=(0.5, 0.4, 0.6), device=cuda)
    sol, orc = _pair(sc)
    a, b = sc.model.state(), sc.model.state()
    for k in range(steps):
        sol.step(a, b, None, None, sc.dt)
        a, b = b, a
        orc.step(sc.dt)
        q, qd = orc.state()
        rep, orep = sol.report(), orc.report()
        assert rep.iters_density[0] == orep["iters_density"][0], k
        assert rep.iters_divergence[0] == orep["iters_divergence"][0], k
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
        assert rep.density_err[0] == orep["density_err"][0]
        assert rep.divergence_err[0] == orep["divergence_err"][0]
    kv, kd = orc.warm()
    np.testing.assert_array_equal(sol.alloy_state_arrays()["sph.kappa_v"].cpu().numpy(), kv)
    np.testing.assert_array_equal(sol.alloy_state_arrays()["sph.kappa_d"].cpu().numpy(), kd)


def test_graph_replay_equals_kernel_by_kernel_and_caller_capture(cuda):
    """The step replayed as one CUDA graph (WHILE nodes for the pressure iterations), launched kernel by kernel, and
    captured by the caller into its own torch CUDA graph give the same bits."""
    sc = dam_break(counts=(10, 8, 12), box=(0.4, 0.3, 0.5), device=cuda)
    runs = {}
    for mode in ("graph", "eager", "caller"):
        sol = SolverDFSPH(sc.model, sc.config)
        sol.use_graphs(mode == "graph")
        a, b = sc.model.state(), sc.model.state()
        if mode == "caller":
            sol.step(a, b, None, None, sc.dt)  # warm-up outside capture (first use builds nothing here)
            a, b = b, a
            g = torch.cuda.CUDAGraph()
            s = torch.cuda.Stream(cuda)
            s.wait_stream(torch.cuda.current_stream(cuda))
            with torch.cuda.stream(s):
                with torch.cuda.graph(g, stream=s):
                    sol.step(a, b, None, None, sc.dt)
            torch.cuda.current_stream(cuda).wait_stream(s)
            # the captured step maps a -> b; replay it with copies to advance the same states
            for _ in range(11):
                g.replay()
                a.particle_q.copy_(b.particle_q)
                a.particle_qd.copy_(b.particle_qd)
        else:
            for _ in range(12):
                sol.step(a, b, None, None, sc.dt)
                a.particle_q.copy_(b.particle_q)
                a.particle_qd.copy_(b.particle_qd)
        torch.cuda.synchronize(cuda)
        runs[mode] = (a.particle_q.cpu().numpy(), sol.report())
    for mode in ("eager", "caller"):
        np.testing.assert_array_equal(runs[mode][0], runs["graph"][0], err_msg=mode)
        assert runs[mode][1].iters_density[0] == runs["graph"][1].iters_density[0]


def test_moving_particle_wall_bit_exact(cuda):
    """A slab of boundary particles moving at (0.1, 0, -0.2) m/s under a small liquid block: the wall advance, the
    slot's wall velocity and the projection out of the advected plane agree with the oracle bit for bit, and the
    slab keeps its own velocity through every step (particle_walls.py:131-135)."""
    from alloy_b200.solvers.sph.build import add_fluid_block, add_wall_particles
    from alloy_b200.solvers.sph.model import ModelBuilder
    from alloy_b200.solvers.sph.testing import benchmark_config

    cfg = benchmark_config(0.02)
    ax = np.arange(-8, 9) * 0.02
    x, y, z = np.meshgrid(ax, ax, -np.arange(3) * 0.02 - 0.01, indexing="ij")
    slab = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    b = ModelBuilder()
    b.begin_world()
    add_fluid_block(b, cfg, (-0.06, -0.06, 0.0), (6, 6, 4), jitter=0.01, seed=4)
    walls = add_wall_particles(b, cfg, slab, velocity=(0.1, 0.0, -0.2))
    b.end_world()
    model = b.finalize(cuda)
    sol = SolverDFSPH(model, cfg)
    orc = Oracle(model.host(), cfg)
    a, s = model.state(), model.state()
    for k in range(15):
        sol.step(a, s, None, None, 1.0e-3)
        a, s = s, a
        orc.step(1.0e-3)
        q, qd = orc.state()
        np.testing.assert_array_equal(a.particle_q.cpu().numpy(), q, err_msg=f"q step {k}")
        np.testing.assert_array_equal(a.particle_qd.cpu().numpy(), qd, err_msg=f"qd step {k}")
    v = a.particle_qd.cpu().numpy()[walls.start:walls.stop]
    np.testing.assert_array_equal(v, np.tile(np.float32([0.1, 0.0, -0.2]), (len(v), 1)))
