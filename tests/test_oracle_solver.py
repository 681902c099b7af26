# SPDX-License-Identifier: Apache-2.0
"""The oracle's DFSPH step against the reference's own solver-level known answers (CPU).

Ports tests/solvers/sph/test_neighbors_reduce.py:19-44 (grouped, sorted, counted rows; overflow keeps the lowest ids),
tests/integration/test_sph_mpm_walls.py:84-100 (a slab of boundary particles reads as a plane; another world's
particles are no wall), tests/solvers/sph/test_mass.py:13-40 (exact int64 ledger with emitter, sink and escape box),
tests/solvers/sph/test_determinism.py:36-63 (per-world independence bitwise; a seeded blow-up is reported)."""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph.build import add_fluid_block, add_fluid_points, add_spares, add_wall_particles
from alloy_b200.solvers.sph.config import DFSPHConfig
from alloy_b200.solvers.sph.model import ModelBuilder
from alloy_b200.solvers.sph.solver import layer_offsets
from alloy_b200.solvers.sph.testing import benchmark_config, dam_break
from oracle.pyoracle import Oracle


def _lattice(n: int, sp: float) -> np.ndarray:
    ax = np.arange(n) * sp
    return np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3).astype(np.float32)


def _two_world_lattice(capacity: int):
    cfg = DFSPHConfig(particle_radius=0.5, neighbor_capacity=capacity, rest_jitter_speed=None,
                      pressure_solver="jacobi")
    g = _lattice(5, 1.0)
    b = ModelBuilder()
    for _ in range(2):
        b.begin_world()
        add_fluid_points(b, cfg, g)
        b.end_world()
    arr = b.finalize().host()
    arr["flags"][3] = 0  # an inactive particle in world 0
    return arr, cfg, g


def test_neighbors_grouped_sorted_and_counted():
    arr, cfg, g = _two_world_lattice(64)
    o = Oracle(arr, cfg)
    o.prepare_density()
    rows, cnt = o.lists()
    q, world = arr["q"], arr["world"]
    for i in range(len(q)):
        row = rows[i, : cnt[i]]
        assert np.all(np.diff(row) > 0)
        assert np.all(world[row] == world[i]) and 3 not in row and i not in row
        assert np.all(np.linalg.norm(q[row] - q[i], axis=1) < 2.0)
    assert cnt[3] == 0
    brute = [(np.linalg.norm(g - g[i], axis=1) < 2.0).sum() - 1 for i in range(len(g))]
    assert list(cnt[len(g):]) == brute
    assert o.report()["neighbor_overflow"].tolist() == [0, 0]


def test_overflow_keeps_the_lowest_ids():
    arr, cfg, g = _two_world_lattice(8)
    o = Oracle(arr, cfg)
    o.prepare_density()
    rows, cnt = o.lists()
    assert o.report()["neighbor_overflow"][1] > 0 and cnt.max() == 8
    n = len(g)
    for i in range(n, 2 * n):
        near = [j + n for j in range(n) if j != i - n and np.linalg.norm(g[j] - g[i - n]) < 2.0]
        np.testing.assert_array_equal(rows[i, : cnt[i]], sorted(near)[:8])


def _slab_scene(fluid_world: int, wall_world: int, zs):
    """Boundary particles (spacing A = 2.5 mm, volume A^3) filling z < 0 under fluid particles at (3e-4, 0, z), r = 2 mm:
    the reference's particle-wall rig (test_sph_mpm_walls.py:23-52)."""
    A = 0.0025
    cfg = DFSPHConfig(particle_radius=2.0e-3, rest_jitter_speed=None, pressure_solver="jacobi")
    ax = np.arange(-12, 13) * A
    x, y, z = np.meshgrid(ax, ax, -np.arange(8) * A - A / 2, indexing="ij")
    slab = np.stack([x.ravel(), y.ravel(), z.ravel()], 1)
    b = ModelBuilder(gravity=(0.0, 0.0, 0.0))
    ranges = {}
    for w in range(max(fluid_world, wall_world) + 1):
        b.begin_world()
        if w == wall_world:
            ranges["wall"] = add_wall_particles(b, cfg, slab, spacing=A, velocity=(0.1, 0.0, -0.2))
        if w == fluid_world:
            pts = np.stack([np.full(len(zs), 3e-4), np.zeros(len(zs)), zs], 1)
            ranges["fluid"] = add_fluid_points(b, cfg, pts)
        b.end_world()
    return b.finalize().host(), cfg, ranges


def test_a_slab_reads_as_a_plane_at_its_face():
    zs = np.linspace(-0.004, 0.004, 17)
    arr, cfg, rg = _slab_scene(0, 0, zs)
    o = Oracle(arr, cfg)
    o.prepare_density()
    f = np.arange(rg["fluid"].start, rg["fluid"].stop)
    on = o.slot_on()[f] > 0
    assert on.all()
    assert np.abs(o.field("slot_phi")[f] - zs).max() < 3.0e-4
    np.testing.assert_allclose(o.field("slot_n")[f][:, 2], 1.0, atol=2e-3)
    np.testing.assert_allclose(o.field("slot_vb")[f], np.tile([0.1, 0.0, -0.2], (len(zs), 1)), atol=1e-6)


def test_another_worlds_particles_are_not_a_wall():
    arr, cfg, rg = _slab_scene(0, 1, np.array([0.001]))
    o = Oracle(arr, cfg)
    o.prepare_density()
    assert o.slot_on()[rg["fluid"].start] == 0


def test_interior_rest_lattice_has_rest_density():
    cfg = benchmark_config(0.02)
    b = ModelBuilder()
    b.begin_world()
    add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (9, 9, 9))
    b.end_world()
    arr = b.finalize().host()
    o = Oracle(arr, cfg)
    o.prepare_density()
    ix = np.rint(arr["q"] / 0.02 - 0.5).astype(int)
    interior = np.all((ix >= 2) & (ix <= 6), axis=1)
    np.testing.assert_allclose(o.field("ratio")[interior], 1.0, atol=1e-6)


def test_mass_ledger_is_exact_with_emitter_sink_and_escape_box():
    cfg = benchmark_config(0.02, world_bounds=((-0.5, -0.5, -0.02), (0.45, 0.9, 1.0)))
    b = ModelBuilder()
    b.begin_world()
    add_fluid_block(b, cfg, (0.1, 0.1, 0.3), (6, 6, 6), velocity=(2.0, 0.0, 0.0))
    sp = add_spares(b, cfg, 200)
    b.end_world()
    arr = b.finalize().host()
    o = Oracle(arr, cfg)
    offs = layer_offsets(np.array([0.04, 0.04, 0.01]), np.array([0.0, 0.0, -1.0]), cfg.spacing)
    xform = np.array([0.4, 0.4, 0.6, 0.0, 0.0, 0.0, 1.0], np.float32)
    o.add_emitter(0, xform, offs, (0.0, 0.0, -1.0), 0.004, np.arange(sp.start, sp.stop))
    o.add_sink(0, np.array([0.3, 0.3, 0.05, 0, 0, 0, 1], np.float32), np.array([0.08, 0.08, 0.05], np.float32))
    for _ in range(120):
        o.step(2.0e-3)
    r = o.report()
    assert r["mass_in"][0] > 0 and r["mass_out"][0] > 0 and r["escaped"][0] > 0
    assert r["mass_active"][0] + r["mass_out"][0] == r["mass_initial"][0] + r["mass_in"][0]


def test_per_world_independence_bitwise():
    """Two worlds of different size packed in one model match their one-world runs bit for bit."""
    cfgs = [(6, 6, 8), (6, 6, 5)]
    cfg = benchmark_config(0.02)
    b = ModelBuilder()
    for c in cfgs:
        b.begin_world()
        add_fluid_block(b, cfg, (0.0, 0.0, 0.0), c, jitter=0.01, seed=c[2])
        add_wall_particles(b, cfg, dam_break(counts=c, box=(0.2, 0.2, 0.3), spacing=0.02).model.host()["q"][
            int(np.prod(c)):])
        b.end_world()
    packed = b.finalize().host()
    o = Oracle(packed, cfg)
    for _ in range(25):
        o.step(1.0e-3)
    q, _ = o.state()
    ws = packed["world_start"]
    for k, c in enumerate(cfgs):
        sc = dam_break(counts=c, box=(0.2, 0.2, 0.3), spacing=0.02, seed=c[2])
        o1 = Oracle(sc.model.host(), cfg)
        for _ in range(25):
            o1.step(1.0e-3)
        q1, _ = o1.state()
        assert q[ws[k]:ws[k + 1]].tobytes() == q1.tobytes(), f"world {k}"
        assert o.report()["iters_density"][k] == o1.report()["iters_density"][0]


def test_seeded_blowup_reaches_speed_fail():
    """An over-relaxed Jacobi (omega = 1, rejected by validate) blows a column up; the report shows a speed above
    SPEED_FAIL (20 m/s) instead of waiting for NaN (test_determinism.py:54-63)."""
    sc = dam_break(counts=(4, 4, 8), box=(0.08, 0.08, 0.3), spacing=0.02)
    cfg = sc.config
    cfg.jacobi_omega = 1.0  # seeded instability (bypasses validate on purpose)
    o = Oracle(sc.model.host(), cfg)
    peak = 0.0
    for _ in range(150):
        o.step(1.0e-3)
        peak = max(peak, float(o.report()["max_speed"][0]))
        if peak > 20.0:
            break
    assert peak > 20.0
    with pytest.raises(ValueError, match="jacobi_omega"):
        cfg.validate()


def test_cg_needs_far_fewer_iterations_than_jacobi_on_a_deep_column():
    """krylov.py:1-9: relaxed Jacobi needs O(N^2) iterations for N layers, CG O(N). A 40-layer column at a tight
    tolerance: every CG solve converges, in far fewer iterations than Jacobi (which hits max_iterations)."""
    totals = {}
    for solver in ("jacobi", "cg"):
        sc = dam_break(counts=(6, 6, 40), box=(0.12, 0.12, 1.0), pressure_solver=solver, max_density_error=1e-4,
                       max_divergence_error=1e-4, max_iterations=200)
        o = Oracle(sc.model.host(), sc.config, threads=4)
        assert o.params.cg == (solver == "cg")
        its = []
        for _ in range(10):
            o.step(sc.dt)
            r = o.report()
            its.append(int(r["iters_divergence"][0]) + int(r["iters_density"][0]))
            if solver == "cg":
                assert r["iters_divergence"][0] < 200 and r["iters_density"][0] < 200
                assert r["density_err"][0] <= 1e-4
        totals[solver] = sum(its)
    assert totals["cg"] * 3 < totals["jacobi"], totals
