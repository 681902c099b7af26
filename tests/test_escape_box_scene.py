# SPDX-License-Identifier: Apache-2.0
"""The automatic escape box of a scene-built solver (escape_box.py:44-94, plugin.py:36-61), ported from the
reference's tests/solvers/sph/test_escape_box.py:21-81 on its scene: a ground plane, a 10 cm static plate at
z = 0.1 m and a 4^3 block resting on it, optionally one particle shot up at 8 m/s.

- the box covers the content (the plate's bounding sphere and the particles; the ground plane is left out) with its
  pad, and an empty model has none (CPU);
- an explicit choice (a config, or a world_bounds kwarg) is kept (CPU);
- the factory's solver retires the shot particle and counts it, the block stays on its plate, and the box leaves a
  resting scene bitwise as it is (GPU).
"""

from __future__ import annotations

import numpy as np
import pytest

from alloy_b200.solvers.sph.build import add_fluid_block, add_fluid_points
from alloy_b200.solvers.sph.config import DFSPHConfig
from alloy_b200.solvers.sph.model import ModelBuilder, ParticleFlags
from alloy_b200.solvers.sph.plugin import auto_box, config_from_kwargs

R = 2.0e-3


def _scene(shot: bool, device="cpu"):
    cfg = DFSPHConfig(particle_radius=R)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.add_ground_plane()
    b.begin_world()
    b.add_shape_box(-1, (0.0, 0.0, 0.095), 0.05, 0.05, 0.005)
    add_fluid_block(b, cfg, (-0.008, -0.008, 0.1), (4, 4, 4))
    if shot:
        add_fluid_points(b, cfg, np.array([[0.03, 0.0, 0.11]]), velocity=(0.0, 0.0, 8.0))
    b.end_world()
    return b.finalize(device)


def test_auto_box_covers_the_content_with_its_pad():
    (lo, hi), pad = auto_box(_scene(shot=False))
    rp = float(np.linalg.norm([0.05, 0.05, 0.005]))
    np.testing.assert_allclose(lo, np.array([-rp, -rp, 0.095 - rp]) - 0.25, atol=1e-6)
    np.testing.assert_allclose(hi, np.array([rp, rp, 0.095 + rp]) + 0.25, atol=1e-6)
    assert pad == 0.25
    assert auto_box(ModelBuilder().finalize()) is None


@pytest.mark.parametrize("kw", [{"world_bounds": None}, {"config": DFSPHConfig(particle_radius=R)}])
def test_factory_keeps_an_explicit_choice(kw):
    m = _scene(shot=True)
    cfg, _, auto = config_from_kwargs(m, kw)
    assert cfg.world_bounds is None and auto is None
    box = ((-1.0, -1.0, -1.0), (1.0, 1.0, 1.0))
    cfg, _, auto = config_from_kwargs(m, {"particle_radius": R, "world_bounds": box})
    assert cfg.world_bounds == box and auto is None


def _run(sol, m, steps: int, dt: float = 1.0e-3):
    a, b = m.state(), m.state()
    for _ in range(steps):
        sol.step(a, b, None, None, dt)
        a, b = b, a
    return a


@pytest.mark.gpu
def test_scene_factory_retires_ejecta_and_counts_them(cuda):
    from alloy_b200.solvers.sph.plugin import _factory

    m = _scene(shot=True, device=cuda)
    sol = _factory(m, {"particle_radius": R})
    top = sol.config.world_bounds[1][2]
    assert 0.3 < top < 1.0
    st = _run(sol, m, 120)  # the shot particle passes the top at ~0.05 s
    shot = m.particle_count - 1
    assert (int(m.particle_flags[shot].item()) & int(ParticleFlags.ACTIVE)) == 0
    rep = sol.report()
    assert rep.escaped.tolist() == [1]
    assert np.isclose(rep.mass_out[0], float(m.particle_mass[shot].item()), rtol=1e-6)
    assert np.all(st.particle_q.cpu().numpy()[:shot, 2] < 0.2)  # the block stays on its plate


@pytest.mark.gpu
def test_escape_box_leaves_a_resting_scene_bitwise(cuda):
    from alloy_b200.solvers.sph.plugin import _factory

    q = []
    for kw in ({"particle_radius": R}, {"particle_radius": R, "world_bounds": None}):
        m = _scene(shot=False, device=cuda)
        q.append(_run(_factory(m, kw), m, 40).particle_q.cpu().numpy().copy())
    assert np.array_equal(q[0], q[1])
