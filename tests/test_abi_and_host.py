# SPDX-License-Identifier: Apache-2.0
"""CPU checks of the boundary: the library builds for sm_100a, loads without a GPU and exports every entry point
include/alloy_dfsph.h declares (no compute calls); the host logic of SolverDFSPH (configuration, emitter layers,
scene builders, world sharding) matches the reference's."""

from __future__ import annotations

import re
from pathlib import Path

import numpy as np
import pytest

from alloy_b200 import _lib
from alloy_b200.solvers.sph import config as C
from alloy_b200.solvers.sph.build import box_shell_points
from alloy_b200.solvers.sph.config import DFSPHConfig
from alloy_b200.solvers.sph.sharding import shard_worlds, sub_arrays
from alloy_b200.solvers.sph.solver import layer_offsets, quat_rotate_inv
from alloy_b200.solvers.sph.testing import batched_worlds, dam_break

ROOT = Path(__file__).resolve().parents[1]


def _declared() -> list[str]:
    text = (ROOT / "include" / "alloy_dfsph.h").read_text()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[A-Za-z_0-9]+\s*\**\s*(adf_[a-z_0-9]+)\(", text, re.M)))


def test_library_builds_loads_and_exports_every_declared_entry_point():
    from alloy_b200 import build

    build.build()
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing
    assert set(names) == set(_lib.EXPORTS)


def test_status_codes_map_to_the_reference_exceptions():
    L = _lib.lib()
    # a null solver is refused on the host, before any CUDA call
    with pytest.raises(ValueError, match="null"):
        _lib.check(L.adf_get_report(None, None, None))
    with pytest.raises(ValueError, match="null solver"):
        _lib.check(L.adf_step(None, None, None, None, None, None, 1.0e-3, None))
    with pytest.raises(_lib.CapacityError):
        _lib.check(-_lib.ADF_ERR_CAPACITY)


def test_config_validation_messages_follow_the_reference():
    with pytest.raises(ValueError, match="jacobi_omega must be in"):
        DFSPHConfig(jacobi_omega=0.8).validate()
    with pytest.raises(ValueError, match="need 0 < min_iterations <= max_iterations"):
        DFSPHConfig(min_iterations=5, max_iterations=4).validate()
    with pytest.raises(ValueError, match="neighbor|support_factor"):
        DFSPHConfig(support_factor=1.0).validate()
    f = DFSPHConfig.fast(particle_radius=0.01)
    assert f.rest_jitter_speed is None and f.cfl == 0.4 and f.h == pytest.approx(0.04)
    assert DFSPHConfig(surface_tension="csf").unsupported() == ["surface_tension 'csf'"]
    assert DFSPHConfig().unsupported(viscosity_max=0.5) == ["viscosity weiler2018 (implicit viscosity)"]


def test_time_step_helpers():
    cfg = DFSPHConfig(particle_radius=0.01)
    assert C.stable_dt(cfg, 0.0) == cfg.dt_max
    assert C.stable_dt(cfg, float("inf")) == cfg.dt_min
    assert C.stable_dt(cfg, 10.0) == pytest.approx(0.2 * 0.02 / 10.0)
    assert C.snap_down(3.0e-4, 0.02) == 0.02 / 128 and C.snap_down(3.2e-4, 0.02) == 0.02 / 64
    assert C.snap_down(1e-9, 0.02) == 0.02 / 1024


def test_emitter_layer_matches_the_reference_rule():
    # a 0.3 m nozzle at 0.1 m spacing has 3 columns, not 2 (emitters.py:48-64)
    pts = layer_offsets(np.array([0.15, 0.15, 0.05]), np.array([0.0, 0.0, -1.0]), 0.1)
    assert pts.shape == (9, 3) and np.all(pts[:, 2] == 0.0)
    assert sorted(set(np.round(pts[:, 0], 6))) == [-0.1, 0.0, 0.1]
    v = quat_rotate_inv([0.0, 0.0, np.sin(np.pi / 4), np.cos(np.pi / 4)], [1.0, 0.0, 0.0])
    np.testing.assert_allclose(v, [0.0, -1.0, 0.0], atol=1e-12)


def test_particle_box_counts_and_faces():
    pts = box_shell_points((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.02)
    assert len(pts) == 52**3 - 50**3
    assert np.isclose(pts.min(), -0.01) and np.isclose(pts.max(), 1.01)
    open_top = box_shell_points((0.0, 0.0, 0.0), (1.0, 1.0, 1.0), 0.02, open_top=True)
    assert len(open_top) == len(pts) - 52 * 52 and open_top[:, 2].max() < 1.0
    sc = dam_break()
    assert sc.fluid_count == 8000 and sc.wall_count == 52**3 - 50**3
    h = sc.model.host()
    assert np.all(np.abs(h["q"][:8000] - np.round(h["q"][:8000] / 0.02 - 0.5) * 0.02 - 0.01) <= 0.01 * 0.02 + 1e-7)


def test_world_sharding_balances_and_keeps_world_order():
    sizes = [5000, 100, 3000, 3000, 200, 7000]
    parts = shard_worlds(sizes, 2)
    assert sorted(w for p in parts for w in p) == list(range(6))
    loads = [sum(sizes[w] for w in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes) and all(p == sorted(p) for p in parts)
    sc = batched_worlds(worlds=5, lo=300, hi=900, seed=1)
    arr = sc.model.host()
    sub = sub_arrays(arr, [1, 3])
    ws = arr["world_start"]
    np.testing.assert_array_equal(sub["q"], np.concatenate([arr["q"][ws[1]:ws[2]], arr["q"][ws[3]:ws[4]]]))
    assert sub["world_start"].tolist() == [0, ws[2] - ws[1], ws[2] - ws[1] + ws[4] - ws[3]]


def test_hydrostatic_guess_is_gravity_times_depth():
    """prime.py:20-49: k_i = |g| (z_top - z_i + r) per horizontal 2r column of liquid (here every column is full, so
    z_top is the block's top layer)."""
    import types

    from alloy_b200.solvers.sph.solver import hydrostatic_guess
    from alloy_b200.solvers.sph.testing import dam_break

    sc = dam_break(counts=(4, 3, 10), box=(0.2, 0.2, 0.4), jitter=0.0)
    fake = types.SimpleNamespace(n=sc.model.particle_count, model=sc.model, config=sc.config)
    g = hydrostatic_guess(fake, sc.model.state())
    q = sc.model.host()["q"][: sc.fluid_count].astype(np.float64)
    expect = 9.81 * (q[:, 2].max() - q[:, 2] + 0.5 * sc.config.spacing)
    np.testing.assert_allclose(g[: sc.fluid_count], expect, rtol=1e-6)
    assert (g[sc.fluid_count:] == 0).all()


def test_plugin_factory_contract():
    """plugin.py:36-61: config or DFSPHConfig fields as kwargs, unknown kwargs raise TypeError, the escape box comes
    from the scene's content (padded by max(0.25 m, the largest extent)) unless world_bounds or a config is given."""
    from alloy_b200.solvers.sph.config import DFSPHConfig
    from alloy_b200.solvers.sph.plugin import CAPABILITY, config_from_kwargs, register, REGISTRY
    from alloy_b200.solvers.sph.testing import dam_break

    sc = dam_break(counts=(4, 4, 4), box=(0.2, 0.2, 0.2))
    with pytest.raises(TypeError):
        config_from_kwargs(sc.model, {"no_such_field": 1})
    cfg, cap, auto = config_from_kwargs(sc.model, {"particle_radius": 0.01, "capacity_per_world": 10})
    assert cap == 10 and cfg.particle_radius == 0.01
    lo, hi = (np.array(v) for v in cfg.world_bounds)
    q = sc.model.host()["q"]
    ext = (q.max(0) - q.min(0)).max()
    pad = max(0.25, float(ext))
    np.testing.assert_allclose(lo, q.min(0) - pad, rtol=1e-6)
    np.testing.assert_allclose(hi, q.max(0) + pad, rtol=1e-6)
    assert auto[1] == pytest.approx(pad)
    base = DFSPHConfig(particle_radius=0.02)
    cfg, _, auto = config_from_kwargs(sc.model, {"config": base, "xsph_c": 0.05})
    assert cfg.particle_radius == 0.02 and cfg.xsph_c == 0.05 and cfg.world_bounds is None and auto is None
    assert CAPABILITY.name == "sph" and CAPABILITY.routes == frozenset({"liquid_sph"})
    register()
    assert REGISTRY["sph"]["capability"] is CAPABILITY


def test_speed_harness_scenes_follow_the_reference_harness():
    """The reference's own speed scenes (tests/solvers/sph/test_speed_gpu.py:24-39, alloy/testing/sph.py:49-115):
    sizes, config and dt, in the reference's open tanks of box shapes h thick (build.py:113-137)."""
    from alloy_b200.solvers.sph.testing import tank_dam_break, water_column

    col = water_column(32, 32, 30, r=2.0e-3)
    cfg = col.config
    assert col.fluid_count == 30720 and col.model.world_count == 1
    assert cfg.pressure_solver == "cg" and cfg.cfl == 0.4 and cfg.rest_jitter_speed is None  # the fast preset
    assert col.dt == cfg.dt_max == 1.25e-3
    s = cfg.spacing
    hs = col.model.host()
    assert len(hs["shape_type"]) == 5 and not (hs["phase"] == -1).any()  # floor and four walls, open top
    top = hs["shape_transform"][:, 2] + hs["shape_scale"][:, 2]
    assert np.isclose(top.max(), (30 + 8) * s)  # headroom of 8 layers
    assert np.isclose(hs["shape_scale"][:, 2].min(), 0.5 * cfg.h)  # the floor, h thick
    many = water_column(16, 16, 16, worlds=3, r=2.0e-3)
    assert many.fluid_count == 3 * 4096 and many.model.world_count == 3
    dam = tank_dam_break(32, 30, 32, 96, r=2.0e-3)
    assert dam.fluid_count == 30720 and dam.config.pressure_solver == "cg" and dam.config.cfl == 0.2
    assert dam.config.rest_jitter_speed == 1.5e-3  # the default config: the resting-jitter rule on
    assert dam.dt == C.snap_down(C.stable_dt(dam.config, 2.0 * (9.81 * 30 * s) ** 0.5), 0.02) == 0.02 / 64
    hd = dam.model.host()
    inner_x = hd["shape_transform"][:, 0] - hd["shape_scale"][:, 0]
    assert np.isclose(inner_x.max(), 96 * s)  # the x_hi wall's inner face


def test_bench_reports_the_harness_figures():
    """rt_factor = dt / wall time per step; world-s per wall-s = worlds x dt / wall time per step
    (test_speed_gpu.py:28-39); vs_baseline on the resting column against the published 4.6 ms per step."""
    import bench
    from alloy_b200.solvers.sph.testing import water_column

    sc = water_column(8, 8, 8, worlds=4, r=2.0e-3)
    f = bench.liq9_fields("columns_256x4k", sc, 2.0e-3)
    assert f["world_s_per_wall_s"] == pytest.approx(4 * 1.25e-3 / 2.0e-3)
    col = water_column(8, 8, 8, r=2.0e-3)
    assert bench.liq9_fields("column_30k", col, 1.0e-3)["rt_factor"] == pytest.approx(1.25)
    assert bench.liq9_fields("large_dam_break", col, 1.0e-3) == {}
    assert bench.LIQ9_PUBLISHED["column_30k"] == pytest.approx(30720 / 4.6e-3)
