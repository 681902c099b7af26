# SPDX-License-Identifier: Apache-2.0
"""Seeded synthetic scenes (the role of alloy/testing/sph.py): the benchmark workloads and small test scenes.

- ``dam_break``: a jittered liquid block in the corner of a closed box of boundary particles (one layer). The
  defaults are the 1-world CPU case: 20 x 20 x 20 particles at 0.02 m in a 1 m box. ``large_dam_break`` is the
  1,048,576-particle case: 128 x 64 x 128 at 0.01 m in a 4 x 2 x 2 m tank.
- ``batched_worlds``: many uneven worlds (particle count log-uniform by seed), each a cuboid block in an open box of
  boundary particles 1.5x its extent, with spares for a spout emitter.
Config: cubic kernel, h = 4r = 2 spacings, rho0 1000, XSPH 0.01, Jacobi, tolerances 1e-3, resting-jitter rule off.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .build import add_fluid_block, add_particle_box, add_spares, box_shell_points, add_wall_particles
from .config import DFSPHConfig
from .model import Model, ModelBuilder


def benchmark_config(spacing: float, **overrides) -> DFSPHConfig:
    cfg = DFSPHConfig(particle_radius=0.5 * spacing, pressure_solver="jacobi", rest_jitter_speed=None,
                      xsph_c=0.01, viscosity="xsph", **overrides)
    cfg.validate()
    return cfg


@dataclass
class Scene:
    model: Model
    config: DFSPHConfig
    dt: float
    steps: int
    fluid_count: int
    wall_count: int
    emitters: list[dict] = field(default_factory=list)
    name: str = ""


def dam_break(counts=(20, 20, 20), box=(1.0, 1.0, 1.0), spacing: float = 0.02, jitter: float = 0.01, seed: int = 0,
              dt: float = 1.0e-3, steps: int = 200, open_top: bool = False, device="cpu", **cfg_kw) -> Scene:
    cfg = benchmark_config(spacing, **cfg_kw)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.begin_world()
    fl = add_fluid_block(b, cfg, (0.0, 0.0, 0.0), counts, jitter=jitter, seed=seed)
    wl = add_particle_box(b, cfg, (0.0, 0.0, 0.0), box, open_top=open_top)
    b.end_world()
    return Scene(b.finalize(device), cfg, dt, steps, len(fl), len(wl), name=f"dam_break_{counts}")


def large_dam_break(device="cpu", **kw) -> Scene:
    return dam_break(counts=(128, 64, 128), box=(4.0, 2.0, 2.0), spacing=0.01, dt=5.0e-4, steps=500,
                     device=device, **kw)


def world_sizes(count: int, lo: int, hi: int, seed: int) -> np.ndarray:
    """Particle counts log-uniform in [lo, hi] by seed."""
    rng = np.random.default_rng(seed)
    return np.rint(np.exp(rng.uniform(np.log(lo), np.log(hi), count))).astype(np.int64)


def _block_dims(n: int) -> tuple[int, int, int]:
    """A near-cubic nx x ny x nz block of at least n particles' lattice, height about the side."""
    side = max(int(round(n ** (1.0 / 3.0))), 1)
    nz = max(int(np.ceil(n / (side * side))), 1)
    return side, side, nz


def batched_worlds(worlds: int = 256, lo: int = 2000, hi: int = 32000, spacing: float = 0.01, seed: int = 0,
                   jitter: float = 0.01, spares_fraction: float = 0.25, spout_layer: int = 8,
                   spout_speed: float = 1.5, dt: float = 1.0e-3, steps: int = 1000, device="cpu",
                   **cfg_kw) -> Scene:
    """Uneven worlds in one model: a cuboid block per world in an open box 1.5x its extent, plus spares for a
    spout of ``spout_layer`` x ``spout_layer`` particles per layer at ``spout_speed`` downward."""
    cfg = benchmark_config(spacing, **cfg_kw)
    sizes = world_sizes(worlds, lo, hi, seed)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    emit = []
    fluid = wall = 0
    for w, n_w in enumerate(sizes):
        b.begin_world()
        nx, ny, nz = _block_dims(int(n_w))
        ext = np.array([nx, ny, nz], np.float64) * spacing
        box = tuple(float(v) for v in 1.5 * ext)
        fl = add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (nx, ny, nz), jitter=jitter, seed=seed * 100003 + w)
        wl = add_particle_box(b, cfg, (0.0, 0.0, 0.0), box, open_top=True)
        spares = add_spares(b, cfg, int(round(spares_fraction * len(fl))))
        b.end_world()
        fluid += len(fl)
        wall += len(wl)
        centre = (0.75 * ext[0] + 0.25 * box[0], 0.5 * box[1], 0.9 * box[2])
        emit.append({"world": w, "centre": centre, "half": (0.5 * spout_layer * spacing, 0.5 * spout_layer * spacing,
                                                            0.5 * spacing),
                     "velocity": (0.0, 0.0, -spout_speed), "pool": np.arange(spares.start, spares.stop)})
    return Scene(b.finalize(device), cfg, dt, steps, fluid, wall, emit, name=f"batched_{worlds}")


__all__ = ["Scene", "benchmark_config", "dam_break", "large_dam_break", "batched_worlds", "world_sizes",
           "box_shell_points", "add_wall_particles"]
