# SPDX-License-Identifier: Apache-2.0
"""Seeded synthetic scenes (the role of alloy/testing/sph.py): the benchmark workloads and small test scenes.

- ``dam_break``: a jittered liquid block in the corner of a closed box of boundary particles (one layer). The
  defaults are the 1-world CPU case: 20 x 20 x 20 particles at 0.02 m in a 1 m box. ``large_dam_break`` is the
  1,048,576-particle case: 128 x 64 x 128 at 0.01 m in a 4 x 2 x 2 m tank.
- ``batched_worlds``: many uneven worlds (particle count log-uniform by seed), each a cuboid block in an open box of
  boundary particles 1.5x its extent, with spares for a spout emitter.
- ``water_column``: the reference's resting column (its own speed harness, tests/solvers/sph/test_speed_gpu.py), one
  world or many, primed before stepping; ``tank_dam_break`` is the same harness's 30k-particle dam break.
- ``pour_bowls``: thousands of worlds, each a hemisphere bowl of boundary particles moving on a seeded sinusoid
  (``BowlMotion`` drives the wall velocities between steps) with liquid resting in it and a spout pouring in.
- ``tank_impacts``, ``shape_obstacles``: parity scenes for walls hit hard (box tanks; spheres, capsules, cylinders,
  planes and turned boxes).
Config: cubic kernel, h = 4r = 2 spacings, rho0 1000, XSPH 0.01, Jacobi, tolerances 1e-3, resting-jitter rule off.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .build import (add_box_tank, add_fluid_block, add_fluid_points, add_particle_box, add_spares,
                    add_wall_particles, box_shell_points, jittered)
from .config import DFSPHConfig, snap_down, stable_dt
from .model import Model, ModelBuilder


def benchmark_config(spacing: float, **overrides) -> DFSPHConfig:
    kw = {"pressure_solver": "jacobi", "rest_jitter_speed": None, "xsph_c": 0.01, "viscosity": "xsph", **overrides}
    cfg = DFSPHConfig(particle_radius=0.5 * spacing, **kw)
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
    motion: object = None  # BowlMotion of kinematic walls, if any


def dam_break(counts=(20, 20, 20), box=(1.0, 1.0, 1.0), spacing: float = 0.02, jitter: float = 0.01, seed: int = 0,
              dt: float = 1.0e-3, steps: int = 200, open_top: bool = False, walls: str = "particles", device="cpu",
              **cfg_kw) -> Scene:
    """``walls``: "particles" (one layer of boundary particles) or "sdf" (the reference's box tank, walls h thick,
    alloy/testing/sph.py:101-115)."""
    cfg = benchmark_config(spacing, **cfg_kw)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.begin_world()
    fl = add_fluid_block(b, cfg, (0.0, 0.0, 0.0), counts, jitter=jitter, seed=seed)
    if walls == "sdf":
        add_box_tank(b, (0.0, 0.0, 0.0), box, wall=cfg.h, open_top=open_top)
        nw = 0
    else:
        nw = len(add_particle_box(b, cfg, (0.0, 0.0, 0.0), box, open_top=open_top))
    b.end_world()
    return Scene(b.finalize(device), cfg, dt, steps, len(fl), nw, name=f"dam_break_{counts}_{walls}")


def tank_impacts(spacing: float = 0.02, dt: float = 1.0e-3, steps: int = 10, device="cpu", **cfg_kw) -> Scene:
    """Walls hit hard (a parity scene for the projection, wall friction and sweep paths): the 6 x 6 x 8 jittered block
    thrown at 1 m/s into the corner of an open box tank (the reference's box shapes, walls h thick) and eight lone
    particles: four at 30 m/s, far past the CFL step, towards the floor and the x and y walls (swept), four at
    0.5-2 m/s grazing the walls (pushed out, lone-particle limit and friction)."""
    cfg = benchmark_config(spacing, **cfg_kw)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.begin_world()
    fl = add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (6, 6, 8), jitter=0.01, seed=3, velocity=(-1.0, -0.6, -0.4))
    lone = [((0.17, 0.06, 0.05), (30.0, 0.0, -4.0)), ((0.15, 0.17, 0.12), (0.0, 30.0, 2.0)),
            ((0.16, 0.09, 0.06), (3.0, 1.0, -30.0)), ((0.18, 0.15, 0.20), (-9.0, 28.0, -6.0)),
            ((0.19, 0.05, 0.16), (2.0, -0.5, 0.3)), ((0.14, 0.19, 0.02), (0.7, 1.5, -1.0)),
            ((0.185, 0.185, 0.09), (0.5, 0.5, -0.2)), ((0.15, 0.012, 0.011), (-0.3, -0.8, -1.2))]
    for x, v in lone:
        add_fluid_points(b, cfg, np.asarray([x]), velocity=v)
    add_box_tank(b, (0.0, 0.0, 0.0), (0.2, 0.2, 0.24), wall=cfg.h, open_top=True)
    b.end_world()
    return Scene(b.finalize(device), cfg, dt, steps, len(fl) + len(lone), 0, name="tank_impacts")


def shape_obstacles(spacing: float = 0.02, dt: float = 1.0e-3, steps: int = 20, device="cpu", **cfg_kw) -> Scene:
    """Static shapes other than axis-aligned boxes (a parity scene for their slots, sweep and projection): a 6 x 6 x 5
    jittered block falling at 0.5 m/s onto a sphere (r 0.05 m) and a capsule along z (r 0.025 m, half height 0.04 m)
    standing on the infinite ground plane z = 0, beside a finite plane (a 0.08 m square shelf), a box turned 45 degrees
    about z and a cylinder lying along y, inside side walls of box shapes h thick with no floor; six lone particles at
    30 m/s, past the CFL step, towards the sphere, the capsule's cap and side, the ground, the cylinder and the turned
    box (swept)."""
    cfg = benchmark_config(spacing, **cfg_kw)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.begin_world()
    fl = add_fluid_block(b, cfg, (0.06, 0.06, 0.16), (6, 6, 5), jitter=0.01, seed=4, velocity=(0.0, 0.0, -0.5))
    lone = [((0.15, 0.15, 0.20), (0.0, 0.0, -30.0)), ((0.07, 0.22, 0.17), (0.5, 0.0, -30.0)),
            ((0.25, 0.25, 0.02), (1.0, 0.0, -30.0)), ((0.12, 0.22, 0.08), (-30.0, 0.5, 0.0)),
            ((0.06, 0.08, 0.09), (0.0, 0.3, -30.0)), ((0.24, 0.22, 0.15), (0.2, 0.0, -30.0))]
    for x, v in lone:
        add_fluid_points(b, cfg, np.asarray([x]), velocity=v)
    add_box_tank(b, (0.0, 0.0, 0.0), (0.3, 0.3, 0.4), wall=cfg.h, open_top=True, floor=False)
    b.add_shape_sphere(-1, (0.15, 0.15, 0.08), radius=0.05, mu=0.4)
    b.add_shape_capsule(-1, (0.07, 0.22, 0.08), radius=0.025, half_height=0.04, mu=0.6)
    b.add_shape_plane(-1, (0.23, 0.07, 0.12), width=0.08, length=0.08, mu=0.3)
    b.add_shape_box(-1, (0.24, 0.22, 0.05, 0.0, 0.0, 0.38268343, 0.9238795), 0.03, 0.015, 0.05, mu=0.2)
    b.add_shape_cylinder(-1, (0.06, 0.08, 0.03, 0.70710677, 0.0, 0.0, 0.70710677), radius=0.02, half_height=0.05,
                         mu=0.5)
    b.end_world()
    b.add_ground_plane(0.0, mu=0.5)
    return Scene(b.finalize(device), cfg, dt, steps, len(fl) + len(lone), 0, name="shape_obstacles")


def large_dam_break(device="cpu", **kw) -> Scene:
    return dam_break(counts=(128, 64, 128), box=(4.0, 2.0, 2.0), spacing=0.01, dt=5.0e-4, steps=500,
                     device=device, **kw)


def water_column(nx: int = 6, ny: int = 6, nz: int = 20, *, worlds: int = 1, r: float = 1.0e-3, headroom: int = 8,
                 dt: float = 1.25e-3, steps: int = 400, walls: str = "sdf", device="cpu", **cfg_kw) -> Scene:
    """A resting column nx x ny x nz on the 2r lattice filling the floor of an open box tank per world (the
    reference's ``alloy.testing.sph.water_column``, alloy/testing/sph.py:49-73): ``walls`` "sdf" the reference's tank
    of box shapes h thick, "particles" one layer of boundary particles (closed top) on the same inner box. Config: the
    reference's ``fast`` preset (projected CG, the resting-jitter rule off, config.py:146-157); dt = dt_max."""
    cfg = DFSPHConfig.fast(particle_radius=r, **cfg_kw)
    cfg.validate()
    s = cfg.spacing
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    fluid = wall = 0
    inner_hi = (nx * s, ny * s, (nz + headroom) * s)
    for _ in range(worlds):
        b.begin_world()
        if walls == "sdf":
            add_box_tank(b, (0.0, 0.0, 0.0), inner_hi, wall=cfg.h)
        fl = add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (nx, ny, nz))
        if walls != "sdf":
            wall += len(add_particle_box(b, cfg, (0.0, 0.0, 0.0), inner_hi))
        b.end_world()
        fluid += len(fl)
    return Scene(b.finalize(device), cfg, dt, steps, fluid, wall, name=f"water_column_{worlds}x{nx}x{ny}x{nz}")


def tank_dam_break(width: int = 32, height: int = 30, depth: int = 32, tank: int = 96, *, r: float = 2.0e-3,
                   steps: int = 400, walls: str = "sdf", device="cpu", **cfg_kw) -> Scene:
    """The reference harness's dam break (alloy/testing/sph.py:101-115): a width x depth x height lattice block
    against the x_lo wall of an open tank (tank x depth x (height + 10)) spacings, of box shapes h thick (``walls``
    "sdf", the reference's) or one layer of boundary particles ("particles"). The reference's default config
    (projected CG, CFL 0.2, the resting-jitter rule on); dt is the CFL step at the Ritter front speed 2 sqrt(g H),
    snapped down to 0.02 s / 2^j (test_speed_gpu.py:30-31)."""
    cfg = DFSPHConfig(particle_radius=r, **cfg_kw)
    cfg.validate()
    s = cfg.spacing
    dt = snap_down(stable_dt(cfg, 2.0 * (9.81 * height * s) ** 0.5), 0.02)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    inner_hi = (tank * s, depth * s, (height + 10) * s)
    b.begin_world()
    if walls == "sdf":
        add_box_tank(b, (0.0, 0.0, 0.0), inner_hi, wall=cfg.h)
    fl = add_fluid_block(b, cfg, (0.0, 0.0, 0.0), (width, depth, height))
    nw = 0 if walls == "sdf" else len(add_particle_box(b, cfg, (0.0, 0.0, 0.0), inner_hi))
    b.end_world()
    return Scene(b.finalize(device), cfg, dt, steps, len(fl), nw, name=f"tank_dam_break_{width}x{depth}x{height}")


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


def hemisphere_shell_points(centre, radius: float, spacing: float) -> np.ndarray:
    """One layer of wall-particle centres on the lower half of the sphere of radius ``radius + spacing / 2`` about
    ``centre``: rings of constant latitude one spacing apart along the meridian, each with its circumference / spacing
    points (the innermost face of the layer is then the bowl surface, as for the box walls)."""
    rr = radius + 0.5 * spacing
    rings = max(int(np.ceil(0.5 * np.pi * rr / spacing)), 1)
    pts = []
    for k in range(rings + 1):
        th = 0.5 * np.pi + 0.5 * np.pi * k / rings  # equator (rim) ... bottom pole
        ring_r = rr * np.sin(th)
        m = max(int(round(2.0 * np.pi * ring_r / spacing)), 1)
        ph = 2.0 * np.pi * (np.arange(m) + 0.5 * (k % 2)) / m
        pts.append(np.stack([ring_r * np.cos(ph), ring_r * np.sin(ph), np.full(m, rr * np.cos(th))], axis=1))
    return np.concatenate(pts) + np.asarray(centre, np.float64)


def bowl_interior_points(centre, radius: float, spacing: float) -> np.ndarray:
    """Lattice cell centres inside the bowl (at least half a spacing from its surface, below the rim), lowest first."""
    n = int(np.ceil(radius / spacing)) + 1
    ax = (np.arange(-n, n) + 0.5) * spacing
    g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    keep = (np.linalg.norm(g, axis=1) <= radius - 0.5 * spacing) & (g[:, 2] <= 0.0)
    g = g[keep]
    g = g[np.lexsort((g[:, 1], g[:, 0], g[:, 2]))]
    return g + np.asarray(centre, np.float64)


@dataclass
class BowlMotion:
    """Kinematic bowls: every wall particle of world w moves with the bowl's velocity
    v_w(t) = A (2 pi / T) cos(2 pi t / T + phase_w) d_w (horizontal unit direction d_w), the derivative of a
    sinusoidal path of amplitude A and period T. ``apply`` writes the velocity at the step's midpoint time into the
    state's wall particles before a step (the caller's role for kinematic bodies)."""

    wall_index: np.ndarray   # [n_wall] particle ids
    wall_world: np.ndarray   # [n_wall] world of each
    direction: np.ndarray    # [W, 3]
    phase: np.ndarray        # [W]
    amplitude: float
    period: float
    _dev: dict = field(default_factory=dict)

    def velocities(self, t: float) -> np.ndarray:
        w = 2.0 * np.pi / self.period
        return (self.amplitude * w * np.cos(w * t + self.phase))[:, None] * self.direction

    def apply(self, state, t: float, dt: float) -> None:
        import torch

        qd = state.particle_qd
        key = str(qd.device)
        if key not in self._dev:
            self._dev[key] = (torch.as_tensor(self.wall_index, dtype=torch.int64, device=qd.device),
                              torch.as_tensor(self.wall_world, dtype=torch.int64, device=qd.device))
        idx, wof = self._dev[key]
        v = torch.as_tensor(self.velocities(t + 0.5 * dt).astype(np.float32), device=qd.device)
        qd[idx] = v[wof]

    def host_velocities(self, t: float, dt: float) -> np.ndarray:
        """The same per-particle velocities as float32 host rows (for the CPU oracle)."""
        return self.velocities(t + 0.5 * dt).astype(np.float32)[self.wall_world]


def pour_bowls(worlds: int = 4096, lo: int = 4096, hi: int = 16384, spacing: float = 0.005, radius: float = 0.08,
               amplitude: float = 0.05, period: float = 1.0, spout_speed: float = 1.0, seed: int = 0,
               jitter: float = 0.01, dt: float = 1.0e-3, steps: int = 2000, device="cpu", **cfg_kw) -> Scene:
    """Batched pour: per world n_w SPH particles (log-uniform in [lo, hi] by seed), half of them (at most 80 % of the
    bowl) resting as a jittered lattice in a hemisphere bowl of boundary particles of ``radius``, the rest spares for
    a 4 x 4 spout at ``spout_speed`` downward into the bowl's centre. Every bowl moves on its own seeded sinusoid
    (``BowlMotion``); liquid that leaves the escape box is retired. Spacing 0.005 m lets a 0.08 m bowl hold the
    thousands of particles per world the workload names (at 0.01 m it holds about 1,000)."""
    cfg = benchmark_config(spacing, world_bounds=((-0.3, -0.3, -0.2), (0.3, 0.3, 0.5)), **cfg_kw)
    sizes = world_sizes(worlds, lo, hi, seed)
    # one stream per quantity, so the first k worlds of any build are the same worlds (sizes, paths, phases)
    ang = np.random.default_rng(seed + 7).uniform(0.0, 2.0 * np.pi, worlds)
    phase = np.random.default_rng(seed + 8).uniform(0.0, 2.0 * np.pi, worlds)
    direction = np.stack([np.cos(ang), np.sin(ang), np.zeros(worlds)], axis=1)
    centre = (0.0, 0.0, radius)
    shell = hemisphere_shell_points(centre, radius, spacing)
    inside = bowl_interior_points(centre, radius, spacing)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    emit, wall_index, wall_world = [], [], []
    fluid = wall = 0
    v0 = BowlMotion(np.zeros(0), np.zeros(0), direction, phase, amplitude, period).velocities(0.5 * dt)
    for w, n_w in enumerate(sizes):
        b.begin_world()
        n_liq = int(min(n_w // 2, int(0.8 * len(inside))))
        pts = jittered(inside[:n_liq], spacing, jitter, seed * 100003 + w)
        fl = add_fluid_points(b, cfg, pts)
        wl = add_wall_particles(b, cfg, shell, velocity=tuple(float(c) for c in v0[w]))
        spares = add_spares(b, cfg, int(n_w) - n_liq, park=(0.0, 0.0, radius + 0.05))
        b.end_world()
        fluid += len(fl)
        wall += len(wl)
        wall_index.append(np.arange(wl.start, wl.stop))
        wall_world.append(np.full(len(wl), w))
        emit.append({"world": w, "centre": (0.0, 0.0, radius + 0.02), "half": (2.0 * spacing, 2.0 * spacing,
                                                                             0.5 * spacing),
                     "velocity": (0.0, 0.0, -spout_speed), "pool": np.arange(spares.start, spares.stop),
                     "layer_every": spacing / spout_speed})
    motion = BowlMotion(np.concatenate(wall_index), np.concatenate(wall_world), direction, phase, amplitude, period)
    sc = Scene(b.finalize(device), cfg, dt, steps, fluid, wall, emit, name=f"pour_{worlds}")
    sc.motion = motion
    return sc


__all__ = ["Scene", "benchmark_config", "dam_break", "tank_impacts", "large_dam_break", "batched_worlds", "pour_bowls", "BowlMotion",
           "water_column", "tank_dam_break", "shape_obstacles",
           "world_sizes", "box_shell_points", "add_wall_particles", "hemisphere_shell_points", "bowl_interior_points"]
