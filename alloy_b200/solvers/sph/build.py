# SPDX-License-Identifier: Apache-2.0
"""Scene helpers: liquid blocks on the 2r lattice, spares, and walls made of boundary particles.

Liquid follows the reference's builders (alloy/solvers/sph/build.py:26-81): lattice cell centres ``lo + (i + 0.5) s``
in x-major order (x slowest, z fastest), mass rho0 / S, flags ACTIVE, sph phase 1. Walls are particle walls
(alloy/solvers/sph/particle_walls.py:1-27): particles flagged ACTIVE | PROXY with sph phase -1 and radius s / 2, so
each carries the cuboid volume V = 8 r^3 = s^3; one layer of them on the lattice ``lo - s/2 + k s`` encloses the inner
box ``[lo, hi]``, whose faces then sit half a spacing from the wall particles' centres.
"""

from __future__ import annotations

import numpy as np

from .config import PHASE_LIQUID, PHASE_NONE, PHASE_SPARE, DFSPHConfig, particle_mass
from .model import ModelBuilder, ParticleFlags

Vec3 = tuple[float, float, float]


def lattice_points(lo: Vec3, counts: tuple[int, int, int], spacing: float) -> np.ndarray:
    """Cell centres of an nx x ny x nz lattice with cells of side ``spacing`` starting at corner ``lo`` [n, 3]."""
    axes = [lo[k] + (np.arange(n) + 0.5) * spacing for k, n in enumerate(counts)]
    g = np.meshgrid(*axes, indexing="ij")
    return np.stack([a.ravel() for a in g], axis=1)


def jittered(points: np.ndarray, spacing: float, fraction: float, seed: int) -> np.ndarray:
    """Points plus seeded uniform jitter of +-fraction x spacing per coordinate, cast to float32 after adding."""
    if fraction <= 0.0:
        return points.astype(np.float32)
    rng = np.random.default_rng(seed)
    return (points + rng.uniform(-fraction, fraction, points.shape) * spacing).astype(np.float32)


def add_fluid_points(b: ModelBuilder, cfg: DFSPHConfig, points: np.ndarray, rest_density: float = 1000.0,
                     viscosity: float = 1.0e-3, velocity: Vec3 = (0.0, 0.0, 0.0)) -> range:
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    m = particle_mass(cfg, rest_density)
    return b.add_particles(pts, velocity, m, cfg.particle_radius, int(ParticleFlags.ACTIVE), PHASE_LIQUID,
                           rest_density, viscosity)


def add_fluid_block(b: ModelBuilder, cfg: DFSPHConfig, lo: Vec3, counts: tuple[int, int, int],
                    rest_density: float = 1000.0, jitter: float = 0.0, seed: int = 0,
                    velocity: Vec3 = (0.0, 0.0, 0.0)) -> range:
    pts = jittered(lattice_points(lo, counts, cfg.spacing), cfg.spacing, jitter, seed)
    return add_fluid_points(b, cfg, pts, rest_density, velocity=velocity)


def add_spares(b: ModelBuilder, cfg: DFSPHConfig, count: int, rest_density: float = 1000.0,
               park: Vec3 = (0.0, 0.0, 0.0)) -> range:
    """Inactive spare particles (ACTIVE cleared, phase 0) for emitters (build.py:67-81)."""
    if count <= 0:
        return range(b.particle_count, b.particle_count)
    m = particle_mass(cfg, rest_density)
    return b.add_particles(np.tile(np.asarray(park, np.float32), (count, 1)), (0.0, 0.0, 0.0), m,
                           cfg.particle_radius, 0, PHASE_SPARE, rest_density)


def box_shell_points(inner_lo: Vec3, inner_hi: Vec3, spacing: float, open_top: bool = False) -> np.ndarray:
    """One layer of wall-particle centres around the inner box: the lattice lo - s/2 + k s, k = 0..N per axis,
    keeping the points on the lattice's outer faces (without the top face when ``open_top``)."""
    lo, hi = np.asarray(inner_lo, np.float64), np.asarray(inner_hi, np.float64)
    n = np.rint((hi - lo) / spacing).astype(int) + 1
    axes = [lo[a] - 0.5 * spacing + np.arange(n[a] + 1) * spacing for a in range(3)]
    idx = np.stack(np.meshgrid(*[np.arange(n[a] + 1) for a in range(3)], indexing="ij"), -1).reshape(-1, 3)
    on = np.zeros(len(idx), bool)
    for a in range(3):
        on |= idx[:, a] == 0
        if not (open_top and a == 2):
            on |= idx[:, a] == n[a]
    if open_top:
        on &= idx[:, 2] < n[2]
    idx = idx[on]
    return np.stack([axes[a][idx[:, a]] for a in range(3)], axis=1)


def add_wall_particles(b: ModelBuilder, cfg: DFSPHConfig, points: np.ndarray, spacing: float | None = None,
                       velocity: Vec3 = (0.0, 0.0, 0.0)) -> range:
    """Boundary particles (ACTIVE | PROXY, phase -1, radius s/2: volume s^3) at ``points``."""
    s = cfg.spacing if spacing is None else spacing
    pts = np.asarray(points, np.float32).reshape(-1, 3)
    m = particle_mass(cfg, 1000.0)
    return b.add_particles(pts, velocity, m, 0.5 * s, int(ParticleFlags.ACTIVE | ParticleFlags.PROXY), PHASE_NONE,
                           1000.0)


def add_particle_box(b: ModelBuilder, cfg: DFSPHConfig, inner_lo: Vec3, inner_hi: Vec3,
                     open_top: bool = False) -> range:
    return add_wall_particles(b, cfg, box_shell_points(inner_lo, inner_hi, cfg.spacing, open_top))
