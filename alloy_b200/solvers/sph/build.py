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


BOUNDARY_SDF = 1  # sph:shape_boundary (config.py:41-44)


def wall_box(builder: ModelBuilder, center: Vec3, half: Vec3, mu: float = 1.0) -> int:
    """One static wall the liquid sees through its signed distance field: a box shape (build.py:104-110)."""
    return builder.add_shape_box(-1, tuple(center), *half, mu=mu, sph_boundary=BOUNDARY_SDF)


def add_box_tank(builder: ModelBuilder, inner_lo: Vec3, inner_hi: Vec3, wall: float, *, open_top: bool = True,
                 floor: bool = True, mu: float = 1.0) -> dict[str, int]:
    """A static axis-aligned tank of box walls ``wall`` thick around the inner box (build.py:113-137): the floor spans
    the full footprint, the x walls the full y extent, the y walls sit between them, so every solid point belongs to
    exactly one box. Returns the shape ids by name (floor, x_lo, x_hi, y_lo, y_hi[, lid])."""
    lo, hi = np.asarray(inner_lo, np.float64), np.asarray(inner_hi, np.float64)
    c = 0.5 * (lo + hi)
    hx, hy, hz = 0.5 * (hi - lo)
    t = 0.5 * wall
    ids = {}
    if floor:
        ids["floor"] = wall_box(builder, (c[0], c[1], lo[2] - t), (hx + wall, hy + wall, t), mu)
    for name, sx in (("x_lo", -1.0), ("x_hi", 1.0)):
        ids[name] = wall_box(builder, (c[0] + sx * (hx + t), c[1], c[2]), (t, hy + wall, hz), mu)
    for name, sy in (("y_lo", -1.0), ("y_hi", 1.0)):
        ids[name] = wall_box(builder, (c[0], c[1] + sy * (hy + t), c[2]), (hx, t, hz), mu)
    if not open_top:
        ids["lid"] = wall_box(builder, (c[0], c[1], hi[2] + t), (hx + wall, hy + wall, t), mu)
    return ids


# ------------------------------------------------------------------------------------------------ scene assembly emit
DISK_CLEAR = 0.375  # a cylinder's outer ring of particles stays this many spacings inside its side (build.py:226)


def inside_primitive(pts: np.ndarray, kind: str, size) -> np.ndarray:
    """Points inside a primitive centred at the origin (cylinder and capsule along z; build.py:181-197)."""
    r2 = pts[:, 0] ** 2 + pts[:, 1] ** 2
    if kind == "box":
        return np.all(np.abs(pts) <= np.asarray(size[:3], np.float64), axis=1)
    if kind == "sphere":
        return r2 + pts[:, 2] ** 2 <= size[0] ** 2
    if kind == "cylinder":
        return (r2 <= size[0] ** 2) & (np.abs(pts[:, 2]) <= size[1])
    if kind == "capsule":
        over = np.maximum(np.abs(pts[:, 2]) - size[1], 0.0)
        return r2 + over ** 2 <= size[0] ** 2
    if kind == "ellipsoid":
        return np.sum((pts / np.asarray(size[:3], np.float64)) ** 2, axis=1) <= 1.0
    raise ValueError(f"SPH emit: no liquid volume for primitive {kind!r}")


def disk_rings(pts: np.ndarray, radius: float, spacing: float) -> np.ndarray:
    """A cylinder's lattice points out to the ring of equal axis distance whose per-layer count comes closest to the
    disk's area / spacing^2 without exceeding it, that ring at least ``DISK_CLEAR`` spacings inside the side
    (build.py:229-246): a square lattice in a small disk can hold more points than its area, which starts the liquid
    compressed."""
    if len(pts) == 0:
        return pts
    dist = np.round(np.hypot(pts[:, 0], pts[:, 1]), 9)
    layer = np.sort(dist[pts[:, 2] == pts[0, 2]])
    rings = np.unique(layer)
    within = np.searchsorted(layer, rings, side="right")
    area = np.pi * radius ** 2 / spacing ** 2
    fits = (within <= area + 1.0e-9) & (rings <= radius - DISK_CLEAR * spacing + 1.0e-9)
    miss = np.where(fits, np.abs(within - area), np.inf)
    pick = int(np.argmin(miss)) if np.isfinite(miss).any() else 0
    return pts[dist <= rings[pick]]


def column_layers(pts: np.ndarray, radius: float, half_height: float, spacing: float) -> np.ndarray:
    """``disk_rings``' column topped up with whole layers until its count is closest to the cylinder's volume /
    spacing^3; the bottom layer stays (build.py:249-262)."""
    if len(pts) == 0:
        return pts
    top = float(pts[:, 2].max())
    layer = pts[np.isclose(pts[:, 2], top)]
    have = len(pts) // len(layer)
    want = np.pi * radius ** 2 * 2.0 * half_height / spacing ** 3
    extra = max(int(np.floor(want / len(layer) + 0.5)) - have, 0)
    more = [layer + np.array([0.0, 0.0, k * spacing]) for k in range(1, extra + 1)]
    return np.concatenate([pts, *more]) if more else pts


def liquid_points(shape, spacing: float) -> np.ndarray:
    """Lattice points (spacing 2r) filling a particle-source region (``shape.region`` = (lo, hi)) or a closed
    primitive (``shape.kind``, ``shape.size``; Newton's half-extent conventions), centred so the lattice sits
    symmetrically in the volume (build.py:200-223). Object frame."""
    region = getattr(shape, "region", None)
    kind = getattr(shape, "kind", None)
    if region is not None:
        lo, hi = np.asarray(region[0], np.float64), np.asarray(region[1], np.float64)
    elif kind is not None and kind != "plane":
        size = tuple(float(v) for v in shape.size)
        ext = {"box": size[:3], "sphere": (size[0],) * 3, "ellipsoid": size[:3],
               "cylinder": (size[0], size[0], size[1]) if len(size) > 1 else None,
               "capsule": (size[0], size[0], size[1] + size[0]) if len(size) > 1 else None}.get(kind)
        if ext is None:
            raise ValueError(f"SPH emit: no liquid volume for primitive {kind!r}")
        lo, hi = -np.asarray(ext, np.float64), np.asarray(ext, np.float64)
    else:
        raise ValueError(f"SPH emit: liquid needs a particle-source region or a closed primitive, got {type(shape)}")
    counts = np.maximum(np.floor((hi - lo) / spacing + 1.0e-9).astype(int), 1)
    start = 0.5 * (lo + hi) - 0.5 * counts * spacing
    pts = lattice_points(tuple(start), tuple(int(c) for c in counts), spacing)
    if region is None:
        size = tuple(float(v) for v in shape.size)
        pts = pts[inside_primitive(pts, kind, size)]
        if kind == "cylinder":
            pts = column_layers(disk_rings(pts, size[0], spacing), size[0], size[1], spacing)
    return pts


def emit_object(builder: ModelBuilder, obj, decision) -> range:
    """The plug-in's emit (build.py:265-285): a liquid object -> active lattice particles at the router's particle
    radius (``decision.numbers["particle_radius"]``), mass rho0 / S, the material's viscosity, in ``builder``'s current
    world (object frame). ``obj`` carries ``card.name``, ``card.shape``, ``card.budget.particles`` and
    ``material.density.value`` / ``material.fluid.viscosity.value`` (fluid may be None: 1e-3 Pa s). Raises
    CapacityError over the particle budget."""
    from ... import _lib

    r = float(decision.numbers.get("particle_radius", 0.0))
    if not r > 0.0:
        raise ValueError(f"{obj.card.name}: liquid_sph decision without particle_radius")
    cfg = DFSPHConfig(particle_radius=r)
    pts = liquid_points(obj.card.shape, cfg.spacing)
    budget = obj.card.budget.particles
    if len(pts) > budget:
        raise _lib.CapacityError(f"{obj.card.name}: {len(pts)} SPH particles at r = {r:.3g} m > budget {budget}")
    fluid = obj.material.fluid
    mu = float(fluid.viscosity.value) if fluid is not None else 1.0e-3
    return add_fluid_points(b=builder, cfg=cfg, points=pts, rest_density=float(obj.material.density.value),
                            viscosity=mu)
