# SPDX-License-Identifier: Apache-2.0
"""A minimal Newton-shaped particle model for SolverDFSPH: ``ModelBuilder`` -> ``Model`` -> ``State``.

The reference's solver reads a Newton ``Model`` (alloy/_vendor/newton) whose particle arrays are Warp arrays. This
package has no Warp, so ``Model`` holds the same attributes as torch tensors (on the model's device) with the same
names, shapes and dtypes: ``particle_q``/``particle_qd`` [n, 3] float32, ``particle_mass``/``particle_radius`` [n]
float32, ``particle_flags`` [n] int32 (``ParticleFlags``), ``particle_world`` [n] int32, ``particle_world_start``
[W + 1] (contiguous worlds), ``gravity`` [W, 3] float32, and the ``sph:*`` custom attributes under ``model.sph``
(``phase`` int8, ``rest_density`` float32). ``SolverDFSPH`` also accepts any object with these attributes whose
arrays expose ``__cuda_array_interface__`` (Warp arrays do).
"""

from __future__ import annotations

from dataclasses import dataclass
from enum import IntEnum
from types import SimpleNamespace

import numpy as np
import torch


class ParticleFlags(IntEnum):
    """newton ParticleFlags (geometry/flags.py:9-24)."""

    ACTIVE = 1 << 0
    PROXY = 1 << 1


class ShapeFlags(IntEnum):
    """newton ShapeFlags (geometry/flags.py:27-45): the liquid sees shapes that collide with particles."""

    VISIBLE = 1 << 0
    COLLIDE_SHAPES = 1 << 1
    COLLIDE_PARTICLES = 1 << 2


class GeoType(IntEnum):
    """newton GeoType (geometry/types.py:73-118)."""

    PLANE = 1
    HFIELD = 2
    SPHERE = 3
    CAPSULE = 4
    ELLIPSOID = 5
    CYLINDER = 6
    BOX = 7
    MESH = 8
    CONE = 9
    CONVEX_MESH = 10


@dataclass
class State:
    particle_q: torch.Tensor
    particle_qd: torch.Tensor
    particle_f: torch.Tensor | None = None
    body_q: None = None
    body_qd: None = None


class Model:
    """Finalized particle model (see module doc)."""

    def __init__(self, q, qd, mass, radius, flags, world, world_start, gravity, phase, rest_density, viscosity,
                 device, shapes: dict | None = None):
        dev = torch.device(device)
        t = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=dev)  # noqa: E731
        self.device = dev
        self.particle_count = int(len(mass))
        self.world_count = int(len(world_start) - 1)
        self.particle_q = t(np.asarray(q, np.float32).reshape(-1, 3), torch.float32)
        self.particle_qd = t(np.asarray(qd, np.float32).reshape(-1, 3), torch.float32)
        self.particle_mass = t(mass, torch.float32)
        self.particle_radius = t(radius, torch.float32)
        self.particle_flags = t(flags, torch.int32)
        self.particle_world = t(world, torch.int32)
        self.particle_world_start = t(world_start, torch.int32)
        self.gravity = t(np.asarray(gravity, np.float32).reshape(-1, 3), torch.float32)
        self.sph = SimpleNamespace(phase=t(phase, torch.int8), rest_density=t(rest_density, torch.float32),
                                   viscosity=t(viscosity, torch.float32))
        sh = shapes or {}
        S = len(sh.get("type", ()))
        self.shape_count = S
        self.shape_type = t(np.asarray(sh.get("type", np.zeros(0)), np.int32), torch.int32)
        self.shape_scale = t(np.asarray(sh.get("scale", np.zeros((0, 3))), np.float32).reshape(-1, 3), torch.float32)
        self.shape_transform = t(np.asarray(sh.get("xform", np.zeros((0, 7))), np.float32).reshape(-1, 7),
                                 torch.float32)
        self.shape_world = t(np.asarray(sh.get("world", np.zeros(0)), np.int32), torch.int32)
        self.shape_flags = t(np.asarray(sh.get("flags", np.zeros(0)), np.int32), torch.int32)
        self.shape_body = t(np.asarray(sh.get("body", np.zeros(0)), np.int32), torch.int32)
        self.shape_material_mu = t(np.asarray(sh.get("mu", np.zeros(0)), np.float32), torch.float32)
        self.sph.shape_boundary = t(np.asarray(sh.get("boundary", np.zeros(0)), np.int8), torch.int8)
        self.body_count = 0

    def state(self) -> State:
        return State(self.particle_q.clone(), self.particle_qd.clone())

    def host(self) -> dict[str, np.ndarray]:
        """Host copies of every particle array (tests, the oracle)."""
        c = lambda x: x.detach().cpu().numpy().copy()  # noqa: E731
        return {"q": c(self.particle_q), "qd": c(self.particle_qd), "mass": c(self.particle_mass),
                "radius": c(self.particle_radius), "flags": c(self.particle_flags), "world": c(self.particle_world),
                "world_start": c(self.particle_world_start), "gravity": c(self.gravity), "phase": c(self.sph.phase),
                "rest_density": c(self.sph.rest_density), "viscosity": c(self.sph.viscosity),
                "shape_type": c(self.shape_type),
                "shape_scale": c(self.shape_scale), "shape_transform": c(self.shape_transform),
                "shape_world": c(self.shape_world), "shape_flags": c(self.shape_flags),
                "shape_body": c(self.shape_body), "shape_mu": c(self.shape_material_mu),
                "shape_boundary": c(self.sph.shape_boundary)}


class ModelBuilder:
    """Collects particles world by world (``begin_world``/``end_world``) like newton.ModelBuilder."""

    def __init__(self, gravity=(0.0, 0.0, -9.81)):
        self.gravity = tuple(float(g) for g in gravity)
        self._cols: dict[str, list[np.ndarray]] = {k: [] for k in
                                                   ("q", "qd", "mass", "radius", "flags", "phase", "rho0", "mu",
                                                    "world")}
        self._world = -1
        self._world_count = 0
        self._world_gravity: list[tuple[float, float, float]] = []
        self._shapes: dict[str, list] = {k: [] for k in ("type", "scale", "xform", "world", "flags", "body", "mu",
                                                          "boundary")}

    @property
    def shape_count(self) -> int:
        return len(self._shapes["type"])

    def _add_shape(self, geo: int, scale, body: int, xform, mu: float, collide_particles: bool,
                   sph_boundary: int) -> int:
        x = np.zeros(7, np.float32)
        x[6] = 1.0
        if xform is not None:
            v = np.asarray(tuple(xform), np.float32).reshape(-1)
            x[: v.size] = v
        sh = self._shapes
        sh["type"].append(int(geo))
        sh["scale"].append(tuple(float(a) for a in scale))
        sh["xform"].append(x)
        sh["world"].append(self._world)
        sh["flags"].append(int(ShapeFlags.VISIBLE | ShapeFlags.COLLIDE_SHAPES |
                               (ShapeFlags.COLLIDE_PARTICLES if collide_particles else 0)))
        sh["body"].append(int(body))
        sh["mu"].append(float(mu))
        sh["boundary"].append(int(sph_boundary))
        return len(sh["type"]) - 1

    def add_shape_box(self, body: int = -1, xform=None, hx: float = 0.5, hy: float = 0.5, hz: float = 0.5,
                      mu: float = 1.0, collide_particles: bool = True, sph_boundary: int = 0) -> int:
        """A box shape (half extents hx, hy, hz) at ``xform`` = (px, py, pz[, qx, qy, qz, qw]) in the current world
        (global, world -1, when no world is open), as newton.ModelBuilder.add_shape_box; ``sph_boundary`` is the
        sph:shape_boundary attribute (0 auto, 1 sdf, 2 akinci, 3 ignore). Returns the shape id."""
        return self._add_shape(GeoType.BOX, (hx, hy, hz), body, xform, mu, collide_particles, sph_boundary)

    def add_shape_sphere(self, body: int = -1, xform=None, radius: float = 1.0, mu: float = 1.0,
                         collide_particles: bool = True, sph_boundary: int = 0) -> int:
        """A sphere shape (scale (radius, 0, 0)), as newton.ModelBuilder.add_shape_sphere."""
        return self._add_shape(GeoType.SPHERE, (radius, 0.0, 0.0), body, xform, mu, collide_particles, sph_boundary)

    def add_shape_capsule(self, body: int = -1, xform=None, radius: float = 1.0, half_height: float = 0.5,
                          mu: float = 1.0, collide_particles: bool = True, sph_boundary: int = 0) -> int:
        """A capsule along the shape's z axis (scale (radius, half_height, 0)), as newton.ModelBuilder.add_shape_capsule
        with its axis along z."""
        return self._add_shape(GeoType.CAPSULE, (radius, half_height, 0.0), body, xform, mu, collide_particles,
                               sph_boundary)

    def add_shape_cylinder(self, body: int = -1, xform=None, radius: float = 1.0, half_height: float = 0.5,
                           mu: float = 1.0, collide_particles: bool = True, sph_boundary: int = 0) -> int:
        """A straight cylinder along the shape's z axis (scale (radius, half_height, 0)), as
        newton.ModelBuilder.add_shape_cylinder."""
        return self._add_shape(GeoType.CYLINDER, (radius, half_height, 0.0), body, xform, mu, collide_particles,
                               sph_boundary)

    def add_shape_plane(self, body: int = -1, xform=None, width: float = 0.0, length: float = 0.0, mu: float = 1.0,
                        collide_particles: bool = True, sph_boundary: int = 0) -> int:
        """A plane through the shape's origin with normal along its z axis, finite (width along x, length along y) when
        both are positive, else infinite, as newton.ModelBuilder.add_shape_plane."""
        return self._add_shape(GeoType.PLANE, (width, length, 0.0), body, xform, mu, collide_particles, sph_boundary)

    def add_ground_plane(self, height: float = 0.0, mu: float = 1.0) -> int:
        """The infinite ground plane z = height, normal +z (newton.ModelBuilder.add_ground_plane with z up), global."""
        world, self._world = self._world, -1
        try:
            return self.add_shape_plane(-1, (0.0, 0.0, height), mu=mu)
        finally:
            self._world = world

    @property
    def particle_count(self) -> int:
        return int(sum(len(a) for a in self._cols["mass"]))

    @property
    def current_world(self) -> int:
        return self._world

    def begin_world(self, gravity=None) -> int:
        if self._world >= 0:
            raise ValueError("begin_world: end the current world first")
        self._world = self._world_count
        self._world_count += 1
        self._world_gravity.append(tuple(float(g) for g in (gravity or self.gravity)))
        return self._world

    def end_world(self) -> None:
        self._world = -1

    def add_particles(self, pos, vel, mass, radius, flags, phase, rest_density=1000.0, viscosity=1.0e-3) -> range:
        if self._world < 0:
            raise ValueError("add_particles: particles belong to a world (begin_world first)")
        pos = np.asarray(pos, np.float32).reshape(-1, 3)
        n = len(pos)
        first = self.particle_count
        bc = lambda v, dt: np.broadcast_to(np.asarray(v, dt), (n,) + np.shape(np.asarray(v))[1:]).copy()  # noqa: E731
        self._cols["q"].append(pos)
        self._cols["qd"].append(np.broadcast_to(np.asarray(vel, np.float32), (n, 3)).copy())
        self._cols["mass"].append(bc(mass, np.float32).reshape(n))
        self._cols["radius"].append(bc(radius, np.float32).reshape(n))
        self._cols["flags"].append(bc(flags, np.int32).reshape(n))
        self._cols["phase"].append(bc(phase, np.int8).reshape(n))
        self._cols["rho0"].append(bc(rest_density, np.float32).reshape(n))
        self._cols["mu"].append(bc(viscosity, np.float32).reshape(n))
        self._cols["world"].append(np.full(n, self._world, np.int32))
        return range(first, first + n)

    def finalize(self, device="cpu") -> Model:
        cat = lambda k, dt, shape=(0,): (np.concatenate(self._cols[k]).astype(dt) if self._cols[k]  # noqa: E731
                                         else np.zeros(shape, dt))
        world = cat("world", np.int32)
        W = self._world_count
        if len(world) and np.any(np.diff(world) < 0):
            raise ValueError("particles must be contiguous per world")
        counts = np.bincount(world, minlength=W) if W else np.zeros(0, np.int64)
        ws = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
        return Model(cat("q", np.float32, (0, 3)), cat("qd", np.float32, (0, 3)), cat("mass", np.float32),
                     cat("radius", np.float32), cat("flags", np.int32), world, ws,
                     np.asarray(self._world_gravity or [self.gravity], np.float32).reshape(-1, 3),
                     cat("phase", np.int8), cat("rho0", np.float32), cat("mu", np.float32), device,
                     shapes=self._shapes if self.shape_count else None)
