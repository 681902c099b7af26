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
                 device):
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
        self.shape_count = 0
        self.body_count = 0

    def state(self) -> State:
        return State(self.particle_q.clone(), self.particle_qd.clone())

    def host(self) -> dict[str, np.ndarray]:
        """Host copies of every particle array (tests, the oracle)."""
        c = lambda x: x.detach().cpu().numpy().copy()  # noqa: E731
        return {"q": c(self.particle_q), "qd": c(self.particle_qd), "mass": c(self.particle_mass),
                "radius": c(self.particle_radius), "flags": c(self.particle_flags), "world": c(self.particle_world),
                "world_start": c(self.particle_world_start), "gravity": c(self.gravity), "phase": c(self.sph.phase),
                "rest_density": c(self.sph.rest_density)}


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
                     cat("phase", np.int8), cat("rho0", np.float32), cat("mu", np.float32), device)
