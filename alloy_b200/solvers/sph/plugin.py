# SPDX-License-Identifier: Apache-2.0
"""The ``sph`` solver capability of the B200 DFSPH step: the registration contract of the reference's
``alloy/solvers/sph/plugin.py`` (factory, capability fields, health and state adapters), so that alloy's router can
build this solver where it builds its own.

``_factory(view, kwargs)`` follows ``plugin.py:36-61``: ``config`` (a DFSPHConfig) or DFSPHConfig fields as kwargs,
plus ``capacity_per_world``; unknown kwargs raise ``TypeError``; without ``config`` and without a ``world_bounds``
kwarg the escape box comes from the scene's content (``escape_box.py:44-94``: the box of the finite shapes and the
particles, padded by ``max(0.25 m, its largest extent)`` on every side). ``register(registry)`` hands the capability and the adapters to
alloy's registry when one is given (``alloy.core.registry.register_solver`` and friends), else records them in this
module's ``REGISTRY``.
"""

from __future__ import annotations

import dataclasses
import logging
from collections.abc import Mapping
from dataclasses import dataclass
from typing import Any, Callable

import numpy as np

from .config import DFSPHConfig
from .solver import SolverDFSPH, _host

log = logging.getLogger("alloy.sph")

_CONFIG_FIELDS = frozenset(f.name for f in dataclasses.fields(DFSPHConfig))
AUTO_PAD_MIN = 0.25  # escape_box.py:30
PLANE_RADIUS = 1.0e5  # escape_box.py:32: shapes with a larger bounding radius (planes) are not content


def content_box(model: Any):
    """(lo, hi) of the model's finite shapes (their bounding spheres about their origins; planes are left out) and of
    every particle with a finite position (active ones and spares), over all worlds; None for an empty model
    (escape_box.py:44-75)."""
    pts = np.zeros((0, 3))
    if int(getattr(model, "particle_count", 0) or 0):
        q = _host(model.particle_q).astype(np.float64).reshape(-1, 3)
        pts = q[np.isfinite(q).all(axis=1)]
    lo_s, hi_s = np.zeros((0, 3)), np.zeros((0, 3))
    S = int(getattr(model, "shape_count", 0) or 0)
    if S:
        from .shapes import shape_radius

        geo = _host(model.shape_type).astype(np.int32)
        scale = _host(model.shape_scale).astype(np.float64).reshape(-1, 3)
        c = _host(model.shape_transform).astype(np.float64).reshape(-1, 7)[:, :3]
        r = np.array([shape_radius(int(geo[k]), scale[k]) for k in range(S)])
        keep = np.isfinite(r) & (r < PLANE_RADIUS) & np.isfinite(c).all(axis=1)
        lo_s, hi_s = c[keep] - r[keep, None], c[keep] + r[keep, None]
    if len(pts) == 0 and len(lo_s) == 0:
        return None
    return np.vstack([lo_s, pts]).min(axis=0), np.vstack([hi_s, pts]).max(axis=0)


def auto_box(model: Any, pad_min: float = AUTO_PAD_MIN):
    """((lo, hi), pad): the content box padded by max(pad_min, its largest extent) on every side; None for an empty
    model (escape_box.py:78-94)."""
    box = content_box(model)
    if box is None:
        return None
    lo, hi = box
    pad = max(float(pad_min), float((hi - lo).max()))
    return (tuple(float(v) for v in lo - pad), tuple(float(v) for v in hi + pad)), pad


def config_from_kwargs(view: Any, kwargs: Mapping[str, Any]):
    """(DFSPHConfig, capacity_per_world, automatic box or None) of a factory call (plugin.py:36-57)."""
    kw = dict(kwargs)
    cfg = kw.pop("config", None)
    cap = kw.pop("capacity_per_world", None)
    fields = {k: kw.pop(k) for k in list(kw) if k in _CONFIG_FIELDS}
    if kw:
        raise TypeError(f"sph factory: unknown kwargs {sorted(kw)}")
    auto = None
    if cfg is None:
        if "world_bounds" not in fields:
            auto = auto_box(view)
            fields["world_bounds"] = None if auto is None else auto[0]
            log.info("sph factory: escape box %s from the scene's content", fields["world_bounds"])
        cfg = DFSPHConfig(**fields)
    elif fields:
        cfg = dataclasses.replace(cfg, **fields)
    return cfg, cap, auto


def _factory(view: Any, kwargs: Mapping[str, Any]) -> SolverDFSPH:
    """The capability's factory (plugin.py:36-61)."""
    cfg, cap, auto = config_from_kwargs(view, kwargs)
    solver = SolverDFSPH(view, cfg, capacity_per_world=cap)
    if auto is not None:
        solver.escape_box_pad = auto[1]  # an automatic box: a drive may widen it
    return solver


@dataclass(frozen=True)
class SolverCapability:
    """The fields of alloy's SolverCapability that the sph capability sets (plugin.py:92-105)."""

    name: str
    factory: Callable[[Any, Mapping[str, Any]], Any]
    routes: frozenset
    owns: frozenset
    coupling: bool
    uniform_worlds: bool
    per_contact_friction: bool
    determinism: str
    friction_mix: str
    restitution_path: bool
    emitter: Any = None
    register_attributes: Callable | None = None


class _SPHEmitter:
    """Emitter protocol adapter: SolverDFSPH.add_emitter on the solver the router built."""

    def emit(self, solver: SolverDFSPH, world: int, region, half_extents, rate: float, velocity, pool=None) -> int:
        return solver.add_emitter(world, region, half_extents, rate, velocity, pool)


def register_custom_attributes(builder) -> None:
    """The sph:* particle attributes the solver reads (config.py:244-261: rest_density, viscosity, phase, ...). This
    package's ModelBuilder carries them on every model it builds, so there is nothing to add; a Newton builder gets
    them from alloy's own registration, which the router runs before the factory."""
    del builder


def health(solver: SolverDFSPH) -> dict[str, np.ndarray]:
    """The health adapter's sample (plugin.py:72-86): per world the pressure iterations of the last step and the mean
    density error."""
    r = solver.report()
    return {"iters": (r.iters_density + r.iters_divergence).astype(np.int32),
            "residual": r.density_err.astype(np.float32)}


def state_arrays(solver: SolverDFSPH) -> dict:
    """The state adapter: the arrays a snapshot must hold beside State (coupling_hooks.py:260-271)."""
    return solver.alloy_state_arrays()


CAPABILITY = SolverCapability(
    name="sph",
    factory=_factory,
    routes=frozenset({"liquid_sph"}),
    owns=frozenset({"particle", "body"}),
    coupling=True,
    uniform_worlds=False,
    per_contact_friction=False,
    determinism="native",
    friction_mix="none",
    restitution_path=False,
    emitter=_SPHEmitter(),
    register_attributes=register_custom_attributes,
)

REGISTRY: dict[str, Any] = {}


def register(registry: Any = None) -> None:
    """Register the capability and its adapters with ``registry`` (an object with alloy's ``register_solver``,
    ``register_health_adapter`` and ``register_state_adapter``), or in ``REGISTRY``; idempotent."""
    if registry is not None:
        registry.register_solver(CAPABILITY)
        registry.register_health_adapter(SolverDFSPH, health)
        registry.register_state_adapter(SolverDFSPH, state_arrays)
        return
    REGISTRY[CAPABILITY.name] = {"capability": CAPABILITY, "health": health, "state": state_arrays}
