# SPDX-License-Identifier: Apache-2.0
"""The liquid's shape walls: which model shapes bound it, per world (boundary.py:70-87 ``world_shape_table``,
layout.py:131-164 radius and thinnest wall, layout.py:207-246 ``shape_table``).

A shape bounds the liquid when it collides with particles (``ShapeFlags.COLLIDE_PARTICLES``), has a signed distance
field, and its ``sph:shape_boundary`` is not ``ignore``; each world sees its own shapes, then the global ones
(world -1). This path evaluates static shapes (no body) with closed-form distances, each in its own frame: boxes (the
walls of ``add_box_tank``), spheres, capsules and straight cylinders along their z axis, and planes with normal along
their z axis (a ground plane); the constructor refuses other particle-colliding shapes with a message naming them.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .model import GeoType, ShapeFlags

BOUNDARY_IGNORE = 3  # sph:shape_boundary (config.py:41-44)
SDF_GEOS = (GeoType.PLANE, GeoType.SPHERE, GeoType.CAPSULE, GeoType.ELLIPSOID, GeoType.CYLINDER, GeoType.BOX,
            GeoType.MESH, GeoType.CONE, GeoType.CONVEX_MESH)


@dataclass
class ShapeTable:
    start: np.ndarray   # int32 [W + 1]: world w's shapes are ids[start[w]:start[w + 1]]
    ids: np.ndarray     # int32: shape ids, each world's own then the global ones
    geo: np.ndarray     # int32 [S]
    scale: np.ndarray   # float32 [S][3]: box half extents; sphere radius; capsule/cylinder radius, half height; plane w, l
    xform: np.ndarray   # float32 [S][7]: (p, q xyzw)
    radius: np.ndarray  # float32 [S]: bounding radius about the shape origin (newton geometry/utils.py:77-110)
    mu: np.ndarray      # float32 [S]: Coulomb friction of the wall
    thinnest: float     # [m] thinnest wall of the table (layout.py:131-149), inf without shapes

    @property
    def count(self) -> int:
        return int(len(self.geo))


PATH_GEOS = (int(GeoType.BOX), int(GeoType.SPHERE), int(GeoType.CAPSULE), int(GeoType.CYLINDER), int(GeoType.PLANE))
THIN_AXES = {int(GeoType.BOX): (0, 1, 2), int(GeoType.SPHERE): (0,), int(GeoType.CAPSULE): (0,),
             int(GeoType.CYLINDER): (0, 1)}


def shape_radius(geo: int, scale) -> float:
    """The radius about the shape's origin that encloses it (newton geometry/utils.py:77-110; a plane's is unused:
    planes are never culled by distance, boundary.py:219)."""
    s = np.abs(np.asarray(scale, np.float64))
    if geo == int(GeoType.SPHERE):
        return float(s[0])
    if geo in (int(GeoType.CAPSULE), int(GeoType.CYLINDER)):
        return float(s[0] + s[1])
    if geo == int(GeoType.PLANE):
        return float(np.linalg.norm(s)) * 0.5 if s[0] > 0.0 and s[1] > 0.0 else 1.0e6
    return float(np.linalg.norm(s))


def _host(a) -> np.ndarray:
    return a.detach().cpu().numpy() if hasattr(a, "detach") else np.asarray(a)


def shape_table(model) -> ShapeTable:
    W = int(model.world_count)
    S = int(getattr(model, "shape_count", 0) or 0)
    if S == 0:
        z = np.zeros
        return ShapeTable(z(W + 1, np.int32), z(0, np.int32), z(0, np.int32), z((0, 3), np.float32),
                          z((0, 7), np.float32), z(0, np.float32), z(0, np.float32), float("inf"))
    geo = _host(model.shape_type).astype(np.int32)
    flags = _host(model.shape_flags).astype(np.int32)
    world = _host(model.shape_world).astype(np.int32)
    body = _host(model.shape_body).astype(np.int32)
    scale = _host(model.shape_scale).astype(np.float32).reshape(-1, 3)
    xform = _host(model.shape_transform).astype(np.float32).reshape(-1, 7)
    sb = getattr(getattr(model, "sph", None), "shape_boundary", None)
    boundary = _host(sb).astype(np.int32) if sb is not None and len(sb) == S else np.zeros(S, np.int32)
    usable = ((flags & int(ShapeFlags.COLLIDE_PARTICLES)) != 0) & np.isin(geo, [int(g) for g in SDF_GEOS])
    usable &= boundary != BOUNDARY_IGNORE
    bad = []
    for s in np.flatnonzero(usable):
        name = GeoType(int(geo[s])).name.lower()
        if int(geo[s]) not in PATH_GEOS:
            bad.append(f"shape {s} ({name})")
        elif body[s] >= 0:
            bad.append(f"shape {s} (a {name} on body {body[s]})")
        elif int(geo[s]) == int(GeoType.CYLINDER) and scale[s, 2] != 0.0:
            bad.append(f"shape {s} (a barrel cylinder)")
        elif abs(float(np.linalg.norm(xform[s, 3:].astype(np.float64))) - 1.0) > 1.0e-4:
            bad.append(f"shape {s} (a {name} whose rotation is not a unit quaternion)")
    if bad:
        raise ValueError("SolverDFSPH (B200 build): the liquid's shape walls must be static boxes, spheres, capsules, "
                         "straight cylinders or planes (add_box_tank, wall_box, add_shape_sphere, add_shape_capsule, "
                         "add_shape_cylinder, add_ground_plane); not on the B200 CUDA path: " + ", ".join(bad[:8]))
    glob = np.flatnonzero(usable & (world < 0))
    start, ids = [0], []
    for w in range(W):
        ids.extend(int(s) for s in np.flatnonzero(usable & (world == w)))
        ids.extend(int(s) for s in glob)
        start.append(len(ids))
    ids = np.asarray(ids, np.int32)
    radius = np.array([shape_radius(int(geo[s]), scale[s]) for s in range(S)], np.float32)
    thin = float("inf")  # layout.py:131-149: planes count as thick
    for s in np.unique(ids):
        axes = THIN_AXES.get(int(geo[s]))
        if axes is not None:
            thin = min(thin, 2.0 * float(min(float(scale[s][k]) for k in axes)))
    return ShapeTable(np.asarray(start, np.int32), ids, geo, scale, xform, radius,
                      _host(model.shape_material_mu).astype(np.float32), thin)
