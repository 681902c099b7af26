# SPDX-License-Identifier: Apache-2.0
"""Generate tests/golden/reference_kernels.json from the reference's own source (run in a container that has the
reference checkout; the committed JSON is what the tests read).

warp-lang is not installed, so ``warp`` is replaced by a minimal stand-in: decorators pass functions through and the
few math helpers the scalar functions call (clamp, abs, min, max, vec2/vec3, length) are plain Python. The
reference's scalar functions then evaluate in float64 Python arithmetic: these vectors pin the *mathematics* of
the kernels, the half-space volume, the wall fit, the lattice constants and the colour inversion, not Warp's float32
rounding. Sources used (paths inside the alloy project):
  alloy/solvers/sph/kernels.py    kernel_w, kernel_grad, projected_p, _g0, _g1, halfspace_volume, lattice_sum,
                                  boundary_fit, lattice_diagonal, _half_lattice
  alloy/solvers/sph/config.py     particle_mass, full_neighbor_count (function bodies extracted with ast)
  alloy/solvers/sph/particle_walls.py  colour_distance, pw_project (function bodies extracted with ast)
  alloy/_vendor/newton/_src/geometry/kernels.py  sdf_box, sdf_sphere, sdf_capsule, sdf_cylinder and gradients, and
  alloy/_vendor/newton/_src/geometry/soft_contacts_sdf.py  _eval_plane_sdf (reference_shape_sdf.json)

Usage: python tests/golden/make_golden.py /path/to/alloy-checkout
"""

from __future__ import annotations

import ast
import importlib.util
import json
import math
import sys
import types
from pathlib import Path

import numpy as np

OUT = Path(__file__).resolve().parent / "reference_kernels.json"


def warp_stand_in() -> types.ModuleType:
    wp = types.ModuleType("warp")
    ident = lambda f=None, **kw: f if f is not None else (lambda g: g)  # noqa: E731
    wp.func = wp.kernel = wp.struct = ident
    wp.constant = lambda x: x
    wp.pi = math.pi
    wp.clamp = lambda x, lo, hi: min(max(x, lo), hi)
    wp.abs = abs
    wp.min = min
    wp.max = max
    wp.vec2 = lambda *a: np.array(a, dtype=np.float64)
    wp.vec3 = lambda *a: np.array(a, dtype=np.float64)
    wp.length = lambda v: float(np.linalg.norm(v))
    wp.dot = lambda a, b: float(np.dot(a, b))
    wp.int64 = int
    wp.float64 = float
    wp.round = round
    return wp


def load_module(path: Path, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def extract(path: Path, names: list[str], namespace: dict) -> dict:
    """Exec the named top-level functions of ``path`` (decorators dropped) in ``namespace``."""
    tree = ast.parse(path.read_text())
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in names]
    for n in keep:
        n.decorator_list = []
    mod = ast.Module(body=keep, type_ignores=[])
    exec(compile(mod, str(path), "exec"), namespace)
    return {n: namespace[n] for n in names}


def main(root: Path) -> None:
    sys.modules["warp"] = warp_stand_in()
    sph = root / "alloy" / "solvers" / "sph"
    K = load_module(sph / "kernels.py", "ref_sph_kernels")
    ns = {"math": math, "np": np, "kernel_w_np": K.kernel_w_np, "lattice_sum": K.lattice_sum,
          "halfspace_volume": K.halfspace_volume, "wp": sys.modules["warp"], "BISECT": 30}

    class Cfg:
        def __init__(self, r, kind):
            self.particle_radius, self.support_factor, self.kernel = r, 4.0, kind

        h = property(lambda s: s.support_factor * s.particle_radius)
        spacing = property(lambda s: 2.0 * s.particle_radius)

    fns = extract(sph / "config.py", ["particle_mass", "full_neighbor_count"], ns)
    pw = extract(sph / "particle_walls.py", ["colour_distance", "pw_project"], ns)

    cases = []
    for r, kind in ((0.01, "cubic"), (0.005, "cubic"), (0.001, "cubic"), (0.002, "cubic"), (0.002, "wendland_c2")):
        cfg = Cfg(r, kind)
        s, h = cfg.spacing, cfg.h
        kid = K.KERNEL_IDS[kind]
        delta, amp = K.boundary_fit(s, h, kind)
        deficit, grad = K._half_lattice(s, h, kind)
        rs = np.linspace(0.0, 1.1 * h, 23)
        grads = [[0.3 * h, -0.2 * h, 0.1 * h], [0.6 * h, 0.1 * h, 0.0], [1e-12 * h, 0.0, 0.0], [0.0, 0.0, 0.95 * h]]
        ds = list(np.linspace(-1.2 * h, 1.2 * h, 25))
        cs = list(np.linspace(0.0002, 0.999, 21))
        cases.append({
            "particle_radius": r, "kind": kind, "spacing": s, "h": h,
            "lattice_sum": K.lattice_sum(s, h, kind), "particle_mass_rho1000": fns["particle_mass"](cfg, 1000.0),
            "full_neighbor_count": fns["full_neighbor_count"](cfg), "lattice_diagonal": K.lattice_diagonal(s, h, kind),
            "boundary_fit": [delta, amp], "half_lattice": [deficit, grad],
            "kernel_w": [[float(x), float(K.kernel_w(float(x), h, kid))] for x in rs],
            "kernel_grad": [[g, [float(c) for c in K.kernel_grad(np.array(g), h, kid)]] for g in grads],
            "halfspace": [[float(d), [float(c) for c in K.halfspace_volume(float(d), h, 0.0, kid)]] for d in ds],
            "colour_distance": [[float(c), float(pw["colour_distance"](float(c), h, kid))] for c in cs],
        })
    # build.py's liquid volume fill (emit_object's points): the reference's liquid_points with stand-ins for the card
    # types it tests with isinstance (alloy/cards/types.py ParticleSource and Primitive)
    cards = types.ModuleType("alloy.cards.types")

    class ParticleSource:
        def __init__(self, region):
            self.region = region

    class Primitive:
        def __init__(self, kind, size):
            self.kind, self.size = kind, size

    cards.ParticleSource, cards.Primitive = ParticleSource, Primitive
    for name in ("alloy", "alloy.cards"):
        sys.modules.setdefault(name, types.ModuleType(name))
    sys.modules["alloy.cards.types"] = cards
    bns = {"np": np, "math": math}
    bfn = extract(sph / "build.py", ["lattice_points", "_inside_primitive", "disk_rings", "column_layers",
                                     "liquid_points"], {**bns, "DISK_CLEAR": 0.375})
    bns.update(bfn)
    for f in bfn.values():
        f.__globals__.update(bfn)
    shapes = [("region", ((0.0, 0.0, 0.0), (0.1, 0.06, 0.05)), 0.01), ("box", (0.011, 0.02, 0.013), 0.004),
              ("sphere", (0.02, 0.0, 0.0), 0.004), ("ellipsoid", (0.02, 0.012, 0.016), 0.004), ("cylinder", (0.02, 0.01, 0.0), 0.004),
              ("cylinder", (0.006, 0.01, 0.0), 0.002), ("capsule", (0.01, 0.015, 0.0), 0.004)]
    fills = []
    for kind, size, sp in shapes:
        shape = ParticleSource(size) if kind == "region" else Primitive(kind, size)
        pts = bfn["liquid_points"](shape, sp)
        fills.append({"kind": kind, "size": size, "spacing": sp, "points": np.asarray(pts, np.float64).tolist()})
    (OUT.parent / "reference_liquid_points.json").write_text(json.dumps(
        {"source": "alloy/solvers/sph/build.py liquid_points (float64 numpy, card types stood in)", "cases": fills}))

    shape_sdf_cases(root)
    OUT.write_text(json.dumps({"source": "alloy/solvers/sph kernels.py, config.py, particle_walls.py (float64 Python "
                                         "evaluation with a warp stand-in)", "cases": cases}, indent=1))
    print(f"wrote {OUT} ({len(cases)} cases)")


def shape_sdf_cases(root: Path) -> None:
    """tests/golden/reference_shape_sdf.json: the vendored Newton signed distances and gradients of the analytic shapes
    the liquid's walls use, as eval_shape_sdf (soft_contacts_sdf.py:249-280) calls them: sdf_box, sdf_sphere,
    sdf_capsule and sdf_cylinder (straight) along z and their _grad functions (geometry/kernels.py), and _eval_plane_sdf with depth 0 for planes
    (soft_contacts_sdf.py:73-102), evaluated in float64 at points inside, on and outside each shape."""
    from enum import IntEnum

    class Axis(IntEnum):
        X = 0
        Y = 1
        Z = 2

    wp = sys.modules["warp"]
    wp.vec3 = lambda *a: np.array(a if a else (0.0, 0.0, 0.0), dtype=np.float64)
    wp.normalize = lambda v: v / np.linalg.norm(v)
    wp.sign = lambda x: -1.0 if x < 0.0 else 1.0
    names = ["_sdf_point_to_z_up", "_sdf_vector_from_z_up", "sdf_sphere", "sdf_sphere_grad", "sdf_box", "sdf_box_grad",
             "sdf_capsule", "sdf_capsule_grad", "sdf_cylinder", "sdf_cylinder_grad"]
    geom = root / "alloy" / "_vendor" / "newton" / "_src" / "geometry"
    f = extract(geom / "kernels.py", names, {"wp": wp, "Axis": Axis, "np": np, "math": math})
    f.update(extract(geom / "soft_contacts_sdf.py", ["_eval_plane_sdf"], {"wp": wp, "np": np, "math": math}))
    for fn in f.values():
        fn.__globals__.update(f)
    rng = np.random.default_rng(7)
    shapes = [("box", 7, (0.03, 0.02, 0.05)), ("sphere", 3, (0.04, 0.0, 0.0)), ("capsule", 4, (0.02, 0.05, 0.0)),
              ("plane", 1, (0.0, 0.0, 0.0)), ("finite_plane", 1, (0.1, 0.06, 0.0)),
              ("cylinder", 6, (0.03, 0.04, 0.0))]
    out = []
    for name, geo, sc in shapes:
        pts = list(rng.uniform(-0.09, 0.09, size=(40, 3)))
        pts += [np.array([0.0, 0.0, 0.0]), np.array([0.0, 0.0, sc[1] + 0.01]), np.array([0.0, 0.0, -sc[1] - 0.01]),
                np.array([sc[0], 0.0, 0.0]), np.array([0.0, 0.0, 0.03])]
        rows = []
        for pnt in pts:
            if geo == 7:
                phi, g = f["sdf_box"](pnt, *sc), f["sdf_box_grad"](pnt, *sc)
            elif geo == 3:
                phi, g = f["sdf_sphere"](pnt, sc[0]), f["sdf_sphere_grad"](pnt, sc[0])
            elif geo == 6:
                phi = f["sdf_cylinder"](pnt, sc[0], sc[1], int(Axis.Z), -1.0, sc[2])
                g = f["sdf_cylinder_grad"](pnt, sc[0], sc[1], int(Axis.Z), -1.0, sc[2])
            elif geo == 4:
                phi = f["sdf_capsule"](pnt, sc[0], sc[1], int(Axis.Z))
                g = f["sdf_capsule_grad"](pnt, sc[0], sc[1], int(Axis.Z))
            else:
                _lo, phi, g = f["_eval_plane_sdf"](np.array(sc, np.float64), pnt, 0.0)
            rows.append([[float(c) for c in pnt], float(phi), [float(c) for c in g]])
        out.append({"shape": name, "geo": geo, "scale": list(sc), "samples": rows})
    (OUT.parent / "reference_shape_sdf.json").write_text(json.dumps(
        {"source": "alloy/_vendor/newton/_src/geometry/kernels.py sdf_* and sdf_*_grad (float64, warp stand-in)",
         "cases": out}, indent=1))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        raise SystemExit(__doc__)
    main(Path(sys.argv[1]))
