# SPDX-License-Identifier: Apache-2.0
"""The liquid's static shape walls beyond boxes, on CPU: the shape table (layout.py:131-249) takes static boxes,
spheres, capsules, straight cylinders and planes in any frame, refuses the rest by name, and keeps newton's bounding
radii and the thinnest wall; the oracle's signed distances and gradients of those shapes equal the vendored Newton
functions eval_shape_sdf calls (geometry/kernels.py sdf_box, sdf_sphere, sdf_capsule, sdf_cylinder and gradients;
soft_contacts_sdf.py _eval_plane_sdf for planes, a finite one a two-sided sheet), evaluated from the reference's
source into tests/golden/reference_shape_sdf.json by make_golden.py: in float64 within 5e-8 (the shape table's scales
are float32, as the model's are) and in float32 within 2e-6."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from alloy_b200.solvers.sph.build import add_fluid_block
from alloy_b200.solvers.sph.model import GeoType, ModelBuilder
from alloy_b200.solvers.sph.shapes import shape_table
from alloy_b200.solvers.sph.testing import benchmark_config
from oracle.pyoracle import Oracle

GOLDEN = json.loads((Path(__file__).parent / "golden" / "reference_shape_sdf.json").read_text())


def _model(add):
    cfg = benchmark_config(0.02)
    b = ModelBuilder(gravity=(0.0, 0.0, -9.81))
    b.begin_world()
    add_fluid_block(b, cfg, (0.0, 0.0, 0.1), (3, 3, 3))
    add(b)
    b.end_world()
    return b.finalize(), cfg


def test_shape_table_takes_the_analytic_static_shapes():
    def add(b):
        b.add_shape_box(-1, (0.0, 0.0, 0.0), 0.3, 0.2, 0.05)
        b.add_shape_sphere(-1, (0.1, 0.0, 0.2, 0.0, 0.0, 0.38268343, 0.9238795), radius=0.04)  # rotation is moot
        b.add_shape_capsule(-1, (0.0, 0.1, 0.2), radius=0.02, half_height=0.05)
        b.add_shape_plane(-1, (0.0, 0.0, -0.1), width=0.5, length=0.4)
        b.add_ground_plane(-0.2)
        b.add_shape_box(-1, (0.0, 0.0, 0.0, 0.0, 0.0, 0.38268343, 0.9238795), 0.1, 0.1, 0.1)  # rotated 45 deg
        b.add_shape_cylinder(-1, (0.0, 0.0, 0.0, 0.70710677, 0.0, 0.0, 0.70710677), radius=0.03, half_height=0.1)

    m, _ = _model(add)
    t = shape_table(m)
    assert t.count == 7 and list(t.ids) == [0, 1, 2, 3, 5, 6, 4]  # the world's own shapes, then the global ground
    np.testing.assert_allclose(t.radius[:3], [np.linalg.norm([0.3, 0.2, 0.05]), 0.04, 0.07], rtol=1e-6)
    assert t.thinnest == pytest.approx(0.04)  # the capsule's diameter; planes count as thick (layout.py:131-149)


@pytest.mark.parametrize("add, words", [
    (lambda b: b._add_shape(GeoType.CONE, (0.1, 0.1, 0.0), -1, None, 1.0, True, 0), "cone"),
    (lambda b: b._add_shape(GeoType.CYLINDER, (0.1, 0.1, 0.2), -1, None, 1.0, True, 0), "barrel cylinder"),
    (lambda b: b.add_shape_sphere(3, (0.0, 0.0, 0.0), radius=0.1), "sphere on body 3"),
    (lambda b: b.add_shape_box(-1, (0.0, 0.0, 0.0, 0.0, 0.0, 0.5, 0.5), 0.1, 0.1, 0.1), "not a unit quaternion"),
])
def test_shape_table_refuses_by_name(add, words):
    m, _ = _model(add)
    with pytest.raises(ValueError, match=words):
        shape_table(m)


@pytest.mark.parametrize("f64", [True, False])
def test_oracle_shape_sdf_equals_newton(f64):
    cases = GOLDEN["cases"]

    def add(b):
        for c in cases:
            b._add_shape(c["geo"], c["scale"], -1, (0.0, 0.0, 0.0), 1.0, True, 0)

    m, cfg = _model(add)
    o = Oracle(m.host(), cfg, f64=f64)
    tol = 5e-8 if f64 else 2e-6  # the shape table holds float32 scales (as the model's shape_scale does)
    for sh, c in enumerate(cases):
        for p, phi, grad in c["samples"]:
            ophi, ograd = o.shape_sdf(sh, p)
            assert ophi == pytest.approx(phi, abs=tol), (c["shape"], p)
            np.testing.assert_allclose(ograd, grad, atol=tol, err_msg=f"{c['shape']} {p}")
