# SPDX-License-Identifier: Apache-2.0
"""Host logic of the drop-in without a GPU: the plug-in's ``emit`` (scene assembly's liquid fill) against the
reference's own ``build.liquid_points`` (golden points made by tests/golden/make_golden.py from
alloy/solvers/sph/build.py:181-285), its budget and radius checks, and the port's host bookkeeping."""

from __future__ import annotations

import json
from pathlib import Path
from types import SimpleNamespace as N

import numpy as np
import pytest

from alloy_b200 import _lib
from alloy_b200.solvers.sph.build import emit_object, liquid_points
from alloy_b200.solvers.sph.model import ModelBuilder

GOLDEN = Path(__file__).resolve().parent / "golden" / "reference_liquid_points.json"


def _shape(case):
    return N(region=case["size"]) if case["kind"] == "region" else N(kind=case["kind"], size=tuple(case["size"]))


@pytest.mark.parametrize("k", range(7))
def test_liquid_points_equal_reference(k):
    case = json.loads(GOLDEN.read_text())["cases"][k]
    np.testing.assert_array_equal(liquid_points(_shape(case), case["spacing"]), np.asarray(case["points"]))


def _obj(shape, budget=10**6, fluid=None, density=1000.0):
    return N(card=N(name="water", shape=shape, budget=N(particles=budget)),
             material=N(density=N(value=density), fluid=fluid))


def test_emit_object_adds_liquid_in_the_current_world():
    b = ModelBuilder()
    b.begin_world()
    fluid = N(viscosity=N(value=2.0e-3))
    rg = emit_object(b, _obj(N(kind="sphere", size=(0.02, 0.0, 0.0)), fluid=fluid, density=998.0),
                     N(numbers={"particle_radius": 0.002}))
    b.end_world()
    m = b.finalize("cpu")
    assert len(rg) == 552 == m.particle_count
    assert np.all(m.sph.phase.numpy() == 1) and np.all(m.particle_flags.numpy() == 1)
    np.testing.assert_array_equal(m.sph.viscosity.numpy(), np.float32(2.0e-3))
    np.testing.assert_array_equal(m.sph.rest_density.numpy(), np.float32(998.0))


def test_emit_object_checks_budget_and_radius():
    b = ModelBuilder()
    b.begin_world()
    with pytest.raises(_lib.CapacityError):
        emit_object(b, _obj(N(kind="box", size=(0.02, 0.02, 0.02)), budget=10), N(numbers={"particle_radius": 0.002}))
    with pytest.raises(ValueError):
        emit_object(b, _obj(N(kind="box", size=(0.02, 0.02, 0.02))), N(numbers={}))
    with pytest.raises(ValueError):
        emit_object(b, _obj(N(kind="plane", size=(1.0, 1.0, 0.0))), N(numbers={"particle_radius": 0.002}))
