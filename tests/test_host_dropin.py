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


def test_skin_capacity_is_the_padded_rest_fill():
    """neighbors_skin.py:155-166: 1.75 x the lattice neighbours within h + s, at least 16 (counted here by brute
    force over the lattice)."""
    import itertools
    import math

    from alloy_b200.solvers.sph.config import skin_capacity

    for h, sp, s in ((0.004, 0.002, 0.0004), (0.04, 0.02, 0.004), (0.01, 0.005, 0.005), (0.002, 0.002, 0.0)):
        rad = (h + s) / sp
        m = int(math.ceil(rad)) + 1
        fill = sum(1 for x, y, z in itertools.product(range(-m, m + 1), repeat=3)
                   if x * x + y * y + z * z < rad * rad) - 1
        assert skin_capacity(h, sp, s) == max(16, math.ceil(1.75 * fill))


def test_skin_refuses_particle_walls():
    """neighbors.py:248-253: particle walls need the grid every step, so the skin is refused with them."""
    from alloy_b200.solvers.sph import SolverDFSPH
    from alloy_b200.solvers.sph.testing import dam_break

    sc = dam_break(counts=(4, 4, 4), box=(0.1, 0.1, 0.1), reneighbor_skin=0.1)
    with pytest.raises(ValueError, match="reneighbor_skin off"):
        SolverDFSPH(sc.model, sc.config)
