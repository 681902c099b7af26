# SPDX-License-Identifier: Apache-2.0
"""The oracle's scalar SPH math and the host constants against the reference's known answers.

Ports tests/solvers/sph/test_kernels.py:23-109 (normalisation, gradient, half-space closed form, wall fit) and
tests/integration/test_sph_mpm_walls.py:72-81 (colour inversion), and compares with tests/golden/reference_kernels.json
(the reference's own kernels.py / config.py / particle_walls.py evaluated in float64, see make_golden.py)."""

from __future__ import annotations

import json
from pathlib import Path

import numpy as np
import pytest

from alloy_b200.solvers.sph import kernels as K
from oracle import pyoracle as O

GOLD = json.loads((Path(__file__).parent / "golden" / "reference_kernels.json").read_text())["cases"]
KINDS = [("cubic", 0), ("wendland_c2", 1)]


@pytest.mark.parametrize("case", GOLD, ids=lambda c: f"{c['kind']}-r{c['particle_radius']}")
def test_host_constants_equal_the_reference_bit_for_bit(case):
    s, h, kind = case["spacing"], case["h"], case["kind"]
    assert K.lattice_sum(s, h, kind) == case["lattice_sum"]
    assert K.particle_mass(s, h, 1000.0, kind) == case["particle_mass_rho1000"]
    assert K.full_neighbor_count(s, h, kind) == case["full_neighbor_count"]
    assert K.lattice_diagonal(s, h, kind) == case["lattice_diagonal"]
    assert list(K.boundary_fit(s, h, kind)) == case["boundary_fit"]


@pytest.mark.parametrize("case", GOLD, ids=lambda c: f"{c['kind']}-r{c['particle_radius']}")
def test_oracle_kernel_matches_the_reference_values(case):
    h, kid = case["h"], K.KERNEL_IDS[case["kind"]]
    sigma = K.kernel_sigma(h, case["kind"])
    r = np.array([p[0] for p in case["kernel_w"]])
    want = np.array([p[1] for p in case["kernel_w"]])
    W64, _ = O.kernel_wf(r * r, h, sigma, kid, f64=True)
    np.testing.assert_allclose(W64, want, rtol=1e-12, atol=1e-12 * sigma)
    W32, _ = O.kernel_wf((r * r).astype(np.float32), h, sigma, kid)
    np.testing.assert_allclose(W32, want, rtol=2e-6, atol=2e-6 * sigma)
    for rv, g in case["kernel_grad"]:
        rv = np.array(rv)
        _, F = O.kernel_wf(np.array([rv @ rv]), h, sigma, kid, f64=True)
        np.testing.assert_allclose(rv * F[0], g, rtol=1e-9, atol=1e-9 * sigma / h)


@pytest.mark.parametrize("case", GOLD, ids=lambda c: f"{c['kind']}-r{c['particle_radius']}")
def test_oracle_halfspace_and_colour_match_the_reference(case):
    h, kid = case["h"], K.KERNEL_IDS[case["kind"]]
    d = np.array([p[0] for p in case["halfspace"]])
    want = np.array([p[1] for p in case["halfspace"]])
    psi, dpsi = O.halfspace(d, h, kid, f64=True)
    np.testing.assert_allclose(psi, want[:, 0], atol=1e-12)
    np.testing.assert_allclose(dpsi, want[:, 1], rtol=1e-10, atol=1e-10 / h)
    c = np.array([p[0] for p in case["colour_distance"]], np.float32)
    want_d = np.array([p[1] for p in case["colour_distance"]])
    np.testing.assert_allclose(O.colour_distance(c, h, kid), want_d, atol=2e-6 * h / 0.008)


@pytest.mark.parametrize("name,kind", KINDS)
def test_kernel_normalised(name, kind):
    h, dx = 1.0, 0.02
    ax = np.arange(-1.0, 1.0 + dx / 2, dx)
    g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    r2 = np.einsum("ij,ij->i", g, g)
    W, _ = O.kernel_wf(r2, h, K.kernel_sigma(h, name), kind, f64=True)
    assert abs(W.sum() * dx**3 - 1.0) < 2e-3


@pytest.mark.parametrize("name,kind", KINDS)
def test_kernel_gradient_matches_finite_difference(name, kind, rng):
    h = 1.0
    sigma = K.kernel_sigma(h, name)
    x = rng.uniform(-h, h, (300, 3)).astype(np.float32)
    _, F = O.kernel_wf(np.einsum("ij,ij->i", x, x), h, sigma, kind)
    g = x * F[:, None]
    e = 1.0e-4 * h
    fd = np.zeros_like(x, dtype=np.float64)
    for a in range(3):
        xp, xm = x.astype(np.float64).copy(), x.astype(np.float64).copy()
        xp[:, a] += e
        xm[:, a] -= e
        wp_, _ = O.kernel_wf(np.einsum("ij,ij->i", xp, xp), h, sigma, kind, f64=True)
        wm_, _ = O.kernel_wf(np.einsum("ij,ij->i", xm, xm), h, sigma, kind, f64=True)
        fd[:, a] = (wp_ - wm_) / (2 * e)
    err = np.linalg.norm(g - fd, axis=1)
    assert err.max() < 2e-3 * np.linalg.norm(g, axis=1).max()


def _halfspace_quadrature(d: float, h: float, name: str) -> float:
    dx = 0.01 * h
    ax = np.arange(-h + dx / 2, h, dx)
    g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    w = K.kernel_w_np(np.linalg.norm(g, axis=1), h, name)
    return float(w[g[:, 2] < -d].sum() * dx**3)


@pytest.mark.parametrize("name,kind", KINDS)
def test_halfspace_volume_closed_form(name, kind):
    h = 1.0
    ds = np.array([-1.5, -0.6, -0.25, 0.0, 0.25, 0.5, 0.8, 1.2], dtype=np.float32)
    psi, dpsi = O.halfspace(ds, h, kind)
    for d, p in zip(ds, psi):
        assert abs(p - _halfspace_quadrature(float(d), h, name)) < 1e-3, d
        assert abs(p - K.halfspace_volume_np(float(d), h, name)) < 1e-6
    assert psi[0] == pytest.approx(1.0, abs=1e-6) and psi[3] == pytest.approx(0.5, abs=1e-6) and psi[-1] == 0.0
    e = 1.0e-3 * h
    pp, _ = O.halfspace(ds.astype(np.float64) + e, h, kind, f64=True)
    pm, _ = O.halfspace(ds.astype(np.float64) - e, h, kind, f64=True)
    assert np.abs(dpsi - (pp - pm) / (2 * e)).max() < 2e-3 * np.abs(dpsi).max()


@pytest.mark.parametrize("name", ["cubic", "wendland_c2"])
def test_boundary_fit_matches_lattice_value(name):
    sp, h = 2.0e-3, 4.0e-3
    delta, amp = K.boundary_fit(sp, h, name)
    n = 3
    ax = np.arange(-n, n + 1) * sp
    g = np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)
    w = K.kernel_w_np(np.linalg.norm(g, axis=1), h, name)
    deficit = 1.0 - w[g[:, 2] >= 0].sum() / w.sum()
    assert amp * K.halfspace_volume_np(0.5 * sp + delta, h, name) == pytest.approx(deficit, rel=1e-6)
    assert K.lattice_sum(sp, h, name) == pytest.approx(w.sum(), rel=1e-12)


def test_the_colour_inverts_to_the_half_space_distance():
    H = 0.008
    d = np.linspace(-0.006, 0.006, 25)
    psi, _ = O.halfspace(d.astype(np.float32), H, 0)
    np.testing.assert_allclose(O.colour_distance(psi, H, 0), d, atol=2e-6)


def test_reducer_matches_numpy_and_is_batch_invariant(rng):
    start = np.array([0, 5, 5, 700, 1203, 1203 + 70_000])
    vals = rng.normal(size=start[-1]).astype(np.float32)
    out, mx = O.world_sum(start, vals)
    for w in range(len(start) - 1):
        v = vals[start[w]:start[w + 1]].astype(np.float64)
        assert np.isclose(out[w], v.sum(), rtol=1e-12, atol=1e-12)
        assert mx[w] == (max(float(v.max()), 0.0) if len(v) else 0.0)
    a = rng.normal(size=777).astype(np.float32)
    other = rng.normal(size=300).astype(np.float32)
    o1, _ = O.world_sum(np.array([0, 777]), a)
    o2, _ = O.world_sum(np.array([0, 300, 1077]), np.concatenate([other, a]))
    assert o1[0].tobytes() == o2[1].tobytes()
