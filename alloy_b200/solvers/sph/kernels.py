# SPDX-License-Identifier: Apache-2.0
"""Host-side (float64, numpy) SPH kernel constants: lattice sums, the wall fit, the DFSPH diagonal.

These run once per solver on the host and feed the CUDA kernels as float32 constants. They restate the reference's
host helpers (alloy/solvers/sph/kernels.py:155-282, config.py:225-236):

- ``kernel_w_np``: cubic spline W = 8/(pi h^3) f(q), f = 6q^3 - 6q^2 + 1 (q <= 1/2), 2 (1-q)^3 (q < 1); Wendland C2
  W = 21/(2 pi h^3) (1-q)^4 (1 + 4q); support radius h (W = 0 for r >= h).
- ``lattice_sum``: sum of W over an infinite cubic lattice, self included; the particle mass rho0 / S makes an interior
  lattice particle have rho = rho0 exactly.
- ``halfspace_volume_np``: kernel volume Psi(d) inside a flat solid half-space at signed distance d (closed form in
  the projected kernel p(y) = int over a plane slice; see the oracle and CUDA sources for the polynomials).
- ``boundary_fit``: wall offset delta and amplitude A of Psi_eff(d) = A Psi(d + delta) such that a lattice resting
  at d = r has rho = rho0 (A Psi(r + delta) equals the half-lattice deficit) and the wall slope is twice the
  half-lattice gradient (the hydrostatic rest state is force free).
- ``lattice_diagonal``: sum_j V^2 |dW_ij/dr|^2 over the rest lattice (V = 1/S), the bulk DFSPH diagonal.
"""

from __future__ import annotations

import math

import numpy as np

KERNEL_IDS = {"cubic": 0, "wendland_c2": 1}


def kernel_sigma(h: float, kind: str = "cubic") -> float:
    """Normalisation of W [1/m^3]: W(0) for both kernels."""
    if kind == "wendland_c2":
        return 21.0 / (2.0 * math.pi * h**3)
    return 8.0 / (math.pi * h**3)


def kernel_w_np(r: np.ndarray, h: float, kind: str = "cubic") -> np.ndarray:
    q = np.asarray(r, dtype=np.float64) / h
    s = np.clip(1.0 - q, 0.0, None)
    if kind == "wendland_c2":
        return kernel_sigma(h, kind) * np.where(q < 1.0, s**4 * (1.0 + 4.0 * q), 0.0)
    inner = 1.0 + 6.0 * q * q * (q - 1.0)
    outer = 2.0 * s**3
    return kernel_sigma(h, kind) * np.where(q <= 0.5, inner, np.where(q < 1.0, outer, 0.0))


def _offsets(spacing: float, h: float) -> np.ndarray:
    n = int(math.ceil(h / spacing)) + 1
    ax = np.arange(-n, n + 1, dtype=np.float64) * spacing
    return np.stack(np.meshgrid(ax, ax, ax, indexing="ij"), -1).reshape(-1, 3)


def lattice_sum(spacing: float, h: float, kind: str = "cubic") -> float:
    g = _offsets(spacing, h)
    return float(kernel_w_np(np.linalg.norm(g, axis=1), h, kind).sum())


def particle_mass(spacing: float, h: float, rest_density: float, kind: str = "cubic") -> float:
    """m = rho0 / S [kg] (config.py:225-227)."""
    return float(rest_density / lattice_sum(spacing, h, kind))


def full_neighbor_count(spacing: float, h: float, kind: str = "cubic") -> float:
    """Neighbours of an interior lattice particle with W > 0, self excluded (config.py:230-236)."""
    g = _offsets(spacing, h)
    return float(np.count_nonzero(kernel_w_np(np.linalg.norm(g, axis=1), h, kind) > 0.0) - 1)


def _dw_dr(r: np.ndarray, h: float, kind: str) -> np.ndarray:
    """dW/dr by central differences at 1e-7 h (the same discrete derivative the reference's fit uses)."""
    e = 1.0e-7 * h
    return (kernel_w_np(r + e, h, kind) - kernel_w_np(r - e, h, kind)) / (2.0 * e)


def lattice_diagonal(spacing: float, h: float, kind: str = "cubic") -> float:
    g = _offsets(spacing, h)
    r = np.linalg.norm(g, axis=1)
    m = (r > 0.0) & (r < h)
    vol = 1.0 / lattice_sum(spacing, h, kind)
    return float(np.sum((vol * _dw_dr(r[m], h, kind)) ** 2))


def _g0(y: float, kind: str) -> float:
    """G0(y) = int_0^y p(t) dt, y in [0, 1]."""
    if kind == "wendland_c2":
        c = [0.0, 1.5, 0.0, -3.5, 0.0, 10.5, -14.0, 7.5, -1.5]
        return float(np.polynomial.polynomial.polyval(y, c))
    if y <= 0.5:
        return 1.4 * y - (8.0 / 3.0) * y**3 + 4.8 * y**5 - 3.2 * y**6
    u = 1.0 - y
    return 0.5 - u**5 * (1.6 - (16.0 / 15.0) * u)


def halfspace_volume_np(d: float, h: float, kind: str = "cubic") -> float:
    """Psi(d) of a flat solid half-space at signed distance d (d > 0 outside the solid)."""
    if d >= h:
        return 0.0
    z = min(max(-d / h, -1.0), 1.0)
    return 0.5 + math.copysign(_g0(abs(z), kind), z)


def _half_lattice(spacing: float, h: float, kind: str) -> tuple[float, float]:
    """(1 - F1, |dF1/dz|): density deficit and its z-gradient of a particle in the first lattice layer next to a
    flat wall, the interior lattice normalised to ratio 1."""
    g = _offsets(spacing, h)
    r = np.linalg.norm(g, axis=1)
    w = kernel_w_np(r, h, kind)
    s = float(w.sum())
    up = (g[:, 2] >= 0.0) & (r > 0.0)
    grad_z = float(np.sum(_dw_dr(r[up], h, kind) * (-g[up, 2]) / r[up])) / s
    f1 = float(w[g[:, 2] >= 0.0].sum()) / s
    return 1.0 - f1, abs(grad_z)


def boundary_fit(spacing: float, h: float, kind: str = "cubic", slope_factor: float = 2.0) -> tuple[float, float]:
    """(delta [m], A) of the wall volume Psi_eff(d) = A Psi(d + delta) (kernels.py:221-249)."""
    deficit, grad = _half_lattice(spacing, h, kind)
    target = deficit / (slope_factor * grad)

    def ratio(d: float) -> float:
        e = 1.0e-7 * h
        dpsi = (halfspace_volume_np(d + e, h, kind) - halfspace_volume_np(d - e, h, kind)) / (2.0 * e)
        return halfspace_volume_np(d, h, kind) / max(abs(dpsi), 1.0e-30)

    lo, hi = 0.0, 0.999 * h
    for _ in range(100):
        mid = 0.5 * (lo + hi)
        if ratio(mid) > target:
            lo = mid
        else:
            hi = mid
    d = 0.5 * (lo + hi)
    return d - 0.5 * spacing, deficit / halfspace_volume_np(d, h, kind)
