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
    """W(r) in float64. The polynomial forms and their evaluation order are the reference's (kernels.py:155-170):
    the wall fit below differentiates W numerically, which would amplify any other rounding into the constants."""
    q = np.asarray(r, dtype=np.float64) / h
    out = np.zeros_like(q)
    h3 = h**3
    if kind == "wendland_c2":
        m = q < 1.0
        s = 1.0 - q[m]
        out[m] = 21.0 / (2.0 * math.pi * h3) * s**4 * (1.0 + 4.0 * q[m])
        return out
    k = 8.0 / (math.pi * h3)
    inner = q <= 0.5
    outer = (q > 0.5) & (q < 1.0)
    out[inner] = k * (6.0 * q[inner] ** 3 - 6.0 * q[inner] ** 2 + 1.0)
    out[outer] = k * 2.0 * (1.0 - q[outer]) ** 3
    return out


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


# G0(y) = int_0^y p(t) dt as power series in y (the integral of the projected kernel p, one piece per branch of W);
# the same coefficient tables as the reference's kernels.py:182-186, evaluated with polyval as there.
_G0 = {
    "cubic": ((0.5, [0.0, 1.4, 0.0, -8.0 / 3.0, 0.0, 4.8, -3.2]),
              (1.0, [-1.0 / 30.0, 1.6, 0.0, -16.0 / 3.0, 8.0, -4.8, 16.0 / 15.0])),
    "wendland_c2": ((1.0, [0.0, 1.5, 0.0, -3.5, 0.0, 10.5, -14.0, 7.5, -1.5]),),
}


def _g0(y: float, kind: str) -> float:
    for top, coeffs in _G0[kind]:
        if y <= top:
            return float(np.polynomial.polynomial.polyval(y, coeffs))
    return 0.5


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
