# SPDX-License-Identifier: Apache-2.0
"""SPH report type: the reference's ``SPHReport`` (alloy/solvers/sph/types.py:11-28), same fields."""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True, eq=False)
class SPHReport:
    density_err: np.ndarray
    divergence_err: np.ndarray
    iters_density: np.ndarray
    iters_divergence: np.ndarray
    mass_active: np.ndarray
    mass_in: np.ndarray
    mass_out: np.ndarray
    escaped: np.ndarray
    neighbor_overflow: np.ndarray
    max_speed: np.ndarray
    unconverged: np.ndarray | None = None
    tension: str = "none"
    tension_qualitative: bool = False
    tension_rh_range: tuple[float, float] | None = None
    capillary_dt_violations: int = 0
    density_tol: np.ndarray | None = None
