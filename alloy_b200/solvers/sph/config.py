# SPDX-License-Identifier: Apache-2.0
"""``DFSPHConfig``: the reference's solver configuration (alloy/solvers/sph/config.py:46-199), same field names,
defaults and validation messages, plus the host constants the CUDA path derives from it.

Fields the CUDA path does not implement yet are accepted and validated like the reference; ``SolverDFSPH`` says
which of them it cannot honour (``unsupported``) when it is constructed.
"""

from __future__ import annotations

import numpy as np

import math
from dataclasses import dataclass
from typing import Literal

from . import kernels as K

Vec3 = tuple[float, float, float]

VISCOUS_ABOVE = 1.0e-2
PHASE_NONE = -1
PHASE_SPARE = 0
PHASE_LIQUID = 1
PHASE_RETIRED = -2
PHASE_HELD = -3
PROJECT_EPS = 1.0e-3  # wall projection skin in particle radii (solver.py:483)


@dataclass
class DFSPHConfig:
    particle_radius: float = 2.0e-3
    support_factor: float = 4.0
    kernel: Literal["cubic", "wendland_c2"] = "cubic"
    max_density_error: float = 1.0e-3
    rest_jitter_speed: float | None = 1.5e-3
    rest_jitter_flow_ratio: float = 0.5
    min_density_error: float = 1.0e-5
    max_divergence_error: float = 1.0e-3
    min_iterations: int = 2
    max_iterations: int = 50
    cfl: float = 0.2
    speed_margin: float = 0.25
    dt_min: float = 1.953125e-5
    dt_max: float = 1.25e-3
    viscosity: Literal["auto", "none", "xsph", "weiler2018"] = "auto"
    xsph_c: float = 0.01
    surface_tension: Literal["none", "akinci2013", "csf"] = "none"
    boundary: Literal["sdf_tube", "akinci_particles", "auto"] = "auto"
    boundary_curvature_order: int = 1
    neighbor_capacity: int = 64
    reneighbor_skin: float | None = None
    coupling: Literal["two_way", "one_way"] = "two_way"
    world_bounds: tuple[Vec3, Vec3] | None = None
    integrate_bodies: Literal["proxies", "dynamic", "none"] = "proxies"
    min_neighbors_divergence: float = 20.0
    divergence_solve: bool = True
    divergence_two_sided: bool = False
    jacobi_omega: float = 0.5
    max_error_factor: float = 10.0
    warm_start_density: float = 0.9
    warm_start_divergence: float = 0.5
    grid_dim: int = 128
    viscosity_tolerance: float = 1.0e-3
    boundary_viscosity: float | None = None
    viscosity_max_iterations: int = 100
    diagonal_floor: float = 0.25
    contact_separation_speed: float = 0.5
    compression_relief_speed: float | None = 0.5
    wall_friction: bool = True
    ambient_pressure: float | None = None
    pressure_solver: Literal["cg", "jacobi"] = "cg"

    @property
    def h(self) -> float:
        return self.support_factor * self.particle_radius

    @property
    def spacing(self) -> float:
        return 2.0 * self.particle_radius

    @property
    def kernel_id(self) -> int:
        return K.KERNEL_IDS[self.kernel]

    @classmethod
    def fast(cls, **overrides) -> DFSPHConfig:
        """``rest_jitter_speed=None`` and ``cfl=0.4`` plus ``overrides`` (config.py:146-157)."""
        return cls(**{"rest_jitter_speed": None, "cfl": 0.4, **overrides})

    def validate(self) -> None:
        checks = [
            (self.particle_radius > 0.0, "particle_radius must be > 0"),
            (self.support_factor >= 2.0, "support_factor must be >= 2 (h >= spacing)"),
            (self.kernel in K.KERNEL_IDS, f"unknown kernel {self.kernel!r}"),
            (0 < self.min_iterations <= self.max_iterations, "need 0 < min_iterations <= max_iterations"),
            (self.max_density_error > 0.0 and self.max_divergence_error > 0.0, "error tolerances must be > 0"),
            (self.rest_jitter_speed is None or self.rest_jitter_speed > 0.0, "rest_jitter_speed must be > 0 or None"),
            (self.compression_relief_speed is None or self.compression_relief_speed > 0.0,
             "compression_relief_speed must be > 0 or None"),
            (self.ambient_pressure is None or self.ambient_pressure > 0.0, "ambient_pressure must be > 0 or None"),
            (0.0 <= self.rest_jitter_flow_ratio <= 1.0, "rest_jitter_flow_ratio must be in [0, 1]"),
            (0.0 < self.min_density_error <= self.max_density_error,
             "need 0 < min_density_error <= max_density_error"),
            (0.0 < self.cfl <= 1.0, "cfl must be in (0, 1]"),
            (0.0 < self.speed_margin <= 1.0, "speed_margin must be in (0, 1]"),
            (0.0 < self.dt_min <= self.dt_max, "need 0 < dt_min <= dt_max"),
            (self.viscosity in ("auto", "none", "xsph", "weiler2018"), f"unknown viscosity {self.viscosity!r}"),
            (self.surface_tension in ("none", "akinci2013", "csf"),
             f"unknown surface_tension {self.surface_tension!r}"),
            (self.boundary in ("sdf_tube", "akinci_particles", "auto"), f"unknown boundary {self.boundary!r}"),
            (self.boundary_curvature_order in (0, 1), "boundary_curvature_order must be 0 or 1"),
            (self.coupling in ("two_way", "one_way"), f"unknown coupling {self.coupling!r}"),
            (self.integrate_bodies in ("proxies", "dynamic", "none"), "unknown integrate_bodies"),
            (0.0 <= self.warm_start_density <= 1.0 and 0.0 <= self.warm_start_divergence <= 1.0,
             "warm start factors must be in [0, 1]"),
            (0.0 < self.jacobi_omega <= 0.6, "jacobi_omega must be in (0, 0.6] (0.8 and 1.0 diverge, measured)"),
            (self.max_error_factor >= 1.0, "max_error_factor must be >= 1"),
            (self.reneighbor_skin is None or 0.0 <= self.reneighbor_skin <= 1.0, "reneighbor_skin must be in [0, 1]"),
            (0.0 <= self.diagonal_floor < 1.0, "diagonal_floor must be in [0, 1)"),
            (self.contact_separation_speed >= 0.0, "contact_separation_speed must be >= 0"),
            (self.pressure_solver in ("jacobi", "cg"), f"unknown pressure_solver {self.pressure_solver!r}"),
            (self.viscosity_tolerance > 0.0 and self.viscosity_max_iterations > 0,
             "viscosity solve limits must be > 0"),
            (self.boundary_viscosity is None or self.boundary_viscosity >= 0.0, "boundary_viscosity must be >= 0"),
            (not self.boundary_viscosity or self.viscosity in ("auto", "weiler2018"),
             "boundary_viscosity needs viscosity 'weiler2018' (or 'auto' resolving to it)"),
        ]
        for ok, msg in checks:
            if not ok:
                raise ValueError(f"SolverDFSPH.Config: {msg}")

    def unsupported(self, viscosity_max: float = 1.0e-3) -> list[str]:
        """Settings the B200 CUDA path does not implement (beside the reference's own fallbacks)."""
        out = []
        visc = resolve_viscosity(self, viscosity_max)
        if visc == "weiler2018":
            out.append("viscosity weiler2018 (implicit viscosity)")
        if self.surface_tension != "none":
            out.append(f"surface_tension {self.surface_tension!r}")
        if self.ambient_pressure is not None:
            out.append("ambient_pressure")
        if self.kernel != "cubic" and self.kernel != "wendland_c2":
            out.append(f"kernel {self.kernel!r}")
        return out


SKIN_FILL_MARGIN = 1.75  # superset row capacity / rest fill within h + s (neighbors_skin.py:152)


def skin_capacity(h: float, spacing: float, skin: float) -> int:
    """Superset row capacity of the Verlet skin (neighbors_skin.py:155-166): 1.75 x the neighbours of an interior
    lattice particle within h + skin, at least 16. A fuller row is built plain for its step and its world rebuilds
    the next step, so a small capacity costs reuse, never exactness."""
    rad = (h + skin) / spacing
    m = int(math.ceil(rad)) + 1
    ax = np.arange(-m, m + 1, dtype=np.float64)
    d2 = ax[:, None, None] ** 2 + ax[None, :, None] ** 2 + ax[None, None, :] ** 2
    fill = int(np.count_nonzero(d2 < rad * rad)) - 1
    return max(16, int(math.ceil(SKIN_FILL_MARGIN * fill)))


def resolve_viscosity(cfg: DFSPHConfig, mu_max: float) -> str:
    if cfg.viscosity != "auto":
        return cfg.viscosity
    return "weiler2018" if mu_max > VISCOUS_ABOVE else "xsph"


def stable_dt(cfg: DFSPHConfig, v_max: float) -> float:
    """clamp(cfl 2r / |v|max, dt_min, dt_max) (config.py:209-213)."""
    if v_max <= 0.0 or not math.isfinite(v_max):
        return cfg.dt_max if v_max <= 0.0 else cfg.dt_min
    return float(min(max(cfg.cfl * cfg.spacing / v_max, cfg.dt_min), cfg.dt_max))


def snap_down(dt: float, control_dt: float, j_max: int = 10) -> float:
    """Largest control_dt / 2^j <= dt with j <= j_max (config.py:216-222)."""
    for j in range(j_max + 1):
        g = control_dt / float(2**j)
        if g <= dt:
            return g
    return control_dt / float(2**j_max)


def particle_mass(cfg: DFSPHConfig, rest_density: float) -> float:
    return K.particle_mass(cfg.spacing, cfg.h, rest_density, cfg.kernel)


@dataclass(frozen=True)
class HostConstants:
    """Float64 host constants of one configuration (the kernels take them as float32)."""

    h: float
    sigma: float
    n_full: float
    tot_min: float
    lattice_grad: float
    wall_offset: float
    wall_amplitude: float
    taper0: float
    taper1: float
    reach: float
    project_eps: float


def host_constants(cfg: DFSPHConfig) -> HostConstants:
    s, h, kind = cfg.spacing, cfg.h, cfg.kernel
    delta, amp = K.boundary_fit(s, h, kind)
    diag = K.lattice_diagonal(s, h, kind)
    # slots are kept for phi < reach: 1.5 spacings, or h with a wall viscosity (layout.py:195-198)
    reach = float(h) if cfg.boundary_viscosity else 1.5 * s
    return HostConstants(
        h=h, sigma=K.kernel_sigma(h, kind), n_full=K.full_neighbor_count(s, h, kind),
        tot_min=cfg.diagonal_floor * diag, lattice_grad=math.sqrt(diag), wall_offset=delta, wall_amplitude=amp,
        taper0=0.5 * s, taper1=1.5 * s, reach=reach, project_eps=PROJECT_EPS * cfg.particle_radius,
    )


def uniform_layout(mass: np.ndarray, rest_density: np.ndarray, rel: float = 1.0e-6) -> bool:
    """One particle mass and one rest density among the SPH particles (layout.py:97-100): the DFSPH operator is then
    symmetric, which the projected CG pressure solve needs; otherwise the reference falls back to Jacobi."""
    if len(mass) == 0:
        return True

    def spread(a):
        a = np.asarray(a, np.float64)
        return float(np.ptp(a)) / max(float(np.max(np.abs(a))), 1.0e-30)

    return spread(mass) <= rel and spread(rest_density) <= rel
