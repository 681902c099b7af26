# SPDX-License-Identifier: Apache-2.0
"""``SolverDFSPH``: the reference's DFSPH liquid solver interface (alloy/solvers/sph/solver.py:57-479) over the
B200 CUDA library (include/alloy_dfsph.h, liballoy_dfsph.so).

The class keeps the reference's constructor, ``step(state_in, state_out, control, contacts, dt)`` contract (dt > 0,
early return for an empty model, state_out may alias state_in, nothing allocated per step), its report, ledger,
reset, emitter and protocol methods and the ``alloy_state_arrays`` keys. Everything the step computes runs in the
library's sm_100a kernels; this module holds host logic only (validation, constants, emitter tables) and has no CPU
fallback: without a CUDA device or the library it raises.

Scope of the CUDA path: cubic or Wendland kernel, projected preconditioned CG (the reference's default, krylov.py)
or relaxed Jacobi pressure solves, XSPH, particle walls (boundary particles flagged PROXY), static shape walls
(boxes, spheres, capsules, straight cylinders and planes, each in its own frame) evaluated through their SDF (up to four wall slots
per particle, projection and the sweep past fast steps, wall friction), emitters, sinks and the escape box.
Settings outside it are refused in the constructor (``DFSPHConfig.unsupported``); CG falls back to Jacobi with a
warning when particle masses or rest densities differ, as the reference does (solver.py:89-91). The resting-jitter
rule sets each world's density tolerance per step (solve_driver.py:1-118).
"""

from __future__ import annotations

import ctypes as C
import logging
from typing import ClassVar

import numpy as np
import torch

from ... import _lib
from .config import (PHASE_HELD, PHASE_SPARE, DFSPHConfig, host_constants, skin_capacity, snap_down, stable_dt,
                     uniform_layout)
from .model import ParticleFlags
from .types import SPHReport

log = logging.getLogger("alloy.sph")

FIX_SCALE = float(2**40)
_ACTIVE = int(ParticleFlags.ACTIVE)


class _DevView:
    """A raw device pointer seen as an array (``__cuda_array_interface__``) so torch can wrap library storage."""

    def __init__(self, ptr: int, shape: tuple, typestr: str):
        self.__cuda_array_interface__ = {"shape": shape, "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2, "strides": None}


def _ptr(a, dtype=None, shape0=None, what="array") -> int:
    """Device pointer of a contiguous CUDA array (torch tensor, or anything with __cuda_array_interface__)."""
    if a is None:
        return 0
    if isinstance(a, torch.Tensor):
        if not a.is_cuda:
            raise ValueError(f"SolverDFSPH: {what} must be on a CUDA device")
        if not a.is_contiguous():
            raise ValueError(f"SolverDFSPH: {what} must be contiguous")
        if dtype is not None and a.dtype != dtype:
            raise ValueError(f"SolverDFSPH: {what} must be {dtype}, got {a.dtype}")
        if shape0 is not None and a.shape[0] != shape0:
            raise ValueError(f"SolverDFSPH: {what} has {a.shape[0]} rows, expected {shape0}")
        return a.data_ptr()
    cai = getattr(a, "__cuda_array_interface__", None)
    if cai is None:
        raise TypeError(f"SolverDFSPH: {what} is not a CUDA array")
    return int(cai["data"][0])


def _host(a) -> np.ndarray:
    if isinstance(a, torch.Tensor):
        return a.detach().cpu().numpy()
    if hasattr(a, "numpy"):
        return a.numpy()
    return np.asarray(a)


def sph_phase(phase: np.ndarray) -> np.ndarray:
    """The SPH solver's particles at build: liquid, spares and held (config.py:36-38)."""
    return (phase >= PHASE_SPARE) | (phase == PHASE_HELD)


def layer_offsets(half_extents: np.ndarray, velocity_local: np.ndarray, spacing: float) -> np.ndarray:
    """Lattice points on the region's mid cross-section perpendicular to the velocity, whole spacings across each
    side with 1e-6 of a cell's slack (emitters.py:48-64)."""
    v = np.asarray(velocity_local, dtype=np.float64)
    axis = int(np.argmax(np.abs(v))) if float(np.linalg.norm(v)) > 0.0 else 2
    others = [a for a in range(3) if a != axis]
    grids = []
    for a in others:
        n = max(int(np.floor(2.0 * half_extents[a] / spacing + 1.0e-6)), 1)
        grids.append((np.arange(n) - 0.5 * (n - 1)) * spacing)
    ga, gb = np.meshgrid(grids[0], grids[1], indexing="ij")
    pts = np.zeros((ga.size, 3))
    pts[:, others[0]] = ga.ravel()
    pts[:, others[1]] = gb.ravel()
    return pts.astype(np.float32)


def quat_rotate_inv(q, v) -> np.ndarray:
    """v rotated by the inverse of unit quaternion q = (x, y, z, w)."""
    u = -np.asarray(q[:3], np.float64)
    w = float(q[3])
    v = np.asarray(v, np.float64)
    return v * (2.0 * w * w - 1.0) + 2.0 * w * np.cross(u, v) + 2.0 * u * np.dot(u, v)


def _xform7(region) -> np.ndarray:
    x = np.asarray(tuple(region), np.float32).reshape(-1)
    if x.size == 3:
        x = np.concatenate([x, np.array([0.0, 0.0, 0.0, 1.0], np.float32)])
    if x.size != 7:
        raise ValueError("region must be a transform (px, py, pz, qx, qy, qz, qw)")
    return x


def hydrostatic_guess(solver, state) -> np.ndarray:
    """k_i = |g| (z_top - z_i + r) per (world, horizontal 2r bin) column of active liquid, measured along gravity: the
    initial guess ``prime`` refines (prime.py:20-49; k = p / rho0 [m^2/s^2]). Host float64, float32 result."""
    n = solver.n
    out = np.zeros(max(n, 1), dtype=np.float32)
    m = solver.model
    q = _host(state.particle_q).astype(np.float64).reshape(-1, 3)
    act = (_host(m.sph.phase) >= 1) & ((_host(m.particle_flags) & _ACTIVE) != 0)
    world = _host(m.particle_world)
    grav = _host(m.gravity).astype(np.float64).reshape(-1, 3)
    sp = solver.config.spacing
    for w in np.unique(world[act]):
        g = grav[w]
        gn = float(np.linalg.norm(g))
        if gn == 0.0:
            continue
        up = -g / gn
        sel = np.nonzero(act & (world == w))[0]
        z = q[sel] @ up
        e1 = np.cross(up, [1.0, 0.0, 0.0] if abs(up[0]) < 0.9 else [0.0, 1.0, 0.0])
        e1 /= np.linalg.norm(e1)
        e2 = np.cross(up, e1)
        key = np.stack([np.floor(q[sel] @ e1 / sp), np.floor(q[sel] @ e2 / sp)], 1).astype(np.int64)
        _, inv = np.unique(key, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        top = np.full(inv.max() + 1, -np.inf)
        np.maximum.at(top, inv, z)
        out[sel] = (gn * np.maximum(top[inv] - z + 0.5 * sp, 0.0)).astype(np.float32)
    return out[:n]


class SolverDFSPH:
    """Divergence-free SPH (Bender & Koschier 2017) on B200: sorted-cell neighbour lists, particle walls,
    per-world float64 convergence (module doc)."""

    plugin_name: ClassVar[str] = "sph"
    routes: ClassVar[frozenset[str]] = frozenset({"liquid_sph"})
    determinism: ClassVar[str] = "native"  # bitwise repeatable, independent of batch composition (D9)
    alloy_clock_safety: ClassVar[float] = 1.0
    Config = DFSPHConfig

    @staticmethod
    def register_custom_attributes(builder) -> None:
        """solver.py:60-70; see plugin.register_custom_attributes."""
        from .plugin import register_custom_attributes

        register_custom_attributes(builder)

    def __init__(self, model, config: DFSPHConfig | None = None, *, capacity_per_world: int | None = None,
                 soft_particles=None, soft_half_thickness: float = 0.0, soft_inertia: bool = True,
                 skin_rows: int | None = None):
        self.model = model
        self.config = cfg = config or DFSPHConfig()
        cfg.validate()
        if soft_particles is not None:
            raise ValueError("SolverDFSPH: soft walls (VBD faces) are not part of the B200 CUDA path")
        self._lib = _lib.lib()
        n = int(model.particle_count)
        W = int(model.world_count)
        self.n, self.world_count = n, W
        ns = getattr(model, "sph", None)
        if ns is None or getattr(ns, "phase", None) is None or getattr(ns, "rest_density", None) is None:
            raise ValueError("SolverDFSPH needs the sph:* custom attributes; call SolverDFSPH.register_custom_attributes"
                             "(builder) before adding particles")
        phase = _host(ns.phase).astype(np.int8) if n else np.zeros(0, np.int8)
        world = _host(model.particle_world).astype(np.int32) if n else np.zeros(0, np.int32)
        sph = sph_phase(phase)
        if np.any(world[sph] < 0):
            raise ValueError("SPH particles must belong to a world (particle_world >= 0)")
        if n and np.any(np.diff(world[world >= 0]) < 0):
            raise ValueError("particles must be contiguous per world (Model.particle_world sorted)")
        ws = np.zeros(W + 1, np.int32)
        if n:
            ws[:] = _host(model.particle_world_start)[: W + 1]
        self.world_start = ws
        flags = _host(model.particle_flags).astype(np.int32) if n else np.zeros(0, np.int32)
        proxy = (flags & int(ParticleFlags.PROXY)) != 0
        if np.any(proxy & (world < 0)):
            raise ValueError(f"SolverDFSPH: {int(np.sum(proxy & (world < 0)))} particle-wall particles are in no "
                             "world (world -1); a wall needs the world of the liquid it bounds")
        mu = _host(getattr(ns, "viscosity", None)) if getattr(ns, "viscosity", None) is not None and n else np.zeros(0)
        mu_max = float(np.max(mu[sph])) if n and np.any(sph) and len(mu) else 0.0
        missing = cfg.unsupported(mu_max)
        if missing:
            raise ValueError("SolverDFSPH (B200 build): not implemented on the CUDA path: " + ", ".join(missing))
        self.pressure_solver = cfg.pressure_solver
        if self.pressure_solver == "cg" and n:
            m_all = _host(model.particle_mass)
            r_all = _host(ns.rest_density)
            if not uniform_layout(m_all[sph], r_all[sph]):  # solver.py:89-91
                log.warning("SolverDFSPH: pressure_solver 'cg' needs one particle mass and rest density; using "
                            "'jacobi'")
                self.pressure_solver = "jacobi"
        self._check_capacity(capacity_per_world, phase, ws)
        from .shapes import shape_table

        self.shapes = shape_table(model)  # refuses shape walls this path does not evaluate
        if cfg.reneighbor_skin and n and np.any((_host(model.particle_flags) & int(ParticleFlags.PROXY)) != 0):
            raise ValueError("SolverDFSPH: particle walls need the grid rebuilt every step (reneighbor_skin off)")
        if n and isinstance(model.particle_mass, torch.Tensor) and not model.particle_mass.is_cuda:
            raise ValueError("SolverDFSPH: the model must live on a CUDA device (Model.finalize(device='cuda'))")
        self.device = model.particle_mass.device if isinstance(model.particle_mass, torch.Tensor) else \
            torch.device("cuda", 0)
        self.hc = host_constants(cfg)
        self._params = self._make_params(cfg, self.hc)
        if cfg.reneighbor_skin:  # Verlet-skin reuse (solver.py:130-133)
            self._params.skin = float(cfg.reneighbor_skin) * self.hc.h
            self._params.skin_cap = skin_rows or skin_capacity(self.hc.h, cfg.spacing, self._params.skin)
        self._params.cg = int(self.pressure_solver == "cg")
        q_host = np.ascontiguousarray(_host(model.particle_q), np.float32).reshape(-1) if n else np.zeros(0, np.float32)
        md = _lib.ModelDesc()
        md.n, md.world_count = n, W
        md.world_start = ws.ctypes.data_as(C.POINTER(C.c_int32))
        md.q_host = q_host.ctypes.data_as(C.POINTER(C.c_float))
        md.mass = _ptr(model.particle_mass, torch.float32, n, "particle_mass")
        md.rest_density = _ptr(ns.rest_density, torch.float32, n, "sph.rest_density")
        md.radius = _ptr(model.particle_radius, torch.float32, n, "particle_radius")
        md.flags = _ptr(model.particle_flags, torch.int32, n, "particle_flags")
        md.phase = _ptr(ns.phase, torch.int8, n, "sph.phase")
        md.world = _ptr(model.particle_world, torch.int32, n, "particle_world")
        md.gravity = _ptr(model.gravity, torch.float32, None, "gravity")
        tab = self.shapes  # static box walls (layout.py:207-246), kept alive for the create call
        box = np.zeros((max(tab.count, 1), 8), np.float32)
        if tab.count:
            box[:, 0:3] = tab.xform[:, 0:3]
            box[:, 3] = tab.radius
            box[:, 4:7] = tab.scale
            box[:, 7] = tab.mu
        sh_start = np.ascontiguousarray(tab.start, np.int32)
        sh_ids = np.ascontiguousarray(tab.ids if len(tab.ids) else np.zeros(1, np.int32), np.int32)
        md.n_shapes = tab.count
        md.shape_start = sh_start.ctypes.data_as(C.POINTER(C.c_int32))
        md.shape_ids = sh_ids.ctypes.data_as(C.POINTER(C.c_int32))
        md.shape_box = box.ctypes.data_as(C.POINTER(C.c_float))
        geo = np.ascontiguousarray(tab.geo if tab.count else np.full(1, 7), np.int32)
        md.shape_geo = geo.ctypes.data_as(C.POINTER(C.c_int32))
        quat = np.ascontiguousarray(tab.xform[:, 3:7] if tab.count else np.array([[0.0, 0.0, 0.0, 1.0]]), np.float32)
        md.shape_quat = quat.ctypes.data_as(C.POINTER(C.c_float))
        md.sweep_len = min(0.5 * cfg.h, 0.5 * tab.thinnest)  # integrate.py:42-49
        handle = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.adf_create(C.byref(self._params), C.byref(md), self.device.index or 0,
                                            C.byref(handle)), "SolverDFSPH")
        self._h = handle
        kv, kd = C.c_void_p(), C.c_void_p()
        _lib.check(self._lib.adf_state_arrays(self._h, C.byref(kv), C.byref(kd)))
        self._kv = torch.as_tensor(_DevView(kv.value, (max(n, 1),), "<f4"), device=self.device)[:n]
        self._kd = torch.as_tensor(_DevView(kd.value, (max(n, 1),), "<f4"), device=self.device)[:n]
        self._flags0 = model.particle_flags.clone() if n else None
        self._phase0 = ns.phase.clone() if n else None
        # emitter host table (runtime.py:452-525)
        self._em_world: list[int] = []
        self._em_pool: list[np.ndarray] = []
        self._em_own: list[bool] = []
        self._patches: list[dict[int, np.ndarray]] = []  # per patch group: world -> reserved spare ids
        self._sinks = 0
        self.bounds = None if cfg.world_bounds is None else cfg.world_bounds
        from .ports import SPHPort

        self.port = SPHPort(self)  # absorb / emit / retire between steps (ports.py)
        self._saved: dict[str, torch.Tensor] = {}  # coupling restarts (coupling_notify_input_state_update)
        log.info("SolverDFSPH (B200): %d particles in %d worlds, r=%g m, h=%g m, kernel=%s", n, W,
                 cfg.particle_radius, cfg.h, cfg.kernel)

    # ------------------------------------------------------------------------------------------------- setup
    @staticmethod
    def _make_params(cfg: DFSPHConfig, hc) -> _lib.Params:
        p = _lib.Params()
        p.kind = cfg.kernel_id
        p.particle_radius = cfg.particle_radius
        p.h, p.sigma, p.n_full, p.tot_min, p.lattice_grad = hc.h, hc.sigma, hc.n_full, hc.tot_min, hc.lattice_grad
        p.wall_offset, p.wall_amplitude = hc.wall_offset, hc.wall_amplitude
        p.taper0, p.taper1, p.reach = hc.taper0, hc.taper1, hc.reach
        p.tol_den, p.tol_div = cfg.max_density_error, cfg.max_divergence_error
        p.max_error_factor = cfg.max_error_factor
        p.min_it, p.max_it = cfg.min_iterations, cfg.max_iterations
        p.omega, p.warm_den, p.warm_div = cfg.jacobi_omega, cfg.warm_start_density, cfg.warm_start_divergence
        p.min_nb = cfg.min_neighbors_divergence
        p.divergence_solve, p.two_sided = int(cfg.divergence_solve), int(cfg.divergence_two_sided)
        p.xsph_c = cfg.xsph_c if cfg.viscosity in ("xsph", "auto") else 0.0
        p.capacity = cfg.neighbor_capacity
        p.v_sep = cfg.contact_separation_speed
        p.relief_speed = cfg.compression_relief_speed or 0.0
        p.project_eps = hc.project_eps
        p.wall_friction = int(bool(cfg.wall_friction))
        p.jitter_speed = cfg.rest_jitter_speed or 0.0  # the resting-jitter rule (solve_driver.py:1-118)
        p.jitter_ratio = cfg.rest_jitter_flow_ratio
        p.tol_den_min = min(cfg.min_density_error, cfg.max_density_error)
        if cfg.world_bounds is not None:
            p.has_bounds = 1
            for a in range(3):
                p.bounds_lo[a], p.bounds_hi[a] = cfg.world_bounds[0][a], cfg.world_bounds[1][a]
        return p

    def _check_capacity(self, capacity_per_world, phase, ws) -> None:
        if capacity_per_world is None:
            return
        for w in range(self.world_count):
            have = int(np.count_nonzero(sph_phase(phase[ws[w]:ws[w + 1]])))
            if have < capacity_per_world:
                raise _lib.CapacityError(f"SolverDFSPH: world {w} has {have} SPH particle slots, "
                                         f"capacity_per_world={capacity_per_world}")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            try:
                self._lib.adf_destroy(h)
            finally:
                self._h = None

    def _stream(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    # ------------------------------------------------------------------------------------------------- step
    def step(self, state_in, state_out, control, contacts, dt: float, *, observables=None) -> None:
        del control, contacts, observables
        if not dt > 0.0:
            raise ValueError(f"SolverDFSPH.step: dt must be > 0, got {dt}")
        if self.n == 0:
            return
        n = self.n
        f = getattr(state_in, "particle_f", None)
        rc = self._lib.adf_step(self._h, _ptr(state_in.particle_q, torch.float32, n, "particle_q"),
                                _ptr(state_in.particle_qd, torch.float32, n, "particle_qd"),
                                _ptr(state_out.particle_q, torch.float32, n, "particle_q"),
                                _ptr(state_out.particle_qd, torch.float32, n, "particle_qd"),
                                _ptr(f, torch.float32, n, "particle_f") if f is not None else None,
                                float(dt), self._stream())
        _lib.check(rc, "SolverDFSPH.step")

    # ------------------------------------------------------------------------------------------------- reports
    def _world_arrays(self) -> dict[str, np.ndarray]:
        W = max(self.world_count, 1)
        arrs = {"density_err": np.zeros(W, np.float32), "divergence_err": np.zeros(W, np.float32),
                "iters_density": np.zeros(W, np.int32), "iters_divergence": np.zeros(W, np.int32),
                "mass_in": np.zeros(W, np.int64), "mass_out": np.zeros(W, np.int64),
                "mass_initial": np.zeros(W, np.int64), "escaped": np.zeros(W, np.int32),
                "neighbor_overflow": np.zeros(W, np.int32), "max_speed": np.zeros(W, np.float32),
                "density_err_max": np.zeros(W, np.float32), "projected": np.zeros(W, np.int32),
                "nonfinite": np.zeros(W, np.int32), "emitter_overflow": np.zeros(W, np.int32),
                "density_tol": np.zeros(W, np.float32), "learned_divergence": np.zeros(W, np.int32),
                "learned_density": np.zeros(W, np.int32), "swept": np.zeros(W, np.int32)}
        r = _lib.Report(**{k: v.ctypes.data for k, v in arrs.items()})
        _lib.check(self._lib.adf_get_report(self._h, C.byref(r), self._stream()), "report")
        return {k: v[: self.world_count] for k, v in arrs.items()}

    def _active_mass(self) -> np.ndarray:
        out = np.zeros(max(self.world_count, 1), np.int64)
        _lib.check(self._lib.adf_active_mass(self._h, out.ctypes.data, self._stream()), "mass")
        return out[: self.world_count]

    def report(self) -> SPHReport:
        a = self._world_arrays()
        it_den, it_div = a["iters_density"].copy(), a["iters_divergence"].copy()
        mx = self.config.max_iterations
        return SPHReport(
            density_err=a["density_err"].astype(np.float64), divergence_err=a["divergence_err"].astype(np.float64),
            iters_density=it_den, iters_divergence=it_div,
            mass_active=self._active_mass().astype(np.float64) / FIX_SCALE,
            mass_in=a["mass_in"].astype(np.float64) / FIX_SCALE, mass_out=a["mass_out"].astype(np.float64) / FIX_SCALE,
            escaped=a["escaped"].copy(), neighbor_overflow=a["neighbor_overflow"].copy(),
            max_speed=a["max_speed"].astype(np.float64), unconverged=(it_den >= mx) | (it_div >= mx),
            density_tol=a["density_tol"].astype(np.float64))

    def diagnostics(self) -> dict[str, np.ndarray]:
        """Per-world counters beyond SPHReport (runtime.py:410-418)."""
        a = self._world_arrays()
        return {"density_err_max": a["density_err_max"].astype(np.float64), "projected": a["projected"],
                "nonfinite": a["nonfinite"], "emitter_overflow": a["emitter_overflow"],
                "swept": a["swept"], "cavitating": np.zeros(self.world_count, np.int32),
                "learned_divergence": a["learned_divergence"], "learned_density": a["learned_density"]}

    def mass_ledger(self) -> dict[str, np.ndarray]:
        """Exact int64 fixed-point ledger per world: initial, in, out, active (active + out == initial + in)."""
        a = self._world_arrays()
        return {"initial": a["mass_initial"].copy(), "in": a["mass_in"].copy(), "out": a["mass_out"].copy(),
                "active": self._active_mass(), "scale": np.float64(FIX_SCALE)}

    def density_ratio(self, state) -> tuple[np.ndarray, np.ndarray]:
        """Density ratio rho/rho0 of every particle of ``state`` and the active-liquid mask (solver.py:386-393)."""
        if self.n == 0:
            return np.zeros(0), np.zeros(0, dtype=bool)
        ratio = torch.zeros(self.n, dtype=torch.float32, device=self.device)
        active = torch.zeros(self.n, dtype=torch.float32, device=self.device)
        _lib.check(self._lib.adf_density_ratio(self._h, _ptr(state.particle_q), _ptr(state.particle_qd),
                                               ratio.data_ptr(), active.data_ptr(), self._stream()), "density_ratio")
        return ratio.cpu().numpy(), active.cpu().numpy() > 0.0

    def neighbor_rows(self) -> tuple[np.ndarray, np.ndarray]:
        """The last lists as global particle ids [n, capacity] (-1 past count) and counts (neighbors.py:285-295)."""
        K = self.config.neighbor_capacity
        rows = np.zeros((self.n, K), np.int32)
        cnt = np.zeros(self.n, np.int32)
        _lib.check(self._lib.adf_neighbor_rows(self._h, rows.ctypes.data, cnt.ctypes.data, self._stream()),
                   "neighbor_rows")
        return rows, cnt

    # ------------------------------------------------------------------------------------------ learned start
    def set_warm_model(self, model) -> None:
        """Start both pressure solves from the warm-start network ``model`` (a ``warmstart.WarmModel``; None: the
        reference's plain start). Each world keeps the plain start whenever the learned one's first sweep leaves
        the larger residual, and every world iterates to the same tolerance (include/alloy_dfsph.h)."""
        if model is None:
            _lib.check(self._lib.adf_set_warm_model(self._h, None, None), "set_warm_model")
            return
        from .warmstart import Network

        net = Network(model.params, self.device.index or 0)
        norm = np.ascontiguousarray(model.norm_vector(), np.float32)
        _lib.check(self._lib.adf_set_warm_model(self._h, net.handle, norm.ctypes.data), "set_warm_model")
        del net  # the solver holds its own copy of the weights

    def autotune(self, enable: bool = True) -> None:
        """Tune block size and gathers in flight of the neighbour-loop kernels at the next step (on by default;
        include/alloy_dfsph.h adf_set_autotune). Off: the default configuration."""
        _lib.check(self._lib.adf_set_autotune(self._h, int(bool(enable))), "autotune")

    def persistent(self, enable: bool = True) -> None:
        """Run each projected-CG pressure solve of a model of at most 131,072 particles as one persistent launch with
        grid-wide barriers (include/alloy_dfsph.h adf_set_persistent; off by default, the multi-launch path measured
        slightly faster). The results are the same bits either way."""
        _lib.check(self._lib.adf_set_persistent(self._h, int(bool(enable))), "persistent")

    def halo(self, mode: int = 1) -> None:
        """Item halos of the Jacobi iterations (include/alloy_dfsph.h adf_set_halo): 1 staged, 0 global gathers (the
        default, measured faster), -1 the autotuner times both forms for the acceleration and Jacobi kernels. Same
        bits either way."""
        _lib.check(self._lib.adf_set_halo(self._h, int(mode)), "halo")

    def halo_stats(self) -> dict:
        """The halo choice in use and, after a step that built them, the items staged and left on global gathers,
        the staged records summed and the largest item's (adf_halo_stats)."""
        use = np.zeros(2, np.int32)
        st = np.zeros(4, np.int64)
        _lib.check(self._lib.adf_halo_stats(self._h, use.ctypes.data, st.ctypes.data, self._stream()), "halo_stats")
        return {"accel": bool(use[0]), "jacobi": bool(use[1]), "staged": int(st[0]), "global": int(st[1]),
                "records": int(st[2]), "max_records": int(st[3])}

    def barrier_wait(self, polls: int = 1 << 22, extra_arrivals: int = 0) -> None:
        """Test hook of the persistent solve's bounded barrier waits (adf_set_barrier_wait): polls per wait, and
        arrivals a barrier waits for beyond the grid's blocks (nonzero makes every wait run out)."""
        _lib.check(self._lib.adf_set_barrier_wait(self._h, int(polls), int(extra_arrivals)), "barrier_wait")

    def clear_status(self) -> None:
        """Clear the status of the bounded waits after one gave up (adf_clear_status)."""
        _lib.check(self._lib.adf_clear_status(self._h), "clear_status")

    def tuned_configs(self) -> dict[str, dict]:
        """{kernel: {"block", "nb", "ms"}} of the configuration in use (ms < 0: not tuned)."""
        k = len(_lib.TUNE_KERNELS)
        blk, nb, ms = np.zeros(k, np.int32), np.zeros(k, np.int32), np.zeros(k, np.float32)
        _lib.check(self._lib.adf_tuned_configs(self._h, blk.ctypes.data, nb.ctypes.data, ms.ctypes.data), "tuned")
        return {name: {"block": int(blk[i]), "nb": int(nb[i]), "ms": float(ms[i])}
                for i, name in enumerate(_lib.TUNE_KERNELS)}

    def set_tuned_config(self, kernel: str, block: int, nb: int) -> None:
        """Pin one kernel's launch configuration (a tuner candidate; for "lists", nb = particles per warp)."""
        _lib.check(self._lib.adf_set_tuned_config(self._h, _lib.TUNE_KERNELS.index(kernel), int(block), int(nb)),
                   "set_tuned_config")

    def warm_judging(self, enable: bool = True) -> None:
        """Judge the learned start by one sweep from both starts (default). Off: the learned start is taken outright
        (a measurement of the network alone; every world still iterates to the same tolerance)."""
        _lib.check(self._lib.adf_set_warm_judging(self._h, int(bool(enable))), "warm_judging")

    def record_features(self, enable: bool = True) -> None:
        """Record the network's features of every liquid particle at the start of each step's first solve."""
        _lib.check(self._lib.adf_set_feature_recording(self._h, int(bool(enable))), "record_features")

    def warm_features(self) -> torch.Tensor:
        """The last step's recorded features, [n, 16] float32 on the device (zero rows for non-liquid particles)."""
        out = torch.empty((self.n, 16), dtype=torch.float32, device=self.device)
        _lib.check(self._lib.adf_warm_features(self._h, out.data_ptr(), self._stream()), "warm_features")
        return out

    def debug_field(self, name: str) -> np.ndarray:
        """A per-particle field of the last step in particle order (parity tests); slot fields take ``:k`` for slot k
        (include/alloy_dfsph.h adf_debug_field)."""
        three = name.split(":")[0] in ("acc", "slot_g", "slot_vb", "slot_n")
        out = torch.zeros((self.n, 3) if three else self.n, dtype=torch.float32, device=self.device)
        _lib.check(self._lib.adf_debug_field(self._h, name.encode(), out.data_ptr(), self._stream()), "debug_field")
        return out.cpu().numpy()

    def skin_flags(self) -> np.ndarray:
        """Per-world rebuild flags of the last step's Verlet-skin update (neighbors_skin.py:206-208
        ``rebuilt_worlds``); ValueError without ``reneighbor_skin``."""
        if not self._params.skin:
            raise ValueError("SolverDFSPH.skin_flags: reneighbor_skin is off")
        out = np.zeros(max(self.world_count, 1), np.int32)
        _lib.check(self._lib.adf_skin_flags(self._h, out.ctypes.data, self._stream()), "skin_flags")
        return out[:self.world_count].astype(bool)

    def kernel_launches(self) -> int:
        return int(self._lib.adf_kernel_launches(self._h))

    def use_graphs(self, enable: bool) -> None:
        """Replay each step as one CUDA graph (default) or launch its kernels one by one (include/alloy_dfsph.h)."""
        _lib.check(self._lib.adf_set_graphs(self._h, int(bool(enable))), "use_graphs")

    def profile(self, enable: bool) -> None:
        """Time every kernel group with CUDA events on the launch stream (``profile_read``)."""
        _lib.check(self._lib.adf_profile_enable(self._h, int(bool(enable))), "profile")

    def profile_read(self) -> dict[str, tuple[float, int]]:
        """{kind: (milliseconds, launches)} since the last read (include/alloy_dfsph.h ADF_PROF_KINDS)."""
        ms = np.zeros(len(_lib.PROF_KINDS), np.float64)
        cnt = np.zeros(len(_lib.PROF_KINDS), np.int64)
        _lib.check(self._lib.adf_profile_read(self._h, ms.ctypes.data, cnt.ctypes.data), "profile_read")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.PROF_KINDS)}

    def iteration_work(self) -> int:
        """Liquid particles processed by the Jacobi iterations so far (their work lists cover the worlds still
        iterating)."""
        v = np.zeros(1, np.int64)
        _lib.check(self._lib.adf_iteration_work(self._h, v.ctypes.data, self._stream()), "iteration_work")
        return int(v[0])

    def list_stats(self) -> tuple[int, int]:
        """(liquid particles, neighbour-row entries) of the last list build."""
        nf = np.zeros(1, np.int32)
        ne = np.zeros(1, np.int64)
        _lib.check(self._lib.adf_list_stats(self._h, nf.ctypes.data, ne.ctypes.data, self._stream()), "list_stats")
        return int(nf[0]), int(ne[0])

    # ------------------------------------------------------------------------------------------------- control
    def prime(self, state, dt: float, tol: float = 1.0e-6, max_iterations: int = 2000) -> int:
        """Give a fluid at rest its hydrostatic pressure before the first step (solver.py:369-372, prime.py:52-87):
        the hydrostatic guess per liquid column, refined by one divergence solve of the velocity a gravity step
        adds, becomes the first density solve's warm start. ``state`` is not changed. Returns the iterations."""
        if self.n == 0:
            return 0
        guess = hydrostatic_guess(self, state)
        kv = torch.as_tensor(guess * np.float32(dt), dtype=torch.float32, device=self.device)
        _lib.check(self._lib.adf_set_warm_starts(self._h, kv.data_ptr(), self._kd.data_ptr(), self._stream()),
                   "prime")
        it = np.zeros(1, np.int32)
        _lib.check(self._lib.adf_prime(self._h, _ptr(state.particle_q, torch.float32, self.n, "particle_q"),
                                       _ptr(state.particle_qd, torch.float32, self.n, "particle_qd"), float(dt),
                                       float(tol), int(max_iterations), it.ctypes.data, self._stream()), "prime")
        return int(it[0])

    def reset(self, state=None, world_mask=None, flags: int | None = None) -> None:
        """Masked worlds (all when None) back to their build-time SPH configuration (solver.py:353-362)."""
        del state, flags
        if self.n == 0:
            return
        mask = None
        if world_mask is not None:
            m = _host(world_mask).astype(np.uint8)[: self.world_count]
            mask = np.ascontiguousarray(m)
        _lib.check(self._lib.adf_reset(self._h, mask.ctypes.data if mask is not None else None,
                                       self._flags0.data_ptr(), self._phase0.data_ptr(), self._stream()), "reset")

    def choose_dt(self, control_dt: float) -> float:
        """CFL step from the last step's max speed, snapped down to the control grid (solver.py:424-426)."""
        a = self._world_arrays()
        v = float(np.max(a["max_speed"])) if self.world_count else 0.0
        return snap_down(stable_dt(self.config, v), control_dt)

    def alloy_stable_dt(self, state, contacts, out) -> None:
        """out[w] (device float32 [W]) = clamp(cfl 2r / |v|max, dt_min, dt_max) over the state's liquid, dt_max at
        rest (runtime.py:411-421); one pass over the particles on the device, nothing allocated."""
        del contacts
        if self.world_count == 0:
            return
        cfg = self.config
        _lib.check(self._lib.adf_stable_dt(self._h, _ptr(state.particle_qd, torch.float32, self.n, "particle_qd"),
                                           float(cfg.cfl), float(cfg.dt_min), float(cfg.dt_max),
                                           _ptr(out, torch.float32, self.world_count, "out"), self._stream()),
                   "alloy_stable_dt")

    def alloy_energy(self, state, z_ref, out) -> None:
        """Kinetic + gravity energy [J] of each world's liquid about (0, 0, z_ref[w]) into ``out`` (device float64
        [W]); float64 per-world sums in a fixed order (runtime.py:66-79, 423-430)."""
        if self.world_count == 0:
            return
        W = self.world_count
        _lib.check(self._lib.adf_energy(self._h, _ptr(state.particle_q, torch.float32, self.n, "particle_q"),
                                        _ptr(state.particle_qd, torch.float32, self.n, "particle_qd"),
                                        _ptr(z_ref, torch.float64, W, "z_ref"), _ptr(out, torch.float64, W, "out"),
                                        self._stream()), "alloy_energy")

    def alloy_capacity_report(self) -> dict[str, int]:
        a = self._world_arrays()
        return {"neighbor_overflow": int(a["neighbor_overflow"].sum()),
                "emitter_overflow": int(a["emitter_overflow"].sum())}

    def _storage(self) -> dict[str, torch.Tensor]:
        """Views of the library's own device arrays behind the snapshot keys (include/alloy_dfsph.h
        adf_state_storage). The emitter views change when emitters are added."""
        st = _lib.StateStorage()
        _lib.check(self._lib.adf_get_state_storage(self._h, C.byref(st)), "state storage")
        W, n = self.world_count, self.n

        def view(ptr, count, typestr):
            return torch.as_tensor(_DevView(ptr, (max(count, 1),), typestr), device=self.device)[:count]

        out = {"mass_in": view(st.mass_in, W, "<i8"), "mass_out": view(st.mass_out, W, "<i8"),
               "escaped": view(st.escaped, W, "<i4"), "port_stack": view(st.port_stack, n, "<i4"),
               "port_top": view(st.port_top, W, "<i4"), "port_absorbed": view(st.port_absorbed, W, "<i4"),
               "port_emitted": view(st.port_emitted, W, "<i4"), "port_retired": view(st.port_retired, W, "<i4"),
               "taken": view(st.port_taken, W, "<i4"), "granted": view(st.port_granted, W, "<i4")}
        if st.warm_probe_gap:
            out.update({"warm_probe_gap": view(st.warm_probe_gap, 2 * W, "<i4"),
                        "warm_probe_wait": view(st.warm_probe_wait, 2 * W, "<i4")})
        P_ = int(st.n_patch_entries)
        if P_:
            out.update({"patch_pending": view(st.patch_pending, P_, "<i4"),
                        "patch_fired": view(st.patch_fired, P_, "<i4"), "patch_world": view(st.patch_world, P_, "<i4")})
        E = int(st.n_emitters)
        if E:
            out.update({"emit_t": view(st.emit_t, E, "<f4"), "emit_cursor": view(st.emit_cursor, E, "<i4"),
                        "emit_world": view(st.emit_world, E, "<i4")})
        return out

    def alloy_state_arrays(self, state=None) -> dict:
        """The solver state a snapshot must hold beside State (coupling_hooks.py:115-126): warm starts, phase and
        flags, the mass ledger (runtime.py:173-174), the emitters' clocks and cursors (runtime.py:389-393) and the
        port (ports.py:201-203). Every value is the library's own storage: a snapshot copies it out and back in
        place between steps."""
        del state
        a = self._storage()
        arrays = {"sph.kappa_v": self._kv, "sph.kappa_d": self._kd, "sph.phase": self.model.sph.phase,
                  "particle_flags": self.model.particle_flags, "sph.mass_in": a["mass_in"],
                  "sph.mass_out": a["mass_out"], "sph.escaped": a["escaped"]}
        if "emit_t" in a:
            arrays.update({"sph.emit_t": a["emit_t"], "sph.emit_cursor": a["emit_cursor"]})
        arrays.update(self.port.state_arrays())
        arrays.update(self._patch_views(a, "patch_pending", "patch_fired"))  # patch.py:236-241
        if "warm_probe_gap" in a:  # the learned start's evaluation schedule (no counterpart in the reference)
            arrays.update({"sph.warm_probe_gap": a["warm_probe_gap"], "sph.warm_probe_wait": a["warm_probe_wait"]})
        return arrays

    def _patch_views(self, a: dict, pending: str, fired: str) -> dict:
        """Group k's slices of the patch entry arrays under the reference's keys sph.patch_pending{k} / fired{k}."""
        out, e = {}, 0
        for k, g in enumerate(self._patches):
            if g:
                out[f"sph.patch_pending{k}"] = a[pending][e:e + len(g)]
                out[f"sph.patch_fired{k}"] = a[fired][e:e + len(g)]
            e += len(g)
        return out

    def alloy_state_worlds(self) -> dict:
        """Item -> world maps of the per-item arrays in ``alloy_state_arrays`` (coupling_hooks.py:128-138); per-world
        arrays are world-major and need none. The port stack holds world w's particles in that world's own index
        range, so its map is the particles' world."""
        pw = self.model.particle_world
        maps = {"sph.kappa_v": pw, "sph.kappa_d": pw, "sph.phase": pw, "particle_flags": pw, "sph.port_stack": pw}
        a = self._storage()
        if "emit_world" in a:
            maps.update({"sph.emit_t": a["emit_world"], "sph.emit_cursor": a["emit_world"]})
        if self._patches and "patch_world" in a:
            maps.update(self._patch_views(a, "patch_world", "patch_world"))
        if "warm_probe_gap" in a:  # [2][W]: divergence then density, world-major within each
            two = torch.arange(2 * self.world_count, dtype=torch.int32, device=self.device) % max(self.world_count, 1)
            maps.update({"sph.warm_probe_gap": two, "sph.warm_probe_wait": two})
        return maps

    # ------------------------------------------------------------------------------------------------ port
    def retire(self, state, mask) -> None:
        """Retire the masked liquid particles for good (``mask [n]`` int32; one launch, capture-safe): their mass
        leaves the ledger as at a sink; ``port.taken[w]`` counts them (solver.py:428-431, ports.py:187-189)."""
        self.port.retire(state, mask)

    # ------------------------------------------------------------------------------------------------ model
    def notify_model_changed(self, flags: int) -> None:
        """solver.py:343-351. The reference re-derives its body modes when body properties change and rebuilds its
        shape table when shape properties change. This path has no bodies, its box walls are static (the constructor
        refuses moving or rotated shapes, and their table is fixed at construction), and every step reads the particle
        arrays, masses, rest densities and gravity live from the model, so no flag leaves anything to rebuild."""
        int(flags)

    @staticmethod
    def emit(builder, obj, decision) -> None:
        """Scene assembly's emit (solver.py:475-479, build.py:265-285): a liquid object -> active lattice particles
        in ``builder``'s current world (``build.emit_object``)."""
        from .build import emit_object

        emit_object(builder, obj, decision)

    # ------------------------------------------------------------------------------------------------ coupling
    def coupling_notify_input_state_update(self, state, flags: int, *, iteration_restart: bool = False,
                                           dt: float = 0.0) -> None:
        """coupling_hooks.py:41-72: every pass of one exchange starts from the same solver state. A restart copies
        back the warm starts, flags, phase, ledgers and emitter clocks saved at the exchange's first pass; any other
        notification saves them."""
        del state, flags, dt
        if self.n == 0:
            return
        live = {"kv": self._kv, "kd": self._kd, "flags": self.model.particle_flags, "phase": self.model.sph.phase}
        live.update({k: v for k, v in self._storage().items() if k in ("mass_in", "mass_out", "escaped", "emit_t",
                                                                          "emit_cursor")})
        if iteration_restart:
            for k, a in live.items():
                if k in self._saved and self._saved[k].shape == a.shape:
                    a.copy_(self._saved[k])
        else:
            self._saved = {k: a.clone() for k, a in live.items()}

    def coupling_prepare_proxy_contacts(self, state, contacts, *, contacts_freshly_detected: bool = False):
        del state, contacts_freshly_detected
        return contacts  # the liquid reads no contact rows: its walls are particle walls

    def coupling_supports_full_surface_soft_contacts(self) -> bool:
        return True  # contacts are ignored, so any soft-contact layout is acceptable

    def coupling_supports_inertial_property_refresh(self) -> bool:
        return False

    def coupling_harvest_proxy_wrenches(self, body_local_to_proxy_global, out_body_f, **kwargs) -> None:
        """This path has no proxy bodies (coupling_hooks.py:74-86 integrates them): only an empty mapping is valid."""
        del out_body_f, kwargs
        if len(body_local_to_proxy_global):
            raise ValueError("SolverDFSPH (B200 build): proxy bodies are not part of the B200 CUDA path")

    def coupling_rewind_proxy_particle(self, particle_local_to_proxy_global, state, coupling_forces,
                                       particle_gravity_acceleration, dt: float) -> None:
        """coupling_hooks.py:88-95: lagged particle proxies are refused beside walls."""
        del state, coupling_forces, particle_gravity_acceleration, dt
        if len(particle_local_to_proxy_global):
            raise ValueError("SolverDFSPH particle walls need a staggered proxy pair (PairPolicy / Proxy mode "
                             "'staggered' with Aitken relaxation); lagged proxies diverge for a liquid-wall pair")

    def coupling_harvest_proxy_particle_forces(self, particle_local_to_proxy_global, out_particle_f, *, dt: float,
                                               **kwargs) -> None:
        """coupling_hooks.py:97-105 returns the liquid's force on two-way particle walls. This path's walls are
        one-way (prescribed): the wall reactions are not accumulated, so a non-empty mapping is refused."""
        del out_particle_f, kwargs
        if len(particle_local_to_proxy_global) == 0:
            return
        if not dt > 0.0:
            raise ValueError("SolverDFSPH harvest requires dt > 0")
        raise ValueError("SolverDFSPH (B200 build): two-way particle walls (reaction forces on proxies) are not part "
                         "of the B200 CUDA path")

    # ------------------------------------------------------------------------------------------------ emitters
    def _spares(self, w: int) -> np.ndarray:
        """Inactive spares of world w not reserved by a patch emitter, ascending (runtime.py:215-219)."""
        ph = _host(self.model.sph.phase)
        wo = _host(self.model.particle_world)
        fl = _host(self.model.particle_flags)
        ids = np.nonzero((ph == PHASE_SPARE) & (wo == w) & ((fl & _ACTIVE) == 0))[0].astype(np.int32)
        held = [g[w] for g in self._patches if w in g]
        return np.setdiff1d(ids, np.concatenate(held)).astype(np.int32) if held else ids

    def _unowned_spares(self, w: int) -> np.ndarray:
        """``_spares`` minus the pools emitters own, for patch emitters to reserve (runtime.py:221-226)."""
        owned = [self._em_pool[e] for e, w2 in enumerate(self._em_world) if w2 == w and self._em_own[e]]
        sp = self._spares(w)
        return np.setdiff1d(sp, np.concatenate(owned)).astype(np.int32) if owned else sp

    def add_patch_emitter(self, world_mask, body, local_points, velocity=(0.0, 0.0, 0.0)) -> int:
        """Triggered one-shot emitter (solver.py:449-453, patch.py): for each masked world w, ``local_points[w]``
        (N_w, 3) in the world frame (``body`` -1: this path has no bodies), emitted with ``velocity`` once a
        ``trigger`` armed the world; N_w spares are reserved now (CapacityError if short), and the world's box
        emitters re-split the rest, so they must not have emitted yet (runtime.py:228-241). Returns the id."""
        W = self.world_count
        mask = np.asarray(world_mask, bool)
        if mask.shape != (W,) or len(local_points) != W:
            raise ValueError(f"add_patch_emitter: world_mask and local_points need one entry per world ({W})")
        bodies = np.full(W, int(body), np.int32) if np.ndim(body) == 0 else np.asarray(body, np.int32)
        if bodies.shape != (W,):
            raise ValueError(f"add_patch_emitter: body must be one index or one per world ({W})")
        body_count = int(getattr(self.model, "body_count", 0) or 0)
        if np.any((bodies < -1) | (bodies >= body_count)):
            raise ValueError("add_patch_emitter: body indices must be in [-1, body_count)")
        for w in np.nonzero(mask)[0]:
            a = np.asarray(local_points[w])
            if a.size and a.reshape(-1, 3).shape[1] != 3:
                raise ValueError(f"add_patch_emitter: local_points[{w}] must be (N, 3)")
        worlds = [w for w in range(W) if mask[w] and len(local_points[w])]
        box = [e for e, w in enumerate(self._em_world) if w in set(worlds)]
        if box:
            cursors = np.zeros(len(self._em_world), np.int32)
            _lib.check(self._lib.adf_emitter_state(self._h, None, cursors.ctypes.data), "emitters")
            if np.any(cursors[box] > 0):
                raise ValueError("add_patch_emitter: a box emitter of these worlds has emitted; add patch emitters "
                                 "first")
        pts = [np.asarray(local_points[w], np.float32).reshape(-1, 3) for w in worlds]
        reserved = {}
        for w, q in zip(worlds, pts, strict=True):
            free = self._unowned_spares(w)
            if len(free) < len(q):
                raise _lib.CapacityError(f"add_patch_emitter: world {w} has {len(free)} free spares, needs {len(q)}")
            reserved[w] = free[:len(q)].astype(np.int32)
        wa = np.asarray(worlds if worlds else [0], np.int32)
        counts = np.asarray([len(q) for q in pts] if worlds else [0], np.int32)
        pool = np.ascontiguousarray(np.concatenate([reserved[w] for w in worlds]) if worlds else np.zeros(1, np.int32))
        flat = np.ascontiguousarray(np.concatenate(pts) if worlds else np.zeros((1, 3), np.float32), np.float32)
        vel = np.ascontiguousarray(np.asarray(velocity, np.float32).reshape(3))
        pid = self._lib.adf_add_patch_emitter(self._h, len(worlds), wa.ctypes.data, counts.ctypes.data,
                                              pool.ctypes.data, flat.ctypes.data, vel.ctypes.data)
        _lib.check(pid if pid < 0 else 0, "add_patch_emitter")
        self._patches.append(reserved)
        for w in sorted({self._em_world[e] for e in box}):
            self._split_pools(w)
        log.info("SPH patch emitter %d: %d worlds, up to %d particles each", pid, len(worlds),
                 int(counts.max()) if worlds else 0)
        return int(pid)

    def trigger(self, pid: int, world_flags) -> None:
        """Arm patch emitter ``pid`` in the worlds where ``world_flags`` (device int32 or bool, one per world) is
        set; the next step emits there once (solver.py:455-458; one launch, capture-safe)."""
        if not 0 <= pid < len(self._patches):
            raise ValueError(f"trigger: no patch emitter {pid}")
        if not self._patches[pid]:
            return
        if world_flags.shape[0] < self.world_count:
            raise ValueError(f"trigger: world_flags needs >= {self.world_count} entries")
        is_bool = world_flags.dtype == torch.bool
        if not is_bool and world_flags.dtype != torch.int32:
            raise ValueError("trigger: world_flags must be int32 or bool")
        _lib.check(self._lib.adf_trigger(self._h, int(pid), _ptr(world_flags), int(is_bool), self._stream()),
                   "trigger")

    def _first_sph(self, world: int) -> int:
        ws = self.world_start
        ph = _host(self.model.sph.phase)[ws[world]:ws[world + 1]]
        idx = np.nonzero(sph_phase(ph))[0]
        if len(idx) == 0:
            raise ValueError(f"world {world} has no SPH particles or spares")
        return int(ws[world] + idx[0])

    def add_emitter(self, world: int, region, half_extents, rate: float, velocity, pool=None) -> int:
        """Emit liquid from a box region at ``rate`` [m^3/s] with ``velocity`` [m/s] by activating spares
        (runtime.py:498-525)."""
        return self.add_emitters([(world, region, half_extents, rate, velocity, pool)])[0]

    def add_emitters(self, specs) -> list[int]:
        """Several emitters at once, each ``(world, region, half_extents, rate, velocity, pool)`` as in
        ``add_emitter``: the host arrays are read once and the library uploads its emitter tables once."""
        cfg = self.config
        ph = _host(self.model.sph.phase)
        fl = _host(self.model.particle_flags)
        mass = _host(self.model.particle_mass)
        rho = _host(self.model.sph.rest_density)
        ws = self.world_start
        sph_ids = np.nonzero(sph_phase(ph))[0]
        spare_ids = np.nonzero((ph == PHASE_SPARE) & ((fl & _ACTIVE) == 0))[0].astype(np.int32)
        rows = []
        packing = []
        for world, region, half_extents, rate, velocity, pool in specs:
            if not 0 <= world < self.world_count:
                raise ValueError(f"add_emitter: world {world} out of range")
            if rate <= 0.0:
                raise ValueError("add_emitter: rate must be > 0 [m^3/s]")
            X = _xform7(region)
            v_local = quat_rotate_inv(X[3:], np.asarray(velocity, np.float64))
            offs = layer_offsets(np.asarray(half_extents, dtype=np.float64), v_local, cfg.spacing)
            k = np.searchsorted(sph_ids, ws[world])
            if k >= len(sph_ids) or sph_ids[k] >= ws[world + 1]:
                raise ValueError(f"world {world} has no SPH particles or spares")
            i0 = int(sph_ids[k])
            interval = len(offs) * (float(mass[i0]) / float(rho[i0])) / rate
            speed = float(np.linalg.norm(v_local))
            if speed > 0.0:
                packing.append(rate / (len(offs) * cfg.spacing * cfg.spacing * speed))
            own = pool is not None
            if own:
                lo_, hi_ = np.searchsorted(spare_ids, [ws[world], ws[world + 1]])
                pool_ids = np.intersect1d(np.asarray(pool), spare_ids[lo_:hi_]).astype(np.int32)
            else:
                pool_ids = np.zeros(0, np.int32)
            rows.append((int(world), X, offs, np.asarray(velocity, np.float32), interval, pool_ids, own))
        bad = [r for r in packing if not 0.8 <= r <= 1.25]
        if bad:
            log.warning("SPH emitters: %d of %d have rate / (area |v|) outside [0.8, 1.25] (e.g. %.3g): layers will "
                        "over/under-pack", len(bad), len(packing), bad[0])
        if not rows:
            return []
        cnt = len(rows)
        world_a = np.array([r[0] for r in rows], np.int32)
        xform = np.ascontiguousarray(np.stack([r[1] for r in rows]), np.float32)
        n_off = np.array([len(r[2]) for r in rows], np.int32)
        offsets = np.ascontiguousarray(np.concatenate([r[2] for r in rows]).reshape(-1, 3), np.float32)
        vel = np.ascontiguousarray(np.stack([r[3] for r in rows]), np.float32)
        interval = np.array([r[4] for r in rows], np.float32)
        psize = np.array([len(r[5]) for r in rows], np.int32)
        pools = np.ascontiguousarray(np.concatenate([r[5] for r in rows]), np.int32)
        first = self._lib.adf_add_emitters(self._h, cnt, world_a.ctypes.data, xform.ctypes.data, n_off.ctypes.data,
                                           offsets.ctypes.data, vel.ctypes.data, interval.ctypes.data,
                                           psize.ctypes.data, pools.ctypes.data)
        _lib.check(first if first < 0 else 0, "add_emitter")
        for r in rows:
            self._em_world.append(r[0])
            self._em_pool.append(r[5])
            self._em_own.append(r[6])
        for w in sorted({r[0] for r in rows if not r[6]}):
            self._split_pools(w)
        log.info("SPH emitters %d..%d added", first, first + cnt - 1)
        return list(range(int(first), int(first) + cnt))

    def _split_pools(self, world: int) -> None:
        """Share the world's unused spares evenly among its emitters given no pool (emitters.py:225-238)."""
        spares = self._spares(world)
        owned = [self._em_pool[e] for e, w in enumerate(self._em_world) if w == world and self._em_own[e]]
        free = np.setdiff1d(spares, np.concatenate(owned)) if owned else spares
        mine = [e for e, w in enumerate(self._em_world) if w == world and not self._em_own[e]]
        if not mine:
            return
        cursors = np.zeros(len(self._em_world), np.int32)
        _lib.check(self._lib.adf_emitter_state(self._h, None, cursors.ctypes.data), "emitters")
        new = {}
        if any(cursors[e] > 0 for e in mine[:-1]):
            used = np.concatenate([self._em_pool[e] for e in mine[:-1]]) if len(mine) > 1 else np.zeros(0, np.int32)
            new[mine[-1]] = np.setdiff1d(free, used).astype(np.int32)
        else:
            for k, part in enumerate(np.array_split(free, len(mine))):
                new[mine[k]] = part.astype(np.int32)
        for e, pool in new.items():
            pool = np.ascontiguousarray(pool, np.int32)
            self._em_pool[e] = pool
            _lib.check(self._lib.adf_set_emitter_pool(self._h, int(e), pool.ctypes.data, len(pool)), "emitter pool")

    def set_emitter_enabled(self, e: int, on: bool) -> None:
        _lib.check(self._lib.adf_set_emitter_enabled(self._h, int(e), int(bool(on))), "set_emitter_enabled")

    def add_sink(self, world: int, region, half_extents) -> int:
        """Retire particles that enter a box region; their mass goes to ``mass_out`` (runtime.py:557-565)."""
        X = _xform7(region)
        half = np.asarray(half_extents, np.float32)
        k = self._lib.adf_add_sink(self._h, int(world), X.ctypes.data, half.ctypes.data)
        _lib.check(k if k < 0 else 0, "add_sink")
        return int(k)
