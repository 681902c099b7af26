# TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
"""ctypes front end of the CPU oracle (dfsph_oracle.cpp): the reference DFSPH step restated on the CPU.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs use it, as the parity checker or the timed CPU
baseline. The product (alloy_b200) never imports it.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle_dfsph.so"
SRC = HERE / "dfsph_oracle.cpp"
CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC", "-shared",
            "-std=c++17"]


def build(force: bool = False) -> Path:
    """Compile the oracle (g++, OpenMP) next to its source."""
    if force or not LIB.exists() or LIB.stat().st_mtime < SRC.stat().st_mtime:
        tmp = LIB.with_suffix(f".{os.getpid()}.tmp")
        subprocess.run(["g++", *CXXFLAGS, "-o", str(tmp), str(SRC)], check=True)
        os.replace(tmp, LIB)
    return LIB


class OrcParams(C.Structure):
    _fields_ = [("kind", C.c_int), ("particle_radius", C.c_double), ("h", C.c_double), ("sigma", C.c_double),
                ("n_full", C.c_double), ("tot_min", C.c_double), ("lattice_grad", C.c_double),
                ("wall_offset", C.c_double), ("wall_amplitude", C.c_double), ("taper0", C.c_double),
                ("taper1", C.c_double), ("reach", C.c_double), ("tol_den", C.c_double), ("tol_div", C.c_double),
                ("max_error_factor", C.c_double), ("min_it", C.c_int), ("max_it", C.c_int), ("omega", C.c_double),
                ("warm_den", C.c_double), ("warm_div", C.c_double), ("min_nb", C.c_double),
                ("divergence_solve", C.c_int), ("two_sided", C.c_int), ("xsph_c", C.c_double),
                ("capacity", C.c_int), ("v_sep", C.c_double), ("relief_speed", C.c_double),
                ("project_eps", C.c_double), ("has_bounds", C.c_int), ("bounds_lo", C.c_double * 3),
                ("bounds_hi", C.c_double * 3), ("cg", C.c_int), ("wall_friction", C.c_int),
                ("jitter_speed", C.c_double), ("jitter_ratio", C.c_double), ("tol_den_min", C.c_double)]


def params_from_config(cfg) -> OrcParams:
    from alloy_b200.solvers.sph.config import host_constants

    hc = host_constants(cfg)
    p = OrcParams()
    p.kind = cfg.kernel_id
    p.particle_radius = cfg.particle_radius
    p.h, p.sigma, p.n_full, p.tot_min, p.lattice_grad = hc.h, hc.sigma, hc.n_full, hc.tot_min, hc.lattice_grad
    p.wall_offset, p.wall_amplitude, p.taper0, p.taper1, p.reach = (hc.wall_offset, hc.wall_amplitude, hc.taper0,
                                                                   hc.taper1, hc.reach)
    p.tol_den, p.tol_div, p.max_error_factor = cfg.max_density_error, cfg.max_divergence_error, cfg.max_error_factor
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
    p.jitter_speed = cfg.rest_jitter_speed or 0.0
    p.jitter_ratio = cfg.rest_jitter_flow_ratio
    p.tol_den_min = min(cfg.min_density_error, cfg.max_density_error)
    if cfg.world_bounds is not None:
        p.has_bounds = 1
        for a in range(3):
            p.bounds_lo[a], p.bounds_hi[a] = cfg.world_bounds[0][a], cfg.world_bounds[1][a]
    return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(str(build()))
        P = C.c_void_p
        fp, ip, dp = C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_double)
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.POINTER(OrcParams), C.c_int, C.c_int, ip, fp, fp, ip, C.c_void_p, ip, fp, fp,
                                 C.c_int]
        for name in ("orc_destroy", "orc_prepare_density"):
            getattr(L, name).argtypes = [P]
        L.orc_set_threads.argtypes = [P, C.c_int]
        L.orc_set_state.argtypes = [P, fp, fp]
        L.orc_set_velocity.argtypes = [P, C.c_int, ip, fp]
        L.orc_get_state.argtypes = [P, fp, fp]
        L.orc_get_state_f64.argtypes = [P, dp, dp]
        L.orc_set_warm.argtypes = [P, fp, fp]
        L.orc_get_warm.argtypes = [P, fp, fp]
        L.orc_get_flags_phase.argtypes = [P, ip, C.c_void_p]
        L.orc_step.argtypes = [P, C.c_double]
        L.orc_prime.argtypes = [P, C.c_double, C.c_double, C.c_int]
        L.orc_get_field.argtypes = [P, C.c_char_p, fp]
        L.orc_get_slot_on.argtypes = [P, ip]
        L.orc_get_slot_shapes.argtypes = [P, ip]
        L.orc_set_shapes.argtypes = [P, C.c_int, ip, ip, fp, fp, fp, fp, C.c_double, ip, fp]
        L.orc_shape_sdf.argtypes = [P, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.orc_get_lists.argtypes = [P, ip, ip]
        L.orc_get_report.argtypes = [P, ip, fp, C.POINTER(C.c_int64)]
        L.orc_active_mass.argtypes = [P, C.POINTER(C.c_int64)]
        L.orc_add_emitter.argtypes = [P, C.c_int, fp, fp, C.c_int, fp, C.c_float, ip, C.c_int]
        L.orc_add_sink.argtypes = [P, C.c_int, fp, fp]
        L.orc_kernel_wf.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, fp, fp, fp]
        L.orc_kernel_wf64.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, dp, dp, dp]
        L.orc_halfspace.argtypes = [C.c_int, C.c_double, C.c_int, fp, fp, fp]
        L.orc_halfspace64.argtypes = [C.c_int, C.c_double, C.c_int, dp, dp, dp]
        L.orc_colour_distance.argtypes = [C.c_int, C.c_double, C.c_int, fp, fp]
        L.orc_world_sum.argtypes = [C.c_int, ip, fp, dp, fp]
        _lib = L
    return _lib


def _p(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Oracle:
    """One oracle solver over host copies of a model's arrays (``Model.host()``)."""

    def __init__(self, arrays: dict, cfg, f64: bool = False, threads: int | None = None):
        self.L = lib()
        self.cfg = cfg
        self.f64 = f64
        a = {k: np.ascontiguousarray(v) for k, v in arrays.items()}
        self.n = n = len(a["mass"])
        self.W = W = len(a["world_start"]) - 1
        proxy = (a["flags"] & 2) != 0
        r64 = a["radius"].astype(np.float64)
        self.wall_vol = np.where(proxy, 8.0 * r64 * r64 * r64, 0.0).astype(np.float32)
        self._keep = [np.ascontiguousarray(a["world_start"], np.int32), np.ascontiguousarray(a["mass"], np.float32),
                      np.ascontiguousarray(a["rest_density"], np.float32), np.ascontiguousarray(a["flags"], np.int32),
                      np.ascontiguousarray(a["phase"], np.int8), np.ascontiguousarray(a["world"], np.int32),
                      self.wall_vol, np.ascontiguousarray(a["gravity"], np.float32).reshape(-1)]
        ws, m, r0, fl, ph, wo, wv, g = self._keep
        self.params = params_from_config(cfg)
        from alloy_b200.solvers.sph.config import PHASE_HELD, PHASE_SPARE, uniform_layout

        sph = (a["phase"] >= PHASE_SPARE) | (a["phase"] == PHASE_HELD)
        self.params.cg = int(cfg.pressure_solver == "cg" and uniform_layout(a["mass"][sph], a["rest_density"][sph]))
        self.h = self.L.orc_create(C.byref(self.params), n, W, _p(ws, C.c_int), _p(m, C.c_float), _p(r0, C.c_float),
                                   _p(fl, C.c_int), ph.ctypes.data, _p(wo, C.c_int), _p(wv, C.c_float),
                                   _p(g, C.c_float), int(f64))
        if threads is not None:
            self.L.orc_set_threads(self.h, int(threads))
        self.set_state(a["q"], a["qd"])
        if "shape_type" in a and len(a["shape_type"]):
            self.set_shapes(a)

    def set_shapes(self, a: dict):
        """The model's static box walls (``alloy_b200.solvers.sph.shapes.shape_table`` of the same arrays)."""
        from types import SimpleNamespace

        import torch

        from alloy_b200.solvers.sph.shapes import shape_table

        t = lambda k: torch.from_numpy(np.ascontiguousarray(a[k]))  # noqa: E731
        m = SimpleNamespace(world_count=self.W, shape_count=len(a["shape_type"]), shape_type=t("shape_type"),
                            shape_flags=t("shape_flags"), shape_world=t("shape_world"), shape_body=t("shape_body"),
                            shape_scale=t("shape_scale"), shape_transform=t("shape_transform"),
                            shape_material_mu=t("shape_mu"), sph=SimpleNamespace(shape_boundary=t("shape_boundary")))
        tab = shape_table(m)
        keep = [np.ascontiguousarray(tab.start, np.int32), np.ascontiguousarray(tab.ids if len(tab.ids) else
                                                                                np.zeros(1, np.int32), np.int32),
                np.ascontiguousarray(tab.xform[:, :3], np.float32), np.ascontiguousarray(tab.scale, np.float32),
                np.ascontiguousarray(tab.radius, np.float32), np.ascontiguousarray(tab.mu, np.float32),
                np.ascontiguousarray(tab.geo if tab.count else np.full(1, 7), np.int32),
                np.ascontiguousarray(tab.xform[:, 3:7] if tab.count else np.array([[0.0, 0.0, 0.0, 1.0]]), np.float32)]
        self._shape_keep = keep
        self.L.orc_set_shapes(self.h, tab.count, _p(keep[0], C.c_int), _p(keep[1], C.c_int), _p(keep[2], C.c_float),
                              _p(keep[3], C.c_float), _p(keep[4], C.c_float), _p(keep[5], C.c_float),
                              float(tab.thinnest), _p(keep[6], C.c_int), _p(keep[7], C.c_float))

    def shape_sdf(self, sh: int, p) -> tuple[float, np.ndarray]:
        """(phi, outward unit gradient) of shape ``sh`` at shape-local point ``p``."""
        x = np.ascontiguousarray(p, np.float64)
        out = np.zeros(4, np.float64)
        self.L.orc_shape_sdf(self.h, int(sh), x.ctypes.data_as(C.POINTER(C.c_double)),
                             out.ctypes.data_as(C.POINTER(C.c_double)))
        return float(out[0]), out[1:].copy()

    def __del__(self):
        if getattr(self, "h", None):
            self.L.orc_destroy(self.h)
            self.h = None

    def set_state(self, q, qd):
        q = np.ascontiguousarray(q, np.float32).reshape(-1)
        qd = np.ascontiguousarray(qd, np.float32).reshape(-1)
        self.L.orc_set_state(self.h, _p(q, C.c_float), _p(qd, C.c_float))

    def set_velocity(self, idx, v):
        """Velocities of the particles ``idx`` (kinematic walls), keeping the rest of the state's precision."""
        idx = np.ascontiguousarray(idx, np.int32)
        v = np.ascontiguousarray(v, np.float32).reshape(-1)
        self.L.orc_set_velocity(self.h, len(idx), _p(idx, C.c_int), _p(v, C.c_float))

    def state(self):
        q = np.zeros((self.n, 3), np.float32)
        qd = np.zeros((self.n, 3), np.float32)
        self.L.orc_get_state(self.h, _p(q, C.c_float), _p(qd, C.c_float))
        return q, qd

    def state64(self):
        q = np.zeros((self.n, 3), np.float64)
        qd = np.zeros((self.n, 3), np.float64)
        self.L.orc_get_state_f64(self.h, _p(q, C.c_double), _p(qd, C.c_double))
        return q, qd

    def warm(self):
        kv = np.zeros(self.n, np.float32)
        kd = np.zeros(self.n, np.float32)
        self.L.orc_get_warm(self.h, _p(kv, C.c_float), _p(kd, C.c_float))
        return kv, kd

    def set_warm(self, kv, kd):
        kv = np.ascontiguousarray(kv, np.float32)
        kd = np.ascontiguousarray(kd, np.float32)
        self.L.orc_set_warm(self.h, _p(kv, C.c_float), _p(kd, C.c_float))

    def flags_phase(self):
        fl = np.zeros(self.n, np.int32)
        ph = np.zeros(self.n, np.int8)
        self.L.orc_get_flags_phase(self.h, _p(fl, C.c_int), ph.ctypes.data)
        return fl, ph

    def active_fluid(self) -> int:
        """Active liquid particles (ACTIVE flag, phase >= 1): the count the throughput metric sums per step."""
        fl, ph = self.flags_phase()
        return int(np.count_nonzero(((fl & 1) != 0) & (ph >= 1)))

    def step(self, dt: float):
        self.L.orc_step(self.h, float(dt))

    def prime(self, dt: float, tol: float = 1.0e-6, max_iterations: int = 2000) -> int:
        """prime.py:52-87 after the caller set kv to the hydrostatic guess x dt; returns the iterations."""
        return int(self.L.orc_prime(self.h, float(dt), float(tol), int(max_iterations)))

    def prepare_density(self):
        self.L.orc_prepare_density(self.h)

    def field(self, name: str) -> np.ndarray:
        three = name.split(":")[0] in ("slot_g", "slot_vb", "slot_n", "acc")
        out = np.zeros((self.n, 3) if three else self.n, np.float32)
        if self.L.orc_get_field(self.h, name.encode(), _p(out, C.c_float)) != 0:
            raise KeyError(name)
        return out

    def slot_on(self) -> np.ndarray:
        """Boundary slots per particle (0: none)."""
        out = np.zeros(self.n, np.int32)
        self.L.orc_get_slot_on(self.h, _p(out, C.c_int))
        return out

    def slot_shapes(self) -> np.ndarray:
        """[n, 4] wall id of each slot (-1 empty; the particle wall's id is the shape count)."""
        out = np.zeros((self.n, 4), np.int32)
        self.L.orc_get_slot_shapes(self.h, _p(out, C.c_int))
        return out

    def lists(self):
        K = self.cfg.neighbor_capacity
        rows = np.zeros((self.n, K), np.int32)
        cnt = np.zeros(self.n, np.int32)
        self.L.orc_get_lists(self.h, _p(rows, C.c_int), _p(cnt, C.c_int))
        return rows, cnt

    def report(self) -> dict:
        W = self.W
        ints = np.zeros((8, W), np.int32)
        fl = np.zeros((5, W), np.float32)
        led = np.zeros((3, W), np.int64)
        self.L.orc_get_report(self.h, _p(ints, C.c_int), _p(fl, C.c_float), _p(led, C.c_int64))
        names_i = ("iters_density", "iters_divergence", "neighbor_overflow", "escaped", "projected", "nonfinite",
                   "emitter_overflow", "swept")
        names_f = ("density_err", "divergence_err", "density_err_max", "max_speed", "density_tol")
        out = {k: ints[i].copy() for i, k in enumerate(names_i)}
        out.update({k: fl[i].copy() for i, k in enumerate(names_f)})
        out.update({"mass_in": led[0].copy(), "mass_out": led[1].copy(), "mass_initial": led[2].copy()})
        act = np.zeros(W, np.int64)
        self.L.orc_active_mass(self.h, _p(act, C.c_int64))
        out["mass_active"] = act
        return out

    def add_emitter(self, world, xform, offsets, velocity, interval, pool):
        xf = np.ascontiguousarray(xform, np.float32)
        off = np.ascontiguousarray(offsets, np.float32).reshape(-1)
        v = np.ascontiguousarray(velocity, np.float32)
        pool = np.ascontiguousarray(pool, np.int32)
        self.L.orc_add_emitter(self.h, int(world), _p(xf, C.c_float), _p(off, C.c_float), len(off) // 3,
                               _p(v, C.c_float), C.c_float(interval), _p(pool, C.c_int), len(pool))

    def add_sink(self, world, xform, half):
        xf = np.ascontiguousarray(xform, np.float32)
        hf = np.ascontiguousarray(half, np.float32)
        self.L.orc_add_sink(self.h, int(world), _p(xf, C.c_float), _p(hf, C.c_float))


# ---------------------------------------------------------------------------------------------- scalar primitives
def kernel_wf(r2: np.ndarray, h: float, sigma: float, kind: int = 0, f64: bool = False):
    dt = np.float64 if f64 else np.float32
    ct = C.c_double if f64 else C.c_float
    r2 = np.ascontiguousarray(r2, dt)
    W = np.zeros_like(r2)
    F = np.zeros_like(r2)
    fn = lib().orc_kernel_wf64 if f64 else lib().orc_kernel_wf
    fn(kind, h, sigma, len(r2), _p(r2, ct), _p(W, ct), _p(F, ct))
    return W, F


def halfspace(d: np.ndarray, h: float, kind: int = 0, f64: bool = False):
    dt = np.float64 if f64 else np.float32
    ct = C.c_double if f64 else C.c_float
    d = np.ascontiguousarray(d, dt)
    psi = np.zeros_like(d)
    dpsi = np.zeros_like(d)
    fn = lib().orc_halfspace64 if f64 else lib().orc_halfspace
    fn(kind, h, len(d), _p(d, ct), _p(psi, ct), _p(dpsi, ct))
    return psi, dpsi


def colour_distance(c: np.ndarray, h: float, kind: int = 0) -> np.ndarray:
    c = np.ascontiguousarray(c, np.float32)
    out = np.zeros_like(c)
    lib().orc_colour_distance(kind, h, len(c), _p(c, C.c_float), _p(out, C.c_float))
    return out


def world_sum(world_start: np.ndarray, values: np.ndarray):
    ws = np.ascontiguousarray(world_start, np.int32)
    v = np.ascontiguousarray(values, np.float32)
    W = len(ws) - 1
    out = np.zeros(W, np.float64)
    mx = np.zeros(W, np.float32)
    lib().orc_world_sum(W, _p(ws, C.c_int), _p(v, C.c_float), _p(out, C.c_double), _p(mx, C.c_float))
    return out, mx
