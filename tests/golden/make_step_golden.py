# TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
"""Generate tests/golden/reference_steps.npz: DFSPH steps computed by the reference's OWN kernels and solve driver.

The reference's modules on the liquid step's path (alloy/solvers/sph: kernels, pressure, reduce, neighbors,
particle_walls, boundary_slots, boundary, soft_walls, integrate, krylov, solve_driver, config) are loaded from the
checkout and run on the CPU under ``refrun``'s float32 warp stand-in. ``RefStep.step`` performs
``SolverDFSPH.step`` (solver.py:218-268) for a model whose walls are particle walls and that has no SDF shapes, soft
faces, bodies, surface tension, implicit viscosity, ambient pressure or emitters: every launch below is one the
reference makes, with the arguments it passes, in its order; the pressure solves are the reference's own
``PressureSolves._solve`` / ``_jacobi`` (solve_driver.py:121-186), run as its host code with the stand-in's
``capture_while``. The only pieces written here are the object plumbing those methods read from ``self``
(solver.py:127-162 allocations), ``NeighborLists.build`` (neighbors.py:241-269: groups, grid, local rows) and
``WorldStats``'s three recorders (runtime.py:111-124), each a line or two of host code around the reference's
kernels. Particle-wall reactions (``ParticleWalls.accumulate``) are skipped: they write the walls' impulse
counters only.

Cases (``CASES``), each a single world of one layer of boundary particles around a jittered liquid block in its
corner, dt 1 ms, the plain settings (resting-jitter rule off, XSPH 0.01):
- ``dam_break_jacobi``: 6 x 6 x 8 particles at 0.02 m (the corner block of the 20 x 20 x 20 single-world dam
  break) in a 0.2 x 0.2 x 0.24 m box, relaxed Jacobi, tolerances 1e-3;
- ``dam_break_cg``: the same with the projected CG solve (krylov.py, the reference's default);
- ``column_jacobi_tight``: a 4 x 4 x 16 column in a 0.08 x 0.08 x 0.4 m box at tolerances 1e-4, which takes
  several Jacobi iterations per solve;
- ``tank_impacts``: the block thrown into a corner of that tank and eight lone particles, four of them beyond the
  CFL step (testing.tank_impacts): projections onto the walls, lone-particle limits and friction, the sweep;
- ``tank_sdf_jacobi`` / ``tank_sdf_cg``: the dam-break block in the reference's own open box tank of five box shapes,
  walls h thick (build.py:113-137), seen through their signed distance fields: up to four boundary slots per
  particle at the tank's edges and corners, the pressure and projection passes of the shape branch, wall friction.
Recorded per step: the start state and warm starts, the neighbour rows, the particle-wall slot, density ratio,
factor, effective neighbour count, per-solve iterations and mean errors, the warm starts each solve stores and the
end state. One file per case: tests/golden/reference_steps_<case>.npz.

Usage: python tests/golden/make_step_golden.py <alloy checkout> [case ...]
"""

from __future__ import annotations

import sys
import time
from pathlib import Path
from types import SimpleNamespace

import numpy as np

HERE = Path(__file__).resolve().parent
for p in (HERE, HERE.parents[1]):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

import refrun  # noqa: E402

_BLOCK = {"counts": (6, 6, 8), "box": (0.2, 0.2, 0.24), "spacing": 0.02, "jitter": 0.01, "seed": 0, "dt": 1.0e-3}
_COLUMN = {"counts": (4, 4, 16), "box": (0.08, 0.08, 0.4), "spacing": 0.02, "jitter": 0.01, "seed": 1, "dt": 1.0e-3}
CASES = {
    "dam_break_jacobi": {"scene": _BLOCK, "config": {"pressure_solver": "jacobi"}, "steps": 10},
    "dam_break_cg": {"scene": _BLOCK, "config": {"pressure_solver": "cg"}, "steps": 10},
    "column_jacobi_tight": {"scene": _COLUMN, "config": {"pressure_solver": "jacobi", "max_density_error": 1.0e-4,
                                                         "max_divergence_error": 1.0e-4}, "steps": 10},
    "tank_sdf_jacobi": {"scene": {**_BLOCK, "walls": "sdf", "open_top": True}, "config": {"pressure_solver": "jacobi"},
                        "steps": 12},
    "tank_sdf_cg": {"scene": {**_BLOCK, "walls": "sdf", "open_top": True}, "config": {"pressure_solver": "cg"},
                    "steps": 12},
    "tank_impacts": {"scene": {"dt": 1.0e-3}, "builder": "tank_impacts", "config": {"pressure_solver": "jacobi"},
                     "steps": 10},
}
PROJECT_EPS = 1.0e-3  # solver.py:483


def out_path(case: str) -> Path:
    return HERE / f"reference_steps_{case}.npz"


def scene_arrays(case: str) -> tuple[dict, object]:
    """The case's host arrays (this package's builders; the test builds the same scene the same way)."""
    from alloy_b200.solvers.sph.testing import dam_break

    c = CASES[case]
    if c.get("builder") == "tank_impacts":
        from alloy_b200.solvers.sph.testing import tank_impacts

        sc = tank_impacts(device="cpu", dt=c["scene"]["dt"], **c["config"])
    else:
        sc = dam_break(device="cpu", **c["scene"], **c["config"])
    return sc.model.host(), sc.config


class RefStep:
    """The reference's step over host arrays (module doc)."""

    def __init__(self, R, a: dict, cfg):
        wp, pr = R.wp, R.pressure
        self.R, self.wp, self.pr = R, wp, pr
        self.config = cfg
        n, W = len(a["mass"]), len(a["world_start"]) - 1
        self.layout = SimpleNamespace(n=n, world_count=W)
        self.device = "cpu"
        self._h, self._kind = float(cfg.h), int(cfg.kernel_id)
        self._n_full = R.config.full_neighbor_count(cfg)
        self._tot_min = cfg.diagonal_floor * R.kernels.lattice_diagonal(cfg.spacing, cfg.h, cfg.kernel)
        ws = np.asarray(a["world_start"], np.int32)
        # model and state arrays
        self.q = wp.array(a["q"], dtype=wp.vec3)
        self.qd = wp.array(a["qd"], dtype=wp.vec3)
        self.mass = wp.array(a["mass"], dtype=wp.float32)
        self.rho0 = wp.array(a["rest_density"], dtype=wp.float32)
        self.flags = wp.array(a["flags"], dtype=wp.int32)
        self.phase = wp.array(a["phase"], dtype=wp.int8)
        self.world = wp.array(a["world"], dtype=wp.int32)
        self.model = SimpleNamespace(gravity=wp.array(a["gravity"], dtype=wp.vec3))
        # neighbour lists (neighbors.py:205-239, world-local rows)
        K = int(cfg.neighbor_capacity)
        self.K = K
        self.nbr = wp.zeros((K, n), dtype=wp.uint16)
        self.hi = wp.zeros((1, 1), dtype=wp.uint8)
        self.base = wp.array(ws[:-1], dtype=wp.int32)
        self.count = wp.zeros(n, dtype=wp.int32)
        self.group = wp.zeros(n, dtype=wp.int32)
        self.overflow = wp.zeros(max(W, 1), dtype=wp.int32)
        # solver.py:127-162
        self._slots = R.boundary.BoundarySlots.allocate(n, "cpu")
        self._slot_impulse = wp.zeros((n, 4), dtype=wp.vec3)
        self._w = pr.SolveArrays.allocate(n, "cpu")
        self._kv, self._kd = wp.zeros(n, dtype=wp.float32), wp.zeros(n, dtype=wp.float32)
        self._vtmp = wp.zeros(n, dtype=wp.vec3)
        self._lower = wp.zeros(n, dtype=wp.float32)
        self._reducer = R.reduce.WorldReducer(ws, "cpu")
        self._n_active = wp.zeros(W, dtype=wp.float64)
        self._err_sum = wp.zeros(W, dtype=wp.float64)
        self._converged = wp.zeros(W, dtype=wp.int32)
        self._iters = wp.zeros(W, dtype=wp.int32)
        self._err_mean = wp.zeros(W, dtype=wp.float32)
        self._err_max = wp.zeros(W, dtype=wp.float32)
        self._n_unconv = wp.zeros(1, dtype=wp.int32)
        self._ctl = R.krylov.SolveControl(self._converged, self._iters, self._err_mean, self._err_max, self._n_unconv,
                                          self._n_active)
        self._cg = (R.krylov.ProjectedCG(n, W, "cpu", self._reducer, self._w, self._lower, self._ctl)
                    if cfg.pressure_solver == "cg" else None)  # solver.py:158-159 (uniform masses here)
        self._ambient = None
        self._empty_vec3 = wp.zeros(1, dtype=wp.vec3)
        # shapes: none, soft faces: none, particle walls: the PROXY particles (layout.py:207-246,
        # particle_walls.py:224-247, coupling_hooks.py:156-168)
        sh = R.boundary.ShapeArrays()
        z32 = lambda: wp.zeros(1, dtype=wp.int32)  # noqa: E731
        S = int(len(a.get("shape_type", ())))
        self.S = S
        if S:  # the model's shapes (layout.py:207-230): Newton's box radius |half extents| (geometry/utils.py:83-84)
            start, ids = R.boundary.world_shape_table(a["shape_world"], a["shape_flags"], a["shape_type"], W,
                                                      a["shape_boundary"] == 3)
            sh.start = wp.array(start, dtype=wp.int32)
            sh.ids = wp.array(ids if len(ids) else np.zeros(1, np.int32), dtype=wp.int32)
            sh.geo = wp.array(a["shape_type"], dtype=wp.int32)
            sh.scale = wp.array(a["shape_scale"], dtype=wp.vec3)
            sh.xform = refrun.TfArray(a["shape_transform"])
            sh.body = wp.array(a["shape_body"], dtype=wp.int32)
            sh.radius = wp.array(np.linalg.norm(np.abs(a["shape_scale"].astype(np.float64)), axis=1)
                                 .astype(np.float32), dtype=wp.float32)
            sh.mu = wp.array(a["shape_mu"], dtype=wp.float32)
            sh.sdf_index = wp.full(S, -1, dtype=wp.int32)
            sh.bvh = wp.zeros(S, dtype=wp.int32)
            sh.mesh = wp.zeros(S, dtype=wp.uint64)
            self.thinnest = float(2.0 * a["shape_scale"][np.unique(ids)].astype(np.float64).min()) if len(ids) \
                else float("inf")  # layout.py:135-148 (boxes)
        else:
            sh.start, sh.ids = wp.zeros(W + 1, dtype=wp.int32), z32()
            sh.geo, sh.body, sh.sdf_index, sh.bvh = z32(), z32(), z32(), z32()
            sh.mesh, sh.scale, sh.radius, sh.mu = (wp.zeros(1, dtype=wp.uint64), wp.zeros(1, dtype=wp.vec3),
                                                   wp.zeros(1, dtype=wp.float32), wp.zeros(1, dtype=wp.float32))
            sh.xform = refrun.TfArray(np.array([[0, 0, 0, 0, 0, 0, 1]], np.float32))
            self.thinnest = float("inf")
        sh.tex = None
        sh.curvature = int(cfg.boundary_curvature_order)
        off, amp = R.kernels.boundary_fit(cfg.spacing, cfg.h, cfg.kernel)
        sh.offset, sh.amplitude = np.float32(off), np.float32(amp)
        sh.taper0, sh.taper1 = np.float32(0.5 * cfg.spacing), np.float32(1.5 * cfg.spacing)
        sh.reach = np.float32(1.5 * cfg.spacing)
        sh.bvh_dist = np.float32(2.0 * cfg.h)
        sh.soft = R.soft_walls.empty_soft(S, "cpu")  # soft faces would follow the shapes; none here
        pw = R.particle_walls.empty_walls(S, cfg.h, cfg.kernel_id, "cpu")  # the particle wall's id: soft.base + 0
        vid = np.flatnonzero((a["flags"] & 2) != 0)
        r64 = a["radius"].astype(np.float64)
        vol, mask = np.zeros(n, np.float32), np.zeros(n, np.int32)
        vol[vid], mask[vid] = (8.0 * r64[vid] ** 3).astype(np.float32), 1
        pw.count, pw.vol, pw.h, pw.kind = int(vid.size), wp.array(vol, dtype=wp.float32), np.float32(cfg.h), self._kind
        sh.pw, sh.friction = pw, int(bool(cfg.wall_friction))
        self.sa = sh
        self.shapes = SimpleNamespace(arrays=sh)  # the ShapeTable the solve driver reads (layout.py:207-246)
        self.vid = wp.array(vid.astype(np.int32), dtype=wp.int32)
        self.wall_mask = wp.array(mask, dtype=wp.int32)
        self.bq, self.bqd, self.com = wp.zeros(1, dtype=wp.transform), wp.zeros(1, dtype=wp.spatial_vector), \
            wp.zeros(1, dtype=wp.vec3)
        self.projected = wp.zeros(W, dtype=wp.int32)
        self.swept = wp.zeros(W, dtype=wp.int32)
        self.shape_work = wp.zeros(1, dtype=wp.int64)
        self.max_speed = wp.zeros(W, dtype=wp.float32)
        self.nonfinite = wp.zeros(W, dtype=wp.int32)
        self.stats = _Stats(R, W)
        self.solver = _Solves(self)  # the reference's PressureSolves mixin over this object's arrays
        self.solver._alloc_tolerance()

    # ------------------------------------------------------------------------------------------------------ the step
    def particles(self):
        p = self.pr.Particles()
        p.q, p.qd, p.mass, p.rho0, p.flags = self.q, self.qd, self.mass, self.rho0, self.flags
        p.phase, p.world = self.phase, self.world
        p.nbr, p.nbr_hi, p.nbr_wide, p.wstart, p.count = self.nbr, self.hi, 0, self.base, self.count
        return p

    def slot_struct(self):
        s = self.pr.Slots()
        sl = self._slots
        s.shape, s.psi, s.gpsi, s.vb, s.reg = sl.shape, sl.psi, sl.gpsi, sl.vb, self._w.reg
        return s

    def launch(self, kernel, inputs, dim=None):
        self.wp.launch(kernel, dim=self.layout.n if dim is None else dim, inputs=inputs)

    def build_lists(self):
        """NeighborLists.build (neighbors.py:241-269) with the particle walls set (set_walls, has_wall 1)."""
        R, n = self.R, self.layout.n
        self.launch(R.neighbors._set_groups_kernel, [self.flags, self.phase, self.world, self.wall_mask, 1, self.group])
        self.grid = refrun.Grid(self.q, self._h, np.asarray(self.group))
        self.launch(R.neighbors._build_local_kernel, [self.grid, self.q, self.group, self.base, self._h, self.K,
                                                      self.nbr, self.hi, 0, self.count, self.overflow], dim=n)

    def step(self, dt: float, rec: dict) -> None:
        R, pr, cfg, w = self.R, self.pr, self.config, self._w
        p = self.particles()
        self._slot_impulse.zero_()
        self.build_lists()
        cnt = np.asarray(self.count).copy()
        rows = np.full((self.layout.n, self.K), -1, np.int32)
        for i in np.flatnonzero(cnt):
            rows[i, :cnt[i]] = np.asarray(self.nbr)[:cnt[i], i].astype(np.int32) + int(self.base[0])
        rec["count"], rec["rows"] = cnt, rows
        pw = self.sa.pw
        pw.x, pw.v, pw.grid = self.q, self.qd, self.grid  # ParticleWalls.begin
        R.boundary.compute_slots(self.q, self.flags, self.phase, self.world, self.sa, self.bq, self.bqd,
                                 self.com, self._h, self._kind, self._slots, "cpu")
        sl = self.slot_struct()
        rec["slot_shape"] = self._slots.shape.numpy()[:, 0].copy()
        rec["slot_psi"] = self._slots.psi.numpy()[:, 0].copy()
        rec["slot_phi"] = self._slots.phi.numpy()[:, 0].copy()
        rec["slot_g"] = self._slots.gpsi.numpy()[:, 0].copy()
        rec["slot_shapes"] = self._slots.shape.numpy().copy()  # [n, 4]
        rec["slot_psi4"] = self._slots.psi.numpy().copy()
        rec["slot_g4"] = self._slots.gpsi.numpy().copy()
        self.launch(pr.density_alpha_kernel, [p, sl, self._h, self._kind, self._n_full, self._tot_min, w.ratio,
                                              w.alpha, w.neff, w.active])
        rec["ratio"], rec["alpha"], rec["neff"] = (np.asarray(w.ratio).copy(), np.asarray(w.alpha).copy(),
                                                   np.asarray(w.neff).copy())
        rec["reg"] = np.asarray(w.reg).copy()
        self._reducer.sum(w.active, self._n_active)
        self.solver._flow_speed(p)
        if cfg.divergence_solve:
            self.solver._solve(p, sl, pr.MODE_DIVERGENCE, dt)
        rec["kv"] = np.asarray(self._kv).copy()
        xsph = cfg.xsph_c if cfg.viscosity in ("xsph", "auto") else 0.0  # resolve_viscosity: xsph below 1e-2 Pa s
        self.launch(R.integrate.nonpressure_kernel, [p, self._h, self._kind, dt, self.model.gravity,
                                                     self._empty_vec3, 0, w.ratio, xsph, self._vtmp])
        self.wp.copy(p.qd, self._vtmp, count=self.layout.n)
        self.solver._solve(p, sl, pr.MODE_DENSITY, dt)
        rec["kd"] = np.asarray(self._kd).copy()
        self.launch(R.integrate.advect_kernel, [p, dt])
        self.wp.launch(R.particle_walls._advance_kernel, dim=int(self.vid.shape[0]),
                       inputs=[self.vid, dt, self.q, self.qd])  # ParticleWalls.advance
        s_ = self._slots
        r = float(cfg.particle_radius)
        sweep = R.integrate.sweep_length(self._h, self.thinnest)
        self.launch(R.integrate.project_kernel, [p, s_.shape, s_.phi, s_.xbl, s_.nbl, s_.face, s_.vb, self.sa,
                                                 self.bq, self.bqd, self.com, PROJECT_EPS * r, self.projected,
                                                 self.bq, dt, sweep, r, self.swept, self.shape_work])
        self.max_speed.zero_()
        self.launch(R.integrate.speed_kernel, [p, self.max_speed, self.nonfinite])
        st = self.stats
        rec["iters_div"], rec["iters_den"] = st.iters_div.copy(), st.iters_den.copy()
        rec["div_err"], rec["den_err"], rec["den_err_max"] = st.div_err.copy(), st.den_err.copy(), st.den_err_max.copy()
        rec["max_speed"] = np.asarray(self.max_speed).copy()
        rec["projected"] = np.asarray(self.projected).copy()
        rec["swept"] = np.asarray(self.swept).copy()


def _Solves(host: RefStep):
    """An instance of the reference's ``PressureSolves`` mixin whose attributes are ``host``'s arrays."""
    cls = type("Solves", (host.R.solve_driver.PressureSolves,), {})
    s = cls()
    for k in ("config", "layout", "device", "model", "_h", "_kind", "_w", "_kv", "_kd", "_lower", "_reducer",
              "_n_active", "_err_sum", "_converged", "_iters", "_err_mean", "_err_max", "_n_unconv", "_ctl", "_cg",
              "_ambient", "_slot_impulse", "stats", "shapes"):
        setattr(s, k, getattr(host, k))
    s._launch = host.launch
    return s


class _Stats:
    """WorldStats' solve recorders (runtime.py:111-124): copies of the per-world iterations and mean errors, the
    reference's max_err_kernel and scale_kernel."""

    def __init__(self, R, W):
        self.R, self.W = R, W
        wp = R.wp
        self.den_err_max = wp.zeros(W, dtype=wp.float32)
        self.den_tol = wp.zeros(W, dtype=wp.float32)
        self.iters_div = self.iters_den = np.zeros(W, np.int32)
        self.div_err = self.den_err = np.zeros(W, np.float32)

    def record_solve(self, divergence, iters, err_mean):
        if divergence:
            self.iters_div, self.div_err = np.asarray(iters).copy(), np.asarray(err_mean).copy()
        else:
            self.iters_den, self.den_err = np.asarray(iters).copy(), np.asarray(err_mean).copy()

    def record_density_tolerance(self, scale, tol):
        self.R.wp.launch(self.R.pressure.scale_kernel, dim=self.W, inputs=[scale, float(tol), self.den_tol])

    def record_max_density_error(self, p, err):
        self.den_err_max.zero_()
        self.R.wp.launch(self.R.pressure.max_err_kernel, dim=err.shape[0], inputs=[p, err, self.den_err_max])


def run_case(root: Path, case: str) -> None:
    c = CASES[case]
    a, ours = scene_arrays(case)  # before the stand-in replaces ``warp`` and ``alloy`` in sys.modules
    R = refrun.load_reference(root)
    kw = {"pressure_solver": "jacobi", "rest_jitter_speed": None, "xsph_c": 0.01, "viscosity": "xsph", **c["config"]}
    cfg = R.config.DFSPHConfig(particle_radius=ours.particle_radius, **kw)
    cfg.validate()
    m_ref = np.float32(R.config.particle_mass(cfg, 1000.0))
    fluid = a["phase"] >= 1
    if not np.all(a["mass"][fluid] == m_ref):
        raise AssertionError(f"liquid mass {a['mass'][fluid][0]!r} differs from the reference's {m_ref!r}")
    ref = RefStep(R, a, cfg)
    out: dict[str, list] = {}
    t0 = time.time()
    dt = c["scene"]["dt"]
    for s in range(c["steps"]):
        rec = {"q0": ref.q.numpy().copy(), "qd0": ref.qd.numpy().copy(), "kv0": np.asarray(ref._kv).copy(),
               "kd0": np.asarray(ref._kd).copy()}
        ref.step(dt, rec)
        rec["q1"], rec["qd1"] = ref.q.numpy().copy(), ref.qd.numpy().copy()
        for k, v in rec.items():
            out.setdefault(k, []).append(v)
        print(f"{case} step {s}: iterations div {rec['iters_div'][0]} den {rec['iters_den'][0]}, density error "
              f"{rec['den_err'][0]:.3e}, {time.time() - t0:.0f} s", flush=True)
    arrays = {k: np.stack(v) for k, v in out.items()}
    kmax = max(int(arrays["count"].max()), 1)
    arrays["rows"] = arrays["rows"][:, :, :kmax].astype(np.int16)  # ids < 32,768; -1 past the row's count
    np.savez_compressed(out_path(case), **arrays, scene=np.array(repr(c)), steps=np.int32(c["steps"]),
                        source=np.array("alloy/solvers/sph kernels under tests/golden/refrun.py (float32 warp "
                                        "stand-in)"))
    print(f"wrote {out_path(case)}")


def main(root: Path, cases: list[str]) -> None:
    for case in cases:  # one process per case: the stand-in owns sys.modules' warp and alloy entries
        import subprocess

        subprocess.run([sys.executable, __file__, "--case", case, str(root)], check=True)


if __name__ == "__main__":
    if len(sys.argv) >= 4 and sys.argv[1] == "--case":
        run_case(Path(sys.argv[3]), sys.argv[2])
    elif len(sys.argv) >= 2:
        main(Path(sys.argv[1]), sys.argv[2:] or list(CASES))
    else:
        raise SystemExit(__doc__)
