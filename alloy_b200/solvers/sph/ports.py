# SPDX-License-Identifier: Apache-2.0
"""The SPH port of a ``SolverDFSPH`` (alloy/solvers/sph/ports.py): calls other stages make between its steps.

- ``absorb(state, mask)``: the masked liquid particles leave the liquid and are held for ``emit`` (phase held, on
  their world's stack), booked out of the mass ledger;
- ``emit(state, pos, vel, n)``: per world up to ``n[w]`` held particles become liquid at the given world-frame
  positions and velocities (written into ``state``), booked into the ledger; ``granted[w]`` says how many;
- ``retire(state, mask)``: as ``absorb``, but gone for good (phase retired).

Each call is one kernel launch (``adf_port_take`` / ``adf_port_emit``) with no host work, so it can run inside a
captured graph. The held particles at build (phase ``PHASE_HELD``) are the reservoir; emitters never take them.
``reset`` restores the build-time reservoir. The reference also books the flux energy of what a port moves
(``emitters.flux_add``, for a health monitor's external work); this port keeps the mass ledger only.
"""

from __future__ import annotations

import weakref

import numpy as np
import torch

from ... import _lib
from .config import PHASE_HELD


class SPHPort:
    """The port of one ``SolverDFSPH`` (``solver.port``)."""

    def __init__(self, solver):
        self.solver = weakref.proxy(solver)  # no reference cycle: the solver's device memory goes with the solver
        W = solver.world_count
        n = solver.n
        ph = solver._phase0.cpu().numpy() if n else np.zeros(0, np.int8)
        ws = solver.world_start
        self.reservoir = int(sum(int(np.count_nonzero(ph[ws[w]:ws[w + 1]] == PHASE_HELD)) for w in range(W)))
        mass = solver.model.particle_mass.cpu().numpy() if n else np.zeros(0, np.float32)
        rho = solver.model.sph.rest_density.cpu().numpy() if n else np.zeros(0, np.float32)
        from .solver import sph_phase

        sph = sph_phase(ph) if n else np.zeros(0, bool)
        self.particle_volume = float(np.median(mass[sph] / rho[sph])) if sph.any() else 0.0
        self.rest_density = float(np.median(rho[sph])) if sph.any() else 0.0

    @property
    def world_count(self) -> int:
        return self.solver.world_count

    def _arrays(self) -> dict[str, torch.Tensor]:
        return self.solver._storage()

    @property
    def taken(self) -> torch.Tensor:
        """[W] int32: particles the last ``absorb`` / ``retire`` took per world."""
        return self._arrays()["taken"]

    @property
    def granted(self) -> torch.Tensor:
        """[W] int32: particles the last ``emit`` made liquid per world."""
        return self._arrays()["granted"]

    def _take(self, state, mask, keep: bool) -> None:
        s = self.solver
        if s.n == 0:
            return
        from .solver import _ptr

        m = _ptr(mask, torch.int32, s.n, "mask")
        _lib.check(s._lib.adf_port_take(s._h, _ptr(state.particle_qd, torch.float32, s.n, "particle_qd"), m,
                                        int(keep), s._stream()), "port")

    def absorb(self, state, mask) -> None:
        """Masked liquid particles (``mask [n]`` int32, non-zero) leave the liquid and are held for ``emit``."""
        self._take(state, mask, True)

    def retire(self, state, mask) -> None:
        """Masked liquid particles leave for good (phase retired); ``taken[w]`` counts them."""
        self._take(state, mask, False)

    def emit(self, state, pos, vel, n) -> None:
        """Up to ``n[w]`` held particles per world become liquid at ``pos [W, R, 3]`` with ``vel [W, R, 3]`` (world
        frame, written into ``state``); ``granted[w]`` says how many (fewer when the reservoir is empty)."""
        s = self.solver
        if s.n == 0 or s.world_count == 0:
            return
        from .solver import _ptr

        if pos.shape[:2] != vel.shape[:2] or pos.shape[0] != s.world_count or pos.shape[-1] != 3:
            raise ValueError(f"port emit: pos and vel must be [W={s.world_count}, R, 3], got {tuple(pos.shape)} and "
                             f"{tuple(vel.shape)}")
        R = int(pos.shape[1])
        _lib.check(s._lib.adf_port_emit(s._h, _ptr(state.particle_q, torch.float32, s.n, "particle_q"),
                                        _ptr(state.particle_qd, torch.float32, s.n, "particle_qd"),
                                        _ptr(pos, torch.float32, None, "pos"), _ptr(vel, torch.float32, None, "vel"),
                                        R, _ptr(n, torch.int32, s.world_count, "n"), s._stream()), "port emit")

    def state_arrays(self) -> dict[str, torch.Tensor]:
        a = self._arrays()
        return {"sph.port_stack": a["port_stack"], "sph.port_top": a["port_top"],
                "sph.port_absorbed": a["port_absorbed"], "sph.port_emitted": a["port_emitted"],
                "sph.port_retired": a["port_retired"]}

    def counts(self) -> dict[str, np.ndarray]:
        """Host copies per world: held (reservoir now), absorbed, emitted, retired (cumulative)."""
        a = self._arrays()
        return {"held": a["port_top"].cpu().numpy().copy(), "absorbed": a["port_absorbed"].cpu().numpy().copy(),
                "emitted": a["port_emitted"].cpu().numpy().copy(), "retired": a["port_retired"].cpu().numpy().copy()}
