# SPDX-License-Identifier: Apache-2.0
"""Learned warm start of the two pressure solves: a per-particle network 16 -> 64 -> 64 -> 2 (SiLU, BF16 weights,
FP32 accumulation) run and trained by the tensor-core kernels of ``liballoy_dfsph.so`` (``adf_mlp_*``).

The reference warm-starts each solve from the previous step's kappa scaled by a constant (0.5 for the divergence
solve, 0.9 for the density solve; ``alloy/solvers/sph/pressure.py:214-261``). The network predicts both solves'
starting kappa from the particle's state at the start of the step instead. The solver keeps judging every step: the
first Jacobi sweep runs from both starts and each world keeps the one with the smaller error (the plain start when
the learned one does worse), and every world still iterates to the same tolerance, so the network changes the
iteration count, never the convergence test.

Features (raw values, written by the solver at the start of each step's first solve, in this order):
  0 ratio - 1          density deviation rho/rho0 - 1
  1 n_eff / n_full     neighbour count relative to a full lattice neighbourhood
  2 dt * rate          density change over the step from the velocity divergence
  3 kappa_v (prev)     previous step's divergence warm start (kappa dt)
  4 kappa_d (prev)     previous step's density warm start (kappa dt^2)
  5 alpha              DFSPH factor
  6 |v|                speed
  7 phi                distance to the boundary-particle wall (the support radius when there is none)
  8 psi                boundary volume term
  9 ratio + dt rate - 1 predicted density error (the density solve's source)
 10 plain kappa_v      the reference's divergence start, 0.5 min(kappa_v, 0.5)
 11 plain kappa_d      the reference's density start, 0.9 min(kappa_d, 2.5e-4)
 12 v_z                vertical velocity
 13 |grad psi|         boundary gradient magnitude
 14 (ratio - 1) alpha
 15 dt rate alpha
Targets: corrections to the plain starts, in the dt-free units the solver stores: the converged kappa dt of the
divergence solve minus feature 10, and the converged kappa dt^2 of the density solve minus feature 11. A network
that outputs zero therefore reproduces the reference's start exactly.
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from ... import _lib

N_FEATURES = _lib.MLP_FEATURES
N_PARAMS = _lib.MLP_PARAMS
HIDDEN = 64
OFF_W1, OFF_B1 = 0, 64 * 16
OFF_W2 = OFF_B1 + 64
OFF_B2 = OFF_W2 + 64 * 64
OFF_W3 = OFF_B2 + 64
OFF_B3 = OFF_W3 + 2 * 64


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initial parameters in the packed order (W1, b1, W2, b2, W3, b3)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(N_PARAMS, np.float32)
    p[OFF_W1:OFF_B1] = rng.normal(0.0, np.sqrt(2.0 / 16), 64 * 16)
    p[OFF_W2:OFF_B2] = rng.normal(0.0, np.sqrt(2.0 / 64), 64 * 64)
    p[OFF_W3:OFF_B3] = rng.normal(0.0, np.sqrt(1.0 / 64), 2 * 64)
    return p


def unpack(p: np.ndarray) -> dict[str, np.ndarray]:
    p = np.asarray(p, np.float32)
    return {"w1": p[OFF_W1:OFF_B1].reshape(64, 16), "b1": p[OFF_B1:OFF_W2], "w2": p[OFF_W2:OFF_B2].reshape(64, 64),
            "b2": p[OFF_B2:OFF_W3], "w3": p[OFF_W3:OFF_B3].reshape(2, 64), "b3": p[OFF_B3:]}


def _ptr(t) -> int:
    return t.data_ptr() if hasattr(t, "data_ptr") else int(t.__cuda_array_interface__["data"][0])


class Network:
    """The device-resident network (``adf_mlp``): inference, gradients and Adam steps on the tensor cores."""

    def __init__(self, params: np.ndarray | None = None, device: int = 0):
        L = _lib.lib()
        p = np.ascontiguousarray(init_params() if params is None else params, dtype=np.float32)
        if p.size != N_PARAMS:
            raise ValueError(f"expected {N_PARAMS} parameters, got {p.size}")
        h = C.c_void_p()
        _lib.check(L.adf_mlp_create(p.ctypes.data, int(device), C.byref(h)), "adf_mlp_create")
        self._h = h
        self.device = int(device)

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            _lib.lib().adf_mlp_destroy(h)
            self._h = None

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def params(self) -> np.ndarray:
        out = np.empty(N_PARAMS, np.float32)
        _lib.check(_lib.lib().adf_mlp_get_params(self._h, out.ctypes.data), "adf_mlp_get_params")
        return out

    def set_params(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        _lib.check(_lib.lib().adf_mlp_set_params(self._h, p.ctypes.data), "adf_mlp_set_params")

    def forward(self, x, y=None, stream: int = 0):
        """y[n][2] = network(x[n][16]) for float32 CUDA tensors (normalised units)."""
        import torch

        n = int(x.shape[0])
        if y is None:
            y = torch.empty((n, 2), dtype=torch.float32, device=x.device)
        _lib.check(_lib.lib().adf_mlp_forward(self._h, _ptr(x), n, _ptr(y), stream or None), "adf_mlp_forward")
        return y

    def gradient(self, x, t, idx, stream: int = 0) -> tuple[np.ndarray, float]:
        g = np.empty(N_PARAMS, np.float32)
        loss = np.empty(1, np.float32)
        _lib.check(_lib.lib().adf_mlp_gradient(self._h, _ptr(x), _ptr(t), _ptr(idx), int(idx.shape[0]),
                                               g.ctypes.data, loss.ctypes.data, stream or None), "adf_mlp_gradient")
        return g, float(loss[0])

    def train_step(self, x, t, idx, lr: float, want_loss: bool = False, stream: int = 0) -> float | None:
        loss = np.empty(1, np.float32)
        _lib.check(_lib.lib().adf_mlp_train_step(self._h, _ptr(x), _ptr(t), _ptr(idx), int(idx.shape[0]), float(lr),
                                                 loss.ctypes.data if want_loss else None, stream or None),
                   "adf_mlp_train_step")
        return float(loss[0]) if want_loss else None

    def status(self) -> None:
        _lib.check(_lib.lib().adf_mlp_status(self._h), "adf_mlp_status")


@dataclass
class WarmModel:
    """A trained network with its feature and target statistics (x_n = (x - f_mean) / f_std, y = t_mean + t_std y_n)."""

    params: np.ndarray
    f_mean: np.ndarray
    f_std: np.ndarray
    t_mean: np.ndarray
    t_std: np.ndarray

    def norm_vector(self) -> np.ndarray:
        """fmu[16], finv[16], tmu[2], tsig[2] as the solver takes them."""
        return np.concatenate([self.f_mean, 1.0 / self.f_std, self.t_mean, self.t_std]).astype(np.float32)

    def save(self, path) -> None:
        np.savez(path, params=self.params, f_mean=self.f_mean, f_std=self.f_std, t_mean=self.t_mean, t_std=self.t_std)

    @classmethod
    def load(cls, path) -> WarmModel:
        d = np.load(path)
        return cls(*(np.asarray(d[k], np.float32) for k in ("params", "f_mean", "f_std", "t_mean", "t_std")))


DEFAULT_MODEL = __import__("pathlib").Path(__file__).resolve().parent / "data" / "warm_model.npz"


def default_model() -> WarmModel:
    """The network shipped with the package: trained by ``python -m alloy_b200.solvers.sph.warmstart --out
    alloy_b200/solvers/sph/data/warm_model.npz`` (2,000,000 pairs from a seed-1 run of 256 worlds of the pour, moving
    bowls and spouts, 200 steps, Adam at 1e-3, batch 65,536, 20 epochs). Trained on the pour alone, it lowers the
    iterations more on every measured workload than networks trained on the dam break and the batched worlds, or on
    all three."""
    return WarmModel.load(DEFAULT_MODEL)


def statistics(x: np.ndarray, floor: float = 1e-12) -> tuple[np.ndarray, np.ndarray]:
    """Per-column mean and deviation (float64 accumulation); constant columns get deviation 1."""
    x = np.asarray(x, np.float64)
    mu = x.mean(axis=0)
    sd = x.std(axis=0)
    sd = np.where(sd > floor, sd, 1.0)
    return mu.astype(np.float32), sd.astype(np.float32)


def train(features: np.ndarray, targets: np.ndarray, *, epochs: int = 20, batch: int = 65536, lr: float = 1e-3,
          seed: int = 0, device: int = 0, log=None) -> WarmModel:
    """Adam on the normalised pairs (feature rows [N][16], targets [N][2]); batches drawn from a seeded permutation
    per epoch. Returns the trained model with its statistics."""
    import torch

    f_mean, f_std = statistics(features)
    t_mean, t_std = statistics(targets)
    dev = torch.device("cuda", device)
    x = torch.from_numpy(((features - f_mean) / f_std).astype(np.float32)).to(dev)
    t = torch.from_numpy(((targets - t_mean) / t_std).astype(np.float32)).to(dev)
    net = Network(init_params(seed), device)
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    n = x.shape[0]
    for ep in range(epochs):
        perm = torch.randperm(n, generator=gen, device=dev).to(torch.int32)
        losses = []
        for b in range(0, n, batch):
            idx = perm[b:b + batch].contiguous()
            losses.append(net.train_step(x, t, idx, lr, want_loss=log is not None))
        if log is not None:
            log(f"epoch {ep}: loss {np.mean(losses):.4e}")
    net.status()
    return WarmModel(net.params(), f_mean, f_std, t_mean, t_std)


def collect_pairs(solver, state_a, state_b, dt: float, steps: int, every: int = 1, per_record: int | None = None,
                  seed: int = 0, drive=None):
    """Run ``steps`` steps of ``solver`` (the plain start unless a model is set) and gather (features, corrections of
    the converged warm starts to the plain starts) of the liquid particles every ``every`` steps; ``per_record`` rows
    drawn without replacement per record (all when None); ``drive(state, k)`` before step k moves the scene's
    kinematic walls. Returns float32 arrays [N][16] and [N][2] and the final (state_a, state_b)."""
    import torch

    solver.record_features(True)
    rng = np.random.default_rng(seed)
    feats, targs = [], []
    model = solver.model
    for k in range(steps):
        live = None
        if k % every == 0:
            live = ((model.particle_flags & 1) != 0) & (model.sph.phase >= 1)
        if drive is not None:
            drive(state_a, k)
        solver.step(state_a, state_b, None, None, dt)
        state_a, state_b = state_b, state_a
        if live is None:
            continue
        idx = torch.nonzero(live).squeeze(1)
        if per_record is not None and idx.numel() > per_record:
            pick = rng.choice(idx.numel(), per_record, replace=False)
            idx = idx[torch.from_numpy(np.sort(pick)).to(idx.device)]
        f = solver.warm_features()[idx]
        arr = solver.alloy_state_arrays()
        t = torch.stack([arr["sph.kappa_v"][idx] - f[:, 10], arr["sph.kappa_d"][idx] - f[:, 11]], dim=1)
        feats.append(f.cpu().numpy())
        targs.append(t.cpu().numpy())
    solver.record_features(False)
    return np.concatenate(feats).astype(np.float32), np.concatenate(targs).astype(np.float32), state_a, state_b


SOURCES = ("large_dam_break", "batched_worlds", "pour_bowls")


def generate_pairs(device=None, pairs: int = 2_000_000, seed: int = 1, steps: int = 200, log=None,
                   sources=("pour_bowls",)):
    """Training pairs from seeded runs of plain workloads (an equal share each): the 1,048,576-particle dam break, the
    256 batched worlds with spouts, and 256 worlds of the pour (moving bowls, spouts), ``steps`` steps each, a record
    every 4 steps."""
    import torch

    from .solver import SolverDFSPH, layer_offsets
    from .testing import batched_worlds, large_dam_break, pour_bowls

    dev = device or torch.device("cuda", 0)
    every = 4
    per = int(np.ceil(pairs / len(sources) / (steps // every)))
    out_f, out_t = [], []
    makers = {"large_dam_break": large_dam_break, "batched_worlds": batched_worlds,
              "pour_bowls": lambda device, seed: pour_bowls(worlds=256, device=device, seed=seed)}
    for name in sources:
        sc = makers[name](device=dev, seed=seed)
        sol = SolverDFSPH(sc.model, sc.config)
        host = sc.model.host()
        specs = []
        for e in sc.emitters:
            i0 = int(host["world_start"][e["world"]])
            vol = float(host["mass"][i0]) / float(host["rest_density"][i0])
            offs = layer_offsets(np.asarray(e["half"], np.float64), np.asarray(e["velocity"], np.float64),
                                 sc.config.spacing)
            rate = len(offs) * vol / e.get("layer_every", 10.0 * sc.dt)
            specs.append((e["world"], e["centre"], e["half"], rate, e["velocity"], e["pool"]))
        sol.add_emitters(specs)
        a, b = sc.model.state(), sc.model.state()
        drive = None if sc.motion is None else (lambda st, k, m=sc.motion, dt=sc.dt: m.apply(st, k * dt, dt))
        f, t, _, _ = collect_pairs(sol, a, b, sc.dt, steps, every=every, per_record=per, seed=seed, drive=drive)
        if log is not None:
            log(f"{sc.name}: {len(f)} pairs")
        out_f.append(f)
        out_t.append(t)
        del sol
    return np.concatenate(out_f)[:pairs], np.concatenate(out_t)[:pairs]


def main(argv=None) -> None:
    """python -m alloy_b200.solvers.sph.warmstart --out model.npz: pairs from the plain solver, then training."""
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--pairs", type=int, default=2_000_000)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=65536)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--sources", default="pour_bowls",
                    help="comma-separated workloads to draw pairs from: " + ", ".join(SOURCES))
    a = ap.parse_args(argv)
    f, t = generate_pairs(pairs=a.pairs, seed=a.seed, log=print, sources=tuple(a.sources.split(",")))
    m = train(f, t, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, log=print)
    m.save(a.out)
    print(f"saved {a.out}: {len(f)} pairs")


if __name__ == "__main__":
    main()
