# SPDX-License-Identifier: Apache-2.0
"""World sharding across GPUs: worlds never interact (each has its own neighbour groups and reductions), so a
batched model splits into per-rank sub-models of whole worlds with no per-step collective. Worlds are assigned by
longest-processing-time on particle counts (largest first, to the least loaded rank), then kept in their original
order inside each rank so a world's particle order, and therefore every sum, is the same as in the full model."""

from __future__ import annotations

import heapq

import numpy as np

from .model import Model


def shard_worlds(sizes, ranks: int) -> list[list[int]]:
    """World indices per rank, balanced by ``sizes`` (particles per world); each list ascending."""
    if ranks < 1:
        raise ValueError("ranks must be >= 1")
    heap = [(0, r) for r in range(ranks)]
    out: list[list[int]] = [[] for _ in range(ranks)]
    for w in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        load, r = heapq.heappop(heap)
        out[r].append(w)
        heapq.heappush(heap, (load + int(sizes[w]), r))
    return [sorted(ws) for ws in out]


SHAPE_KEYS = ("shape_type", "shape_scale", "shape_transform", "shape_flags", "shape_body", "shape_mu",
              "shape_boundary")


def sub_arrays(arrays: dict, worlds: list[int]) -> dict:
    """Host arrays (``Model.host()``) of the listed worlds only, renumbered 0..len(worlds)-1: their particles, and
    the shapes of those worlds and the global ones in their original order (so each world sees the same walls in the
    same order as in the full model)."""
    ws = np.asarray(arrays["world_start"])
    idx = np.concatenate([np.arange(ws[w], ws[w + 1]) for w in worlds]) if worlds else np.zeros(0, np.int64)
    out = {k: arrays[k][idx] for k in ("q", "qd", "mass", "radius", "flags", "phase", "rest_density")}
    counts = np.array([ws[w + 1] - ws[w] for w in worlds], np.int64)
    out["world"] = np.repeat(np.arange(len(worlds), dtype=np.int32), counts)
    out["world_start"] = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    g = np.asarray(arrays["gravity"]).reshape(-1, 3)
    out["gravity"] = g[worlds] if len(g) > 1 else np.repeat(g, max(len(worlds), 1), axis=0)[: max(len(worlds), 1)]
    visc = arrays.get("viscosity")
    out["viscosity"] = np.asarray(visc)[idx] if visc is not None else np.full(len(idx), 1.0e-3, np.float32)
    sw = np.asarray(arrays.get("shape_world", np.zeros(0, np.int32)))
    new = {w: k for k, w in enumerate(worlds)}
    keep = [s for s in range(len(sw)) if sw[s] < 0 or int(sw[s]) in new]
    for k in SHAPE_KEYS:
        if k in arrays:
            out[k] = np.asarray(arrays[k])[keep]
    out["shape_world"] = np.array([int(sw[s]) if sw[s] < 0 else new[int(sw[s])] for s in keep], np.int32)
    return out


def sub_model(model: Model, worlds: list[int], device) -> Model:
    a = sub_arrays(model.host(), worlds)
    shapes = {"type": a.get("shape_type", []), "scale": a.get("shape_scale", np.zeros((0, 3))),
              "xform": a.get("shape_transform", np.zeros((0, 7))), "world": a["shape_world"],
              "flags": a.get("shape_flags", []), "body": a.get("shape_body", []), "mu": a.get("shape_mu", []),
              "boundary": a.get("shape_boundary", [])}
    return Model(a["q"], a["qd"], a["mass"], a["radius"], a["flags"], a["world"], a["world_start"], a["gravity"],
                 a["phase"], a["rest_density"], a["viscosity"], device, shapes=shapes)
