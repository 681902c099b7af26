# SPDX-License-Identifier: Apache-2.0
"""adf_world_sum_noalloc through the C ABI: the per-world float64 residual sum for callers that cannot allocate
device memory (a host loop that must not enter the CUDA allocator, or a process whose device memory another
framework's pool already holds). It keeps its scratch in a static device array shared by every call, so two calls
in a row must each equal the solver's own reducer (adf_world_sum) bit for bit, the tolerance every reduction test
here uses; sizes beyond the static scratch are refused with a message."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from alloy_b200 import _lib
from alloy_b200.solvers.sph import SolverDFSPH
from alloy_b200.solvers.sph.testing import batched_worlds

pytestmark = pytest.mark.gpu


def test_noalloc_world_sum_equals_the_solver_reducer_on_two_calls(cuda):
    sc = batched_worlds(worlds=7, lo=300, hi=5000, seed=3, device=cuda)  # uneven worlds, spares included
    sol = SolverDFSPH(sc.model, sc.config)
    L = _lib.lib()
    n, W = sol.n, sol.world_count
    ws = torch.as_tensor(sol.world_start, dtype=torch.int32, device=cuda)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    gen = torch.Generator().manual_seed(0)
    for call in range(2):
        vals = (torch.randn(n, generator=gen) * 10.0 ** (call - 3)).to(torch.float32).to(cuda)
        ref_sum = torch.zeros(W, dtype=torch.float64, device=cuda)
        ref_max = torch.zeros(W, dtype=torch.float32, device=cuda)
        _lib.check(L.adf_world_sum(sol._h, vals.data_ptr(), ref_sum.data_ptr(), ref_max.data_ptr(), stream))
        out_sum = torch.full((W,), float("nan"), dtype=torch.float64, device=cuda)
        out_max = torch.full((W,), float("nan"), dtype=torch.float32, device=cuda)
        _lib.check(L.adf_world_sum_noalloc(vals.data_ptr(), n, ws.data_ptr(), W, out_sum.data_ptr(),
                                           out_max.data_ptr(), stream))
        torch.cuda.synchronize(cuda)
        assert torch.equal(out_sum, ref_sum), call
        assert torch.equal(out_max, ref_max), call
        v = vals.double().cpu().numpy()
        b = sol.world_start
        np.testing.assert_allclose(out_sum.cpu().numpy(), [v[b[w]:b[w + 1]].sum() for w in range(W)], rtol=1e-12,
                                   atol=1e-12)


def _many_worlds(device, worlds=3000, seed=11):
    """Worlds of 0..400 particles: every seventh and a run of ten consecutive ones empty, some of exactly 256 and 257
    (chunk edges), so one thread of the chunk table covers several worlds and the world search meets equal starts."""
    from alloy_b200.solvers.sph.build import add_fluid_points
    from alloy_b200.solvers.sph.model import ModelBuilder
    from alloy_b200.solvers.sph.testing import benchmark_config

    cfg = benchmark_config(0.02)
    rng = np.random.default_rng(seed)
    sizes = rng.integers(1, 401, worlds)
    sizes[::7] = 0
    sizes[100:110] = 0
    sizes[[5, 6, 500]] = (256, 257, 512)
    b = ModelBuilder()
    for w in range(worlds):
        b.begin_world()
        if sizes[w]:
            add_fluid_points(b, cfg, rng.uniform(0.0, 0.3, (int(sizes[w]), 3)))
        b.end_world()
    return b.finalize(device), cfg, sizes


def test_noalloc_world_sum_many_worlds_with_empty_ones(cuda):
    model, cfg, sizes = _many_worlds(cuda)
    sol = SolverDFSPH(model, cfg)
    L = _lib.lib()
    n, W = sol.n, sol.world_count
    assert W == 3000 and n == int(sizes.sum())
    ws = torch.as_tensor(sol.world_start, dtype=torch.int32, device=cuda)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    gen = torch.Generator().manual_seed(1)
    for call in range(2):
        vals = torch.randn(n, generator=gen).to(torch.float32).to(cuda)
        ref_sum = torch.zeros(W, dtype=torch.float64, device=cuda)
        ref_max = torch.zeros(W, dtype=torch.float32, device=cuda)
        _lib.check(L.adf_world_sum(sol._h, vals.data_ptr(), ref_sum.data_ptr(), ref_max.data_ptr(), stream))
        out_sum = torch.full((W,), float("nan"), dtype=torch.float64, device=cuda)
        out_max = torch.full((W,), float("nan"), dtype=torch.float32, device=cuda)
        _lib.check(L.adf_world_sum_noalloc(vals.data_ptr(), n, ws.data_ptr(), W, out_sum.data_ptr(),
                                           out_max.data_ptr(), stream))
        torch.cuda.synchronize(cuda)
        assert torch.equal(out_sum, ref_sum), call
        assert torch.equal(out_max, ref_max), call
        empty = torch.as_tensor(sizes == 0, device=cuda)
        assert torch.all(out_sum[empty] == 0.0) and torch.all(out_max[empty] == 0.0)


def test_noalloc_world_sum_of_no_values_is_zero(cuda):
    L = _lib.lib()
    W = 5
    ws = torch.zeros(W + 1, dtype=torch.int32, device=cuda)
    out_sum = torch.full((W,), float("nan"), dtype=torch.float64, device=cuda)
    out_max = torch.full((W,), float("nan"), dtype=torch.float32, device=cuda)
    stream = torch.cuda.current_stream(cuda).cuda_stream
    _lib.check(L.adf_world_sum_noalloc(None, 0, ws.data_ptr(), W, out_sum.data_ptr(), out_max.data_ptr(), stream))
    torch.cuda.synchronize(cuda)
    assert torch.all(out_sum == 0.0) and torch.all(out_max == 0.0)


def test_noalloc_world_sum_refuses_sizes_beyond_its_scratch(cuda):
    L = _lib.lib()
    dummy = torch.zeros(4, dtype=torch.float64, device=cuda)
    too_many_worlds = _lib.ADF_NOALLOC_MAX_WORLDS + 1
    with pytest.raises(_lib.CapacityError, match="world limit"):
        _lib.check(L.adf_world_sum_noalloc(dummy.data_ptr(), 0, dummy.data_ptr(), too_many_worlds, dummy.data_ptr(),
                                           dummy.data_ptr(), None))
    with pytest.raises(_lib.CapacityError, match="static scratch limit"):
        _lib.check(L.adf_world_sum_noalloc(dummy.data_ptr(), 256 * _lib.ADF_NOALLOC_MAX_CHUNKS, dummy.data_ptr(), 1,
                                           dummy.data_ptr(), dummy.data_ptr(), None))
