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
