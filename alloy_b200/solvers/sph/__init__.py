# SPDX-License-Identifier: Apache-2.0
"""B200 DFSPH liquid solver: the reference's ``alloy.solvers.sph`` interface (SolverDFSPH, DFSPHConfig) over
hand-written sm_100a CUDA kernels (include/alloy_dfsph.h)."""

from .config import DFSPHConfig
from .solver import SolverDFSPH
from .types import SPHReport

__all__ = ["DFSPHConfig", "SolverDFSPH", "SPHReport"]
