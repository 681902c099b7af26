# SPDX-License-Identifier: Apache-2.0
"""alloy_b200: a B200-native DFSPH liquid step with the reference's SolverDFSPH interface."""

__version__ = "0.1.0"
