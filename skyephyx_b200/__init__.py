"""B200-native augmented vertex block descent (AVBD) step.

Drop-in for SkyePhyX's ``Solver::Step()``: scenes are built through the
reference's Solver API (bodies, box colliders, joints, springs, Neo-Hookean
tets, StVK triangles) and stepped by hand-written sm_100a CUDA kernels in the
in-tree ``libavbd.so`` (C-ABI in ``include/avbd.h``).
"""
from ._lib import AvbdError, AvbdParams, load  # noqa: F401
from .solver import GROUP_FLAT, Batch, INF, Solver  # noqa: F401

__all__ = ["Solver", "Batch", "AvbdError", "AvbdParams", "INF", "GROUP_FLAT", "load"]
