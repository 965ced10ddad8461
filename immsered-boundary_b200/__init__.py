"""B200 explicit time step for the cell-based AMR compressible Navier-Stokes
solver with immersed bodies (drop-in for the reference's
NS_Solver::TimeMarching step; see include/ibgpu.h for the C ABI).

The directory name is not a Python identifier; load it with
``importlib`` under the module name ``immsered_boundary_b200`` (tests/,
bench.py and __graft_entry__.py do so).
"""
from . import ibgpu, indicator, workloads  # noqa: F401

__all__ = ["ibgpu", "indicator", "workloads"]
