"""B200 hierarchical domain-decomposition PCG Poisson solver (uwgraphics/hierarchicaldd hot path).

The compute path is libhdd_b200.so (hand-written sm_100a CUDA kernels behind the
C ABI in include/hdd.h); this package holds the Python host mirror of the
reference solver API and the synthetic domain generator.
"""
from . import domains  # noqa: F401

__all__ = ["domains", "SPGrid_Domain_Decomposition_Solver", "HddError"]


def __getattr__(name):
    if name in ("SPGrid_Domain_Decomposition_Solver", "HddError"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)
