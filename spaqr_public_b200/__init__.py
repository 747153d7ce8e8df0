"""spaQR-B200: B200-native hierarchical sparsified QR (spaQR) with GMRES/CGLS drivers.

The numerical path lives in the in-tree CUDA library (``_build/libspaqr_b200.so``,
C ABI in ``include/spaqr_b200.h``); this package is its Python mirror of the
reference's ``Tree`` / ``gmres`` / ``cgls`` surface plus the seeded workload
generators.
"""
from .tree import (FP32, FP64, Tree, autotune, cgls, column_normalize, factorize_batch, gmres,  # noqa: F401
                   gmres_adjoint, graph_parts, launches, solve_to_residual)

__all__ = ["Tree", "gmres", "gmres_adjoint", "cgls", "solve_to_residual", "launches", "column_normalize",
           "factorize_batch", "autotune", "graph_parts", "FP32", "FP64"]
