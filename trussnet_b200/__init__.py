"""trussnet_b200 -- v2mesh's truss/particle relaxation loop on NVIDIA B200 (sm_100a).

The native library libv2m_cuda.so (csrc/, C ABI in include/v2m_cuda.h) holds
the kernels and the loop; this package is the host-side mirror of the
reference's relaxation interface (tn::relax_cl / tn::relax_cpu and their types,
fangq/trussnet src/v2m_gpu.h, src/v2m_particles.h) plus seeded synthetic inputs.
"""
from .types import (V2M_CORNER, V2M_INTERFACE, V2M_INTERIOR, V2M_JUNCTION, V2M_K, V2M_NOLAB, Grid, GridParams,
                    Nodes, RelaxParams, RelaxStats)
from .relax import Session, device_count, grid_cl, points_cl, relax_cl, relax_cl_batch, seed_cl, validate_lists
from ._lib import V2mError

__all__ = ["Grid", "Nodes", "RelaxParams", "RelaxStats", "Session", "relax_cl", "relax_cl_batch", "seed_cl", "device_count",
           "validate_lists", "grid_cl", "points_cl", "GridParams",
           "V2mError", "V2M_INTERIOR", "V2M_INTERFACE", "V2M_JUNCTION", "V2M_CORNER", "V2M_NOLAB", "V2M_K"]
