"""hydropol2d_b200 -- B200-native surface-flow step of HydroPol2D.

The product is the C-ABI library ``libhp2d.so`` (include/hp2d.h): sm_100a kernels for
the local-inertial D4 routing (Local_Inertial_Model_D4 / Inertial_Solver), Green-Ampt
infiltration at the Infiltration_Module boundary, the CFL timestep of
refreshing_timestep, and the fused step of HydroPol2D_Main_While.  This package is the
host-side mirror: ``SurfaceFlow`` (one resident grid), the MATLAB-signature functions
in ``reference_api`` and the seeded benchmark inputs in ``synthetic``.
"""
from ._abi import HP2DError, default_params  # noqa: F401
from .surface import SurfaceFlow  # noqa: F401

__all__ = ["SurfaceFlow", "HP2DError", "default_params"]
