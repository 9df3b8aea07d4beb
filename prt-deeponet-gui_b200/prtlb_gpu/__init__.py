"""prtlb_gpu -- PRT-LB's flow and transport hot path on one NVIDIA B200.

Drop-in for the reference's NumPy simulator (3D/tools/prtlb_2d.py,
3D/tools/prtlb_3d.py): the same function names, signatures, outputs and
refusals, computed by hand-written sm_100a CUDA in libprtlb.so through a
C ABI (include/prtlb.h).  There is no CPU fallback.

    from prtlb_gpu import stokes_d3q19, solve_adr, check_physics
"""

from ._lib import Context, PrtError, default_context, lib  # noqa: F401
from .adr import solve_adr, prepare  # noqa: F401
from .chemistry import (Chemistry, Sorption, default_chemistry,  # noqa: F401
                        first_order_chemistry, monod_chemistry,
                        reversible_sorption_chemistry)
from .flow import permeability, stokes_d2q9, stokes_d3q19, trt_minus  # noqa: F401
from .geometry import (assert_finite_distance, coat_with_biofilm,  # noqa: F401
                       random_pack, sphere_pack_3d, disk_pack_2d)
from .prep import keep_inlet_connected  # noqa: F401  (the GPU walk)
from .physics import check_physics  # noqa: F401
from . import prep  # noqa: F401  (the inlet walk on the GPU: keep_inlet_connected, geodesic_steps, ...)

SOLID, WALL, PORE = 0, 1, 2

__all__ = ["stokes_d2q9", "stokes_d3q19", "solve_adr", "check_physics", "Chemistry",
           "default_chemistry", "keep_inlet_connected", "coat_with_biofilm",
           "assert_finite_distance", "permeability", "Context", "PrtError",
           "SOLID", "WALL", "PORE"]
