"""Drop-in for the reference module 3D/tools/prtlb_2d.py: the names its
callers import (build_dataset_2d.py:61-63, build_toy_pack_2d.py:66)."""

from . import SOLID, WALL, PORE  # noqa: F401
from .adr import solve_adr, _wanted_steps, _nearest_unused  # noqa: F401
from .chemistry import Chemistry, default_chemistry  # noqa: F401
from .flow import stokes_d2q9, trt_minus as _trt_minus  # noqa: F401
from .geometry import assert_finite_distance, coat_with_biofilm  # noqa: F401
from .prep import keep_inlet_connected  # noqa: F401
from .physics import check_physics  # noqa: F401
