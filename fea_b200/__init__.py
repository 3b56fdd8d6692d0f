"""fea_b200 — the C3D4/C3D8 Neo-Hookean element, assembly and solver path of
sssnnn7119/FEA as hand-written sm_100a kernels behind the reference's API.

The kernels live in ``libfea_b200.so`` (C ABI: include/fea_b200.h), built
in-tree by ``python fea_b200/_build.py``.  Importing the package loads the
library and raises ImportError when it is missing; there is no fallback.
"""
from . import _lib  # noqa: F401  (loads the native library or raises)
from . import materials, elements, loads, boundarys, constraints
from .part import Part, Instance
from .reference_points import ReferencePoint
from .assembly import Assembly
from .controller import FEAController
from . import solver
from .plan import DevicePlan
from .inp import FEA_INP, from_inp

__all__ = ["Part", "Instance", "ReferencePoint", "Assembly", "FEAController", "materials", "elements", "loads",
           "boundarys", "constraints", "solver", "DevicePlan", "FEA_INP", "from_inp"]
