"""B200 (sm_100a) implementation of fmm3dbie's combined-field Dirichlet path:
the locally corrected layer-potential matvec (lpcomp_{lap,helm}_comb_dir) and
the GMRES solvers built on it, behind the reference's calling sequences.

    from fmm3dbie_b200 import surface, layer, Plan
"""
from ._lib import BieError, lib  # noqa: F401
from . import surface  # noqa: F401
from .surface import Surface, NearField, Oversampled, Setup  # noqa: F401
from . import layer  # noqa: F401
from .plan import Plan  # noqa: F401

__version__ = "0.1.0"
