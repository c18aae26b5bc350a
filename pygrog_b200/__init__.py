"""pygrog_b200: the GROG gridding hot path of pygrog, re-built for NVIDIA B200 (sm_100a).

Public API mirrors FiRMLAB-Pisa/pygrog: ``calib.GrogInterpolator``,
``operator.SparseFFT`` / ``operator.MaskedFFT`` and the ``cg`` / ``lsmr`` /
``solve`` solvers.  Every array operation on the path runs in hand-written
CUDA kernels (``libpygrog_b200.so``) or cuFFT; there is no CPU fallback.
"""

from . import calib  # noqa: F401
from . import operator  # noqa: F401
from ._lib import load_library  # noqa: F401

__version__ = "0.1.0"

from ._solve import cg, lsmr, solve  # noqa: F401
from ._toep import GrogToeplitzOp  # noqa: F401
