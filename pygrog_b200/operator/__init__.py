"""Cartesian operators on GROG-gridded data (GPU)."""

from ._masked_fft import MaskedFFT, MaskedFFTPlan  # noqa: F401
from ._sparse_fft import SparseFFT, gather, scatter_add  # noqa: F401
from ._subspace import (  # noqa: F401
    SubspaceMaskedFFT,
    SubspaceProjection,
    SubspaceSparseFFT,
    SubspaceToeplitzOp,
    with_subspace,
)

__all__ = ["SparseFFT", "MaskedFFT", "MaskedFFTPlan", "gather", "scatter_add", "SubspaceProjection",
           "SubspaceMaskedFFT", "SubspaceSparseFFT", "SubspaceToeplitzOp", "with_subspace"]
