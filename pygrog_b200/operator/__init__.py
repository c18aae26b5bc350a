"""Cartesian operators on GROG-gridded data (GPU)."""

from ._masked_fft import MaskedFFTPlan  # noqa: F401

__all__ = ["MaskedFFTPlan"]

try:  # filled in as the operator modules land
    from ._sparse_fft import SparseFFT, gather, scatter_add  # noqa: F401
    from ._masked_fft import MaskedFFT  # noqa: F401

    __all__ += ["SparseFFT", "MaskedFFT", "gather", "scatter_add"]
except ImportError:  # pragma: no cover
    pass
