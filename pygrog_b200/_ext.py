"""Torch-facing mirror of the reference native module ``pygrog._pygrog_torch``.

Same seven names, argument meaning, return conventions and RuntimeError
messages as the pybind11 bindings in ``csrc/torch/module.cpp:54-87`` and the
argument checks of ``grog_interp.cpp:117-129``, ``sparse_ops.cpp:239-245,
275-279, 307-316`` and ``toep_psf.cpp:247-254, 282-292, 329-340``.  Each call
goes through the C ABI of ``libpygrog_b200.so`` on torch's current stream.

Differences from the reference, all deliberate:
* CUDA tensors only: a CPU tensor raises (the reference runs OpenMP loops);
* in-place targets (``grid``, ``psf``) must be contiguous: the reference
  silently updates a temporary copy of a non-contiguous target;
* data and weights must agree in precision (complex64 with float32,
  complex128 with float64); the reference CUDA scatter dispatches on the
  weights' dtype and misreads a complex128 grid given float32 weights;
* ``grog_interpolate`` writes zeros for an out-of-range table index where the
  reference CUDA kernel leaves the output uninitialised.
"""

from __future__ import annotations

import torch

from . import _lib


def _chk(cond: bool, msg: str) -> None:
    if not cond:
        raise RuntimeError(msg)


def _real_of(t: torch.Tensor) -> torch.dtype:
    return torch.float32 if t.dtype == torch.complex64 else torch.float64


def _check_pair(data: torch.Tensor, weights: torch.Tensor, what: str) -> int:
    code = _lib.dtype_code(data, what)
    _chk(data.is_complex(), f"{what}: data must be complex, got {data.dtype}")
    _chk(
        weights.dtype == _real_of(data),
        f"{what}: weights dtype {weights.dtype} does not match data dtype {data.dtype}",
    )
    return code


def grog_interpolate(data: torch.Tensor, indexes: torch.Tensor, kernel: torch.Tensor) -> torch.Tensor:
    """``out[n,b,:] = kernel[indexes[n]] @ data[n,b,:]`` (new tensor)."""
    _chk(data.dim() == 3, f"data must be 3-D (nsamples, nbatches, ncoils), got {data.dim()}-D")
    _chk(indexes.dim() == 1, f"indexes must be 1-D (nsamples,), got {indexes.dim()}-D")
    _chk(kernel.dim() == 3, f"kernel must be 3-D (n_kernels, ncoils, ncoils), got {kernel.dim()}-D")
    _chk(indexes.dtype == torch.int64, f"indexes must be int64, got {indexes.dtype}")
    _chk(
        data.size(0) == indexes.size(0),
        f"data.size(0) ({data.size(0)}) != indexes.size(0) ({indexes.size(0)})",
    )
    _chk(
        data.size(2) == kernel.size(1) and kernel.size(1) == kernel.size(2),
        f"ncoils mismatch between data ({data.size(2)}) and kernel "
        f"({kernel.size(1)}×{kernel.size(2)})",
    )
    code = _lib.dtype_code(data, "grog_interpolate")
    _chk(data.is_complex(), f"grog_interpolate: expected ComplexFloat or ComplexDouble, got {data.dtype}")
    _chk(kernel.dtype == data.dtype, f"kernel dtype {kernel.dtype} does not match data dtype {data.dtype}")
    _lib.require_cuda(data, indexes, kernel, what="grog_interpolate")
    data = data.contiguous()
    indexes = indexes.contiguous()
    kernel = kernel.contiguous()
    out = torch.empty_like(data)
    N, B, C = data.shape
    _lib.call(
        "pgb_grog_interpolate",
        data.data_ptr(), indexes.data_ptr(), kernel.data_ptr(), out.data_ptr(),
        N, B, C, kernel.size(0), code, _lib.stream_ptr(data.device),
    )
    return out


def _check_1d_scatter(grid, data, indices, weights, who):
    _chk(grid.dim() == 1, f"grid must be 1-D, got {grid.dim()}-D")
    _chk(data.dim() == 1, f"data must be 1-D, got {data.dim()}-D")
    _chk(indices.dim() == 1, "indices must be 1-D")
    _chk(weights.dim() == 1, "weights must be 1-D")
    _chk(data.size(0) == indices.size(0), "data/indices size mismatch")
    _chk(data.size(0) == weights.size(0), "data/weights size mismatch")
    _chk(indices.dtype == torch.int64, "indices must be int64")
    _chk(grid.is_contiguous(), f"{who}: grid must be contiguous (updated in place)")
    _chk(grid.dtype == data.dtype, f"{who}: grid dtype {grid.dtype} != data dtype {data.dtype}")
    _lib.require_cuda(grid, data, indices, weights, what=who)
    return _check_pair(data, weights, who)


def scatter_add(grid: torch.Tensor, data: torch.Tensor, indices: torch.Tensor, weights: torch.Tensor) -> None:
    """``grid[indices[i]] += weights[i] * data[i]`` in place."""
    code = _check_1d_scatter(grid, data, indices, weights, "scatter_add")
    data, indices, weights = data.contiguous(), indices.contiguous(), weights.contiguous()
    _lib.call(
        "pgb_scatter_add",
        grid.data_ptr(), grid.numel(), data.data_ptr(), indices.data_ptr(), weights.data_ptr(),
        data.numel(), code, _lib.stream_ptr(grid.device),
    )


def scatter_add_binned(
    grid: torch.Tensor,
    data: torch.Tensor,
    indices: torch.Tensor,
    weights: torch.Tensor,
    bin_starts: torch.Tensor,
    bin_size: int,
) -> None:
    """Binned shared-memory scatter-add (same result as :func:`scatter_add`)."""
    _chk(bin_starts.dim() == 1, "bin_starts must be 1-D")
    _chk(bin_starts.dtype == torch.int64, "bin_starts must be int64")
    _chk(int(bin_size) > 0, "bin_size must be positive")
    code = _check_1d_scatter(grid, data, indices, weights, "scatter_add_binned")
    _lib.require_cuda(bin_starts, what="scatter_add_binned")
    data, indices, weights = data.contiguous(), indices.contiguous(), weights.contiguous()
    bin_starts = bin_starts.contiguous()
    _lib.call(
        "pgb_scatter_add_binned",
        grid.data_ptr(), grid.numel(), data.data_ptr(), indices.data_ptr(), weights.data_ptr(),
        data.numel(), bin_starts.data_ptr(), bin_starts.numel() - 1, int(bin_size), code,
        _lib.stream_ptr(grid.device),
    )


def gather(grid: torch.Tensor, indices: torch.Tensor, weights: torch.Tensor) -> torch.Tensor:
    """``out[i] = weights[i] * grid[indices[i]]`` (new tensor)."""
    _chk(grid.dim() == 1, f"grid must be 1-D, got {grid.dim()}-D")
    _chk(indices.dim() == 1, "indices must be 1-D")
    _chk(weights.dim() == 1, "weights must be 1-D")
    _chk(indices.size(0) == weights.size(0), "indices/weights size mismatch")
    _chk(indices.dtype == torch.int64, "indices must be int64")
    _lib.require_cuda(grid, indices, weights, what="gather")
    code = _check_pair(grid, weights, "gather")
    grid, indices, weights = grid.contiguous(), indices.contiguous(), weights.contiguous()
    out = torch.empty(indices.numel(), dtype=grid.dtype, device=grid.device)
    _lib.call(
        "pgb_gather",
        grid.data_ptr(), grid.numel(), indices.data_ptr(), weights.data_ptr(), out.data_ptr(),
        indices.numel(), code, _lib.stream_ptr(grid.device),
    )
    return out


def psf_scatter_scalar(psf: torch.Tensor, indices: torch.Tensor, w_sq: torch.Tensor) -> None:
    """``psf[indices[i]] += w_sq[i]`` in place (real psf)."""
    _chk(psf.dim() == 1, f"psf must be 1-D, got {psf.dim()}-D")
    _chk(indices.dim() == 1, "indices must be 1-D")
    _chk(w_sq.dim() == 1, "w_sq must be 1-D")
    _chk(indices.size(0) == w_sq.size(0), "indices/w_sq size mismatch")
    _chk(indices.dtype == torch.int64, "indices must be int64")
    _chk(psf.dtype == w_sq.dtype, "psf/w_sq dtype mismatch")
    _chk(psf.dtype in (torch.float32, torch.float64), f"psf_scatter_scalar: unsupported dtype {psf.dtype}")
    _chk(psf.is_contiguous(), "psf_scatter_scalar: psf must be contiguous (updated in place)")
    _lib.require_cuda(psf, indices, w_sq, what="psf_scatter_scalar")
    code = _lib.dtype_code(psf, "psf_scatter_scalar")
    indices, w_sq = indices.contiguous(), w_sq.contiguous()
    _lib.call(
        "pgb_psf_scatter_scalar",
        psf.data_ptr(), psf.numel(), indices.data_ptr(), w_sq.data_ptr(), indices.numel(), code,
        _lib.stream_ptr(psf.device),
    )


def psf_scatter_outer(
    psf: torch.Tensor, indices: torch.Tensor, w_sq: torch.Tensor, basis_per_sample: torch.Tensor
) -> None:
    """``psf[idx, l, l'] += w_sq * conj(b[l]) * b[l']`` in place."""
    _chk(psf.dim() == 3, "psf must be 3-D (grid_size, M, M)")
    _chk(psf.size(1) == psf.size(2), "psf last two dims must be equal")
    _chk(indices.dim() == 1 and w_sq.dim() == 1, "indices and w_sq must be 1-D")
    _chk(basis_per_sample.dim() == 2, "basis must be 2-D (N, M)")
    _chk(
        indices.size(0) == w_sq.size(0) and indices.size(0) == basis_per_sample.size(0),
        "indices/w_sq/basis sample-count mismatch",
    )
    _chk(basis_per_sample.size(1) == psf.size(1), "basis M does not match psf M")
    _chk(indices.dtype == torch.int64, "indices must be int64")
    _chk(psf.is_contiguous(), "psf_scatter_outer: psf must be contiguous (updated in place)")
    _chk(basis_per_sample.dtype == psf.dtype, "psf_scatter_outer: basis dtype must match psf")
    _lib.require_cuda(psf, indices, w_sq, basis_per_sample, what="psf_scatter_outer")
    code = _check_pair(psf, w_sq, "psf_scatter_outer")
    indices, w_sq, b = indices.contiguous(), w_sq.contiguous(), basis_per_sample.contiguous()
    _lib.call(
        "pgb_psf_scatter_outer",
        psf.data_ptr(), psf.size(0), psf.size(1), indices.data_ptr(), w_sq.data_ptr(), b.data_ptr(),
        indices.numel(), code, _lib.stream_ptr(psf.device),
    )


def psf_scatter_outer_basis(
    psf: torch.Tensor,
    indices: torch.Tensor,
    w_sq: torch.Tensor,
    basis: torch.Tensor,
    time_index: torch.Tensor,
) -> None:
    """``psf[idx, k, k'] += w_sq * conj(B[k, t]) * B[k', t]`` in place."""
    _chk(psf.dim() == 3, "psf must be 3-D (grid_size, K, K)")
    _chk(psf.size(1) == psf.size(2), "psf last two dims must be equal")
    _chk(basis.dim() == 2, "basis must be 2-D (K, T)")
    _chk(basis.size(0) == psf.size(1), "basis K does not match psf K")
    _chk(
        indices.dim() == 1 and w_sq.dim() == 1 and time_index.dim() == 1,
        "indices, w_sq, time_index must be 1-D",
    )
    _chk(
        indices.size(0) == w_sq.size(0) and indices.size(0) == time_index.size(0),
        "indices/w_sq/time_index size mismatch",
    )
    _chk(indices.dtype == torch.int64, "indices must be int64")
    _chk(time_index.dtype == torch.int64, "time_index must be int64")
    _chk(psf.is_contiguous(), "psf_scatter_outer_basis: psf must be contiguous (updated in place)")
    _chk(basis.dtype == psf.dtype, "psf_scatter_outer_basis: basis dtype must match psf")
    _lib.require_cuda(psf, indices, w_sq, basis, time_index, what="psf_scatter_outer_basis")
    code = _check_pair(psf, w_sq, "psf_scatter_outer_basis")
    indices, w_sq, basis, time_index = (
        indices.contiguous(), w_sq.contiguous(), basis.contiguous(), time_index.contiguous(),
    )
    _lib.call(
        "pgb_psf_scatter_outer_basis",
        psf.data_ptr(), psf.size(0), psf.size(1), indices.data_ptr(), w_sq.data_ptr(),
        basis.data_ptr(), basis.size(1), time_index.data_ptr(), indices.numel(), code,
        _lib.stream_ptr(psf.device),
    )


__all__ = [
    "grog_interpolate",
    "scatter_add",
    "scatter_add_binned",
    "gather",
    "psf_scatter_scalar",
    "psf_scatter_outer",
    "psf_scatter_outer_basis",
]
