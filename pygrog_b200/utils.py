"""Pre-processing of multi-coil k-space: PCA coil compression.

Mirrors ``pygrog.utils.coil_compress`` (``utils/_coil_compress.py:23-57``),
which forwards to ``mrinufft.extras.smaps.coil_compression``: the principal
components of the coil data (optionally only the samples within
``krad_thresh`` of the k-space centre, relative to the largest radius of
``traj``) give a ``(K, C)`` compression matrix, and the virtual coils are the
matrix times the data.  ``n_coils`` is the number of virtual coils (int) or
the fraction of the calibration energy to keep (float in (0, 1]).

The coil covariance is accumulated in FP64 on the GPU
(``pgb_coil_covariance``), its ``C x C`` eigendecomposition is solved on the
host in FP64, and the compression is one HBM-bound kernel
(``pgb_coil_compress``).  Each virtual coil is scaled so that its
largest-magnitude weight is real and positive (eigenvectors are defined only
up to a phase).
"""

from __future__ import annotations

__all__ = ["coil_compress", "compression_matrix"]

import numpy as np
import torch

from . import _lib


def _as_device(x, device):
    t = torch.as_tensor(x)
    if not t.is_complex():
        t = t.to(torch.complex64)
    return t.to(device=device, dtype=torch.complex64).contiguous()


def compression_matrix(calib: torch.Tensor, n_coils) -> torch.Tensor:
    """``(K, C)`` complex64 matrix from calibration samples ``calib (C, M)`` (on the GPU)."""
    C, M = int(calib.shape[0]), int(calib.shape[1])
    cov = torch.empty(C, C, dtype=torch.complex128, device=calib.device)
    _lib.call("pgb_coil_covariance", calib.data_ptr(), M, C, cov.data_ptr(), _lib.stream_ptr(calib.device))
    w, v = torch.linalg.eigh(cov.cpu())  # ascending, FP64
    w = w.flip(0).clamp(min=0.0)
    v = v.flip(1)
    if isinstance(n_coils, float) and not float(n_coils).is_integer() or (isinstance(n_coils, float) and n_coils <= 1):
        frac = float(n_coils)
        if not 0.0 < frac <= 1.0:
            raise ValueError("an energy fraction must lie in (0, 1]")
        energy = torch.cumsum(w, 0) / max(float(w.sum()), 1e-300)
        K = int(torch.searchsorted(energy, torch.tensor(frac - 1e-12, dtype=energy.dtype)).item()) + 1
    else:
        K = int(n_coils)
    if not 1 <= K <= C:
        raise ValueError(f"number of virtual coils must be in 1..{C}, got {K}")
    mat = v[:, :K].conj().T.contiguous()  # (K, C)
    # phase convention: the largest-magnitude weight of every row is real and positive
    idx = mat.abs().argmax(dim=1)
    ph = mat[torch.arange(K), idx]
    mat = mat * (ph.abs() / ph).unsqueeze(1)  # times conj(ph) / |ph|
    return mat.to(torch.complex64).to(calib.device).contiguous()


def coil_compress(kspace_data, n_coils, traj=None, krad_thresh=None, *, device=None, precision: str = "fp32"):
    """``(compressed (K, n_samples), compression_matrix (K, C))`` like the reference.

    numpy input returns numpy arrays; a torch tensor returns tensors on its device.
    ``precision="bf16x3"`` runs the compression on the tensor cores (~1e-5
    relative to FP64; needs K <= 16 and C <= 32).
    """
    is_numpy = isinstance(kspace_data, np.ndarray)
    src_dev = kspace_data.device if isinstance(kspace_data, torch.Tensor) else torch.device("cpu")
    dev = torch.device(device) if device is not None else (src_dev if src_dev.type == "cuda" else torch.device("cuda"))
    if dev.type != "cuda":
        raise RuntimeError("coil_compress runs on a CUDA device (no CPU fallback)")
    data = _as_device(kspace_data, dev)
    C = int(data.shape[0])
    flat = data.reshape(C, -1)
    calib = flat
    if krad_thresh is not None and traj is not None:
        tr = torch.as_tensor(np.asarray(traj) if not isinstance(traj, torch.Tensor) else traj).to(dev).float()
        rad = torch.sqrt((tr.reshape(-1, tr.shape[-1]) ** 2).sum(-1))
        sel = rad < float(krad_thresh) * rad.max()
        calib = flat[:, sel].contiguous()
    mat = compression_matrix(calib, n_coils)
    K, N = int(mat.shape[0]), int(flat.shape[1])
    out = torch.empty(K, N, dtype=torch.complex64, device=dev)
    fn = {"fp32": "pgb_coil_compress", "bf16x3": "pgb_coil_compress_tc"}.get(precision)
    if fn is None:
        raise ValueError("precision must be 'fp32' or 'bf16x3'")
    _lib.call(fn, flat.data_ptr(), N, C, K, 1, mat.data_ptr(), out.data_ptr(), _lib.stream_ptr(dev))
    out = out.reshape(K, *data.shape[1:])
    if is_numpy:
        return out.cpu().numpy(), mat.cpu().numpy()
    return out.to(src_dev), mat.to(src_dev)
