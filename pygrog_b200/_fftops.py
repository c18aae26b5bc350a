"""Shared GPU stages of the Cartesian operators: cuFFT plus the pointwise
kernels of ``csrc/fft_stage.cu``.

Buffers passed to cuFFT are kept in FFT order (centred index p stored at
m = (p - g//2) mod g), so the centred ortho transforms of the reference
(``_base/_fftc.py:114-139``: ifftshift -> fftn -> fftshift, ortho) become
one unscaled cuFFT call between two index-remapping kernels, with the ortho
scale folded into those kernels.
"""

from __future__ import annotations

import functools
import math

import numpy as np
import torch

from . import _lib


def with_torch(fn):
    """numpy arrays in -> torch tensors inside -> numpy arrays out (container only)."""

    @functools.wraps(fn)
    def wrapper(*args, **kwargs):
        was_numpy = any(isinstance(a, np.ndarray) for a in args) or any(
            isinstance(v, np.ndarray) for v in kwargs.values()
        )
        args = tuple(torch.as_tensor(a) if isinstance(a, np.ndarray) else a for a in args)
        kwargs = {k: (torch.as_tensor(v) if isinstance(v, np.ndarray) else v) for k, v in kwargs.items()}
        out = fn(*args, **kwargs)
        if was_numpy and isinstance(out, torch.Tensor):
            return out.detach().cpu().numpy()
        return out

    return wrapper


def compute_device(device) -> torch.device:
    """The CUDA device that runs the kernels (the reference's ``device`` argument
    may name the CPU; computation here is always on a GPU)."""
    if device is not None:
        d = torch.device(device)
        if d.type == "cuda":
            return d
    return torch.device("cuda", torch.cuda.current_device() if torch.cuda.is_available() else 0)


class FFTStage:
    """Shapes and launchers for one (grid_shape, image_shape) pair."""

    def __init__(self, grid_shape, image_shape):
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.image_shape = tuple(int(s) for s in image_shape)
        self.ndim = len(self.grid_shape)
        if self.ndim not in (2, 3):
            raise ValueError(f"only 2-D and 3-D grids are supported, got {self.ndim}-D")
        if len(self.image_shape) != self.ndim:
            raise ValueError("image_shape and grid_shape must have the same length")
        self.G = int(np.prod(self.grid_shape))
        self.I = int(np.prod(self.image_shape))
        self.axes = tuple(range(-self.ndim, 0))
        self._g = np.ascontiguousarray(self.grid_shape, dtype=np.int64)
        self._n = np.ascontiguousarray(self.image_shape, dtype=np.int64)
        self.ortho = 1.0 / math.sqrt(self.G)

    # -- index maps ---------------------------------------------------------
    def fft_order_index(self, centred_flat: torch.Tensor) -> torch.Tensor:
        """FFT-order flat index of centred flat grid indices."""
        idx = centred_flat.to(torch.int64)
        out = torch.zeros_like(idx)
        rem = idx
        mult = 1
        for d in reversed(range(self.ndim)):
            g = self.grid_shape[d]
            p = rem % g
            rem = rem // g
            m = (p - g // 2) % g
            out = out + m * mult
            mult *= g
        return out

    def to_fft_order(self, grid_centred: torch.Tensor) -> torch.Tensor:
        """Real or complex array (..., *grid) centred -> FFT order (ifftshift)."""
        return torch.fft.ifftshift(grid_centred, dim=self.axes)

    # -- launchers --------------------------------------------------------------
    def expand(self, x, smaps, u, B, C, scale, x_has_coils):
        _lib.call(
            "pgb_fft_expand", x.data_ptr(), smaps.data_ptr() if smaps is not None else None, u.data_ptr(),
            B, C, self.ndim, self._g.ctypes.data, self._n.ctypes.data, float(scale), int(x_has_coils),
            _lib.stream_ptr(u.device),
        )
        return u

    def combine(self, v, smaps, out, B, C, scale, add=None, add_scale=0.0):
        _lib.call(
            "pgb_fft_combine", v.data_ptr(), smaps.data_ptr() if smaps is not None else None, out.data_ptr(),
            B, C, self.ndim, self._g.ctypes.data, self._n.ctypes.data, float(scale),
            add.data_ptr() if add is not None else None, float(add_scale), _lib.stream_ptr(v.device),
        )
        return out

    def shift(self, src, mask, dst, BC, scale, to_centred):
        _lib.call(
            "pgb_fft_shift", src.data_ptr(), mask.data_ptr() if mask is not None else None, dst.data_ptr(),
            BC, self.ndim, self._g.ctypes.data, float(scale), int(to_centred), _lib.stream_ptr(src.device),
        )
        return dst

    def fft(self, u):
        """Unscaled forward DFT over the grid axes of an FFT-order buffer."""
        return torch.fft.fftn(u, dim=self.axes, norm="backward")

    def ifft(self, U):
        """Unscaled inverse DFT over the grid axes."""
        return torch.fft.ifftn(U, dim=self.axes, norm="forward")

    @staticmethod
    def scatter(data, cellpos, w, u, BC, R, G):
        _lib.call("pgb_sparse_scatter", data.data_ptr(), cellpos.data_ptr(), w.data_ptr(), u.data_ptr(),
                  BC, R, G, _lib.stream_ptr(u.device))

    @staticmethod
    def gather(U, cellpos, w, out, BC, R, G):
        _lib.call("pgb_sparse_gather", U.data_ptr(), cellpos.data_ptr(), w.data_ptr(), out.data_ptr(),
                  BC, R, G, _lib.stream_ptr(U.device))

    @staticmethod
    def psf_apply(U, psf, BC, G):
        _lib.call("pgb_psf_apply", U.data_ptr(), psf.data_ptr(), BC, G, _lib.stream_ptr(U.device))


def as_c64(t: torch.Tensor, device) -> torch.Tensor:
    """complex64, contiguous, on ``device`` (the kernels compute in complex64)."""
    t = torch.as_tensor(t)
    if t.dtype != torch.complex64:
        if t.is_complex() or t.is_floating_point():
            t = t.to(torch.complex64)
        else:
            raise TypeError(f"expected a complex tensor, got {t.dtype}")
    return t.to(device).contiguous()
