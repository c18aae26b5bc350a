"""GROG Toeplitz normal operator on the GPU.

Mirrors ``_toep/_grog_toep.py`` (``GrogToeplitzOp``, 30-209) of
FiRMLAB-Pisa/pygrog: the PSF is the per-cell sum of squared sqrt-weights,
``PSF[j] = sum_i w_i delta(j == idx_i)`` built once with
``psf_scatter_scalar`` (or the ``density`` grid of a MaskedFFT), and
``A^H A x = sum_c conj(S_c) crop(IFFT(PSF * FFT(pad(S_c x))))``.

Here: one coil-expansion kernel, one batched cuFFT, one PSF multiply (PSF
stored in FFT order with the two ortho scales folded in), one batched inverse
cuFFT and one crop + coil-sum kernel per call, for all coils at once.
"""

from __future__ import annotations

__all__ = ["GrogToeplitzOp"]

import numpy as np
import torch

from . import _ext
from ._fftops import FFTStage, as_c64, compute_device


class GrogToeplitzOp:
    """Self-adjoint ``A^H A`` of a :class:`SparseFFT` or :class:`MaskedFFT`."""

    def __init__(self, sparse_fft, device=None):
        self.sparse_fft = sparse_fft
        self.device = compute_device(device if device is not None else getattr(sparse_fft, "device", None))
        self.grid_shape = tuple(sparse_fft.grid_shape)
        self.image_shape = tuple(sparse_fft.image_shape)
        self.fft_axes = sparse_fft.fft_axes
        self._pad_slices = sparse_fft._pad_slices
        self.stack_shape = tuple(getattr(sparse_fft, "stack_shape", ()) or ())
        self._stage = FFTStage(self.grid_shape, self.image_shape)
        S = int(np.prod(self.stack_shape)) if self.stack_shape else 1
        G = self._stage.G
        dens = getattr(sparse_fft, "density", None)
        if dens is not None:
            psf = torch.as_tensor(dens).to(self.device, torch.float32).reshape(S, *self.grid_shape).clone()
        else:
            idx = sparse_fft.indices.reshape(S, -1).to(self.device)
            sw = sparse_fft.sqrt_weights.reshape(S, -1).to(self.device, torch.float32)
            psf = torch.zeros(S, G, dtype=torch.float32, device=self.device)
            for s in range(S):
                _ext.psf_scatter_scalar(psf[s], idx[s].contiguous(), (sw[s] * sw[s]).contiguous())
            psf = psf.reshape(S, *self.grid_shape)
        # reference attribute: PSF on the centred grid
        self.psf = psf.reshape(*self.stack_shape, *self.grid_shape) if self.stack_shape else psf[0]
        self._psf_fft = (self._stage.to_fft_order(psf) * (1.0 / G)).reshape(S, G).contiguous()

    def _n_coils(self, x):
        sm = self.sparse_fft.smaps
        return int(sm.shape[0]) if sm is not None else int(x.shape[1])

    def _apply_frames(self, x: torch.Tensor, s: int, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """x (B, *img) [smaps] or (B, C, *img) on device -> out (same shape)."""
        st = self._stage
        smaps = getattr(self.sparse_fft, "_smaps_d", None)
        B = int(x.shape[0])
        C = self._n_coils(x)
        u = torch.empty(B, C, *st.grid_shape, dtype=torch.complex64, device=x.device)
        st.expand(x, smaps, u, B, C, 1.0, x_has_coils=smaps is None)
        U = st.fft(u)
        st.psf_apply(U, self._psf_fft[s], B * C, st.G)
        V = st.ifft(U)
        st.combine(V, smaps, out, B, C, 1.0, add=x if damp else None, add_scale=damp)
        return out

    def _apply_into(self, x: torch.Tensor, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """One frame, stack element 0: ``out = A^H A x + damp * x``."""
        return self._apply_frames(x.reshape(1, *x.shape), 0, out.reshape(1, *out.shape), damp)

    def __call__(self, image):
        x = torch.as_tensor(image)
        src_dev = x.device
        sf = self.sparse_fft
        s_shape = self.stack_shape
        single_ndim = len(self.image_shape) + (0 if sf.smaps is not None else 1)
        prefix = tuple(int(s) for s in x.shape[: x.ndim - single_ndim])
        if s_shape:
            if len(prefix) < len(s_shape) or tuple(prefix[-len(s_shape):]) != s_shape:
                raise ValueError(f"image prefix {prefix} must end with stack_shape {s_shape}")
            B_shape = prefix[: len(prefix) - len(s_shape)]
        else:
            B_shape = prefix
        single = tuple(int(s) for s in x.shape[x.ndim - single_ndim:])
        S = int(np.prod(s_shape)) if s_shape else 1
        Bt = int(np.prod(B_shape)) if B_shape else 1
        xd = as_c64(x, self.device).reshape(Bt, S, *single)
        out = torch.empty_like(xd)
        for s in range(S):
            xs = xd[:, s].contiguous()
            os_ = torch.empty_like(xs)
            self._apply_frames(xs, s, os_)
            out[:, s] = os_
        return out.reshape(x.shape).to(src_dev)
