"""Masked FFT operator on gridded k-space (reference ``operator/_masked_fft.py``)."""

from __future__ import annotations

import torch


class MaskedFFTPlan:
    """Plan returned by ``interpolate(grid=True)`` (reference ``_masked_fft.py:54-119``)."""

    def __init__(self, grid_shape, image_shape, stack_shape, mask, density, *, coords=None, dcf=None):
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.image_shape = tuple(int(s) for s in image_shape)
        self.stack_shape = tuple(int(s) for s in stack_shape)
        self.mask = torch.as_tensor(mask).float()
        self.density = torch.as_tensor(density).float()
        self._coords = None if coords is None else torch.as_tensor(coords)
        self._dcf = None if dcf is None else torch.as_tensor(dcf).float()

    def __repr__(self):
        return (
            f"MaskedFFTPlan(grid_shape={self.grid_shape}, image_shape={self.image_shape}, "
            f"stack_shape={self.stack_shape}, mask={tuple(self.mask.shape)}, "
            f"density={tuple(self.density.shape)})"
        )


import numpy as np

from .._fftops import FFTStage, as_c64, compute_device, with_torch
from .._solve import SolveMixin

__all__ = ["MaskedFFTPlan", "MaskedFFT"]


class MaskedFFT(SolveMixin):
    """Masked FFT / IFFT operator on gridded k-space (reference ``_masked_fft.py:122-561``).

    ``adjoint``: gridded k-space ``(*B, *S, C, *grid)`` -> image (mask, centred
    IFFT, crop, conj-smaps coil sum); ``forward``: image -> masked gridded
    k-space; ``normal``: Toeplitz with ``density`` as the PSF when enabled.
    One batched pass over all coils per call.
    """

    def __init__(self, grid_shape=None, image_shape=None, mask=None, density=None, smaps=None, stack_shape=None,
                 device=None, *, toeplitz=None, plan=None, coords=None, dcf=None):
        _pc = None if coords is None else torch.as_tensor(coords)
        _pd = None if dcf is None else torch.as_tensor(dcf).float()
        if plan is not None and isinstance(plan, MaskedFFTPlan):
            grid_shape, image_shape, mask, density = plan.grid_shape, plan.image_shape, plan.mask, plan.density
            if stack_shape is None:
                stack_shape = plan.stack_shape
            _pc = plan._coords if _pc is None else _pc
            _pd = plan._dcf if _pd is None else _pd
        if grid_shape is None or image_shape is None or mask is None:
            raise ValueError(
                "Either 'plan' (MaskedFFTPlan) or explicit 'grid_shape', 'image_shape', and 'mask' are required."
            )
        self._cdev = compute_device(device)
        self.grid_shape = tuple(int(s) for s in grid_shape)
        self.image_shape = tuple(int(s) for s in image_shape)
        self.ndim = len(self.grid_shape)
        self.grid_size = int(np.prod(self.grid_shape))
        self.fft_axes = tuple(range(-self.ndim, 0))
        mask_t = torch.as_tensor(mask).float()
        if stack_shape is None:
            stack_shape = tuple(int(s) for s in mask_t.shape[: -self.ndim]) if mask_t.ndim > self.ndim else ()
        self.stack_shape = tuple(int(s) for s in stack_shape)
        self.mask = mask_t
        self.density = torch.as_tensor(density).float() if density is not None else None
        self._coords = _pc
        self._dcf = _pd
        self.natural_shape = self.grid_shape
        self.n_samples = self.grid_size
        if smaps is not None:
            self.smaps = torch.as_tensor(smaps)
            self._conj_smaps = self.smaps.conj()
            self._smaps_d = as_c64(self.smaps, self._cdev)
        else:
            self.smaps = None
            self._conj_smaps = None
            self._smaps_d = None
        self._pad_slices = tuple(
            slice((gs - is_) // 2, (gs - is_) // 2 + is_) for gs, is_ in zip(self.grid_shape, self.image_shape)
        )
        self.device = torch.device(device) if device is not None else None
        if toeplitz is None:
            target = self.device if self.device is not None else torch.device("cpu")
            toeplitz = target.type == "cpu"
        if toeplitz and self.density is None:
            toeplitz = False
        self.toeplitz = bool(toeplitz)
        self._toep_op = None
        self._plan = plan
        self._stage = FFTStage(self.grid_shape, self.image_shape)
        S = int(np.prod(self.stack_shape)) if self.stack_shape else 1
        self._mask_d = self.mask.to(self._cdev, torch.float32).reshape(S, self.grid_size).contiguous()

    def _stack_mask(self, s_flat_idx: int):
        if not self.stack_shape:
            return self.mask, self.density
        S = int(np.prod(self.stack_shape))
        m = self.mask.reshape(S, *self.grid_shape)[s_flat_idx]
        d = self.density.reshape(S, *self.grid_shape)[s_flat_idx] if self.density is not None else None
        return m, d

    def _split(self, x, single_ndim):
        prefix = tuple(int(s) for s in x.shape[: x.ndim - single_ndim])
        s_shape = self.stack_shape
        if s_shape:
            if len(prefix) < len(s_shape) or tuple(prefix[-len(s_shape):]) != s_shape:
                raise ValueError(f"prefix {prefix} must end with stack_shape {s_shape}")
            return prefix[: len(prefix) - len(s_shape)]
        return prefix

    @with_torch
    def adjoint(self, kspace_grid):
        x = torch.as_tensor(kspace_grid)
        src_dev = x.device
        st = self._stage
        B_shape = self._split(x, 1 + self.ndim)
        C = int(x.shape[-self.ndim - 1])
        S = int(np.prod(self.stack_shape)) if self.stack_shape else 1
        Bt = int(np.prod(B_shape)) if B_shape else 1
        xd = as_c64(x, self._cdev).reshape(Bt, S, C, *self.grid_shape)
        single = tuple(self.image_shape) if self.smaps is not None else (C, *self.image_shape)
        out = torch.empty(Bt, S, *single, dtype=torch.complex64, device=self._cdev)
        for s in range(S):
            xs = xd[:, s].contiguous()
            u = torch.empty_like(xs)
            st.shift(xs, self._mask_d[s], u, Bt * C, 1.0, to_centred=False)
            v = st.ifft(u)
            o = torch.empty(Bt, *single, dtype=torch.complex64, device=self._cdev)
            st.combine(v, self._smaps_d, o, Bt, C, st.ortho)
            out[:, s] = o
        return out.reshape(*B_shape, *self.stack_shape, *single).to(src_dev)

    @with_torch
    def forward(self, image):
        x = torch.as_tensor(image)
        src_dev = x.device
        st = self._stage
        single_ndim = self.ndim + (0 if self.smaps is not None else 1)
        B_shape = self._split(x, single_ndim)
        single = tuple(int(s) for s in x.shape[x.ndim - single_ndim:])
        C = int(self.smaps.shape[0]) if self.smaps is not None else single[0]
        S = int(np.prod(self.stack_shape)) if self.stack_shape else 1
        Bt = int(np.prod(B_shape)) if B_shape else 1
        xd = as_c64(x, self._cdev).reshape(Bt, S, *single)
        out = torch.empty(Bt, S, C, *self.grid_shape, dtype=torch.complex64, device=self._cdev)
        for s in range(S):
            xs = xd[:, s].contiguous()
            u = torch.empty(Bt, C, *self.grid_shape, dtype=torch.complex64, device=self._cdev)
            st.expand(xs, self._smaps_d, u, Bt, C, 1.0, x_has_coils=self._smaps_d is None)
            U = st.fft(u)
            o = torch.empty_like(U)
            st.shift(U, self._mask_d[s], o, Bt * C, st.ortho, to_centred=True)
            out[:, s] = o
        return out.reshape(*B_shape, *self.stack_shape, C, *self.grid_shape).to(src_dev)

    def __call__(self, x, adjoint=False):
        return self.adjoint(x) if adjoint else self.forward(x)

    @with_torch
    def normal(self, image):
        if self.toeplitz:
            if self._toep_op is None:
                from .._toep import GrogToeplitzOp

                self._toep_op = GrogToeplitzOp(self, device=self._cdev)
            return self._toep_op(image)
        return self.adjoint(self.forward(image))

    def _normal_into(self, x, out, damp: float = 0.0):
        if self.stack_shape:
            raise NotImplementedError("device CG loop covers unstacked operators")
        if self.toeplitz:
            if self._toep_op is None:
                from .._toep import GrogToeplitzOp

                self._toep_op = GrogToeplitzOp(self, device=self._cdev)
            return self._toep_op._apply_into(x, out, damp)
        y = self.adjoint(self.forward(x))
        out.copy_(y + damp * x if damp else y)
        return out

    def _mask_ifft_crop_batch(self, batch_kspace_grid, s_flat_idx: int = 0):
        x = torch.as_tensor(batch_kspace_grid)
        src_dev = x.device
        B = int(x.shape[0])
        st = self._stage
        xd = as_c64(x, self._cdev).reshape(B, *self.grid_shape)
        u = torch.empty_like(xd)
        st.shift(xd, self._mask_d[s_flat_idx], u, B, 1.0, to_centred=False)
        v = st.ifft(u)
        out = torch.empty(B, 1, *self.image_shape, dtype=torch.complex64, device=self._cdev)
        st.combine(v.reshape(B, 1, *self.grid_shape), None, out, B, 1, st.ortho)
        return out.reshape(B, *self.image_shape).to(src_dev)

    def _fft_pad_mask_batch(self, batch_imgs, s_flat_idx: int = 0):
        x = torch.as_tensor(batch_imgs)
        src_dev = x.device
        B = int(x.shape[0])
        st = self._stage
        xd = as_c64(x, self._cdev).reshape(B, 1, *self.image_shape)
        u = torch.empty(B, 1, *self.grid_shape, dtype=torch.complex64, device=self._cdev)
        st.expand(xd, None, u, B, 1, 1.0, x_has_coils=True)
        U = st.fft(u)
        o = torch.empty_like(U)
        st.shift(U, self._mask_d[s_flat_idx], o, B, st.ortho, to_centred=True)
        return o.reshape(B, *self.grid_shape).to(src_dev)
