"""Masked FFT operator on gridded k-space (reference ``operator/_masked_fft.py``)."""

from __future__ import annotations

__all__ = ["MaskedFFTPlan"]

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
