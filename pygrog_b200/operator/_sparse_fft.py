"""Sparse FFT operator on GROG-gridded samples (GPU).

Mirrors ``operator/_sparse_fft.py`` of FiRMLAB-Pisa/pygrog: ``SparseFFT``
(187-1242) with ``adjoint`` (sparse k-space -> image, 505-572), ``forward``
(image -> sparse k-space, 685-701), ``normal`` (858-887), the batch helpers
(1050-1149), ``solve`` and the module functions ``scatter_add`` / ``gather``
(123-181).  Convention as in the reference: ``forward = A`` (image -> k),
``adjoint = A^H``; both apply ``sqrt(weights)`` and callers pre-multiply the
data by ``plan.pre_weights`` once.

Each call is one batched pass over all coils: coil expansion + zero pad +
shift (one kernel), one batched cuFFT, one natural-order gather (forward);
or one natural-order scatter, one batched cuFFT, one crop + shift +
conj-smaps coil sum (adjoint).  The reference instead loops over coils,
re-sorts the data and shifts with separate passes.
"""

from __future__ import annotations

__all__ = ["SparseFFT", "gather", "scatter_add"]

import numpy as np
import torch

from .. import _ext
from .._fftops import FFTStage, as_c64, compute_device, with_torch
from .._solve import SolveMixin


def scatter_add(grid, data, indices, weights) -> None:
    """``grid[indices[i]] += weights[i] * data[i]`` in place (reference ``scatter_add``)."""
    _ext.scatter_add(grid, data, indices, weights)


def gather(grid, indices, weights):
    """``out[i] = weights[i] * grid[indices[i]]`` (reference ``gather``)."""
    return _ext.gather(grid, indices, weights)


class _StackArrays:
    """Natural-order device arrays of one stack element."""

    def __init__(self, stage: FFTStage, idx_nat: torch.Tensor, sw_nat: torch.Tensor):
        self.cellpos = stage.fft_order_index(idx_nat).to(torch.int32).contiguous()
        self.w = sw_nat.to(torch.float32).contiguous()
        self.w_fwd = (self.w * stage.ortho).contiguous()
        self.R = int(idx_nat.numel())


class SparseFFT(SolveMixin):
    """Sparse FFT / IFFT operator with SENSE coil combination (GPU).

    Same constructor as the reference; ``device`` names where results may
    live (computation is always on a CUDA device).  ``toeplitz=None``
    follows the reference's policy (enabled unless ``device`` is CUDA).
    """

    def __init__(
        self,
        grid_shape=None,
        image_shape=None,
        indices=None,
        weights=None,
        smaps=None,
        device=None,
        *,
        plan=None,
        toeplitz=None,
    ):
        self._cdev = compute_device(device)
        if plan is not None:
            self.grid_shape = tuple(plan.grid_shape)
            self.image_shape = tuple(plan.image_shape)
            self.grid_size = int(plan.grid_size)
            self.indices = plan.indices
            self.sqrt_weights = plan.sqrt_weights
            self.sort_perm = plan.sort_perm
            self.inv_perm = plan.inv_perm
            self.natural_shape = tuple(int(s) for s in getattr(plan, "natural_shape", (int(plan.n_samples),)))
            self.stack_shape = tuple(int(s) for s in getattr(plan, "stack_shape", ()) or ())
        else:
            if grid_shape is None or image_shape is None:
                raise ValueError("Either 'plan' or both 'grid_shape'/'image_shape' required")
            self.grid_shape = tuple(int(s) for s in grid_shape)
            self.image_shape = tuple(int(s) for s in image_shape)
            self.grid_size = int(np.prod(self.grid_shape))
            idx = torch.as_tensor(indices).reshape(-1).to(torch.int64).to(self._cdev)
            w = torch.as_tensor(weights).reshape(-1).to(torch.float32).to(self._cdev)
            sqrt_w = torch.sqrt(w)
            sort_perm = torch.sort(idx, stable=True).indices
            self.sort_perm = sort_perm
            self.indices = idx[sort_perm]
            self.sqrt_weights = sqrt_w[sort_perm]
            inv = torch.empty_like(sort_perm)
            inv[sort_perm] = torch.arange(sort_perm.numel(), device=self._cdev)
            self.inv_perm = inv
            self.natural_shape = (int(idx.numel()),)
            self.stack_shape = ()
        self.n_samples = int(self.indices.shape[-1])
        self.ndim = len(self.grid_shape)
        self.fft_axes = tuple(range(-self.ndim, 0))
        self._stage = FFTStage(self.grid_shape, self.image_shape)
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
        self.toeplitz = bool(toeplitz)
        self._toep_op = None
        self._arrays = None

    # ------------------------------------------------------------------
    def _stack_arrays_dev(self, s: int) -> _StackArrays:
        if self._arrays is None:
            S = int(np.prod(self.stack_shape)) if self.stack_shape else 1
            idx = self.indices.reshape(S, -1).to(self._cdev)
            sw = self.sqrt_weights.reshape(S, -1).to(self._cdev)
            ip = self.inv_perm.reshape(S, -1).to(self._cdev)
            self._arrays = [
                _StackArrays(self._stage, torch.gather(idx[k], 0, ip[k]), torch.gather(sw[k], 0, ip[k]))
                for k in range(S)
            ]
        return self._arrays[s]

    def _stack_arrays(self, s_flat_idx: int):
        """``(indices, sqrt_weights, sort_perm, inv_perm)`` of one stack element."""
        if not self.stack_shape:
            return self.indices, self.sqrt_weights, self.sort_perm, self.inv_perm
        S = int(np.prod(self.stack_shape))
        n = self.n_samples
        return tuple(t.reshape(S, n)[s_flat_idx] for t in (self.indices, self.sqrt_weights, self.sort_perm, self.inv_perm))

    def _n_coils(self, fallback: int) -> int:
        return int(self.smaps.shape[0]) if self.smaps is not None else fallback

    # ------------------------------------------------------------------
    # core (one stack element, B frames, all coils in one pass)
    # ------------------------------------------------------------------
    def _adjoint_core(self, sparse: torch.Tensor, s: int) -> torch.Tensor:
        """sparse (B, C, n) complex64 on device -> image (B, *img) or (B, C, *img)."""
        B, C, n = sparse.shape
        st = self._stage
        a = self._stack_arrays_dev(s)
        u = torch.zeros(B, C, *st.grid_shape, dtype=torch.complex64, device=sparse.device)
        st.scatter(sparse, a.cellpos, a.w, u, B * C, n, st.G)
        v = st.ifft(u)
        if self._smaps_d is not None:
            out = torch.empty(B, *st.image_shape, dtype=torch.complex64, device=sparse.device)
        else:
            out = torch.empty(B, C, *st.image_shape, dtype=torch.complex64, device=sparse.device)
        st.combine(v, self._smaps_d, out, B, C, st.ortho)
        return out

    def _forward_core(self, image: torch.Tensor, s: int, C: int) -> torch.Tensor:
        """image (B, *img) [smaps] or (B, C, *img) -> sparse (B, C, n) natural order."""
        st = self._stage
        B = image.shape[0]
        a = self._stack_arrays_dev(s)
        u = torch.empty(B, C, *st.grid_shape, dtype=torch.complex64, device=image.device)
        st.expand(image, self._smaps_d, u, B, C, 1.0, x_has_coils=self._smaps_d is None)
        U = st.fft(u)
        out = torch.empty(B, C, a.R, dtype=torch.complex64, device=image.device)
        st.gather(U, a.cellpos, a.w_fwd, out, B * C, a.R, st.G)
        return out

    # ------------------------------------------------------------------
    # adjoint: sparse k-space -> image
    # ------------------------------------------------------------------
    @with_torch
    def adjoint(self, sparse_kspace):
        """Sparse k-space ``(*B, *S, C, *natural_shape | n_samples)`` to image."""
        nat = self.natural_shape
        x = torch.as_tensor(sparse_kspace)
        src_dev = x.device
        if len(nat) > 1 and tuple(int(s) for s in x.shape[-len(nat):]) == nat:
            x = x.reshape(*x.shape[: -len(nat)], self.n_samples)
        s_shape = self.stack_shape
        prefix = tuple(int(s) for s in x.shape[:-2])
        if s_shape:
            if len(prefix) < len(s_shape) or tuple(prefix[-len(s_shape):]) != s_shape:
                raise ValueError(f"sparse_kspace prefix {prefix} must end with stack_shape {s_shape}")
            B_shape = prefix[: len(prefix) - len(s_shape)]
        else:
            B_shape = prefix
        C = int(x.shape[-2])
        if x.shape[-1] != self.n_samples:
            raise ValueError(f"sparse_kspace has {x.shape[-1]} samples, plan has {self.n_samples}")
        if self.smaps is not None and C != self.smaps.shape[0]:
            raise ValueError(f"{C} coils in the data, {self.smaps.shape[0]} sensitivity maps")
        S = int(np.prod(s_shape)) if s_shape else 1
        Bt = int(np.prod(B_shape)) if B_shape else 1
        xd = as_c64(x, self._cdev).reshape(Bt, S, C, self.n_samples)
        outs = [self._adjoint_core(xd[:, s].contiguous(), s) for s in range(S)]
        out = torch.stack(outs, dim=1)  # (Bt, S, ...)
        single = tuple(self.image_shape) if self.smaps is not None else (C, *self.image_shape)
        out = out.reshape(*B_shape, *s_shape, *single)
        return out.to(src_dev)

    # ------------------------------------------------------------------
    # forward: image -> sparse k-space
    # ------------------------------------------------------------------
    @with_torch
    def forward(self, image):
        """Image ``(*B, *S, [C,] *image_shape)`` to sparse k-space ``(*B, *S, C, *natural_shape)``."""
        out = self._adjoint_flat(image)
        nat = self.natural_shape
        if len(nat) > 1:
            out = out.reshape(*out.shape[:-1], *nat)
        return out

    @with_torch
    def _adjoint_flat(self, image):
        """Flat-output forward: ``(*B, *S, C, n_samples)`` (reference naming)."""
        x = torch.as_tensor(image)
        src_dev = x.device
        s_shape = self.stack_shape
        single_ndim = len(self.image_shape) + (0 if self.smaps is not None else 1)
        prefix = tuple(int(s) for s in x.shape[: x.ndim - single_ndim])
        if s_shape:
            if len(prefix) < len(s_shape) or tuple(prefix[-len(s_shape):]) != s_shape:
                raise ValueError(f"image prefix {prefix} must end with stack_shape {s_shape}")
            B_shape = prefix[: len(prefix) - len(s_shape)]
        else:
            B_shape = prefix
        single = tuple(int(s) for s in x.shape[x.ndim - single_ndim:])
        C = self._n_coils(single[0] if self.smaps is None else 0)
        S = int(np.prod(s_shape)) if s_shape else 1
        Bt = int(np.prod(B_shape)) if B_shape else 1
        xd = as_c64(x, self._cdev).reshape(Bt, S, *single)
        outs = [self._forward_core(xd[:, s].contiguous(), s, C) for s in range(S)]
        out = torch.stack(outs, dim=1)  # (Bt, S, C, n)
        return out.reshape(*B_shape, *s_shape, C, self.n_samples).to(src_dev)

    def __call__(self, x, adjoint=False):
        return self.adjoint(x) if adjoint else self.forward(x)

    # ------------------------------------------------------------------
    # normal operator
    # ------------------------------------------------------------------
    @with_torch
    def normal(self, image):
        """``A^H A image`` (Toeplitz PSF when ``self.toeplitz``, else adjoint(forward))."""
        if self.toeplitz:
            if self._toep_op is None:
                from .._toep import GrogToeplitzOp

                self._toep_op = GrogToeplitzOp(self, device=self._cdev)
            return self._toep_op(image)
        return self.adjoint(self.forward(image))

    def _normal_into(self, x: torch.Tensor, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """``out = A^H A x + damp * x`` for one frame already on the device
        (used by the device-side CG loop; no host synchronisation)."""
        if self.stack_shape:
            raise NotImplementedError("device CG loop covers unstacked operators")
        if self.toeplitz:
            if self._toep_op is None:
                from .._toep import GrogToeplitzOp

                self._toep_op = GrogToeplitzOp(self, device=self._cdev)
            return self._toep_op._apply_into(x, out, damp)
        C = self._n_coils(x.shape[0] if x.ndim > len(self.image_shape) else 1)
        k = self._forward_core(x.reshape(1, *x.shape), 0, C)
        st = self._stage
        a = self._stack_arrays_dev(0)
        u = torch.zeros(1, C, *st.grid_shape, dtype=torch.complex64, device=x.device)
        st.scatter(k, a.cellpos, a.w, u, C, a.R, st.G)
        v = st.ifft(u)
        st.combine(v, self._smaps_d, out, 1, C, st.ortho, add=x if damp else None, add_scale=damp)
        return out

    def _normal_frames_into(self, x: torch.Tensor, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """``out[f] = A^H A x[f] + damp * x[f]`` for F independent frames ``x (F, *single)``
        already on the device (one batched pass; no host synchronisation)."""
        if self.stack_shape:
            raise NotImplementedError("frame-batched normal operator covers unstacked operators")
        if self.toeplitz:
            if self._toep_op is None:
                from .._toep import GrogToeplitzOp

                self._toep_op = GrogToeplitzOp(self, device=self._cdev)
            return self._toep_op._apply_frames(x, 0, out, damp)
        F = int(x.shape[0])
        C = self._n_coils(x.shape[1] if x.ndim > len(self.image_shape) + 1 else 1)
        k = self._forward_core(x, 0, C)
        st = self._stage
        a = self._stack_arrays_dev(0)
        u = torch.zeros(F, C, *st.grid_shape, dtype=torch.complex64, device=x.device)
        st.scatter(k, a.cellpos, a.w, u, F * C, a.R, st.G)
        v = st.ifft(u)
        st.combine(v, self._smaps_d, out, F, C, st.ortho, add=x if damp else None, add_scale=damp)
        return out

    # ------------------------------------------------------------------
    # batch helpers (reference 1050-1149)
    # ------------------------------------------------------------------
    def _scatter_ifft_crop_batch(self, batch_kspace, s_flat_idx: int = 0):
        """``(B, n_samples)`` unsorted rows -> ``(B, *image_shape)`` (no coil combination)."""
        x = torch.as_tensor(batch_kspace)
        src_dev = x.device
        B = int(x.shape[0])
        st = self._stage
        a = self._stack_arrays_dev(s_flat_idx)
        xd = as_c64(x, self._cdev).reshape(B, 1, -1)
        u = torch.zeros(B, 1, *st.grid_shape, dtype=torch.complex64, device=xd.device)
        st.scatter(xd, a.cellpos, a.w, u, B, a.R, st.G)
        v = st.ifft(u)
        out = torch.empty(B, 1, *st.image_shape, dtype=torch.complex64, device=xd.device)
        st.combine(v, None, out, B, 1, st.ortho)
        return out.reshape(B, *st.image_shape).to(src_dev)

    def _fft_pad_gather_batch(self, batch_imgs, s_flat_idx: int = 0):
        """``(B, *image_shape)`` -> ``(B, n_samples)`` in natural order."""
        x = torch.as_tensor(batch_imgs)
        src_dev = x.device
        B = int(x.shape[0])
        st = self._stage
        a = self._stack_arrays_dev(s_flat_idx)
        xd = as_c64(x, self._cdev).reshape(B, 1, *st.image_shape)
        u = torch.empty(B, 1, *st.grid_shape, dtype=torch.complex64, device=xd.device)
        st.expand(xd, None, u, B, 1, 1.0, x_has_coils=True)
        U = st.fft(u)
        out = torch.empty(B, 1, a.R, dtype=torch.complex64, device=xd.device)
        st.gather(U, a.cellpos, a.w_fwd, out, B, a.R, st.G)
        return out.reshape(B, a.R).to(src_dev)
