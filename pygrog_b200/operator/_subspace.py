"""Low-rank subspace operators on the GPU.

Mirrors ``gadgets/_subspace.py`` (``SubspaceProjection`` 44-90,
``with_subspace`` 96-131, ``SubspaceSparseFFT`` 134-508) and
``_toep/_sub_toep.py`` (``SubspaceToeplitzOp`` 30-303) of
FiRMLAB-Pisa/pygrog.  With basis ``Phi (K, T)`` and the sample weights
``w = pre_w * sqrt_w`` of the GROG plan:

    forward:  y_c[i] = w_i * sum_k conj(Phi[k, t_i]) * FFT(pad(S_c x_k))[cell_i]
    adjoint:  x_k    = sum_c conj(S_c) crop(IFFT(sum_i w_i Phi[k, t_i] y_c[i] delta_cell_i))
    normal (Toeplitz): x_k <- sum_c conj(S_c) crop(IFFT(sum_k' P[k, k'] FFT(pad(S_c x_k'))))
              with P[g, k, k'] = sum_{i: cell_i = g} w_i^2 Phi[k, t_i] conj(Phi[k', t_i]).

The reference loops over coils and components with one scatter / FFT per
(c, k); here one kernel reads every sample once for all K components, the
FFTs run batched over (frames, K, C), and the K x K PSF matvec is one kernel.

``SubspaceMaskedFFT`` (``gadgets/_subspace.py:761-1004``) wraps a
:class:`MaskedFFT` whose grid carries the encoding axis: with ``t(g)`` the
encoding index of grid cell ``g`` and the reference's centred transform over
every grid axis,

    forward:  y_c = sum_k conj(Phi[k, t]) * mask * FFT(pad(S_c x_k))
    adjoint:  x_k = sum_c conj(S_c) crop(IFFT(mask * Phi[k, t] * y_c))
    normal (Toeplitz): the K x K PSF P[g, a, b] = density[g] Phi[b, t(g)]
              conj(Phi[a, t(g)]) of ``_toep/_sub_toep.py:64-105`` (the
              reference builds the masked PSF in this order; for a complex
              basis it is the conjugate of the nested operator's).
"""

from __future__ import annotations

__all__ = ["SubspaceMaskedFFT", "SubspaceProjection", "SubspaceSparseFFT", "SubspaceToeplitzOp", "with_subspace"]

import numpy as np
import torch

from .. import _ext, _lib
from .._fftops import as_c64, with_torch
from .._solve import SolveMixin


class SubspaceProjection:
    """Low-rank projection by truncated SVD (reference ``SubspaceProjection``)."""

    def __init__(self, n_components: int):
        self.n_components = n_components
        self._basis = None

    def fit(self, calib_data) -> "SubspaceProjection":
        U, _S, _Vh = torch.linalg.svd(torch.as_tensor(calib_data), full_matrices=False)
        self._basis = U[:, : self.n_components].T.conj()
        return self

    @property
    def basis(self) -> torch.Tensor:
        if self._basis is None:
            raise RuntimeError("Call fit() first.")
        return self._basis

    @with_torch
    def forward(self, data: torch.Tensor) -> torch.Tensor:
        flat = data.reshape(data.shape[0], -1)
        return (self.basis.to(flat.device) @ flat).reshape(self.n_components, *data.shape[1:])

    @with_torch
    def adjoint(self, coefficients: torch.Tensor) -> torch.Tensor:
        flat = coefficients.reshape(self.n_components, -1)
        return (self.basis.to(flat.device).conj().T @ flat).reshape(-1, *coefficients.shape[1:])


def with_subspace(base_op, subspace_basis, encoding_axis: int = -4, *, toeplitz=None):
    """Wrap a :class:`SparseFFT` or :class:`MaskedFFT` with a subspace projection
    (reference ``with_subspace``, ``gadgets/_subspace.py:91-122``)."""
    from ._masked_fft import MaskedFFT

    if isinstance(base_op, MaskedFFT):
        return SubspaceMaskedFFT(base_op, subspace_basis, encoding_axis=encoding_axis, toeplitz=toeplitz)
    return SubspaceSparseFFT(base_op, subspace_basis, encoding_axis=encoding_axis, toeplitz=toeplitz)


class SubspaceSparseFFT(SolveMixin):
    """SparseFFT with low-rank subspace projection (reference ``SubspaceSparseFFT``).

    ``k_chunk`` is accepted for API compatibility; every component is handled
    in one pass."""

    def __init__(self, base_op, subspace_basis, encoding_axis: int = -4, *, toeplitz=None, k_chunk: int = 1):
        self._base = base_op
        self.basis = torch.as_tensor(subspace_basis)
        self.K, self.T = (int(s) for s in self.basis.shape)
        self.encoding_axis = encoding_axis
        self.k_chunk = max(1, int(k_chunk))
        self.grid_shape = base_op.grid_shape
        self.image_shape = base_op.image_shape
        self.natural_shape = tuple(base_op.natural_shape)
        self.stack_shape = tuple(getattr(base_op, "stack_shape", ()) or ())
        self.smaps = getattr(base_op, "smaps", None)
        nat_ndim = len(self.natural_shape)
        ax = encoding_axis if encoding_axis >= 0 else encoding_axis + (1 + nat_ndim)
        self._t_axis_in_nat = ax - 1
        if not (0 <= self._t_axis_in_nat < nat_ndim):
            raise ValueError(
                f"encoding_axis={encoding_axis} does not land inside natural_shape "
                f"{base_op.natural_shape} (computed nat-axis {self._t_axis_in_nat})"
            )
        if self.natural_shape[self._t_axis_in_nat] != self.T:
            raise ValueError(
                f"basis T={self.T} does not match natural_shape"
                f"[{self._t_axis_in_nat}]={self.natural_shape[self._t_axis_in_nat]}"
            )
        if toeplitz is None:
            toeplitz = bool(getattr(base_op, "toeplitz", False))
        self.toeplitz = bool(toeplitz)
        self._toep_op = None
        self._cdev = base_op._cdev
        self._single_ndim = 1 + len(self.image_shape)  # (K, *image) frames for the device CG
        dev = self._cdev
        self._basis_d = as_c64(self.basis, dev).contiguous()
        view = [1] * nat_ndim
        view[self._t_axis_in_nat] = self.T
        self._tidx = (torch.arange(self.T, dtype=torch.int32, device=dev).view(view)
                      .expand(self.natural_shape).reshape(-1).contiguous())
        self._w2 = {}

    # -- helpers -----------------------------------------------------------------
    def _require_smaps(self):
        if self._base.smaps is None:
            raise NotImplementedError("SubspaceSparseFFT requires base_op.smaps")

    def _weights(self, s: int):
        """(stack arrays, w = pre_w * sqrt_w natural, w * ortho)."""
        if s not in self._w2:
            a = self._base._stack_arrays_dev(s)
            w2 = (a.w * a.w).contiguous()
            self._w2[s] = (a, w2, (w2 * self._base._stage.ortho).contiguous())
        return self._w2[s]

    def _split(self, x: torch.Tensor, single_ndim: int):
        prefix = tuple(int(v) for v in x.shape[: x.ndim - single_ndim])
        s_shape = self.stack_shape
        if s_shape:
            if len(prefix) < len(s_shape) or tuple(prefix[-len(s_shape):]) != s_shape:
                raise ValueError(f"input prefix {prefix} must end with stack_shape {s_shape}")
            B_shape = prefix[: len(prefix) - len(s_shape)]
        else:
            B_shape = prefix
        S = int(np.prod(s_shape)) if s_shape else 1
        Bt = int(np.prod(B_shape)) if B_shape else 1
        return prefix, B_shape, S, Bt

    # -- cores (device tensors, one stack element) --------------------------------
    def _adjoint_core(self, y: torch.Tensor, s: int) -> torch.Tensor:
        """y (Bt, C, R) -> (Bt, K, *image)."""
        Bt, C, R = y.shape
        st = self._base._stage
        a, w2, _ = self._weights(s)
        u = torch.zeros(Bt, self.K, C, *st.grid_shape, dtype=torch.complex64, device=y.device)
        _lib.call("pgb_subspace_scatter", y.data_ptr(), a.cellpos.data_ptr(), w2.data_ptr(), self._tidx.data_ptr(),
                  self._basis_d.data_ptr(), u.data_ptr(), Bt, C, self.K, self.T, R, st.G, _lib.stream_ptr(y.device))
        v = st.ifft(u)
        out = torch.empty(Bt, self.K, *st.image_shape, dtype=torch.complex64, device=y.device)
        st.combine(v, self._base._smaps_d, out, Bt * self.K, C, st.ortho)
        return out

    def _forward_core(self, x: torch.Tensor, s: int) -> torch.Tensor:
        """x (Bt, K, *image) -> (Bt, C, R)."""
        Bt = int(x.shape[0])
        st = self._base._stage
        sm = self._base._smaps_d
        C = int(sm.shape[0])
        a, _, w2o = self._weights(s)
        u = torch.empty(Bt, self.K, C, *st.grid_shape, dtype=torch.complex64, device=x.device)
        st.expand(x, sm, u, Bt * self.K, C, 1.0, x_has_coils=False)
        U = st.fft(u)
        out = torch.empty(Bt, C, a.R, dtype=torch.complex64, device=x.device)
        _lib.call("pgb_subspace_gather", U.data_ptr(), a.cellpos.data_ptr(), w2o.data_ptr(), self._tidx.data_ptr(),
                  self._basis_d.data_ptr(), out.data_ptr(), Bt, C, self.K, self.T, a.R, st.G,
                  _lib.stream_ptr(x.device))
        return out

    # -- public ------------------------------------------------------------------
    @with_torch
    def adjoint(self, sparse_kspace):
        """Sparse k-space ``(*B, *S, C, *natural)`` -> coefficients ``(*B, *S, K, *image)``."""
        self._require_smaps()
        x = torch.as_tensor(sparse_kspace)
        src = x.device
        nat_ndim = len(self.natural_shape)
        if x.ndim < 1 + nat_ndim:
            raise ValueError(f"Expected (C, *natural)=(C, {self.natural_shape}); got {tuple(x.shape)}")
        prefix, B_shape, S, Bt = self._split(x, 1 + nat_ndim)
        C = int(x.shape[x.ndim - 1 - nat_ndim])
        xd = as_c64(x, self._cdev).reshape(Bt, S, C, -1)
        outs = [self._adjoint_core(xd[:, s].contiguous(), s) for s in range(S)]
        out = torch.stack(outs, dim=1)
        return out.reshape(*prefix, self.K, *self.image_shape).to(src)

    @with_torch
    def forward(self, coeffs):
        """Coefficients ``(*B, *S, K, *image)`` -> sparse k-space ``(*B, *S, C, *natural)``."""
        self._require_smaps()
        x = torch.as_tensor(coeffs)
        src = x.device
        single = 1 + len(self.image_shape)
        if x.shape[x.ndim - single] != self.K:
            raise ValueError(f"coeffs.shape[0]={x.shape[x.ndim - single]} != K={self.K}")
        if tuple(int(v) for v in x.shape[x.ndim - single + 1:]) != tuple(self.image_shape):
            raise ValueError(f"coeffs spatial {tuple(x.shape[x.ndim - single + 1:])} != image_shape "
                             f"{tuple(self.image_shape)}")
        prefix, B_shape, S, Bt = self._split(x, single)
        xd = as_c64(x, self._cdev).reshape(Bt, S, self.K, *self.image_shape)
        outs = [self._forward_core(xd[:, s].contiguous(), s) for s in range(S)]
        out = torch.stack(outs, dim=1)
        C = int(out.shape[2])
        return out.reshape(*prefix, C, *self.natural_shape).to(src)

    def __call__(self, x, adjoint=False):
        return self.adjoint(x) if adjoint else self.forward(x)

    def _toeplitz(self):
        if self._toep_op is None:
            self._toep_op = SubspaceToeplitzOp(self, device=self._cdev)
        return self._toep_op

    @with_torch
    def normal(self, coeffs):
        """``A^H A coeffs`` (Toeplitz K x K PSF when ``self.toeplitz``)."""
        if self.toeplitz:
            return self._toeplitz()(coeffs)
        return self.adjoint(self.forward(coeffs))

    def _normal_frames_into(self, x: torch.Tensor, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """``out[f] = A^H A x[f] + damp x[f]`` for frames ``x (F, K, *image)`` on the device."""
        if self.stack_shape:
            raise NotImplementedError("frame-batched normal operator covers unstacked operators")
        if self.toeplitz:
            return self._toeplitz()._apply_frames(x, 0, out, damp)
        y = self._adjoint_core(self._forward_core(x, 0), 0)
        torch.add(y, x, alpha=damp, out=out) if damp else out.copy_(y)
        return out

    def _normal_into(self, x: torch.Tensor, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """``out = A^H A x + damp x`` for one frame ``(K, *image)`` on the device."""
        if self.stack_shape:
            raise NotImplementedError("device CG loop covers unstacked operators")
        if self.toeplitz:
            return self._toeplitz()._apply_frames(x.unsqueeze(0), 0, out.unsqueeze(0), damp)
        y = self._adjoint_core(self._forward_core(x.unsqueeze(0), 0), 0)
        torch.add(y[0], x, alpha=damp, out=out) if damp else out.copy_(y[0])
        return out


class SubspaceMaskedFFT(SubspaceSparseFFT):
    """MaskedFFT with low-rank subspace projection (reference ``SubspaceMaskedFFT``,
    ``gadgets/_subspace.py:761-1004``).

    The base operator's grid (its natural shape) carries the encoding axis
    ``T`` (``encoding_axis`` counts in the layout ``(C, *grid)``; default -3:
    ``(C, T, gy, gx)``).  Gridded k-space ``(*B, *S, C, *grid)`` <->
    coefficients ``(*B, *S, K, *image)``; as in the reference, the centred
    transforms run over every grid axis and the crop pairs grid and image
    axes in order, so the image shape has the grid's rank.  All coils and
    components go through one batched masked transform per stack element.
    """

    def __init__(self, base_op, subspace_basis, encoding_axis: int = -3, *, toeplitz=None):
        self._base = base_op
        self.basis = torch.as_tensor(subspace_basis)
        self.K, self.T = (int(v) for v in self.basis.shape)
        self.encoding_axis = encoding_axis
        self.k_chunk = 1
        self.grid_shape = tuple(base_op.grid_shape)
        self.image_shape = tuple(base_op.image_shape)
        self.natural_shape = tuple(base_op.natural_shape)  # the grid
        self.stack_shape = tuple(getattr(base_op, "stack_shape", ()) or ())
        self.smaps = getattr(base_op, "smaps", None)
        nat_ndim = len(self.natural_shape)
        ax = encoding_axis if encoding_axis >= 0 else encoding_axis + (1 + nat_ndim)
        self._t_axis_in_nat = ax - 1
        if not (0 <= self._t_axis_in_nat < nat_ndim):
            raise ValueError(
                f"encoding_axis={encoding_axis} does not land inside natural_shape "
                f"{base_op.natural_shape} (computed nat-axis {self._t_axis_in_nat})"
            )
        if self.natural_shape[self._t_axis_in_nat] != self.T:
            raise ValueError(
                f"basis T={self.T} does not match natural_shape"
                f"[{self._t_axis_in_nat}]={self.natural_shape[self._t_axis_in_nat]}"
            )
        if toeplitz is None:
            toeplitz = bool(getattr(base_op, "toeplitz", False))
        if toeplitz and getattr(base_op, "density", None) is None:
            raise ValueError("a Toeplitz SubspaceMaskedFFT needs base_op.density")
        self.toeplitz = bool(toeplitz)
        self._toep_op = None
        self._cdev = base_op._cdev
        self._single_ndim = 1 + len(self.image_shape)
        dev = self._cdev
        self._basis_d = as_c64(self.basis, dev).contiguous()
        view = [1] * nat_ndim
        view[self._t_axis_in_nat] = self.T
        # encoding index of every grid cell, and Phi[k, t(g)] on the grid
        self._tcell = (torch.arange(self.T, dtype=torch.int64, device=dev).view(view)
                       .expand(self.natural_shape).reshape(-1).contiguous())
        G = int(np.prod(self.grid_shape))
        self._phi = self._basis_d[:, self._tcell].reshape(1, self.K, 1, G).contiguous()
        self._phi_conj = self._phi.conj().contiguous()

    def _require_smaps(self):
        if self._base.smaps is None:
            raise NotImplementedError("SubspaceMaskedFFT requires base_op.smaps")

    def _adjoint_core(self, y: torch.Tensor, s: int) -> torch.Tensor:
        """y (Bt, C, G) centred grid -> (Bt, K, *image): mask, Phi[k, t], IFFT, crop, coil sum."""
        Bt, C, G = (int(v) for v in y.shape)
        st = self._base._stage
        w = (y.reshape(Bt, 1, C, G) * self._phi).contiguous()  # (Bt, K, C, G)
        u = torch.empty(Bt, self.K, C, *st.grid_shape, dtype=torch.complex64, device=y.device)
        st.shift(w, self._base._mask_d[s], u, Bt * self.K * C, 1.0, to_centred=False)
        v = st.ifft(u)
        out = torch.empty(Bt, self.K, *st.image_shape, dtype=torch.complex64, device=y.device)
        st.combine(v, self._base._smaps_d, out, Bt * self.K, C, st.ortho)
        return out

    def _forward_core(self, x: torch.Tensor, s: int) -> torch.Tensor:
        """x (Bt, K, *image) -> (Bt, C, G) centred grid: smaps, pad, FFT, mask, sum_k conj(Phi[k, t])."""
        Bt = int(x.shape[0])
        st = self._base._stage
        sm = self._base._smaps_d
        C = int(sm.shape[0])
        u = torch.empty(Bt, self.K, C, *st.grid_shape, dtype=torch.complex64, device=x.device)
        st.expand(x, sm, u, Bt * self.K, C, 1.0, x_has_coils=False)
        U = st.fft(u)
        o = torch.empty_like(U)
        st.shift(U, self._base._mask_d[s], o, Bt * self.K * C, st.ortho, to_centred=True)
        return (o.reshape(Bt, self.K, C, st.G) * self._phi_conj).sum(1)


class SubspaceToeplitzOp:
    """``A^H A`` of a :class:`SubspaceSparseFFT` or :class:`SubspaceMaskedFFT`
    with a per-cell K x K PSF (reference ``SubspaceToeplitzOp``; ``psf`` holds
    the PSF on the centred grid in the reference's ``(*grid, K, K)`` layout)."""

    def __init__(self, sub_op: SubspaceSparseFFT, device=None):
        base = sub_op._base
        if base.smaps is None:
            raise NotImplementedError("SubspaceToeplitzOp requires base_op.smaps")
        self._sub = sub_op
        self._base = base
        self.device = torch.device(device) if device is not None else sub_op._cdev
        self.grid_shape = tuple(base.grid_shape)
        self.image_shape = tuple(base.image_shape)
        self.K, self.T = sub_op.K, sub_op.T
        self.stack_shape = sub_op.stack_shape
        st = base._stage
        S = int(np.prod(self.stack_shape)) if self.stack_shape else 1
        basis = sub_op._basis_d
        if isinstance(sub_op, SubspaceMaskedFFT):
            # one encoding index per grid cell: P[g, a, b] = density[g] Phi[b, t(g)]
            # conj(Phi[a, t(g)]), in the order of _toep/_sub_toep.py:64-105
            dens = base.density.to(self.device, torch.float32).reshape(S, st.G)
            Bj = basis[:, sub_op._tcell].T  # (G, K): Phi[k, t(g)]
            P = dens.reshape(S, st.G, 1, 1) * (Bj.conj()[None, :, :, None] * Bj[None, :, None, :])
            P = P.to(torch.complex64).reshape(S, *self.grid_shape, self.K, self.K)
        else:
            nat = sub_op.natural_shape
            n_per = int(np.prod(nat))
            t_nat = sub_op._tidx.to(torch.int64)
            idx_all = base.indices.reshape(S, -1).to(self.device)
            sw_all = base.sqrt_weights.reshape(S, -1).to(self.device, torch.float32)
            sp_all = base.sort_perm.reshape(S, -1).to(self.device)
            psfs = []
            for s in range(S):
                w = sw_all[s] * sw_all[s]
                w_eff = (w * w).contiguous()
                t_sorted = t_nat[sp_all[s] % n_per].contiguous()
                pf = torch.zeros(st.G, self.K, self.K, dtype=torch.complex64, device=self.device)
                _ext.psf_scatter_outer_basis(pf, idx_all[s].contiguous(), w_eff, basis, t_sorted)
                psfs.append(pf.transpose(-2, -1).contiguous())  # P[g, k, k']
            P = torch.stack(psfs).reshape(S, *self.grid_shape, self.K, self.K)
        self.psf = P[0] if not self.stack_shape else P.reshape(*self.stack_shape, *self.grid_shape, self.K, self.K)
        # FFT order, 1/G of the two unscaled transforms folded in
        Pf = torch.fft.ifftshift(P, dim=tuple(range(1, 1 + len(self.grid_shape))))
        self._psf_fft = (Pf.reshape(S, st.G, self.K, self.K) * (1.0 / st.G)).contiguous()

    def _apply_frames(self, x: torch.Tensor, s: int, out: torch.Tensor, damp: float = 0.0) -> torch.Tensor:
        """x (Bt, K, *image) on the device -> out (same shape)."""
        st = self._base._stage
        sm = self._base._smaps_d
        C = int(sm.shape[0])
        Bt = int(x.shape[0])
        u = torch.empty(Bt, self.K, C, *st.grid_shape, dtype=torch.complex64, device=x.device)
        st.expand(x, sm, u, Bt * self.K, C, 1.0, x_has_coils=False)
        U = st.fft(u)
        _lib.call("pgb_psf_apply_kk", U.data_ptr(), self._psf_fft[s].data_ptr(), Bt, self.K, C, st.G,
                  _lib.stream_ptr(x.device))
        V = st.ifft(U)
        st.combine(V, sm, out, Bt * self.K, C, 1.0, add=x if damp else None, add_scale=damp)
        return out

    def __call__(self, coeffs):
        x = torch.as_tensor(coeffs)
        src = x.device
        single = 1 + len(self.image_shape)
        if x.shape[x.ndim - single] != self.K:
            raise ValueError(f"coeffs K-dim {x.shape[x.ndim - single]} != K={self.K}")
        prefix, B_shape, S, Bt = self._sub._split(x, single)
        xd = as_c64(x, self.device).reshape(Bt, S, self.K, *self.image_shape)
        out = torch.empty_like(xd)
        for s in range(S):
            xs = xd[:, s].contiguous()
            os_ = torch.empty_like(xs)
            self._apply_frames(xs, s, os_)
            out[:, s] = os_
        return out.reshape(x.shape).to(src)
