"""GRAPPA unit-shift operators and the fractional-shift GROG table.

Restates the reference algorithm of ``calib/_grappa.py`` (FiRMLAB-Pisa/pygrog):

* ``lstsq`` (``_grappa.py:16-59``): Tikhonov least squares through the
  augmented system ``[A; sqrt(lam) I] X = [B; 0]`` solved by LAPACK gelsd;
* unit operators (``_grappa.py:264-367``): the calibration block is scaled to
  unit Frobenius norm and, per spatial axis, ``S @ G.T = T`` is solved for
  neighbour pairs along that axis;
* fractional powers (``_grappa.py:62-72, 184-208``): ``G^d = expm(d logm G)``
  with ``logm`` through a complex128 eigendecomposition;
* the table (``_grappa.py:75-181``): ``nsteps = 2*radius/10^-p + 1`` shifts
  per axis and ``table[i*n + j] = Gx[j] @ Gy[i]`` (2-D) or
  ``table[i*n^2 + j*n + k] = Gx[k] @ Gy[j] @ Gz[i]`` (3-D).

The operator naming follows the reference exactly, including its axis
convention: in 2-D ``Gx`` shifts along spatial axis 0 and ``Gy`` along axis
1; in 3-D ``Gz`` shifts along axis 0, ``Gy`` along axis 1, ``Gx`` along
axis 2.  The same library calls (torch.linalg on the host CPU) are used so
that a table computed here is bit-identical to the reference's on the same
machine.

The fit is tiny (a few C x C solves) and stays on the host CPU in the
caller's precision; ``fit_dtype=torch.complex128`` runs the whole fit in
FP64 and casts only the finished table.
"""

from __future__ import annotations

__all__ = ["KernelTable", "lstsq", "grappa_power", "prepare_grappa_table", "table_factors", "train_grappa"]

from types import SimpleNamespace

import numpy as np
import torch


def lstsq(A, b, lamda: float = 0.0):
    """Tikhonov-regularised least squares ``min ||A X - B||^2 + lamda ||X||^2``."""
    A_t = torch.as_tensor(A)
    b_t = torch.as_tensor(b)
    n = A_t.shape[-1]
    if lamda > 0:
        reg = (lamda**0.5) * torch.eye(n, dtype=A_t.dtype, device=A_t.device)
        if A_t.dim() > 2:
            reg = reg.expand(*A_t.shape[:-2], n, n)
        pad = torch.zeros(*A_t.shape[:-2], n, b_t.shape[-1], dtype=b_t.dtype, device=b_t.device)
        A_t = torch.cat([A_t, reg], dim=-2)
        b_t = torch.cat([b_t, pad], dim=-2)
    sol = torch.linalg.lstsq(A_t, b_t, driver="gelsd").solution
    return sol.numpy() if isinstance(A, np.ndarray) else sol


def _logm(A: torch.Tensor) -> torch.Tensor:
    """Matrix logarithm ``V diag(log lam) V^-1`` evaluated in complex128."""
    out_dtype = A.dtype if A.is_complex() else torch.complex64
    vals, vecs = torch.linalg.eig(A.to(torch.complex128))
    return (vecs @ torch.diag_embed(torch.log(vals)) @ torch.linalg.inv(vecs)).to(out_dtype)


def grappa_power_device(G_unit: torch.Tensor, exponents: torch.Tensor) -> torch.Tensor:
    """``G_unit ** e`` for each exponent in complex128 on ``G_unit``'s device:
    ``expm(e logm(G))`` of ``calib/_grappa.py:184-208``, evaluated in the
    eigenbasis of the logarithm, ``V diag(exp(e l)) V^-1`` with
    ``logm(G) = V diag(l) V^-1`` (the eigendecomposition form of
    :func:`_logm`).  The ``C x C`` eigendecomposition (complex128, C <= 32)
    runs on the host -- there is no eigensolver for non-Hermitian matrices on
    the GPU here; the exponentials and the products of every power run
    batched on the device.  This form is used instead of the device matrix
    exponential, whose scaling and squaring loses accuracy on the large
    norms of nearly singular operators (strong regularisation off, many
    coils), while the host FP64 ``matrix_exp`` and this form agree to FP64
    rounding."""
    dev = G_unit.device
    L = _logm(G_unit.detach().to("cpu", torch.complex128))
    lam, V = torch.linalg.eig(L)
    Vi = torch.linalg.inv(V)
    lam, V, Vi = lam.to(dev), V.to(dev), Vi.to(dev)
    e = torch.as_tensor(exponents, dtype=torch.float64, device=dev).to(lam.dtype)
    ph = torch.exp(e.view(-1, 1) * lam.view(1, -1))  # (n_steps, C)
    return (V.unsqueeze(0) * ph.unsqueeze(1)) @ Vi.unsqueeze(0)


def grappa_power(G_unit: torch.Tensor, exponents: torch.Tensor) -> torch.Tensor:
    """Stack of ``G_unit ** e`` for each exponent, shape ``(len(e), C, C)``."""
    G_unit = torch.as_tensor(G_unit)
    e = torch.as_tensor(exponents, dtype=torch.float32)
    L = _logm(G_unit)
    return torch.linalg.matrix_exp(e.to(L.dtype).view(-1, 1, 1) * L.unsqueeze(0)).to(G_unit.dtype)


def _unit_operators(calib: torch.Tensor, lamda: float) -> list[torch.Tensor]:
    """Per-axis unit shift operators; entry ``a`` shifts along spatial axis a."""
    calib = calib / torch.linalg.norm(calib)
    cal = calib.movedim(0, -1)  # (*spatial, C)
    nc = cal.shape[-1]
    ops = []
    for axis in range(cal.ndim - 1):
        m = cal.shape[axis] - 1
        src = cal.narrow(axis, 0, m).reshape(-1, nc)
        dst = cal.narrow(axis, 1, m).reshape(-1, nc)
        ops.append(lstsq(src, dst, lamda).mT)
    return ops


def _unit_operators_device(calib: torch.Tensor, lamda: float, device) -> list[torch.Tensor]:
    """The unit operators of :func:`_unit_operators` fitted in FP64 with the
    O(samples) work on the GPU: the Gram matrices ``src^H src`` and
    ``src^H dst`` of every axis's neighbour pairs are accumulated in FP64 by
    ``pgb_coil_cross_covariance``; the regularised ``C x C`` normal equations
    ``(src^H src + lamda I) X = src^H dst`` (the calibration block scaled to
    unit norm, as in the reference) are solved on the host in FP64.  The
    samples enter as complex64 (k-space calibration data).  The
    least-squares solution equals the augmented-system one of
    ``_grappa.py:16-59`` up to FP64 rounding (the regularised Gram matrix has
    condition number <= 1 / lamda + 1)."""
    from .. import _lib

    dev = torch.device(device)
    cal = torch.as_tensor(calib).to(dev)
    norm2 = float(torch.linalg.norm(cal.to(torch.complex128)) ** 2)
    cal = cal.to(torch.complex64)
    nc = int(cal.shape[0])
    st = _lib.stream_ptr(dev)
    ops = []
    for axis in range(1, cal.ndim):
        m = cal.shape[axis] - 1
        # (C, M) coil-major copies of the source and target samples of this axis
        src = cal.narrow(axis, 0, m).reshape(nc, -1).contiguous()
        dst = cal.narrow(axis, 1, m).reshape(nc, -1).contiguous()
        M = int(src.shape[1])
        g_ss = torch.empty(nc, nc, dtype=torch.complex128, device=dev)
        g_sd = torch.empty(nc, nc, dtype=torch.complex128, device=dev)
        _lib.call("pgb_coil_cross_covariance", src.data_ptr(), src.data_ptr(), M, nc, g_ss.data_ptr(), st)
        _lib.call("pgb_coil_cross_covariance", src.data_ptr(), dst.data_ptr(), M, nc, g_sd.data_ptr(), st)
        # kernel: sum_m a[i, m] conj(b[j, m]); src^H src = its conjugate, likewise src^H dst
        A = g_ss.conj() / norm2 + lamda * torch.eye(nc, dtype=torch.complex128, device=dev)
        Bm = g_sd.conj() / norm2
        X = torch.linalg.solve(A, Bm)  # FP64 on the device
        ops.append(X.mT)
    return ops


def train_grappa(train_data, lamda: float | None = None, device=None) -> SimpleNamespace:
    """Unit GROG operators ``x``, ``y`` (and ``z`` in 3-D) from a Cartesian ACR.

    With ``device`` (a CUDA device) the fit runs in FP64 with its Gram
    matrices accumulated on that GPU (:func:`_unit_operators_device`)."""
    if lamda is None:
        lamda = 0.01
    t = torch.as_tensor(train_data)
    ndim = t.ndim - 1
    ops = _unit_operators_device(t, lamda, device) if device is not None else _unit_operators(t, lamda)
    if ndim == 2:
        return SimpleNamespace(x=ops[0], y=ops[1], z=None)
    if ndim == 3:
        return SimpleNamespace(x=ops[2], y=ops[1], z=ops[0])
    raise ValueError(f"GROG interpolation only supports 2D or 3D data, got {ndim}D")


def prepare_grappa_table(Gx, Gy, Gz, nsteps: int, ndim: int) -> torch.Tensor:  # noqa: ARG001
    """Product table of per-axis fractional operators (row-major shift index)."""
    Gx = torch.as_tensor(Gx)
    Gy = torch.as_tensor(Gy)
    if ndim == 2:
        return (Gx[None] @ Gy[:, None]).reshape(-1, *Gx.shape[-2:])
    if ndim == 3:
        if Gz is None:
            raise ValueError("3D interpolation requires Z operator")
        Gz = torch.as_tensor(Gz)
        return (Gx[None, None] @ Gy[None, :, None] @ Gz[:, None, None]).reshape(-1, *Gx.shape[-2:])
    raise ValueError(f"GROG interpolation only supports 2D or 3D data, got {ndim}D")


def shift_steps(radius: float, precision: int) -> tuple[float, int, torch.Tensor]:
    """Quantisation step, number of steps and the float32 shift of each step."""
    stepsize = 10 ** (-precision)
    nsteps = int(2 * radius / stepsize + 1)
    deltas = (torch.arange(nsteps).float() - (nsteps - 1) / 2) * stepsize
    return stepsize, nsteps, deltas


def table_factors(Gx, Gy, Gz, ndim: int):
    """Split the table as ``T[e] = outer[e % n] @ inner[e // n]``.

    2-D: ``T[i*n + j] = Gx[j] @ Gy[i]``          -> outer = Gx, inner = Gy.
    3-D: ``T[i*n^2 + j*n + k] = Gx[k] @ Gy[j] @ Gz[i]``
                                                   -> outer = Gx,
                                                      inner[i*n + j] = Gy[j] @ Gz[i].
    The fused kernels keep ``inner`` in shared memory and apply ``outer`` once
    per run of replicas that share its index and target cell.
    """
    Gx = torch.as_tensor(Gx)
    Gy = torch.as_tensor(Gy)
    if ndim == 2:
        return Gx.contiguous(), Gy.contiguous()
    Gz = torch.as_tensor(Gz)
    inner = (Gy[None, :] @ Gz[:, None]).reshape(-1, *Gx.shape[-2:])
    return Gx.contiguous(), inner.contiguous()


def KernelTable(
    train_data,
    radius: float,
    precision: int = 1,
    lamda: float = 0.01,
    fit_dtype: torch.dtype | None = None,
    return_factors: bool = False,
    fit_device=None,
):
    """Return ``(table (nsteps**ndim, C, C) ndarray, nsteps, ndim)``.

    ``fit_dtype`` (e.g. ``torch.complex128``) runs the least squares, logm and
    expm in that precision and casts the table back to the ACR's dtype.
    With ``return_factors`` a fourth item ``(outer, inner)`` is returned (see
    :func:`table_factors`), cast like the table.  ``fit_device`` (a CUDA
    device) runs the fit in FP64 on that GPU: the least-squares Gram
    matrices and solves (:func:`_unit_operators_device`), the matrix
    exponentials of the fractional powers and the table product
    (:func:`grappa_power_device`); only the ``C x C`` eigendecomposition
    behind each logarithm runs on the host, and the finished table is copied
    to the host.
    """
    t = torch.as_tensor(np.asarray(train_data)) if isinstance(train_data, np.ndarray) else torch.as_tensor(train_data)
    t = t.detach().cpu()
    out_dtype = t.dtype if t.is_complex() else torch.complex64
    if fit_device is not None and t.dtype == torch.complex128:
        fit_device = None  # complex128 calibration data: the host FP64 fit keeps every bit
        fit_dtype = torch.complex128
    if fit_dtype is not None and fit_device is None:
        t = t.to(fit_dtype)
    ops = train_grappa(t, lamda, device=fit_device)
    _, nsteps, deltas = shift_steps(radius, precision)
    # the device fit stays in FP64 on the GPU through the powers and the product
    power = grappa_power_device if fit_device is not None else grappa_power
    Gx = power(ops.x, deltas)
    Gy = power(ops.y, deltas)
    if ops.z is not None:
        Gz = power(ops.z, deltas)
        ndim = 3
    else:
        Gz = None
        ndim = 2
    table = prepare_grappa_table(Gx, Gy, Gz, nsteps, ndim).to(out_dtype).cpu()
    if return_factors:
        outer, inner = table_factors(Gx, Gy, Gz, ndim)
        return table.numpy(), nsteps, ndim, (outer.to(out_dtype).cpu(), inner.to(out_dtype).cpu())
    return table.numpy(), nsteps, ndim


def eigen_factors(train_data, radius: float, precision: int = 1, lamda: float = 0.01,
                  fit_dtype: torch.dtype | None = None) -> SimpleNamespace:
    """Eigendecompositions of the per-axis shift generators behind the table.

    The reference forms each fractional operator as ``G_a(d) = expm(d L_a)``
    with ``L_a = logm(G_a)`` cast to the ACR's dtype (``_grappa.py:62-72,
    184-208``).  With ``L_a = V_a diag(l_a) V_a^-1`` (complex128 ``eig``) this is
    ``G_a(d) = V_a diag(exp(d l_a)) V_a^-1``, so the table product
    ``T[i, j, k] = Gx(d_k) Gy(d_j) Gz(d_i)`` becomes fixed dense basis changes
    with per-replica diagonal phases in between (the tensor-core gridder).

    Returns ``ndim``, ``nsteps``, the float32 ``deltas`` and ``axes``: the
    ``(V, l)`` pairs (complex128) in the order the forward applies them
    (3-D: z, y, x; 2-D: y, x), matching the table index split
    ``e = q * nsteps + k`` with ``q = i * nsteps + j`` (3-D) or ``q = i`` (2-D).
    """
    t = torch.as_tensor(np.asarray(train_data)) if isinstance(train_data, np.ndarray) else torch.as_tensor(train_data)
    t = t.detach().cpu()
    if fit_dtype is not None:
        t = t.to(fit_dtype)
    ops = train_grappa(t, lamda)
    _, nsteps, deltas = shift_steps(radius, precision)
    order = [ops.z, ops.y, ops.x] if ops.z is not None else [ops.y, ops.x]
    axes = []
    for G in order:
        L = _logm(torch.as_tensor(G))
        lam, V = torch.linalg.eig(L.to(torch.complex128))
        axes.append((V, lam))
    return SimpleNamespace(ndim=len(order), nsteps=int(nsteps), deltas=deltas, axes=axes)
