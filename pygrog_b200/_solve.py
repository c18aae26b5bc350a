"""Iterative solvers: CG with device-side FP64 scalars, LSMR, ``solve``.

Mirrors ``_solve/_solvers.py`` (``cg`` 49-139, ``lsmr`` 145-262, ``solve``
268-302) and ``_solve/_mixin.py`` (``SolveMixin`` 84-158) of
FiRMLAB-Pisa/pygrog.

CG on an operator of this package runs as a fixed sequence of kernels per
iteration -- ``Ap = A^H A p + damp p`` (Toeplitz or fused forward/adjoint),
FP64 ``<p, Ap>``, x/r update, FP64 ``|r|^2`` with the relative-residual test,
p update -- with every scalar kept in device memory and a device flag
replacing the host-side ``break``.  Without a callback one iteration is
captured in a CUDA graph and replayed ``max_iter`` times: no host
synchronisation inside the loop.  Other duck-typed operators use the
reference recurrence with torch tensors (inner products in FP64).
"""

from __future__ import annotations

__all__ = ["cg", "lsmr", "solve", "SolveMixin", "DeviceCG", "BatchedDeviceCG", "DeviceLSMR"]

import gc
import math
import weakref
from collections.abc import Callable
from typing import Any

import numpy as np
import torch

from . import _lib


def _normalize_kspace_shape(op: Any, b: torch.Tensor) -> torch.Tensor:
    nat = getattr(op, "natural_shape", None)
    if nat is None or len(nat) <= 1:
        return b
    nat = tuple(int(s) for s in nat)
    n = int(np.prod(nat))
    if b.shape[-1] != n:
        return b
    return b.reshape(*b.shape[:-1], *nat)


def _vdot_re64(a: torch.Tensor, b: torch.Tensor) -> torch.Tensor:
    return torch.vdot(a.reshape(-1).to(torch.complex128), b.reshape(-1).to(torch.complex128)).real


class DeviceCG:
    """CG state for one frame on the device (FP64 scalars, optional CUDA graph)."""

    def __init__(self, op, AHb: torch.Tensor, damp: float, tol: float, x0=None, weak_op: bool = False):
        # a solver cached on its operator refers to it weakly: no reference cycle whose
        # collection (at any time, e.g. inside another graph capture) would free a graph
        self.op = weakref.proxy(op) if weak_op else op
        dev = AHb.device
        self.damp = float(damp)
        self.x = torch.zeros_like(AHb) if x0 is None else x0.to(dev, torch.complex64).clone()
        self.Ap = torch.empty_like(AHb)
        if x0 is None:
            self.r = AHb.clone()
        else:
            op._normal_into(self.x, self.Ap, self.damp)
            self.r = AHb - self.Ap
        self.p = self.r.clone()
        self.n = int(AHb.numel())
        lib = _lib.load_library()
        nbytes = int(lib.pgb_reduce_scratch_bytes())
        self.scratch = torch.zeros((nbytes + 7) // 8, dtype=torch.float64, device=dev)
        self.scal = torch.zeros(8, dtype=torch.float64, device=dev)
        self.scal[6] = float(tol)
        self.tol = float(tol)
        st = _lib.stream_ptr(dev)
        _lib.call("pgb_dot_f64", self.r.data_ptr(), None, self.n, self.scratch.data_ptr(),
                  self.scal.data_ptr(), 0, 2, st)
        self.graph = None

    def reset(self, AHb: torch.Tensor, x0=None):
        """Start a new solve in the same buffers (a captured iteration graph stays valid)."""
        if x0 is None:
            self.x.zero_()
            self.r.copy_(AHb)
        else:
            self.x.copy_(x0)
            self.op._normal_into(self.x, self.Ap, self.damp)
            torch.sub(AHb, self.Ap, out=self.r)
        self.p.copy_(self.r)
        self.scal.zero_()
        self.scal[6] = self.tol
        _lib.call("pgb_dot_f64", self.r.data_ptr(), None, self.n, self.scratch.data_ptr(),
                  self.scal.data_ptr(), 0, 2, _lib.stream_ptr(self.p.device))

    def step(self):
        st = _lib.stream_ptr(self.p.device)
        self.op._normal_into(self.p, self.Ap, self.damp)
        _lib.call("pgb_dot_f64", self.p.data_ptr(), self.Ap.data_ptr(), self.n, self.scratch.data_ptr(),
                  self.scal.data_ptr(), 1, 0, st)
        # x, r update and rr = |r|^2 with the residual check, one pass
        _lib.call("pgb_cg_update_xr_rr", self.x.data_ptr(), self.r.data_ptr(), self.p.data_ptr(),
                  self.Ap.data_ptr(), self.n, self.scal.data_ptr(), self.scratch.data_ptr(), st)
        _lib.call("pgb_cg_update_p", self.p.data_ptr(), self.r.data_ptr(), self.n, self.scal.data_ptr(),
                  self.scratch.data_ptr(), st)

    def capture(self):
        """Capture one iteration in a CUDA graph (after a warm-up of the FFT plans)."""
        side = torch.cuda.Stream(self.p.device)
        side.wait_stream(torch.cuda.current_stream(self.p.device))
        saved = [t.clone() for t in (self.x, self.r, self.p, self.scal)]
        with torch.cuda.stream(side):
            self.step()  # warm-up: cuFFT plans and workspaces exist before capture
        torch.cuda.current_stream(self.p.device).wait_stream(side)
        for t, v in zip((self.x, self.r, self.p, self.scal), saved):
            t.copy_(v)
        g = torch.cuda.CUDAGraph()
        gc_on = gc.isenabled()
        gc.disable()  # no collection (and no CUDA frees it may trigger) while capturing
        try:
            with torch.cuda.graph(g):
                self.step()
        finally:
            if gc_on:
                gc.enable()
        self.graph = g

    def run(self, max_iter: int, callback: Callable | None = None, use_graph: bool = True):
        if callback is None and use_graph and max_iter > 1:
            if self.graph is None:
                self.capture()
            for _ in range(max_iter):
                self.graph.replay()
            return self.x
        for k in range(max_iter):
            self.step()
            if callback is not None or self.scal[6] > 0:
                rel = float(self.scal[4].item())
                if callback is not None:
                    callback(k, self.x, rel)
                if self.scal[5].item() != 0.0:
                    break
        return self.x


class BatchedDeviceCG:
    """Independent CG solves of up to ``frames`` systems in lock step: one
    frame-batched normal operator per iteration and per-frame FP64 scalars
    (each frame follows the single-frame recurrence of ``DeviceCG``, with its
    own alpha, beta, residual and done flag).  The buffers persist, so one
    object serves many batches (``load`` F <= frames right-hand sides, then
    ``run``); everything is stream-ordered on the current stream."""

    def __init__(self, op, frames: int, single_shape, device, damp: float = 0.0, tol: float = 0.0):
        self.op = op
        self.cap = int(frames)
        self.damp = float(damp)
        self.tol = float(tol)
        shape = (self.cap, *tuple(int(s) for s in single_shape))
        self._x = torch.zeros(shape, dtype=torch.complex64, device=device)
        self._r = torch.empty_like(self._x)
        self._p = torch.empty_like(self._x)
        self._Ap = torch.empty_like(self._x)
        self.n = int(self._x[0].numel())
        self.words = (int(_lib.load_library().pgb_reduce_scratch_bytes()) + 7) // 8
        self.scratch = torch.zeros(self.cap * self.words, dtype=torch.float64, device=device)
        self._scal = torch.zeros(self.cap, 8, dtype=torch.float64, device=device)
        self.F = 0
        self._graphs: dict = {}
        self._pool = None

    def load(self, AHb: torch.Tensor):
        """Start from x = 0 with right-hand sides ``AHb (F, *single)``."""
        F = int(AHb.shape[0])
        if not 1 <= F <= self.cap:
            raise ValueError(f"BatchedDeviceCG: {F} frames, capacity {self.cap}")
        self.F = F
        self.x, self.r, self.p, self.Ap = (t[:F] for t in (self._x, self._r, self._p, self._Ap))
        self.scal = self._scal[:F]
        st = _lib.stream_ptr(AHb.device)
        self.x.zero_()
        self.r.copy_(AHb)
        self.p.copy_(AHb)
        self.scal.zero_()
        self.scal[:, 6] = self.tol
        _lib.call("pgb_dot_f64_batched", self.r.data_ptr(), None, self.n, F, self.scratch.data_ptr(),
                  self.scal.data_ptr(), 0, 2, st)

    def step(self):
        st = _lib.stream_ptr(self.p.device)
        F = self.F
        self.op._normal_frames_into(self.p, self.Ap, self.damp)
        _lib.call("pgb_dot_f64_batched", self.p.data_ptr(), self.Ap.data_ptr(), self.n, F,
                  self.scratch.data_ptr(), self.scal.data_ptr(), 1, 0, st)
        _lib.call("pgb_cg_update_xr_rr_batched", self.x.data_ptr(), self.r.data_ptr(), self.p.data_ptr(),
                  self.Ap.data_ptr(), self.n, F, self.scal.data_ptr(), self.scratch.data_ptr(), st)
        _lib.call("pgb_cg_update_p_batched", self.p.data_ptr(), self.r.data_ptr(), self.n, F,
                  self.scal.data_ptr(), self.scratch.data_ptr(), st)

    def capture(self, frames: int, max_iter: int):
        """Record ``max_iter`` iterations for ``frames`` frames as one CUDA graph
        (operator and FFT plans must have run once for this shape already).
        Graphs of one object share a memory pool: replay them on one stream."""
        self.load(torch.zeros((frames, *self._x.shape[1:]), dtype=torch.complex64, device=self._x.device))
        if self._pool is None:
            self._pool = torch.cuda.graph_pool_handle()
        g = torch.cuda.CUDAGraph()
        gc_on = gc.isenabled()
        gc.disable()  # no collection (and no CUDA frees it may trigger) while capturing
        try:
            with torch.cuda.graph(g, pool=self._pool):
                for _ in range(int(max_iter)):
                    self.step()
        finally:
            if gc_on:
                gc.enable()
        self._graphs[(int(frames), int(max_iter))] = g

    def run(self, max_iter: int) -> torch.Tensor:
        g = self._graphs.get((self.F, int(max_iter)))
        if g is not None:
            g.replay()
            return self.x
        for _ in range(int(max_iter)):
            self.step()
        return self.x


def _device_cg_applicable(op, AHb, preconditioner) -> bool:
    return (
        preconditioner is None
        and hasattr(op, "_normal_into")
        and isinstance(AHb, torch.Tensor)
        and AHb.device.type == "cuda"
        and AHb.dtype == torch.complex64
        and not getattr(op, "stack_shape", ())
        and AHb.ndim == getattr(op, "_single_ndim",
                                len(op.image_shape) + (0 if getattr(op, "smaps", None) is not None else 1))
    )


_CG_GRAPHS_PER_OP = 4


def _cached_solver(op, AHb: torch.Tensor, damp: float, tol: float, x0d) -> DeviceCG:
    """Graph-replayed CG solver of ``op`` for this right-hand side shape, damp
    and tolerance, kept on the operator so that repeated solves replay the
    captured iteration instead of capturing it again (the key includes the
    coil maps' buffer, the state the captured normal operator reads)."""
    smaps = getattr(op, "_smaps_d", None)
    key = (tuple(AHb.shape), str(AHb.device), float(damp), float(tol), bool(getattr(op, "toeplitz", False)),
           smaps.data_ptr() if isinstance(smaps, torch.Tensor) else 0)
    cache = getattr(op, "_cg_graphs", None)
    if cache is None:
        cache = {}
        op._cg_graphs = cache
    solver = cache.pop(key, None)
    if solver is None:
        solver = DeviceCG(op, AHb, damp, tol, x0d, weak_op=True)
        while len(cache) >= _CG_GRAPHS_PER_OP:
            cache.pop(next(iter(cache)))
    else:
        solver.reset(AHb, x0d)
    cache[key] = solver  # most recently used last
    return solver


def cg(
    op: Any,
    b: torch.Tensor,
    *,
    damp: float = 0.0,
    x0: torch.Tensor | None = None,
    max_iter: int = 20,
    tol: float = 1e-6,
    preconditioner: Any | None = None,
    callback: Callable | None = None,
    use_graph: bool = True,
) -> torch.Tensor:
    """CG on ``(A^H A + damp I) x = A^H b`` (``forward = A``, ``adjoint = A^H``)."""
    b = _normalize_kspace_shape(op, b)
    src_dev = b.device
    if hasattr(op, "_cdev") and src_dev.type != "cuda":
        b = b.to(op._cdev)
    AHb = op.adjoint(b)
    if _device_cg_applicable(op, AHb, preconditioner):
        x0d = None if x0 is None else torch.as_tensor(x0).to(AHb.device, torch.complex64)
        if use_graph and callback is None and int(max_iter) > 1:
            solver = _cached_solver(op, AHb, damp, tol, x0d)
            return solver.run(int(max_iter), None, True).clone().to(src_dev)
        solver = DeviceCG(op, AHb, damp, tol, x0d)
        x = solver.run(int(max_iter), callback, use_graph)
        return x.to(src_dev)
    # generic duck-typed operators: reference recurrence, FP64 inner products
    AHA = getattr(op, "normal", None)
    if AHA is None:

        def AHA(v):
            return op.adjoint(op.forward(v))

    x = torch.zeros_like(AHb) if x0 is None else torch.as_tensor(x0).clone()
    r = AHb - AHA(x) - damp * x
    z = preconditioner.apply(r) if preconditioner is not None else r
    p = z.clone()
    rz_old = _vdot_re64(r, z)
    r0 = torch.linalg.vector_norm(r.to(torch.complex128)) + 1e-30
    for k in range(max_iter):
        Ap = AHA(p) + damp * p
        alpha = (rz_old / (_vdot_re64(p, Ap) + 1e-30)).to(torch.float32)
        x = x + alpha * p
        r = r - alpha * Ap
        rel = float((torch.linalg.vector_norm(r.to(torch.complex128)) / r0).item())
        if callback is not None:
            callback(k, x, rel)
        if rel < tol:
            break
        z = preconditioner.apply(r) if preconditioner is not None else r
        rz_new = _vdot_re64(r, z)
        beta = (rz_new / (rz_old + 1e-30)).to(torch.float32)
        p = z + beta * p
        rz_old = rz_new
    return x.to(src_dev) if isinstance(x, torch.Tensor) else x


class DeviceLSMR:
    """LSMR state for one right-hand side on the device (``_solvers.py:145-262``).

    Vectors are complex64 device tensors; every scalar of the recurrence is
    FP64 in a device block (``include/pygrog_b200.h``, ``pgb_lsmr_*``), the
    two branch tests and the stopping test are device flags, so an iteration
    issues no host synchronisation and can be captured in a CUDA graph and
    replayed (iterations after the stopping test leave the state unchanged).
    The operator's ``forward`` / ``adjoint`` are called on device tensors.
    """

    def __init__(self, op, b: torch.Tensor, damp: float, tol: float, x0: torch.Tensor | None = None):
        self.op = op
        dev = b.device
        st = _lib.stream_ptr(dev)
        if x0 is not None:
            b = b - op.forward(x0)
        beta = float(torch.linalg.vector_norm(b.to(torch.complex128)))  # set-up syncs only
        self.trivial = None
        if beta == 0.0:
            self.trivial = x0.clone() if x0 is not None else op.adjoint(b)
            return
        self.u = (b / beta).to(torch.complex64).contiguous()
        v_full = op.adjoint(self.u)
        alpha = float(torch.linalg.vector_norm(v_full.to(torch.complex128)))
        if alpha == 0.0:
            self.trivial = x0.clone() if x0 is not None else torch.zeros_like(v_full)
            return
        self.v = (v_full / alpha).to(torch.complex64).contiguous()
        self.vf = torch.empty_like(self.v)
        self.h = self.v.clone()
        self.hbar = torch.zeros_like(self.v)
        self.x = torch.zeros_like(self.v) if x0 is None else x0.to(dev, torch.complex64).clone()
        self.nu, self.nv = int(self.u.numel()), int(self.v.numel())
        lib = _lib.load_library()
        self.scratch = torch.zeros((int(lib.pgb_lsmr_scratch_bytes()) + 7) // 8, dtype=torch.float64, device=dev)
        sc = np.zeros(32, dtype=np.float64)
        sc[[0, 1, 2, 3, 4, 5, 6, 7, 9, 11, 12]] = [alpha, beta, alpha, 1.0, 1.0, 1.0, 0.0, alpha * beta, beta,
                                                  float(tol), float(damp)]
        self.scal = torch.from_numpy(sc).to(dev)
        self.graph = None
        del st

    def step(self):
        st = _lib.stream_ptr(self.u.device)
        Av = self.op.forward(self.v)
        _lib.call("pgb_lsmr_u_update", self.u.data_ptr(), Av.data_ptr(), self.nu, self.scal.data_ptr(),
                  self.scratch.data_ptr(), st)
        _lib.call("pgb_lsmr_u_scale", self.u.data_ptr(), self.nu, self.scal.data_ptr(), st)
        Atu = self.op.adjoint(self.u)
        _lib.call("pgb_lsmr_v_full", self.vf.data_ptr(), Atu.data_ptr(), self.v.data_ptr(), self.nv,
                  self.scal.data_ptr(), self.scratch.data_ptr(), st)
        _lib.call("pgb_lsmr_scalars", self.scal.data_ptr(), st)
        _lib.call("pgb_lsmr_vec_update", self.x.data_ptr(), self.h.data_ptr(), self.hbar.data_ptr(),
                  self.v.data_ptr(), self.vf.data_ptr(), self.nv, self.scal.data_ptr(), st)

    def capture(self):
        """Capture one iteration in a CUDA graph (the operator runs once first,
        on a copy of the state, so its FFT plans exist before the capture)."""
        dev = self.u.device
        state = (self.u, self.v, self.vf, self.h, self.hbar, self.x, self.scal)
        saved = [t.clone() for t in state]
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):
            self.step()
        torch.cuda.current_stream(dev).wait_stream(side)
        for t, v in zip(state, saved):
            t.copy_(v)
        g = torch.cuda.CUDAGraph()
        gc_on = gc.isenabled()
        gc.disable()  # no collection (and no CUDA frees it may trigger) while capturing
        try:
            with torch.cuda.graph(g):
                self.step()
        finally:
            if gc_on:
                gc.enable()
        self.graph = g

    def run(self, max_iter: int, callback: Callable | None = None, use_graph: bool = True) -> torch.Tensor:
        if self.trivial is not None:
            return self.trivial
        if callback is None and use_graph and max_iter > 1:
            if self.graph is None:
                self.capture()
            for _ in range(int(max_iter)):
                self.graph.replay()
            return self.x
        for k in range(int(max_iter)):
            self.step()
            if callback is not None:
                sc = self.scal.cpu()
                if sc[18] != 0.0:
                    callback(k, self.x, float(sc[19]))
                if sc[10] != 0.0:
                    break
        return self.x


def _device_lsmr_applicable(op, b) -> bool:
    from .operator._masked_fft import MaskedFFT
    from .operator._sparse_fft import SparseFFT

    return (
        isinstance(op, (SparseFFT, MaskedFFT))
        and isinstance(b, torch.Tensor)
        and b.device.type == "cuda"
        and b.dtype == torch.complex64
    )


def lsmr(
    op: Any,
    b: torch.Tensor,
    *,
    damp: float = 0.0,
    x0: torch.Tensor | None = None,
    max_iter: int = 20,
    atol: float = 1e-6,
    btol: float = 1e-6,
    callback: Callable | None = None,
    use_graph: bool = True,
) -> torch.Tensor:
    """LSMR (Fong & Saunders) for ``argmin ||A x - b||^2 + damp^2 ||x||^2``.

    The recurrence of the reference (``_solvers.py:145-262``).  On this
    package's operators with complex64 device data it runs as
    :class:`DeviceLSMR` (FP64 device scalars, no host synchronisation inside
    the loop, one iteration replayed from a CUDA graph when there is no
    callback); other operators use the same recurrence on the host with FP64
    scalars.
    """
    b = _normalize_kspace_shape(op, b)
    src_dev = b.device
    if hasattr(op, "_cdev") and src_dev.type != "cuda":
        b = b.to(op._cdev)
    if _device_lsmr_applicable(op, b):
        x0d = None if x0 is None else torch.as_tensor(x0).to(b.device, torch.complex64)
        solver = DeviceLSMR(op, b, damp, atol + btol, x0d)
        return solver.run(int(max_iter), callback, use_graph).to(src_dev)
    if x0 is not None:
        b = b - op.forward(torch.as_tensor(x0).to(b.device))

    def nrm(t):
        return float(torch.linalg.vector_norm(t.to(torch.complex128)))

    beta = nrm(b)
    if beta == 0:
        out = torch.as_tensor(x0).clone() if x0 is not None else op.adjoint(b)
        return out.to(src_dev)
    u = b / beta
    v_full = op.adjoint(u)
    alpha = nrm(v_full)
    if alpha == 0:
        out = torch.as_tensor(x0).clone() if x0 is not None else torch.zeros_like(v_full)
        return out.to(src_dev)
    v = v_full / alpha
    zetabar = alpha * beta
    alphabar = alpha
    rho = rhobar = cbar = 1.0
    sbar = 0.0
    h = v.clone()
    hbar = torch.zeros_like(v)
    x = torch.zeros_like(v) if x0 is None else torch.as_tensor(x0).to(v.device).clone()
    normb = beta
    for k in range(max_iter):
        u = op.forward(v) - alpha * u
        beta = nrm(u)
        if beta > 0:
            u = u / beta
            v_full = op.adjoint(u) - beta * v
            alpha = nrm(v_full)
            if alpha > 0:
                v = v_full / alpha
        alphahat = math.sqrt(alphabar * alphabar + damp * damp)
        rhoold = rho
        rho = math.sqrt(alphahat * alphahat + beta * beta)
        c = alphahat / rho
        s = beta / rho
        thetanew = s * alpha
        alphabar = c * alpha
        rhobarold = rhobar
        thetabar = sbar * rho
        rhotemp = cbar * rho
        rhobar = math.sqrt(rhotemp * rhotemp + thetanew * thetanew)
        cbar = rhotemp / rhobar
        sbar = thetanew / rhobar
        zeta = cbar * zetabar
        zetabar = -sbar * zetabar
        hbar = h - (thetabar * rho / (rhoold * rhobarold)) * hbar
        x = x + (zeta / (rho * rhobar)) * hbar
        h = v - (thetanew / rho) * h
        rel = abs(zetabar) / (normb + 1e-30)
        if callback is not None:
            callback(k, x, rel)
        if rel < atol + btol:
            break
    return x.to(src_dev)


def solve(op: Any, b: torch.Tensor, *, method: str = "cg", **kwargs) -> torch.Tensor:
    """Dispatch to :func:`cg` or :func:`lsmr` (reference ``solve``)."""
    method = method.lower()
    if method == "cg":
        return cg(op, b, **kwargs)
    if method == "lsmr":
        return lsmr(op, b, **kwargs)
    raise ValueError(f"Unknown solver method: {method!r}. Use 'cg' or 'lsmr'.")


def _backend(x) -> str:
    if isinstance(x, torch.Tensor):
        return "torch"
    if isinstance(x, np.ndarray):
        return "numpy"
    return "torch"


class SolveMixin:
    """``op.solve(b, method=None, damp, x0, max_iter, tol, preconditioner, callback)``.

    ``method=None`` picks ``cg`` when ``self.toeplitz`` else ``lsmr`` (reference
    ``_mixin.py:131-132``); numpy inputs give numpy outputs.
    """

    def solve(self, b, *, method=None, damp=0.0, x0=None, max_iter=20, tol=1e-6, preconditioner=None,
              callback=None, **kwargs):
        backend = _backend(b)
        b_t = torch.as_tensor(b)
        x0_t = None if x0 is None else torch.as_tensor(x0)
        if method is None:
            method = "cg" if getattr(self, "toeplitz", False) else "lsmr"
        method = method.lower()
        if method == "cg":
            out = cg(self, b_t, damp=damp, x0=x0_t, max_iter=max_iter, tol=tol, preconditioner=preconditioner,
                     callback=callback, **kwargs)
        elif method == "lsmr":
            out = lsmr(self, b_t, damp=damp, x0=x0_t, max_iter=max_iter, callback=callback, **kwargs)
        else:
            raise ValueError(f"Unknown method: {method!r}")
        return out.detach().cpu().numpy() if backend == "numpy" else out
