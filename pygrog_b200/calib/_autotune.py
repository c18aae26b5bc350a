"""Autotuner of the fused GROG gridder: kernel family and brick shape.

The fused kernels (``csrc/grog_tc.cu``, ``grog_v8.cu``, ``grog_v6.cu``) are
parametrised by the brick of grid cells a CTA owns (its shared-memory tile)
and, through the plan, by how replicas are cut into sub-chunks.  The best
choice depends on the trajectory's density, the coil count and the table
size, so it is measured: every candidate (family x brick that fits shared
memory) is built on the caller's trajectory and timed forward + adjoint with
CUDA events on random data of the caller's batch size; the fastest is kept on
the interpolator and cached per problem signature.

Precision gates the families twice.  The tensor-core bf16x3 family
(``"tc"``) is a candidate only when the caller accepts a relative error of
1e-4 against FP64, plain bf16 (``"tc1"``) only at 1e-2; the FP32 families
(``"v8"``, ``"v6"``, ``"global"`` above 16 coils) always are.  Then every
tensor-core candidate's forward and adjoint outputs are compared with those
of an FP32 family on the same data (whose own error against FP64 is about
1e-6): a candidate above the tolerance is rejected, since the error of the
eigen-factored chain grows with the conditioning of the table's per-axis
eigenvectors, which depends on the calibration data.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib

__all__ = ["autotune_gridder", "clear_cache"]

_CACHE: dict = {}


def clear_cache() -> None:
    _CACHE.clear()


def _signature(g, batch: int, tolerance: float):
    plan = g.plan
    kw = int(plan.target_idx.shape[-1])
    n_valid = int((plan.target_idx.reshape(-1) >= 0).sum())
    return (tuple(int(s) for s in plan.grid_shape), int(g._interp_kernel.shape[-1]), kw, n_valid,
            int(g._nsteps), int(batch), float(tolerance))


def _rel(a: torch.Tensor, b: torch.Tensor) -> float:
    return float((a - b).norm() / b.norm().clamp(min=1e-30))


def _time(bp, data: torch.Tensor, G: int, reps: int, warmup: int):
    """Median forward + adjoint milliseconds and the two outputs."""
    B, C, N = data.shape
    kg = torch.empty(B, C, G, dtype=torch.complex64, device=data.device)
    out = torch.empty(B, C, N, dtype=torch.complex64, device=data.device)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    ts = []
    for it in range(warmup + reps):
        ev[0].record()
        bp.forward(data, kg)
        bp.adjoint(kg, out)
        ev[1].record()
        torch.cuda.synchronize(data.device)
        if bp.tc is not None:  # a timed-out tile wait leaves the output incomplete: never time or pick it
            _lib.check_tc_timeouts(f"autotune_gridder ({bp.mode})")
        if it >= warmup:
            ts.append(ev[0].elapsed_time(ev[1]))
    return float(np.median(ts)), kg, out


def autotune_gridder(g, batch: int = 1, tolerance: float = 1e-4, families=None, reps: int = 3, warmup: int = 1,
                     use_cache: bool = True) -> dict:
    """Pick the fastest fused gridder for ``g`` (a ``GrogInterpolator`` after
    ``calc_interp_table``) and install it (``g.gridder_mode``, ``g.gridder_brick``).

    Returns ``{"mode", "brick", "ms", "trials": [(mode, brick, ms, err), ...],
    "rejected": [(mode, brick, err), ...], "cached"}``.  ``ms`` is the forward +
    adjoint time on stack entry 0; ``err`` the larger relative L2 difference of
    the forward and adjoint outputs from the FP32 reference candidate.
    """
    from ._grog import GrogGridder

    if not getattr(g, "_interpolator_set", False):
        raise RuntimeError("autotune_gridder: call calc_interp_table() first")
    key = _signature(g, batch, tolerance)
    if use_cache and key in _CACHE:
        best = _CACHE[key]
        g.gridder_mode, g.gridder_brick = best["mode"], best["brick"]
        g._brick_plans = None
        return dict(best, cached=True)
    C = int(g._interp_kernel.shape[-1])
    ndim = len(g.plan.grid_shape)
    if families is None:
        families = ["v8", "v6"] if C <= 16 else ["global"]  # FP32 shared-memory families cover C <= 16
        if C <= 32 and tolerance >= 1e-4:
            families.insert(0, "tc")
        if C <= 32 and tolerance >= 1e-2:
            families.insert(1, "tc1")
    bricks = GrogGridder.BRICKS3 if ndim == 3 else GrogGridder.BRICKS2
    plan = g.plan
    s_total = int(np.prod(plan.stack_shape)) if plan.stack_shape else 1
    kw = int(plan.target_idx.shape[-1])
    tgt = plan.target_idx.reshape(s_total, -1)[0]
    sw = torch.sqrt(plan.weights.reshape(s_total, -1)[0].clamp(min=0.0))
    rep_w = sw * sw
    idx = g._interp_idx.reshape(s_total, -1)[0]
    N = tgt.numel() // kw
    G = int(np.prod(plan.grid_shape))
    gen = torch.Generator(device=g.device).manual_seed(0)
    data = torch.randn(batch, C, N, dtype=torch.complex64, device=g.device, generator=gen)
    trials = []
    rejected = []
    best = None
    best_bp = None
    ref = None  # (grid, samples) of the first FP32 candidate
    tc_fams = ("tc", "tc1")
    order = [m for m in families if m not in tc_fams] + [m for m in families if m in tc_fams]
    if order and order[0] in tc_fams:  # no FP32 family asked for: the global gridder is the reference
        bp = GrogGridder(tgt, idx, rep_w, kw, plan.grid_shape, g._interp_kernel, g._factors, g._nsteps,
                         mode="global")
        ref = _time(bp, data, G, 1, 0)[1:]
        del bp
    for mode in order:
        tc_ops = g._tc_operands() if mode in tc_fams else None
        for br in bricks:
            try:
                bp = GrogGridder(tgt, idx, rep_w, kw, plan.grid_shape, g._interp_kernel, g._factors, g._nsteps,
                                 mode=mode, brick=br, tc_ops=tc_ops)
            except ValueError:
                continue  # this family / brick does not fit shared memory
            if bp.mode != mode and not (mode == "v8" and bp.mode == "v8"):
                continue
            ms, kg, out = _time(bp, data, G, reps, warmup)
            if ref is None:
                ref = (kg, out)
            err = max(_rel(kg, ref[0]), _rel(out, ref[1]))
            if mode in tc_fams and err > tolerance:
                rejected.append((mode, tuple(br), err))
                del bp
                continue
            trials.append((mode, tuple(br), ms, err))
            if best is None or ms < best["ms"]:
                best = {"mode": mode, "brick": tuple(br), "ms": ms}
                best_bp = bp
            else:
                del bp
    if best is None:
        raise RuntimeError("autotune_gridder: no candidate gridder fits this problem")
    best["trials"] = trials
    best["rejected"] = rejected
    g.gridder_mode, g.gridder_brick = best["mode"], best["brick"]
    g._brick_plans = {0: best_bp} if s_total == 1 else None
    if use_cache:
        _CACHE[key] = best
    torch.cuda.empty_cache()
    return dict(best, cached=False)
