"""GROG interpolator on the GPU: plan, shift table, interpolation and gridding.

Mirrors the public API of ``calib/_grog.py`` (FiRMLAB-Pisa/pygrog):
``GrogPlan`` (27-181), ``GrogInterpolator(shape, coords, oversamp,
kernel_width, kernel_shape, time_map, image_shape, stack_shape)`` (302-331),
``calc_interp_table`` (382-422), ``interpolate`` (437-555), shot-by-shot
gridding (697-731, 904-912) and ``fft_plan`` (348-376).

What runs where:
* plan geometry, EGROG weights and shift quantisation: CUDA kernels with
  bit-exact float32 integer keys (``csrc/plan.cu``); sorting by cell:
  device radix sort;
* GRAPPA table fit: host LAPACK, as in the reference (a few C x C solves);
* ``interpolate``: one replica-expansion kernel (``csrc/grog_fused.cu``)
  instead of replicate / transpose / matvec / copy-back passes;
* ``interpolate(grid=True)``: one fused kernel (shift matvec, EGROG weight,
  scatter) writing every grid cell once;
* :meth:`GrogInterpolator.degrid`: its exact adjoint (new; the reference has
  no adjoint of the GROG shift).

Plan fields live on the GPU.  Inputs may be numpy arrays or tensors on any
device; numpy inputs give numpy outputs like the reference.
"""

from __future__ import annotations

__all__ = ["GrogInterpolator", "GrogPlan", "BrickPlan", "GrogGridder"]

import math
import os
from types import SimpleNamespace

import numpy as np
import torch

from .. import _lib
from ._grappa import KernelTable
from ._plan6 import BrickPlan6, _sm_count, lane_chunk

_DEFAULT_DEVICE = "cuda"
# check the tensor-core timeout counter after every degrid (synchronising)
_SYNC_CHECK = os.environ.get("PYGROG_B200_SYNC_CHECK", "0") not in ("", "0")


# ---------------------------------------------------------------------------
# Plan container
# ---------------------------------------------------------------------------
class GrogPlan(SimpleNamespace):
    """Namespace of GROG / FFT plan fields (reference ``GrogPlan``).

    ``pre_weights`` is computed from ``sqrt_weights`` and ``inv_perm`` so it
    always matches :meth:`GrogInterpolator.interpolate` output order.
    """

    @property
    def stack_shape(self) -> tuple:
        return tuple(getattr(self, "_stack_shape", ()))

    @stack_shape.setter
    def stack_shape(self, value):
        self._stack_shape = tuple(int(s) for s in (value or ()))

    @property
    def is_stacked(self) -> bool:
        return len(self.stack_shape) > 0

    @property
    def pre_weights(self) -> torch.Tensor:
        sw = self.sqrt_weights
        ip = self.inv_perm
        if not self.is_stacked:
            return sw[ip]
        return torch.gather(sw, -1, ip)

    @classmethod
    def _stack(cls, plans: list) -> "GrogPlan":
        if not plans:
            raise ValueError("Cannot stack an empty list of plans.")
        for p in plans:
            if getattr(p, "stack_shape", ()) != ():
                raise ValueError("GrogPlan.stack requires unstacked input plans.")
        ref = plans[0]
        global_fields = (
            "shape", "oversamp", "grid_shape", "kernel_width", "kernel_shape", "radius",
            "image_shape", "grid_size", "n_samples", "natural_shape",
        )
        for f in global_fields:
            v = getattr(ref, f, None)
            for p in plans[1:]:
                if getattr(p, f, None) != v:
                    raise ValueError(f"GrogPlan.stack: field '{f}' differs across plans")
        out = cls(**{f: getattr(ref, f) for f in global_fields})
        out.stack_shape = (len(plans),)
        for f in ("target_idx", "weights", "indices", "sqrt_weights", "sort_perm", "inv_perm"):
            setattr(out, f, torch.stack([getattr(p, f) for p in plans], dim=0))
        if all(getattr(p, "distances", None) is not None for p in plans):
            out.distances = torch.stack([p.distances for p in plans], dim=0)
        else:
            out.distances = None
        if any(p.time_map is not None for p in plans):
            if any(p.time_map is None for p in plans):
                raise ValueError("GrogPlan.stack: all plans must agree on time_map presence")
            out.time_map = torch.stack([p.time_map for p in plans], dim=0)
        else:
            out.time_map = None
        return out


# ---------------------------------------------------------------------------
# Plan helpers (host: tiny integer tables and the coordinate rescale)
# ---------------------------------------------------------------------------
def _kernel_offsets(ndim: int, width: int, shape: str) -> np.ndarray:
    """Integer neighbourhood offsets ``(kw, ndim)`` (reference ``_grog.py:1240-1277``).

    Width ``w`` spans ``arange(w) - floor((w-1)/2)`` per axis; ``circle`` /
    ``sphere`` keep ``|o| <= (w-1)/2 + 0.5``, ``cross`` keeps offsets with at
    most one non-zero component, ``square`` / ``cube`` keep all, in C order.
    """
    half = (width - 1) / 2.0
    ax = np.arange(width) - int(np.floor(half))
    grids = np.meshgrid(*([ax] * ndim), indexing="ij")
    offs = np.stack([g.ravel() for g in grids], axis=-1).astype(np.int32)
    key = shape.lower()
    if key in ("square", "cube"):
        return offs
    if key in ("circle", "sphere"):
        r = np.sqrt((offs.astype(np.float32) ** 2).sum(axis=-1))
        return offs[r <= half + 0.5]
    if key == "cross":
        return offs[(offs != 0).sum(axis=-1) <= 1]
    raise ValueError(
        f"Unknown kernel_shape '{shape}'. Use 'circle'/'sphere', 'square'/'cube', or 'cross'."
    )


def _default_shape(ndim, shape):
    if np.isscalar(shape):
        shape = ndim * [shape]
    return tuple(int(s) for s in shape)


def _default_oversamp(ndim, oversamp):
    if oversamp is None:
        oversamp = (1.0, 1.0) if ndim == 2 else (1.0, 1.0, 1.2)
    if np.isscalar(oversamp):
        oversamp = ndim * [oversamp]
    oversamp = tuple(oversamp)
    if len(oversamp) != ndim:
        raise ValueError(f"Oversampling {oversamp} does not match ndim={ndim}")
    return oversamp


def _rescale_coords(coords: torch.Tensor, amp) -> torch.Tensor:
    """``0.5 * amp * coords / max|coords|`` per axis, in float32 (``_grog.py:1318-1322``).

    ``coords`` is a float32 ``(npts, ndim)`` tensor (on the device for plans);
    the products and the quotient are IEEE float32 operations in the same
    order as the reference's, so the result is bit-identical wherever it runs.
    """
    ndim = int(coords.shape[-1])
    cmax = coords.abs().amax(dim=0)
    if np.isscalar(amp):
        amp = ndim * [amp]
    half_amp = torch.as_tensor(0.5 * np.asarray(amp, dtype=np.float32), device=coords.device)
    return (half_amp * coords) / cmax


def _create_plan_single(shape, coords, oversamp, kernel_width, kernel_shape, time_map, device):
    """Per-replica target cells, shifts and EGROG weights on the device.

    Follows ``_create_plan_single`` (``_grog.py:1081-1234``); the arithmetic is
    in ``pgb_plan_geometry`` / ``pgb_plan_gauss_sum`` / ``pgb_plan_weights``.
    """
    if not isinstance(coords, torch.Tensor):
        coords = np.asarray(coords)
    ndim = int(coords.shape[-1])
    if ndim not in (2, 3):
        raise ValueError(f"GROG interpolation only supports 2D or 3D data, got {ndim}D")
    shape = _default_shape(ndim, shape)
    oversamp = _default_oversamp(ndim, oversamp)
    grid_shape = tuple(int(np.ceil(s * o)) for s, o in zip(shape, oversamp))
    amp = [2 * (s - 1 - s // 2) for s in shape]
    offsets = _kernel_offsets(ndim, kernel_width, kernel_shape)
    kw = int(offsets.shape[0])
    origins = np.asarray([-(s // 2) for s in shape], dtype=np.float32)
    steps = np.asarray(
        [(s - 1) / (gs - 1) if gs > 1 else 1.0 for s, gs in zip(shape, grid_shape)], dtype=np.float32
    )
    lead = coords.shape[:-1]
    npts = int(np.prod(lead)) if lead else 1
    R = npts * kw
    G = int(np.prod(grid_shape))
    dev = torch.device(device)
    # cast to float32 first (as the reference does), then rescale on the device
    c_in = coords if isinstance(coords, torch.Tensor) else torch.from_numpy(np.ascontiguousarray(coords))
    c_d = c_in.reshape(npts, ndim).to(dev, non_blocking=False).to(torch.float32)
    c_d = _rescale_coords(c_d, amp).contiguous()
    off_d = torch.from_numpy(np.ascontiguousarray(offsets)).to(dev)
    # per-axis parameters are read by the host launcher: pass host arrays
    gs_h = np.ascontiguousarray(grid_shape, dtype=np.int64)
    org_h = np.ascontiguousarray(origins, dtype=np.float32)
    stp_h = np.ascontiguousarray(steps, dtype=np.float32)
    target = torch.empty(R, dtype=torch.int64, device=dev)
    dist = torch.empty(R, ndim, dtype=torch.float32, device=dev)
    gauss = torch.empty(R, dtype=torch.float32, device=dev)
    s = _lib.stream_ptr(dev)
    _lib.call(
        "pgb_plan_geometry", c_d.data_ptr(), npts, ndim, off_d.data_ptr(), kw, gs_h.ctypes.data,
        org_h.ctypes.data, stp_h.ctypes.data, target.data_ptr(), dist.data_ptr(), gauss.data_ptr(), s,
    )
    gsum = torch.zeros(G, dtype=torch.float64, device=dev)
    _lib.call("pgb_plan_gauss_sum", target.data_ptr(), gauss.data_ptr(), R, gsum.data_ptr(), G, s)
    weights = torch.empty(R, dtype=torch.float32, device=dev)
    _lib.call(
        "pgb_plan_weights", target.data_ptr(), gauss.data_ptr(), gsum.data_ptr(), R,
        weights.data_ptr(), s,
    )
    del gsum, gauss
    if time_map is not None:
        tm = torch.as_tensor(np.asarray(time_map, dtype=np.float32), device=dev)
        time_map = tm.reshape(*lead, 1).expand(*lead, kw).contiguous()
    return GrogPlan(
        shape=shape,
        oversamp=oversamp,
        grid_shape=grid_shape,
        kernel_width=kernel_width,
        kernel_shape=kernel_shape,
        radius=0.5,
        target_idx=target.reshape(*lead, kw),
        distances=dist.reshape(*lead, kw, ndim),
        weights=weights.reshape(*lead, kw),
        time_map=time_map,
    )


def _attach_fft_plan(plan, image_shape=None):
    """Sorted-by-cell FFT fields (``_grog.py:918-998``), on the device.

    Invalid replicas keep index 0 and weight 0 so ``n_samples = N * kw``.
    The sort is stable (the reference's is not; only the order among
    replicas of the same cell can differ, which no result depends on).
    """
    grid_shape = tuple(plan.grid_shape)
    if image_shape is None:
        image_shape = tuple(plan.shape)
    elif np.isscalar(image_shape):
        image_shape = len(grid_shape) * (int(image_shape),)
    image_shape = tuple(int(s) for s in image_shape)
    grid_size = int(np.prod(grid_shape))
    s_shape = tuple(getattr(plan, "stack_shape", ()) or ())
    tgt = plan.target_idx
    natural_shape = tuple(int(s) for s in tgt.shape[len(s_shape):])
    n_per = int(np.prod(natural_shape)) if natural_shape else 0
    idx = tgt.reshape(*s_shape, n_per).to(torch.int64).clone()
    w = plan.weights.reshape(*s_shape, n_per).to(torch.float32)
    sqrt_w = torch.sqrt(w.clamp(min=0.0))
    invalid = idx < 0
    idx = torch.where(invalid, torch.zeros_like(idx), idx)
    sqrt_w = torch.where(invalid, torch.zeros_like(sqrt_w), sqrt_w)
    sorted_idx, sort_perm = torch.sort(idx, dim=-1, stable=True)
    sorted_w = torch.gather(sqrt_w, -1, sort_perm)
    inv_perm = torch.empty_like(sort_perm)
    ar = torch.arange(n_per, dtype=torch.int64, device=idx.device).expand(sort_perm.shape)
    inv_perm.scatter_(-1, sort_perm, ar)
    plan.image_shape = image_shape
    plan.grid_size = grid_size
    plan.n_samples = n_per
    plan.natural_shape = natural_shape
    plan.indices = sorted_idx
    plan.sqrt_weights = sorted_w
    plan.sort_perm = sort_perm
    plan.inv_perm = inv_perm


def _create_plan(shape, coords, oversamp, kernel_width, kernel_shape, time_map, stack_shape, device):
    s_shape = tuple(int(s) for s in (stack_shape or ()))
    if not s_shape:
        return _create_plan_single(shape, coords, oversamp, kernel_width, kernel_shape, time_map, device)
    coords = np.asarray(coords)
    if tuple(coords.shape[: len(s_shape)]) != s_shape:
        raise ValueError(
            f"coords leading shape {coords.shape[: len(s_shape)]} does not match stack_shape {s_shape}"
        )
    s_total = int(np.prod(s_shape))
    cflat = coords.reshape(s_total, *coords.shape[len(s_shape):])
    if time_map is not None:
        tm = np.asarray(time_map)
        if tm.shape[: len(s_shape)] != s_shape:
            raise ValueError(
                f"time_map leading shape {tm.shape[: len(s_shape)]} does not match stack_shape {s_shape}"
            )
        tflat = tm.reshape(s_total, *tm.shape[len(s_shape):])
    else:
        tflat = [None] * s_total
    plans = [
        _create_plan_single(shape, cflat[i], oversamp, kernel_width, kernel_shape, tflat[i], device)
        for i in range(s_total)
    ]
    for p in plans:
        _attach_fft_plan(p, image_shape=None)
    out = GrogPlan._stack(plans)
    if len(s_shape) > 1:
        for f in ("target_idx", "weights", "indices", "sqrt_weights", "sort_perm", "inv_perm"):
            t = getattr(out, f)
            setattr(out, f, t.reshape(s_shape + tuple(t.shape[1:])))
        if out.time_map is not None:
            out.time_map = out.time_map.reshape(s_shape + tuple(out.time_map.shape[1:]))
        out.stack_shape = s_shape
    return out


# ---------------------------------------------------------------------------
# Brick work plan for the fused grid / degrid kernels
# ---------------------------------------------------------------------------
def _u32_to_i32(x: torch.Tensor) -> torch.Tensor:
    return torch.where(x >= 2**31, x - 2**32, x).to(torch.int32)


class BrickPlan:
    """Valid replicas sorted by (brick, cell) with packed per-replica metadata.

    Per replica: ``rep_src`` int32 source sample, ``rep_meta`` uint32 (table
    entry in the low 20 bits, cell-in-brick above), ``rep_w`` float32 weight.
    ``work`` rows ``{brick, begin, end, split}`` give each CTA one brick or one
    chunk of at most ``chunk`` replicas of a hot brick.
    """

    def __init__(
        self,
        target_idx: torch.Tensor,
        interp_idx: torch.Tensor,
        rep_weight: torch.Tensor,
        kw: int,
        grid_shape,
        brick=None,
        chunk: int = 2048,
        n_outer: int = 1,
        pack: str = "wide",
        mask: torch.Tensor | None = None,
        order: str = "cell",
    ):
        dev = target_idx.device
        grid_shape = tuple(int(s) for s in grid_shape)
        self.n_outer = int(n_outer)
        if len(grid_shape) == 2:
            gz, gy, gx = 1, grid_shape[0], grid_shape[1]
            bz, by, bx = brick if brick is not None else (1, 16, 32)
        else:
            gz, gy, gx = grid_shape
            bz, by, bx = brick if brick is not None else (8, 8, 8)
        # partial bricks at the grid edge are bounds-checked by the kernels
        self.grid = (gz, gy, gx)
        self.brick = (bz, by, bx)
        self.nb = ((gz + bz - 1) // bz, (gy + by - 1) // by, (gx + bx - 1) // bx)
        self.cells = bz * by * bx
        if self.cells > 4096:
            raise ValueError("brick too large (max 4096 cells)")
        n_bricks = self.nb[0] * self.nb[1] * self.nb[2]
        tgt = target_idx.reshape(-1)
        R = tgt.numel()
        self.n_src = R // kw
        valid = tgt >= 0
        if mask is not None:
            valid = valid & mask.reshape(-1)
        r = torch.nonzero(valid).squeeze(1)
        t = tgt[r]
        z = t // (gy * gx)
        rem = t - z * (gy * gx)
        y = rem // gx
        x = rem - y * gx
        brick_id = ((z // bz) * self.nb[1] + (y // by)) * self.nb[2] + (x // bx)
        cl = ((z % bz) * by + (y % by)) * bx + (x % bx)
        # sort key (brick, outer table index, cell): runs sharing the outer
        # factor and the target cell are contiguous inside each brick
        e_all = interp_idx.reshape(-1)[r].to(torch.int64)
        kout = e_all % self.n_outer
        if order == "inner":
            # (brick, inner index, outer index, cell): a warp's lanes share operators
            n_in = int(e_all.max()) // self.n_outer + 1 if e_all.numel() else 1
            key = ((brick_id * n_in + e_all // self.n_outer) * self.n_outer + kout) * self.cells + cl
            span = n_in * self.n_outer * self.cells
        else:
            # (brick, outer index, cell): runs sharing the outer factor and cell
            key = (brick_id * self.n_outer + kout) * self.cells + cl
            span = self.n_outer * self.cells
        key_sorted, perm = torch.sort(key, stable=True)
        r = r[perm]
        brick_sorted = key_sorted // span
        cl_sorted = key_sorted % self.cells
        entry = interp_idx.reshape(-1)[r].to(torch.int64)
        if entry.numel() and int(entry.max()) >= 2**20:
            raise ValueError("shift table too large for the fused kernels (max 2^20 entries)")
        self.rep_src = (r // kw).to(torch.int32).contiguous()
        if pack == "split":
            # cell | inner << 11 | outer << 25  (T[e] = outer[e % n] @ inner[e // n])
            inner_i = entry // self.n_outer
            outer_i = entry % self.n_outer
            if self.cells > 2048 or (entry.numel() and (int(inner_i.max()) >= 16384 or self.n_outer > 128)):
                raise ValueError("split metadata needs cells <= 2048, inner < 16384, outer <= 128")
            self.rep_meta = _u32_to_i32(cl_sorted | (inner_i << 11) | (outer_i << 25)).contiguous()
        else:
            self.rep_meta = _u32_to_i32(entry | (cl_sorted << 20)).contiguous()
        self.rep_w = rep_weight.reshape(-1)[r].to(torch.float32).contiguous()
        self.n_valid = int(r.numel())
        counts = torch.bincount(brick_sorted, minlength=n_bricks)
        starts = torch.cumsum(counts, 0) - counts
        nch = torch.clamp((counts + chunk - 1) // chunk, min=1)
        bricks_rep = torch.repeat_interleave(torch.arange(n_bricks, device=dev), nch)
        first = torch.cumsum(nch, 0) - nch
        k = torch.arange(bricks_rep.numel(), device=dev) - first[bricks_rep]
        b0 = starts[bricks_rep] + k * chunk
        b1 = torch.minimum(b0 + chunk, starts[bricks_rep] + counts[bricks_rep])
        split = (nch[bricks_rep] > 1).to(torch.int64)
        self.work = torch.stack([bricks_rep, b0, b1, split], dim=1).to(torch.int32).contiguous()
        nonempty = b1 > b0
        self.work_nonempty = self.work[nonempty].contiguous()
        self.split_bricks = torch.nonzero(nch > 1).squeeze(1).to(torch.int32).contiguous()
        # Samples with no valid replica (zeroed by the adjoint) and whether any
        # sample has more than one (the adjoint then accumulates atomically).
        per_src = torch.bincount(self.rep_src.to(torch.int64), minlength=self.n_src)
        self.multi = bool(int(per_src.max()) > 1) if per_src.numel() else False
        self.zero_src = torch.nonzero(per_src == 0).squeeze(1).to(torch.int32).contiguous()
        self._c_all = self._struct(self.work)
        self._c_nonempty = self._struct(self.work_nonempty)

    def _struct(self, work: torch.Tensor) -> _lib.BrickPlanC:
        gz, gy, gx = self.grid
        bz, by, bx = self.brick
        nbz, nby, nbx = self.nb
        return _lib.BrickPlanC(
            self.rep_src.data_ptr(), self.rep_meta.data_ptr(), self.rep_w.data_ptr(),
            work.data_ptr(), int(work.shape[0]), gz, gy, gx, bz, by, bx, nbz, nby, nbx,
            self.split_bricks.data_ptr() if self.split_bricks.numel() else None,
            int(self.split_bricks.numel()),
        )


def _ctypes_ref(s):
    import ctypes

    return ctypes.byref(s)


_SMEM_BUDGET = 220 * 1024
_SMEM_V3 = 227 * 1024


def _first_valid_mask(target_idx: torch.Tensor, kw: int) -> torch.Tensor:
    """True for the first valid replica (lowest replica index) of each sample."""
    tgt = target_idx.reshape(-1, kw)
    valid = tgt >= 0
    first = torch.argmax(valid.to(torch.int8), dim=1)  # first True per row (0 if none)
    m = torch.zeros_like(valid)
    rows = torch.arange(tgt.shape[0], device=tgt.device)
    m[rows, first] = True
    return (m & valid).reshape(-1)


def _pack_axis_indices(bp: BrickPlan6, nsteps: int, ndim: int) -> None:
    """Rewrite ``meta.y = q | k << 16`` (``e = q * nsteps + k``) of a v6 plan as
    the per-axis shift indices the tensor-core kernels read: ``i | j << 8 |
    k << 16`` in 3-D (``q = i * nsteps + j``, ``nsteps <= 255``), ``i | k << 16``
    in 2-D."""
    if ndim == 3 and nsteps > 255:
        raise ValueError("tc kernels: 3-D tables need nsteps <= 255")
    if bp.meta.numel() == 0:
        return
    y = bp.meta[:, 1].to(torch.int64)
    q, k = y & 0xFFFF, y >> 16
    if ndim == 3:
        y = (q // nsteps) | ((q % nsteps) << 8) | (k << 16)
    bp.meta[:, 1] = y.to(torch.int32)


class GrogGridder:
    """Fused GROG gridding operator for one trajectory: brick plans + tables.

    Kernel families (chosen from the shared-memory budget of one CTA):
      ``"tc"``        C <= 32: eigen-factored table as a chain of dense
                      coil matrices on the tensor cores (bf16x3 split
                      products, FP32 accumulate) with per-replica phases;
      ``"tc1"``       the same chain with plain bf16 products;
      ``"v8"``        C <= 16: one lane per replica on balanced sub-chunk
                      streams, replicas ordered (outer, inner, cell) so
                      operator loads are conflict-free or broadcast; the
                      forward sums each cell's replicas without atomics
                      (the FP32 default);
      ``"v8pair"``    the v8 adjoint with the v6 forward;
      ``"v6"``        C <= 16: operator-stationary slots (outer factor rows
                      in registers along sorted runs, inner factor or whole
                      table in shared memory), dynamic work queue;
      ``"global"``    table read through L1/L2 (any C <= 32, K < 2^20): the
                      FP32 gridder above 16 coils or when no table fits
                      shared memory.
    With a factored table ``T[e] = outer[e % n] @ inner[e // n]``, the outer
    factor is applied once per run of replicas sharing (outer index, cell).
    """

    BRICKS3 = ((8, 8, 8), (4, 8, 8), (4, 4, 8), (2, 4, 8))
    # v8 plans: deal replicas round-robin over inner residues q mod 8 inside
    # outer runs (BrickPlan6 lane_order): fewer shared-memory bank conflicts
    LANE_ORDER_V8 = True
    # v8 forward: longest run of one cell's replicas summed by one thread
    SEG_LEN_V8 = 24
    BRICKS2 = ((1, 16, 32), (1, 16, 16), (1, 8, 16), (1, 8, 8))
    # tensor-core forward plans: cell runs packed into 16-row m-tiles (0: off)
    PACK_ROWS_TC = 16

    def __init__(self, target_idx, interp_idx, rep_weight, kw, grid_shape, table, factors, nsteps,
                 mode: str | None = None, brick=None, chunk: int = 2048, tc_ops: dict | None = None):
        C = int(table.shape[-1])
        K = int(table.shape[0])
        self.C = C
        ndim = len(grid_shape)
        lib = _lib.load_library()
        cand = self.BRICKS3 if ndim == 3 else self.BRICKS2
        if brick is not None:
            cand = (tuple(brick),)
        self.tc = None
        if mode in ("tc", "tc1"):
            self._init_tc(mode, tc_ops, target_idx, interp_idx, rep_weight, kw, grid_shape, cand, lib)
            return
        n_fact = int(factors[1].shape[0]) if factors is not None else None

        def v6_fits(n_in, n_out, br, sub):
            cells = br[0] * br[1] * br[2]
            return lib.pgb_grog_v6_smem_bytes(C, cells, n_in, n_out, sub) <= _SMEM_V3

        def v8_fits(n_in, n_out, br, sub):
            cells = br[0] * br[1] * br[2]
            return lib.pgb_grog_v8_smem_bytes(C, cells, n_in, n_out, sub) <= _SMEM_V3

        chosen = None
        self.sub_cap = None
        self.fwd6 = None  # (brick, sub_cap, factored) of the v6 forward used with the v8 adjoint
        if mode in (None, "v8", "v8pair") and C <= 16:
            n_out_f = int(factors[0].shape[0]) if factors is not None else None
            for sub in (256, 192, 128):
                for br in cand:
                    if K <= 65535 and v8_fits(K, 1, br, sub):
                        chosen = ("v8", br, False)
                    elif n_fact is not None and n_fact <= 65535 and v8_fits(n_fact, n_out_f, br, sub):
                        chosen = ("v8", br, True)
                    if chosen is not None:
                        self.sub_cap = sub
                        break
                if chosen is not None:
                    break
            if chosen is not None and mode == "v8pair":
                # the operator-stationary v6 forward with the same table factoring
                fact8 = chosen[2]
                for sub6 in (128, 96, 64):
                    for br6 in cand:
                        ok = (v6_fits(n_fact, n_out_f, br6, sub6) if fact8 else v6_fits(K, 1, br6, sub6))
                        if ok:
                            self.fwd6 = (br6, sub6, fact8)
                            break
                    if self.fwd6 is not None:
                        break
        if chosen is None and mode in (None, "v6") and C <= 16:
            n_out_f = int(factors[0].shape[0]) if factors is not None else None
            for sub in (128, 96, 64):
                for br in cand:
                    if K <= 65535 and v6_fits(K, 1, br, sub):
                        chosen = ("v6", br, False)
                    elif n_fact is not None and n_fact <= 65535 and v6_fits(n_fact, n_out_f, br, sub):
                        chosen = ("v6", br, True)
                    if chosen is not None:
                        self.sub_cap = sub
                        break
                if chosen is not None:
                    break
        if chosen is None:
            if mode in ("v6", "v8", "v8pair"):
                raise ValueError(f"{mode} kernels need C <= 16 and a table that fits shared memory")
            if mode not in (None, "global"):
                raise ValueError(f"unknown gridder mode {mode!r} (tc, tc1, v8, v8pair, v6, global)")
            br = cand[0] if C <= 16 else ((4, 8, 8) if ndim == 3 else (1, 16, 16))
            if brick is not None:
                br = tuple(brick)
            chosen = ("global", br, False)
        self.mode, brick, factored = chosen
        self.brick = brick
        dev = target_idx.device
        if factored:
            outer, inner = factors
            self.n_outer = int(outer.shape[0])
            self.inner = inner.to(dev).contiguous()
            self.outer = outer.to(dev).contiguous()
            self.inner_h = self.inner.conj().transpose(-1, -2).contiguous()
            self.outer_h = self.outer.conj().transpose(-1, -2).contiguous()
        else:
            self.n_outer = 1
            self.inner = torch.as_tensor(table).to(dev).contiguous()
            self.inner_h = self.inner.conj().transpose(-1, -2).contiguous()
            self.outer = self.outer_h = None
        self.plan2 = None  # adjoint secondary replicas (v3 / v5 / v6 / v8)
        if self.mode == "v8":
            kw8 = dict(brick=brick, n_outer=self.n_outer, sub_cap=self.sub_cap, lane_order=self.LANE_ORDER_V8)
            if self.fwd6 is not None:
                br6, sub6, _ = self.fwd6
                self.inner_lc = lane_chunk(self.inner)
                self.outer_lc = lane_chunk(self.outer) if self.outer is not None else None
                self.plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, brick=br6,
                                       n_outer=self.n_outer, sub_cap=sub6)
            else:
                self.plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, cell_order=True,
                                       seg_len=self.SEG_LEN_V8, **kw8)
            first = _first_valid_mask(target_idx, kw)
            self.adj_plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, mask=first, **kw8)
            if self.plan.n_valid > self.adj_plan.n_valid:
                self.plan2 = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, mask=~first, **kw8)
            return
        if self.mode == "v6":
            self.inner_lc = lane_chunk(self.inner)
            self.inner_h_lc = lane_chunk(self.inner_h)
            self.outer_lc = lane_chunk(self.outer) if self.outer is not None else None
            self.outer_h_lc = lane_chunk(self.outer_h) if self.outer_h is not None else None
            kw6 = dict(brick=brick, n_outer=self.n_outer, sub_cap=self.sub_cap)
            self.plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, **kw6)
            first = _first_valid_mask(target_idx, kw)
            self.adj_plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, mask=first, **kw6)
            if self.plan.n_valid > self.adj_plan.n_valid:
                self.plan2 = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, mask=~first, **kw6)
            return
        kwargs = dict(brick=brick, chunk=chunk, n_outer=self.n_outer, pack="wide", order="cell")
        self.plan = BrickPlan(target_idx, interp_idx, rep_weight, kw, grid_shape, **kwargs)
        self.adj_plan = self.plan

    def _init_tc(self, mode, tc_ops, target_idx, interp_idx, rep_weight, kw, grid_shape, cand, lib):
        """Tensor-core gridder (``csrc/grog_tc.cu``): sample-ordered v6 plans
        with ``n_outer = nsteps`` and the eigen-factored table operands."""
        C = self.C
        if tc_ops is None:
            raise ValueError("tensor-core gridding needs the eigen-factored table (calc_interp_table first)")
        if C > 32:
            raise ValueError("tc kernels cover C <= 32")
        cap = 256 if C <= 16 else 128  # one m-tile per warp above 16 coils
        nd, nsteps = int(tc_ops["ndim"]), int(tc_ops["nsteps"])
        if nd != len(grid_shape):
            raise ValueError("table and plan dimensionality differ")
        bps = int(lib.pgb_grog_tc_blocks_per_sm(C, nd))
        budget = _SMEM_V3 if bps <= 1 else (_SMEM_V3 // bps) - 1024
        chosen = None
        for br in cand:
            cells = br[0] * br[1] * br[2]
            if lib.pgb_grog_tc_smem_bytes(C, cells, nsteps, nd, cap) <= budget:
                chosen = tuple(br)
                break
        if chosen is None:
            raise ValueError("tc kernels: no brick fits shared memory")
        self.mode = mode
        self.brick = chosen
        self.sub_cap = cap
        self.tc = tc_ops
        self.terms = 3 if mode == "tc" else 1
        self.n_outer = nsteps
        self.fwd6 = None
        dev = target_idx.device
        kwt = dict(brick=chosen, n_outer=nsteps, sub_cap=cap, n_cta=_sm_count(dev) * max(bps, 1), sample_order=True,
                   full_subs=True)
        self.plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, cell_rows=True,
                               pack_rows=self.PACK_ROWS_TC, **kwt)
        first = _first_valid_mask(target_idx, kw)
        self.adj_plan = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, mask=first, **kwt)
        self.plan2 = None
        if self.plan.n_valid > self.adj_plan.n_valid:
            self.plan2 = BrickPlan6(target_idx, interp_idx, rep_weight, kw, grid_shape, mask=~first, **kwt)
        for bp in (self.plan, self.adj_plan, self.plan2):
            if bp is not None:
                _pack_axis_indices(bp, nsteps, nd)

    @property
    def n_valid(self):
        return self.plan.n_valid

    def kernel_names(self) -> tuple[str, str]:
        """Names of the (forward, adjoint) main kernels of this gridder."""
        m = self.mode
        if m in ("tc", "tc1"):
            return "grog_grid_tc_kernel", "grog_degrid_tc_kernel"
        if m == "v8":
            return ("grog_grid_v6_kernel" if self.fwd6 is not None else "grog_grid_v8_kernel", "grog_degrid_v8_kernel")
        k = {"v6": "v6_kernel", "global": "kernel"}[m]
        return f"grog_grid_{k}", f"grog_degrid_{k}"

    def launches_per_call(self, adjoint: bool) -> int:
        bp = self.plan
        if adjoint:
            if self.mode in ("v6", "v8", "tc", "tc1"):
                return 1 + (1 if self.plan2 is not None else 0) + (1 if self.adj_plan.zero_src.numel() else 0)
            return 1 + (1 if (not bp.multi and bp.zero_src.numel()) else 0)
        if self.mode in ("tc", "tc1") and self._tile_copies():
            return 1 + (1 if bp.zero_bricks.numel() > bp.n_empty_tail else 0)
        if self.mode in ("v6", "v8", "tc", "tc1"):
            return 1 + (1 if bp.zero_bricks.numel() else 0)
        return 1 + (1 if bp.split_bricks.numel() else 0)

    def _tile_copies(self) -> bool:
        """Whether the tensor-core kernels move brick tiles by tensor copies
        (the launcher's test: coil count a kernel width, even grid and brick
        width, copies switched on); their forward then clears empty bricks
        inside the gridding kernel."""
        C = self.C
        width = (C + 3) // 4 * 4 if C <= 16 else (C + 7) // 8 * 8
        gx, bx = self.plan.grid[-1], self.plan.brick[-1]
        return C == width and gx % 2 == 0 and bx % 2 == 0 and _lib.lib().pgb_grog_tc_use_tma(-1) == 1

    def _outer_ptr(self, h: bool):
        t = self.outer_h if h else self.outer
        return t.data_ptr() if t is not None else None

    def forward(self, data: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """``out (B, C, G)`` <- fused gridding of ``data (B, C, N)``."""
        B, C, N = data.shape
        G = out.shape[-1]
        bp = self.plan
        st = _lib.stream_ptr(data.device)
        if self.tc is not None:
            wf, dt = self.tc["fwd"]
            _lib.call("pgb_grog_grid_tc", data.data_ptr(), N, out.data_ptr(), G, wf.data_ptr(), dt.data_ptr(),
                      self.tc["nsteps"], self.tc["ndim"], C, B, self.terms, _ctypes_ref(bp._c), st)
        elif self.mode == "v8" and self.fwd6 is not None:
            olc = self.outer_lc.data_ptr() if self.outer_lc is not None else None
            _lib.call("pgb_grog_grid_v6", data.data_ptr(), N, out.data_ptr(), G, self.inner_lc.data_ptr(),
                      self.inner.shape[0], olc, self.n_outer, C, B, _ctypes_ref(bp._c), st)
        elif self.mode == "v8":
            _lib.call("pgb_grog_grid_v8", data.data_ptr(), N, out.data_ptr(), G, self.inner.data_ptr(),
                      self.inner.shape[0], self._outer_ptr(False), self.n_outer, C, B, _ctypes_ref(bp._c), st)
        elif self.mode == "v6":
            olc = self.outer_lc.data_ptr() if self.outer_lc is not None else None
            _lib.call("pgb_grog_grid_v6", data.data_ptr(), N, out.data_ptr(), G, self.inner_lc.data_ptr(),
                      self.inner.shape[0], olc, self.n_outer, C, B, _ctypes_ref(bp._c), st)
        else:
            _lib.call("pgb_grog_grid", data.data_ptr(), N, out.data_ptr(), G, self.inner.data_ptr(),
                      self.inner.shape[0], C, B, _ctypes_ref(bp._c_all), st)
        return out

    def adjoint(self, grid: torch.Tensor, out: torch.Tensor) -> torch.Tensor:
        """``out (B, C, N)`` <- adjoint of :meth:`forward` applied to ``grid (B, C, G)``."""
        B, C, G = grid.shape
        N = out.shape[-1]
        bp = self.adj_plan
        st = _lib.stream_ptr(grid.device)
        zs = bp.zero_src.data_ptr() if bp.zero_src.numel() else None
        if self.tc is not None:
            wf, dt = self.tc["adj"]
            sec = _ctypes_ref(self.plan2._c) if self.plan2 is not None else None
            _lib.call("pgb_grog_degrid_tc", grid.data_ptr(), G, out.data_ptr(), N, wf.data_ptr(), dt.data_ptr(),
                      self.tc["nsteps"], self.tc["ndim"], C, B, self.terms, _ctypes_ref(bp._c), sec, zs,
                      int(bp.zero_src.numel()), st)
        elif self.mode == "v8":
            sec = _ctypes_ref(self.plan2._c) if self.plan2 is not None else None
            _lib.call("pgb_grog_degrid_v8", grid.data_ptr(), G, out.data_ptr(), N, self.inner_h.data_ptr(),
                      self.inner_h.shape[0], self._outer_ptr(True), self.n_outer, C, B,
                      _ctypes_ref(bp._c), sec, zs, int(bp.zero_src.numel()), st)
        elif self.mode == "v6":
            sec = _ctypes_ref(self.plan2._c) if self.plan2 is not None else None
            olc = self.outer_h_lc.data_ptr() if self.outer_h_lc is not None else None
            _lib.call("pgb_grog_degrid_v6", grid.data_ptr(), G, out.data_ptr(), N, self.inner_h_lc.data_ptr(),
                      self.inner_h.shape[0], olc, self.n_outer, C, B,
                      _ctypes_ref(bp._c), sec, zs, int(bp.zero_src.numel()), st)
        else:
            _lib.call("pgb_grog_degrid", grid.data_ptr(), G, out.data_ptr(), N, self.inner_h.data_ptr(),
                      self.inner_h.shape[0], C, B, _ctypes_ref(bp._c_nonempty), 1 if bp.multi else 0,
                      zs, int(bp.zero_src.numel()), st)
        return out


# ---------------------------------------------------------------------------
# GrogInterpolator
# ---------------------------------------------------------------------------
class GrogInterpolator:
    """Data-driven GROG interpolator (reference ``GrogInterpolator``).

    Extra keyword ``device`` (default ``"cuda"``) selects the GPU that holds
    the plan and runs every kernel.
    """

    _interpolator_set = False
    _dataset_shape_set = False
    _data: list | None = None

    def __init__(
        self,
        shape,
        coords,
        oversamp=None,
        kernel_width: int = 2,
        kernel_shape: str = "circle",
        time_map=None,
        image_shape=None,
        stack_shape: tuple = (),
        *,
        device=None,
    ):
        self.device = torch.device(device if device is not None else _DEFAULT_DEVICE)
        coords_arr = coords.detach().cpu().numpy() if isinstance(coords, torch.Tensor) else np.asarray(coords)
        s_eff = tuple(int(s) for s in (stack_shape or ()))
        if not s_eff and coords_arr.ndim == 4:
            s_eff = (int(coords_arr.shape[0]),)
        self.plan = _create_plan(
            shape, coords_arr, oversamp, kernel_width, kernel_shape, time_map, s_eff, self.device
        )
        _attach_fft_plan(self.plan, image_shape)
        self._brick_plans = None
        self._density = None

    # -- metadata -----------------------------------------------------------
    def metadata(self):
        oshape = np.ceil(np.asarray(self.plan.shape) * np.asarray(self.plan.oversamp)).astype(int).tolist()
        return SimpleNamespace(
            shape=tuple(self.plan.shape),
            oshape=tuple(oshape),
            target_idx=self.plan.target_idx,
            weights=self.plan.weights,
            time_map=self.plan.time_map,
        )

    def fft_plan(self, image_shape=None):
        if image_shape is not None and tuple(np.atleast_1d(image_shape)) != tuple(self.plan.image_shape):
            import copy

            plan = copy.copy(self.plan)
            _attach_fft_plan(plan, image_shape)
            return plan
        return self.plan

    # -- table ----------------------------------------------------------------
    def calc_interp_table(self, train_data, lamda: float = 0.01, precision: int = 1, *, fit_dtype=None,
                          fit_on_device: bool = False):
        """Fit the GRAPPA shift table and quantise every replica's shift.

        ``fit_dtype=torch.complex128`` runs the fit in FP64 (table cast back);
        ``fit_on_device=True`` runs it in FP64 with the least-squares Gram
        matrices accumulated on this interpolator's GPU.
        """
        if isinstance(train_data, torch.Tensor):
            train_data = train_data.detach().cpu()
        table, nsteps, ndim, factors = KernelTable(
            train_data, self.plan.radius, precision, lamda, fit_dtype, return_factors=True,
            fit_device=self.device if fit_on_device else None,
        )
        self._factors = factors
        self._nsteps = int(nsteps)
        dist = self.plan.distances
        if dist is None:
            raise RuntimeError("calc_interp_table: plan distances were already released")
        K = int(table.shape[0])
        pfac = 10.0**precision
        stepsize = 10 ** (-precision)
        lead = tuple(dist.shape[:-1])
        R = int(np.prod(lead))
        idx = torch.empty(lead, dtype=torch.int64, device=self.device)
        d = dist.contiguous()
        _lib.call(
            "pgb_plan_quantize", d.data_ptr(), R, int(dist.shape[-1]), float(self.plan.radius),
            float(np.float32(pfac)), float(np.float32(stepsize)), int(nsteps), K, idx.data_ptr(),
            _lib.stream_ptr(self.device),
        )
        self.plan.distances = None
        self._interp_kernel = torch.as_tensor(table)  # host copy (reference field)
        self._table_d = self._interp_kernel.to(self.device).contiguous()
        self._table_h_d = self._table_d.conj().transpose(-1, -2).contiguous()
        self._interp_idx = idx
        self._interpolator_set = True
        self._brick_plans = None
        self._fit_args = (train_data, float(self.plan.radius), precision, lamda, fit_dtype)
        self._tc_ops = None

    def _tc_operands(self) -> dict:
        """Eigen-factored table operands of the tensor-core gridder (built once)."""
        if getattr(self, "_tc_ops", None) is None:
            from ._grappa import eigen_factors
            from ._tc import tc_operands

            train, radius, precision, lamda, fit_dtype = self._fit_args
            ef = eigen_factors(train, radius, precision, lamda, fit_dtype)
            self._tc_ops = tc_operands(ef, int(self._interp_kernel.shape[-1]), self.device)
        return self._tc_ops

    def set_dataset_shape(self, shape):
        if self._dataset_shape_set:
            return
        self.dataset_shape = tuple(shape)
        self._dataset_shape_set = True

    # -- helpers ----------------------------------------------------------------
    def _to_device(self, data):
        is_numpy = isinstance(data, np.ndarray)
        t = torch.as_tensor(data)
        src_dev = t.device
        if not t.is_complex():
            t = t.to(torch.complex64)
        if t.device.type == "cpu" and t.is_pinned():
            # page-locked input: DMA straight from the caller's buffer
            return t.to(self.device, non_blocking=True), is_numpy, src_dev
        return t.to(self.device), is_numpy, src_dev

    @staticmethod
    def _to_host(res: torch.Tensor, is_numpy: bool, src_dev):
        """Return a result to the caller's device; host results land in page-locked memory."""
        if not is_numpy and src_dev.type != "cpu":
            return res.to(src_dev)
        host = torch.empty(res.shape, dtype=res.dtype, pin_memory=True)
        host.copy_(res, non_blocking=True)
        torch.cuda.current_stream(res.device).synchronize()
        return host.numpy() if is_numpy else host

    def _check_c64(self, t):
        if t.dtype != torch.complex64:
            raise RuntimeError(
                f"GrogInterpolator: the fused GROG kernels compute in complex64, got {t.dtype}"
            )

    def _split_layout(self, data: torch.Tensor):
        plan = self.plan
        s_shape = tuple(plan.stack_shape)
        s_ndim = len(s_shape)
        spatial = tuple(int(s) for s in plan.target_idx.shape[s_ndim:-1])
        kw = int(plan.target_idx.shape[-1])
        cpos = data.ndim - len(spatial) - 1
        if cpos < s_ndim:
            raise ValueError(
                f"data.ndim={data.ndim} too small for stack_shape={s_shape} + spatial={spatial} (+coils)"
            )
        if s_ndim and tuple(int(s) for s in data.shape[cpos - s_ndim : cpos]) != s_shape:
            raise ValueError(
                f"data stack prefix {tuple(data.shape[cpos - s_ndim:cpos])} != plan.stack_shape {s_shape}"
            )
        if tuple(int(s) for s in data.shape[cpos + 1 :]) != spatial:
            raise ValueError(f"data spatial dims {tuple(data.shape[cpos + 1:])} != plan {spatial}")
        batch = tuple(int(s) for s in data.shape[: cpos - s_ndim])
        return batch, s_shape, int(data.shape[cpos]), spatial, kw

    def _brick(self, s: int) -> "GrogGridder":
        if self._brick_plans is None:
            self._brick_plans = {}
        bp = self._brick_plans.get(s)
        if bp is None:
            plan = self.plan
            s_total = int(np.prod(plan.stack_shape)) if plan.stack_shape else 1
            kw = int(plan.target_idx.shape[-1])
            tgt = plan.target_idx.reshape(s_total, -1)[s]
            w = plan.weights.reshape(s_total, -1)[s].clamp(min=0.0)
            sw = torch.sqrt(w)
            rep_w = sw * sw
            idx = self._interp_idx.reshape(s_total, -1)[s]
            mode = getattr(self, "gridder_mode", None)
            tc_ops = self._tc_operands() if mode in ("tc", "tc1") else None
            bp = GrogGridder(tgt, idx, rep_w, kw, plan.grid_shape, self._interp_kernel, self._factors,
                             self._nsteps, mode=mode, tc_ops=tc_ops, brick=getattr(self, "gridder_brick", None))
            self._brick_plans[s] = bp
        return bp

    # -- forward interpolation ------------------------------------------------
    def interpolate(self, data, shot_index=None, ret_image: bool = False, grid: bool = False):
        """GROG-shifted replicas ``(*batch, *stack, C, n_samples)`` (see reference)."""
        if not self._interpolator_set:
            raise RuntimeError("GRAPPA kernels not set. Call calc_interp_table() first.")
        if grid and ret_image:
            raise ValueError("'grid' and 'ret_image' are mutually exclusive.")
        t, is_numpy, src_dev = self._to_device(data)
        if shot_index is not None:
            if np.isscalar(shot_index):
                shot_index = (shot_index,)
            g = self._grid_shot(t, tuple(shot_index))
            if self._data is None:
                self._data = []
            self._data.append(g)
            return None
        if grid:
            kgrid, mplan = self._grid_kspace(t)
            if is_numpy:
                from ..operator._masked_fft import MaskedFFTPlan

                npplan = MaskedFFTPlan(
                    grid_shape=mplan.grid_shape, image_shape=mplan.image_shape,
                    stack_shape=mplan.stack_shape, mask=mplan.mask.cpu().numpy(),
                    density=mplan.density.cpu().numpy(),
                )
                return self._to_host(kgrid, True, src_dev), npplan
            return self._to_host(kgrid, False, src_dev), mplan
        sparse = self._sparse_flat(t)
        if ret_image:
            from ..operator._sparse_fft import SparseFFT

            plan = self.plan
            op = SparseFFT(plan=plan)
            pre_w = plan.pre_weights.to(sparse.dtype)
            pw = pre_w.unsqueeze(-2) if pre_w.ndim > 1 else pre_w.unsqueeze(0)
            img = op.adjoint(sparse * pw)
            ax = img.ndim - len(plan.image_shape) - 1
            image = img.abs().square().sum(ax).sqrt()
            return image.cpu().numpy() if is_numpy else image.to(src_dev)
        return self._to_host(sparse, is_numpy, src_dev)

    def __call__(self, data, shot_index=None, ret_image=False, grid=False):
        return self.interpolate(data, shot_index, ret_image, grid)

    def _sparse_flat(self, data: torch.Tensor) -> torch.Tensor:
        """Replica expansion, returned as ``(*batch, *stack, C, n_samples)``."""
        self._check_c64(data)
        batch, s_shape, C, spatial, kw = self._split_layout(data)
        B = int(np.prod(batch)) if batch else 1
        S = int(np.prod(s_shape)) if s_shape else 1
        N = int(np.prod(spatial))
        d = data.reshape(B, S, C, N)
        out = torch.empty(B, S, C, N * kw, dtype=data.dtype, device=data.device)
        idx = self._interp_idx.reshape(S, N * kw)
        st = _lib.stream_ptr(data.device)
        for s in range(S):
            ds = d[:, s].contiguous() if S > 1 else d.reshape(B, C, N).contiguous()
            os_ = torch.empty(B, C, N * kw, dtype=data.dtype, device=data.device) if S > 1 else out.view(B, C, N * kw)
            _lib.call(
                "pgb_grog_expand", ds.data_ptr(), N, kw, idx[s].contiguous().data_ptr(),
                self._table_d.data_ptr(), self._table_d.shape[0], C, B, os_.data_ptr(), st,
            )
            if S > 1:
                out[:, s] = os_
        return out.reshape(*batch, *s_shape, C, N * kw)

    # -- gridded output (fused kernel) ------------------------------------------
    def _density_grid(self) -> torch.Tensor:
        """Sum of squared sorted sqrt-weights per cell, ``(*stack, *grid_shape)``."""
        if self._density is None:
            plan = self.plan
            S = int(np.prod(plan.stack_shape)) if plan.stack_shape else 1
            G = int(plan.grid_size)
            dens = torch.zeros(S, G, dtype=torch.float32, device=self.device)
            idx = plan.indices.reshape(S, -1)
            sw = plan.sqrt_weights.reshape(S, -1)
            from .. import _ext

            for s in range(S):
                w_sq = (sw[s] * sw[s]).contiguous()
                _ext.psf_scatter_scalar(dens[s], idx[s].contiguous(), w_sq)
            self._density = dens.reshape(*plan.stack_shape, *plan.grid_shape)
        return self._density

    def _grid_kspace(self, data: torch.Tensor):
        from ..operator._masked_fft import MaskedFFTPlan

        self._check_c64(data)
        plan = self.plan
        batch, s_shape, C, spatial, kw = self._split_layout(data)
        B = int(np.prod(batch)) if batch else 1
        S = int(np.prod(s_shape)) if s_shape else 1
        N = int(np.prod(spatial))
        G = int(plan.grid_size)
        d = data.reshape(B, S, C, N)
        out = torch.empty(B, S, C, G, dtype=data.dtype, device=data.device)
        for s in range(S):
            bp = self._brick(s)
            ds = d[:, s].contiguous()
            o = torch.empty(B, C, G, dtype=data.dtype, device=data.device) if S > 1 else out.view(B, C, G)
            bp.forward(ds, o)
            if S > 1:
                out[:, s] = o
        density = self._density_grid()
        mask = (density > 0).float()
        kgrid = out.reshape(*batch, *s_shape, C, *plan.grid_shape)
        mplan = MaskedFFTPlan(
            grid_shape=tuple(plan.grid_shape), image_shape=tuple(plan.image_shape),
            stack_shape=tuple(s_shape), mask=mask, density=density,
        )
        return kgrid, mplan

    def grid(self, data) -> torch.Tensor:
        """Fused gridding only: ``interpolate(data, grid=True)[0]`` without the plan object."""
        if not self._interpolator_set:
            raise RuntimeError("GRAPPA kernels not set. Call calc_interp_table() first.")
        t, is_numpy, src_dev = self._to_device(data)
        self._check_c64(t)
        plan = self.plan
        batch, s_shape, C, spatial, kw = self._split_layout(t)
        B = int(np.prod(batch)) if batch else 1
        S = int(np.prod(s_shape)) if s_shape else 1
        N = int(np.prod(spatial))
        G = int(plan.grid_size)
        d = t.reshape(B, S, C, N)
        out = torch.empty(B, S, C, G, dtype=t.dtype, device=t.device)
        for s in range(S):
            ds = d[:, s].contiguous()
            o = torch.empty(B, C, G, dtype=t.dtype, device=t.device) if S > 1 else out.view(B, C, G)
            self._brick(s).forward(ds, o)
            if S > 1:
                out[:, s] = o
        res = out.reshape(*batch, *s_shape, C, *plan.grid_shape)
        return self._to_host(res, is_numpy, src_dev)

    def degrid(self, kgrid):
        """Adjoint of :meth:`grid` / ``interpolate(grid=True)`` with respect to ``data``.

        ``kgrid (*batch, *stack, C, *grid_shape)`` -> ``(*batch, *stack, C, *spatial)``:
        ``x[n] = sum_{valid replicas r of n} w_r * T[e_r]^H @ kgrid[cell_r]``.
        """
        if not self._interpolator_set:
            raise RuntimeError("GRAPPA kernels not set. Call calc_interp_table() first.")
        t, is_numpy, src_dev = self._to_device(kgrid)
        self._check_c64(t)
        plan = self.plan
        s_shape = tuple(plan.stack_shape)
        gnd = len(plan.grid_shape)
        if tuple(t.shape[-gnd:]) != tuple(plan.grid_shape):
            raise ValueError(f"kgrid trailing dims {tuple(t.shape[-gnd:])} != grid_shape {plan.grid_shape}")
        C = int(t.shape[-gnd - 1])
        lead = tuple(int(s) for s in t.shape[: t.ndim - gnd - 1])
        if s_shape and tuple(lead[len(lead) - len(s_shape):]) != s_shape:
            raise ValueError(f"kgrid stack prefix {lead} must end with {s_shape}")
        batch = lead[: len(lead) - len(s_shape)]
        B = int(np.prod(batch)) if batch else 1
        S = int(np.prod(s_shape)) if s_shape else 1
        spatial = tuple(int(s) for s in plan.target_idx.shape[len(s_shape):-1])
        N = int(np.prod(spatial))
        G = int(plan.grid_size)
        g = t.reshape(B, S, C, G)
        out = torch.empty(B, S, C, N, dtype=t.dtype, device=t.device)
        for s in range(S):
            gs = g[:, s].contiguous()
            o = torch.empty(B, C, N, dtype=t.dtype, device=t.device) if S > 1 else out.view(B, C, N)
            bp = self._brick(s)
            bp.adjoint(gs, o)
            if bp.tc is not None:
                self._tc_pending = True
            if S > 1:
                out[:, s] = o
        res = out.reshape(*batch, *s_shape, C, *spatial)
        host = self._to_host(res, is_numpy, src_dev)
        if is_numpy or src_dev.type == "cpu" or _SYNC_CHECK:
            self.check_errors()  # the launching stream has been synchronised (or is, here)
        return host

    def check_errors(self) -> None:
        """Raise RuntimeError if a tensor-core adjoint launched by this
        interpolator since the last check gave up waiting for a brick tile
        (its result is then incomplete).  Synchronises the device.

        ``degrid`` runs this check itself when it returns a host result, and
        after every call when ``PYGROG_B200_SYNC_CHECK=1``; a device-resident
        result is checked here, or by the next host-returning ``degrid``.
        """
        if not getattr(self, "_tc_pending", False):
            return
        if torch.cuda.is_current_stream_capturing():
            return
        torch.cuda.synchronize(self.device)
        self._tc_pending = False
        _lib.check_tc_timeouts("GrogInterpolator.degrid")

    # -- shot-by-shot ---------------------------------------------------------------
    def _grid_shot(self, data: torch.Tensor, shot_index: tuple) -> torch.Tensor:
        """Grid one shot ``(C, npts)`` with the plan weights (reference ``_grid_shot``)."""
        from .. import _ext

        plan = self.plan
        tgt = plan.target_idx[shot_index].reshape(-1)
        w = plan.weights[shot_index].reshape(-1).to(torch.float32)
        idx = self._interp_idx[shot_index].reshape(-1)
        C = int(data.shape[0])
        npts = int(data.shape[-1])
        kw = int(plan.target_idx.shape[-1])
        self._check_c64(data)
        rep = data.reshape(C, npts, 1).expand(C, npts, kw).reshape(C, npts * kw)
        x = rep.transpose(0, 1).reshape(npts * kw, 1, C).contiguous()
        y = _ext.grog_interpolate(x, idx.contiguous(), self._table_d)[:, 0, :]  # (npts*kw, C)
        valid = tgt >= 0
        G = int(np.prod(plan.grid_shape))
        out = torch.zeros(C, G, dtype=data.dtype, device=data.device)
        cells = torch.where(valid, tgt, torch.zeros_like(tgt)).contiguous()
        wv = torch.where(valid, w, torch.zeros_like(w)).contiguous()
        for c in range(C):
            _ext.scatter_add(out[c], y[:, c].contiguous(), cells, wv)
        return out

    def collect_shots(self) -> torch.Tensor:
        if self._data is None or len(self._data) == 0:
            raise RuntimeError("No shots accumulated.")
        out = torch.stack(self._data, dim=0).sum(dim=0)
        self._data = None
        return out.reshape(out.shape[0], *self.plan.grid_shape)
