"""Timed CPU arm: the reference's own CPU implementation of the GROG fwd+adj path.

TEST/BASELINE INFRASTRUCTURE ONLY (used by ``bench.py``'s CPU baseline and
``--impl reference``; never by the product).

Forward = ``GrogInterpolator.interpolate(data, grid=True)`` of the reference:
the Python glue of ``calib/_grog.py:668-695`` (replicate, transpose,
``grog_interpolate``, copy back, permute) and ``calib/_grog.py:736-821``
(``pre_weights`` multiply, per-coil sort + ``scatter_add``), restated here
step for step, calling the reference's compiled C++ kernels from
``oracle/_ref`` (built from its sources by ``oracle/build_ref.py``).

Adjoint: the reference has no adjoint of the GROG shift; it is composed from
the same reference kernels (per-coil ``gather`` in sorted order, un-sort,
``pre_weights``, ``grog_interpolate`` with the conjugate-transposed table,
sum over the kw replicas of each sample).

When ``oracle/_ref`` is not built, the numpy restatement in ``oracle.grog``
is timed instead (``kind="port"``).
"""

from __future__ import annotations

import os
import time

import numpy as np

from . import grog as og


class ReferenceCPU:
    def __init__(self, shape, coords, oversamp, kernel_width, kernel_shape, acr, precision, lamda,
                 threads: int | None = None):
        import torch

        self.torch = torch
        self.threads = threads or os.cpu_count() or 1
        torch.set_num_threads(self.threads)
        os.environ.setdefault("OMP_NUM_THREADS", str(self.threads))
        self.plan = og.create_plan(shape, coords, oversamp, kernel_width, kernel_shape)
        self.fplan = og.fft_plan(self.plan)
        tab, n, nd = og.kernel_table(acr, 0.5, precision, lamda)
        K = tab.shape[0]
        self.interp_idx = og.quantize(self.plan["distances"], precision, n, K)
        self.table = tab
        self.kw = int(self.plan["kw"])
        self.N = int(np.prod(coords.shape[:-1]))
        self.G = int(np.prod(self.plan["grid_shape"]))
        try:
            from . import build_ref

            self.ext = build_ref.load()
            self.kind = "reference"
        except Exception:  # noqa: BLE001 - fall back to the numpy port
            self.ext = None
            self.kind = "port"
        t = torch
        self.t_idx = t.from_numpy(self.interp_idx.reshape(-1).astype(np.int64))
        self.t_tab = t.from_numpy(np.ascontiguousarray(tab))
        self.t_tabh = t.from_numpy(np.ascontiguousarray(np.conj(np.swapaxes(tab, -1, -2))))
        self.t_indices = t.from_numpy(self.fplan["indices"])
        self.t_sqw = t.from_numpy(self.fplan["sqrt_weights"])
        self.t_sort = t.from_numpy(self.fplan["sort_perm"])
        self.t_inv = t.from_numpy(self.fplan["inv_perm"])
        self.t_prew = self.t_sqw[self.t_inv]

    def use_table(self, table: np.ndarray) -> None:
        """Run the reference kernels with ``table`` (K, C, C) instead of the
        oracle's own fit (isolates the gridding path from the table fit)."""
        t = self.torch
        self.table = np.ascontiguousarray(table)
        self.t_tab = t.from_numpy(self.table)
        self.t_tabh = t.from_numpy(np.ascontiguousarray(np.conj(np.swapaxes(self.table, -1, -2))))

    def _interpolate(self, data: np.ndarray):
        """calib/_grog.py:668-695: replicate every sample kw times, shift each
        replica by its table entry (``grog_interpolate``), back to (C, N kw)."""
        t = self.torch
        C, N = data.shape
        kw = self.kw
        x = t.from_numpy(np.ascontiguousarray(data))
        rep = x.unsqueeze(-1).expand(-1, -1, kw).reshape(C, N * kw)
        di = rep.T.reshape(N * kw, 1, C).contiguous()
        res = self.ext.grog_interpolate(di, self.t_idx, self.t_tab)
        di.copy_(res)
        return di.permute(1, 2, 0).contiguous().reshape(C, N * kw)

    def interpolate(self, data: np.ndarray) -> np.ndarray:
        """data (C, N) complex64 -> shifted replicas (C, N kw) (``interpolate(data)``)."""
        if self.ext is None:
            return og.interpolate(data[None], self.interp_idx.reshape(self.N, -1), self.table)[0]
        return self._interpolate(data).numpy()

    def forward(self, data: np.ndarray) -> np.ndarray:
        """data (C, N) complex64 -> kgrid (C, G)."""
        if self.ext is None:
            return og.grid(data[None], self.interp_idx, self.table, self.plan, self.fplan)[0][0]
        t = self.torch
        C, N = data.shape
        sparse = self._interpolate(data)
        sdc = sparse * self.t_prew.to(sparse.dtype)
        grid = t.zeros(C, self.G, dtype=sparse.dtype)
        for c in range(C):
            self.ext.scatter_add(grid[c], sdc[c][self.t_sort], self.t_indices, self.t_sqw)
        return grid.numpy()

    def adjoint(self, kgrid: np.ndarray) -> np.ndarray:
        """kgrid (C, G) -> samples (C, N)."""
        if self.ext is None:
            return og.degrid(kgrid[None], self.interp_idx, self.table, self.plan)[0]
        t = self.torch
        C = kgrid.shape[0]
        kw = self.kw
        g = t.from_numpy(kgrid)
        sp = t.empty(C, self.N * kw, dtype=g.dtype)
        for c in range(C):
            sp[c] = self.ext.gather(g[c], self.t_indices, self.t_sqw)[self.t_inv]
        sp = sp * self.t_prew.to(sp.dtype)
        di = sp.T.reshape(self.N * kw, 1, C).contiguous()
        res = self.ext.grog_interpolate(di, self.t_idx, self.t_tabh)
        return res.reshape(self.N, kw, C).sum(1).T.contiguous().numpy()

    def time_step(self, data: np.ndarray, repeats: int = 1) -> float:
        """Seconds per fwd+adj step (minimum over ``repeats``)."""
        best = float("inf")
        for _ in range(repeats):
            t0 = time.perf_counter()
            kg = self.forward(data)
            self.adjoint(kg)
            best = min(best, time.perf_counter() - t0)
        return best
