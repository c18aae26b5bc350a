"""Served GROG + CG-SENSE reconstructions on one GPU.

A *protocol* is a trajectory with its GROG plan and table, coil maps and
Toeplitz PSF, all resident on the device (built once, as the reference's
``GrogInterpolator`` / ``SparseFFT(plan, smaps, toeplitz=True)`` /
``solve(method="cg")`` chain would build them, ``calib/_grog.py:302-555``,
``operator/_sparse_fft.py:221-318``, ``_solve/_mixin.py:84-158``).  A
*request* brings new non-Cartesian k-space for one protocol and asks for
``x = argmin |A x - b|^2 + damp |x|^2`` by ``max_iter`` CG iterations.

The server loop runs continuous batching:

* requests that have arrived wait in per-protocol queues;
* whenever one of ``n_slots`` CUDA streams is free, the protocol whose oldest
  request waited longest is served: up to ``max_batch`` of its queued
  requests are stacked into one batch -- one GROG interpolation, one SparseFFT
  adjoint and one frame-batched CG (``BatchedDeviceCG``) for all of them --
  provided the batch's device-memory estimate fits the budget still free;
* batches on different streams overlap on the device; completion is
  detected with CUDA events, results land in page-locked host memory.

Each frame of a batch runs the single-request recurrence with its own
scalars, so a request's result does not depend on what it was batched with
(up to FP32 reduction order in cuFFT's batched transforms).
"""

from __future__ import annotations

__all__ = ["ReconProtocol", "Request", "ReconServer", "poisson_arrivals"]

import collections
import dataclasses
import time

import numpy as np
import torch

from ._solve import BatchedDeviceCG
from .calib import GrogInterpolator
from .operator import SparseFFT, with_subspace


@dataclasses.dataclass
class Request:
    rid: int
    protocol: str
    arrival: float  # seconds after the start of the run
    data: torch.Tensor  # (C, *spatial) complex64, page-locked host memory
    keep: bool = False  # keep the reconstructed image in ``result``
    t_start: float | None = None
    t_done: float | None = None
    batch: int = 0
    result: torch.Tensor | None = None

    @property
    def latency(self) -> float:
        return float(self.t_done - self.arrival)


class ReconProtocol:
    """Resident GROG plan + table + SENSE maps + Toeplitz PSF of one trajectory."""

    def __init__(self, name: str, shape, coords, acr, smaps, *, oversamp=None, kernel_width: int = 2,
                 kernel_shape: str = "circle", precision: int = 1, lamda: float = 0.01, max_iter: int = 20,
                 damp: float = 1e-3, basis=None, encoding_axis: int = -3, device="cuda"):
        self.name = name
        self.device = torch.device(device)
        self.interp = GrogInterpolator(shape=shape, coords=coords, oversamp=oversamp, kernel_width=kernel_width,
                                       kernel_shape=kernel_shape, device=self.device)
        self.interp.calc_interp_table(acr, lamda=lamda, precision=precision)
        sm = torch.as_tensor(smaps).to(self.device, torch.complex64)
        base = SparseFFT(plan=self.interp.plan, smaps=sm, toeplitz=True, device=self.device)
        self.subspace = basis is not None
        if self.subspace:
            # low-rank subspace (gadgets/_subspace.py): unknowns are K coefficient images
            self.op = with_subspace(base, torch.as_tensor(basis), encoding_axis=encoding_axis)
            self.image_shape = (self.op.K, *tuple(base.image_shape))
        else:
            self.op = base
            self.image_shape = tuple(base.image_shape)
        self.pre_w = self.interp.plan.pre_weights.to(self.device, torch.float32)
        self.natural_shape = tuple(base.natural_shape)
        self.C = int(sm.shape[0])
        self.spatial = tuple(int(s) for s in np.asarray(coords).shape[:-1])
        self.max_iter = int(max_iter)
        self.damp = float(damp)
        self._solvers: dict = {}
        self._io: dict = {}  # slot -> (device input, page-locked output), allocated once
        self._cap = 1

    @property
    def data_shape(self):
        return (self.C, *self.spatial)

    def bytes_per_request(self) -> int:
        """Device-memory estimate of one request inside a batch (inputs, replicas,
        FFT buffers, CG vectors)."""
        n_s = int(np.prod(self.spatial))
        n_rep = int(self.interp.plan.n_samples)
        G = int(np.prod(self.op.grid_shape)) * (self.op.K if self.subspace else 1)
        img = int(np.prod(self.image_shape))
        return 8 * (self.C * n_s + 3 * self.C * n_rep + 3 * self.C * G + 6 * img)

    def prepare(self, max_batch: int, n_slots: int, graphs: bool = True):
        """Allocate the per-slot solvers, warm cuFFT plans and the PSF for every batch
        size, and record each slot's CG loop as a CUDA graph per batch size."""
        self._cap = int(max_batch)
        self._prepared_for = (int(max_batch), int(n_slots), bool(graphs))
        self._solvers, self._io = {}, {}
        for s in range(n_slots):
            self._solvers[s] = BatchedDeviceCG(self.op, self._cap, self.image_shape, self.device,
                                               damp=self.damp, tol=0.0)
            self._io[s] = (torch.empty((self._cap, *self.data_shape), dtype=torch.complex64, device=self.device),
                           torch.empty((self._cap, *self.image_shape), dtype=torch.complex64, pin_memory=True))
        x = torch.zeros(max_batch, *self.data_shape, dtype=torch.complex64, device=self.device)
        for F in range(1, max_batch + 1):
            self.recon(x[:F], 0, max_iter=1)
        torch.cuda.synchronize(self.device)
        if graphs:
            for s in range(n_slots):
                for F in range(1, max_batch + 1):
                    self._solvers[s].capture(F, self.max_iter)
            torch.cuda.synchronize(self.device)

    def recon(self, data_dev: torch.Tensor, slot: int, max_iter: int | None = None) -> torch.Tensor:
        """``data_dev (F, C, *spatial)`` on the device -> images ``(F, *image_shape)`` (stream-ordered)."""
        sparse = self.interp.interpolate(data_dev)  # (F, C, n_samples)
        if self.subspace:  # the subspace operator applies the sample weights itself
            AHb = self.op.adjoint(sparse.reshape(sparse.shape[0], self.C, *self.natural_shape))
        else:
            AHb = self.op.adjoint(sparse * self.pre_w)  # (F, *image_shape)
        cg = self._solvers[slot]
        cg.load(AHb)
        return cg.run(self.max_iter if max_iter is None else max_iter)


def poisson_arrivals(rate: float, duration: float, rng: np.random.Generator) -> np.ndarray:
    """Arrival times of a Poisson process of ``rate`` per second over ``duration`` seconds."""
    t, out = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            return np.asarray(out)
        out.append(t)


class ReconServer:
    """Continuous-batching request loop over resident protocols (module docstring)."""

    def __init__(self, protocols: dict, *, mem_budget: int, max_batch: int = 8, n_slots: int = 4,
                 device="cuda", graphs: bool = True):
        self.protocols = protocols
        self.device = torch.device(device)
        self.mem_budget = int(mem_budget)
        self.max_batch = int(max_batch)
        self.n_slots = int(n_slots)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(self.n_slots)]
        self._key = (self.max_batch, self.n_slots, bool(graphs))
        for p in protocols.values():
            p.prepare(self.max_batch, self.n_slots, graphs=graphs)
            if p.bytes_per_request() > self.mem_budget:
                raise ValueError(f"protocol {p.name} needs more than the memory budget for one request")

    def _ensure_prepared(self) -> None:
        """A protocol keeps the per-slot buffers and graphs of the last server
        that prepared it; re-prepare the ones another server configuration
        has taken over since (a protocol serves one server at a time)."""
        for p in self.protocols.values():
            if getattr(p, "_prepared_for", None) != self._key:
                p.prepare(self._key[0], self._key[1], graphs=self._key[2])

    def _launch(self, slot: int, proto: ReconProtocol, reqs: list):
        s = self.streams[slot]
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            F = len(reqs)
            d_all, h_all = proto._io[slot]  # the slot's buffers: free while the slot is free
            d = d_all[:F]
            for i, r in enumerate(reqs):
                d[i].copy_(r.data, non_blocking=True)
            x = proto.recon(d, slot)
            host = h_all[:F]
            host.copy_(x, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(s)
        return ev, host

    def run(self, requests: list, realtime: bool = True) -> dict:
        """Serve ``requests`` (arrival times relative to the start); returns a report.

        ``realtime=False`` admits every request at time 0 (closed-loop throughput)."""
        self._ensure_prepared()
        torch.cuda.synchronize(self.device)
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        ready = {name: collections.deque() for name in self.protocols}
        free = list(range(self.n_slots))
        inflight = []
        used = 0
        done = 0
        n = len(requests)
        t0 = time.perf_counter()
        while done < n:
            now = time.perf_counter() - t0
            progressed = False
            while pending and (not realtime or pending[0].arrival <= now):
                r = pending.popleft()
                ready[r.protocol].append(r)
                progressed = True
            for item in list(inflight):
                ev, host, reqs, slot, nbytes = item
                if ev.query():
                    t = time.perf_counter() - t0
                    for i, r in enumerate(reqs):
                        r.t_done = t
                        if r.keep:
                            r.result = host[i].clone()
                    inflight.remove(item)
                    free.append(slot)
                    used -= nbytes
                    done += len(reqs)
                    progressed = True
            while free:
                cands = [(q[0].arrival, name) for name, q in ready.items() if q]
                if not cands:
                    break
                _, name = min(cands)
                proto = self.protocols[name]
                q = ready[name]
                F = min(len(q), self.max_batch)
                per = proto.bytes_per_request()
                F = min(F, max(0, (self.mem_budget - used) // per))
                if F == 0:
                    break  # admission waits for memory to free up
                reqs = [q.popleft() for _ in range(F)]
                slot = free.pop()
                t = time.perf_counter() - t0
                for r in reqs:
                    r.t_start = t
                    r.batch = F
                ev, host = self._launch(slot, proto, reqs)
                inflight.append((ev, host, reqs, slot, F * per))
                used += F * per
                progressed = True
            if not progressed:
                time.sleep(2e-5)
        t_end = time.perf_counter() - t0
        if not realtime:  # closed loop: every request was there at time 0
            for r in requests:
                r.arrival = 0.0
        lat = np.asarray([r.latency for r in requests]) * 1e3
        first = min(r.arrival for r in requests) if realtime else 0.0
        return {
            "requests": n,
            "recons_per_s": n / (t_end - first),
            "p50_ms": float(np.percentile(lat, 50)),
            "p95_ms": float(np.percentile(lat, 95)),
            "p99_ms": float(np.percentile(lat, 99)),
            "mean_batch": float(np.mean([r.batch for r in requests])),
            "wall_s": t_end,
        }
