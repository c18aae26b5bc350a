"""Many reconstructions of uneven shape in one CUDA graph launch.

Config c3 reconstructs a batch of independent 2-D slices whose trajectory
length, grid size and coil count all differ.  The reference has no batched
form for that: stacking needs equal shapes (``calib/_grog.py:114-132``,
``operator/_sparse_fft.py:461-500``), so it loops over the slices.  Here
the whole batch -- for every slice the host-to-device copy of its k-space,
the GROG interpolation (``calib/_grog.py:437-555``), the pre-weighted
SparseFFT adjoint (``operator/_sparse_fft.py:505-680``), ``max_iter`` CG
iterations on the Toeplitz normal operator (``_solve/_solvers.py:49-139``,
FP64 device scalars) and the device-to-host copy of the image -- is recorded
once as one CUDA graph in which every slice is its own branch.  A batch is
then a single graph launch: the GPU runs the branches side by side, so the
small kernels and FFTs of the small slices fill the device while the large
slices run, with no host work between stages.

Each branch owns its buffers (k-space, replicas, FFT grids, CG vectors and
its reduction scratch), so a slice's result does not depend on the others
in the batch; the branch runs exactly the kernels of
:meth:`pygrog_b200.serve.ReconProtocol.recon`.
"""

from __future__ import annotations

__all__ = ["UnevenBatch"]

import gc
import math

import torch

from ._solve import BatchedDeviceCG


class UnevenBatch:
    """One CUDA graph reconstructing one request of each protocol in ``protocols``.

    ``protocols``: :class:`pygrog_b200.serve.ReconProtocol` objects (their
    plans, tables, coil maps and PSFs resident on ``device``).  ``lanes``:
    number of parallel chains in the graph (default: one per protocol).  Inputs go in
    :attr:`host_in` (page-locked, one ``(C, *spatial)`` tensor per protocol),
    :meth:`run` launches the graph and returns :attr:`host_out` (page-locked
    ``image_shape`` tensors).  The graph copies from and to these very
    tensors: write into them, and replace them (other page-locked tensors of
    the same shapes) only before the graph is captured.
    """

    def __init__(self, protocols, device=None, lanes: int | None = None):
        self.protos = list(protocols)
        if not self.protos:
            raise ValueError("UnevenBatch needs at least one protocol")
        self.device = torch.device(device) if device is not None else self.protos[0].device
        self.host_in = [torch.zeros(p.data_shape, dtype=torch.complex64, pin_memory=True) for p in self.protos]
        self.host_out = [torch.empty(p.image_shape, dtype=torch.complex64, pin_memory=True) for p in self.protos]
        self._dev_in = [torch.empty((1, *p.data_shape), dtype=torch.complex64, device=self.device)
                        for p in self.protos]
        self._cg = [BatchedDeviceCG(p.op, 1, p.image_shape, self.device, damp=p.damp, tol=0.0) for p in self.protos]
        # parallel chains of the graph: every slice its own branch by default;
        # with `lanes`, the slices are dealt largest first (samples x coils x
        # CG iterations) to the lane with the least work, each lane a chain
        n = len(self.protos) if lanes is None else max(1, min(int(lanes), len(self.protos)))
        cost = [p.C * max(math.prod(p.spatial), 1) * max(p.max_iter, 1) for p in self.protos]
        load = [0.0] * n
        self._lane_of = [0] * len(self.protos)
        self._order = sorted(range(len(self.protos)), key=lambda j: -cost[j])  # capture order: largest first
        for i in self._order:
            ln = min(range(n), key=lambda k: load[k])
            self._lane_of[i] = ln
            load[ln] += cost[i]
        self._streams = [torch.cuda.Stream(self.device) for _ in range(n)]
        self.graph = None

    def _branch(self, i: int) -> None:
        """The reconstruction of protocol ``i`` on the current stream."""
        p = self.protos[i]
        x = self._dev_in[i]
        x[0].copy_(self.host_in[i], non_blocking=True)
        sparse = p.interp.interpolate(x)
        if p.subspace:
            AHb = p.op.adjoint(sparse.reshape(1, p.C, *p.natural_shape))
        else:
            AHb = p.op.adjoint(sparse * p.pre_w)
        cg = self._cg[i]
        cg.load(AHb)
        for _ in range(p.max_iter):
            cg.step()
        self.host_out[i].copy_(cg.x[0], non_blocking=True)

    def _all_branches(self) -> None:
        main = torch.cuda.current_stream(self.device)
        for s in self._streams:
            s.wait_stream(main)
        for i in self._order:
            with torch.cuda.stream(self._streams[self._lane_of[i]]):
                self._branch(i)
        for s in self._streams:
            main.wait_stream(s)

    def capture(self) -> None:
        """Run every branch once (cuFFT plans, PSFs and workspaces exist
        before the capture), then record the whole batch as one graph."""
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            self._all_branches()
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        g = torch.cuda.CUDAGraph()
        gc_on = gc.isenabled()
        gc.disable()  # no collection (and no CUDA frees it may trigger) while capturing
        try:
            with torch.cuda.graph(g):
                self._all_branches()
        finally:
            if gc_on:
                gc.enable()
        self.graph = g
        self._bound = ([id(t) for t in self.host_in], [id(t) for t in self.host_out])

    def run(self, inputs=None, sync: bool = True) -> list:
        """Reconstruct the batch.  ``inputs`` (optional): one ``(C, *spatial)``
        complex64 tensor per protocol, copied into :attr:`host_in` first."""
        if inputs is not None:
            if len(inputs) != len(self.protos):
                raise ValueError(f"{len(inputs)} inputs for {len(self.protos)} protocols")
            for dst, src in zip(self.host_in, inputs):
                dst.copy_(torch.as_tensor(src))
        if self.graph is None:
            self.capture()
        elif self._bound != ([id(t) for t in self.host_in], [id(t) for t in self.host_out]):
            raise RuntimeError("UnevenBatch: host_in / host_out were replaced after the graph was captured; "
                               "copy into the captured tensors instead")
        self.graph.replay()
        if sync:
            torch.cuda.current_stream(self.device).synchronize()
        return self.host_out
