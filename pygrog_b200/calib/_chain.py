"""The eigen-factored shift chain alone, in its two tensor-core forms.

``y = W3 Dx[k] W2 Dy[j] W1 Dz[i] W0 x`` per replica is the table product of
the reference (``calib/_grappa.py:62-72, 184-208``: every per-axis operator is
``expm(d logm G)``) in the form the tensor-core gridders run it.  This module
calls ``pgb_shift_chain`` (``csrc/shift_chain.cu``), which runs only the chain
(no staging, row sums or brick tiles) with ``mma.sync`` (``variant="mma"``) or
with ``tcgen05.mma`` and the accumulator in tensor memory
(``variant="tcgen05"``), so that the two MMA flavours can be measured on the
same work.  Used by ``bench.py --chain`` and ``tests/test_gpu_chain.py``.
"""

from __future__ import annotations

import numpy as np
import torch

from .. import _lib
from ._tc import realify

STEPS = 11  # shift steps per axis (precision 1)
VARIANTS = {"mma": 0, "tcgen05": 1}


def chain_operands(W: np.ndarray, phases: np.ndarray, device) -> tuple[torch.Tensor, torch.Tensor]:
    """Complex ``W (4, C, C)`` and ``phases (3, 11, C)`` -> the kernel's realified
    ``(4, 2C, 2C)`` float32 matrices ([stage][output][input]) and complex64 phases."""
    C = int(W.shape[-1])
    Wr = np.stack([realify(W[s], C).T for s in range(4)])  # realify gives x B = M x; the kernel wants M
    ph = np.ascontiguousarray(phases, dtype=np.complex64)
    return (torch.from_numpy(Wr.astype(np.float32)).to(device).contiguous(),
            torch.view_as_real(torch.from_numpy(ph)).to(device).contiguous())


def pack_shift_indices(ijk: torch.Tensor) -> torch.Tensor:
    """``(3, R)`` per-axis shift indices (each < 11) -> int32 ``i | j << 8 | k << 16``."""
    t = ijk.to(torch.int32)
    return (t[0] | (t[1] << 8) | (t[2] << 16)).contiguous()


def shift_chain(x: torch.Tensor, idx: torch.Tensor, W: torch.Tensor, ph: torch.Tensor, out: torch.Tensor,
                rep: int = 1, variant: str = "tcgen05", timeouts: torch.Tensor | None = None) -> torch.Tensor:
    """``out (2C, R) = chain^rep (x (2C, R))`` on the device, asynchronously on the
    current stream.  ``timeouts``: int32 device counter for the tcgen05 form
    (allocated when omitted; read it with :func:`check_timeouts`)."""
    C = int(x.shape[0]) // 2
    R = int(x.shape[1])
    for t in (x, idx, W, ph, out):
        if not t.is_cuda or not t.is_contiguous():
            raise ValueError("shift_chain: every tensor must be a contiguous CUDA tensor")
    if timeouts is None:
        timeouts = torch.zeros(1, dtype=torch.int32, device=x.device)
    _lib.call("pgb_shift_chain", x.data_ptr(), idx.data_ptr(), W.data_ptr(), ph.data_ptr(), out.data_ptr(), R, C,
              int(rep), VARIANTS[variant], timeouts.data_ptr(), _lib.stream_ptr(x.device))
    return timeouts


def check_timeouts(timeouts: torch.Tensor) -> None:
    """Raise ``RuntimeError`` if a tcgen05 chain launch gave up a wait (synchronises)."""
    n = int(timeouts.item())
    if n:
        raise RuntimeError(f"shift_chain: {n} CTA(s) gave up waiting for their tensor-core MMAs; "
                           "the result is incomplete")
