"""Operands of the tensor-core gridder (``csrc/grog_tc.cu``).

With the per-axis eigendecompositions of :func:`._grappa.eigen_factors`, the
table operator of a replica with axis indices ``(i, j, k)`` is

    T x = V2 D2[k] V2^-1 V1 D1[j] V1^-1 V0 D0[i] V0^-1 x        (3-D)

i.e. dense matrices ``M0 = V0^-1``, ``M_s = V_s^-1 V_{s-1}``, ``M_ndim =
V_{ndim-1}`` applied to every replica, and diagonal phases ``D_s[step] =
exp(delta_step * l_s)`` between them.  The adjoint applies ``M_ndim^H, ...,
M0^H`` with conjugated phases in reverse axis order.

Each complex ``C x C`` matrix is realified with (re, im) interleaved,
``B[2c + a, 2r + b]``, so that ``y = x B`` on interleaved rows is ``y = M x``,
padded to ``CP = 4 ceil(C / 4)`` coils and split into bf16 heads and tails
(``B = hi + lo``).  The words are laid out per lane in the register order of
the kernel's mma.sync B fragments: for every n-tile ``nt`` (8 real output
columns), each k16 chunk contributes two words (rows ``2t, 2t+1`` and
``2t+8, 2t+9`` of column ``8 nt + g``, ``g = lane / 4``, ``t = lane % 4``)
and a trailing k8 chunk one word; a word holds the lower-row element in its
low 16 bits.
"""

from __future__ import annotations

import numpy as np
import torch


def padded_coils(C: int) -> int:
    return 4 * ((int(C) + 3) // 4)


def realify(M: np.ndarray, CP: int) -> np.ndarray:
    """Complex ``(C, C)`` -> real ``(2 CP, 2 CP)`` with ``(x B)`` = ``M x`` on interleaved rows."""
    C = M.shape[0]
    W = np.zeros((CP, CP), dtype=np.complex128)
    W[:C, :C] = M
    WT = W.T
    B = np.zeros((2 * CP, 2 * CP), dtype=np.float64)
    B[0::2, 0::2] = WT.real
    B[1::2, 0::2] = -WT.imag
    B[0::2, 1::2] = WT.imag
    B[1::2, 1::2] = WT.real
    return B


def _bf16_bits(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Round-to-nearest bf16 head and tail of ``x`` as uint16 bit patterns."""
    t = torch.from_numpy(np.ascontiguousarray(x, dtype=np.float32))
    hi = t.to(torch.bfloat16)
    lo = (t - hi.to(torch.float32)).to(torch.bfloat16)
    as_u16 = lambda h: h.view(torch.int16).numpy().astype(np.int64) & 0xFFFF  # noqa: E731
    return as_u16(hi), as_u16(lo)


def fragment_words(B: np.ndarray, CP: int) -> np.ndarray:
    """``(2, NFR, 32)`` uint32 head / tail fragment words of one realified matrix."""
    NT = CP // 4
    K16, K8 = NT // 2, NT % 2
    lane = np.arange(32)
    g, t = lane // 4, lane % 4
    rows, cols = [], []  # (NFR, 32) row index of the low element, column
    for nt in range(NT):
        for kc in range(K16):
            for half in (0, 8):
                rows.append(16 * kc + half + 2 * t)
                cols.append(8 * nt + g)
        if K8:
            rows.append(16 * K16 + 2 * t)
            cols.append(8 * nt + g)
    rows = np.stack(rows)
    cols = np.stack(cols)
    lo_el = B[rows, cols]
    hi_el = B[rows + 1, cols]
    out = np.zeros((2,) + rows.shape, dtype=np.uint32)
    for part in range(2):
        a = _bf16_bits(lo_el)[part]
        b = _bf16_bits(hi_el)[part]
        out[part] = (a | (b << 16)).astype(np.uint32)
    return out


def tc_operands(ef, C: int, device) -> dict:
    """Device operands ``{"fwd": (wfrag, dtab), "adj": (wfrag, dtab), "CP", "ndim", "nsteps"}``.

    ``wfrag``: int32 ``(ndim + 1, 2, NFR, 32)``; ``dtab``: complex64
    ``(ndim, nsteps, CP)`` phases in the order the kernel applies them.
    """
    CP = padded_coils(C)
    V = [np.asarray(v.numpy(), dtype=np.complex128) for v, _ in ef.axes]
    lam = [np.asarray(l.numpy(), dtype=np.complex128) for _, l in ef.axes]
    Vi = [np.linalg.inv(v) for v in V]
    nd = ef.ndim
    mats = [Vi[0]] + [Vi[s] @ V[s - 1] for s in range(1, nd)] + [V[nd - 1]]
    d = ef.deltas.numpy().astype(np.float32).astype(np.float64)
    D = []
    for s in range(nd):
        ph = np.zeros((ef.nsteps, CP), dtype=np.complex128)
        ph[:, :C] = np.exp(d[:, None] * lam[s][None, :])
        D.append(ph)
    adj_mats = [m.conj().T for m in reversed(mats)]
    adj_D = [np.conj(p) for p in reversed(D)]

    def pack(ms, ds):
        w = np.stack([fragment_words(realify(m, CP), CP) for m in ms])  # (nd + 1, 2, NFR, 32)
        wt = torch.from_numpy(w.view(np.int32).copy()).to(device)
        dt = torch.from_numpy(np.stack(ds).astype(np.complex64)).to(device).contiguous()
        return wt.contiguous(), dt

    return {"fwd": pack(mats, D), "adj": pack(adj_mats, adj_D), "CP": CP, "ndim": nd, "nsteps": ef.nsteps,
            "mats": mats, "phases": D}
