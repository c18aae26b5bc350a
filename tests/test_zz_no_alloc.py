"""pgb_dot_f64_noalloc (static-scratch row inner products) against pgb_dot_f64.

Both are called through the C-ABI.  The two reduce in FP64 with the same
block partitioning per vector, so they agree to FP64 rounding; the test
allows 1e-12 relative.
"""

import ctypes

import pytest
import torch

import pygrog_b200
from pygrog_b200 import _lib

PGB_ERR_RANGE = 5
MAX_ROWS = 64


def _dot_existing(a, b, dev):
    """Per-row dot through pgb_dot_f64 mode 0 (caller-owned scratch)."""
    lib = pygrog_b200.load_library()
    scratch = torch.zeros((int(lib.pgb_reduce_scratch_bytes()) + 7) // 8, dtype=torch.float64, device=dev)
    scal = torch.zeros(8, dtype=torch.float64, device=dev)
    st = _lib.stream_ptr(dev)
    res = []
    for r in range(a.shape[0]):
        _lib.call("pgb_dot_f64", a[r].data_ptr(), None if b is None else b[r].data_ptr(), a.shape[1],
                  scratch.data_ptr(), scal.data_ptr(), 0, 0, st)
        res.append(scal[0].item())
    return torch.tensor(res, dtype=torch.float64)


def _dot_noalloc(a, b, out, dev):
    _lib.call("pgb_dot_f64_noalloc", a.data_ptr(), None if b is None else b.data_ptr(), a.shape[1], a.shape[0],
              out.data_ptr(), _lib.stream_ptr(dev))
    torch.cuda.synchronize(dev)
    return out.cpu()


def test_rows_above_maximum_are_rejected():
    lib = pygrog_b200.load_library()
    st = lib.pgb_dot_f64_noalloc(None, None, 10, MAX_ROWS + 1, None, None)
    assert st == PGB_ERR_RANGE
    assert b"exceeds the static scratch maximum" in lib.pgb_last_error()


@pytest.mark.gpu
def test_noalloc_matches_dot_f64_twice_in_a_row(cuda):
    g = torch.Generator(device="cpu").manual_seed(7)
    out = torch.empty(MAX_ROWS, dtype=torch.float64, device=cuda)
    for rows, n, with_b in [(5, 100_003, True), (5, 100_003, False), (MAX_ROWS, 4099, True), (1, 3, True)]:
        a = torch.randn(rows, n, dtype=torch.complex64, generator=g).to(cuda)
        b = torch.randn(rows, n, dtype=torch.complex64, generator=g).to(cuda) if with_b else None
        ref = _dot_existing(a, b, cuda)
        for _ in range(2):  # the second call reuses the counters the first one left
            got = _dot_noalloc(a, b, out[:rows], cuda)
            torch.testing.assert_close(got, ref, rtol=1e-12, atol=1e-9)
    # n = 0 gives zeros
    a = torch.empty(3, 0, dtype=torch.complex64, device=cuda)
    out.fill_(1.0)
    assert torch.all(_dot_noalloc(a, a, out[:3], cuda) == 0)


@pytest.mark.gpu
def test_noalloc_back_to_back_on_one_stream(cuda):
    """Several calls with different inputs queued on one stream with no host
    synchronisation between them, then one sync: each call's kernel must see
    the counters that its own clear left, so every output must still match
    pgb_dot_f64."""
    g = torch.Generator(device="cpu").manual_seed(11)
    cases = [(7, 50_001), (MAX_ROWS, 2_053), (3, 300_007), (MAX_ROWS, 17), (1, 1)]
    data = []
    for rows, n in cases:
        a = torch.randn(rows, n, dtype=torch.complex64, generator=g).to(cuda)
        b = torch.randn(rows, n, dtype=torch.complex64, generator=g).to(cuda)
        data.append((a, b, _dot_existing(a, b, cuda)))
    torch.cuda.synchronize(cuda)
    outs = [torch.full((a.shape[0],), float("nan"), dtype=torch.float64, device=cuda) for a, _, _ in data]
    stream = _lib.stream_ptr(cuda)
    for (a, b, _), out in zip(data, outs):
        _lib.call("pgb_dot_f64_noalloc", a.data_ptr(), b.data_ptr(), a.shape[1], a.shape[0], out.data_ptr(), stream)
    torch.cuda.synchronize(cuda)
    for (_, _, ref), out in zip(data, outs):
        torch.testing.assert_close(out.cpu(), ref, rtol=1e-12, atol=1e-9)
