"""GPU parity of the seven native functions (reference tests + golden fixtures).

Mirrors tests/test_sparse_fft.py:45-106, tests/test_fast_binning.py and
tests/test_toeplitz_kernels.py of the reference, running through the C ABI.
"""

import numpy as np
import pytest
import torch

from conftest import golden, rel_l2
from pygrog_b200 import _ext

pytestmark = pytest.mark.gpu


def _sorted(n, G, dev, seed=0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    idx = torch.randint(0, G, (n,), generator=g).sort().values.to(dev)
    w = torch.rand(n, generator=g).to(dev)
    d = torch.randn(n, dtype=torch.complex64, generator=g).to(dev)
    return idx, w, d


def test_scatter_accumulates(cuda):
    grid = torch.zeros(8, dtype=torch.complex64, device=cuda)
    _ext.scatter_add(grid, torch.ones(3, dtype=torch.complex64, device=cuda),
                     torch.tensor([0, 0, 4], device=cuda), torch.ones(3, device=cuda))
    assert grid[0].real.item() == pytest.approx(2.0)
    assert grid[4].real.item() == pytest.approx(1.0)
    assert grid[1].real.item() == 0.0


def test_gather_selects_and_weights(cuda):
    grid = torch.arange(8).to(torch.complex64).to(cuda)
    out = _ext.gather(grid, torch.tensor([0, 3, 7], device=cuda), torch.tensor([2.0, 0.5, 3.0], device=cuda))
    torch.testing.assert_close(out.cpu(), torch.tensor([0.0, 1.5, 21.0], dtype=torch.complex64))


@pytest.mark.parametrize("n,G", [(512, 64), (100000, 4096), (4096, 1024)])
def test_scatter_matches_torch(cuda, n, G):
    idx, w, d = _sorted(n, G, cuda, seed=n)
    grid = torch.ones(G, dtype=torch.complex64, device=cuda)
    ref = grid.clone()
    _ext.scatter_add(grid, d, idx, w)
    ref.index_add_(0, idx, d * w.to(torch.complex64))
    torch.testing.assert_close(grid, ref, rtol=1e-4, atol=1e-4)


def test_scatter_unsorted_and_out_of_range(cuda):
    g = torch.Generator().manual_seed(5)
    G = 50
    idx = torch.randint(-10, G + 10, (3000,), generator=g)
    w = torch.rand(3000, generator=g)
    d = torch.randn(3000, dtype=torch.complex64, generator=g)
    ref = torch.zeros(G, dtype=torch.complex64)
    ok = (idx >= 0) & (idx < G)
    ref.index_add_(0, idx[ok], (d * w)[ok])
    grid = torch.zeros(G, dtype=torch.complex64, device=cuda)
    _ext.scatter_add(grid, d.to(cuda), idx.to(cuda), w.to(cuda))
    torch.testing.assert_close(grid.cpu(), ref, rtol=1e-4, atol=1e-4)
    out = _ext.gather(torch.arange(G).to(torch.complex64).to(cuda), idx.to(cuda), w.to(cuda)).cpu()
    exp = torch.where(ok, w * idx.clamp(0, G - 1).float(), torch.zeros_like(w)).to(torch.complex64)
    torch.testing.assert_close(out, exp)


def test_scatter_empty_single_and_all_same_bin(cuda):
    grid = torch.zeros(16, dtype=torch.complex64, device=cuda)
    e = torch.empty(0, device=cuda)
    _ext.scatter_add(grid, e.to(torch.complex64), e.long(), e)
    assert grid.abs().max().item() == 0.0
    assert _ext.gather(grid, e.long(), e).numel() == 0
    g2 = torch.zeros(10, dtype=torch.complex64, device=cuda)
    _ext.scatter_add(g2, torch.tensor([1 + 2j], dtype=torch.complex64, device=cuda),
                     torch.tensor([3], device=cuda), torch.tensor([0.5], device=cuda))
    assert abs(g2[3].item() - (0.5 + 1j)) < 1e-6 and g2.abs().sum().item() == pytest.approx(abs(0.5 + 1j))
    n = 1 << 16
    g3 = torch.zeros(16, dtype=torch.complex64, device=cuda)
    _ext.scatter_add(g3, torch.ones(n, dtype=torch.complex64, device=cuda),
                     torch.full((n,), 7, device=cuda), torch.ones(n, device=cuda))
    assert abs(g3[7].real.item() - n) < 1e-3 * n and g3[7].imag.abs().item() < 1e-5


def test_scatter_binned_matches_simple(cuda):
    G, n, bs = 1024, 4096, 256
    idx, w, d = _sorted(n, G, cuda, seed=9)
    a = torch.zeros(G, dtype=torch.complex64, device=cuda)
    _ext.scatter_add(a, d, idx, w)
    edges = torch.arange(G // bs + 1, device=cuda) * bs
    starts = torch.searchsorted(idx, edges)
    b = torch.zeros(G, dtype=torch.complex64, device=cuda)
    _ext.scatter_add_binned(b, d, idx, w, starts, bs)
    torch.testing.assert_close(a, b, rtol=1e-4, atol=1e-4)


def test_round_trip_identity(cuda):
    G = 32
    idx = torch.arange(G, device=cuda)
    w = torch.ones(G, device=cuda)
    d = torch.randn(G, dtype=torch.complex64, device=cuda)
    grid = torch.zeros(G, dtype=torch.complex64, device=cuda)
    _ext.scatter_add(grid, d, idx, w)
    torch.testing.assert_close(_ext.gather(grid, idx, w), d)


def test_golden_l0(cuda):
    z = golden("l0_ops.npz")
    t = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(cuda)  # noqa: E731
    out = _ext.grog_interpolate(t(z["gi_data"]), t(z["gi_idx"]), t(z["gi_kernel"]))
    assert rel_l2(out.cpu().numpy(), z["ref_gi"]) < 1e-6
    out = _ext.grog_interpolate(t(z["gi_data"]).to(torch.complex128), t(z["gi_idx"]),
                                t(z["gi_kernel"]).to(torch.complex128))
    assert rel_l2(out.cpu().numpy(), z["ref_gi128"]) < 1e-12
    g = t(z["sa_grid0"]).clone()
    _ext.scatter_add(g, t(z["sa_data"]), t(z["sa_idx"]), t(z["sa_w"]))
    assert rel_l2(g.cpu().numpy(), z["ref_sa"]) < 1e-6
    assert rel_l2(_ext.gather(t(z["ga_grid"]), t(z["sa_idx"]), t(z["sa_w"])).cpu().numpy(), z["ref_ga"]) < 1e-7
    G = z["ref_ps"].size
    ps = torch.zeros(G, device=cuda)
    _ext.psf_scatter_scalar(ps, t(z["sa_idx"]), t(z["ps_wsq"]))
    np.testing.assert_allclose(ps.cpu().numpy(), z["ref_ps"], rtol=1e-6, atol=1e-5)
    M = z["po_basis"].shape[1]
    po = torch.zeros(G, M, M, dtype=torch.complex64, device=cuda)
    _ext.psf_scatter_outer(po, t(z["sa_idx"]), t(z["ps_wsq"]), t(z["po_basis"]))
    assert rel_l2(po.cpu().numpy(), z["ref_po"]) < 1e-6
    K = z["pb_basis"].shape[0]
    pb = torch.zeros(G, K, K, dtype=torch.complex64, device=cuda)
    _ext.psf_scatter_outer_basis(pb, t(z["sa_idx"]), t(z["ps_wsq"]), t(z["pb_basis"]), t(z["pb_tix"]))
    assert rel_l2(pb.cpu().numpy(), z["ref_pb"]) < 1e-6


@pytest.mark.parametrize("C", [1, 3, 8, 12, 16, 31, 32, 40])
def test_grog_interpolate_vs_matmul(cuda, C):
    g = torch.Generator().manual_seed(C)
    N, B, K = 777, 3, 13
    d = torch.randn(N, B, C, dtype=torch.complex64, generator=g)
    idx = torch.randint(0, K, (N,), generator=g)
    ker = torch.randn(K, C, C, dtype=torch.complex64, generator=g)
    ref = torch.einsum("nij,nbj->nbi", ker[idx], d)
    out = _ext.grog_interpolate(d.to(cuda), idx.to(cuda), ker.to(cuda)).cpu()
    assert rel_l2(out.numpy(), ref.numpy()) < 1e-6


def test_psf_kernels_hermitian_and_fp64(cuda):
    g = torch.Generator().manual_seed(8)
    G, K, T, n = 16, 4, 12, 80
    idx = torch.randint(0, G, (n,), generator=g).sort().values.to(cuda)
    wsq = (torch.rand(n, generator=g) + 0.1).to(cuda)
    basis = torch.randn(K, T, dtype=torch.complex64, generator=g).to(cuda)
    tix = torch.randint(0, T, (n,), generator=g).to(cuda)
    psf = torch.zeros(G, K, K, dtype=torch.complex64, device=cuda)
    _ext.psf_scatter_outer_basis(psf, idx, wsq, basis, tix)
    torch.testing.assert_close(psf, psf.conj().transpose(-2, -1), rtol=1e-5, atol=1e-5)
    p64 = torch.zeros(G, dtype=torch.float64, device=cuda)
    w64 = wsq.double()
    _ext.psf_scatter_scalar(p64, idx, w64)
    ref = torch.zeros(G, dtype=torch.float64, device=cuda).index_add_(0, idx, w64)
    torch.testing.assert_close(p64, ref, rtol=1e-12, atol=1e-12)
