"""GPU parity of SparseFFT / MaskedFFT / Toeplitz normal / CG / LSMR.

Golden outputs come from the reference operators on the same GROG plans
(tests/golden/ops_*.npz).  Tolerances: 1e-5 relative L2 for single
operator applications (FP32), 1e-4 for iterative solves (the reference
accumulates its CG / LSMR inner products in FP32, these in FP64).
Mirrors the reference's adjointness, shape and batch-helper tests
(tests/test_sparse_fft.py:108-278, tests/test_toeplitz.py:128-150,
tests/test_masked_fft.py).
"""

import numpy as np
import pytest
import torch

from conftest import golden, parse_meta, rel_l2
from pygrog_b200.calib import GrogInterpolator
from pygrog_b200.operator import MaskedFFT, SparseFFT

pytestmark = pytest.mark.gpu


def _plan(name, cuda):
    z = golden(f"ops_{name}.npz")
    _, shape, img, osf, C = parse_meta(z["meta"])
    g = GrogInterpolator(shape=shape, coords=z["in_coords"], oversamp=osf, kernel_width=2, image_shape=img,
                         device=cuda)
    g.calc_interp_table(z["in_calib"], lamda=0.01, precision=1)
    return z, g, C


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_sparse_fft_matches_reference(cuda, name):
    z, g, C = _plan(name, cuda)
    sm = torch.from_numpy(z["in_smaps"])
    op = SparseFFT(plan=g.plan, smaps=sm, toeplitz=True)
    b = torch.from_numpy(z["in_b"])
    assert rel_l2(op.adjoint(b).numpy(), z["ref_adjoint"]) < 1e-5
    x = torch.from_numpy(z["in_x"])
    assert rel_l2(op.forward(x).reshape(C, -1).numpy(), z["ref_forward"]) < 1e-5
    opc = SparseFFT(plan=g.plan, toeplitz=False)
    assert rel_l2(opc.adjoint(b).numpy(), z["ref_adjoint_nosmaps"]) < 1e-5
    xc = torch.from_numpy(z["in_xc"])
    assert rel_l2(opc.forward(xc).reshape(C, -1).numpy(), z["ref_forward_nosmaps"]) < 1e-5
    # numpy in -> numpy out, like the reference's with_torch
    out = op.adjoint(z["in_b"])
    assert isinstance(out, np.ndarray)


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_toeplitz_and_nested_normal_match_reference(cuda, name):
    z, g, C = _plan(name, cuda)
    sm = torch.from_numpy(z["in_smaps"])
    x = torch.from_numpy(z["in_x"])
    op_t = SparseFFT(plan=g.plan, smaps=sm, toeplitz=True)
    op_n = SparseFFT(plan=g.plan, smaps=sm, toeplitz=False)
    yt = op_t.normal(x).numpy()
    yn = op_n.normal(x).numpy()
    assert rel_l2(yt, z["ref_normal_toep"]) < 1e-5
    assert rel_l2(yn, z["ref_normal_notoep"]) < 1e-5
    np.testing.assert_allclose(op_t._toep_op.psf.cpu().numpy(), z["ref_psf"], rtol=1e-5, atol=1e-6)
    # Toeplitz == nested (reference test_toeplitz.py:128-150 bar)
    assert np.abs(yt - yn).max() / np.abs(yn).max() < 1e-4


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_cg_and_lsmr_match_reference(cuda, name):
    z, g, C = _plan(name, cuda)
    sm = torch.from_numpy(z["in_smaps"])
    op = SparseFFT(plan=g.plan, smaps=sm, toeplitz=True)
    bn = torch.from_numpy(z["in_b"]).reshape(C, *op.natural_shape)
    x = op.solve(bn, method="cg", max_iter=8, damp=1e-3, tol=0.0)
    assert rel_l2(x.numpy(), z["ref_cg"]) < 1e-4
    # graph replay and the host loop agree
    x2 = op.solve(bn, method="cg", max_iter=8, damp=1e-3, tol=0.0, use_graph=False)
    assert rel_l2(x2.numpy(), x.numpy()) < 1e-6
    opn = SparseFFT(plan=g.plan, smaps=sm, toeplitz=False)
    xl = opn.solve(bn, method="lsmr", max_iter=8, damp=1e-3)
    assert rel_l2(xl.numpy(), z["ref_lsmr"]) < 1e-4
    # default method: cg when toeplitz (reference _mixin.py:131-132)
    assert op.toeplitz is True and opn.toeplitz is False


def test_cg_with_a_preconditioner_object(cuda):
    """``preconditioner=`` takes any object with ``.apply(r)`` (``_solvers.py:115, 133``)
    and runs the host-driven loop; a scalar preconditioner leaves the CG
    iterates unchanged, so the result equals the unpreconditioned solve and
    the reference's."""

    class Scaled:
        calls = 0

        def apply(self, r):
            Scaled.calls += 1
            return 0.37 * r

    z, g, C = _plan("op2d", cuda)
    op = SparseFFT(plan=g.plan, smaps=torch.from_numpy(z["in_smaps"]), toeplitz=True)
    bn = torch.from_numpy(z["in_b"]).reshape(C, *op.natural_shape)
    x = op.solve(bn, method="cg", max_iter=8, damp=1e-3, tol=0.0, preconditioner=Scaled())
    assert Scaled.calls == 9  # once before the loop and once per iteration
    assert rel_l2(x.numpy(), z["ref_cg"]) < 1e-4
    x0 = op.solve(bn, method="cg", max_iter=8, damp=1e-3, tol=0.0)
    assert rel_l2(x.numpy(), x0.numpy()) < 1e-5


def test_device_lsmr_graph_eager_and_early_stop(cuda):
    """Device LSMR: the graph-replayed iteration and the eager loop agree; a
    stopping tolerance freezes the state at the iteration where the
    reference's loop breaks (same result as that many iterations run alone),
    and the eager loop's callback sees the reference's relative residuals."""
    from pygrog_b200._solve import lsmr

    z, g, C = _plan("op2d", cuda)
    sm = torch.from_numpy(z["in_smaps"])
    opn = SparseFFT(plan=g.plan, smaps=sm, toeplitz=False)
    bn = torch.from_numpy(z["in_b"]).reshape(C, *opn.natural_shape).to(cuda)
    xg = lsmr(opn, bn, damp=1e-3, max_iter=12)
    xe = lsmr(opn, bn, damp=1e-3, max_iter=12, use_graph=False)
    assert rel_l2(xe.cpu().numpy(), xg.cpu().numpy()) < 1e-6
    seen = []
    lsmr(opn, bn, damp=1e-3, max_iter=40, callback=lambda k, x, r: seen.append(r))
    assert len(seen) > 6
    tol = seen[5] * 1.0000001  # the test fires at iteration 5 at the latest (0-based)
    k_stop = next(k for k, r in enumerate(seen) if r < tol)
    x_tol = lsmr(opn, bn, damp=1e-3, max_iter=40, atol=tol / 2, btol=tol / 2)
    x_k = lsmr(opn, bn, damp=1e-3, max_iter=k_stop + 1)
    assert rel_l2(x_tol.cpu().numpy(), x_k.cpu().numpy()) < 1e-6


def test_cg_early_exit_matches_break(cuda):
    z, g, C = _plan("op2d", cuda)
    sm = torch.from_numpy(z["in_smaps"])
    op = SparseFFT(plan=g.plan, smaps=sm, toeplitz=True)
    bn = torch.from_numpy(z["in_b"]).reshape(C, *op.natural_shape)
    seen = []
    x_cb = op.solve(bn, method="cg", max_iter=50, damp=1e-3, tol=1e-2, callback=lambda k, x, r: seen.append(r))
    assert seen[-1] < 1e-2 and all(r >= 1e-2 for r in seen[:-1])
    x_gr = op.solve(bn, method="cg", max_iter=50, damp=1e-3, tol=1e-2)
    assert rel_l2(x_gr.numpy(), x_cb.numpy()) < 1e-6


def test_repeated_solves_replay_the_cached_graph(cuda):
    """Solves on one operator reuse its captured CG iteration: each result
    equals a fresh host-loop solve, earlier results are not overwritten, and
    a warm start (x0) and another damp take their own paths."""
    z, g, C = _plan("op2d", cuda)
    sm = torch.from_numpy(z["in_smaps"])
    op = SparseFFT(plan=g.plan, smaps=sm, toeplitz=True)
    bn = torch.from_numpy(z["in_b"]).reshape(C, *op.natural_shape)
    x1 = op.solve(bn, method="cg", max_iter=8, damp=1e-3, tol=0.0)
    b2 = bn * 0.5 + 0.25j * torch.roll(bn, 3, dims=-1)
    x2 = op.solve(b2, method="cg", max_iter=8, damp=1e-3, tol=0.0)
    assert len(op._cg_graphs) == 1
    assert rel_l2(x1.numpy(), z["ref_cg"]) < 1e-4  # x1 kept its values
    ref2 = op.solve(b2, method="cg", max_iter=8, damp=1e-3, tol=0.0, use_graph=False)
    assert rel_l2(x2.numpy(), ref2.numpy()) < 1e-6
    x3 = op.solve(b2, method="cg", max_iter=8, damp=1e-2, tol=0.0)
    assert len(op._cg_graphs) == 2
    assert rel_l2(x3.numpy(), op.solve(b2, method="cg", max_iter=8, damp=1e-2, tol=0.0, use_graph=False).numpy()) < 1e-6
    x4 = op.solve(b2, method="cg", max_iter=8, damp=1e-3, tol=0.0, x0=x1)
    ref4 = op.solve(b2, method="cg", max_iter=8, damp=1e-3, tol=0.0, x0=x1, use_graph=False)
    assert rel_l2(x4.numpy(), ref4.numpy()) < 1e-6


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_masked_fft_matches_reference(cuda, name):
    z, g, C = _plan(name, cuda)
    sm = torch.from_numpy(z["in_smaps"])
    kg, mp = g.interpolate(torch.from_numpy(z["in_data"]), grid=True)
    mop = MaskedFFT(plan=mp, smaps=sm, toeplitz=True)
    assert rel_l2(mop.adjoint(kg).cpu().numpy(), z["ref_masked_adjoint"]) < 1e-5
    x = torch.from_numpy(z["in_x"])
    assert rel_l2(mop.forward(x).numpy(), z["ref_masked_forward"]) < 1e-5
    assert rel_l2(mop.normal(x).numpy(), z["ref_masked_normal"]) < 1e-5
    xs = mop.solve(kg.cpu(), method="cg", max_iter=8, damp=1e-3, tol=0.0)
    assert rel_l2(xs.numpy(), z["ref_masked_cg"]) < 1e-4


def _cdot(a, b):
    return torch.vdot(a.flatten().to(torch.complex128), b.flatten().to(torch.complex128))


def _rand_op(grid, img, n, smaps=None, seed=0, weighted=False):
    rng = np.random.default_rng(seed)
    G = int(np.prod(grid))
    idx = rng.integers(0, G, size=n)
    w = rng.uniform(0.5, 2.0, size=n).astype(np.float32) if weighted else np.ones(n, np.float32)
    return SparseFFT(grid, img, idx, w, smaps=smaps)


@pytest.mark.parametrize("grid,img,C,with_smaps,weighted", [
    ((32, 32), (24, 24), 4, False, False),
    ((32, 32), (24, 24), 4, True, False),
    ((16, 16, 16), (12, 12, 12), 2, False, False),
    ((32, 32), (24, 24), 3, False, True),
    ((33, 31), (20, 19), 2, True, True),   # odd extents exercise the shift remap
])
def test_adjointness(cuda, grid, img, C, with_smaps, weighted):
    torch.manual_seed(1)
    sm = torch.randn(C, *img, dtype=torch.complex64) if with_smaps else None
    op = _rand_op(grid, img, 300, smaps=sm, seed=2, weighted=weighted)
    x = torch.randn(C, 300, dtype=torch.complex64)
    y = torch.randn(*((img) if with_smaps else (C, *img)), dtype=torch.complex64)
    lhs = _cdot(op.adjoint(x), y)
    rhs = _cdot(x, op.forward(y))
    assert abs(lhs - rhs) / abs(lhs) < 1e-4


def test_shapes_and_call_flag(cuda):
    op = _rand_op((32, 32), (24, 24), 256)
    ksp = torch.randn(4, 256, dtype=torch.complex64, device=cuda)
    img = torch.randn(4, 24, 24, dtype=torch.complex64, device=cuda)
    assert op.adjoint(ksp).shape == (4, 24, 24) and op.adjoint(ksp).device.type == "cuda"
    assert op.forward(img).shape == (4, 256)
    torch.testing.assert_close(op(img), op.forward(img))
    torch.testing.assert_close(op(ksp, adjoint=True), op.adjoint(ksp))
    op3 = _rand_op((16, 16, 16), (12, 12, 12), 128)
    assert op3.adjoint(torch.randn(2, 128, dtype=torch.complex64)).shape == (2, 12, 12, 12)


def test_batch_helpers_match_per_row(cuda):
    from pygrog_b200 import _ext

    op = _rand_op((32, 32), (24, 24), 256, seed=4)
    B = 6
    ksp = torch.randn(B, 256, dtype=torch.complex64, device=cuda)
    out = op._scatter_ifft_crop_batch(ksp)
    sp, idx, sw = op.sort_perm.to(cuda), op.indices.to(cuda), op.sqrt_weights.to(cuda)
    ref = []
    for b in range(B):
        grid = torch.zeros(op.grid_size, dtype=torch.complex64, device=cuda)
        _ext.scatter_add(grid, ksp[b][sp].contiguous(), idx, sw)
        full = torch.fft.fftshift(torch.fft.ifftn(torch.fft.ifftshift(grid.reshape(op.grid_shape)), norm="ortho"))
        ref.append(full[op._pad_slices])
    torch.testing.assert_close(out, torch.stack(ref), rtol=1e-5, atol=1e-5)
    imgs = torch.randn(B, 24, 24, dtype=torch.complex64, device=cuda)
    outk = op._fft_pad_gather_batch(imgs)
    lhs = _cdot(op._scatter_ifft_crop_batch(ksp), imgs)
    rhs = _cdot(ksp, outk)
    assert abs(lhs - rhs) / abs(lhs) < 1e-4


def test_batched_and_stacked_layouts(cuda):
    """(*B) batches and stacked plans equal per-element loops (reference test_batch_stack.py)."""
    from pygrog_b200.workloads import radial2d

    rng = np.random.default_rng(0)
    co = np.stack([radial2d(6, 32, 8.0), radial2d(6, 32, 8.0)[:, ::-1]])  # (S=2, 6, 32, 2)
    calib = (rng.standard_normal((3, 8, 8)) + 1j * rng.standard_normal((3, 8, 8))).astype(np.complex64)
    g = GrogInterpolator(shape=(16, 16), coords=co, oversamp=2.0, kernel_width=2, device=cuda)
    g.calc_interp_table(calib)
    assert g.plan.stack_shape == (2,)
    data = (rng.standard_normal((4, 2, 3, 6, 32)) + 1j * rng.standard_normal((4, 2, 3, 6, 32))).astype(np.complex64)
    sp = g.interpolate(data)
    assert sp.shape == (4, 2, 3, g.plan.n_samples)
    op = SparseFFT(plan=g.plan)
    imgs = op.adjoint(torch.from_numpy(sp))
    assert imgs.shape == (4, 2, 3, 16, 16)
    for s in range(2):
        gs = GrogInterpolator(shape=(16, 16), coords=co[s], oversamp=2.0, kernel_width=2, device=cuda)
        gs.calc_interp_table(calib)
        sps = gs.interpolate(data[:, s])
        assert rel_l2(sp[:, s], sps) < 1e-6
        ims = SparseFFT(plan=gs.plan).adjoint(torch.from_numpy(sps))
        assert rel_l2(imgs[:, s].numpy(), ims.numpy()) < 1e-5


def test_ret_image_matches_sparsefft_rss(cuda):
    """interpolate(ret_image=True) == SparseFFT.adjoint(pre_weights * sparse) + RSS
    (reference tests/test_grog_interpolator.py:42-88), and against the golden image."""
    z = golden("plan_p2d_circle_osf2.npz")
    name, shape, osf, kwd, ks, prec, C = parse_meta(z["meta"])
    g = GrogInterpolator(shape=shape, coords=z["in_coords"], oversamp=osf, kernel_width=kwd, kernel_shape=ks,
                         device=cuda)
    g.calc_interp_table(z["in_calib"], lamda=0.01, precision=prec)
    image = g.interpolate(z["in_data"], ret_image=True)
    assert rel_l2(image, z["ref_image"]) < 1e-5
    sparse = torch.as_tensor(g.interpolate(z["in_data"]))
    op = SparseFFT(plan=g.plan)
    exp = op.adjoint(sparse * g.plan.pre_weights.cpu().unsqueeze(0)).abs().square().sum(0).sqrt()
    np.testing.assert_allclose(image, exp.numpy(), rtol=1e-5, atol=1e-5)
