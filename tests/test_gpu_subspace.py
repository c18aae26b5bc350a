"""GPU parity of the low-rank subspace operator against the reference fixture
``tests/golden/sub_sub2d.npz`` and ``sub_masked.npz`` (reference ``gadgets/_subspace.py`` and
``_toep/_sub_toep.py`` run on the same seeded inputs).  FP32 operator
outputs <= 1e-5 relative L2, CG <= 1e-4."""

import numpy as np
import pytest
import torch

from conftest import golden, parse_meta, rel_l2
from pygrog_b200.calib import GrogInterpolator
from pygrog_b200.operator import SparseFFT, with_subspace

pytestmark = pytest.mark.gpu


def _ops(cuda):
    z = golden("sub_sub2d.npz")
    _, shape, img, osf, C, K, T = parse_meta(z["meta"])
    g = GrogInterpolator(shape=shape, coords=z["in_coords"], oversamp=osf, kernel_width=2, image_shape=img,
                         device=cuda)
    g.calc_interp_table(z["in_calib"], lamda=0.01, precision=1)
    sm = torch.from_numpy(z["in_smaps"])
    basis = torch.from_numpy(z["in_basis"])
    sub_t = with_subspace(SparseFFT(plan=g.plan, smaps=sm, toeplitz=True), basis, encoding_axis=-3)
    sub_n = with_subspace(SparseFFT(plan=g.plan, smaps=sm, toeplitz=False), basis, encoding_axis=-3)
    return z, sub_t, sub_n


def test_subspace_operator_matches_reference(cuda):
    z, sub_t, sub_n = _ops(cuda)
    b = torch.from_numpy(z["in_b"])
    xk = torch.from_numpy(z["in_xk"])
    assert rel_l2(sub_t.adjoint(b).numpy(), z["ref_sub_adjoint"]) < 1e-5
    assert rel_l2(sub_t.forward(xk).numpy(), z["ref_sub_forward"]) < 1e-5
    assert rel_l2(sub_t.normal(xk).numpy(), z["ref_sub_normal_toep"]) < 1e-5
    assert rel_l2(sub_t._toep_op.psf.cpu().numpy(), z["ref_sub_psf"]) < 1e-5
    assert rel_l2(sub_n.normal(xk).numpy(), z["ref_sub_normal_notoep"]) < 1e-5
    x = sub_t.solve(b, method="cg", max_iter=6, damp=1e-3, tol=0.0)
    assert rel_l2(x.numpy(), z["ref_sub_cg"]) < 1e-4
    xn = sub_n.solve(b, method="cg", max_iter=6, damp=1e-3, tol=0.0)
    assert rel_l2(xn.numpy(), z["ref_sub_cg"]) < 1e-4


def test_subspace_adjointness_and_batches(cuda):
    z, sub_t, _ = _ops(cuda)
    g = torch.Generator().manual_seed(3)
    y = torch.randn(*z["in_b"].shape, dtype=torch.complex64, generator=g)
    x = torch.randn(*z["in_xk"].shape, dtype=torch.complex64, generator=g)
    lhs = torch.vdot(sub_t.adjoint(y).flatten().to(torch.complex128), x.flatten().to(torch.complex128))
    rhs = torch.vdot(y.flatten().to(torch.complex128), sub_t.forward(x).flatten().to(torch.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-4
    yb = torch.stack([y, 2 * y + 1j])
    xb = sub_t.adjoint(yb)
    assert xb.shape == (2, *z["in_xk"].shape)
    assert rel_l2(xb[1].numpy(), sub_t.adjoint(yb[1]).numpy()) < 1e-6
    fb = sub_t.forward(torch.stack([x, x * 0.5]))
    assert rel_l2(fb[1].numpy(), 0.5 * sub_t.forward(x).numpy()) < 1e-6
    nb = sub_t.normal(torch.stack([x, 3 * x]))
    assert rel_l2(nb[1].numpy(), 3 * sub_t.normal(x).numpy()) < 1e-5
    with pytest.raises(ValueError, match="does not match natural_shape"):
        with_subspace(sub_t._base, torch.zeros(2, 7, dtype=torch.complex64), encoding_axis=-3)


def _masked_ops(cuda):
    from pygrog_b200.operator import MaskedFFT

    z = golden("sub_masked.npz")
    _, grid, img, C, K, T = parse_meta(z["meta"])
    mk = dict(grid_shape=grid, image_shape=img, mask=torch.from_numpy(z["in_mask"]),
              density=torch.from_numpy(z["in_density"]), smaps=torch.from_numpy(z["in_smaps"]), device=cuda)
    basis = torch.from_numpy(z["in_basis"])
    sub_t = with_subspace(MaskedFFT(**mk, toeplitz=True), basis, encoding_axis=-3)
    sub_n = with_subspace(MaskedFFT(**mk, toeplitz=False), basis, encoding_axis=-3)
    return z, sub_t, sub_n


def test_subspace_masked_operator_matches_reference(cuda):
    """SubspaceMaskedFFT (``gadgets/_subspace.py:761-1004``) against the reference
    fixture ``sub_masked.npz``: adjoint, forward, both normals, the density PSF
    and CG (the device CG loop and the nested operator)."""
    from pygrog_b200.operator import SubspaceMaskedFFT

    z, sub_t, sub_n = _masked_ops(cuda)
    assert isinstance(sub_t, SubspaceMaskedFFT)
    b = torch.from_numpy(z["in_b"])
    xk = torch.from_numpy(z["in_xk"])
    assert rel_l2(sub_t.adjoint(b).numpy(), z["ref_sub_adjoint"]) < 1e-5
    assert rel_l2(sub_t.forward(xk).numpy(), z["ref_sub_forward"]) < 1e-5
    assert rel_l2(sub_t.normal(xk).numpy(), z["ref_sub_normal_toep"]) < 1e-5
    assert rel_l2(sub_t._toep_op.psf.cpu().numpy(), z["ref_sub_psf"]) < 1e-5
    assert rel_l2(sub_n.normal(xk).numpy(), z["ref_sub_normal_notoep"]) < 1e-5
    x = sub_t.solve(b, method="cg", max_iter=8, damp=1e-3, tol=0.0)
    assert rel_l2(x.numpy(), z["ref_sub_cg"]) < 1e-4
    xd = sub_t.solve(b.to(cuda), method="cg", max_iter=8, damp=1e-3, tol=0.0)  # device CG loop
    assert xd.is_cuda and rel_l2(xd.cpu().numpy(), z["ref_sub_cg"]) < 1e-4


def test_subspace_masked_adjointness_and_batches(cuda):
    z, _, sub_n = _masked_ops(cuda)
    g = torch.Generator().manual_seed(4)
    y = torch.randn(*z["in_b"].shape, dtype=torch.complex64, generator=g)
    x = torch.randn(*z["in_xk"].shape, dtype=torch.complex64, generator=g)
    lhs = torch.vdot(sub_n.adjoint(y).flatten().to(torch.complex128), x.flatten().to(torch.complex128))
    rhs = torch.vdot(y.flatten().to(torch.complex128), sub_n.forward(x).flatten().to(torch.complex128))
    assert abs(lhs - rhs) / abs(lhs) < 1e-4
    yb = torch.stack([y, 2 * y + 1j])
    xb = sub_n.adjoint(yb)
    assert xb.shape == (2, *z["in_xk"].shape)
    assert rel_l2(xb[1].numpy(), sub_n.adjoint(yb[1]).numpy()) < 1e-6
    fb = sub_n.forward(torch.stack([x, x * 0.5]))
    assert fb.shape == (2, *z["in_b"].shape)
    assert rel_l2(fb[1].numpy(), 0.5 * sub_n.forward(x).numpy()) < 1e-6
    with pytest.raises(ValueError, match="does not match natural_shape"):
        with_subspace(sub_n._base, torch.zeros(2, 7, dtype=torch.complex64), encoding_axis=-3)
