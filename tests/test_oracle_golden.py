"""The oracle (numpy restatement) against golden fixtures from the reference itself.

Integer keys (target cells, shift indices, sorted cell indices) bit-exact;
distances bit-exact (float32 chain); floats within 1e-5 relative L2.
"""

import numpy as np
import pytest

from conftest import golden, golden_plan_cases, parse_meta, rel_l2
from oracle import grog as og


@pytest.mark.parametrize("case", golden_plan_cases())
def test_oracle_plan_matches_reference(case):
    z = golden(case)
    name, shape, osf, kwd, ks, prec, C = parse_meta(z["meta"])
    p = og.create_plan(shape, z["in_coords"], osf, kwd, ks)
    assert tuple(p["grid_shape"]) == tuple(z["ref_grid_shape"])
    np.testing.assert_array_equal(p["target_idx"], z["ref_target_idx"])
    np.testing.assert_array_equal(p["distances"], z["ref_distances"])
    np.testing.assert_allclose(p["weights"], z["ref_weights"], rtol=1e-6, atol=1e-7)
    fp = og.fft_plan(p)
    np.testing.assert_array_equal(fp["indices"], z["ref_indices"])
    # sqrt weights: same multiset per cell (sort ties may be ordered differently)
    np.testing.assert_allclose(np.sort(fp["sqrt_weights"]), np.sort(z["ref_sqrt_weights"]), rtol=1e-6, atol=1e-7)
    K = int(z["ref_table_size"][0])
    nsteps = int(round(K ** (1.0 / len(shape))))
    qi = og.quantize(p["distances"], prec, nsteps, K)
    np.testing.assert_array_equal(qi, z["ref_interp_idx"])


@pytest.mark.parametrize("case", golden_plan_cases())
def test_oracle_table_and_grid_match_reference(case):
    z = golden(case)
    name, shape, osf, kwd, ks, prec, C = parse_meta(z["meta"])
    tab, n, nd = og.kernel_table(z["in_calib"], 0.5, prec, 0.01)
    used = z["ref_table_used_idx"]
    assert tab.shape == tuple(z["ref_table_size"])
    assert rel_l2(tab[used], z["ref_table_used"]) < 1e-5
    # interpolation / gridding with the reference's own table entries
    full = np.zeros(tuple(z["ref_table_size"]), dtype=np.complex64)
    full[used] = z["ref_table_used"]
    p = og.create_plan(shape, z["in_coords"], osf, kwd, ks)
    data = z["in_data"].reshape(1, C, -1)
    rep = og.interpolate(data, z["ref_interp_idx"], full)[0]
    assert rel_l2(rep, z["ref_interpolate"]) < 1e-6
    kg, dens = og.grid(data, z["ref_interp_idx"], full, p, og.fft_plan(p))
    assert rel_l2(kg[0], z["ref_kgrid"].reshape(C, -1)) < 1e-5
    np.testing.assert_allclose(dens, z["ref_density"].reshape(-1), rtol=1e-5, atol=1e-6)


def test_oracle_degrid_is_adjoint_of_grid():
    z = golden("plan_p2d_circle_osf2.npz")
    name, shape, osf, kwd, ks, prec, C = parse_meta(z["meta"])
    full = np.zeros(tuple(z["ref_table_size"]), dtype=np.complex64)
    full[z["ref_table_used_idx"]] = z["ref_table_used"]
    p = og.create_plan(shape, z["in_coords"], osf, kwd, ks)
    rng = np.random.default_rng(3)
    N = z["in_coords"].size // 2
    G = int(np.prod(p["grid_shape"]))
    x = (rng.standard_normal((1, C, N)) + 1j * rng.standard_normal((1, C, N))).astype(np.complex128)
    y = (rng.standard_normal((1, C, G)) + 1j * rng.standard_normal((1, C, G))).astype(np.complex128)
    fx, _ = og.grid(x, z["ref_interp_idx"], full.astype(np.complex128), p, og.fft_plan(p))
    ahy = og.degrid(y, z["ref_interp_idx"], full.astype(np.complex128), p)
    lhs = np.vdot(y.ravel(), fx.ravel())
    rhs = np.vdot(ahy.ravel(), x.ravel())
    assert abs(lhs - rhs) / abs(lhs) < 1e-10


def test_oracle_l0_primitives_match_reference():
    z = golden("l0_ops.npz")
    ref = np.einsum("nij,nbj->nbi", z["gi_kernel"][z["gi_idx"]], z["gi_data"])
    assert rel_l2(ref, z["ref_gi"]) < 1e-6
    sa = og.scatter_add(z["sa_grid0"], z["sa_data"], z["sa_idx"], z["sa_w"])
    assert rel_l2(sa, z["ref_sa"]) < 1e-6
    ga = og.gather(z["ga_grid"], z["sa_idx"], z["sa_w"])
    assert rel_l2(ga, z["ref_ga"]) < 1e-7
    G = z["ref_ps"].size
    ps = og.psf_scalar(G, z["sa_idx"], z["ps_wsq"])
    np.testing.assert_allclose(ps, z["ref_ps"], rtol=1e-6, atol=1e-6)
    po = og.psf_outer(G, z["po_basis"].shape[1], z["sa_idx"], z["ps_wsq"], z["po_basis"])
    assert rel_l2(po, z["ref_po"]) < 1e-6
    pb = og.psf_outer_basis(G, z["pb_basis"].shape[0], z["sa_idx"], z["ps_wsq"], z["pb_basis"], z["pb_tix"])
    assert rel_l2(pb, z["ref_pb"]) < 1e-6


# ---------------------------------------------------------------------------
# Cartesian operators (SparseFFT / Toeplitz / MaskedFFT / CG)
# ---------------------------------------------------------------------------
from oracle import operators as oo  # noqa: E402


def _op_setup(name):
    z = golden(f"ops_{name}.npz")
    _, shape, img, osf, C = parse_meta(z["meta"])
    p = og.create_plan(shape, z["in_coords"], osf, 2, "circle")
    fp = og.fft_plan(p)
    idx_nat = fp["indices"][fp["inv_perm"]]
    sw_nat = fp["sqrt_weights"][fp["inv_perm"]].astype(np.float64)
    return z, shape, tuple(img), p, idx_nat, sw_nat, C


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_oracle_sparse_fft_matches_reference(name):
    z, shape, img, p, idx, sw, C = _op_setup(name)
    gs = tuple(p["grid_shape"])
    sm = z["in_smaps"].astype(np.complex128)
    b = z["in_b"].astype(np.complex128)
    assert rel_l2(oo.sparse_adjoint(b, idx, sw, gs, img, sm), z["ref_adjoint"]) < 1e-5
    assert rel_l2(oo.sparse_forward(z["in_x"], idx, sw, gs, img, sm), z["ref_forward"]) < 1e-5
    assert rel_l2(oo.sparse_adjoint(b, idx, sw, gs, img), z["ref_adjoint_nosmaps"]) < 1e-5
    assert rel_l2(oo.sparse_forward(z["in_xc"], idx, sw, gs, img), z["ref_forward_nosmaps"]) < 1e-5
    pg = oo.psf(idx, sw, gs)
    np.testing.assert_allclose(pg, z["ref_psf"], rtol=1e-5, atol=1e-6)
    assert rel_l2(oo.toeplitz_normal(z["in_x"], pg, gs, img, sm), z["ref_normal_toep"]) < 1e-5
    assert rel_l2(oo.toeplitz_normal(z["in_x"], pg, gs, img, sm), z["ref_normal_notoep"]) < 1e-4


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_oracle_cg_matches_reference(name):
    z, shape, img, p, idx, sw, C = _op_setup(name)
    gs = tuple(p["grid_shape"])
    sm = z["in_smaps"].astype(np.complex128)
    pg = oo.psf(idx, sw, gs)
    AHb = oo.sparse_adjoint(z["in_b"].astype(np.complex128), idx, sw, gs, img, sm)
    x = oo.cg(lambda v: oo.toeplitz_normal(v, pg, gs, img, sm), AHb, damp=1e-3, max_iter=8)
    # the reference iterates in complex64 with FP32 inner products
    assert rel_l2(x, z["ref_cg"]) < 1e-4


@pytest.mark.parametrize("name", ["op2d", "op3d"])
def test_oracle_lsmr_matches_reference(name):
    z, shape, img, p, idx, sw, C = _op_setup(name)
    gs = tuple(p["grid_shape"])
    sm = z["in_smaps"].astype(np.complex128)
    x = oo.lsmr(lambda v: oo.sparse_forward(v, idx, sw, gs, img, sm),
                lambda u: oo.sparse_adjoint(u, idx, sw, gs, img, sm),
                z["in_b"].astype(np.complex128), damp=1e-3, max_iter=8)
    # the reference iterates in complex64 with FP32 norms
    assert rel_l2(x, z["ref_lsmr"]) < 1e-4


def _sub_setup():
    z = golden("sub_sub2d.npz")
    _, shape, img, osf, C, K, T = parse_meta(z["meta"])
    p = og.create_plan(shape, z["in_coords"], osf, 2, "circle")
    fp = og.fft_plan(p)
    idx = fp["indices"][fp["inv_perm"]]
    sw = fp["sqrt_weights"][fp["inv_perm"]].astype(np.float64)
    nat = z["in_b"].shape[1:]
    tidx = np.broadcast_to(np.arange(T).reshape(T, 1, 1), nat).reshape(-1)
    return z, tuple(p["grid_shape"]), tuple(img), idx, sw, tidx


def test_oracle_subspace_matches_reference():
    z, gs, img, idx, sw, tidx = _sub_setup()
    sm = z["in_smaps"].astype(np.complex128)
    B = z["in_basis"].astype(np.complex128)
    C = sm.shape[0]
    b = z["in_b"].reshape(C, -1).astype(np.complex128)
    assert rel_l2(oo.sub_adjoint(b, idx, sw, tidx, B, gs, img, sm), z["ref_sub_adjoint"]) < 1e-5
    y = oo.sub_forward(z["in_xk"].astype(np.complex128), idx, sw, tidx, B, gs, img, sm)
    assert rel_l2(y, z["ref_sub_forward"].reshape(C, -1)) < 1e-5
    P = oo.sub_psf(idx, sw, tidx, B, gs)
    assert rel_l2(P, z["ref_sub_psf"]) < 1e-5
    xk = z["in_xk"].astype(np.complex128)
    assert rel_l2(oo.sub_toeplitz_normal(xk, P, gs, img, sm), z["ref_sub_normal_toep"]) < 1e-5
    nested = oo.sub_adjoint(oo.sub_forward(xk, idx, sw, tidx, B, gs, img, sm), idx, sw, tidx, B, gs, img, sm)
    assert rel_l2(nested, z["ref_sub_normal_notoep"]) < 1e-5
    AHb = oo.sub_adjoint(b, idx, sw, tidx, B, gs, img, sm)
    x = oo.cg(lambda v: oo.sub_toeplitz_normal(v, P, gs, img, sm), AHb, damp=1e-3, max_iter=6)
    assert rel_l2(x, z["ref_sub_cg"]) < 1e-4


def test_oracle_subspace_masked_matches_reference():
    """SubspaceMaskedFFT on a (T, gy, gx) grid with T = 5 frames on axis 0."""
    z = golden("sub_masked.npz")
    _, grid, img, C, K, T = parse_meta(z["meta"])
    sm = z["in_smaps"].astype(np.complex128)
    B = z["in_basis"].astype(np.complex128)
    mask = z["in_mask"].astype(np.float64)
    b = z["in_b"].astype(np.complex128)
    xk = z["in_xk"].astype(np.complex128)
    adj = oo.submasked_adjoint(b, mask, B, 0, grid, img, sm)
    assert rel_l2(adj, z["ref_sub_adjoint"]) < 1e-5
    assert rel_l2(oo.submasked_forward(xk, mask, B, 0, grid, img, sm), z["ref_sub_forward"]) < 1e-5
    P = oo.submasked_psf(z["in_density"].astype(np.float64), B, 0, grid)
    assert rel_l2(P, z["ref_sub_psf"]) < 1e-5
    assert rel_l2(oo.sub_toeplitz_normal(xk, P, grid, img, sm), z["ref_sub_normal_toep"]) < 1e-5
    nested = oo.submasked_adjoint(oo.submasked_forward(xk, mask, B, 0, grid, img, sm), mask, B, 0, grid, img, sm)
    assert rel_l2(nested, z["ref_sub_normal_notoep"]) < 1e-5
    x = oo.cg(lambda v: oo.sub_toeplitz_normal(v, P, grid, img, sm), adj, damp=1e-3, max_iter=8)
    assert rel_l2(x, z["ref_sub_cg"]) < 1e-4
