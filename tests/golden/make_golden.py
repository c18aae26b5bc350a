"""Generate golden fixtures by running the reference pygrog (CPU) on seeded inputs.

Run in a container that has the reference checkout (see ``refimport.py``):

    python tests/golden/make_golden.py [plans] [l0] [operators] [subspace] [submasked]

Writes ``tests/golden/*.npz``.  Every array stored under ``ref_*`` is an output
of the reference implementation itself (its Python package plus its C++
extension built from source); ``in_*`` arrays are the seeded inputs.  The
GPU parity tests and the oracle tests read these files; nothing reads the
reference checkout at test time.
"""

from __future__ import annotations

import pathlib
import sys

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
import refimport  # noqa: E402


def _c(rng, *shape, dtype=np.complex64):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)).astype(dtype)


PLAN_CASES = [
    # name, shape, coords shape, oversamp, kernel_width, kernel_shape, precision, C
    ("p2d_circle_osf2", (16, 16), (6, 40, 2), 2.0, 2, "circle", 1, 3),
    ("p2d_square_osf1_p2", (20, 20), (5, 48, 2), 1.0, 5, "square", 2, 4),
    ("p2d_cross_osf15", (18, 14), (4, 36, 2), 1.5, 3, "cross", 1, 2),
    ("p3d_sphere_osf1", (12, 12, 12), (7, 30, 3), 1.0, 2, "sphere", 1, 4),
    ("p3d_cube_default_osf", (10, 10, 10), (5, 24, 3), None, 3, "cube", 1, 3),
    ("p3d_sphere_osf2_p2", (8, 8, 8), (4, 20, 3), 2.0, 2, "sphere", 2, 2),
]


def make_plan_cases(pg, out):
    for k, (name, shape, cshape, osf, kwd, ks, prec, C) in enumerate(PLAN_CASES):
        rng = np.random.default_rng(100 + k)
        coords = (rng.standard_normal(cshape) * 4).astype(np.float32)
        ndim = cshape[-1]
        g = pg.calib.GrogInterpolator(
            shape=shape, coords=coords, oversamp=osf, kernel_width=kwd, kernel_shape=ks
        )
        calib = _c(rng, C, *([8] * ndim))
        plan = g.plan
        rec = dict(
            in_coords=coords,
            in_calib=calib,
            meta=np.array([repr((name, shape, osf, kwd, ks, prec, C))]),
            ref_grid_shape=np.asarray(plan.grid_shape),
            ref_target_idx=plan.target_idx.numpy(),
            ref_distances=plan.distances.numpy(),
            ref_weights=plan.weights.numpy(),
            ref_indices=plan.indices.numpy(),
            ref_sqrt_weights=plan.sqrt_weights.numpy(),
        )
        g.calc_interp_table(calib, lamda=0.01, precision=prec)
        rec["ref_interp_idx"] = g._interp_idx.numpy()
        table = g._interp_kernel.numpy()
        used = np.unique(rec["ref_interp_idx"])
        rec["ref_table_size"] = np.asarray(table.shape)
        rec["ref_table_used_idx"] = used
        rec["ref_table_used"] = table[used]
        data = _c(rng, C, *cshape[:-1])
        rec["in_data"] = data
        rec["ref_interpolate"] = np.asarray(g.interpolate(data))
        kg, mp = g.interpolate(data, grid=True)
        rec["ref_kgrid"] = np.asarray(kg)
        rec["ref_density"] = np.asarray(mp.density)
        rec["ref_mask"] = np.asarray(mp.mask)
        if ndim == 2:
            rec["ref_image"] = np.asarray(g.interpolate(data, ret_image=True))
        np.savez_compressed(out / f"plan_{name}.npz", **rec)
        print("wrote", name)


def make_fp64_case(pg, out):
    rng = np.random.default_rng(7)
    shape = (16, 16)
    coords = (rng.standard_normal((6, 32, 2)) * 4).astype(np.float32)
    g = pg.calib.GrogInterpolator(shape=shape, coords=coords, oversamp=2.0, kernel_width=2)
    calib = _c(rng, 3, 8, 8, dtype=np.complex128)
    g.calc_interp_table(calib, lamda=0.01, precision=1)
    data = _c(rng, 3, 6, 32, dtype=np.complex128)
    np.savez_compressed(
        out / "fp64_interp.npz",
        in_coords=coords,
        in_calib=calib,
        in_data=data,
        ref_table=g._interp_kernel.numpy(),
        ref_interp_idx=g._interp_idx.numpy(),
        ref_interpolate=np.asarray(g.interpolate(data)),
    )
    print("wrote fp64_interp")


def make_l0_cases(pg, out):
    ext = sys.modules["pygrog._pygrog_torch"]
    rng = np.random.default_rng(11)
    rec = {}
    # grog_interpolate
    N, B, C, K = 50, 2, 5, 9
    d = torch.from_numpy(_c(rng, N, B, C))
    idx = torch.from_numpy(rng.integers(0, K, N).astype(np.int64))
    ker = torch.from_numpy(_c(rng, K, C, C))
    rec.update(gi_data=d.numpy(), gi_idx=idx.numpy(), gi_kernel=ker.numpy(),
               ref_gi=ext.grog_interpolate(d, idx, ker).numpy())
    d2 = d.to(torch.complex128)
    k2 = ker.to(torch.complex128)
    rec["ref_gi128"] = ext.grog_interpolate(d2, idx, k2).numpy()
    # scatter_add / gather (sorted, with a hot cell and out-of-range indices)
    G, n = 64, 300
    ix = np.sort(rng.integers(0, G, n)).astype(np.int64)
    ix[100:180] = ix[100]
    w = rng.random(n).astype(np.float32)
    dat = _c(rng, n)
    grid = torch.from_numpy(_c(rng, G))
    g0 = grid.clone()
    ext.scatter_add(grid, torch.from_numpy(dat), torch.from_numpy(ix), torch.from_numpy(w))
    rec.update(sa_grid0=g0.numpy(), sa_idx=ix, sa_w=w, sa_data=dat, ref_sa=grid.numpy())
    gsrc = torch.from_numpy(_c(rng, G))
    rec.update(ga_grid=gsrc.numpy(),
               ref_ga=ext.gather(gsrc, torch.from_numpy(ix), torch.from_numpy(w)).numpy())
    # psf kernels
    wsq = (rng.random(n) + 0.1).astype(np.float32)
    psf = torch.zeros(G, dtype=torch.float32)
    ext.psf_scatter_scalar(psf, torch.from_numpy(ix), torch.from_numpy(wsq))
    rec.update(ps_wsq=wsq, ref_ps=psf.numpy())
    M = 3
    bps = _c(rng, n, M)
    po = torch.zeros(G, M, M, dtype=torch.complex64)
    ext.psf_scatter_outer(po, torch.from_numpy(ix), torch.from_numpy(wsq), torch.from_numpy(bps))
    rec.update(po_basis=bps, ref_po=po.numpy())
    Kb, T = 4, 16
    basis = _c(rng, Kb, T)
    tix = rng.integers(0, T, n).astype(np.int64)
    pb = torch.zeros(G, Kb, Kb, dtype=torch.complex64)
    ext.psf_scatter_outer_basis(pb, torch.from_numpy(ix), torch.from_numpy(wsq), torch.from_numpy(basis),
                                torch.from_numpy(tix))
    rec.update(pb_basis=basis, pb_tix=tix, ref_pb=pb.numpy())
    np.savez_compressed(out / "l0_ops.npz", **rec)
    print("wrote l0_ops")


def make_operator_cases(pg, out):
    """SparseFFT / MaskedFFT / Toeplitz / CG on a small GROG plan (2-D and 3-D)."""
    for name, shape, img, cshape, osf, C in [
        ("op2d", (24, 24), (20, 20), (8, 48, 2), 2.0, 4),
        ("op3d", (10, 10, 10), (10, 10, 10), (6, 20, 3), 1.0, 3),
    ]:
        rng = np.random.default_rng(len(name) * 31 + C)
        coords = (rng.standard_normal(cshape) * 4).astype(np.float32)
        g = pg.calib.GrogInterpolator(shape=shape, coords=coords, oversamp=osf, kernel_width=2,
                                      image_shape=img)
        ndim = cshape[-1]
        calib = _c(rng, C, *([8] * ndim))
        g.calc_interp_table(calib, lamda=0.01, precision=1)
        data = _c(rng, C, *cshape[:-1])
        smaps = (_c(rng, C, *img) * 0.5).astype(np.complex64)
        sparse = torch.as_tensor(np.asarray(g.interpolate(data)))
        b = sparse * g.plan.pre_weights.unsqueeze(0)
        op = pg.operator.SparseFFT(plan=g.plan, smaps=torch.from_numpy(smaps), toeplitz=True)
        opn = pg.operator.SparseFFT(plan=g.plan, smaps=torch.from_numpy(smaps), toeplitz=False)
        opc = pg.operator.SparseFFT(plan=g.plan, toeplitz=False)  # no smaps (coil images)
        x = torch.from_numpy(_c(rng, *img))
        xc = torch.from_numpy(_c(rng, C, *img))
        rec = dict(
            in_coords=coords, in_calib=calib, in_data=data, in_smaps=smaps,
            in_x=x.numpy(), in_xc=xc.numpy(), in_b=b.numpy(),
            meta=np.array([repr((name, shape, img, osf, C))]),
            ref_adjoint=op.adjoint(b).numpy(),
            ref_forward=op.forward(x).numpy().reshape(C, -1),
            ref_adjoint_nosmaps=opc.adjoint(b).numpy(),
            ref_forward_nosmaps=opc.forward(xc).numpy().reshape(C, -1),
            ref_normal_toep=op.normal(x).numpy(),
            ref_normal_notoep=opn.normal(x).numpy(),
            ref_psf=op._toep_op.psf.numpy(),
        )
        bn = b.reshape(C, *op.natural_shape)
        rec["ref_cg"] = op.solve(bn, method="cg", max_iter=8, damp=1e-3, tol=0.0).numpy()
        rec["ref_lsmr"] = opn.solve(bn, method="lsmr", max_iter=8, damp=1e-3).numpy()
        # Masked FFT path (grid=True output)
        kg, mp = g.interpolate(data, grid=True)
        mop = pg.operator.MaskedFFT(plan=mp, smaps=torch.from_numpy(smaps), toeplitz=True)
        kgt = torch.as_tensor(np.asarray(kg))
        rec["ref_masked_adjoint"] = mop.adjoint(kgt).numpy()
        rec["ref_masked_forward"] = mop.forward(x).numpy()
        rec["ref_masked_normal"] = mop.normal(x).numpy()
        rec["ref_masked_cg"] = mop.solve(kgt, method="cg", max_iter=8, damp=1e-3, tol=0.0).numpy()
        np.savez_compressed(out / f"ops_{name}.npz", **rec)
        print("wrote", name)


def make_subspace_cases(pg, out):
    """SubspaceSparseFFT adjoint / forward / normal (Toeplitz and nested) / CG on
    a 2-D plan whose natural shape (T, 160, kw) carries T = 5 frames on the
    encoding axis -3 of the sparse layout (C, T, 160, kw)."""
    import importlib

    gad = importlib.import_module("pygrog.gadgets")
    rng = np.random.default_rng(2024)
    shape, img, C, K, T = (20, 20), (20, 20), 3, 2, 5
    coords = (rng.standard_normal((T, 160, 2)) * 4).astype(np.float32)
    g = pg.calib.GrogInterpolator(shape=shape, coords=coords, oversamp=2.0, kernel_width=2, image_shape=img)
    calib = _c(rng, C, 8, 8)
    g.calc_interp_table(calib, lamda=0.01, precision=1)
    smaps = (_c(rng, C, *img) * 0.5).astype(np.complex64)
    q, _ = np.linalg.qr(_c(rng, T, K, dtype=np.complex128))
    basis = q.T.astype(np.complex64)  # (K, T) orthonormal rows
    base_t = pg.operator.SparseFFT(plan=g.plan, smaps=torch.from_numpy(smaps), toeplitz=True)
    base_n = pg.operator.SparseFFT(plan=g.plan, smaps=torch.from_numpy(smaps), toeplitz=False)
    sub_t = gad.with_subspace(base_t, torch.from_numpy(basis), encoding_axis=-3)
    sub_n = gad.with_subspace(base_n, torch.from_numpy(basis), encoding_axis=-3)
    nat = tuple(int(v) for v in base_t.natural_shape)
    b = torch.from_numpy(_c(rng, C, *nat))
    xk = torch.from_numpy(_c(rng, K, *img))
    rec = dict(
        in_coords=coords, in_calib=calib, in_smaps=smaps, in_basis=basis, in_b=b.numpy(), in_xk=xk.numpy(),
        meta=np.array([repr(("sub2d", shape, img, 2.0, C, K, T))]),
        ref_sub_adjoint=sub_t.adjoint(b).numpy(),
        ref_sub_forward=sub_t.forward(xk).numpy(),
        ref_sub_normal_toep=sub_t.normal(xk).numpy(),
        ref_sub_normal_notoep=sub_n.normal(xk).numpy(),
    )
    rec["ref_sub_psf"] = sub_t._toep_op.psf.numpy()
    rec["ref_sub_cg"] = sub_t.solve(b, method="cg", max_iter=6, damp=1e-3, tol=0.0).numpy()
    np.savez_compressed(out / "sub_sub2d.npz", **rec)
    print("wrote sub2d")


def make_subspace_masked_case(pg, out):
    """SubspaceMaskedFFT adjoint / forward / normal (Toeplitz with the density
    PSF, and nested) / CG on a MaskedFFT whose grid (T, gy, gx) carries T = 5
    frames on its first axis (encoding axis -3 of the layout (C, T, gy, gx));
    the reference transforms and crops every grid axis, so the image shape
    has the grid's rank (T, ny, nx)."""
    import importlib

    gad = importlib.import_module("pygrog.gadgets")
    rng = np.random.default_rng(2025)
    grid, img, C, K, T = (5, 12, 10), (5, 8, 8), 3, 2, 5
    mask = (rng.random(grid) < 0.55).astype(np.float32)
    density = (mask * rng.uniform(0.5, 2.0, grid)).astype(np.float32)
    smaps = (_c(rng, C, *img) * 0.5).astype(np.complex64)
    q, _ = np.linalg.qr(_c(rng, T, K, dtype=np.complex128))
    basis = q.T.astype(np.complex64)  # (K, T) orthonormal rows
    mk = dict(grid_shape=grid, image_shape=img, mask=torch.from_numpy(mask), density=torch.from_numpy(density),
              smaps=torch.from_numpy(smaps))
    base_t = pg.operator.MaskedFFT(**mk, toeplitz=True)
    base_n = pg.operator.MaskedFFT(**mk, toeplitz=False)
    sub_t = gad.with_subspace(base_t, torch.from_numpy(basis), encoding_axis=-3)
    sub_n = gad.with_subspace(base_n, torch.from_numpy(basis), encoding_axis=-3)
    b = torch.from_numpy(_c(rng, C, *grid))
    xk = torch.from_numpy(_c(rng, K, *img))
    rec = dict(
        in_mask=mask, in_density=density, in_smaps=smaps, in_basis=basis, in_b=b.numpy(), in_xk=xk.numpy(),
        meta=np.array([repr(("submasked", grid, img, C, K, T))]),
        ref_sub_adjoint=sub_t.adjoint(b).numpy(),
        ref_sub_forward=sub_t.forward(xk).numpy(),
        ref_sub_normal_toep=sub_t.normal(xk).numpy(),
        ref_sub_normal_notoep=sub_n.normal(xk).numpy(),
    )
    rec["ref_sub_psf"] = sub_t._toep_op.psf.numpy()
    rec["ref_sub_cg"] = sub_t.solve(b, method="cg", max_iter=8, damp=1e-3, tol=0.0).numpy()
    np.savez_compressed(out / "sub_masked.npz", **rec)
    print("wrote submasked")


def main():
    pg = refimport.import_reference()
    torch.set_num_threads(4)
    out = HERE
    only = set(sys.argv[1:])
    if not only or "plans" in only:
        make_plan_cases(pg, out)
        make_fp64_case(pg, out)
    if not only or "l0" in only:
        make_l0_cases(pg, out)
    if not only or "operators" in only:
        make_operator_cases(pg, out)
    if not only or "subspace" in only:
        make_subspace_cases(pg, out)
    if not only or "submasked" in only:
        make_subspace_masked_case(pg, out)


if __name__ == "__main__":
    main()
