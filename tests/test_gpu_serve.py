"""Served reconstructions: each result is the same alone and in a batched,
overlapping mix, and within 1e-4 of an FP64 CG-SENSE on the same inputs.

The FP64 reference restates the reference chain
``interpolate -> * pre_weights -> SparseFFT.adjoint -> cg(Toeplitz normal)``
(``calib/_grog.py:437-555``, ``operator/_sparse_fft.py:574-621``,
``_toep/_grog_toep.py:154-209``, ``_solve/_solvers.py:49-139``) in complex128
with the oracle.
"""

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import grog as og
from oracle import operators as oo
from pygrog_b200.serve import ReconProtocol, ReconServer, Request, poisson_arrivals
from pygrog_b200.workloads import gaussian_coils, radial2d, spiral2d

pytestmark = pytest.mark.gpu


def _protocols(cuda):
    rng = np.random.default_rng(11)
    out = {}
    for name, n, C, coords, osf in [
        ("radial", 48, 4, radial2d(24, 96, 24.0), 1.0),
        ("spiral", 40, 6, spiral2d(6, 600, 20.0), 2.0),
    ]:
        acr = (rng.standard_normal((C, 12, 12)) + 1j * rng.standard_normal((C, 12, 12))).astype(np.complex64)
        maps = gaussian_coils((n, n), C, rng).astype(np.complex64)
        out[name] = ReconProtocol(name, (n, n), coords, acr, maps, oversamp=osf, kernel_width=2, max_iter=12,
                                  damp=1e-3, device=cuda)
    return out


def _requests(protos, n_req, rng, rate=400.0):
    arr = poisson_arrivals(rate, n_req / rate * 3, rng)[:n_req]
    names = list(protos)
    reqs = []
    for i, t in enumerate(arr):
        p = protos[names[i % len(names)]]
        d = (rng.standard_normal(p.data_shape) + 1j * rng.standard_normal(p.data_shape)).astype(np.complex64)
        reqs.append(Request(i, p.name, float(t), torch.from_numpy(d).pin_memory(), keep=True))
    return reqs


def _fp64_recon(p: ReconProtocol, data: np.ndarray) -> np.ndarray:
    g = p.interp
    plan = g.plan
    table = g._interp_kernel.numpy().astype(np.complex128)
    idx = g._interp_idx.cpu().numpy().reshape(int(np.prod(p.spatial)), -1)
    rep = og.interpolate(data.reshape(1, p.C, -1).astype(np.complex128), idx, table)[0]
    ip = plan.inv_perm.cpu().numpy()
    idx_nat = plan.indices.cpu().numpy()[ip]
    sw_nat = plan.sqrt_weights.cpu().numpy().astype(np.float64)[ip]
    b = rep * sw_nat  # pre_weights
    sm = p.op.smaps.cpu().numpy().astype(np.complex128)
    grid, img = tuple(p.op.grid_shape), tuple(p.op.image_shape)
    AHb = oo.sparse_adjoint(b, idx_nat, sw_nat, grid, img, sm)
    psf = oo.psf(idx_nat, sw_nat, grid)
    return oo.cg(lambda x: oo.toeplitz_normal(x, psf, grid, img, sm), AHb, damp=p.damp, max_iter=p.max_iter)


def test_served_results_match_alone_and_fp64(cuda):
    protos = _protocols(cuda)
    server = ReconServer(protos, mem_budget=2 << 30, max_batch=4, n_slots=3, device=cuda)
    rng = np.random.default_rng(5)
    reqs = _requests(protos, 24, rng)
    rep = server.run(reqs, realtime=False)  # all queued at t=0: batches must form
    assert rep["requests"] == 24 and rep["p99_ms"] >= rep["p50_ms"] > 0
    assert rep["mean_batch"] > 1.0
    live = _requests(protos, 12, np.random.default_rng(8))
    rep2 = server.run(live)  # Poisson arrivals in real time
    assert rep2["requests"] == 12 and rep2["p99_ms"] >= rep2["p50_ms"] > 0
    reqs = reqs + live
    for r in reqs:
        p = protos[r.protocol]
        alone = p.recon(r.data.to(cuda).unsqueeze(0), 0)[0].cpu()
        assert rel_l2(r.result.numpy(), alone.numpy()) < 1e-5
    for name in protos:
        r = next(q for q in reqs if q.protocol == name)
        ref = _fp64_recon(protos[name], r.data.numpy())
        assert rel_l2(r.result.numpy(), ref) < 1e-4


def test_memory_budget_limits_batches(cuda):
    protos = _protocols(cuda)
    one = max(p.bytes_per_request() for p in protos.values())
    server = ReconServer(protos, mem_budget=one * 2 + 1, max_batch=8, n_slots=4, device=cuda)
    rng = np.random.default_rng(6)
    reqs = _requests(protos, 16, rng, rate=5000.0)
    rep = server.run(reqs, realtime=False)
    assert rep["requests"] == 16
    for r in reqs:  # admission never put more requests in flight than the budget holds
        assert r.batch <= (2 * one + 1) // protos[r.protocol].bytes_per_request()


def test_subspace_requests_in_the_mix(cuda):
    from pygrog_b200.workloads import t2_subspace_basis

    rng = np.random.default_rng(21)
    T, ro, n, C = 24, 64, 32, 4
    coords = radial2d(T, ro, n / 2.0).reshape(T, ro, 2)
    acr = (rng.standard_normal((C, 12, 12)) + 1j * rng.standard_normal((C, 12, 12))).astype(np.complex64)
    maps = gaussian_coils((n, n), C, rng).astype(np.complex64)
    sub = ReconProtocol("sub", (n, n), coords, acr, maps, oversamp=2.0, max_iter=8,
                        basis=t2_subspace_basis(T, 3), encoding_axis=-3, device=cuda)
    protos = {"sub": sub, **_protocols(cuda)}
    server = ReconServer(protos, mem_budget=2 << 30, max_batch=3, n_slots=2, device=cuda)
    reqs = _requests(protos, 12, np.random.default_rng(22))
    rep = server.run(reqs, realtime=False)
    assert rep["mean_batch"] > 1.0
    for r in reqs:
        p = protos[r.protocol]
        alone = p.recon(r.data.to(cuda).unsqueeze(0), 0)[0].cpu()
        assert r.result.shape == alone.shape
        assert rel_l2(r.result.numpy(), alone.numpy()) < 1e-5
    r = next(q for q in reqs if q.protocol == "sub")
    sparse = sub.interp.interpolate(r.data.to(cuda).unsqueeze(0))
    ref = sub.op.solve(sparse.reshape(sub.C, *sub.natural_shape), method="cg", max_iter=sub.max_iter,
                       damp=sub.damp, tol=0.0)
    assert rel_l2(r.result.numpy(), ref.cpu().numpy()) < 1e-5


def test_uneven_batch_graph_matches_alone(cuda):
    """Protocols of different grid size, coil count and trajectory length
    reconstructed as one CUDA graph (each a branch): every image equals the
    same request reconstructed alone, and one equals an FP64 CG-SENSE; a
    second launch with new k-space gives that k-space's reconstructions."""
    from pygrog_b200.batch import UnevenBatch

    protos = _protocols(cuda)
    rng = np.random.default_rng(31)
    for name, n, C, sp, ro in [("r32", 32, 8, 17, 64), ("r56", 56, 3, 40, 112)]:
        acr = (rng.standard_normal((C, 12, 12)) + 1j * rng.standard_normal((C, 12, 12))).astype(np.complex64)
        maps = gaussian_coils((n, n), C, rng).astype(np.complex64)
        protos[name] = ReconProtocol(name, (n, n), radial2d(sp, ro, n / 2.0), acr, maps, oversamp=1.0,
                                     kernel_width=2, max_iter=9, damp=1e-3, device=cuda)
    plist = list(protos.values())
    for p in plist:
        p.prepare(1, 1, graphs=False)  # the single-request path used for comparison
    batch = UnevenBatch(plist, cuda)
    for launch in range(2):
        data = [(rng.standard_normal(p.data_shape) + 1j * rng.standard_normal(p.data_shape)).astype(np.complex64)
                for p in plist]
        outs = batch.run([torch.from_numpy(d) for d in data])
        assert batch.graph is not None
        for p, d, o in zip(plist, data, outs):
            alone = p.recon(torch.from_numpy(d).to(cuda).unsqueeze(0), 0)[0].cpu()
            assert o.shape == alone.shape
            assert rel_l2(o.numpy(), alone.numpy()) < 1e-5, p.name
        if launch == 0:
            ref = _fp64_recon(protos["spiral"], data[plist.index(protos["spiral"])])
            assert rel_l2(outs[plist.index(protos["spiral"])].numpy(), ref) < 1e-4


def test_servers_sharing_protocols_take_turns(cuda):
    """Two servers of different batch / slot configuration over the same
    protocols, used alternately: each re-prepares the protocols the other
    took over, and every result equals the request reconstructed alone."""
    protos = _protocols(cuda)
    a = ReconServer(protos, mem_budget=2 << 30, max_batch=4, n_slots=2, device=cuda)
    b = ReconServer(protos, mem_budget=2 << 30, max_batch=1, n_slots=1, device=cuda)
    rng = np.random.default_rng(41)
    done = []
    for srv in (a, b, a):
        reqs = _requests(protos, 8, rng)
        rep = srv.run(reqs, realtime=False)
        assert rep["requests"] == 8
        done += reqs
    for p in protos.values():
        p.prepare(1, 1, graphs=False)
    for r in done:
        alone = protos[r.protocol].recon(r.data.to(cuda).unsqueeze(0), 0)[0].cpu()
        assert rel_l2(r.result.numpy(), alone.numpy()) < 1e-5
