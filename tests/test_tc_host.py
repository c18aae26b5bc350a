"""Host side of the tensor-core gridder, checked on the CPU.

The fragment words and phase tables of ``calib/_tc.py`` are run through a
numpy model of the kernel's register dataflow (``csrc/grog_tc.cu``:
``mm_stage`` / ``chain``) on the documented mma.sync m16n8k16 / m16n8k8
fragment layouts, and the result is compared with the table product applied
in FP64.  This pins the realification, the fragment packing, the C -> A
register hand-off between stages and the phase ordering without a GPU.
"""

import numpy as np
import pytest
import torch

from pygrog_b200.calib._grappa import KernelTable, eigen_factors
from pygrog_b200.calib._tc import padded_coils, tc_operands


def _bf16(x):
    return torch.from_numpy(np.asarray(x, dtype=np.float32)).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)


def _unpack(word):
    w = np.asarray(word, dtype=np.uint32)
    lo = (w & 0xFFFF).astype(np.uint32) << 16
    hi = (w >> 16).astype(np.uint32) << 16
    return lo.view(np.float32).astype(np.float64), hi.view(np.float32).astype(np.float64)


# ---- hardware model: PTX fragment layouts (g = lane // 4, t = lane % 4) ----
def _mma(d, a_regs, b_regs, k):
    """d (32, 4) += A B for m16n8k{k}; a_regs (32, k // 4) pairs, b_regs (32, k // 8) pairs."""
    A = np.zeros((16, k))
    B = np.zeros((k, 8))
    for lane in range(32):
        g, t = divmod(lane, 4)
        for i, (row, col) in enumerate([(g, 2 * t), (g + 8, 2 * t), (g, 2 * t + 8), (g + 8, 2 * t + 8)][: k // 4]):
            A[row, col], A[row, col + 1] = a_regs[lane][i]
        for i, krow in enumerate([2 * t, 2 * t + 8][: k // 8]):
            B[krow, g], B[krow + 1, g] = b_regs[lane][i]
    D = A @ B
    for lane in range(32):
        g, t = divmod(lane, 4)
        d[lane] += [D[g, 2 * t], D[g, 2 * t + 1], D[g + 8, 2 * t], D[g + 8, 2 * t + 1]]


def _model_tile(x16, ix16, ops, fwd: bool, terms: int):
    """Mirror of the kernel's chain on one 16-row m-tile; returns (16, CP) complex."""
    wfrag, dtab = ops["fwd" if fwd else "adj"]
    wfrag = wfrag.cpu().numpy().view(np.uint32)
    dtab = dtab.cpu().numpy()
    CP, nd = ops["CP"], ops["ndim"]
    NT, K16, K8 = CP // 4, CP // 8, (CP // 4) % 2
    v = np.zeros((32, 2, NT), dtype=np.complex128)
    for lane in range(32):
        g, t = divmod(lane, 4)
        for r in range(2):
            for m in range(NT):
                v[lane, r, m] = x16[g + 8 * r, 4 * m + t]
    for s in range(nd + 1):
        hi_a = np.stack([_bf16(v.real), _bf16(v.imag)], -1)  # (32, 2, NT, 2)
        lo_a = np.stack([_bf16(v.real - hi_a[..., 0]), _bf16(v.imag - hi_a[..., 1])], -1)
        bh = [_unpack(wfrag[s, 0, f]) for f in range(wfrag.shape[2])]
        bl = [_unpack(wfrag[s, 1, f]) for f in range(wfrag.shape[2])]
        bh = [np.stack(p, -1) for p in bh]  # (32, 2)
        bl = [np.stack(p, -1) for p in bl]
        out = np.zeros((32, 2, NT), dtype=np.complex128)
        for nt in range(NT):
            d = np.zeros((32, 4))
            f = nt * (2 * K16 + K8)
            terms_l = ([(lo_a, bh), (hi_a, bl)] if terms == 3 else []) + [(hi_a, bh)]
            for kc in range(K16):
                for a, b in terms_l:
                    regs = [[a[l, 0, 2 * kc], a[l, 1, 2 * kc], a[l, 0, 2 * kc + 1], a[l, 1, 2 * kc + 1]] for l in range(32)]
                    _mma(d, regs, [[b[f][l], b[f + 1][l]] for l in range(32)], 16)
                f += 2
            if K8:
                for a, b in terms_l:
                    regs = [[a[l, 0, NT - 1], a[l, 1, NT - 1]] for l in range(32)]
                    _mma(d, regs, [[b[f][l]] for l in range(32)], 8)
            out[:, 0, nt] = d[:, 0] + 1j * d[:, 1]
            out[:, 1, nt] = d[:, 2] + 1j * d[:, 3]
        v = out
        if s < nd:
            for lane in range(32):
                g, t = divmod(lane, 4)
                for r in range(2):
                    a = s if fwd else nd - 1 - s
                    step = ix16[g + 8 * r, a]
                    for m in range(NT):
                        v[lane, r, m] *= dtab[s, step, 4 * m + t]
    res = np.zeros((16, CP), dtype=np.complex128)
    for lane in range(32):
        g, t = divmod(lane, 4)
        for r in range(2):
            for m in range(NT):
                res[g + 8 * r, 4 * m + t] = v[lane, r, m]
    return res


def _acr(C, ndim, seed):
    """Smooth multi-coil calibration block (Gaussian coil bumps on a disc phantom)."""
    rng = np.random.default_rng(seed)
    n = 24
    ax = np.linspace(-1, 1, n)
    grids = np.meshgrid(*([ax] * ndim), indexing="ij")
    r2 = sum(a * a for a in grids)
    ph = (r2 < 0.6).astype(np.float64) + 0.5 * (r2 < 0.2)
    out = []
    for _ in range(C):
        c = rng.uniform(-0.7, 0.7, ndim)
        bump = np.exp(-sum((a - ci) ** 2 for a, ci in zip(grids, c)) / 0.5)
        img = ph * bump * np.exp(1j * rng.uniform(0, 2 * np.pi))
        k = np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(img), norm="ortho"))
        lo = n // 2 - 6
        out.append(k[tuple(slice(lo, lo + 12) for _ in range(ndim))])
    return np.stack(out).astype(np.complex64)


@pytest.mark.parametrize("ndim,C,terms", [(3, 12, 3), (2, 8, 3), (2, 5, 3), (3, 4, 1), (2, 16, 3), (2, 20, 3),
                                          (3, 32, 3)])
def test_tc_dataflow_matches_table(ndim, C, terms):
    acr = _acr(C, ndim, seed=C + ndim)
    table, nsteps, nd, _ = KernelTable(acr, 1.0, 1, 0.01, return_factors=True)
    ef = eigen_factors(acr, 1.0, 1, 0.01)
    assert ef.nsteps == nsteps and ef.ndim == nd == ndim
    ops = tc_operands(ef, C, "cpu")
    CP = padded_coils(C)
    rng = np.random.default_rng(7)
    x = np.zeros((16, CP), dtype=np.complex128)
    x[:, :C] = rng.standard_normal((16, C)) + 1j * rng.standard_normal((16, C))
    ix = rng.integers(0, nsteps, (16, ndim))
    # table index: 3-D e = i n^2 + j n + k with (i, j, k) in the forward axis order (z, y, x);
    # 2-D e = i n + j with (i, j) = (y, x)
    e = ix[:, 0] * nsteps + ix[:, 1] if ndim == 2 else (ix[:, 0] * nsteps + ix[:, 1]) * nsteps + ix[:, 2]
    T = table[e].astype(np.complex128)
    ref = np.einsum("nrc,nc->nr", T, x[:, :C])
    got = _model_tile(x, ix, ops, True, terms)
    tol = 1e-4 if terms == 3 else 2e-2
    assert np.linalg.norm(got[:, :C] - ref) / np.linalg.norm(ref) < tol
    assert np.abs(got[:, C:]).max(initial=0.0) == 0.0
    # adjoint chain: T^H y
    refa = np.einsum("nrc,nr->nc", T.conj(), x[:, :C])
    gota = _model_tile(x, ix, ops, False, terms)
    assert np.linalg.norm(gota[:, :C] - refa) / np.linalg.norm(refa) < tol


@pytest.mark.parametrize("C,CP", [(1, 4), (12, 12), (16, 16), (17, 24), (24, 24), (25, 32), (32, 32)])
def test_tc_padding_and_sub_chunk_budget(C, CP):
    """Coil padding of the operands matches the kernels; above 16 coils the
    sub-chunks hold 128 entries and one of them still fits shared memory."""
    from pygrog_b200 import _lib

    assert padded_coils(C) == CP
    lib = _lib.lib()
    cap = 256 if C <= 16 else 128
    for nd in (2, 3):
        assert lib.pgb_grog_tc_blocks_per_sm(C, nd) >= 1
        cells = 4 * 4 * 8 if nd == 3 else 8 * 16  # second-smallest bricks of the gridder's candidates
        assert lib.pgb_grog_tc_smem_bytes(C, cells, 9, nd, cap) <= 227 * 1024
    assert lib.pgb_grog_tc_blocks_per_sm(33, 3) == 0


def test_tc_operands_pick_the_lower_modeled_error():
    """The eigenvector scaling of the operands is the one with the lower
    modeled bf16x3 error; the model's plain-bf16 error is reported too."""
    from pygrog_b200.calib._tc import _chain, balance_eigenvectors, chain_rounding_error

    C, ndim = 20, 2
    acr = _acr(C, ndim, seed=3)
    ef = eigen_factors(acr, 1.0, 1, 0.01)
    ops = tc_operands(ef, C, "cpu")
    CP = padded_coils(C)
    V0 = [np.asarray(v.numpy(), dtype=np.complex128) for v, _ in ef.axes]
    lam = [np.asarray(l.numpy(), dtype=np.complex128) for _, l in ef.axes]
    d = ef.deltas.numpy().astype(np.float32).astype(np.float64)
    errs = []
    for V in (V0, [balance_eigenvectors(v) for v in V0]):
        # same operator whatever the scaling
        mats, D = _chain(V, lam, d, C, CP)
        errs.append(chain_rounding_error(mats, D, C, CP, 3))
        for s in range(ndim):
            np.testing.assert_allclose(V[s] @ np.diag(np.exp(0.3 * lam[s])) @ np.linalg.inv(V[s]),
                                       V0[s] @ np.diag(np.exp(0.3 * lam[s])) @ np.linalg.inv(V0[s]), atol=1e-10)
    assert ops["model_err"][3] == min(errs) < 1e-4
    assert 1e-4 < ops["model_err"][1] < 5e-2
