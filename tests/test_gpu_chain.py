"""The shift chain in both tensor-core forms (mma.sync, tcgen05 with the
accumulator in tensor memory) against an FP64 restatement of
``y = W3 Dx[k] W2 Dy[j] W1 Dz[i] W0 x`` (the eigen-factored table product of
``calib/_grappa.py:62-72, 184-208``), at 12 and 32 coils, on a replica count
that leaves ragged last tiles for both forms (128-replica and 16-replica
tiles)."""

import numpy as np
import pytest
import torch

from conftest import rel_l2
from pygrog_b200.calib import _chain

pytestmark = pytest.mark.gpu


def _unitary(rng, n):
    z = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    q, _ = np.linalg.qr(z)
    return q


def _case(C, R, seed, device):
    rng = np.random.default_rng(seed)
    W = np.stack([_unitary(rng, C) for _ in range(4)])
    ph = np.exp(1j * rng.uniform(-np.pi, np.pi, (3, _chain.STEPS, C)))
    ijk = rng.integers(0, _chain.STEPS, (3, R))
    xc = rng.standard_normal((C, R)) + 1j * rng.standard_normal((C, R))
    x = np.empty((2 * C, R), dtype=np.float32)
    x[0::2], x[1::2] = xc.real, xc.imag
    Wd, phd = _chain.chain_operands(W, ph, device)
    return (W, ph, ijk, xc), (torch.from_numpy(x).to(device), _chain.pack_shift_indices(torch.from_numpy(ijk).to(device)),
                              Wd, phd)


def _reference(W, ph, ijk, xc, rep):
    y = xc.astype(np.complex128)
    for _ in range(rep):
        for s in range(4):
            y = W[s] @ y
            if s < 3:
                y = y * ph[s][ijk[s]].T
    return y


@pytest.mark.parametrize("C", [12, 32])
@pytest.mark.parametrize("variant", ["mma", "tcgen05"])
@pytest.mark.parametrize("rep", [1, 2])
def test_shift_chain_matches_fp64(cuda, C, variant, rep):
    R = 10000 + 7  # 78 full tiles of 128 + 23, 625 m-tiles of 16 + 7
    (W, ph, ijk, xc), (x, idx, Wd, phd) = _case(C, R, 11 + C, cuda)
    out = torch.full_like(x, float("nan"))
    t = _chain.shift_chain(x, idx, Wd, phd, out, rep=rep, variant=variant)
    torch.cuda.synchronize(cuda)
    _chain.check_timeouts(t)
    o = out.double().cpu().numpy()
    got = o[0::2] + 1j * o[1::2]
    assert np.isfinite(got).all()
    assert rel_l2(got, _reference(W, ph, ijk, xc, rep)) < 1e-4 * rep


def test_shift_chain_forms_agree_and_reject_bad_arguments(cuda):
    C, R = 12, 4096
    _, (x, idx, Wd, phd) = _case(C, R, 5, cuda)
    a = torch.empty_like(x)
    b = torch.empty_like(x)
    _chain.shift_chain(x, idx, Wd, phd, a, variant="mma")
    t = _chain.shift_chain(x, idx, Wd, phd, b, variant="tcgen05")
    torch.cuda.synchronize(cuda)
    _chain.check_timeouts(t)
    assert rel_l2(a.cpu().numpy(), b.cpu().numpy()) < 3e-5
    x16 = torch.zeros(32, R, device=cuda)  # 16 coils: not built
    with pytest.raises(RuntimeError, match="12 and 32 coils"):
        _chain.shift_chain(x16, idx, Wd, phd, torch.empty_like(x16))
