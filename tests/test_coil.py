"""Coil compression: the PCA step before the GROG path (utils/_coil_compress.py:23-57).

CPU: properties of the FP64 oracle.  GPU: the device covariance, matrix and
compression against the oracle on the same seeded data."""

import numpy as np
import pytest
import torch

from conftest import rel_l2
from oracle import coil as oc


def _coil_data(C=32, n=4000, rank=6, seed=0):
    """Samples of a few strong spatial modes mixed into C coils plus weak noise
    (a clear eigenvalue spectrum, like real coil arrays)."""
    rng = np.random.default_rng(seed)
    mix = rng.standard_normal((C, rank)) + 1j * rng.standard_normal((C, rank))
    scale = np.geomspace(10.0, 1.0, rank)
    src = (rng.standard_normal((rank, n)) + 1j * rng.standard_normal((rank, n))) * scale[:, None]
    noise = 0.01 * (rng.standard_normal((C, n)) + 1j * rng.standard_normal((C, n)))
    traj = rng.uniform(-64, 64, (n, 2)).astype(np.float32)
    return (mix @ src + noise).astype(np.complex64), traj


def test_oracle_matrix_is_orthonormal_and_ordered():
    d, _ = _coil_data()
    mat = oc.compression_matrix(d, 8)
    assert mat.shape == (8, 32)
    np.testing.assert_allclose(mat @ mat.conj().T, np.eye(8), atol=1e-10)
    energy = np.linalg.norm(mat @ d.astype(np.complex128), axis=1)
    assert (np.diff(energy) <= 1e-9 * energy[0]).all()
    idx = np.abs(mat).argmax(axis=1)
    ph = mat[np.arange(8), idx]
    assert np.allclose(ph.imag, 0) and (ph.real > 0).all()


def test_oracle_energy_fraction_and_calibration_subset():
    d, traj = _coil_data()
    comp, mat = oc.coil_compress(d, 0.999)
    w = np.linalg.eigvalsh(d.astype(np.complex128) @ d.conj().T.astype(np.complex128))[::-1]
    k = int(np.searchsorted(np.cumsum(w) / w.sum(), 0.999 - 1e-12)) + 1
    assert mat.shape[0] == k and comp.shape == (k, d.shape[1])
    comp2, mat2 = oc.coil_compress(d, 6, traj=traj, krad_thresh=0.3)
    assert mat2.shape == (6, 32)
    assert rel_l2(comp2, mat2 @ d.astype(np.complex128)) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("n_coils,thresh", [(12, None), (8, 0.4), (0.99, None)])
def test_gpu_coil_compress_matches_oracle(cuda, n_coils, thresh):
    from pygrog_b200.utils import coil_compress

    d, traj = _coil_data(seed=3)
    comp, mat = coil_compress(d, n_coils, traj=traj if thresh else None, krad_thresh=thresh)
    rcomp, rmat = oc.coil_compress(d, n_coils, traj=traj if thresh else None, krad_thresh=thresh)
    assert isinstance(comp, np.ndarray) and mat.shape == rmat.shape
    # well-separated leading components: the matrices agree; the last kept
    # component may share its eigenvalue with discarded noise, so compare
    # the leading rank-6 part strictly and the compressed data through the
    # projector onto the kept subspace
    k6 = min(6, mat.shape[0])
    assert rel_l2(mat[:k6], rmat[:k6]) < 1e-5
    P = mat.conj().T @ mat
    rP = rmat.conj().T @ rmat
    assert rel_l2(P @ d, rP @ d.astype(np.complex128)) < 1e-4
    assert rel_l2(comp[:k6], rcomp[:k6]) < 1e-5


@pytest.mark.gpu
def test_gpu_coil_compress_batched_kernel(cuda):
    """pgb_coil_compress on a (B, C, N) batch equals mat @ data per batch entry."""
    from pygrog_b200 import _lib

    rng = np.random.default_rng(9)
    B, C, K, N = 3, 20, 7, 5003
    x = (rng.standard_normal((B, C, N)) + 1j * rng.standard_normal((B, C, N))).astype(np.complex64)
    m = (rng.standard_normal((K, C)) + 1j * rng.standard_normal((K, C))).astype(np.complex64)
    xd, md = torch.from_numpy(x).to(cuda), torch.from_numpy(m).to(cuda)
    out = torch.empty(B, K, N, dtype=torch.complex64, device=cuda)
    _lib.call("pgb_coil_compress", xd.data_ptr(), N, C, K, B, md.data_ptr(), out.data_ptr(), _lib.stream_ptr(cuda))
    ref = np.einsum("kc,bcn->bkn", m.astype(np.complex128), x.astype(np.complex128))
    assert rel_l2(out.cpu().numpy(), ref) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("C,K,B,N", [(32, 12, 1, 4099), (32, 16, 2, 1000), (12, 5, 1, 777), (20, 9, 3, 64),
                                     (32, 12, 2, 200_000), (8, 8, 1, 130)])
def test_gpu_coil_compress_tensor_cores(cuda, C, K, B, N):
    """bf16x3 tensor-core compression within 1e-5 of the FP64 product."""
    from pygrog_b200 import _lib

    rng = np.random.default_rng(C * K + N)
    x = (rng.standard_normal((B, C, N)) + 1j * rng.standard_normal((B, C, N))).astype(np.complex64)
    m = (rng.standard_normal((K, C)) + 1j * rng.standard_normal((K, C))).astype(np.complex64)
    xd, md = torch.from_numpy(x).to(cuda), torch.from_numpy(m).to(cuda)
    out = torch.empty(B, K, N, dtype=torch.complex64, device=cuda)
    _lib.call("pgb_coil_compress_tc", xd.data_ptr(), N, C, K, B, md.data_ptr(), out.data_ptr(), _lib.stream_ptr(cuda))
    ref = np.einsum("kc,bcn->bkn", m.astype(np.complex128), x.astype(np.complex128))
    assert rel_l2(out.cpu().numpy(), ref) < 1e-5
