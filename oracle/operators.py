"""Oracle: CPU restatement of the reference Cartesian operators (numpy).

TEST INFRASTRUCTURE ONLY (never imported by the product).  Parity pinned by
``tests/test_oracle_golden.py`` against fixtures produced by the reference
itself (``tests/golden/ops_*.npz``).

References (FiRMLAB-Pisa/pygrog):
  centred ortho FFT           _base/_fftc.py:114-139
  SparseFFT adjoint / forward operator/_sparse_fft.py:574-621, 741-789, 1154-1177
  Toeplitz normal             _toep/_grog_toep.py:154-209
  MaskedFFT                   operator/_masked_fft.py:322-430
  CG                          _solve/_solvers.py:49-139
  LSMR                        _solve/_solvers.py:145-262
"""

from __future__ import annotations

import os

import numpy as np


try:  # the same pocketfft algorithm, multi-threaded (large FP64 CG-SENSE checks)
    import scipy.fft as _fft

    _FFT_KW = {"workers": os.cpu_count() or 1}
except ImportError:  # pragma: no cover
    _fft = np.fft
    _FFT_KW = {}


def fftc(x, axes):
    return np.fft.fftshift(_fft.fftn(np.fft.ifftshift(x, axes=axes), axes=axes, norm="ortho", **_FFT_KW),
                           axes=axes)


def ifftc(x, axes):
    return np.fft.fftshift(_fft.ifftn(np.fft.ifftshift(x, axes=axes), axes=axes, norm="ortho", **_FFT_KW),
                           axes=axes)


def _slices(grid_shape, image_shape):
    return tuple(slice((g - i) // 2, (g - i) // 2 + i) for g, i in zip(grid_shape, image_shape))


def sparse_adjoint(sparse, idx_nat, sw_nat, grid_shape, image_shape, smaps=None):
    """sparse (C, R) natural order -> image (*img) with smaps, else (C, *img)."""
    C = sparse.shape[0]
    G = int(np.prod(grid_shape))
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    grid = np.zeros((C, G), dtype=np.complex128)
    for c in range(C):
        np.add.at(grid[c], idx_nat, sw_nat * sparse[c])
    img = ifftc(grid.reshape(C, *grid_shape), axes)[(slice(None), *_slices(grid_shape, image_shape))]
    if smaps is None:
        return img
    return (np.conj(smaps) * img).sum(0)


def sparse_forward(image, idx_nat, sw_nat, grid_shape, image_shape, smaps=None):
    """image (*img) [smaps] or (C, *img) -> sparse (C, R) natural order."""
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    coil = smaps * image if smaps is not None else image
    C = coil.shape[0]
    pad = np.zeros((C, *grid_shape), dtype=np.complex128)
    pad[(slice(None), *_slices(grid_shape, image_shape))] = coil
    k = fftc(pad, axes).reshape(C, -1)
    return sw_nat * k[:, idx_nat]


def psf(idx_nat, sw_nat, grid_shape):
    p = np.zeros(int(np.prod(grid_shape)), dtype=np.float64)
    np.add.at(p, idx_nat, sw_nat.astype(np.float64) ** 2)
    return p.reshape(grid_shape)


def toeplitz_normal(x, psf_grid, grid_shape, image_shape, smaps=None):
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    coil = smaps * x if smaps is not None else x
    C = coil.shape[0]
    pad = np.zeros((C, *grid_shape), dtype=np.complex128)
    sl = (slice(None), *_slices(grid_shape, image_shape))
    pad[sl] = coil
    img = ifftc(psf_grid * fftc(pad, axes), axes)[sl]
    if smaps is None:
        return img
    return (np.conj(smaps) * img).sum(0)


def masked_adjoint(kgrid, mask, grid_shape, image_shape, smaps=None):
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    img = ifftc(kgrid * mask, axes)[(slice(None), *_slices(grid_shape, image_shape))]
    return img if smaps is None else (np.conj(smaps) * img).sum(0)


def masked_forward(image, mask, grid_shape, image_shape, smaps=None):
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    coil = smaps * image if smaps is not None else image
    pad = np.zeros((coil.shape[0], *grid_shape), dtype=np.complex128)
    pad[(slice(None), *_slices(grid_shape, image_shape))] = coil
    return fftc(pad, axes) * mask


def cg(normal, AHb, damp=0.0, max_iter=20, tol=0.0):
    """_solvers.py:49-139 in complex128 (x0 = 0, no preconditioner)."""
    x = np.zeros_like(AHb)
    r = AHb.copy()
    p = r.copy()
    rz = np.vdot(r, r).real
    r0 = np.linalg.norm(r) + 1e-30
    for _ in range(max_iter):
        Ap = normal(p) + damp * p
        alpha = rz / (np.vdot(p, Ap).real + 1e-30)
        x = x + alpha * p
        r = r - alpha * Ap
        if np.linalg.norm(r) / r0 < tol:
            break
        rz_new = np.vdot(r, r).real
        p = r + rz_new / (rz + 1e-30) * p
        rz = rz_new
    return x


def lsmr(forward, adjoint, b, damp=0.0, max_iter=20, atol=1e-6, btol=1e-6):
    """_solvers.py:145-262 in complex128 / FP64 scalars (x0 = 0)."""
    beta = np.linalg.norm(b)
    if beta == 0:
        return adjoint(b)
    u = b / beta
    v = adjoint(u)
    alpha = np.linalg.norm(v)
    if alpha == 0:
        return np.zeros_like(v)
    v = v / alpha
    zetabar, alphabar = alpha * beta, alpha
    rho = rhobar = cbar = 1.0
    sbar = 0.0
    h, hbar = v.copy(), np.zeros_like(v)
    x = np.zeros_like(v)
    normb = beta
    for _ in range(max_iter):
        u = forward(v) - alpha * u
        beta = np.linalg.norm(u)
        if beta > 0:
            u = u / beta
            vf = adjoint(u) - beta * v
            alpha = np.linalg.norm(vf)
            if alpha > 0:
                v = vf / alpha
        alphahat = np.sqrt(alphabar**2 + damp**2)
        rhoold = rho
        rho = np.sqrt(alphahat**2 + beta**2)
        c, s = alphahat / rho, beta / rho
        thetanew = s * alpha
        alphabar = c * alpha
        rhobarold = rhobar
        thetabar = sbar * rho
        rhotemp = cbar * rho
        rhobar = np.sqrt(rhotemp**2 + thetanew**2)
        cbar, sbar = rhotemp / rhobar, thetanew / rhobar
        zeta = cbar * zetabar
        zetabar = -sbar * zetabar
        hbar = h - (thetabar * rho / (rhoold * rhobarold)) * hbar
        x = x + (zeta / (rho * rhobar)) * hbar
        h = v - (thetanew / rho) * h
        if abs(zetabar) / (normb + 1e-30) < atol + btol:
            break
    return x


# ---------------------------------------------------------------------------
# Low-rank subspace operator (gadgets/_subspace.py:311-508, _toep/_sub_toep.py:120-303)
# ---------------------------------------------------------------------------
def sub_adjoint(y, idx_nat, sw_nat, tidx, basis, grid_shape, image_shape, smaps):
    """y (C, R) natural order -> coefficients (K, *img).

    x_k = sum_c conj(S_c) crop(IFFT(scatter(sw^2 * basis[k, t] * y_c))) (pre_w = sw).
    """
    K = basis.shape[0]
    out = np.zeros((K, *image_shape), dtype=np.complex128)
    for k in range(K):  # pre-weight sw here, sparse_adjoint applies the second sw
        out[k] = sparse_adjoint(y * sw_nat * basis[k, tidx], idx_nat, sw_nat, grid_shape, image_shape, smaps)
    return out


def sub_forward(x, idx_nat, sw_nat, tidx, basis, grid_shape, image_shape, smaps):
    """coefficients (K, *img) -> y (C, R): y_c = sw^2 sum_k conj(basis[k, t]) FFT(pad(S_c x_k))[idx]."""
    K = basis.shape[0]
    acc = 0
    for k in range(K):
        acc = acc + np.conj(basis[k, tidx]) * sparse_forward(x[k], idx_nat, sw_nat, grid_shape, image_shape, smaps)
    return acc * sw_nat


def sub_psf(idx_nat, sw_nat, tidx, basis, grid_shape):
    """P[g, k, k'] = sum_{i: idx_i = g} sw_i^4 basis[k, t_i] conj(basis[k', t_i]) -> (*grid, K, K)."""
    K = basis.shape[0]
    G = int(np.prod(grid_shape))
    w4 = sw_nat.astype(np.float64) ** 4
    P = np.zeros((G, K, K), dtype=np.complex128)
    for k in range(K):
        for kp in range(K):
            np.add.at(P[:, k, kp], idx_nat, w4 * basis[k, tidx] * np.conj(basis[kp, tidx]))
    return P.reshape(*grid_shape, K, K)


def sub_toeplitz_normal(x, P, grid_shape, image_shape, smaps):
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    K = x.shape[0]
    sl = (slice(None), *_slices(grid_shape, image_shape))
    out = np.zeros_like(x, dtype=np.complex128)
    for c in range(smaps.shape[0]):
        pad = np.zeros((K, *grid_shape), dtype=np.complex128)
        pad[sl] = smaps[c] * x
        Kk = fftc(pad, axes)
        mixed = np.einsum("...ab,b...->a...", P, Kk)
        out += np.conj(smaps[c]) * ifftc(mixed, axes)[sl]
    return out


# ---- SubspaceMaskedFFT (gadgets/_subspace.py:761-1004, _toep/_sub_toep.py:64-117) ----
def submasked_tcell(grid_shape, t_axis):
    """Encoding (frame) index of every grid cell: its coordinate along ``t_axis``."""
    T = grid_shape[t_axis]
    shp = [1] * len(grid_shape)
    shp[t_axis] = T
    return np.broadcast_to(np.arange(T).reshape(shp), grid_shape).reshape(-1)


def submasked_adjoint(kgrid, mask, basis, t_axis, grid_shape, image_shape, smaps):
    """kgrid (C, *grid) -> (K, *img): x_k = sum_c conj(S_c) crop(ifftc(mask * basis[k, t] * y_c)),
    the centred transform over every grid axis (``_subspace.py:879-907``)."""
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    K = basis.shape[0]
    phi = basis[:, submasked_tcell(grid_shape, t_axis)].reshape(K, *grid_shape)
    sl = (slice(None), *_slices(grid_shape, image_shape))
    out = np.zeros((K, *image_shape), dtype=np.complex128)
    for c in range(kgrid.shape[0]):
        out += np.conj(smaps[c]) * ifftc(phi * kgrid[c] * mask, axes)[sl]
    return out


def submasked_forward(x, mask, basis, t_axis, grid_shape, image_shape, smaps):
    """(K, *img) -> (C, *grid): y_c = sum_k conj(basis[k, t]) mask fftc(pad(S_c x_k)) (``_subspace.py:950-988``)."""
    nd = len(grid_shape)
    axes = tuple(range(-nd, 0))
    K = basis.shape[0]
    phi = basis[:, submasked_tcell(grid_shape, t_axis)].reshape(K, *grid_shape)
    sl = (slice(None), *_slices(grid_shape, image_shape))
    out = np.zeros((smaps.shape[0], *grid_shape), dtype=np.complex128)
    for c in range(smaps.shape[0]):
        pad = np.zeros((K, *grid_shape), dtype=np.complex128)
        pad[sl] = smaps[c] * x
        out[c] = (np.conj(phi) * fftc(pad, axes) * mask).sum(0)
    return out


def submasked_psf(density, basis, t_axis, grid_shape):
    """The reference's masked PSF (``_sub_toep.py:64-105``): P[j, a, b] = density[j] *
    basis[b, t_j] * conj(basis[a, t_j]) -> (*grid, K, K); applied by
    :func:`sub_toeplitz_normal` as out_a = sum_b P[a, b] in_b."""
    K = basis.shape[0]
    Bj = basis[:, submasked_tcell(grid_shape, t_axis)].T  # (G, K)
    P = density.reshape(-1, 1, 1) * (np.conj(Bj)[:, :, None] * Bj[:, None, :])
    return P.reshape(*grid_shape, K, K)
