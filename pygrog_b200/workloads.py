"""Seeded synthetic workloads with the shapes of the GROG benchmark configurations.

No dataset is available offline, so trajectories, phantoms, coil maps and
k-space are generated from seeds (``numpy.random.default_rng(1000 + config)``):

* ``radial2d``   golden-angle radial (angle ``k*pi*(3-sqrt(5))``);
* ``kooshball``  3-D radial with directions from the 2-D golden means
  (phi1 = 0.4656, phi2 = 0.6823);
* ``spiral2d``   variable-density spiral interleaves;
* ``ellipse_phantom2d`` / ``gaussian_coils`` for images and coil maps.

Configurations (sizes as in the benchmark definitions):
  c0  256^2 image, 64 spokes x 512 readout, 8 coils, 5x5 square kernel
  c1  192^3 grid, 20,000 spokes x 384 readout, 32 -> 12 coils, sphere kw=4
  c2  320^2, spiral 24 x 4096, 16 coils, oversamp 2, CG-SENSE 30 iterations
  c3  64 uneven 2-D radial slices
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

GOLDEN_ANGLE = math.pi * (3.0 - math.sqrt(5.0))
PHI1, PHI2 = 0.4656, 0.6823


def radial2d(n_spokes: int, n_readout: int, half_extent: float) -> np.ndarray:
    """Golden-angle radial coordinates ``(n_spokes, n_readout, 2)`` in ``[-h, h)``."""
    r = np.linspace(-half_extent, half_extent, n_readout, endpoint=False, dtype=np.float64)
    ang = np.arange(n_spokes) * GOLDEN_ANGLE
    c = np.stack([np.cos(ang), np.sin(ang)], axis=-1)  # (S, 2)
    return (r[None, :, None] * c[:, None, :]).astype(np.float32)


def kooshball(n_spokes: int, n_readout: int, half_extent: float) -> np.ndarray:
    """3-D golden-means radial coordinates ``(n_spokes, n_readout, 3)``."""
    m = np.arange(n_spokes, dtype=np.float64)
    cz = 2.0 * np.mod(m * PHI1, 1.0) - 1.0
    az = 2.0 * math.pi * np.mod(m * PHI2, 1.0)
    sz = np.sqrt(np.clip(1.0 - cz * cz, 0.0, None))
    d = np.stack([sz * np.cos(az), sz * np.sin(az), cz], axis=-1)
    r = np.linspace(-half_extent, half_extent, n_readout, endpoint=False, dtype=np.float64)
    return (r[None, :, None] * d[:, None, :]).astype(np.float32)


def spiral2d(n_interleaves: int, n_samples: int, half_extent: float, alpha: float = 2.0) -> np.ndarray:
    """Variable-density Archimedean-like spiral ``(n_interleaves, n_samples, 2)``.

    Radius grows as ``t**alpha`` (alpha > 1 oversamples the centre); turns are
    chosen so that the outer ring spacing is about one Nyquist step.
    """
    t = np.linspace(0.0, 1.0, n_samples, dtype=np.float64)
    turns = half_extent / max(n_interleaves, 1)
    r = half_extent * t**alpha
    th = 2.0 * math.pi * turns * t
    out = []
    for i in range(n_interleaves):
        a = th + 2.0 * math.pi * i / n_interleaves
        out.append(np.stack([r * np.cos(a), r * np.sin(a)], axis=-1))
    return np.stack(out).astype(np.float32)


def ellipse_phantom2d(n: int, rng: np.random.Generator, n_ellipses: int = 10) -> np.ndarray:
    """Sum of random ellipses on an ``n x n`` grid (intensities U(0.1, 1))."""
    y, x = np.mgrid[-1:1:complex(0, n), -1:1:complex(0, n)]
    img = np.zeros((n, n), dtype=np.float64)
    for _ in range(n_ellipses):
        cx, cy = rng.uniform(-0.6, 0.6, 2)
        a, b = rng.uniform(0.05, 0.4, 2)
        th = rng.uniform(0, math.pi)
        v = rng.uniform(0.1, 1.0)
        xr = (x - cx) * math.cos(th) + (y - cy) * math.sin(th)
        yr = -(x - cx) * math.sin(th) + (y - cy) * math.cos(th)
        img[(xr / a) ** 2 + (yr / b) ** 2 <= 1.0] += v
    return img


def gaussian_coils(shape, n_coils: int, rng: np.random.Generator, radius: float = 0.7,
                   sigma: float = 0.35) -> np.ndarray:
    """Smooth complex Gaussian-bump coil maps placed on a ring (2-D) or sphere (3-D)."""
    nd = len(shape)
    axes = np.meshgrid(*[np.linspace(-1, 1, s) for s in shape], indexing="ij")
    maps = np.empty((n_coils, *shape), dtype=np.complex64)
    for c in range(n_coils):
        if nd == 2:
            a = 2 * math.pi * c / n_coils
            centre = radius * np.array([math.cos(a), math.sin(a)])
        else:
            u = rng.standard_normal(3)
            centre = radius * u / np.linalg.norm(u)
        d2 = sum((ax - centre[i]) ** 2 for i, ax in enumerate(axes))
        ph = rng.uniform(0, 2 * math.pi)
        maps[c] = (np.exp(-d2 / (2 * (2 * sigma) ** 2)) * np.exp(1j * ph)).astype(np.complex64)
    return maps


def centered_fft(x: np.ndarray, axes) -> np.ndarray:
    return np.fft.fftshift(np.fft.fftn(np.fft.ifftshift(x, axes=axes), axes=axes, norm="ortho"), axes=axes)


def center_crop(x: np.ndarray, width: int, ndim: int) -> np.ndarray:
    sl = [slice(None)] * (x.ndim - ndim)
    for s in x.shape[-ndim:]:
        st = (s - width) // 2
        sl.append(slice(st, st + width))
    return x[tuple(sl)]


@dataclass
class Workload:
    name: str
    shape: tuple
    coords: np.ndarray
    oversamp: float
    kernel_width: int
    kernel_shape: str
    precision: int
    lamda: float
    acr: np.ndarray
    data: np.ndarray | None
    smaps: np.ndarray | None = None
    image_shape: tuple | None = None


def config0(seed: int = 1000, ndft: bool = False) -> Workload:
    """Plain 2-D GROG: 256^2, 64 golden-angle spokes x 512, 8 coils, 5x5 square, p=2."""
    rng = np.random.default_rng(seed)
    n, C = 256, 8
    coords = radial2d(64, 512, 128.0)
    img = ellipse_phantom2d(n, rng)
    maps = gaussian_coils((n, n), C, rng)
    coil_img = maps * img
    acr = center_crop(centered_fft(coil_img, axes=(-2, -1)), 24, 2).astype(np.complex64)
    if ndft:
        data = ndft2d(coil_img, coords)
    else:
        data = (rng.standard_normal((C, 64, 512)) + 1j * rng.standard_normal((C, 64, 512))).astype(np.complex64)
    return Workload("c0", (n, n), coords, 1.0, 5, "square", 2, 1e-2, acr, data, maps, (n, n))


def ndft2d(coil_img: np.ndarray, coords: np.ndarray, snr_db: float = 30.0, seed: int = 1000) -> np.ndarray:
    """Direct NDFT (FP64, separable GEMMs) of coil images at ``coords`` + noise."""
    C, n, _ = coil_img.shape
    k = coords.reshape(-1, 2).astype(np.float64)
    pos = np.arange(n) - n // 2
    ex = np.exp(-2j * np.pi * np.outer(k[:, 0], pos) / n)  # (M, n) along axis 0
    ey = np.exp(-2j * np.pi * np.outer(k[:, 1], pos) / n)
    out = np.empty((C, k.shape[0]), dtype=np.complex128)
    for c in range(C):
        t = ex @ coil_img[c].astype(np.complex128)  # (M, n)
        out[c] = np.einsum("mj,mj->m", t, ey) / n
    rng = np.random.default_rng(seed + 1)
    p = np.mean(np.abs(out) ** 2)
    sigma = math.sqrt(p / (10 ** (snr_db / 10)) / 2)
    out = out + sigma * (rng.standard_normal(out.shape) + 1j * rng.standard_normal(out.shape))
    return out.reshape(C, *coords.shape[:-1]).astype(np.complex64)


def ndft2d_device(coil_img: np.ndarray, coords: np.ndarray, device, noise: float = 0.01,
                  seed: int = 1002) -> np.ndarray:
    """Direct NDFT of coil images at ``coords`` in FP64 on ``device`` (torch
    complex128, separable GEMMs), plus complex Gaussian noise of standard
    deviation ``noise`` x the RMS of the signal; complex64 ``(C, *coords.shape[:-1])``."""
    import torch

    C, n, _ = coil_img.shape
    k = torch.as_tensor(coords.reshape(-1, 2), dtype=torch.float64, device=device)
    pos = torch.arange(n, dtype=torch.float64, device=device) - n // 2
    ex = torch.exp(-2j * math.pi * torch.outer(k[:, 0], pos) / n)  # (M, n) along axis 0
    ey = torch.exp(-2j * math.pi * torch.outer(k[:, 1], pos) / n)
    img = torch.as_tensor(coil_img, dtype=torch.complex128, device=device)
    out = torch.empty(C, k.shape[0], dtype=torch.complex128, device=device)
    for c in range(C):
        out[c] = ((ex @ img[c]) * ey).sum(1) / n
    rms = float(out.abs().square().mean().sqrt())
    rng = np.random.default_rng(seed + 1)
    sig = noise * rms / math.sqrt(2.0)
    nz = sig * (rng.standard_normal(out.shape) + 1j * rng.standard_normal(out.shape))
    res = out.cpu().numpy() + nz
    return res.reshape(C, *coords.shape[:-1]).astype(np.complex64)


def config1_geometry(n_spokes: int = 20000, n_readout: int = 384, n: int = 192):
    """Kooshball trajectory of the 3-D roofline configuration."""
    return kooshball(n_spokes, n_readout, n / 2.0)


def config2(seed: int = 1002, ndft_device=None) -> Workload:
    """CG-SENSE: 320^2, spiral 24 x 4096, 16 coils, oversamp 2, kernel_width 2.

    With ``ndft_device`` the k-space is the FP64 NDFT of the phantom's coil
    images computed on that device, plus 1% complex Gaussian noise; otherwise
    seeded complex Gaussian samples of the same shape."""
    rng = np.random.default_rng(seed)
    n, C = 320, 16
    coords = spiral2d(24, 4096, n / 2.0)
    img = ellipse_phantom2d(n, rng)
    maps = gaussian_coils((n, n), C, rng)
    coil_img = maps * img
    acr = center_crop(centered_fft(coil_img, axes=(-2, -1)), 24, 2).astype(np.complex64)
    if ndft_device is not None:
        data = ndft2d_device(coil_img, coords, ndft_device, 0.01, seed)
    else:
        data = (rng.standard_normal((C, 24, 4096)) + 1j * rng.standard_normal((C, 24, 4096))).astype(np.complex64)
    return Workload("c2", (n, n), coords, 2.0, 2, "circle", 1, 1e-3, acr, data, maps, (n, n))


def config3_slices(seed: int = 1003, n_slices: int = 64):
    """Uneven 2-D radial slices: spokes U{13..233}, readout U{256..768}, grid U{128..384}, coils U{8..32}."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_slices):
        sp = int(rng.integers(13, 234))
        ro = int(rng.integers(256, 769))
        g = int(rng.integers(128, 385))
        C = int(rng.integers(8, 33))
        out.append(dict(spokes=sp, readout=ro, grid=g, coils=C))
    return out


def serving_protocols(seed: int = 1004, n_slices: int = 2) -> list[dict]:
    """Protocol specs of the served-recon mix: the c0 and c2 configurations and
    ``n_slices`` uneven radial slices of c3 (coil maps from seeded Gaussian
    bumps, ACR = centre 24^2 of the coil k-space of a seeded phantom).
    Keyword sets for ``pygrog_b200.serve.ReconProtocol``."""
    out = []
    w0 = config0()
    out.append(dict(name="c0", shape=w0.shape, coords=w0.coords, acr=w0.acr, smaps=w0.smaps, oversamp=1.0,
                    kernel_width=5, kernel_shape="square", precision=2, lamda=1e-2, max_iter=10))
    w2 = config2()
    out.append(dict(name="c2", shape=w2.shape, coords=w2.coords, acr=w2.acr, smaps=w2.smaps, oversamp=2.0,
                    kernel_width=2, kernel_shape="circle", precision=1, lamda=1e-3, max_iter=30))
    return out + c3_protocols(seed, n_slices)


def c3_protocols(seed: int = 1004, n_slices: int = 64) -> list[dict]:
    """The first ``n_slices`` uneven radial slices of c3 as ``ReconProtocol``
    keyword sets (coil maps from seeded Gaussian bumps, ACR = centre 24^2 of the
    coil k-space of a seeded phantom, 20 CG iterations)."""
    out = []
    rng = np.random.default_rng(seed)
    for i, s in enumerate(config3_slices(seed=1003, n_slices=n_slices)):
        n, C = s["grid"], s["coils"]
        coords = radial2d(s["spokes"], s["readout"], n / 2.0)
        img = ellipse_phantom2d(n, rng)
        maps = gaussian_coils((n, n), C, rng)
        acr = center_crop(centered_fft(maps * img, axes=(-2, -1)), 24, 2).astype(np.complex64)
        out.append(dict(name=f"c3s{i}", shape=(n, n), coords=coords, acr=acr, smaps=maps.astype(np.complex64),
                        oversamp=1.0, kernel_width=2, kernel_shape="circle", precision=1, lamda=1e-2,
                        max_iter=20))
    return out


def t2_subspace_basis(n_frames: int = 500, rank: int = 4, n_atoms: int = 200, te_ms: float = 1.0,
                      seed: int = 1005) -> np.ndarray:
    """Rank-``rank`` temporal basis ``(rank, n_frames)`` complex64: leading right singular
    vectors of a seeded dictionary of mono-exponential decays, T2 ~ U(20, 300) ms."""
    rng = np.random.default_rng(seed)
    t2 = rng.uniform(20.0, 300.0, n_atoms)
    t = (np.arange(n_frames) + 1) * te_ms
    D = np.exp(-t[None, :] / t2[:, None])
    _, _, vh = np.linalg.svd(D, full_matrices=False)
    return vh[:rank].astype(np.complex64)


def subspace_protocol(seed: int = 1006, n_frames: int = 500, readout: int = 256, n: int = 192,
                      coils: int = 8, rank: int = 4) -> dict:
    """Served subspace protocol: one golden-angle spoke per frame, ``n_frames`` frames,
    rank-``rank`` T2 basis on the frame axis (keyword set for ``ReconProtocol``)."""
    rng = np.random.default_rng(seed)
    coords = radial2d(n_frames, readout, n / 2.0).reshape(n_frames, readout, 2)
    img = ellipse_phantom2d(n, rng)
    maps = gaussian_coils((n, n), coils, rng)
    acr = center_crop(centered_fft(maps * img, axes=(-2, -1)), 24, 2).astype(np.complex64)
    return dict(name="sub", shape=(n, n), coords=coords, acr=acr, smaps=maps.astype(np.complex64), oversamp=2.0,
                kernel_width=2, kernel_shape="circle", precision=1, lamda=1e-2, max_iter=20,
                basis=t2_subspace_basis(n_frames, rank), encoding_axis=-3)
