"""Oracle (test infrastructure only): PCA coil compression on the CPU.

Restates the method behind the reference's ``utils/_coil_compress.py:23-57``
(``coil_compress`` forwards to ``mrinufft.extras.smaps.coil_compression``,
a package absent here and not pinned by the reference): the virtual coils are
the leading principal components of the (calibration) coil data, i.e. the
leading eigenvectors of the coil covariance ``D D^H``, computed here in FP64
with numpy.  Parity with mrinufft itself is unpinned; the phase convention
(largest-magnitude weight of every row real and positive) is this build's.
"""

import numpy as np


def compression_matrix(calib: np.ndarray, n_coils) -> np.ndarray:
    d = np.asarray(calib, dtype=np.complex128).reshape(calib.shape[0], -1)
    cov = d @ d.conj().T
    w, v = np.linalg.eigh(cov)
    w, v = np.clip(w[::-1], 0.0, None), v[:, ::-1]
    if isinstance(n_coils, float) and (n_coils <= 1 or not float(n_coils).is_integer()):
        energy = np.cumsum(w) / max(w.sum(), 1e-300)
        K = int(np.searchsorted(energy, n_coils - 1e-12)) + 1
    else:
        K = int(n_coils)
    mat = v[:, :K].conj().T
    idx = np.abs(mat).argmax(axis=1)
    ph = mat[np.arange(K), idx]
    return mat * np.conj(ph / np.abs(ph))[:, None]


def coil_compress(kspace_data, n_coils, traj=None, krad_thresh=None):
    data = np.asarray(kspace_data)
    C = data.shape[0]
    flat = data.reshape(C, -1)
    calib = flat
    if krad_thresh is not None and traj is not None:
        tr = np.asarray(traj, dtype=np.float32).reshape(-1, np.asarray(traj).shape[-1])
        rad = np.sqrt((tr.astype(np.float64) ** 2).sum(-1))
        calib = flat[:, rad < krad_thresh * rad.max()]
    mat = compression_matrix(calib, n_coils)
    return (mat @ flat.astype(np.complex128)).reshape((mat.shape[0],) + data.shape[1:]), mat
